// C++ host layer over the b200la C ABI, with the names, argument meaning and
// results of HiFlow3's lmp / linear_solver interface for the PCG path:
//
//   B200_lVector<T>      ~ lVector<T>       (lmp/lvector.h:38-321)
//   B200_CSR_lMatrix<T>  ~ CSR_lMatrix<T>   (lmp/lmatrix.h:39-468)
//   B200_LinearSolver<T> ~ LinearSolver<LAD> (linear_solver/linear_solver.h):
//                          InitControl, SetupOperator, Solve, iter, res
//   B200_CG<T>           ~ CG<LAD>          (linear_solver/cg.h:39-247) with
//                          PreconditionerBlockJacobiStand::Init_Jacobi
//   B200_Jacobi<T>       ~ Jacobi<LAD>      (linear_solver/jacobi.h:30-80)
//   B200_BiCGSTAB<T>     ~ BiCGSTAB<LAD>    (linear_solver/bicgstab.h:37-495)
//   B200_GMRES<T>        ~ GMRES<LAD>       (linear_solver/gmres.h:46-746)
//   B200_MPIR            ~ MPIR<CoupledD, CoupledS> (linear_solver/mpir.h:29-150)
//
// Header-only; link with ba_b200/libb200la.so.  Errors throw
// b200la::Error (the reference calls exit(-1) instead).
#pragma once

#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "b200la.h"

namespace b200la {

enum LinearSolverState { kSolverSuccess = 0, kSolverExceeded = 1, kSolverError = 2 };

struct Error : std::runtime_error {
  int status;
  Error(int st, const std::string &msg) : std::runtime_error(msg), status(st) {}
};

inline void check(int st) {
  if (st != B200LA_OK) throw Error(st, b200la_last_error());
}

template <typename T> constexpr int dtype_of();
template <> constexpr int dtype_of<double>() { return B200LA_F64; }
template <> constexpr int dtype_of<float>() { return B200LA_F32; }

// One device context (init_platform_gpu).
class Platform {
 public:
  explicit Platform(int device = 0) { check(b200la_ctx_create(device, &ctx_)); }
  ~Platform() { b200la_ctx_destroy(ctx_); }
  Platform(const Platform &) = delete;
  Platform &operator=(const Platform &) = delete;
  b200la_ctx get() const { return ctx_; }
  void Sync() const { check(b200la_ctx_synchronize(ctx_)); }

 private:
  b200la_ctx ctx_ = nullptr;
};

template <typename T> class B200_lVector {
 public:
  B200_lVector(Platform &p, int size, const std::string &name = "") : p_(&p), name_(name) { Init(size, name); }
  ~B200_lVector() { Clear(); }
  B200_lVector(const B200_lVector &) = delete;
  B200_lVector &operator=(const B200_lVector &) = delete;

  void Init(int size, const std::string &name) {
    Clear();
    name_ = name;
    size_ = size;
    check(b200la_vec_create(p_->get(), size, dtype_of<T>(), &h_));
  }
  void Clear() {
    if (h_) b200la_vec_destroy(h_);
    h_ = nullptr;
  }
  int get_size() const { return size_; }
  void Zeros() { check(b200la_vec_zeros(h_)); }
  void SetBlockValues(int start, int end, const T *values) {
    if (start != 0 || end != size_) throw Error(B200LA_ERR_INVALID, "SetBlockValues: full range only");
    check(b200la_vec_upload(h_, values, size_));
  }
  void GetBlockValues(int start, int end, T *values) const {
    if (start != 0 || end != size_) throw Error(B200LA_ERR_INVALID, "GetBlockValues: full range only");
    check(b200la_vec_download(h_, values, size_));
  }
  void SetValues(const int *index, int size, const T *values) { check(b200la_vec_set_values(h_, index, values, size)); }
  void GetValues(const int *index, int size, T *values) const { check(b200la_vec_get_values(h_, index, values, size)); }
  void CopyFrom(const B200_lVector &v) { check(b200la_vec_copy(h_, v.h_)); }
  template <typename S> void CastFrom(const B200_lVector<S> &v) { check(b200la_vec_cast(h_, v.handle())); }
  T Dot(const B200_lVector &v) const {
    double d = 0.0;
    check(b200la_vec_dot(h_, v.h_, &d));
    return (T)d;
  }
  T Norm2() const {
    double d = 0.0;
    check(b200la_vec_norm2(h_, &d));
    return (T)d;
  }
  void Axpy(const B200_lVector &v, T scalar) { check(b200la_vec_axpy(h_, v.h_, scalar)); }        // this += s v
  void ScaleAdd(T scalar, const B200_lVector &v) { check(b200la_vec_scaleadd(h_, scalar, v.h_)); }  // this = s this + v
  void Scale(T scalar) { check(b200la_vec_scale(h_, scalar)); }
  void ElementWiseMult(const B200_lVector &v) { check(b200la_vec_elementwise_mult(h_, v.h_)); }
  T *GetBuffer() const {
    void *p = nullptr;
    check(b200la_vec_info(h_, nullptr, nullptr, &p));
    return (T *)p;
  }
  b200la_vec handle() const { return h_; }

 private:
  Platform *p_;
  std::string name_;
  int size_ = 0;
  b200la_vec h_ = nullptr;
};

template <typename T> class B200_CSR_lMatrix {
 public:
  // Init + CopyStructureFrom + CopyFrom from a host CSR with double values.
  B200_CSR_lMatrix(Platform &p, int nrow, int ncol, int64_t nnz, const int *rowptr, const int *col,
                   const double *val, const std::string &name = "")
      : name_(name), nrow_(nrow), ncol_(ncol), nnz_(nnz) {
    check(b200la_csr_upload(p.get(), nrow, ncol, nnz, rowptr, col, val, B200LA_F64, dtype_of<T>(), &h_));
  }
  ~B200_CSR_lMatrix() { b200la_mat_destroy(h_); }
  B200_CSR_lMatrix(const B200_CSR_lMatrix &) = delete;
  B200_CSR_lMatrix &operator=(const B200_CSR_lMatrix &) = delete;
  int get_num_row() const { return nrow_; }
  int get_num_col() const { return ncol_; }
  int64_t get_nnz() const { return nnz_; }
  void VectorMult(const B200_lVector<T> &in, B200_lVector<T> *out) const { check(b200la_spmv(h_, in.handle(), out->handle())); }
  void VectorMultAdd(const B200_lVector<T> &in, B200_lVector<T> *out) const {
    check(b200la_spmv_add(h_, in.handle(), out->handle()));
  }
  void extract_invdiagelements(B200_lVector<T> *vec) const { check(b200la_mat_inv_diag(h_, vec->handle())); }
  void ZeroRows(const int *index_set, int size, T alpha) { check(b200la_mat_zero_rows(h_, index_set, size, alpha)); }
  void Tune() { check(b200la_mat_tune(h_, nullptr, nullptr, nullptr)); }
  // CastFrom: a copy of this matrix holding its values as S.
  template <typename S> std::unique_ptr<B200_CSR_lMatrix<S>> CastTo() const {
    b200la_mat h = nullptr;
    check(b200la_mat_cast(h_, dtype_of<S>(), &h));
    return std::unique_ptr<B200_CSR_lMatrix<S>>(new B200_CSR_lMatrix<S>(h, nrow_, ncol_, nnz_, name_));
  }
  b200la_mat handle() const { return h_; }
  // adopts a matrix handle
  B200_CSR_lMatrix(b200la_mat h, int nrow, int ncol, int64_t nnz, const std::string &name)
      : name_(name), nrow_(nrow), ncol_(ncol), nnz_(nnz), h_(h) {}

 private:
  std::string name_;
  int nrow_, ncol_;
  int64_t nnz_;
  b200la_mat h_ = nullptr;
};

// LinearSolver<LAD>'s part of the interface the MPIR loop drives.
template <typename T> class B200_LinearSolver {
 public:
  virtual ~B200_LinearSolver() = default;
  virtual void InitControl(int maxits, double atol, double rtol, double dtol) = 0;
  virtual void SetupOperator(B200_CSR_lMatrix<T> &op) = 0;
  virtual LinearSolverState Solve(const B200_lVector<T> &b, B200_lVector<T> *x) = 0;
  virtual int iter() const = 0;
  virtual double res() const = 0;
};

// CG<LAD> with IterateControl(maxits, atol, rtol, dtol); SetupPreconditioner
// with Jacobi switches to right preconditioning (linear_solver.h:97-100).
template <typename T> class B200_CG : public B200_LinearSolver<T> {
 public:
  B200_CG() = default;
  ~B200_CG() override { release(); }
  void InitControl(int maxits, double atol, double rtol, double dtol) override {
    prm_.maxits = maxits;
    prm_.atol = atol;
    prm_.rtol = rtol;
    prm_.dtol = dtol;
    release();
  }
  void InitParameter(const std::string &method) {
    prm_.precond = method == "NoPreconditioning" ? 0 : 1;
    release();
  }
  void SetupOperator(B200_CSR_lMatrix<T> &op) override {
    op_ = &op;
    release();
  }
  void SetupPreconditionerJacobi() {
    prm_.precond = 1;
    release();
  }
  LinearSolverState Solve(const B200_lVector<T> &b, B200_lVector<T> *x) override {
    if (!op_) throw Error(B200LA_ERR_INVALID, "CG: SetupOperator was not called");
    if (!s_) check(b200la_cg_create(op_->handle(), &prm_, &s_));
    check(b200la_cg_solve(s_, b.handle(), x->handle(), &res_));
    return (LinearSolverState)res_.solver_state;
  }
  int iter() const override { return res_.iters; }
  double res() const override { return res_.res; }
  double res_init() const { return res_.res_init; }
  double res_rel() const { return res_.res_rel; }

 private:
  void release() {
    if (s_) b200la_cg_destroy(s_);
    s_ = nullptr;
  }
  B200_CSR_lMatrix<T> *op_ = nullptr;
  b200la_cg_params prm_{1000, 1e-12, 1e-8, 1e8, 0};  // IterateControl defaults (iterate_control.cc:26-29)
  b200la_cg s_ = nullptr;
  b200la_cg_result res_{};
};

// Jacobi, BiCGSTAB and GMRES on the device (b200la_solver_*).
template <typename T> class B200_DeviceSolver : public B200_LinearSolver<T> {
 public:
  ~B200_DeviceSolver() override { release(); }
  void InitControl(int maxits, double atol, double rtol, double dtol) override {
    prm_.maxits = maxits;
    prm_.atol = atol;
    prm_.rtol = rtol;
    prm_.dtol = dtol;
    release();
  }
  void SetupOperator(B200_CSR_lMatrix<T> &op) override {
    op_ = &op;
    release();
  }
  LinearSolverState Solve(const B200_lVector<T> &b, B200_lVector<T> *x) override {
    if (!op_) throw Error(B200LA_ERR_INVALID, "solver: SetupOperator was not called");
    if (!s_) check(b200la_solver_create(op_->handle(), &prm_, &s_));
    check(b200la_solver_solve(s_, b.handle(), x->handle(), &res_));
    iter_ = counts_on() ? iter_ + res_.iters : res_.iters;
    return (LinearSolverState)res_.solver_state;
  }
  int iter() const override { return iter_; }
  double res() const override { return res_.res; }
  int restarts() const { return res_.restarts; }

 protected:
  explicit B200_DeviceSolver(int method) {
    prm_.method = method;
    prm_.maxits = 1000;  // IterateControl defaults (iterate_control.cc:26-29)
    prm_.atol = 1e-12;
    prm_.rtol = 1e-8;
    prm_.dtol = 1e8;
    prm_.inner_iter = 1;
    prm_.smooth_iter = 1;
    prm_.w = 1.0;
    prm_.size_basis = 100;
  }
  // Jacobi's smoothing modes add their sweeps to iter_ (jacobi.cc:256-285)
  virtual bool counts_on() const { return false; }
  void release() {
    if (s_) b200la_solver_destroy(s_);
    s_ = nullptr;
  }
  B200_CSR_lMatrix<T> *op_ = nullptr;
  b200la_solver_params prm_{};
  b200la_solver s_ = nullptr;
  b200la_solver_result res_{};
  int iter_ = 0;
};

// Jacobi<LAD>: SetSolveMode (0 SolveNormal, 1 SolveDamped, 2 SmoothNormal,
// 3 SmoothDamped), SetNumIter, SetInnerIter, SetDampingParameter.
template <typename T> class B200_Jacobi : public B200_DeviceSolver<T> {
 public:
  B200_Jacobi() : B200_DeviceSolver<T>(B200LA_METHOD_JACOBI) {}
  void SetSolveMode(int mode) { this->prm_.mode = mode; this->release(); }
  void SetNumIter(int it) { this->prm_.smooth_iter = it; this->release(); }
  void SetInnerIter(int it) { this->prm_.inner_iter = it; this->release(); }
  void SetDampingParameter(T w) { this->prm_.w = w; this->release(); }

 protected:
  bool counts_on() const override { return this->prm_.mode >= B200LA_JACOBI_SMOOTH_NORMAL; }
};

// BiCGSTAB<LAD>: InitParameter("NoPreconditioning" | "RightPreconditioning").
template <typename T> class B200_BiCGSTAB : public B200_DeviceSolver<T> {
 public:
  B200_BiCGSTAB() : B200_DeviceSolver<T>(B200LA_METHOD_BICGSTAB) {}
  void InitParameter(const std::string &method) {
    if (method == "LeftPreconditioning") throw Error(B200LA_ERR_UNSUPPORTED, "BiCGSTAB: left preconditioning");
    this->prm_.precond = method == "RightPreconditioning" ? 1 : 0;
    this->release();
  }
  void SetupPreconditionerJacobi() { this->prm_.precond = 1; this->release(); }
};

// GMRES<LAD>: InitParameter(size_basis, "NoPreconditioning" | "RightPreconditioning").
template <typename T> class B200_GMRES : public B200_DeviceSolver<T> {
 public:
  B200_GMRES() : B200_DeviceSolver<T>(B200LA_METHOD_GMRES) {}
  void InitParameter(int size_basis, const std::string &method) {
    if (method == "LeftPreconditioning") throw Error(B200LA_ERR_UNSUPPORTED, "GMRES: left preconditioning");
    this->prm_.size_basis = size_basis;
    this->prm_.precond = method == "RightPreconditioning" ? 1 : 0;
    this->release();
  }
  void SetupPreconditionerJacobi() { this->prm_.precond = 1; this->release(); }
};


// MPIR<LADescriptorCoupledD, LADescriptorCoupledS> (linear_solver/mpir.cc:
// 52-297).  With SetLowPrecErrCorSolver (and optionally a high-precision
// error-correction solver and smoothers) Solve runs SolveImpl's loop over the
// device solvers: FP64 residual; while ContinueIteration(): high
// pre-smoothing, a low-precision pass (cast, low pre-smoothing, correction
// solve, low post-smoothing, cast back) while max_ecl allows, else a
// high-precision pass, x += correction, high post-smoothing, FP64 residual,
// res0 = res (mpir.cc:240).  Kept from the reference: component parameters
// default to 0 iterations, the pass counters are not reset by Solve.
// Without an error-correction solver Solve is one fused device solve
// (b200la_mp: FP32 Jacobi-PCG inside FP64 refinement, outer test relative to
// the initial residual); max_ech must be 0 there.
class B200_MPIR {
 public:
  explicit B200_MPIR(Platform &p) : p_(&p) {}
  ~B200_MPIR() { release(); }
  void SetupOperator(B200_CSR_lMatrix<double> &op) {
    op_ = &op;
    release();
  }
  void SetHighPrecMatrix(B200_CSR_lMatrix<double> &m) { SetupOperator(m); }
  void SetLowPrecMatrix(B200_CSR_lMatrix<float> &m) { al_ = &m; }
  void SetHighPrecResVector(B200_lVector<double> &v) { resh_ = &v; }
  void SetHighPrecCorVector(B200_lVector<double> &v) { corh_ = &v; }
  void SetLowPrecResVector(B200_lVector<float> &v) { resl_ = &v; }
  void SetLowPrecCorVector(B200_lVector<float> &v) { corl_ = &v; }
  void SetHighPrecPreSmoother(B200_LinearSolver<double> &s) { preh_ = &s; }
  void SetHighPrecPostSmoother(B200_LinearSolver<double> &s) { posth_ = &s; }
  void SetLowPrecPreSmoother(B200_LinearSolver<float> &s) { prel_ = &s; }
  void SetLowPrecPostSmoother(B200_LinearSolver<float> &s) { postl_ = &s; }
  void SetHighPrecErrCorSolver(B200_LinearSolver<double> &s) { ech_ = &s; }
  void SetLowPrecErrCorSolver(B200_LinearSolver<float> &s) { ecl_ = &s; }
  void UseHighPrecPreSmoother(bool u) { use_preh_ = u; }
  void UseHighPrecPostSmoother(bool u) { use_posth_ = u; }
  void UseLowPrecPreSmoother(bool u) { use_prel_ = u; }
  void UseLowPrecPostSmoother(bool u) { use_postl_ = u; }
  void SetMpirParameters(int max_ech, int max_ecl, double abs_tol, double rel_tol, double div_tol) {
    max_ech_ = max_ech;
    max_ecl_ = max_ecl;
    abs_ = abs_tol;
    rel_ = rel_tol;
    div_ = div_tol;
    prm_.max_outer = max_ecl;
    prm_.atol = abs_tol;
    prm_.rtol = rel_tol;
    prm_.dtol = div_tol;
    release();
  }
  void SetHighPrecPreSmootherParameters(int it, double a, double r, double d) { par_[kPreH] = {it, a, r, d}; }
  void SetHighPrecPostSmootherParameters(int it, double a, double r, double d) { par_[kPostH] = {it, a, r, d}; }
  void SetLowPrecPreSmootherParameters(int it, double a, double r, double d) { par_[kPreL] = {it, a, r, d}; }
  void SetLowPrecPostSmootherParameters(int it, double a, double r, double d) { par_[kPostL] = {it, a, r, d}; }
  void SetHighPrecErrCorSolverParameters(int it, double a, double r, double d) { par_[kEcH] = {it, a, r, d}; }
  void SetLowPrecErrCorSolverParameters(int max_iter, double abs_tol, double rel_tol, double div_tol) {
    par_[kEcL] = {max_iter, abs_tol, rel_tol, div_tol};
    prm_.inner_maxits = max_iter;
    prm_.inner_rtol = rel_tol;
    release();
  }
  LinearSolverState Solve(const B200_lVector<double> &b, B200_lVector<double> *x) {
    if (!op_) throw Error(B200LA_ERR_INVALID, "MPIR: SetupOperator was not called");
    if (ecl_ || ech_) return SolveGeneric(b, x);
    if (max_ech_ != 0) throw Error(B200LA_ERR_UNSUPPORTED, "MPIR: high-precision passes need SetHighPrecErrCorSolver");
    if (!s_) check(b200la_mp_create(op_->handle(), &prm_, &s_));
    check(b200la_mp_solve(s_, b.handle(), x->handle(), &res_));
    iter_ = res_.inner_iters;
    outer_ = res_.outer;
    r_ = res_.res;
    r_init_ = res_.res_init;
    return (LinearSolverState)res_.solver_state;
  }
  int iter() const { return iter_; }
  int outer() const { return outer_; }
  int n_ecl() const { return n_ecl_; }
  int n_ech() const { return n_ech_; }
  double res() const { return r_; }
  double res_rel() const { return r_init_ > 0 ? r_ / r_init_ : 0.0; }

 private:
  enum { kPreH, kPostH, kPreL, kPostL, kEcH, kEcL, kRoles };
  struct Params {
    int it;
    double atol, rtol, dtol;
  };
  template <typename S> void Reset(B200_LinearSolver<S> *s, int role) {
    if (s) s->InitControl(par_[role].it, par_[role].atol, par_[role].rtol, par_[role].dtol);
  }
  bool Passes(int n, int max, int role) const {
    return n < max && r_ > par_[role].atol && r_ > r0_ * par_[role].rtol && r_ < par_[role].dtol;
  }
  bool ContinueIteration() const {
    return r_ > abs_ && r_ > r0_ * rel_ && r_ < div_ && (Passes(n_ech_, max_ech_, kEcH) || Passes(n_ecl_, max_ecl_, kEcL));
  }
  void Residual(const B200_lVector<double> &b, B200_lVector<double> *x) {
    op_->VectorMult(*x, resh_);
    resh_->ScaleAdd(-1.0, b);  // coupled resh.ScaleAdd(b, -1)
    r_ = resh_->Norm2();
  }
  LinearSolverState SolveGeneric(const B200_lVector<double> &b, B200_lVector<double> *x) {
    const int n = op_->get_num_row();
    if (!al_) {
      al_own_ = op_->CastTo<float>();
      al_ = al_own_.get();
    }
    if (!resh_) { resh_own_.reset(new B200_lVector<double>(*p_, n, "resh")); resh_ = resh_own_.get(); }
    if (!corh_) { corh_own_.reset(new B200_lVector<double>(*p_, n, "corh")); corh_ = corh_own_.get(); }
    if (!resl_) { resl_own_.reset(new B200_lVector<float>(*p_, n, "resl")); resl_ = resl_own_.get(); }
    if (!corl_) { corl_own_.reset(new B200_lVector<float>(*p_, n, "corl")); corl_ = corl_own_.get(); }
    iter_ = 0;
    if (use_preh_) { Reset(preh_, kPreH); preh_->SetupOperator(*op_); }
    if (use_prel_) { Reset(prel_, kPreL); prel_->SetupOperator(*al_); }
    if (ecl_) { ecl_->SetupOperator(*al_); Reset(ecl_, kEcL); }
    if (use_postl_) { Reset(postl_, kPostL); postl_->SetupOperator(*al_); }
    if (ech_) { Reset(ech_, kEcH); ech_->SetupOperator(*op_); }
    if (use_posth_) { Reset(posth_, kPostH); posth_->SetupOperator(*op_); }
    Residual(b, x);
    r_init_ = r0_ = r_;
    outer_ = 0;
    while (ContinueIteration()) {
      ++outer_;
      if (use_preh_) {
        preh_->Solve(b, x);
        iter_ += preh_->iter();
        Residual(b, x);
      }
      if (ecl_ && Passes(n_ecl_, max_ecl_, kEcL)) {
        ++n_ecl_;
        resl_->CastFrom(*resh_);
        corl_->Zeros();
        if (use_prel_) { prel_->Solve(*resl_, corl_); iter_ += prel_->iter(); }
        ecl_->Solve(*resl_, corl_);
        iter_ += ecl_->iter();
        if (use_postl_) { postl_->Solve(*resl_, corl_); iter_ += postl_->iter(); }
        corh_->CastFrom(*corl_);
      } else if (ech_ && Passes(n_ech_, max_ech_, kEcH)) {
        ++n_ech_;
        corh_->Zeros();
        ech_->Solve(*resh_, corh_);
        iter_ += ech_->iter();
      }
      x->Axpy(*corh_, 1.0);
      if (use_posth_) {
        posth_->Solve(b, x);
        iter_ += posth_->iter();
      }
      Residual(b, x);
      r0_ = r_;
    }
    return (r_ < abs_ || r_ < r0_ * rel_) ? kSolverSuccess : kSolverExceeded;
  }
  void release() {
    if (s_) b200la_mp_destroy(s_);
    s_ = nullptr;
  }
  Platform *p_;
  B200_CSR_lMatrix<double> *op_ = nullptr;
  B200_CSR_lMatrix<float> *al_ = nullptr;
  std::unique_ptr<B200_CSR_lMatrix<float>> al_own_;
  B200_lVector<double> *resh_ = nullptr, *corh_ = nullptr;
  B200_lVector<float> *resl_ = nullptr, *corl_ = nullptr;
  std::unique_ptr<B200_lVector<double>> resh_own_, corh_own_;
  std::unique_ptr<B200_lVector<float>> resl_own_, corl_own_;
  B200_LinearSolver<double> *preh_ = nullptr, *posth_ = nullptr, *ech_ = nullptr;
  B200_LinearSolver<float> *prel_ = nullptr, *postl_ = nullptr, *ecl_ = nullptr;
  bool use_preh_ = false, use_posth_ = false, use_prel_ = false, use_postl_ = false;
  Params par_[kRoles] = {};
  int max_ech_ = 0, max_ecl_ = 0, n_ech_ = 0, n_ecl_ = 0, iter_ = 0, outer_ = 0;
  double abs_ = 0.0, rel_ = 0.0, div_ = 0.0, r_ = 0.0, r0_ = 0.0, r_init_ = 0.0;
  b200la_mp_params prm_{50, 0.0, 1e-10, 1e6, 100000, 1e-5, 1, 1};
  b200la_mp s_ = nullptr;
  b200la_mp_result res_{};
};

}  // namespace b200la
