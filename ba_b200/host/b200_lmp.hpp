// C++ host layer over the b200la C ABI, with the names, argument meaning and
// results of HiFlow3's lmp / linear_solver interface for the PCG path:
//
//   B200_lVector<T>      ~ lVector<T>       (lmp/lvector.h:38-321)
//   B200_CSR_lMatrix<T>  ~ CSR_lMatrix<T>   (lmp/lmatrix.h:39-468)
//   B200_CG<T>           ~ CG<LAD>          (linear_solver/cg.h:39-247) with
//                          PreconditionerBlockJacobiStand::Init_Jacobi
//   B200_MPIR            ~ MPIR<CoupledD, CoupledS> (linear_solver/mpir.h)
//
// Header-only; link with ba_b200/libb200la.so.  Errors throw
// b200la::Error (the reference calls exit(-1) instead).
#pragma once

#include <cstdint>
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
  b200la_mat handle() const { return h_; }

 private:
  std::string name_;
  int nrow_, ncol_;
  int64_t nnz_;
  b200la_mat h_ = nullptr;
};

// CG<LAD> with IterateControl(maxits, atol, rtol, dtol); SetupPreconditioner
// with Jacobi switches to right preconditioning (linear_solver.h:97-100).
template <typename T> class B200_CG {
 public:
  B200_CG() = default;
  ~B200_CG() { release(); }
  void InitControl(int maxits, double atol, double rtol, double dtol) {
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
  void SetupOperator(B200_CSR_lMatrix<T> &op) {
    op_ = &op;
    release();
  }
  void SetupPreconditionerJacobi() {
    prm_.precond = 1;
    release();
  }
  LinearSolverState Solve(const B200_lVector<T> &b, B200_lVector<T> *x) {
    if (!op_) throw Error(B200LA_ERR_INVALID, "CG: SetupOperator was not called");
    if (!s_) check(b200la_cg_create(op_->handle(), &prm_, &s_));
    check(b200la_cg_solve(s_, b.handle(), x->handle(), &res_));
    return (LinearSolverState)res_.solver_state;
  }
  int iter() const { return res_.iters; }
  double res() const { return res_.res; }
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

// MPIR<LADescriptorCoupledD, LADescriptorCoupledS> with an FP32 Jacobi-PCG as
// the low-precision error-correction solver.
class B200_MPIR {
 public:
  ~B200_MPIR() { release(); }
  void SetupOperator(B200_CSR_lMatrix<double> &op) {
    op_ = &op;
    release();
  }
  void SetMpirParameters(int max_ech, int max_ecl, double abs_tol, double rel_tol, double div_tol) {
    if (max_ech != 0) throw Error(B200LA_ERR_UNSUPPORTED, "MPIR: high-precision passes are not on this path");
    prm_.max_outer = max_ecl;
    prm_.atol = abs_tol;
    prm_.rtol = rel_tol;
    prm_.dtol = div_tol;
    release();
  }
  void SetLowPrecErrCorSolverParameters(int max_iter, float abs_tol, float rel_tol, float div_tol) {
    (void)abs_tol;
    (void)div_tol;
    prm_.inner_maxits = max_iter;
    prm_.inner_rtol = rel_tol;
    release();
  }
  LinearSolverState Solve(const B200_lVector<double> &b, B200_lVector<double> *x) {
    if (!op_) throw Error(B200LA_ERR_INVALID, "MPIR: SetupOperator was not called");
    if (!s_) check(b200la_mp_create(op_->handle(), &prm_, &s_));
    check(b200la_mp_solve(s_, b.handle(), x->handle(), &res_));
    return (LinearSolverState)res_.solver_state;
  }
  int iter() const { return res_.inner_iters; }
  int outer() const { return res_.outer; }
  double res() const { return res_.res; }
  double res_rel() const { return res_.res_rel; }

 private:
  void release() {
    if (s_) b200la_mp_destroy(s_);
    s_ = nullptr;
  }
  B200_CSR_lMatrix<double> *op_ = nullptr;
  b200la_mp_params prm_{50, 0.0, 1e-10, 1e6, 100000, 1e-5, 1, 1};
  b200la_mp s_ = nullptr;
  b200la_mp_result res_{};
};

}  // namespace b200la
