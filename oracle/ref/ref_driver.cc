// Reference CPU checker driver (TEST INFRASTRUCTURE ONLY).
//
// Linked against HiFlow3's own lmp CPU sources, compiled unmodified from the
// reference tree by oracle/ref/Makefile into oracle/_ref/libhiflow_lmp_ref.so.
// Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline legs load
// it, and only as the checker / the timed CPU reference.  The product path
// (ba_b200/) never links or calls it.
//
// Exposes a plain C ABI over the reference classes:
//   * ref_spmv_*      -> CPUsimple_CSR_lMatrix / CPUopenmp_CSR_lMatrix
//                        ::VectorMult (lmp/CPUsimple_csr_lmatrix.cc:92-111,
//                        lmp/openmp/CPUopenmp_csr_lmatrix.cc:145-165)
//   * ref_cg_solve_*  -> a single-rank restatement of CG<LAD>::SolveNoPrecond
//                        / SolvePrecond (linear_solver/cg.h:87-246) with the
//                        stopping test of IterateControl::Check
//                        (common/iterate_control.cc:80-107), issued as the
//                        same sequence of compiled lVector/lMatrix calls and
//                        lPreconditioner_Jacobi (lmp/lpreconditioner.cc:125-200).
//                        On one rank CoupledVector::Dot is the interior Dot plus
//                        an identity all-reduce and CoupledMatrix::VectorMult is
//                        the diagonal block's VectorMult, so the restatement
//                        issues exactly the arithmetic the reference does.
//   * ref_lmp_cg_*    -> the reference's own lmp cg() (lmp/solvers/cg.cc:35).
//   * ref_jacobi_solve_d, ref_bicgstab_solve_d, ref_gmres_solve_d ->
//                        single-rank restatements of Jacobi<LAD>
//                        (linear_solver/jacobi.cc:145-356), BiCGSTAB<LAD>
//                        (linear_solver/bicgstab.h:127-473) and GMRES<LAD>
//                        (linear_solver/gmres.h:229-746) over the same
//                        compiled lmp calls.
//   * ref_coo_to_csr_d -> CPU_CSR_lMatrix::TransformFromCOO.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>

#include "config.h"
#include "lmatrix_csr_cpu.h"
#include "lpreconditioner.h"
#include "lvector_cpu.h"
#include "solvers/cg.h"

using namespace hiflow::la;

namespace {

enum { IMPL_NAIVE = 0, IMPL_OPENMP = 1 };

// IterateControl states (common/iterate_control.h): kIterate,
// kFailureDivergenceTol, kFailureMaxitsExceeded, kSuccessAbsoluteTol,
// kSuccessRelativeTol.  Numbered as in the B200 library's solver status.
enum { CTRL_ITERATE = 0, CTRL_SUCCESS_ABS = 1, CTRL_SUCCESS_REL = 2,
       CTRL_FAIL_DIV = 3, CTRL_FAIL_MAXITS = 4 };

// IterateControl::Check, common/iterate_control.cc:80-107.
int control_check(int step, double value, int maxits, double atol, double rtol,
                  double dtol, double *first_value) {
  if (step == 0) *first_value = value;
  if (value <= atol) return CTRL_SUCCESS_ABS;
  if (value < rtol * (*first_value)) return CTRL_SUCCESS_REL;
  if (value > dtol * (*first_value)) return CTRL_FAIL_DIV;
  if (step >= maxits) return CTRL_FAIL_MAXITS;
  return CTRL_ITERATE;
}

template < typename T >
lVector< T > *make_vector(int impl, int n, const char *name) {
  if (impl == IMPL_OPENMP) return new CPUopenmp_lVector< T >(n, name);
  return new CPUsimple_lVector< T >(n, name);
}

// Builds a CPU CSR matrix through the reference's own COO->CSR path
// (CPU_CSR_lMatrix::TransformFromCOO, lmp/lmatrix_csr_cpu.cc:883-906), which
// also sets diag_ptr_ used by extract_invdiagelements.
template < typename T >
CPU_CSR_lMatrix< T > *make_matrix(int impl, int nthreads, int n, int nnz,
                                  const int *rowptr, const int *col,
                                  const T *val) {
  std::vector< int > rows(nnz);
  for (int i = 0; i < n; ++i)
    for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) rows[j] = i;
  CPUsimple_CSR_lMatrix< T > *sm =
      new CPUsimple_CSR_lMatrix< T >(nnz, n, n, "A");
  sm->TransformFromCOO(rows.data(), col, val, n, n, nnz);
  if (impl != IMPL_OPENMP) return sm;
  CPUopenmp_CSR_lMatrix< T > *om = new CPUopenmp_CSR_lMatrix< T >();
  om->CopyStructureFrom(*sm);
  om->CopyFrom(*sm);
  om->set_num_threads(nthreads);
  delete sm;
  return om;
}

template < typename T >
int cg_solve_on(int impl, CPU_CSR_lMatrix< T > *A, int precond, int n,
                const T *bh, T *xh, int maxits, double atol, double rtol,
                double dtol, int *iters, double *res_out, double *res_init_out,
                double *res_rel_out, double *seconds) {
  lVector< T > *b = make_vector< T >(impl, n, "b");
  lVector< T > *x = make_vector< T >(impl, n, "x");
  lVector< T > *r = make_vector< T >(impl, n, "r");
  lVector< T > *p = make_vector< T >(impl, n, "p");
  lVector< T > *z = make_vector< T >(impl, n, "z");
  lVector< T > *Ap = make_vector< T >(impl, n, "Ap");
  b->SetBlockValues(0, n, bh);
  x->SetBlockValues(0, n, xh);

  lPreconditioner_Jacobi< T > jac;
  if (precond) {
    jac.Init();
    jac.SetupOperator(*A);
    jac.SetReuse(true);
    jac.Build(r, z);
  }

  int state = CTRL_ITERATE;
  double first = 0.;
  int iter = 0;
  T alpha, beta, gamma, ressquared;
  double res;
  const auto t0 = std::chrono::steady_clock::now();

  // initialization step (cg.h:104-121 / :184-204)
  A->VectorMult(*x, r);
  r->ScaleAdd(static_cast< T >(-1.), *b); // coupled r.ScaleAdd(b, -1)
  ressquared = r->Dot(*r);
  res = std::sqrt(ressquared);
  const double res_init = res;
  state = control_check(iter, res, maxits, atol, rtol, dtol, &first);
  if (precond) {
    z->Zeros();
    jac.ApplylPreconditioner(*r, z);
    p->CopyFrom(*z);
    beta = r->Dot(*z);
  } else {
    p->CopyFrom(*r);
    beta = ressquared;
  }

  // main loop (cg.h:124-148 / :207-233)
  while (state == CTRL_ITERATE) {
    ++iter;
    A->VectorMult(*p, Ap);
    alpha = beta / (Ap->Dot(*p));
    x->Axpy(*p, alpha);
    r->Axpy(*Ap, -alpha);
    ressquared = r->Dot(*r);
    res = std::sqrt(ressquared);
    state = control_check(iter, res, maxits, atol, rtol, dtol, &first);
    if (state != CTRL_ITERATE) break;
    if (precond) {
      z->Zeros();
      jac.ApplylPreconditioner(*r, z);
      gamma = r->Dot(*z);
      beta = gamma / beta;
      p->ScaleAdd(beta, *z); // coupled p.ScaleAdd(z, beta)
      beta = gamma;
    } else {
      beta = ressquared / beta;
      p->ScaleAdd(beta, *r);
      beta = ressquared;
    }
  }

  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration< double >(t1 - t0).count();
  x->GetBlockValues(0, n, xh);
  *iters = iter;
  *res_out = res;
  *res_init_out = res_init;
  *res_rel_out = res_init > 0. ? res / res_init : 0.;
  if (precond) jac.Clear();
  delete Ap; delete z; delete p; delete r; delete x; delete b;
  return state;
}

template < typename T >
int cg_solve(int impl, int nthreads, int precond, int n, int nnz,
             const int *rowptr, const int *col, const T *val, const T *bh,
             T *xh, int maxits, double atol, double rtol, double dtol,
             int *iters, double *res_out, double *res_init_out,
             double *res_rel_out) {
  CPU_CSR_lMatrix< T > *A = make_matrix< T >(impl, nthreads, n, nnz, rowptr,
                                             col, val);
  int st = cg_solve_on< T >(impl, A, precond, n, bh, xh, maxits, atol, rtol,
                            dtol, iters, res_out, res_init_out, res_rel_out,
                            nullptr);
  delete A;
  return st;
}

template < typename T >
int spmv(int impl, int nthreads, int n, int nnz, const int *rowptr,
         const int *col, const T *val, const T *xh, T *yh) {
  CPU_CSR_lMatrix< T > *A = make_matrix< T >(impl, nthreads, n, nnz, rowptr,
                                             col, val);
  lVector< T > *x = make_vector< T >(impl, n, "x");
  lVector< T > *y = make_vector< T >(impl, n, "y");
  x->SetBlockValues(0, n, xh);
  A->VectorMult(*x, y);
  y->GetBlockValues(0, n, yh);
  delete y; delete x; delete A;
  return 0;
}

template < typename T >
int lmp_cg(int impl, int nthreads, int n, int nnz, const int *rowptr,
           const int *col, const T *val, const T *bh, T *xh, T rel_eps,
           T abs_eps, int *max_iter) {
  CPU_CSR_lMatrix< T > *A = make_matrix< T >(impl, nthreads, n, nnz, rowptr,
                                             col, val);
  lVector< T > *b = make_vector< T >(impl, n, "b");
  lVector< T > *x = make_vector< T >(impl, n, "x");
  b->SetBlockValues(0, n, bh);
  x->SetBlockValues(0, n, xh);
  int rv = cg(x, b, A, rel_eps, abs_eps, *max_iter, -1);
  x->GetBlockValues(0, n, xh);
  delete x; delete b; delete A;
  return rv;
}

// Jacobi<LAD> (linear_solver/jacobi.cc) on one rank: Prepare/BuildImpl
// (:35-63: SwapDiagElementsToRowFront, extract_invdiagelements), then
// SolveNormal/SolveDamped (:145-254: residual b - A x, Check(iter, ||r||) once
// per inner_iter sweeps) or SmoothNormal (smooth_iter * inner_iter sweeps) /
// SmoothDamped (maxits * inner_iter sweeps, :256-285).  One sweep is
// DoNormalIteration/DoDampedIteration (:288-356): y = A_nodiag x,
// y.ScaleAdd(-1, b), y .*= inv_D, then x = y or x = (1 - w) x + w y.
// Smoothing modes return CTRL_ITERATE (no stopping test).
template < typename T >
int jacobi_solve(int impl, int nthreads, int mode, int n, int nnz,
                 const int *rowptr, const int *col, const T *val, const T *bh,
                 T *xh, int maxits, int inner_iter, int smooth_iter, double w,
                 double atol, double rtol, double dtol, int *iters,
                 double *res_out, double *res_init_out, double *seconds) {
  CPU_CSR_lMatrix< T > *A = make_matrix< T >(impl, nthreads, n, nnz, rowptr,
                                             col, val);
  A->SwapDiagElementsToRowFront();
  lVector< T > *b = make_vector< T >(impl, n, "b");
  lVector< T > *x = make_vector< T >(impl, n, "x");
  lVector< T > *y = make_vector< T >(impl, n, "y");
  lVector< T > *r = make_vector< T >(impl, n, "res");
  lVector< T > *invd = make_vector< T >(impl, n, "inv_diag");
  b->SetBlockValues(0, n, bh);
  x->SetBlockValues(0, n, xh);
  A->extract_invdiagelements(0, n, invd);
  const bool damped = mode == 1 || mode == 3;
  int iter = 0;
  auto sweep = [&]() {
    ++iter;
    A->VectorMultNoDiag(*x, y);
    y->ScaleAdd(static_cast< T >(-1.0), *b);
    y->ElementWiseMult(*invd);
    if (damped) {
      x->Scale(static_cast< T >(1.0 - static_cast< T >(w)));
      x->Axpy(*y, static_cast< T >(w));
    } else {
      x->CopyFrom(*y);
    }
  };
  auto residual = [&]() -> double {
    A->VectorMult(*x, r);
    r->ScaleAdd(static_cast< T >(-1.0), *b);
    return r->Norm2();
  };
  int state = CTRL_ITERATE;
  double res = 0., first = 0.;
  *res_init_out = 0.;
  const auto t0 = std::chrono::steady_clock::now();
  if (mode <= 1) {
    res = residual();
    *res_init_out = res;
    state = control_check(iter, res, maxits, atol, rtol, dtol, &first);
    while (state == CTRL_ITERATE) {
      for (int i = 0; i < inner_iter; ++i) sweep();
      res = residual();
      state = control_check(iter, res, maxits, atol, rtol, dtol, &first);
    }
  } else {
    const int outer = mode == 2 ? smooth_iter : maxits;
    for (int k = 0; k < outer; ++k)
      for (int i = 0; i < inner_iter; ++i) sweep();
  }
  if (seconds)
    *seconds = std::chrono::duration< double >(
                   std::chrono::steady_clock::now() - t0).count();
  x->GetBlockValues(0, n, xh);
  *iters = iter;
  *res_out = res;
  delete invd; delete r; delete y; delete x; delete b; delete A;
  return state;
}

// BiCGSTAB<LAD>::SolveNoPrecond / SolvePrecondRight (linear_solver/
// bicgstab.h:127-293, :297-473) on one rank with the block-Jacobi(Jacobi)
// preconditioner: the same sequence of compiled lVector/lMatrix calls,
// including the restart when |sigma| <= tol1 (r0 recomputed from the current
// x, the iteration count carried on) and the short update when ||s|| is at
// rounding level.  The coupled calls map to the interior ones as
// r0.ScaleAdd(b, -1) -> r0.ScaleAdd(-1, b) and p.ScaleAdd(r, beta) ->
// p.ScaleAdd(beta, r) (coupled_vector.cc:353-358).
template < typename T >
int bicgstab_solve(int impl, int nthreads, int precond, int n, int nnz,
                   const int *rowptr, const int *col, const T *val,
                   const T *bh, T *xh, int maxits, double atol, double rtol,
                   double dtol, int *iters, int *restarts, double *res_out,
                   double *res_init_out, double *seconds) {
  CPU_CSR_lMatrix< T > *A = make_matrix< T >(impl, nthreads, n, nnz, rowptr,
                                             col, val);
  const char *names[] = {"b", "x", "r", "r0", "p", "Ap", "s", "t", "h", "h1"};
  lVector< T > *v[10];
  for (int i = 0; i < 10; ++i) v[i] = make_vector< T >(impl, n, names[i]);
  lVector< T > &b = *v[0], &x = *v[1], &r = *v[2], &r0 = *v[3], &p = *v[4];
  lVector< T > &Ap = *v[5], &s = *v[6], &t = *v[7], &h = *v[8], &h1 = *v[9];
  b.SetBlockValues(0, n, bh);
  x.SetBlockValues(0, n, xh);
  lPreconditioner_Jacobi< T > jac;
  if (precond) {
    jac.Init();
    jac.SetupOperator(*A);
    jac.SetReuse(true);
    jac.Build(&r, &h);
  }
  const T eps = precond ? static_cast< T >(5.e-16) : static_cast< T >(1.e-15);
  T alpha, beta, ressquared, rho, rho_old, omega, sigma, tol1;
  int iter = 0, nrestart = -1, conv = CTRL_ITERATE;
  double res = 0., first = 0.;
  bool restart = true;
  const auto t0 = std::chrono::steady_clock::now();
  while (restart) {
    restart = false;
    ++nrestart;
    r.Zeros(); r0.Zeros(); p.Zeros(); Ap.Zeros(); s.Zeros(); t.Zeros();
    h.Zeros(); h1.Zeros();
    A->VectorMult(x, &r0);
    r0.ScaleAdd(static_cast< T >(-1.), b);
    r.CopyFrom(r0);
    ressquared = r.Dot(r);
    rho = rho_old = ressquared;
    res = std::sqrt(ressquared);
    *res_init_out = res;
    conv = control_check(iter, res, maxits, atol, rtol, dtol, &first);
    p.CopyFrom(r);
    while (conv == CTRL_ITERATE && !restart) {
      ++iter;
      if (precond) {
        h.Zeros();
        jac.ApplylPreconditioner(p, &h);
        A->VectorMult(h, &Ap);
      } else {
        A->VectorMult(p, &Ap);
      }
      sigma = Ap.Dot(r0);
      tol1 = eps * Ap.Norm2() * r0.Norm2();
      if (std::abs(sigma) > tol1) {
        alpha = rho / sigma;
        s.CopyFrom(r);
        s.Axpy(Ap, -alpha);
        if (s.Norm2() > eps) {
          if (precond) {
            h.Zeros();
            jac.ApplylPreconditioner(s, &h);
            A->VectorMult(h, &t);
          } else {
            A->VectorMult(s, &t);
          }
          omega = t.Dot(s) / t.Dot(t);
          if (precond) {
            h.Zeros();
            h1.Zeros();
            h1.Axpy(p, alpha);
            h1.Axpy(s, omega);
            jac.ApplylPreconditioner(h1, &h);
            x.Axpy(h, static_cast< T >(1.));
          } else {
            x.Axpy(p, alpha);
            x.Axpy(s, omega);
          }
          r.CopyFrom(s);
          r.Axpy(t, -omega);
          ressquared = r.Dot(r);
          res = std::sqrt(ressquared);
          conv = control_check(iter, res, maxits, atol, rtol, dtol, &first);
          if (conv != CTRL_ITERATE) break;
          rho = r.Dot(r0);
          beta = (alpha * rho) / (omega * rho_old);
          rho_old = rho;
          p.ScaleAdd(beta, r);
          p.Axpy(Ap, -omega * beta);
        } else {
          if (precond) {
            h1.Zeros();
            h1.Axpy(p, alpha);
            h.Zeros();
            jac.ApplylPreconditioner(h1, &h);
            x.Axpy(h, static_cast< T >(1.));
          } else {
            x.Axpy(p, alpha);
          }
          r.CopyFrom(s);
          ressquared = r.Dot(r);
          res = std::sqrt(ressquared);
          conv = control_check(iter, res, maxits, atol, rtol, dtol, &first);
          if (conv != CTRL_ITERATE) break;
        }
      } else {
        restart = true;
      }
    }
  }
  if (seconds)
    *seconds = std::chrono::duration< double >(
                   std::chrono::steady_clock::now() - t0).count();
  x.GetBlockValues(0, n, xh);
  *iters = iter;
  *restarts = nrestart;
  *res_out = res;
  if (precond) jac.Clear();
  for (int i = 9; i >= 0; --i) delete v[i];
  delete A;
  return conv;
}

// GMRES<LAD, PreLAD>::SolveNoPrecond / SolveRight (linear_solver/gmres.h:
// 229-389, 462-713) on one rank over the compiled lmp objects, with the
// Givens helpers (:97-115) and UpdateSolution (:727-746).  H is the
// reference's SeqDenseMatrix H(row j, column i) of m rows and m + 1 columns.
template < typename T >
int gmres_solve(int impl, int nthreads, int precond, int n, int nnz,
                const int *rowptr, const int *col, const T *val, const T *bh,
                T *xh, int size_basis, int maxits, double atol, double rtol,
                double dtol, int *iters, double *res_out, double *res_init_out,
                double *seconds) {
  CPU_CSR_lMatrix< T > *A = make_matrix< T >(impl, nthreads, n, nnz, rowptr,
                                             col, val);
  const int m = std::min(size_basis, maxits);
  std::vector< lVector< T > * > V(m + 1);
  for (int i = 0; i <= m; ++i) V[i] = make_vector< T >(impl, n, "V");
  lVector< T > *b = make_vector< T >(impl, n, "b");
  lVector< T > *x = make_vector< T >(impl, n, "x");
  lVector< T > *w = make_vector< T >(impl, n, "w");
  lVector< T > *z = make_vector< T >(impl, n, "z");
  b->SetBlockValues(0, n, bh);
  x->SetBlockValues(0, n, xh);
  lPreconditioner_Jacobi< T > jac;
  if (precond) {
    jac.Init();
    jac.SetupOperator(*A);
    jac.SetReuse(true);
    jac.Build(w, z);
  }
  const int ld = m + 1;
  std::vector< T > H((size_t)std::max(m, 1) * ld), g(ld), cs(ld), sn(ld);
  auto rot = [](T c, T s_, T *dx, T *dy) {
    const T temp = c * (*dx) + s_ * (*dy);
    *dy = -s_ * (*dx) + c * (*dy);
    *dx = temp;
  };
  auto update = [&](int k, lVector< T > *out) {
    std::vector< T > y(g);
    for (int i = k + 1; (i--) != 0;) {
      y[i] /= H[i * ld + i];
      const T temp = y[i];
      for (int j = 0; j < i; ++j) y[j] -= H[i * ld + j] * temp;
    }
    for (int j = 0; j <= k; ++j) out->Axpy(*V[j], y[j]);
  };
  int iter = 0, conv;
  double first = 0.;
  const auto t0 = std::chrono::steady_clock::now();
  A->VectorMult(*x, V[0]);
  V[0]->ScaleAdd(static_cast< T >(-1.), *b);
  T res = V[0]->Norm2();
  *res_init_out = res;
  conv = control_check(iter, res, maxits, atol, rtol, dtol, &first);
  while (conv == CTRL_ITERATE) {
    std::fill(g.begin(), g.end(), static_cast< T >(0.));
    std::fill(H.begin(), H.end(), static_cast< T >(0.));
    V[0]->Scale(static_cast< T >(1.) / res);
    g[0] = res;
    int j = 0;
    for (; j != m; ++j) {
      ++iter;
      if (precond) {
        z->Zeros();
        jac.ApplylPreconditioner(*V[j], z);
        A->VectorMult(*z, w);
      } else {
        A->VectorMult(*V[j], w);
      }
      for (int i = 0; i <= j; ++i) {
        H[j * ld + i] = w->Dot(*V[i]);
        w->Axpy(*V[i], static_cast< T >(-1.) * H[j * ld + i]);
      }
      H[j * ld + j + 1] = w->Norm2();
      w->Scale(static_cast< T >(1.) / H[j * ld + j + 1]);
      V[j + 1]->CopyFrom(*w);
      for (int k = 0; k != j; ++k) rot(cs[k], sn[k], &H[j * ld + k], &H[j * ld + k + 1]);
      {
        const T dx = H[j * ld + j], dy = H[j * ld + j + 1];
        const T beta = std::sqrt(dx * dx + dy * dy);
        cs[j] = dx / beta;
        sn[j] = dy / beta;
      }
      rot(cs[j], sn[j], &H[j * ld + j], &H[j * ld + j + 1]);
      rot(cs[j], sn[j], &g[j], &g[j + 1]);
      res = std::abs(g[j + 1]);
      conv = control_check(iter, res, maxits, atol, rtol, dtol, &first);
      if (conv != CTRL_ITERATE) break;
    }
    const int k = conv != CTRL_ITERATE ? j : m - 1;
    if (precond) {
      z->Zeros();
      update(k, z);
      w->Zeros();
      jac.ApplylPreconditioner(*z, w);
      x->Axpy(*w, static_cast< T >(1.));
    } else {
      update(k, x);
    }
    if (conv == CTRL_ITERATE) {
      A->VectorMult(*x, V[0]);
      V[0]->ScaleAdd(static_cast< T >(-1.), *b);
    }
  }
  if (seconds)
    *seconds = std::chrono::duration< double >(
                   std::chrono::steady_clock::now() - t0).count();
  x->GetBlockValues(0, n, xh);
  *iters = iter;
  *res_out = res;
  if (precond) jac.Clear();
  delete z; delete w; delete x; delete b;
  for (int i = m; i >= 0; --i) delete V[i];
  delete A;
  return conv;
}

struct RefSystem {
  int impl;
  int n;
  CPU_CSR_lMatrix< double > *A;
};

} // namespace

extern "C" {

// A matrix built once (reference COO->CSR path), for repeated timed solves:
// the solve time reported by ref_system_cg excludes matrix construction.
void *ref_system_create(int impl, int nthreads, int n, int nnz,
                        const int *rowptr, const int *col, const double *val) {
  RefSystem *s = new RefSystem;
  s->impl = impl;
  s->n = n;
  s->A = make_matrix< double >(impl, nthreads, n, nnz, rowptr, col, val);
  return s;
}

void ref_system_destroy(void *h) {
  RefSystem *s = static_cast< RefSystem * >(h);
  if (!s) return;
  delete s->A;
  delete s;
}

int ref_system_cg(void *h, int precond, const double *b, double *x,
                  int maxits, double atol, double rtol, double dtol,
                  int *iters, double *res, double *res_init, double *seconds) {
  RefSystem *s = static_cast< RefSystem * >(h);
  double rel = 0.;
  return cg_solve_on< double >(s->impl, s->A, precond, s->n, b, x, maxits,
                               atol, rtol, dtol, iters, res, res_init, &rel,
                               seconds);
}

int ref_spmv_d(int impl, int nthreads, int n, int nnz, const int *rowptr,
               const int *col, const double *val, const double *x, double *y) {
  return spmv< double >(impl, nthreads, n, nnz, rowptr, col, val, x, y);
}

int ref_spmv_f(int impl, int nthreads, int n, int nnz, const int *rowptr,
               const int *col, const float *val, const float *x, float *y) {
  return spmv< float >(impl, nthreads, n, nnz, rowptr, col, val, x, y);
}

int ref_cg_solve_d(int impl, int nthreads, int precond, int n, int nnz,
                   const int *rowptr, const int *col, const double *val,
                   const double *b, double *x, int maxits, double atol,
                   double rtol, double dtol, int *iters, double *res,
                   double *res_init, double *res_rel) {
  return cg_solve< double >(impl, nthreads, precond, n, nnz, rowptr, col, val,
                            b, x, maxits, atol, rtol, dtol, iters, res,
                            res_init, res_rel);
}

int ref_cg_solve_f(int impl, int nthreads, int precond, int n, int nnz,
                   const int *rowptr, const int *col, const float *val,
                   const float *b, float *x, int maxits, double atol,
                   double rtol, double dtol, int *iters, double *res,
                   double *res_init, double *res_rel) {
  return cg_solve< float >(impl, nthreads, precond, n, nnz, rowptr, col, val,
                           b, x, maxits, atol, rtol, dtol, iters, res,
                           res_init, res_rel);
}

int ref_jacobi_solve_d(int impl, int nthreads, int mode, int n, int nnz,
                       const int *rowptr, const int *col, const double *val,
                       const double *b, double *x, int maxits, int inner_iter,
                       int smooth_iter, double w, double atol, double rtol,
                       double dtol, int *iters, double *res,
                       double *res_init, double *seconds) {
  return jacobi_solve< double >(impl, nthreads, mode, n, nnz, rowptr, col, val,
                                b, x, maxits, inner_iter, smooth_iter, w, atol,
                                rtol, dtol, iters, res, res_init, seconds);
}

int ref_bicgstab_solve_d(int impl, int nthreads, int precond, int n, int nnz,
                         const int *rowptr, const int *col, const double *val,
                         const double *b, double *x, int maxits, double atol,
                         double rtol, double dtol, int *iters, int *restarts,
                         double *res, double *res_init, double *seconds) {
  return bicgstab_solve< double >(impl, nthreads, precond, n, nnz, rowptr, col,
                                  val, b, x, maxits, atol, rtol, dtol, iters,
                                  restarts, res, res_init, seconds);
}

int ref_gmres_solve_d(int impl, int nthreads, int precond, int n, int nnz,
                      const int *rowptr, const int *col, const double *val,
                      const double *b, double *x, int size_basis, int maxits,
                      double atol, double rtol, double dtol, int *iters,
                      double *res, double *res_init, double *seconds) {
  return gmres_solve< double >(impl, nthreads, precond, n, nnz, rowptr, col,
                               val, b, x, size_basis, maxits, atol, rtol, dtol,
                               iters, res, res_init, seconds);
}

// CPU_CSR_lMatrix::TransformFromCOO (lmp/lmatrix_csr_cpu.cc:883-906, which
// calls coo_2_csr, lmp/lmatrix_formats.h:320-452) on host COO arrays; the CSR
// arrays are copied out of the matrix's storage.
int ref_coo_to_csr_d(int nrow, int ncol, int nnz, const int *rows,
                     const int *cols, const double *vals, int *rowptr_out,
                     int *col_out, double *val_out) {
  CPUsimple_CSR_lMatrix< double > m(nnz, nrow, ncol, "coo");
  m.TransformFromCOO(rows, cols, vals, nrow, ncol, nnz);
  for (int i = 0; i <= nrow; ++i) rowptr_out[i] = m.matrix.row[i];
  for (int k = 0; k < nnz; ++k) {
    col_out[k] = m.matrix.col[k];
    val_out[k] = m.matrix.val[k];
  }
  return 0;
}

int ref_lmp_cg_d(int impl, int nthreads, int n, int nnz, const int *rowptr,
                 const int *col, const double *val, const double *b, double *x,
                 double rel_eps, double abs_eps, int *max_iter) {
  return lmp_cg< double >(impl, nthreads, n, nnz, rowptr, col, val, b, x,
                          rel_eps, abs_eps, max_iter);
}

} // extern "C"
