/*
 * CPU oracle for the PCG hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of HiFlow3's CPU algorithms for the Jacobi-PCG path,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as
 * the checker.  The product library (ba_b200/) never links or calls this.
 * Built by oracle/Makefile into oracle/liboracle.so.
 *
 * Parity is pinned in two ways: against the known answers in the reference's
 * own tests (tests/cg_test.cc:92-94, tests/lmp_test.cc:80-82,
 * tests/cuda_test.cc:76-78; committed as tests/golden/), and against the
 * reference's own lmp sources compiled into oracle/_ref/ (oracle/ref/).
 *
 * Every routine is instantiated for double (suffix _d) and float (suffix _f);
 * arithmetic and accumulation happen in that type, as in the reference's
 * templates.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* IterateControl states, numbered as the B200 library's solver status. */
enum { CTRL_ITERATE = 0, CTRL_SUCCESS_ABS = 1, CTRL_SUCCESS_REL = 2,
       CTRL_FAIL_DIV = 3, CTRL_FAIL_MAXITS = 4 };

/* IterateControl::Check (common/iterate_control.cc:80-107): the first call
 * (step 0) records the initial residual; success if res <= atol or
 * res < rtol * res0 (strict); divergence if res > dtol * res0; failure once
 * step >= maxits. */
int orc_iterate_check(int step, double value, int maxits, double atol,
                      double rtol, double dtol, double *first_value) {
  if (step == 0) *first_value = value;
  if (value <= atol) return CTRL_SUCCESS_ABS;
  if (value < rtol * (*first_value)) return CTRL_SUCCESS_REL;
  if (value > dtol * (*first_value)) return CTRL_FAIL_DIV;
  if (step >= maxits) return CTRL_FAIL_MAXITS;
  return CTRL_ITERATE;
}

#define ORACLE_INSTANTIATE(T, S, SQRT)                                            \
  /* CPUsimple_CSR_lMatrix::VectorMult (lmp/CPUsimple_csr_lmatrix.cc:92-111):  \
   * y_i = sum_j val[j] * x[col[j]] in stored order, accumulated in T. */      \
  void orc_spmv_##S(int n, const int *rowptr, const int *col, const T *val,    \
                    const T *x, T *y) {                                        \
    for (int i = 0; i < n; ++i) {                                              \
      T res = 0;                                                               \
      for (int j = rowptr[i]; j != rowptr[i + 1]; ++j)                         \
        res += val[j] * x[col[j]];                                             \
      y[i] = res;                                                              \
    }                                                                          \
  }                                                                            \
  /* CPUsimple_lVector::Dot (lmp/CPUsimple_lvector.cc:162-222): that file     \
   * defines CLANG_VECTORIZE (:29), so the sum is one accumulator fed first    \
   * with the n % 5 leading products one by one, then with groups of five      \
   * products each summed left to right before being added. */                \
  T orc_dot_##S(int n, const T *a, const T *b) {                               \
    T acc = 0;                                                                 \
    const int m = n % 5;                                                       \
    for (int i = 0; i < m; ++i) acc += a[i] * b[i];                            \
    for (int i = m; i + 4 < n; i += 5)                                         \
      acc += a[i] * b[i] + a[i + 1] * b[i + 1] + a[i + 2] * b[i + 2] +         \
             a[i + 3] * b[i + 3] + a[i + 4] * b[i + 4];                        \
    return acc;                                                                \
  }                                                                            \
  /* CPUsimple_lVector::Axpy (lmp/CPUsimple_lvector.cc:254-310):               \
   * this += scalar * vec. */                                                  \
  void orc_axpy_##S(int n, T *y, const T *x, T alpha) {                        \
    for (int i = 0; i < n; ++i) y[i] += alpha * x[i];                          \
  }                                                                            \
  /* CPUsimple_lVector::ScaleAdd (lmp/CPUsimple_lvector.cc:329-395):           \
   * this = scalar * this + vec. */                                            \
  void orc_scaleadd_##S(int n, T *y, T scalar, const T *x) {                   \
    for (int i = 0; i < n; ++i) y[i] = scalar * y[i] + x[i];                   \
  }                                                                            \
  /* CPU_lVector::ElementWiseMult (lmp/lvector_cpu.cc:485-493). */             \
  void orc_ewmult_##S(int n, T *y, const T *x) {                               \
    for (int i = 0; i < n; ++i) y[i] *= x[i];                                  \
  }                                                                            \
  /* CPU_CSR_lMatrix::extract_invdiagelements (lmp/lmatrix_csr_cpu.cc:         \
   * 2426-2441): inv_D[i] = 1 / a_ii, a_ii the first stored entry of row i     \
   * whose column is i (diag_ptr_).  Returns the first row without a nonzero   \
   * diagonal, or -1. */                                                       \
  int orc_invdiag_##S(int n, const int *rowptr, const int *col, const T *val,  \
                      T *invd) {                                               \
    for (int i = 0; i < n; ++i) {                                              \
      int k = -1;                                                              \
      for (int j = rowptr[i]; j < rowptr[i + 1]; ++j)                          \
        if (col[j] == i) { k = j; break; }                                     \
      if (k < 0 || val[k] == 0) return i;                                      \
      invd[i] = (T)(1. / val[k]);                                              \
    }                                                                          \
    return -1;                                                                 \
  }                                                                            \
  /* CG<LAD>::SolveNoPrecond / SolvePrecond (linear_solver/cg.h:87-246) on one \
   * rank, with the block-Jacobi(Jacobi) preconditioner                        \
   * (lmp/lpreconditioner.cc:184-200: z = copy(r) .* inv_D).  work must hold   \
   * 4n (no precond) or 5n (Jacobi) values.  Returns the IterateControl        \
   * state; iters/res/res_init follow CG's iter_/res_/res_init_. */            \
  int orc_cg_##S(int n, const int *rowptr, const int *col, const T *val,       \
                 const T *b, T *x, int maxits, double atol, double rtol,       \
                 double dtol, int precond, const T *invd, T *work, int *iters, \
                 double *res_out, double *res_init_out) {                      \
    T *r = work, *p = work + n, *Ap = work + 2 * (size_t)n;                    \
    T *z = work + 3 * (size_t)n;                                               \
    T alpha, beta, gamma, ressq;                                               \
    double res, first = 0.;                                                    \
    int iter = 0, state;                                                       \
    orc_spmv_##S(n, rowptr, col, val, x, r);                                   \
    orc_scaleadd_##S(n, r, (T)-1., b);                                         \
    ressq = orc_dot_##S(n, r, r);                                              \
    res = (double)SQRT(ressq);                                                 \
    *res_init_out = res;                                                       \
    state = orc_iterate_check(iter, res, maxits, atol, rtol, dtol, &first);    \
    if (precond) {                                                             \
      for (int i = 0; i < n; ++i) z[i] = r[i];                                 \
      orc_ewmult_##S(n, z, invd);                                              \
      for (int i = 0; i < n; ++i) p[i] = z[i];                                 \
      beta = orc_dot_##S(n, r, z);                                             \
    } else {                                                                   \
      for (int i = 0; i < n; ++i) p[i] = r[i];                                 \
      beta = ressq;                                                            \
    }                                                                          \
    while (state == CTRL_ITERATE) {                                            \
      ++iter;                                                                  \
      orc_spmv_##S(n, rowptr, col, val, p, Ap);                                \
      alpha = beta / orc_dot_##S(n, Ap, p);                                    \
      orc_axpy_##S(n, x, p, alpha);                                            \
      orc_axpy_##S(n, r, Ap, -alpha);                                          \
      ressq = orc_dot_##S(n, r, r);                                            \
      res = (double)SQRT(ressq);                                               \
      state = orc_iterate_check(iter, res, maxits, atol, rtol, dtol, &first);  \
      if (state != CTRL_ITERATE) break;                                        \
      if (precond) {                                                           \
        for (int i = 0; i < n; ++i) z[i] = r[i];                               \
        orc_ewmult_##S(n, z, invd);                                            \
        gamma = orc_dot_##S(n, r, z);                                          \
        beta = gamma / beta;                                                   \
        orc_scaleadd_##S(n, p, beta, z);                                       \
        beta = gamma;                                                          \
      } else {                                                                 \
        beta = ressq / beta;                                                   \
        orc_scaleadd_##S(n, p, beta, r);                                       \
        beta = ressq;                                                          \
      }                                                                        \
    }                                                                          \
    *iters = iter;                                                             \
    *res_out = res;                                                            \
    return state;                                                              \
  }                                                                            \
  /* lmp cg() / CGFunctor::operator() (lmp/solvers/cg.h:93-209): plain CG      \
   * (the reference computes z but never uses it, cg.h:153 vs :157), stop on   \
   * norm <= max(rel_eps * norm0, abs_eps) checked after each update; on exit  \
   * max_iter holds the 0-based index of the breaking iteration (cg.h:201). */ \
  int orc_lmp_cg_##S(int n, const int *rowptr, const int *col, const T *val,   \
                     const T *b, T *x, T rel_eps, T abs_eps, int *max_iter,    \
                     T *work) {                                                \
    T *p = work, *q = work + n, *r = work + 2 * (size_t)n;                     \
    for (int i = 0; i < n; ++i) p[i] = 0;                                      \
    orc_spmv_##S(n, rowptr, col, val, x, r);                                   \
    orc_scaleadd_##S(n, r, (T)-1.0, b);                                        \
    T rho = orc_dot_##S(n, r, r);                                              \
    T norm = SQRT(rho);                                             \
    T beta = 0, rho_old;                                                       \
    T crit = rel_eps * norm > abs_eps ? rel_eps * norm : abs_eps;              \
    int iter = 0;                                                              \
    for (; iter < *max_iter; ++iter) {                                         \
      orc_scaleadd_##S(n, p, beta, r);                                         \
      orc_spmv_##S(n, rowptr, col, val, p, q);                                 \
      T alpha = rho / orc_dot_##S(n, p, q);                                    \
      orc_axpy_##S(n, x, p, alpha);                                            \
      orc_axpy_##S(n, r, q, -alpha);                                           \
      rho_old = rho;                                                           \
      rho = orc_dot_##S(n, r, r);                                              \
      beta = rho / rho_old;                                                    \
      norm = SQRT(rho);                                             \
      if (norm <= crit) break;                                                 \
    }                                                                          \
    *max_iter = iter;                                                          \
    return 0;                                                                  \
  }

ORACLE_INSTANTIATE(double, d, sqrt)
ORACLE_INSTANTIATE(float, f, sqrtf)

/*
 * Jacobi<LAD> and BiCGSTAB<LAD> on one rank, over the routines above.
 */
#define ORACLE_KRYLOV(T, S, SQRT, FABS)                                           \
  /* CPU_CSR_lMatrix::SwapDiagElementsToRowFront (lmp/lmatrix_csr_cpu.cc:      \
   * 430-454): in each row the first entry whose column is the row trades      \
   * places (value and column) with the row's first entry. */                 \
  static void orc_swap_diag_##S(int n, const int *rowptr, int *col, T *val) {  \
    for (int i = 0; i < n; ++i)                                                \
      for (int j = rowptr[i]; j < rowptr[i + 1]; ++j)                          \
        if (col[j] == i) {                                                     \
          const int j0 = rowptr[i];                                            \
          T tv = val[j0]; val[j0] = val[j]; val[j] = tv;                       \
          int tc = col[j0]; col[j0] = col[j]; col[j] = tc;                     \
          break;                                                               \
        }                                                                      \
  }                                                                            \
  /* CPU_CSR_lMatrix::VectorMultNoDiag (lmp/lmatrix_csr_cpu.cc:479-492):       \
   * y_i = sum over stored j with col[j] != i, in stored order. */             \
  void orc_spmv_nodiag_##S(int n, const int *rowptr, const int *col,           \
                           const T *val, const T *x, T *y) {                   \
    for (int i = 0; i < n; ++i) {                                              \
      T res = 0;                                                               \
      for (int j = rowptr[i]; j < rowptr[i + 1]; ++j)                          \
        if (col[j] != i) res += val[j] * x[col[j]];                            \
      y[i] = res;                                                              \
    }                                                                          \
  }                                                                            \
  /* Jacobi<LAD> (linear_solver/jacobi.cc): Prepare (:35-63) moves each       \
   * diagonal entry to the front of its row and takes inv_D = 1/a_ii;         \
   * mode 0/1 = SolveNormal/SolveDamped (:145-254): Check(iter, ||b - A x||)   \
   * before the loop and after every inner_iter sweeps; mode 2 = SmoothNormal \
   * (smooth_iter * inner_iter sweeps), mode 3 = SmoothDamped (maxits *       \
   * inner_iter sweeps; the reference loops to maxits_ there, :276).  A sweep \
   * (:288-356): y = A_nodiag x; y = -y + b; y .*= inv_D; x = y, or           \
   * x = (1 - w) x + w y.  Smoothing modes return CTRL_ITERATE; -2 if a       \
   * diagonal entry is missing or zero; -3 if out of memory. */              \
  int orc_jacobi_##S(int n, const int *rowptr, const int *col_in,              \
                     const T *val_in, const T *b, T *x, int mode, int maxits,  \
                     int inner_iter, int smooth_iter, double w, double atol,   \
                     double rtol, double dtol, int *iters, double *res_out,    \
                     double *res_init_out) {                                   \
    const int nnz = rowptr[n];                                                 \
    int *col = (int *)malloc(sizeof(int) * (size_t)(nnz > 0 ? nnz : 1));       \
    T *val = (T *)malloc(sizeof(T) * (size_t)(nnz > 0 ? nnz : 1));             \
    T *work = (T *)malloc(sizeof(T) * 3 * (size_t)(n > 0 ? n : 1));            \
    if (!col || !val || !work) {                                               \
      free(col); free(val); free(work);                                        \
      return -3;                                                               \
    }                                                                          \
    T *invd = work, *y = work + n, *r = work + 2 * (size_t)n;                  \
    memcpy(col, col_in, sizeof(int) * (size_t)nnz);                            \
    memcpy(val, val_in, sizeof(T) * (size_t)nnz);                              \
    orc_swap_diag_##S(n, rowptr, col, val);                                    \
    int state = CTRL_ITERATE, iter = 0;                                        \
    double res = 0., first = 0.;                                               \
    *res_init_out = 0.;                                                        \
    if (orc_invdiag_##S(n, rowptr, col, val, invd) >= 0) {                     \
      state = -2;                                                              \
      goto done;                                                               \
    }                                                                          \
    const int damped = mode == 1 || mode == 3;                                 \
    const T tw = (T)w, keep = (T)(1.0 - tw);                                   \
    for (int k = 0, outer = mode == 2 ? smooth_iter : maxits;; ++k) {          \
      if (mode <= 1) {                                                         \
        orc_spmv_##S(n, rowptr, col, val, x, r);                               \
        orc_scaleadd_##S(n, r, (T)-1., b);                                     \
        res = (double)SQRT(orc_dot_##S(n, r, r));                              \
        if (iter == 0) *res_init_out = res;                                    \
        state = orc_iterate_check(iter, res, maxits, atol, rtol, dtol,        \
                                  &first);                                     \
        if (state != CTRL_ITERATE) break;                                      \
      } else if (k >= outer) {                                                 \
        break;                                                                 \
      }                                                                        \
      for (int i = 0; i < inner_iter; ++i) {                                   \
        ++iter;                                                                \
        orc_spmv_nodiag_##S(n, rowptr, col, val, x, y);                        \
        orc_scaleadd_##S(n, y, (T)-1., b);                                     \
        orc_ewmult_##S(n, y, invd);                                            \
        if (damped) {                                                          \
          for (int q = 0; q < n; ++q) x[q] *= keep;                            \
          orc_axpy_##S(n, x, y, tw);                                           \
        } else {                                                               \
          memcpy(x, y, sizeof(T) * (size_t)n);                                 \
        }                                                                      \
      }                                                                        \
    }                                                                          \
  done:                                                                        \
    *iters = iter;                                                             \
    *res_out = res;                                                            \
    free(col); free(val); free(work);                                          \
    return state;                                                              \
  }                                                                            \
  /* BiCGSTAB<LAD>::SolveNoPrecond / SolvePrecondRight (linear_solver/         \
   * bicgstab.h:127-293, :297-473) with the Jacobi preconditioner h = copy(v) \
   * .* inv_D.  A step: Ap = A (P) p; sigma = Ap.r0; restart (r0 = b - A x,    \
   * r = p = r0, the count carried on) unless |sigma| > eps ||Ap|| ||r0||;    \
   * alpha = rho / sigma; s = r - alpha Ap; if ||s|| > eps: t = A (P) s,       \
   * omega = t.s / t.t, x += (P)(alpha p + omega s), r = s - omega t, check,  \
   * rho = r.r0, beta = alpha rho / (omega rho_old), p = beta p + r - omega    \
   * beta Ap; else x += (P)(alpha p), r = s, check.  eps = 1e-15 without,     \
   * 5e-16 with preconditioner.  restarts counts the restarts after the       \
   * first start; every restart follows a counted step, so IterateControl    \
   * ends the loop at maxits.  Returns the IterateControl state, -3 if out of \
   * memory. */                                                               \
  int orc_bicgstab_##S(int n, const int *rowptr, const int *col, const T *val, \
                       const T *b, T *x, int precond, const T *invd,           \
                       int maxits, double atol, double rtol, double dtol,      \
                       int *iters, int *restarts, double *res_out,             \
                       double *res_init_out) {                                 \
    T *w = (T *)malloc(sizeof(T) * 8 * (size_t)(n > 0 ? n : 1));               \
    if (!w) return -3;                                                         \
    T *r = w, *r0 = w + n, *p = w + 2 * (size_t)n, *Ap = w + 3 * (size_t)n;    \
    T *s = w + 4 * (size_t)n, *t = w + 5 * (size_t)n, *h = w + 6 * (size_t)n;  \
    T *h1 = w + 7 * (size_t)n;                                                 \
    const T eps = precond ? (T)5.e-16 : (T)1.e-15;                             \
    T alpha = 0, beta, ressq, rho, rho_old, omega, sigma, tol1;                \
    int iter = 0, nrestart = -1, conv = CTRL_ITERATE, restart = 1;             \
    double res = 0., first = 0.;                                               \
    while (restart) {                                                          \
      restart = 0;                                                             \
      ++nrestart;                                                              \
      memset(w, 0, sizeof(T) * 8 * (size_t)n);                                 \
      orc_spmv_##S(n, rowptr, col, val, x, r0);                                \
      orc_scaleadd_##S(n, r0, (T)-1., b);                                      \
      memcpy(r, r0, sizeof(T) * (size_t)n);                                    \
      ressq = orc_dot_##S(n, r, r);                                            \
      rho = rho_old = ressq;                                                   \
      res = (double)SQRT(ressq);                                               \
      *res_init_out = res;                                                     \
      conv = orc_iterate_check(iter, res, maxits, atol, rtol, dtol, &first);   \
      memcpy(p, r, sizeof(T) * (size_t)n);                                     \
      while (conv == CTRL_ITERATE && !restart) {                               \
        ++iter;                                                                \
        if (precond) {                                                         \
          memcpy(h, p, sizeof(T) * (size_t)n);                                 \
          orc_ewmult_##S(n, h, invd);                                          \
          orc_spmv_##S(n, rowptr, col, val, h, Ap);                            \
        } else {                                                               \
          orc_spmv_##S(n, rowptr, col, val, p, Ap);                            \
        }                                                                      \
        sigma = orc_dot_##S(n, Ap, r0);                                        \
        tol1 = eps * SQRT(orc_dot_##S(n, Ap, Ap)) * SQRT(orc_dot_##S(n, r0, r0)); \
        if (!(FABS(sigma) > tol1)) {                                           \
          restart = 1;                                                         \
          break;                                                               \
        }                                                                      \
        alpha = rho / sigma;                                                   \
        memcpy(s, r, sizeof(T) * (size_t)n);                                   \
        orc_axpy_##S(n, s, Ap, -alpha);                                        \
        if (SQRT(orc_dot_##S(n, s, s)) > eps) {                                \
          if (precond) {                                                       \
            memcpy(h, s, sizeof(T) * (size_t)n);                               \
            orc_ewmult_##S(n, h, invd);                                        \
            orc_spmv_##S(n, rowptr, col, val, h, t);                           \
          } else {                                                             \
            orc_spmv_##S(n, rowptr, col, val, s, t);                           \
          }                                                                    \
          omega = orc_dot_##S(n, t, s) / orc_dot_##S(n, t, t);                 \
          if (precond) {                                                       \
            memset(h1, 0, sizeof(T) * (size_t)n);                              \
            orc_axpy_##S(n, h1, p, alpha);                                     \
            orc_axpy_##S(n, h1, s, omega);                                     \
            memcpy(h, h1, sizeof(T) * (size_t)n);                              \
            orc_ewmult_##S(n, h, invd);                                        \
            orc_axpy_##S(n, x, h, (T)1.);                                      \
          } else {                                                             \
            orc_axpy_##S(n, x, p, alpha);                                      \
            orc_axpy_##S(n, x, s, omega);                                      \
          }                                                                    \
          memcpy(r, s, sizeof(T) * (size_t)n);                                 \
          orc_axpy_##S(n, r, t, -omega);                                       \
          ressq = orc_dot_##S(n, r, r);                                        \
          res = (double)SQRT(ressq);                                           \
          conv = orc_iterate_check(iter, res, maxits, atol, rtol, dtol, &first); \
          if (conv != CTRL_ITERATE) break;                                     \
          rho = orc_dot_##S(n, r, r0);                                         \
          beta = (alpha * rho) / (omega * rho_old);                            \
          rho_old = rho;                                                       \
          orc_scaleadd_##S(n, p, beta, r);                                     \
          orc_axpy_##S(n, p, Ap, -omega * beta);                               \
        } else {                                                               \
          if (precond) {                                                       \
            memset(h1, 0, sizeof(T) * (size_t)n);                              \
            orc_axpy_##S(n, h1, p, alpha);                                     \
            memcpy(h, h1, sizeof(T) * (size_t)n);                              \
            orc_ewmult_##S(n, h, invd);                                        \
            orc_axpy_##S(n, x, h, (T)1.);                                      \
          } else {                                                             \
            orc_axpy_##S(n, x, p, alpha);                                      \
          }                                                                    \
          memcpy(r, s, sizeof(T) * (size_t)n);                                 \
          ressq = orc_dot_##S(n, r, r);                                        \
          res = (double)SQRT(ressq);                                           \
          conv = orc_iterate_check(iter, res, maxits, atol, rtol, dtol, &first); \
          if (conv != CTRL_ITERATE) break;                                     \
        }                                                                      \
      }                                                                        \
    }                                                                          \
    *iters = iter;                                                             \
    *restarts = nrestart;                                                      \
    *res_out = res;                                                            \
    free(w);                                                                   \
    return conv;                                                               \
  }

ORACLE_KRYLOV(double, d, sqrt, fabs)
ORACLE_KRYLOV(float, f, sqrtf, fabsf)

/*
 * GMRES<LAD, PreLAD>::SolveNoPrecond / SolveRight (linear_solver/gmres.h:
 * 229-389, 462-713) on one rank: restarted GMRES with modified Gram-Schmidt,
 * Givens rotations (ApplyPlaneRotation / GeneratePlaneRotation, :97-115) and
 * UpdateSolution (:727-746: back substitution, then x += V y; with right
 * preconditioning z = V y, x += inv_D .* z).  The basis size is min(m,
 * maxits).  After a restart V[0] = b - A x is scaled by 1 / res with res the
 * recurrence residual |g[j+1]| (not the norm of the new V[0]), as the
 * reference does.  Returns the IterateControl state, -3 if out of memory.
 */
#define ORACLE_GMRES(T, S, SQRT, FABS)                                            \
  static void orc_gm_update_##S(int n, T **V, const T *H, int ld, const T *g,  \
                                int k, T *y, T *x) {                           \
    for (int i = 0; i <= k; ++i) y[i] = g[i];                                  \
    for (int i = k + 1; (i--) != 0;) {                                         \
      y[i] /= H[i * ld + i];                                                   \
      const T temp = y[i];                                                     \
      for (int j = 0; j < i; ++j) y[j] -= H[i * ld + j] * temp;                \
    }                                                                          \
    for (int j = 0; j <= k; ++j) orc_axpy_##S(n, x, V[j], y[j]);               \
  }                                                                            \
  static void orc_gm_rot_##S(T cs, T sn, T *dx, T *dy) {                       \
    const T temp = cs * (*dx) + sn * (*dy);                                    \
    *dy = -sn * (*dx) + cs * (*dy);                                            \
    *dx = temp;                                                                \
  }                                                                            \
  int orc_gmres_##S(int n, const int *rowptr, const int *col, const T *val,    \
                    const T *b, T *x, int precond, const T *invd,              \
                    int size_basis, int maxits, double atol, double rtol,      \
                    double dtol, int *iters, double *res_out,                  \
                    double *res_init_out) {                                    \
    const int m = size_basis < maxits ? size_basis : maxits;                   \
    const int ld = m + 1;                                                      \
    const size_t nn = (size_t)(n > 0 ? n : 1);                                 \
    T *store = (T *)calloc(nn * (size_t)(m + 3), sizeof(T));                   \
    T **V = (T **)calloc((size_t)(m + 1), sizeof(T *));                        \
    T *H = (T *)calloc((size_t)(m > 0 ? m : 1) * (size_t)ld, sizeof(T));       \
    T *gv = (T *)calloc((size_t)(4 * ld), sizeof(T));                          \
    if (!store || !V || !H || !gv) {                                           \
      free(store); free(V); free(H); free(gv);                                 \
      return -3;                                                               \
    }                                                                          \
    for (int i = 0; i <= m; ++i) V[i] = store + (size_t)i * nn;                \
    T *w = store + (size_t)(m + 1) * nn, *z = store + (size_t)(m + 2) * nn;    \
    T *g = gv, *cs = gv + ld, *sn = gv + 2 * ld, *y = gv + 3 * ld;             \
    int iter = 0, conv;                                                        \
    double first = 0.;                                                         \
    T res;                                                                     \
    orc_spmv_##S(n, rowptr, col, val, x, V[0]);                                \
    orc_scaleadd_##S(n, V[0], (T)-1., b);                                      \
    res = SQRT(orc_dot_##S(n, V[0], V[0]));                                    \
    *res_init_out = (double)res;                                               \
    conv = orc_iterate_check(iter, (double)res, maxits, atol, rtol, dtol,      \
                             &first);                                          \
    while (conv == CTRL_ITERATE) {                                             \
      for (int i = 0; i < ld; ++i) g[i] = 0;                                   \
      memset(H, 0, sizeof(T) * (size_t)m * (size_t)ld);                        \
      {                                                                        \
        const T sc = (T)1. / res;                                              \
        for (int q = 0; q < n; ++q) V[0][q] *= sc;                             \
      }                                                                        \
      g[0] = res;                                                              \
      int j = 0;                                                               \
      for (; j != m; ++j) {                                                    \
        ++iter;                                                                \
        if (precond) {                                                         \
          memcpy(z, V[j], sizeof(T) * (size_t)n);                              \
          orc_ewmult_##S(n, z, invd);                                          \
          orc_spmv_##S(n, rowptr, col, val, z, w);                             \
        } else {                                                               \
          orc_spmv_##S(n, rowptr, col, val, V[j], w);                          \
        }                                                                      \
        for (int i = 0; i <= j; ++i) {                                         \
          H[j * ld + i] = orc_dot_##S(n, w, V[i]);                             \
          orc_axpy_##S(n, w, V[i], (T)-1. * H[j * ld + i]);                    \
        }                                                                      \
        H[j * ld + j + 1] = SQRT(orc_dot_##S(n, w, w));                        \
        {                                                                      \
          const T sc = (T)1. / H[j * ld + j + 1];                              \
          for (int q = 0; q < n; ++q) w[q] *= sc;                              \
        }                                                                      \
        memcpy(V[j + 1], w, sizeof(T) * (size_t)n);                            \
        for (int k = 0; k != j; ++k)                                           \
          orc_gm_rot_##S(cs[k], sn[k], &H[j * ld + k], &H[j * ld + k + 1]);    \
        {                                                                      \
          const T dx = H[j * ld + j], dy = H[j * ld + j + 1];                  \
          const T beta = SQRT(dx * dx + dy * dy);                              \
          cs[j] = dx / beta;                                                   \
          sn[j] = dy / beta;                                                   \
        }                                                                      \
        orc_gm_rot_##S(cs[j], sn[j], &H[j * ld + j], &H[j * ld + j + 1]);      \
        orc_gm_rot_##S(cs[j], sn[j], &g[j], &g[j + 1]);                        \
        res = FABS(g[j + 1]);                                                  \
        conv = orc_iterate_check(iter, (double)res, maxits, atol, rtol, dtol,  \
                                 &first);                                      \
        if (conv != CTRL_ITERATE) break;                                       \
      }                                                                        \
      const int k = conv != CTRL_ITERATE ? j : m - 1;                          \
      if (precond) {                                                           \
        memset(z, 0, sizeof(T) * (size_t)n);                                   \
        orc_gm_update_##S(n, V, H, ld, g, k, y, z);                            \
        memcpy(w, z, sizeof(T) * (size_t)n);                                   \
        orc_ewmult_##S(n, w, invd);                                            \
        orc_axpy_##S(n, x, w, (T)1.);                                          \
      } else {                                                                 \
        orc_gm_update_##S(n, V, H, ld, g, k, y, x);                            \
      }                                                                        \
      if (conv == CTRL_ITERATE) {                                              \
        orc_spmv_##S(n, rowptr, col, val, x, V[0]);                            \
        orc_scaleadd_##S(n, V[0], (T)-1., b);                                  \
      }                                                                        \
    }                                                                          \
    *iters = iter;                                                             \
    *res_out = (double)res;                                                    \
    free(store); free(V); free(H); free(gv);                                   \
    return conv;                                                               \
  }

ORACLE_GMRES(double, d, sqrt, fabs)
ORACLE_GMRES(float, f, sqrtf, fabsf)

/*
 * Mixed-precision iterative refinement around a float inner CG, structured
 * like MPIR<LAD_high, LAD_low>::SolveImpl (linear_solver/mpir.cc:52-230)
 * without smoothers: double residual r = b - A x; loop { cast r to float;
 * float Jacobi-PCG on the float matrix from a zero start to inner_rtol; cast
 * the correction to double; x += c; recompute the double residual }.  The
 * outer stopping test is relative to the INITIAL residual.  (The reference
 * overwrites res0_ with the latest residual after every pass, mpir.cc:239,
 * so its relative test compares against the previous pass instead; the
 * north-star tolerance is stated relative to the initial residual.)  An
 * inner solve also stops once its residual is at or below floor_frac * rtol
 * * (initial residual), as the batch's last pass does (floor_frac 0.5; 0 for
 * none).  work must hold 3n doubles + 6n floats.  Returns 0 on success, 1 if
 * max_outer passes did not reach the tolerance.
 */
int orc_mpir_d(int n, const int *rowptr, const int *col, const double *val,
               const float *val32, const double *b, double *x, int max_outer,
               double rtol, double inner_rtol, double floor_frac, int inner_maxits,
               const double *invd, const float *invd32, double *work64,
               float *work32, int *outer_iters, int *inner_iters_total,
               double *res_out, double *res_init_out) {
  double *r = work64, *c = work64 + n;
  float *r32 = work32, *c32 = work32 + n, *w32 = work32 + 2 * (size_t)n;
  (void)invd;
  orc_spmv_d(n, rowptr, col, val, x, r);
  orc_scaleadd_d(n, r, -1., b);
  double res = sqrt(orc_dot_d(n, r, r));
  const double res0 = res;
  *res_init_out = res0;
  int k = 0, inner_total = 0;
  while (res > rtol * res0 && k < max_outer) {
    ++k;
    for (int i = 0; i < n; ++i) { r32[i] = (float)r[i]; c32[i] = 0.f; }
    int it = 0;
    double ires, ires0;
    orc_cg_f(n, rowptr, col, val32, r32, c32, inner_maxits, floor_frac * rtol * res0,
             inner_rtol, 1e30, 1, invd32, w32, &it, &ires, &ires0);
    inner_total += it;
    for (int i = 0; i < n; ++i) c[i] = (double)c32[i];
    orc_axpy_d(n, x, c, 1.);
    orc_spmv_d(n, rowptr, col, val, x, r);
    orc_scaleadd_d(n, r, -1., b);
    res = sqrt(orc_dot_d(n, r, r));
  }
  *outer_iters = k;
  *inner_iters_total = inner_total;
  *res_out = res;
  return res <= rtol * res0 ? 0 : 1;
}

/*
 * Mixed-precision CG with residual replacement -- the B200 library's default
 * fused refinement (b200la_mp with restart_inner = 0, and the batch's mixed
 * mode), not a reference algorithm: the reference's MPIR restarts its inner
 * solver every pass (orc_mpir_d above).  A float Jacobi-PCG runs on the float
 * copy of the matrix; once its recurrence residual has fallen below
 * inner_rtol times its value at the last replacement (IterateControl with
 * rtol = inner_rtol, strict), its correction goes into x in double, the
 * recurrence residual is replaced by the float copy of b - A x computed in
 * double, and the search direction carries on: p = z + beta p with
 * beta = (r.z of the new residual) / (r.z before the last step).  The first
 * pass, a pass after one that took no step, and a pass whose new residual is
 * more than twice the recurrence's last one start from p = z.  The
 * outer test (strict, relative to the first residual) is as orc_mpir_d's.
 * An inner pass never aims below floor_frac * rtol * (first residual): the
 * batch stops its last pass at half the outer target (floor_frac = 0.5), the
 * single-system solver does not (0).  work64 holds n doubles, work32 6n
 * floats.
 */
int orc_mpcg_kept_d(int n, const int *rowptr, const int *col, const double *val,
                    const float *val32, const double *b, double *x, int max_outer,
                    double rtol, double inner_rtol, double floor_frac, int inner_maxits,
                    const float *invd32, double *work64, float *work32,
                    int *outer_iters, int *inner_iters_total, double *res_out,
                    double *res_init_out) {
  double *r = work64;
  float *r32 = work32, *c32 = work32 + n, *p32 = work32 + 2 * (size_t)n;
  float *ap32 = work32 + 3 * (size_t)n, *z32 = work32 + 4 * (size_t)n;
  orc_spmv_d(n, rowptr, col, val, x, r);
  orc_scaleadd_d(n, r, -1., b);
  double res = sqrt(orc_dot_d(n, r, r));
  const double res0 = res;
  *res_init_out = res0;
  int k = 0, inner_total = 0, restart = 1;
  float rz_prev = 0.f;
  double rec_res = 0.; /* recurrence residual at the end of the last pass */
  while (!(res < rtol * res0) && k < max_outer) {
    ++k;
    for (int i = 0; i < n; ++i) {
      r32[i] = (float)r[i];
      c32[i] = 0.f;
      z32[i] = r32[i] * invd32[i];
    }
    float rz = orc_dot_f(n, r32, z32);
    const float beta0 = rz / rz_prev;
    const double rr_new = (double)orc_dot_f(n, r32, r32);
    /* a replaced residual more than twice the recurrence's last one means
     * the float recurrence drifted far from the true residual: the old
     * direction is then restarted (p = z) rather than kept */
    const int keep = !restart && isfinite(beta0) && !(sqrt(rr_new) > 2. * rec_res);
    for (int i = 0; i < n; ++i) p32[i] = keep ? beta0 * p32[i] + z32[i] : z32[i];
    const double ires0 = (double)sqrtf(orc_dot_f(n, r32, r32));
    int it = 0, broke = 0;
    while (!(ires0 <= 0.) && it < inner_maxits) {
      orc_spmv_f(n, rowptr, col, val32, p32, ap32);
      const float pap = orc_dot_f(n, p32, ap32);
      const float alpha = rz / pap;
      if (pap == 0.f || !isfinite(alpha)) { broke = 1; break; }
      orc_axpy_f(n, c32, p32, alpha);
      orc_axpy_f(n, r32, ap32, -alpha);
      ++it;
      for (int i = 0; i < n; ++i) z32[i] = r32[i] * invd32[i];
      const float rz_new = orc_dot_f(n, r32, z32);
      const double ires = (double)sqrtf(orc_dot_f(n, r32, r32));
      rz_prev = rz;
      rz = rz_new;
      rec_res = ires;
      if (ires < fmax(inner_rtol * ires0, floor_frac * rtol * res0)) break;
      const float beta = rz_new / rz_prev;
      orc_scaleadd_f(n, p32, beta, z32);
    }
    inner_total += it;
    restart = it == 0 || broke;
    for (int i = 0; i < n; ++i) x[i] += (double)c32[i];
    orc_spmv_d(n, rowptr, col, val, x, r);
    orc_scaleadd_d(n, r, -1., b);
    res = sqrt(orc_dot_d(n, r, r));
  }
  *outer_iters = k;
  *inner_iters_total = inner_total;
  *res_out = res;
  return res < rtol * res0 ? 0 : 1;
}

/*
 * coo_2_csr (lmp/lmatrix_formats.h:320-452), as CPU_CSR_lMatrix::
 * TransformFromCOO (lmp/lmatrix_csr_cpu.cc:883-906) calls it: count the
 * entries of each row, turn the counts into row offsets, scatter the entries
 * in input order, then sort each row by column with a selection sort (first
 * minimum by strict <, swapped into place; duplicates are kept and are not
 * kept in input order).  work holds nrow ints.  Returns 0, or -1 if an index
 * is out of range.
 */
int orc_coo2csr_d(int nrow, int ncol, int nnz, const int *rows, const int *cols,
                  const double *vals, int *rowptr, int *col, double *val,
                  int *work) {
  for (int i = 0; i < nnz; ++i)
    if (rows[i] < 0 || rows[i] >= nrow || cols[i] < 0 || cols[i] >= ncol)
      return -1;
  memset(rowptr, 0, sizeof(int) * (size_t)(nrow + 1));
  for (int i = 0; i < nnz; ++i) ++rowptr[rows[i]];
  rowptr[nrow] = nnz;
  int acc = 0;
  for (int i = 0; i < nrow; ++i) {
    const int c = rowptr[i];
    rowptr[i] = acc;
    work[i] = acc;
    acc += c;
  }
  for (int i = 0; i < nnz; ++i) {
    const int t = work[rows[i]]++;
    col[t] = cols[i];
    val[t] = vals[i];
  }
  for (int k = 0; k < nrow; ++k) {
    for (int i = rowptr[k], ie = rowptr[k + 1]; i != ie; ++i) {
      int mi = i, mc = col[i];
      for (int j = i + 1; j < ie; ++j)
        if (col[j] < mc) {
          mi = j;
          mc = col[j];
        }
      const int tc = col[i];
      col[i] = col[mi];
      col[mi] = tc;
      const double tv = val[i];
      val[i] = val[mi];
      val[mi] = tv;
    }
  }
  return 0;
}
