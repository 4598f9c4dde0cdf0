// The stationary Jacobi solver/smoother and BiCGSTAB on the device, on the
// same SpMV schedules and reductions as the CG path:
//   Jacobi<LAD>   linear_solver/jacobi.cc:101-356 (SolveNormal/SolveDamped,
//                 SmoothNormal/SmoothDamped, DoNormalIteration/DoDampedIteration)
//   BiCGSTAB<LAD> linear_solver/bicgstab.h:104-473 (SolveNoPrecond,
//                 SolvePrecondRight with PreconditionerBlockJacobiStand)
// with IterateControl::Check (common/iterate_control.cc:80-107).
//
// As for CG, the host never sits in the loop: the kernels of one pass are the
// body of a CUDA-graph WHILE node, every scalar lives in device memory, the
// last block of each reduction (ticket) makes the pass's decision, and the
// last kernel of the body sets the loop condition.  Every device loop is
// bounded: the sweep/pass counters stop the loop past maxits whatever the
// reductions report.
//
// Jacobi, one kernel per sweep k: r = b - A x_k (schedule emitter), ||r||^2,
// and x_{k+1} = x_k + w inv_D r into the other buffer of a pair.  That is the
// reference's sweep y = inv_D (b - A_nodiag x), x = (1 - w) x + w y written
// through the full row, so the residual norm that SolveNormal/SolveDamped
// test after every inner_iter sweeps comes out of the same pass: the test of
// x_k decides in the sweep that already produced x_{k+1}, and x_k is still
// intact in its buffer when the test ends the solve.  One SpMV-sized pass per
// sweep instead of the reference's two SpMVs and five vector passes.
//
// BiCGSTAB, five kernels per iteration:
//   B1  restart pass: r0 = b - A x, r = r0, q = P r0, ||r||, IterateControl;
//       step pass:    Ap = A q, sigma = Ap.r0, Ap.Ap; restart test; alpha
//   B2  s = r - alpha Ap (sh = inv_D s), s.s; the short-update test
//   B3  t = A s (or A sh), t.s, t.t; omega
//   B4  x += alpha q + omega s (sh), r = s - omega t, r.r, r.r0; IterateControl;
//       rho, beta
//   B5  q = beta q + P(r - omega beta Ap); the loop condition
// P is the Jacobi preconditioner (right preconditioning) or the identity; the
// direction is stored as q = P p, so A P p is one SpMV of q.
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "krylov.cuh"
#include "spmv.cuh"

namespace b200la {

// Device-resident scalars of one solve.
struct ItScalars {
  double res, res_init, first;
  double atol, rtol, dtol;
  double w;                 // Jacobi damping
  double rho, rho_old, alpha, omega, beta, r0norm;
  int iter;                 // Jacobi: sweeps done (x_iter is current); BiCGSTAB: iterations
  int state;
  int phase;                // BiCGSTAB: kStart / kFresh / kStep
  int shortb;               // BiCGSTAB: this iteration takes the short update
  int restarts;             // BiCGSTAB: starts - 1
  int maxits, inner, total, mode;
  int guard;                // body passes
  unsigned ticket[4];
};

enum { kStart = 0, kFresh = 1, kStep = 2 };

__device__ __forceinline__ int it_check(int step, double value, const ItScalars &s) {
  if (value <= s.atol) return B200LA_SUCCESS_ABS;
  if (value < s.rtol * s.first) return B200LA_SUCCESS_REL;
  if (value > s.dtol * s.first) return B200LA_FAIL_DIV;
  if (step >= s.maxits) return B200LA_FAIL_MAXITS;
  return B200LA_ITERATE;
}

// ---- Jacobi sweep ------------------------------------------------------------
template <typename T> struct JacobiEmit {
  const T *__restrict__ b;
  const T *__restrict__ invd;
  const T *__restrict__ xc;
  T *__restrict__ xn;
  T w;
  Acc<T> rr;
  __device__ __forceinline__ void operator()(int row, T y) {
    const T r = b[row] - y;
    xn[row] = fma(w * invd[row], r, xc[row]);
    rr.add(r * r);
  }
};

// Sweep k = sc->iter: reads x_k from buf[k & 1], writes x_{k+1} to the other.
// Solve modes test ||b - A x_k|| when k is a multiple of inner_iter; the
// smoothing modes stop after `total` sweeps.
template <typename Op, typename T, bool IN_GRAPH>
__global__ void __launch_bounds__(kBlock) jacobi_sweep_kernel(Op op, T *buf0, T *buf1, const T *__restrict__ b,
                                                              const T *__restrict__ invd, double *part,
                                                              ItScalars *sc, cudaGraphConditionalHandle loop) {
  if (__ldg(&sc->state) != B200LA_ITERATE) return;
  const int k = __ldg(&sc->iter);
  const T *xc = (k & 1) ? buf1 : buf0;
  T *xn = (k & 1) ? buf0 : buf1;
  JacobiEmit<T> e{b, invd, xc, xn, (T)__ldg(&sc->w)};
  op.run(xc, e);
  double s[1] = {e.rr.value()};
  if (grid_sum_last<1>(s, part, &sc->ticket[0]) && threadIdx.x == 0) {
    bool go = true;
    if (sc->mode <= B200LA_JACOBI_SOLVE_DAMPED) {
      if (k % sc->inner == 0) {
        const double res = sqrt(s[0]);
        if (k == 0) {
          sc->res_init = res;
          sc->first = res;
        }
        sc->res = res;
        const int stt = it_check(k, res, *sc);
        if (stt != B200LA_ITERATE) {
          sc->state = stt;
          go = false;
        }
      }
      if (go) {
        sc->iter = k + 1;
        // the test at a multiple of inner_iter >= maxits always stops the
        // loop first; this bound only guards against a broken reduction
        if (k + 1 > sc->maxits + sc->inner) {
          sc->state = B200LA_FAIL_BREAKDOWN;
          go = false;
        }
      }
    } else {
      sc->iter = k + 1;
      go = k + 1 < sc->total;
      if (!go) sc->state = B200LA_DONE_FIXED;
    }
    if (IN_GRAPH) cudaGraphSetConditional(loop, go ? 1u : 0u);
  }
}

// ---- BiCGSTAB ------------------------------------------------------------------
template <typename T> struct BiVecs {
  T *x, *r, *r0, *q, *Ap, *s, *sh, *t;
  const T *b;
  const T *invd;  // nullptr without preconditioner
  int64_t n;
};

template <bool PRE> __device__ __forceinline__ double bicg_eps() { return PRE ? 5.e-16 : 1.e-15; }

// restart: r0 = b - A x, r = r0, q = P r0, r.r
template <typename T, bool PRE> struct RestartEmit {
  BiVecs<T> v;
  Acc<T> rr;
  __device__ __forceinline__ void operator()(int row, T y) {
    const T r = v.b[row] - y;  // r0.ScaleAdd(b, -1): -1*(Ax) + b
    v.r0[row] = r;
    v.r[row] = r;
    v.q[row] = PRE ? r * v.invd[row] : r;
    rr.add(r * r);
  }
};

// step: Ap = A q, Ap.r0, Ap.Ap
template <typename T> struct StepEmit {
  T *__restrict__ Ap;
  const T *__restrict__ r0;
  Acc<T> sig, aa;
  __device__ __forceinline__ void operator()(int row, T y) {
    Ap[row] = y;
    sig.add(y * r0[row]);
    aa.add(y * y);
  }
};

// B1.  Phase kStart (first pass, or after a restart test failed): the
// (re)start and its IterateControl test, then kFresh so that B2-B5 of this
// pass do nothing.  Otherwise (kFresh or kStep): the step's SpMV and the
// restart test of bicgstab.h:205/:382.  Blocks read the phase before any
// block writes it, and the only write in this kernel comes from the last
// block, so kFresh and kStep take the same branch here.
template <typename Op, typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) bicg_spmv_q_kernel(Op op, BiVecs<T> v, double *part, ItScalars *sc) {
  if (__ldg(&sc->state) != B200LA_ITERATE) return;
  if (__ldg(&sc->phase) == kStart) {
    RestartEmit<T, PRE> e{v};
    op.run(v.x, e);
    double s[1] = {e.rr.value()};
    if (grid_sum_last<1>(s, part, &sc->ticket[0]) && threadIdx.x == 0) {
      const double res = sqrt(s[0]);
      sc->restarts += 1;
      sc->rho = sc->rho_old = s[0];
      sc->r0norm = res;  // ||r0|| of the restart tolerance: r = r0 here
      sc->res = res;
      sc->res_init = res;
      if (sc->iter == 0) sc->first = res;  // IterateControl's first step
      sc->state = it_check(sc->iter, res, *sc);
      sc->phase = kFresh;
    }
    return;
  }
  StepEmit<T> e{v.Ap, v.r0};
  op.run(v.q, e);
  double s[2] = {e.sig.value(), e.aa.value()};
  if (grid_sum_last<2>(s, part, &sc->ticket[1]) && threadIdx.x == 0) {
    sc->iter += 1;
    const double tol1 = bicg_eps<PRE>() * sqrt(s[1]) * sc->r0norm;
    if (fabs(s[0]) > tol1) {
      sc->alpha = sc->rho / s[0];
      sc->phase = kStep;
    } else {
      sc->phase = kStart;  // not finite or too small: restart next pass
    }
  }
}

// B2.  s = r - alpha Ap (sh = inv_D s), s.s; the short update when ||s|| <= eps.
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) bicg_s_kernel(BiVecs<T> v, double *part, ItScalars *sc) {
  if (__ldg(&sc->state) != B200LA_ITERATE || __ldg(&sc->phase) != kStep) return;
  const T alpha = (T)__ldg(&sc->alpha);
  Acc<T> ss;
  for_each_chunk<T>(v.n, [&](int64_t i, auto cc) {
    constexpr int C = decltype(cc)::value;
    T r[C], a[C], d[C], s[C];
    ld<C>(v.r + i, r);
    ld<C>(v.Ap + i, a);
    if (PRE) ld<C>(v.invd + i, d);
#pragma unroll
    for (int k = 0; k < C; ++k) {
      s[k] = fma(-alpha, a[k], r[k]);
      ss.add(s[k] * s[k]);
      if (PRE) d[k] = s[k] * d[k];
    }
    st<C>(v.s + i, s);
    if (PRE) st<C>(v.sh + i, d);
  });
  double sm[1] = {ss.value()};
  if (grid_sum_last<1>(sm, part, &sc->ticket[2]) && threadIdx.x == 0)
    sc->shortb = sqrt(sm[0]) > bicg_eps<PRE>() ? 0 : 1;
}

// t = A s, t.s, t.t
template <typename T> struct TEmit {
  T *__restrict__ t;
  const T *__restrict__ s;
  Acc<T> ts, tt;
  __device__ __forceinline__ void operator()(int row, T y) {
    t[row] = y;
    ts.add(y * s[row]);
    tt.add(y * y);
  }
};

// B3.  t = A s (A sh with the preconditioner), omega = t.s / t.t.
template <typename Op, typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) bicg_spmv_s_kernel(Op op, BiVecs<T> v, double *part, ItScalars *sc) {
  if (__ldg(&sc->state) != B200LA_ITERATE || __ldg(&sc->phase) != kStep || __ldg(&sc->shortb)) return;
  TEmit<T> e{v.t, v.s};
  op.run(PRE ? v.sh : v.s, e);
  double s[2] = {e.ts.value(), e.tt.value()};
  if (grid_sum_last<2>(s, part, &sc->ticket[0]) && threadIdx.x == 0) sc->omega = s[0] / s[1];
}

// B4.  x += alpha q + omega s (sh), r = s - omega t, r.r, r.r0, the test;
// short update: x += alpha q, r = s.  Then rho = r.r0 and beta.
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) bicg_update_kernel(BiVecs<T> v, double *part, ItScalars *sc) {
  if (__ldg(&sc->state) != B200LA_ITERATE || __ldg(&sc->phase) != kStep) return;
  const bool shortb = __ldg(&sc->shortb) != 0;
  const T alpha = (T)__ldg(&sc->alpha);
  const T omega = shortb ? T(0) : (T)__ldg(&sc->omega);
  Acc<T> rr, rr0;
  for_each_chunk<T>(v.n, [&](int64_t i, auto cc) {
    constexpr int C = decltype(cc)::value;
    T x[C], q[C], s[C], u[C], t[C], z[C];
    ld<C>(v.x + i, x);
    ld<C>(v.q + i, q);
    ld<C>(v.s + i, s);
    if (shortb) {
#pragma unroll
      for (int k = 0; k < C; ++k) {
        x[k] = fma(alpha, q[k], x[k]);
        rr.add(s[k] * s[k]);
      }
      st<C>(v.r + i, s);
    } else {
      if (PRE) ld<C>(v.sh + i, u);
      ld<C>(v.t + i, t);
      ld<C>(v.r0 + i, z);
#pragma unroll
      for (int k = 0; k < C; ++k) {
        x[k] = fma(omega, PRE ? u[k] : s[k], fma(alpha, q[k], x[k]));
        const T r = fma(-omega, t[k], s[k]);
        s[k] = r;
        rr.add(r * r);
        rr0.add(r * z[k]);
      }
      st<C>(v.r + i, s);
    }
    st<C>(v.x + i, x);
  });
  double sm[2] = {rr.value(), rr0.value()};
  if (grid_sum_last<2>(sm, part, &sc->ticket[1]) && threadIdx.x == 0) {
    const double res = sqrt(sm[0]);
    sc->res = res;
    const int stt = it_check(sc->iter, res, *sc);
    sc->state = stt;
    if (stt == B200LA_ITERATE && !shortb) {
      const double rho = sm[1];
      sc->beta = (sc->alpha * rho) / (sc->omega * sc->rho_old);
      sc->rho = rho;
      sc->rho_old = rho;
    }
  }
}

// B5.  q = beta q + P (r - omega beta Ap) (p.ScaleAdd(r, beta);
// p.Axpy(Ap, -omega beta)), then the loop condition.  The body runs at most
// 2 maxits + 4 passes: each restart pass follows a pass that counted an
// iteration, and IterateControl stops at maxits.
template <typename T, bool PRE, bool IN_GRAPH>
__global__ void __launch_bounds__(kBlock) bicg_direction_kernel(BiVecs<T> v, ItScalars *sc,
                                                                cudaGraphConditionalHandle loop) {
  const int state = __ldg(&sc->state);
  if (IN_GRAPH && blockIdx.x == 0 && threadIdx.x == 0) {
    const int g = sc->guard + 1;
    sc->guard = g;
    bool go = state == B200LA_ITERATE;
    if (go && g > 2 * sc->maxits + 4) {
      sc->state = B200LA_FAIL_BREAKDOWN;
      go = false;
    }
    cudaGraphSetConditional(loop, go ? 1u : 0u);
  }
  if (state != B200LA_ITERATE || __ldg(&sc->phase) != kStep || __ldg(&sc->shortb)) return;
  const T beta = (T)__ldg(&sc->beta);
  const T ob = (T)(__ldg(&sc->omega) * __ldg(&sc->beta));
  for_each_chunk<T>(v.n, [&](int64_t i, auto cc) {
    constexpr int C = decltype(cc)::value;
    T q[C], r[C], a[C], d[C];
    ld<C>(v.q + i, q);
    ld<C>(v.r + i, r);
    ld<C>(v.Ap + i, a);
    if (PRE) ld<C>(v.invd + i, d);
#pragma unroll
    for (int k = 0; k < C; ++k) {
      const T u = fma(-ob, a[k], r[k]);
      q[k] = fma(beta, q[k], PRE ? u * d[k] : u);
    }
    st<C>(v.q + i, q);
  });
}

}  // namespace b200la

using namespace b200la;

struct b200la_solver_s {
  b200la_mat A;
  b200la_ctx ctx;            // kept for destroy, which may come after A's
  b200la_solver_params prm;
  int64_t n;
  // Jacobi: v[0], v[1] = the iterate pair.  BiCGSTAB: x r r0 q Ap s sh t.
  void *v[8];
  void *invd;
  void *bown;                // the right-hand side, copied in per solve
  double *part;              // [2][kMaxReduceBlocks]
  ItScalars *sc;             // device
  ItScalars *sc_host;        // pinned
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int g_format, g_param;     // schedule baked into the graph
  int g_gen;                 // the matrix's schedule generation at capture
  int grid_spmv, grid_ew;
  b200la::GmresState *gm;    // GMRES keeps its own state (gmres.cu)
};

namespace b200la {

template <typename T> static BiVecs<T> bi_vecs(b200la_solver s) {
  return BiVecs<T>{(T *)s->v[0], (T *)s->v[1], (T *)s->v[2], (T *)s->v[3], (T *)s->v[4],
                   (T *)s->v[5], (T *)s->v[6], (T *)s->v[7], (const T *)s->bown, (const T *)s->invd, s->n};
}

// One pass of the loop body on stream `st`: captured into the graph, or
// launched from the host loop.  The body reads the solver's own buffers only
// (x, b are copied in per solve), so one graph serves every solve.
template <typename T, bool PRE, bool IN_GRAPH>
static int solver_body_t(b200la_solver s, cudaStream_t st, cudaGraphConditionalHandle h) {
  b200la_mat A = s->A;
  b200la_ctx c = A->ctx;
  if (s->prm.method == B200LA_METHOD_JACOBI) {
    return with_schedule<T>(A, [&](auto op) -> int {
      using Op = decltype(op);
      B_TRY(grid_for(c, (const void *)jacobi_sweep_kernel<Op, T, IN_GRAPH>, op.work_items(), Op::kRowsPerBlock,
                     &s->grid_spmv));
      jacobi_sweep_kernel<Op, T, IN_GRAPH><<<s->grid_spmv, kBlock, 0, st>>>(
          op, (T *)s->v[0], (T *)s->v[1], (const T *)s->bown, (const T *)s->invd, s->part, s->sc, h);
      return B200LA_OK;
    });
  }
  const BiVecs<T> v = bi_vecs<T>(s);
  B_TRY(with_schedule<T>(A, [&](auto op) -> int {
    using Op = decltype(op);
    B_TRY(grid_for(c, (const void *)bicg_spmv_q_kernel<Op, T, PRE>, op.work_items(), Op::kRowsPerBlock,
                   &s->grid_spmv));
    bicg_spmv_q_kernel<Op, T, PRE><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part, s->sc);
    bicg_s_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->part, s->sc);
    bicg_spmv_s_kernel<Op, T, PRE><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part, s->sc);
    return B200LA_OK;
  }));
  bicg_update_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->part, s->sc);
  bicg_direction_kernel<T, PRE, IN_GRAPH><<<s->grid_ew, kBlock, 0, st>>>(v, s->sc, h);
  return B200LA_OK;
}

template <typename T, bool PRE>
static int solver_build_graph_t(b200la_solver s) {
  b200la_mat A = s->A;
  B_TRY(grid_for(A->ctx, (const void *)bicg_update_kernel<T, PRE>, (s->n + Vec16<T>::n - 1) / Vec16<T>::n, kBlock,
                 &s->grid_ew));
  if (s->exec) { cudaGraphExecDestroy(s->exec); s->exec = nullptr; }
  if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
  cudaGraph_t g;
  B_CUDA(cudaGraphCreate(&g, 0));
  s->graph = g;
  cudaGraphConditionalHandle h;
  B_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  B_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &np));
  cudaGraph_t body = np.conditional.phGraph_out[0];
  cudaStream_t cs;
  B_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  B_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int rc = solver_body_t<T, PRE, true>(s, cs, h);
  cudaGraph_t captured;
  cudaError_t ce = cudaStreamEndCapture(cs, &captured);
  cudaStreamDestroy(cs);
  B_TRY(rc);
  B_CUDA(ce);
  B_CUDA(cudaGraphInstantiate(&s->exec, g, 0));
  s->g_format = A->format;
  s->g_param = A->param;
  s->g_gen = A->sched_gen;
  return B200LA_OK;
}

static bool solver_pre(b200la_solver s) {
  return s->prm.method == B200LA_METHOD_JACOBI || s->prm.precond != 0;
}

static int solver_build_graph(b200la_solver s) {
  const bool pre = solver_pre(s);
  if (s->A->dtype == B200LA_F64)
    return pre ? solver_build_graph_t<double, true>(s) : solver_build_graph_t<double, false>(s);
  return pre ? solver_build_graph_t<float, true>(s) : solver_build_graph_t<float, false>(s);
}

static int solver_fetch(b200la_solver s, ItScalars *out) {
  cudaStream_t st = s->A->ctx->stream;
  B_CUDA(cudaMemcpyAsync(s->sc_host, s->sc, sizeof(ItScalars), cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  *out = *s->sc_host;
  return B200LA_OK;
}

// Host loop with the same kernels (B200LA_GRAPHS=0): the kernels return at
// once after the state leaves "iterate", so polling every 16 passes runs the
// same iterations.
template <typename T, bool PRE>
static int solver_host_loop_t(b200la_solver s) {
  cudaStream_t st = s->A->ctx->stream;
  const int64_t bound = 2 * (int64_t)s->prm.maxits + (int64_t)s->prm.inner_iter * s->prm.smooth_iter + 64;
  for (int64_t pass = 0;; pass += 16) {
    for (int k = 0; k < 16; ++k) B_TRY((solver_body_t<T, PRE, false>(s, st, 0)));
    B_CUDA(cudaGetLastError());
    ItScalars h;
    B_TRY(solver_fetch(s, &h));
    if (h.state != B200LA_ITERATE || pass > bound) break;
  }
  return B200LA_OK;
}

static int solver_host_loop(b200la_solver s) {
  const bool pre = solver_pre(s);
  if (s->A->dtype == B200LA_F64)
    return pre ? solver_host_loop_t<double, true>(s) : solver_host_loop_t<double, false>(s);
  return pre ? solver_host_loop_t<float, true>(s) : solver_host_loop_t<float, false>(s);
}

// Scalars at the start of a solve.
static ItScalars solver_initial(const b200la_solver_s *s) {
  ItScalars init = {};
  const b200la_solver_params &p = s->prm;
  init.atol = p.atol;
  init.rtol = p.rtol;
  init.dtol = p.dtol;
  init.maxits = p.maxits;
  init.inner = p.inner_iter;
  init.mode = p.mode;
  init.w = p.method == B200LA_METHOD_JACOBI && (p.mode == B200LA_JACOBI_SOLVE_DAMPED ||
                                                p.mode == B200LA_JACOBI_SMOOTH_DAMPED)
               ? p.w
               : 1.0;
  init.total = p.mode == B200LA_JACOBI_SMOOTH_NORMAL ? p.smooth_iter * p.inner_iter
                                                     : p.maxits * p.inner_iter;
  init.state = B200LA_ITERATE;
  init.phase = kStart;
  init.restarts = -1;
  return init;
}

}  // namespace b200la

namespace b200la {

// Runs `passes` passes of the body as separate launches with CUDA events
// between the kernels, from the start value x_dev and right-hand side b_dev
// (copied into the solver's buffers); adds the mean ms per launch.
template <typename T, bool PRE>
static int solver_profile_t(b200la_solver s, const void *b_dev, const void *x_dev, int passes, double *ms) {
  b200la_mat A = s->A;
  cudaStream_t st = A->ctx->stream;
  const size_t vb = (size_t)s->n * sizeof(T);
  const ItScalars init = solver_initial(s);
  B_CUDA(cudaMemcpyAsync(s->sc, &init, sizeof(init), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaMemcpyAsync(s->bown, b_dev, vb, cudaMemcpyDeviceToDevice, st));
  B_CUDA(cudaMemcpyAsync(s->v[0], x_dev, vb, cudaMemcpyDeviceToDevice, st));
  const bool jac = s->prm.method == B200LA_METHOD_JACOBI;
  const int nk = jac ? 1 : 5;
  const BiVecs<T> v = bi_vecs<T>(s);
  // every pass is queued before the first wait, after one untimed pass, so
  // the timed kernels run back to back and no host launch gap falls between
  // an event pair
  const int ne = nk + 1;
  std::vector<cudaEvent_t> ev((size_t)(passes > 0 ? passes : 0) * ne);
  for (auto &e : ev) B_CUDA(cudaEventCreate(&e));
  float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  int rc = B200LA_OK;
  auto pass = [&](cudaEvent_t *e) -> int {
    if (e) cudaEventRecord(e[0], st);
    B_TRY(with_schedule<T>(A, [&](auto op) -> int {
      using Op = decltype(op);
      if (jac) {
        jacobi_sweep_kernel<Op, T, false><<<s->grid_spmv, kBlock, 0, st>>>(
            op, (T *)s->v[0], (T *)s->v[1], (const T *)s->bown, (const T *)s->invd, s->part, s->sc, 0);
        if (e) cudaEventRecord(e[1], st);
        return B200LA_OK;
      }
      bicg_spmv_q_kernel<Op, T, PRE><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part, s->sc);
      if (e) cudaEventRecord(e[1], st);
      bicg_s_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->part, s->sc);
      if (e) cudaEventRecord(e[2], st);
      bicg_spmv_s_kernel<Op, T, PRE><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part, s->sc);
      if (e) cudaEventRecord(e[3], st);
      return B200LA_OK;
    }));
    if (!jac) {
      bicg_update_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->part, s->sc);
      if (e) cudaEventRecord(e[4], st);
      bicg_direction_kernel<T, PRE, false><<<s->grid_ew, kBlock, 0, st>>>(v, s->sc, 0);
      if (e) cudaEventRecord(e[5], st);
    }
    return B200LA_OK;
  };
  if (passes > 0) rc = pass(nullptr);
  for (int it = 0; it < passes && rc == B200LA_OK; ++it) rc = pass(&ev[(size_t)it * ne]);
  const cudaError_t se = cudaStreamSynchronize(st);
  for (int it = 0; it < passes && rc == B200LA_OK && se == cudaSuccess; ++it)
    for (int k = 0; k < nk; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[(size_t)it * ne + k], ev[(size_t)it * ne + k + 1]);
      acc[k] += t;
    }
  for (auto &e : ev) cudaEventDestroy(e);
  B_CUDA(se);
  B_CUDA(cudaGetLastError());
  for (int k = 0; k < nk; ++k) ms[k] = passes > 0 ? acc[k] / passes : 0.0;
  return rc;
}

}  // namespace b200la

extern "C" {

int b200la_solver_destroy(b200la_solver s) {
  if (!s) return B200LA_OK;
  if (s->gm) {
    gmres_destroy(s->gm);
    delete s;
    return B200LA_OK;
  }
  cudaStream_t st = s->ctx->stream;
  cudaStreamSynchronize(st);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  for (void *b : s->v)
    if (b) cudaFreeAsync(b, st);
  void *bufs[] = {s->invd, s->bown, s->part, s->sc};
  for (void *b : bufs)
    if (b) cudaFreeAsync(b, st);
  if (s->sc_host) cudaFreeHost(s->sc_host);
  delete s;
  return B200LA_OK;
}

int b200la_solver_create(b200la_mat A, const b200la_solver_params *prm, b200la_solver *out) {
  B_CHECK(A && prm && out, B200LA_ERR_INVALID, "solver_create: null argument");
  B_CHECK(A->nrow == A->ncol, B200LA_ERR_INVALID, "solver_create: matrix is %dx%d, not square", A->nrow, A->ncol);
  B_CHECK(prm->method == B200LA_METHOD_JACOBI || prm->method == B200LA_METHOD_BICGSTAB ||
              prm->method == B200LA_METHOD_GMRES,
          B200LA_ERR_INVALID, "solver_create: unknown method %d", prm->method);
  B_CHECK(prm->maxits >= 0 && prm->maxits <= 10000000, B200LA_ERR_INVALID, "solver_create: maxits %d not in [0, 1e7]",
          prm->maxits);
  B_CHECK(prm->atol >= 0.0 && prm->rtol >= 0.0 && prm->dtol > 0.0, B200LA_ERR_INVALID,
          "solver_create: tolerances must be atol >= 0, rtol >= 0, dtol > 0");
  b200la_solver_params p = *prm;
  if (p.method == B200LA_METHOD_GMRES) {
    p.mode = 0;
    p.inner_iter = 1;
    p.smooth_iter = 1;
    p.w = 1.0;
    b200la_solver s = new b200la_solver_s();
    s->A = A;
    s->ctx = A->ctx;
    s->prm = p;
    s->n = A->nrow;
    const int rc = gmres_create(A, &p, &s->gm);
    if (rc != B200LA_OK) {
      delete s;
      return rc;
    }
    *out = s;
    return B200LA_OK;
  }
  if (p.method == B200LA_METHOD_JACOBI) {
    B_CHECK(p.mode >= 0 && p.mode <= 3, B200LA_ERR_INVALID, "solver_create: Jacobi mode %d not in 0..3", p.mode);
    B_CHECK(p.inner_iter >= 1 && p.smooth_iter >= 1, B200LA_ERR_INVALID,
            "solver_create: Jacobi inner_iter %d and smooth_iter %d must be >= 1", p.inner_iter, p.smooth_iter);
    B_CHECK(p.w > 0.0, B200LA_ERR_INVALID, "solver_create: Jacobi damping %g must be > 0", p.w);
    const int64_t sweeps = (int64_t)(p.mode == B200LA_JACOBI_SMOOTH_NORMAL ? p.smooth_iter : p.maxits) * p.inner_iter;
    B_CHECK(sweeps <= 20000000, B200LA_ERR_INVALID, "solver_create: %lld sweeps exceed 2e7", (long long)sweeps);
  } else {
    p.mode = 0;
    p.inner_iter = 1;
    p.smooth_iter = 1;
    p.w = 1.0;
  }
  b200la_ctx c = A->ctx;
  cudaStream_t st = c->stream;
  b200la_solver s = new b200la_solver_s();
  s->A = A;
  s->ctx = A->ctx;
  s->prm = p;
  s->n = A->nrow;
  const size_t vb = dtype_size(A->dtype) * (size_t)(s->n > 0 ? s->n : 1);
  auto cleanup = [&](int code) { b200la_solver_destroy(s); return code; };
  const bool jac = p.method == B200LA_METHOD_JACOBI;
  const bool pre = jac || p.precond != 0;
  const int nvec = jac ? 2 : 8;
  for (int k = 0; k < nvec; ++k) {
    if (!jac && k == 6 && !pre) continue;  // sh: preconditioned only
    if (cudaMallocAsync(&s->v[k], vb, st) != cudaSuccess)
      return cleanup(fail(B200LA_ERR_NOMEM, "solver_create: allocation of %zu-byte work vectors failed", vb));
  }
  if (cudaMallocAsync(&s->bown, vb, st) != cudaSuccess ||
      cudaMallocAsync(&s->part, sizeof(double) * 2 * kMaxReduceBlocks, st) != cudaSuccess ||
      cudaMallocAsync(&s->sc, sizeof(ItScalars), st) != cudaSuccess ||
      cudaMallocHost(&s->sc_host, sizeof(ItScalars)) != cudaSuccess)
    return cleanup(fail(B200LA_ERR_NOMEM, "solver_create: allocation failed"));
  if (pre) {
    if (cudaMallocAsync(&s->invd, vb, st) != cudaSuccess)
      return cleanup(fail(B200LA_ERR_NOMEM, "solver_create: allocation of the inverse diagonal failed"));
    b200la_vec_s dv{c, s->n, A->dtype, s->invd, false};
    const int rc = b200la_mat_inv_diag(A, &dv);
    if (rc != B200LA_OK) return cleanup(rc);
  }
  if (s->n > 0) {
    const int rc = solver_build_graph(s);
    if (rc != B200LA_OK) return cleanup(rc);
  }
  *out = s;
  return B200LA_OK;
}

int b200la_solver_solve(b200la_solver s, b200la_vec b, b200la_vec x, b200la_solver_result *res) {
  B_CHECK(s && b && x && res, B200LA_ERR_INVALID, "solver_solve: null argument");
  b200la_mat A = s->A;
  B_CHECK(b->n == s->n && x->n == s->n, B200LA_ERR_INVALID, "solver_solve: vector sizes %lld/%lld vs %lld",
          (long long)b->n, (long long)x->n, (long long)s->n);
  B_CHECK(b->dtype == A->dtype && x->dtype == A->dtype, B200LA_ERR_DTYPE, "solver_solve: dtype mismatch");
  if (s->gm) return gmres_solve(s->gm, b, x, res);
  memset(res, 0, sizeof(*res));
  const bool jac = s->prm.method == B200LA_METHOD_JACOBI;
  const bool smooth = jac && s->prm.mode >= B200LA_JACOBI_SMOOTH_NORMAL;
  const ItScalars init = solver_initial(s);
  if (s->n == 0 || (smooth && init.total == 0)) {
    res->state = smooth ? B200LA_DONE_FIXED : B200LA_SUCCESS_ABS;
    return B200LA_OK;
  }
  cudaStream_t st = A->ctx->stream;
  const size_t vb = (size_t)s->n * dtype_size(A->dtype);
  B_CUDA(cudaMemcpyAsync(s->sc, &init, sizeof(init), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaMemcpyAsync(s->bown, b->d, vb, cudaMemcpyDeviceToDevice, st));
  B_CUDA(cudaMemcpyAsync(s->v[0], x->d, vb, cudaMemcpyDeviceToDevice, st));
  if (A->ctx->use_graphs) {
    if (A->format != s->g_format || A->param != s->g_param || A->sched_gen != s->g_gen) B_TRY(solver_build_graph(s));
    B_CUDA(cudaGraphLaunch(s->exec, st));
  } else {
    B_TRY(solver_host_loop(s));
  }
  ItScalars h;
  B_TRY(solver_fetch(s, &h));
  // Jacobi: x_iter sits in buffer iter & 1; BiCGSTAB: x is v[0]
  const void *xs = jac ? s->v[h.iter & 1] : s->v[0];
  B_CUDA(cudaMemcpyAsync(x->d, xs, vb, cudaMemcpyDeviceToDevice, st));
  B_CUDA(cudaStreamSynchronize(st));
  res->iters = h.iter;
  res->state = h.state;
  res->restarts = jac ? 0 : (h.restarts > 0 ? h.restarts : 0);
  res->res = h.res;
  res->res_init = h.res_init;
  res->res_rel = h.res_init > 0.0 ? h.res / h.res_init : 0.0;
  if (h.state == B200LA_SUCCESS_ABS || h.state == B200LA_SUCCESS_REL || h.state == B200LA_DONE_FIXED)
    res->solver_state = B200LA_SOLVER_SUCCESS;
  else if (h.state == B200LA_FAIL_DIV || h.state == B200LA_FAIL_MAXITS)
    res->solver_state = B200LA_SOLVER_EXCEEDED;
  else
    res->solver_state = B200LA_SOLVER_ERROR;
  return B200LA_OK;
}

int b200la_solver_profile(b200la_solver s, b200la_vec b, b200la_vec x, int passes, double *ms) {
  B_CHECK(s && b && x && ms && passes >= 0, B200LA_ERR_INVALID, "solver_profile: bad argument");
  B_CHECK(b->n == s->n && x->n == s->n && s->n > 0, B200LA_ERR_INVALID, "solver_profile: sizes");
  B_CHECK(b->dtype == s->A->dtype && x->dtype == s->A->dtype, B200LA_ERR_DTYPE, "solver_profile: dtype");
  if (s->gm) return gmres_profile(s->gm, b, x, passes, ms);
  const bool pre = solver_pre(s);
  if (s->A->dtype == B200LA_F64)
    return pre ? solver_profile_t<double, true>(s, b->d, x->d, passes, ms)
               : solver_profile_t<double, false>(s, b->d, x->d, passes, ms);
  return pre ? solver_profile_t<float, true>(s, b->d, x->d, passes, ms)
             : solver_profile_t<float, false>(s, b->d, x->d, passes, ms);
}

}  // extern "C"
