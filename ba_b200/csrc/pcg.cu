// Preconditioned CG on the device: CG<LAD>::SolvePrecond / SolveNoPrecond
// (linear_solver/cg.h:87-246) with PreconditionerBlockJacobiStand(Jacobi)
// (preconditioner_bjacobi_standard.cc:188-196, lmp/lpreconditioner.cc:184-200)
// and IterateControl::Check (common/iterate_control.cc:80-107).
//
// The reference runs the loop on the host: per iteration 1 SpMV, 3 blocking
// dot products and 6 more BLAS-1 passes, each its own launch.  Here one
// iteration is three kernels and no host round trip:
//   K1  Ap = A p, fused with the partial sums of p.Ap     (SpMV schedule)
//   K2  alpha = rz/pAp; x += alpha p; r -= alpha Ap; z = invD r;
//       fused sums r.r and r.z; its last block applies IterateControl
//   K3  beta = rz_new/rz_old; p = beta p + z  (z recomputed from r, invD)
// All scalars live in device memory.  The three kernels form the body of a
// CUDA-graph WHILE node, so one graph launch runs the whole solve; K3 clears
// the loop condition once the state leaves "iterate".  K3 also counts body
// passes and stops the loop after maxits + 2 passes whatever K2 reported, so
// the device loop ends even if a reduction misbehaves.
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cg_internal.cuh"
#include "spmv.cuh"

namespace b200la {

// IterateControl::Check; step 0 records the initial residual (res_init).
// Under the lmp cg() rule: no test before the first iteration, success once
// ||r|| <= max(rtol ||r0||, atol), no divergence test.
__device__ __forceinline__ int iterate_check(int step, double value, const CgScalars &s, double first) {
  if (s.stop_rule == B200LA_STOP_LMP_CG) {
    if (step > 0 && value <= fmax(s.rtol * first, s.atol)) return B200LA_SUCCESS_REL;
    if (step >= s.maxits) return B200LA_FAIL_MAXITS;
    return B200LA_ITERATE;
  }
  if (value <= s.atol) return B200LA_SUCCESS_ABS;
  if (value < s.rtol * first) return B200LA_SUCCESS_REL;
  if (value > s.dtol * first) return B200LA_FAIL_DIV;
  if (step >= s.maxits) return B200LA_FAIL_MAXITS;
  return B200LA_ITERATE;
}

template <typename T> struct CgVecs {
  T *x, *r, *p, *Ap;
  const T *invd;  // nullptr without preconditioner
  int64_t n;
};

// ---- init: r = b - A x0, z = invD r, p = z, rz = r.z, res_init -----------------
template <typename T, bool PRE> struct InitEmit {
  const T *__restrict__ b;
  const T *__restrict__ x_user;
  CgVecs<T> v;
  Acc<T> rr, rz;
  __device__ __forceinline__ void operator()(int row, T y) {
    T r = b[row] - y;  // r.ScaleAdd(b, -1): -1*(Ax) + b
    v.x[row] = x_user[row];
    v.r[row] = r;
    T z = PRE ? r * v.invd[row] : r;
    v.p[row] = z;
    rr.add(r * r);
    rz.add(r * z);
  }
};

template <typename Op, typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) cg_init_kernel(Op op, const T *__restrict__ x_user, const T *__restrict__ b,
                                                         CgVecs<T> v, double *part, CgScalars *sc) {
  InitEmit<T, PRE> e{b, x_user, v};
  op.run(x_user, e);
  double s[2] = {e.rr.value(), e.rz.value()};
  if (grid_sum_last<2>(s, part, &sc->ticket[0]) && threadIdx.x == 0) {
    double res = sqrt(s[0]);
    sc->rr = s[0];
    sc->rz = PRE ? s[1] : s[0];
    sc->res = res;
    sc->res_init = res;
    sc->iter = 0;
    sc->guard = 0;
    sc->state = iterate_check(0, res, *sc, res);
  }
}

// Start from x0 = 0: r = b exactly (b - A*0), no SpMV needed.
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) cg_init_zero_kernel(const T *__restrict__ b, CgVecs<T> v, double *part,
                                                              CgScalars *sc) {
  Acc<T> rr, rz;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += stride) {
    const T r = b[i];
    v.x[i] = T(0);
    v.r[i] = r;
    const T z = PRE ? r * v.invd[i] : r;
    v.p[i] = z;
    rr.add(r * r);
    rz.add(r * z);
  }
  double s[2] = {rr.value(), rz.value()};
  if (grid_sum_last<2>(s, part, &sc->ticket[0]) && threadIdx.x == 0) {
    double res = sqrt(s[0]);
    sc->rr = s[0];
    sc->rz = PRE ? s[1] : s[0];
    sc->res = res;
    sc->res_init = res;
    sc->iter = 0;
    sc->guard = 0;
    sc->state = iterate_check(0, res, *sc, res);
  }
}

// ---- K1: Ap = A p and p.Ap --------------------------------------------------------
template <typename T> struct SpmvDotEmit {
  T *__restrict__ Ap;
  const T *__restrict__ p;
  Acc<T> acc;
  __device__ __forceinline__ void operator()(int row, T y) {
    Ap[row] = y;
    acc.add(y * __ldg(p + row));
  }
};

template <typename Op, typename T>
__global__ void __launch_bounds__(kBlock) cg_spmv_kernel(Op op, CgVecs<T> v, double *part, CgScalars *sc) {
  if (__ldg(&sc->state) != B200LA_ITERATE) return;
  SpmvDotEmit<T> e{v.Ap, v.p};
  op.run(v.p, e);
  double s[1] = {e.acc.value()};
  if (grid_sum_last<1>(s, part, &sc->ticket[1]) && threadIdx.x == 0) {
    sc->pAp = s[0];
    double alpha = sc->rz / s[0];
    sc->alpha = alpha;
    if (!(s[0] != 0.0) || !isfinite(alpha)) sc->state = B200LA_FAIL_BREAKDOWN;
  }
}

// ---- K2: x += alpha p, r -= alpha Ap, sums r.r and r.z ----------------------------
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) cg_update_kernel(CgVecs<T> v, double *part, CgScalars *sc) {
  if (__ldg(&sc->state) != B200LA_ITERATE) return;
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  const T alpha = (T)sc->alpha;
  Acc<T> rr, rz;
  const int64_t n = v.n, nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
    V xv = reinterpret_cast<V *>(v.x)[i];
    V pv = reinterpret_cast<const V *>(v.p)[i];
    V rv = reinterpret_cast<V *>(v.r)[i];
    V av = reinterpret_cast<const V *>(v.Ap)[i];
    V dv;
    if (PRE) dv = reinterpret_cast<const V *>(v.invd)[i];
    T *xs = reinterpret_cast<T *>(&xv);
    T *rs = reinterpret_cast<T *>(&rv);
    const T *ps = reinterpret_cast<const T *>(&pv);
    const T *as = reinterpret_cast<const T *>(&av);
    const T *ds = reinterpret_cast<const T *>(&dv);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      xs[k] = fma(alpha, ps[k], xs[k]);
      rs[k] = fma(-alpha, as[k], rs[k]);
      rr.add(rs[k] * rs[k]);
      if (PRE) rz.add(rs[k] * (rs[k] * ds[k]));
    }
    reinterpret_cast<V *>(v.x)[i] = xv;
    reinterpret_cast<V *>(v.r)[i] = rv;
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    v.x[i] = fma(alpha, v.p[i], v.x[i]);
    T r = fma(-alpha, v.Ap[i], v.r[i]);
    v.r[i] = r;
    rr.add(r * r);
    if (PRE) rz.add(r * (r * v.invd[i]));
  }
  double s[2] = {rr.value(), rz.value()};
  if (grid_sum_last<2>(s, part, &sc->ticket[2]) && threadIdx.x == 0) {
    double res = sqrt(s[0]);
    int it = sc->iter + 1;
    sc->iter = it;
    sc->rr = s[0];
    sc->res = res;
    int st = iterate_check(it, res, *sc, sc->res_init);
    double rz_new = PRE ? s[1] : s[0];
    sc->beta = rz_new / sc->rz;
    sc->rz_prev = sc->rz;
    sc->rz = rz_new;
    sc->state = st;
  }
}

// ---- K3: p = beta p + z; ends the device loop ---------------------------------------
template <typename T, bool PRE, bool IN_GRAPH = true>
__global__ void __launch_bounds__(kBlock) cg_direction_kernel(CgVecs<T> v, CgScalars *sc,
                                                              cudaGraphConditionalHandle loop) {
  const int state = __ldg(&sc->state);
  if (IN_GRAPH && blockIdx.x == 0 && threadIdx.x == 0) {
    int g = sc->guard + 1;
    sc->guard = g;
    bool go = state == B200LA_ITERATE;
    if (go && g > sc->maxits + 2) {  // unreachable unless K2 failed to count
      sc->state = B200LA_FAIL_BREAKDOWN;
      go = false;
    }
    cudaGraphSetConditional(loop, go ? 1u : 0u);
  }
  if (state != B200LA_ITERATE) return;
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  const T beta = (T)sc->beta;
  const int64_t n = v.n, nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
    V pv = reinterpret_cast<V *>(v.p)[i];
    V rv = reinterpret_cast<const V *>(v.r)[i];
    V dv;
    if (PRE) dv = reinterpret_cast<const V *>(v.invd)[i];
    T *ps = reinterpret_cast<T *>(&pv);
    const T *rs = reinterpret_cast<const T *>(&rv);
    const T *ds = reinterpret_cast<const T *>(&dv);
#pragma unroll
    for (int k = 0; k < W; ++k) ps[k] = fma(beta, ps[k], PRE ? rs[k] * ds[k] : rs[k]);
    reinterpret_cast<V *>(v.p)[i] = pv;
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    v.p[i] = fma(beta, v.p[i], PRE ? v.r[i] * v.invd[i] : v.r[i]);
}

// ---- resume after a residual replacement: x = 0, p = z + beta p ------------------
// Every block derives beta from the same two scalars; block 0 then resets the
// solve's scalars for the new start (none of which the other blocks read).
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) cg_resume_kernel(CgVecs<T> v, const double *__restrict__ sums,
                                                           CgScalars *sc, int restart) {
  const double rr = sums[0], rz_new = PRE ? sums[1] : sums[0];
  const double beta_d = rz_new / __ldg(&sc->rz_prev);
  const bool keep = !restart && isfinite(beta_d);
  const T beta = keep ? (T)beta_d : T(0);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < v.n; i += stride) {
    const T r = v.r[i];
    const T z = PRE ? r * v.invd[i] : r;
    v.x[i] = T(0);
    v.p[i] = keep ? fma(beta, v.p[i], z) : z;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double res = sqrt(rr);
    sc->rr = rr;
    sc->rz = rz_new;
    sc->res = res;
    sc->res_init = res;
    sc->iter = 0;
    sc->guard = 0;
    sc->state = iterate_check(0, res, *sc, res);
  }
}

}  // namespace b200la

using namespace b200la;

namespace b200la {

// One iteration: K1, K2, K3 on stream `st` (captured into the graph body,
// or launched from the host loop when graphs are off).
// M = stored matrix value type, T = vector type (M == T, or FP32 values over
// FP64 vectors).
template <typename M, typename T, bool PRE, bool IN_GRAPH>
static int cg_launch_body_t(b200la_cg s, cudaStream_t st, cudaGraphConditionalHandle h) {
  b200la_mat A = s->A;
  b200la_ctx c = A->ctx;
  CgVecs<T> v{(T *)s->x, (T *)s->r, (T *)s->p, (T *)s->Ap, (const T *)s->invd, s->n};
  B_TRY((with_schedule<M, T>(A, [&](auto op) -> int {
    using Op = decltype(op);
    B_TRY(grid_for(c, (const void *)cg_spmv_kernel<Op, T>, op.work_items(), Op::kRowsPerBlock, &s->grid_spmv));
    cg_spmv_kernel<Op, T><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part, s->sc);
    return B200LA_OK;
  })));
  cg_update_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->part, s->sc);
  cg_direction_kernel<T, PRE, IN_GRAPH><<<s->grid_ew, kBlock, 0, st>>>(v, s->sc, h);
  return B200LA_OK;
}

// Calls f(M(), T(), std::bool_constant<PRE>()) with the solver's matrix value
// type M, vector type T and preconditioning.
template <typename F> static int cg_types(b200la_cg s, F &&f) {
  const bool pre = s->prm.precond != 0;
  auto go = [&](auto m, auto t) -> int { return pre ? f(m, t, std::true_type()) : f(m, t, std::false_type()); };
  if (s->A->dtype == B200LA_F64) return go(double(), double());
  if (s->vdtype == B200LA_F64) return go(float(), double());
  return go(float(), float());
}

template <typename M, typename T, bool PRE>
static int cg_build_graph_t(b200la_cg s) {
  b200la_mat A = s->A;
  b200la_ctx c = A->ctx;
  if (s->exec) { cudaGraphExecDestroy(s->exec); s->exec = nullptr; }
  if (s->graph) { cudaGraphDestroy(s->graph); s->graph = nullptr; }
  CgVecs<T> v{(T *)s->x, (T *)s->r, (T *)s->p, (T *)s->Ap, (const T *)s->invd, s->n};
  B_TRY(grid_for(c, (const void *)cg_update_kernel<T, PRE>, (s->n + Vec16<T>::n - 1) / Vec16<T>::n, kBlock, &s->grid_ew));
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
  int rc = cg_launch_body_t<M, T, PRE, true>(s, cs, h);
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

static int cg_build_graph(b200la_cg s) {
  return cg_types(s, [&](auto m, auto t, auto pre) -> int {
    return cg_build_graph_t<decltype(m), decltype(t), decltype(pre)::value>(s);
  });
}

template <typename M, typename T, bool PRE>
static int cg_launch_init_t(b200la_cg s, const void *x_user, const void *b) {
  b200la_mat A = s->A;
  CgVecs<T> v{(T *)s->x, (T *)s->r, (T *)s->p, (T *)s->Ap, (const T *)s->invd, s->n};
  cudaStream_t st = A->ctx->stream;
  if (!x_user) {
    int grid;
    B_TRY(grid_for(A->ctx, (const void *)cg_init_zero_kernel<T, PRE>, s->n, kBlock, &grid));
    cg_init_zero_kernel<T, PRE><<<grid, kBlock, 0, st>>>((const T *)b, v, s->part, s->sc);
    B_CUDA(cudaGetLastError());
    return B200LA_OK;
  }
  return with_schedule<M, T>(A, [&](auto op) -> int {
    using Op = decltype(op);
    int grid;
    B_TRY(grid_for(A->ctx, (const void *)cg_init_kernel<Op, T, PRE>, op.work_items(), Op::kRowsPerBlock, &grid));
    cg_init_kernel<Op, T, PRE><<<grid, kBlock, 0, st>>>(op, (const T *)x_user, (const T *)b, v, s->part, s->sc);
    B_CUDA(cudaGetLastError());
    return B200LA_OK;
  });
}

static int cg_launch_init(b200la_cg s, const void *x_user, const void *b) {
  return cg_types(s, [&](auto m, auto t, auto pre) -> int {
    return cg_launch_init_t<decltype(m), decltype(t), decltype(pre)::value>(s, x_user, b);
  });
}

int cg_start(b200la_cg s, const void *x_dev, const void *b_dev) { return cg_launch_init(s, x_dev, b_dev); }

int cg_resume(b200la_cg s, const double *sums, bool restart) {
  cudaStream_t st = s->A->ctx->stream;
  return cg_types(s, [&](auto m, auto t, auto pre) -> int {
    using T = decltype(t);
    constexpr bool PRE = decltype(pre)::value;
    CgVecs<T> v{(T *)s->x, (T *)s->r, (T *)s->p, (T *)s->Ap, (const T *)s->invd, s->n};
    int grid;
    B_TRY(grid_for(s->A->ctx, (const void *)cg_resume_kernel<T, PRE>, s->n, kBlock, &grid));
    cg_resume_kernel<T, PRE><<<grid, kBlock, 0, st>>>(v, sums, s->sc, restart ? 1 : 0);
    B_CUDA(cudaGetLastError());
    return B200LA_OK;
  });
}

template <typename M, typename T, bool PRE>
static int cg_host_loop_t(b200la_cg s) {
  cudaStream_t st = s->A->ctx->stream;
  // the kernels return at once when the state is no longer "iterate", so
  // checking the state every 16 iterations runs the same iterations
  for (int64_t it = 0;; it += 16) {
    for (int k = 0; k < 16; ++k) B_TRY((cg_launch_body_t<M, T, PRE, false>(s, st, 0)));
    B_CUDA(cudaGetLastError());
    CgScalars h;
    B_TRY(cg_fetch(s, &h));
    if (h.state != B200LA_ITERATE || it > (int64_t)s->prm.maxits + 32) break;
  }
  return B200LA_OK;
}

int cg_run(b200la_cg s) {
  b200la_mat A = s->A;
  if (!A->ctx->use_graphs) {
    return cg_types(s, [&](auto m, auto t, auto pre) -> int {
      return cg_host_loop_t<decltype(m), decltype(t), decltype(pre)::value>(s);
    });
  }
  if (A->format != s->g_format || A->param != s->g_param || A->sched_gen != s->g_gen) B_TRY(cg_build_graph(s));
  B_CUDA(cudaGraphLaunch(s->exec, A->ctx->stream));
  return B200LA_OK;
}

int cg_fetch(b200la_cg s, CgScalars *out) {
  cudaStream_t st = s->A->ctx->stream;
  B_CUDA(cudaMemcpyAsync(s->sc_host, s->sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  *out = *s->sc_host;
  return B200LA_OK;
}

// Runs the init kernel and then `iters` iterations as separate launches with
// CUDA events between the kernels; adds the mean time per launch of K1, K2
// and K3 to ms[0..2].  Same kernels as the graph body (K3 without the loop
// condition).
template <typename M, typename T, bool PRE>
static int cg_profile_t(b200la_cg s, const void *x_user, const void *b, int iters, double *ms) {
  b200la_mat A = s->A;
  cudaStream_t st = A->ctx->stream;
  CgVecs<T> v{(T *)s->x, (T *)s->r, (T *)s->p, (T *)s->Ap, (const T *)s->invd, s->n};
  B_TRY((cg_launch_init_t<M, T, PRE>(s, x_user, b)));
  // every pass is queued before the first wait, after one untimed pass, so
  // the timed kernels run back to back and no host launch gap falls between
  // an event pair
  std::vector<cudaEvent_t> ev((size_t)(iters > 0 ? iters : 0) * 4);
  for (auto &e : ev) B_CUDA(cudaEventCreate(&e));
  int rc = B200LA_OK;
  auto pass = [&](cudaEvent_t *e) -> int {
    if (e) cudaEventRecord(e[0], st);
    B_TRY((with_schedule<M, T>(A, [&](auto op) -> int {
      using Op = decltype(op);
      cg_spmv_kernel<Op, T><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part, s->sc);
      return B200LA_OK;
    })));
    if (e) cudaEventRecord(e[1], st);
    cg_update_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->part, s->sc);
    if (e) cudaEventRecord(e[2], st);
    cg_direction_kernel<T, PRE, false><<<s->grid_ew, kBlock, 0, st>>>(v, s->sc, 0);
    if (e) cudaEventRecord(e[3], st);
    return B200LA_OK;
  };
  if (iters > 0) rc = pass(nullptr);
  for (int it = 0; it < iters && rc == B200LA_OK; ++it) rc = pass(&ev[(size_t)it * 4]);
  const cudaError_t se = cudaStreamSynchronize(st);
  float acc[3] = {0.f, 0.f, 0.f};
  for (int it = 0; it < iters && rc == B200LA_OK && se == cudaSuccess; ++it)
    for (int k = 0; k < 3; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[(size_t)it * 4 + k], ev[(size_t)it * 4 + k + 1]);
      acc[k] += t;
    }
  for (auto &e : ev) cudaEventDestroy(e);
  B_CUDA(se);
  B_CUDA(cudaGetLastError());
  for (int k = 0; k < 3; ++k) ms[k] = iters > 0 ? acc[k] / iters : 0.0;
  return rc;
}

}  // namespace b200la

extern "C" {

int b200la_cg_profile(b200la_cg s, b200la_vec b, b200la_vec x, int iters, double *ms) {
  B_CHECK(s && b && x && ms && iters >= 0, B200LA_ERR_INVALID, "cg_profile: bad argument");
  B_CHECK(b->n == s->n && x->n == s->n && s->n > 0, B200LA_ERR_INVALID, "cg_profile: sizes");
  B_CHECK(b->dtype == s->vdtype && x->dtype == s->vdtype, B200LA_ERR_DTYPE, "cg_profile: dtype");
  return cg_types(s, [&](auto m, auto t, auto pre) -> int {
    return cg_profile_t<decltype(m), decltype(t), decltype(pre)::value>(s, x->d, b->d, iters, ms);
  });
}

int b200la_cg_create(b200la_mat A, const b200la_cg_params *prm, b200la_cg *out) {
  B_CHECK(A, B200LA_ERR_INVALID, "cg_create: null argument");
  return cg_create_ex(A, prm, A->dtype, nullptr, out);
}

}  // extern "C"

int b200la::cg_create_ex(b200la_mat A, const b200la_cg_params *prm, int vdtype, b200la_mat invd_src,
                         b200la_cg *out) {
  B_CHECK(A && prm && out, B200LA_ERR_INVALID, "cg_create: null argument");
  B_CHECK(vdtype == A->dtype || (A->dtype == B200LA_F32 && vdtype == B200LA_F64), B200LA_ERR_DTYPE,
          "cg_create: vectors of dtype %d over a matrix of dtype %d", vdtype, A->dtype);
  B_CHECK(vdtype == A->dtype || !prm->precond ||
              (invd_src && invd_src->dtype == vdtype && invd_src->nrow == A->nrow && invd_src->nnz == A->nnz),
          B200LA_ERR_INVALID, "cg_create: mixed storage with Jacobi needs an FP64 matrix of the same structure");
  B_CHECK(A->nrow == A->ncol, B200LA_ERR_INVALID, "cg_create: matrix is %dx%d, not square", A->nrow, A->ncol);
  B_CHECK(prm->maxits >= 0 && prm->maxits <= kMaxIts, B200LA_ERR_INVALID, "cg_create: maxits %d not in [0, %d]",
          prm->maxits, kMaxIts);
  B_CHECK(prm->atol >= 0.0 && prm->rtol >= 0.0 && prm->dtol > 0.0, B200LA_ERR_INVALID,
          "cg_create: tolerances must be atol >= 0, rtol >= 0, dtol > 0");
  B_CHECK(prm->stop_rule == B200LA_STOP_ITERATE_CONTROL || (prm->stop_rule == B200LA_STOP_LMP_CG && !prm->precond),
          B200LA_ERR_INVALID, "cg_create: stop_rule %d (the lmp cg() rule takes no preconditioner)", prm->stop_rule);
  b200la_ctx c = A->ctx;
  cudaStream_t st = c->stream;
  b200la_cg s = new b200la_cg_s();
  s->A = A;
  s->ctx = c;
  s->prm = *prm;
  s->vdtype = vdtype;
  s->n = A->nrow;
  size_t es = dtype_size(vdtype);
  size_t vb = es * (size_t)(s->n > 0 ? s->n : 1);
  int rc = B200LA_OK;
  auto cleanup = [&](int code) { b200la_cg_destroy(s); return code; };
  if (cudaMallocAsync(&s->x, vb, st) != cudaSuccess || cudaMallocAsync(&s->r, vb, st) != cudaSuccess ||
      cudaMallocAsync(&s->p, vb, st) != cudaSuccess || cudaMallocAsync(&s->Ap, vb, st) != cudaSuccess ||
      cudaMallocAsync(&s->part, sizeof(double) * 2 * kMaxReduceBlocks, st) != cudaSuccess ||
      cudaMallocAsync(&s->sc, sizeof(CgScalars), st) != cudaSuccess ||
      cudaMallocHost(&s->sc_host, sizeof(CgScalars)) != cudaSuccess)
    return cleanup(fail(B200LA_ERR_NOMEM, "cg_create: allocation of %zu-byte work vectors failed", vb));
  CgScalars init = {};
  init.atol = prm->atol;
  init.rtol = prm->rtol;
  init.dtol = prm->dtol;
  init.maxits = prm->maxits;
  init.stop_rule = prm->stop_rule;
  init.state = B200LA_ITERATE;
  if (cudaMemcpyAsync(s->sc, &init, sizeof(init), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return cleanup(fail(B200LA_ERR_CUDA, "cg_create: scalar upload failed"));
  if (prm->precond) {
    if (cudaMallocAsync(&s->invd, vb, st) != cudaSuccess)
      return cleanup(fail(B200LA_ERR_NOMEM, "cg_create: allocation of the inverse diagonal failed"));
    b200la_vec_s dv{c, s->n, vdtype, s->invd, false};
    rc = b200la_mat_inv_diag(vdtype == A->dtype ? A : invd_src, &dv);
    if (rc != B200LA_OK) return cleanup(rc);
  }
  if (s->n > 0) {
    rc = cg_build_graph(s);
    if (rc != B200LA_OK) return cleanup(rc);
  }
  *out = s;
  return B200LA_OK;
}

extern "C" {

int b200la_cg_destroy(b200la_cg s) {
  if (!s) return B200LA_OK;
  cudaStream_t st = s->ctx->stream;
  cudaStreamSynchronize(st);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  void *bufs[] = {s->x, s->r, s->p, s->Ap, s->invd, s->part, s->sc};
  for (void *b : bufs)
    if (b) cudaFreeAsync(b, st);
  if (s->sc_host) cudaFreeHost(s->sc_host);
  delete s;
  return B200LA_OK;
}

int b200la_cg_solve(b200la_cg s, b200la_vec b, b200la_vec x, b200la_cg_result *res) {
  B_CHECK(s && b && x && res, B200LA_ERR_INVALID, "cg_solve: null argument");
  b200la_mat A = s->A;
  B_CHECK(b->n == s->n && x->n == s->n, B200LA_ERR_INVALID, "cg_solve: vector sizes %lld/%lld vs %lld",
          (long long)b->n, (long long)x->n, (long long)s->n);
  B_CHECK(b->dtype == s->vdtype && x->dtype == s->vdtype, B200LA_ERR_DTYPE, "cg_solve: dtype mismatch");
  memset(res, 0, sizeof(*res));
  if (s->n == 0) {
    res->state = B200LA_SUCCESS_ABS;
    return B200LA_OK;
  }
  cudaStream_t st = A->ctx->stream;
  B_TRY(cg_start(s, x->d, b->d));
  B_TRY(cg_run(s));
  B_CUDA(cudaMemcpyAsync(x->d, s->x, (size_t)s->n * dtype_size(s->vdtype), cudaMemcpyDeviceToDevice, st));
  CgScalars h;
  B_TRY(cg_fetch(s, &h));
  res->iters = h.iter;
  // the lmp cg() returns the 0-based index of the iteration that met its test
  if (s->prm.stop_rule == B200LA_STOP_LMP_CG && h.state == B200LA_SUCCESS_REL) res->iters = h.iter - 1;
  res->state = h.state;
  res->res = h.res;
  res->res_init = h.res_init;
  res->res_rel = h.res_init > 0.0 ? h.res / h.res_init : 0.0;
  if (h.state == B200LA_SUCCESS_ABS || h.state == B200LA_SUCCESS_REL)
    res->solver_state = B200LA_SOLVER_SUCCESS;
  else if (h.state == B200LA_FAIL_DIV || h.state == B200LA_FAIL_MAXITS)
    res->solver_state = B200LA_SOLVER_EXCEEDED;
  else
    res->solver_state = B200LA_SOLVER_ERROR;
  return B200LA_OK;
}

int b200la_pcg_solve(b200la_mat A, b200la_vec b, b200la_vec x, const b200la_cg_params *prm, b200la_cg_result *res) {
  b200la_cg s = nullptr;
  B_TRY(b200la_cg_create(A, prm, &s));
  int rc = b200la_cg_solve(s, b, x, res);
  b200la_cg_destroy(s);
  return rc;
}

}  // extern "C"
