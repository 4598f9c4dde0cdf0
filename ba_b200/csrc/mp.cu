// Mixed-precision iterative refinement: FP64 outer residual and update
// around an FP32 Jacobi-PCG, structured like MPIR<LAD_high, LAD_low>::
// SolveImpl (linear_solver/mpir.cc:52-230) without smoothers:
//   r = b - A64 x            (FP64 SpMV, fused with ||r|| and the cast r -> float)
//   loop: c = PCG32(A32, r32) from c = 0 to inner_rtol   (device graph)
//         x += c             (FP64 update, fused cast)
//         r = b - A64 x; stop on the FP64 residual
// With inner_storage = B200LA_MP_F32_VALUES the inner PCG keeps its vectors,
// dot products and Jacobi scaling in FP64 over the FP32 matrix values (each
// widened before its FMA): the matrix, most of an iteration's bytes, still
// moves at 4 bytes per value, while the Krylov recurrence no longer loses
// accuracy to FP32 rounding -- on ill-conditioned systems the FP32 recurrence
// needs far more iterations than FP64 PCG to reach the same inner tolerance.
// The outer test is relative to the initial residual; the reference resets
// res0_ to the latest residual after every pass (mpir.cc:239), which would
// make a relative tolerance relative to the previous pass instead.
#include <cmath>
#include <cstddef>
#include <cstring>
#include <type_traits>

#include "cg_internal.cuh"
#include "spmv.cuh"

namespace b200la {

struct MpScalars {
  double rr;
  double res;
  double in[2];     // r.r and r.z of the residual in the inner type (the inner solve's new start)
  unsigned ticket[2];
};

// The FP64 residual r = b - A64 x, its norm, and its copy in the inner
// solve's type R (float, or double under mixed storage) written straight into
// the inner solve's r, with that copy's r.r and r.z (Jacobi) in the inner
// arithmetic, as the inner solve's own kernels form them.
template <typename Op, typename R, bool PRE> struct ResidualEmit {
  const double *__restrict__ b;
  R *__restrict__ rin;
  const R *__restrict__ invd;
  Acc<double> rr;
  Acc<R> rr_in, rz_in;
  __device__ __forceinline__ void operator()(int row, double y) {
    const double r = b[row] - y;
    const R ri = (R)r;
    rin[row] = ri;
    rr.add(r * r);
    rr_in.add(ri * ri);
    if (PRE) rz_in.add(ri * (ri * invd[row]));
  }
};

template <typename Op, typename R, bool PRE>
__global__ void __launch_bounds__(kBlock) mp_residual_kernel(Op op, const double *__restrict__ x,
                                                             const double *__restrict__ b, R *__restrict__ rin,
                                                             const R *__restrict__ invd, double *part,
                                                             MpScalars *sc) {
  ResidualEmit<Op, R, PRE> e{b, rin, invd};
  op.run(x, e);
  double s[3] = {e.rr.value(), e.rr_in.value(), e.rz_in.value()};
  if (grid_sum_last<3>(s, part, &sc->ticket[0]) && threadIdx.x == 0) {
    sc->rr = s[0];
    sc->res = sqrt(s[0]);
    sc->in[0] = s[1];
    sc->in[1] = PRE ? s[2] : s[1];
  }
}

__global__ void __launch_bounds__(kBlock) mp_correct_kernel(int64_t n, double *__restrict__ x,
                                                            const float *__restrict__ c) {
  const int64_t n4 = n / 4;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
    const float4 cv = reinterpret_cast<const float4 *>(c)[i];
    double2 a = reinterpret_cast<double2 *>(x)[2 * i];
    double2 b = reinterpret_cast<double2 *>(x)[2 * i + 1];
    a.x += (double)cv.x;
    a.y += (double)cv.y;
    b.x += (double)cv.z;
    b.y += (double)cv.w;
    reinterpret_cast<double2 *>(x)[2 * i] = a;
    reinterpret_cast<double2 *>(x)[2 * i + 1] = b;
  }
  for (int64_t i = n4 * 4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] += (double)c[i];
}

// x += c with an FP64 correction (mixed storage)
__global__ void __launch_bounds__(kBlock) mp_correct64_kernel(int64_t n, double *__restrict__ x,
                                                              const double *__restrict__ c) {
  const int64_t n2 = n / 2;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n2; i += stride) {
    double2 a = reinterpret_cast<double2 *>(x)[i];
    const double2 cv = reinterpret_cast<const double2 *>(c)[i];
    a.x += cv.x;
    a.y += cv.y;
    reinterpret_cast<double2 *>(x)[i] = a;
  }
  for (int64_t i = n2 * 2 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) x[i] += c[i];
}

}  // namespace b200la

using namespace b200la;

struct b200la_mp_s {
  b200la_mat A64;
  b200la_ctx ctx;            // kept for destroy, which may come after A64's
  b200la_mat A32;
  b200la_mp_params prm;
  b200la_cg inner;
  int64_t n;
  double *part;
  MpScalars *sc;
  MpScalars *sc_host;
};

namespace b200la {

static int mp_residual(b200la_mp s, const double *x, const double *b, double *res) {
  b200la_mat A = s->A64;
  cudaStream_t st = A->ctx->stream;
  const bool f64in = s->prm.inner_storage == B200LA_MP_F32_VALUES;
  auto launch = [&](auto op, auto rtag, auto pre) -> int {
    using Op = decltype(op);
    using R = decltype(rtag);
    constexpr bool PRE = decltype(pre)::value;
    int grid;
    B_TRY(grid_for(A->ctx, (const void *)mp_residual_kernel<Op, R, PRE>, op.work_items(), Op::kRowsPerBlock,
                   &grid));
    mp_residual_kernel<Op, R, PRE><<<grid, kBlock, 0, st>>>(op, x, b, (R *)s->inner->r, (const R *)s->inner->invd,
                                                            s->part, s->sc);
    B_CUDA(cudaGetLastError());
    return B200LA_OK;
  };
  const bool pre = s->prm.precond != 0;
  B_TRY(with_schedule<double>(A, [&](auto op) -> int {
    if (f64in) return pre ? launch(op, double(), std::true_type()) : launch(op, double(), std::false_type());
    return pre ? launch(op, float(), std::true_type()) : launch(op, float(), std::false_type());
  }));
  B_CUDA(cudaMemcpyAsync(s->sc_host, s->sc, sizeof(MpScalars), cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  *res = s->sc_host->res;
  return B200LA_OK;
}

}  // namespace b200la

extern "C" {

int b200la_mp_destroy(b200la_mp s) {
  if (!s) return B200LA_OK;
  cudaStream_t st = s->ctx->stream;
  cudaStreamSynchronize(st);
  if (s->inner) b200la_cg_destroy(s->inner);
  if (s->A32) b200la_mat_destroy(s->A32);
  if (s->part) cudaFreeAsync(s->part, st);
  if (s->sc) cudaFreeAsync(s->sc, st);
  if (s->sc_host) cudaFreeHost(s->sc_host);
  delete s;
  return B200LA_OK;
}

int b200la_mp_create(b200la_mat A64, const b200la_mp_params *prm, b200la_mp *out) {
  B_CHECK(A64 && prm && out, B200LA_ERR_INVALID, "mp_create: null argument");
  B_CHECK(A64->dtype == B200LA_F64, B200LA_ERR_DTYPE, "mp_create: the outer matrix must be FP64");
  B_CHECK(A64->nrow == A64->ncol, B200LA_ERR_INVALID, "mp_create: matrix is not square");
  B_CHECK(prm->max_outer >= 0 && prm->max_outer <= 1000, B200LA_ERR_INVALID, "mp_create: max_outer %d",
          prm->max_outer);
  B_CHECK(prm->inner_rtol > 0.0 && prm->inner_rtol < 1.0, B200LA_ERR_INVALID, "mp_create: inner_rtol %g",
          prm->inner_rtol);
  B_CHECK(prm->atol >= 0.0 && prm->rtol >= 0.0 && prm->dtol > 0.0, B200LA_ERR_INVALID, "mp_create: tolerances");
  B_CHECK(prm->inner_storage == B200LA_MP_F32 || prm->inner_storage == B200LA_MP_F32_VALUES, B200LA_ERR_INVALID,
          "mp_create: inner_storage %d", prm->inner_storage);
  const bool f64in = prm->inner_storage == B200LA_MP_F32_VALUES;
  b200la_mp s = new b200la_mp_s();
  s->A64 = A64;
  s->ctx = A64->ctx;
  s->prm = *prm;
  s->n = A64->nrow;
  cudaStream_t st = A64->ctx->stream;
  int rc = b200la_mat_cast(A64, B200LA_F32, &s->A32);
  if (rc == B200LA_OK && prm->tune) rc = b200la_mat_tune(s->A32, nullptr, nullptr, nullptr);
  if (rc == B200LA_OK) {
    b200la_cg_params ip = {prm->inner_maxits, 0.0, prm->inner_rtol, 1e30, prm->precond};
    rc = f64in ? cg_create_ex(s->A32, &ip, B200LA_F64, A64, &s->inner) : b200la_cg_create(s->A32, &ip, &s->inner);
  }
  if (rc == B200LA_OK &&
      (cudaMallocAsync(&s->part, sizeof(double) * 3 * kMaxReduceBlocks, st) != cudaSuccess ||
       cudaMallocAsync(&s->sc, sizeof(MpScalars), st) != cudaSuccess ||
       cudaMallocHost(&s->sc_host, sizeof(MpScalars)) != cudaSuccess ||
       cudaMemsetAsync(s->sc, 0, sizeof(MpScalars), st) != cudaSuccess))
    rc = fail(B200LA_ERR_NOMEM, "mp_create: allocation failed");
  if (rc == B200LA_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(B200LA_ERR_CUDA, "mp_create: sync");
  if (rc != B200LA_OK) {
    b200la_mp_destroy(s);
    return rc;
  }
  *out = s;
  return B200LA_OK;
}

int b200la_mp_inner_matrix(b200la_mp s, b200la_mat *out) {
  B_CHECK(s && out, B200LA_ERR_INVALID, "mp_inner_matrix: null argument");
  *out = s->A32;
  return B200LA_OK;
}

int b200la_mp_solve(b200la_mp s, b200la_vec b, b200la_vec x, b200la_mp_result *res) {
  B_CHECK(s && b && x && res, B200LA_ERR_INVALID, "mp_solve: null argument");
  B_CHECK(b->n == s->n && x->n == s->n, B200LA_ERR_INVALID, "mp_solve: vector sizes");
  B_CHECK(b->dtype == B200LA_F64 && x->dtype == B200LA_F64, B200LA_ERR_DTYPE, "mp_solve: b and x must be FP64");
  memset(res, 0, sizeof(*res));
  if (s->n == 0) {
    res->state = B200LA_SUCCESS_ABS;
    return B200LA_OK;
  }
  b200la_ctx c = s->A64->ctx;
  cudaStream_t st = c->stream;
  const b200la_mp_params &p = s->prm;
  double r = 0.0;
  B_TRY(mp_residual(s, (const double *)x->d, (const double *)b->d, &r));
  const double r0 = r;
  int outer = 0, inner_total = 0;
  const bool f64in = p.inner_storage == B200LA_MP_F32_VALUES;
  int grid_c;
  if (f64in) B_TRY(grid_for(c, (const void *)mp_correct64_kernel, (s->n + 1) / 2, kBlock, &grid_c));
  else B_TRY(grid_for(c, (const void *)mp_correct_kernel, (s->n + 3) / 4, kBlock, &grid_c));
  auto done = [&](double v) { return v <= p.atol || v < p.rtol * r0 || !(v <= p.dtol * r0); };
  // every pass continues the inner solve from the true residual the last
  // residual kernel wrote into it; its search direction is kept unless
  // restart_inner is set, this is the first pass, or the last pass took no
  // step or broke down
  bool restart = true;
  while (!done(r) && outer < p.max_outer) {
    ++outer;
    const double *sums = reinterpret_cast<const double *>(reinterpret_cast<const char *>(s->sc) +
                                                          offsetof(MpScalars, in));  // device address
    B_TRY(cg_resume(s->inner, sums, restart || p.restart_inner != 0));
    B_TRY(cg_run(s->inner));
    if (f64in) mp_correct64_kernel<<<grid_c, kBlock, 0, st>>>(s->n, (double *)x->d, (const double *)s->inner->x);
    else mp_correct_kernel<<<grid_c, kBlock, 0, st>>>(s->n, (double *)x->d, (const float *)s->inner->x);
    B_CUDA(cudaGetLastError());
    B_TRY(mp_residual(s, (const double *)x->d, (const double *)b->d, &r));
    CgScalars h;
    B_TRY(cg_fetch(s->inner, &h));
    inner_total += h.iter;
    // restart the direction when the pass took no step or broke down, or when
    // the replaced residual is more than twice the recurrence's last one (the
    // inner recurrence drifted far from the true residual)
    restart = h.iter == 0 || h.state == B200LA_FAIL_BREAKDOWN || !(sqrt(s->sc_host->in[0]) <= 2.0 * h.res);
  }
  res->outer = outer;
  res->inner_iters = inner_total;
  res->res = r;
  res->res_init = r0;
  res->res_rel = r0 > 0.0 ? r / r0 : 0.0;
  if (r <= p.atol) res->state = B200LA_SUCCESS_ABS;
  else if (r < p.rtol * r0) res->state = B200LA_SUCCESS_REL;
  else if (!(r <= p.dtol * r0)) res->state = B200LA_FAIL_DIV;
  else res->state = B200LA_FAIL_MAXITS;
  res->solver_state = (res->state == B200LA_SUCCESS_ABS || res->state == B200LA_SUCCESS_REL) ? B200LA_SOLVER_SUCCESS
                                                                                               : B200LA_SOLVER_EXCEEDED;
  return B200LA_OK;
}

}  // extern "C"
