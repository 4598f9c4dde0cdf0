// Restarted GMRES on the device: GMRES<LAD, PreLAD>::SolveNoPrecond /
// SolveRight (linear_solver/gmres.h:229-389, 462-713) with modified
// Gram-Schmidt, the Givens helpers (:97-115) and UpdateSolution (:727-746),
// stopping on IterateControl::Check (common/iterate_control.cc:80-107).
//
// One CUDA-graph WHILE loop runs the whole solve; its body is four kernels:
//   G1  at a cycle end: x += P (sum_i y_i V_i) (y from the back substitution
//       G4 left), one pass over the basis
//   G2  at a (re)start: V0 = (b - A x) / res, z = P V0, reset H and g
//   G3  w = A z (z = P V_j, or V_j itself without preconditioner), fused
//       with the partial sums of w.V_0
//   G4  the rest of the Arnoldi step in one cooperative kernel: for
//       i = 0..j, h_ij from the previous partial sums (every block adds
//       them in the same order), w -= h_ij V_i fused with the next dot
//       (w.V_{i+1}, or w.w at the end), one grid barrier per i; then
//       V_{j+1} = w / ||w||, z = P V_{j+1}; block 0 applies the Givens
//       rotations, the test, and at a cycle end solves H y = g.  When w
//       fits in the SMs' shared memory (up to ~4.3 M FP64 rows on 148
//       SMs) it stays there for the whole step.
// The reference runs the Gram-Schmidt loop as 2 (j+1) separate BLAS-1 calls
// with a blocking scalar read each; here one launch covers it and the host
// never waits.  As in the reference, a restart normalises V0 by the
// recurrence residual |g[j+1]|, not by V0's own norm.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "krylov.cuh"
#include "spmv.cuh"

namespace b200la {

constexpr int kMaxBasis = 512;

struct GmScalars {
  double res, res_init, first;
  double atol, rtol, dtol;
  int iter;          // Arnoldi steps over all cycles
  int j;             // step within the cycle
  int m;             // basis size: min(size_basis, maxits)
  int kend;          // last step of the cycle being applied by G1
  int state;
  int phase;         // kGmRestart / kGmStep / kGmUpdate / kGmDone
  int maxits;
  int guard;         // body passes
  alignas(128) unsigned err;  // a G4 barrier wait ran out
  unsigned ticket[2];
  int stall_block;            // test hook: this block of the resident G4 never reaches its barrier (-1: none)
  // G4's grid barrier: arrivals since the solve started (own line) and the
  // barriers its launches have passed (written by block 0 at the end)
  alignas(128) unsigned long long bar_count;
  unsigned long long bar_done;
};

enum { kGmRestart = 0, kGmStep = 1, kGmUpdate = 2, kGmDone = 3 };

__device__ __forceinline__ int gm_check(int step, double value, const GmScalars &s) {
  if (value <= s.atol) return B200LA_SUCCESS_ABS;
  if (value < s.rtol * s.first) return B200LA_SUCCESS_REL;
  if (value > s.dtol * s.first) return B200LA_FAIL_DIV;
  if (step >= s.maxits) return B200LA_FAIL_MAXITS;
  return B200LA_ITERATE;
}

// Device buffers of one solver.
template <typename T> struct GmBufs {
  T *V;          // (m + 1) vectors of ldv values
  int64_t ldv;
  T *w, *z, *x;
  const T *b, *invd;
  double *H;     // [m][m + 1]: H(j, i) at j * (m + 1) + i
  double *g, *cs, *sn, *y;
  int64_t n;
};

// ---- start: ||b - A x0||, the first test ----------------------------------------
template <typename T> struct NormResEmit {
  const T *__restrict__ b;
  Acc<T> rr;
  __device__ __forceinline__ void operator()(int row, T y) {
    const T r = b[row] - y;
    rr.add(r * r);
  }
};

template <typename Op, typename T>
__global__ void __launch_bounds__(kBlock) gm_start_kernel(Op op, GmBufs<T> v, double *part, GmScalars *sc) {
  NormResEmit<T> e{v.b};
  op.run(v.x, e);
  double s[1] = {e.rr.value()};
  if (grid_sum_last<1>(s, part, &sc->ticket[0]) && threadIdx.x == 0) {
    const double res = (double)(T)sqrt((T)s[0]);  // Norm2 in the value type
    sc->res = sc->res_init = sc->first = res;
    sc->iter = 0;
    sc->state = gm_check(0, res, *sc);
    sc->phase = sc->state == B200LA_ITERATE ? kGmRestart : kGmDone;
  }
}

// ---- G1: x += P (sum_i y_i V_i) at the end of a cycle ----------------------------
template <typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) gm_update_kernel(GmBufs<T> v, GmScalars *sc) {
  if (__ldg(&sc->phase) != kGmUpdate) return;
  const int k = __ldg(&sc->kend);
  for_each_chunk<T>(v.n, [&](int64_t i0, auto cc) {
    constexpr int C = decltype(cc)::value;
    T acc[C], t[C];
    if (PRE) {
#pragma unroll
      for (int q = 0; q < C; ++q) acc[q] = T(0);  // z = 0; z.Axpy(V_i, y_i) ...
    } else {
      ld<C>(v.x + i0, acc);                        // x.Axpy(V_i, y_i) ...
    }
    for (int i = 0; i <= k; ++i) {
      const T yi = (T)__ldg(v.y + i);
      ld<C>(v.V + i * v.ldv + i0, t);
#pragma unroll
      for (int q = 0; q < C; ++q) acc[q] = fma(yi, t[q], acc[q]);
    }
    if (PRE) {  // w = z .* inv_D; x.Axpy(w, 1)
      T xv[C], d[C];
      ld<C>(v.x + i0, xv);
      ld<C>(v.invd + i0, d);
#pragma unroll
      for (int q = 0; q < C; ++q) xv[q] = xv[q] + acc[q] * d[q];
      st<C>(v.x + i0, xv);
    } else {
      st<C>(v.x + i0, acc);
    }
  });
}

// ---- G2: (re)start V0 = (b - A x) / res, z = P V0 ----------------------------------
template <typename T, bool PRE> struct RestartV0Emit {
  GmBufs<T> v;
  T inv_res;
  __device__ __forceinline__ void operator()(int row, T y) {
    const T r = (v.b[row] - y) * inv_res;  // V0 = b - A x; V0.Scale(1 / res)
    v.V[row] = r;
    if (PRE) v.z[row] = r * v.invd[row];
  }
};

template <typename Op, typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) gm_restart_kernel(Op op, GmBufs<T> v, double *part, GmScalars *sc) {
  const int phase = __ldg(&sc->phase);
  const int state = __ldg(&sc->state);
  if (phase == kGmUpdate && state != B200LA_ITERATE) {
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->phase = kGmDone;  // every block does nothing here
    return;
  }
  if (phase != kGmRestart && phase != kGmUpdate) return;
  const T res = (T)__ldg(&sc->res);
  RestartV0Emit<T, PRE> e{v, T(1) / res};
  op.run(v.x, e);
  double s[1] = {0.0};
  if (grid_sum_last<1>(s, part, &sc->ticket[1])) {
    // the last block: a fresh cycle (H = 0, g = (res, 0, ...))
    const int m = sc->m, ldh = m + 1;
    for (int i = threadIdx.x; i < m * ldh; i += blockDim.x) v.H[i] = 0.0;
    for (int i = threadIdx.x; i < ldh; i += blockDim.x) v.g[i] = i == 0 ? (double)res : 0.0;
    if (threadIdx.x == 0) {
      sc->j = 0;
      sc->phase = kGmStep;
    }
  }
}

// ---- G3: w = A z, partial sums of w.V0 ---------------------------------------------
template <typename T> struct ArnoldiSpmvEmit {
  T *__restrict__ w;
  const T *__restrict__ v0;
  Acc<T> acc;
  __device__ __forceinline__ void operator()(int row, T y) {
    w[row] = y;
    acc.add(y * v0[row]);
  }
};

template <typename Op, typename T, bool PRE>
__global__ void __launch_bounds__(kBlock) gm_spmv_kernel(Op op, GmBufs<T> v, double *part3, GmScalars *sc) {
  if (__ldg(&sc->phase) != kGmStep) return;
  const int j = __ldg(&sc->j);
  ArnoldiSpmvEmit<T> e{v.w, v.V};
  op.run(PRE ? v.z : v.V + j * v.ldv, e);
  double s[1] = {e.acc.value()};
  __shared__ double red[32];
  block_sum<1>(s, red);
  if (threadIdx.x == 0) part3[blockIdx.x] = s[0];
}

// Sum of count partials in a fixed order (all threads of the block take part;
// the total is returned in every thread).
__device__ __forceinline__ double block_total(const double *part, int count) {
  __shared__ double red[32];
  __shared__ double total;
  double v[1] = {0.0};
  for (int i = threadIdx.x; i < count; i += blockDim.x) v[0] += __ldcg(part + i);
  block_sum<1>(v, red);
  if (threadIdx.x == 0) total = v[0];
  __syncthreads();
  const double t = total;
  __syncthreads();
  return t;
}

// Givens rotation of (dx, dy) by (cs, sn) (gmres.h:97-103).
__device__ __forceinline__ void gm_rotate(double cs, double sn, double *dx, double *dy) {
  const double temp = cs * (*dx) + sn * (*dy);
  *dy = -sn * (*dx) + cs * (*dy);
  *dx = temp;
}

// ---- G4: the Arnoldi step (cooperative launch: every block resident) -------------
// A pass outside an Arnoldi step only advances the guard and the loop
// condition (lead thread).
template <bool IN_GRAPH>
__device__ __forceinline__ void gm_idle(GmScalars *sc, int phase, cudaGraphConditionalHandle loop) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int g = sc->guard + 1;
    sc->guard = g;
    const bool go = phase != kGmDone;
    if (IN_GRAPH) cudaGraphSetConditional(loop, go ? 1u : 0u);
  }
}

// A grid barrier wait ran out (no block should ever be missing under a
// cooperative launch): end the solve, and clear the loop condition from the
// lead thread, which fails the same barrier.
template <bool IN_GRAPH>
__device__ __forceinline__ void gm_abort(GmScalars *sc, cudaGraphConditionalHandle loop) {
  if (threadIdx.x == 0) {
    sc->state = B200LA_FAIL_BREAKDOWN;
    sc->phase = kGmDone;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && IN_GRAPH) cudaGraphSetConditional(loop, 0u);
}

// Block 0's end of step j (all its threads): H(j, j+1) = ||w||, the Givens
// rotations, the test, at a cycle end the back substitution H y = g, then the
// guard and the loop condition.
template <bool IN_GRAPH>
__device__ __noinline__ void gm_step_end(double *H, double *g, double *cs, double *sn, double *y, GmScalars *sc, int j, int m,
                            double hn, cudaGraphConditionalHandle loop) {
  __shared__ double ysh[kMaxBasis + 1];
  __shared__ int finish;
  const int ldh = m + 1;
  if (threadIdx.x == 0) {
    double *Hj = H + j * ldh;
    Hj[j + 1] = hn;
    for (int k = 0; k != j; ++k) gm_rotate(cs[k], sn[k], &Hj[k], &Hj[k + 1]);
    const double dx = Hj[j], dy = Hj[j + 1];
    const double beta = sqrt(dx * dx + dy * dy);
    cs[j] = dx / beta;
    sn[j] = dy / beta;
    gm_rotate(cs[j], sn[j], &Hj[j], &Hj[j + 1]);
    gm_rotate(cs[j], sn[j], &g[j], &g[j + 1]);
    const double res = fabs(g[j + 1]);
    const int it = sc->iter + 1;
    sc->iter = it;
    sc->res = res;
    const int st8 = gm_check(it, res, *sc);
    sc->state = st8;
    finish = (st8 != B200LA_ITERATE || j + 1 == m) ? 1 : 0;
    if (!finish) sc->j = j + 1;
  }
  __syncthreads();
  if (finish) {
    // UpdateSolution's back substitution (gmres.h:731-740): the per-element
    // order of the reference (i descending) with the j < i updates in parallel
    for (int i = threadIdx.x; i <= j; i += blockDim.x) ysh[i] = g[i];
    __syncthreads();
    for (int i = j; i >= 0; --i) {
      if (threadIdx.x == 0) ysh[i] /= H[i * ldh + i];
      __syncthreads();
      const double temp = ysh[i];
      for (int q = threadIdx.x; q < i; q += blockDim.x) ysh[q] -= H[i * ldh + q] * temp;
      __syncthreads();
    }
    for (int i = threadIdx.x; i <= j; i += blockDim.x) y[i] = ysh[i];
    if (threadIdx.x == 0) {
      sc->kend = j;
      sc->phase = kGmUpdate;
    }
  }
  if (threadIdx.x == 0) {
    // one pass per Arnoldi step (G1 and G2 ride along in the next pass), so
    // IterateControl's maxits ends the loop first; the bound only guards
    // against a broken reduction
    const int gd = sc->guard + 1;
    sc->guard = gd;
    bool go = true;
    if (gd > sc->maxits + 4) {
      sc->state = B200LA_FAIL_BREAKDOWN;
      sc->phase = kGmDone;
      go = false;
    }
    if (IN_GRAPH) cudaGraphSetConditional(loop, go ? 1u : 0u);
  }
}

// Streaming form, for any n: w lives in global memory (the L2 keeps most of
// it).  part4 holds [2][gridDim.x] partial sums, by parity of i, so a block
// that is one barrier ahead never overwrites partials another block still adds.
template <typename T, bool PRE, bool IN_GRAPH>
__global__ void __launch_bounds__(kBlock) gm_arnoldi_kernel(GmBufs<T> v, const double *part3, int n3, double *part4,
                                                            GmScalars *sc, cudaGraphConditionalHandle loop) {
  __shared__ double red[32];
  const int phase = __ldg(&sc->phase);
  if (phase != kGmStep) {
    gm_idle<IN_GRAPH>(sc, phase, loop);
    return;
  }
  const int j = __ldg(&sc->j);
  const int m = __ldg(&sc->m), ldh = m + 1;
  const unsigned long long bar0 = __ldg(&sc->bar_done);
  T *vj1 = v.V + (int64_t)(j + 1) * v.ldv;
  // h_0j from G3's partials; then for each i: w -= h_ij V_i, fused with the
  // next dot (w.V_{i+1}, or w.w after the last i)
  double h = block_total(part3, n3);
  for (int i = 0; i <= j; ++i) {
    if (blockIdx.x == 0 && threadIdx.x == 0) v.H[j * ldh + i] = h;
    const T hi = (T)h;
    const T *vi = v.V + (int64_t)i * v.ldv;
    const T *vn = i < j ? v.V + (int64_t)(i + 1) * v.ldv : nullptr;
    Acc<T> acc;
    for_each_chunk<T>(v.n, [&](int64_t e, auto cc) {
      constexpr int C = decltype(cc)::value;
      T wv[C], a[C], bnext[C];
      ld<C>(v.w + e, wv);
      ld<C>(vi + e, a);
      if (vn) ld<C>(vn + e, bnext);
#pragma unroll
      for (int q = 0; q < C; ++q) {
        wv[q] = fma(-hi, a[q], wv[q]);
        acc.add(wv[q] * (vn ? bnext[q] : wv[q]));
      }
      st<C>(v.w + e, wv);
    });
    double s[1] = {acc.value()};
    block_sum<1>(s, red);
    double *slot = part4 + (i & 1) * gridDim.x;
    if (threadIdx.x == 0) slot[blockIdx.x] = s[0];
    if (!grid_barrier_count(&sc->bar_count, (bar0 + (unsigned long long)i + 1ull) * gridDim.x, &sc->err)) {
      gm_abort<IN_GRAPH>(sc, loop);
      return;
    }
    h = block_total(slot, gridDim.x);
  }
  // h = w.w: H(j, j+1) = ||w||, V_{j+1} = w / ||w||, z = P V_{j+1}
  const T hn = sqrt((T)h);
  const T inv = T(1) / hn;
  for_each_chunk<T>(v.n, [&](int64_t e, auto cc) {
    constexpr int C = decltype(cc)::value;
    T wv[C], d[C];
    ld<C>(v.w + e, wv);
    if (PRE) ld<C>(v.invd + e, d);
#pragma unroll
    for (int q = 0; q < C; ++q) {
      wv[q] = wv[q] * inv;
      if (PRE) d[q] = wv[q] * d[q];
    }
    st<C>(vj1 + e, wv);
    if (PRE) st<C>(v.z + e, d);
  });
  if (blockIdx.x != 0) return;
  if (threadIdx.x == 0) sc->bar_done = bar0 + (unsigned long long)j + 1ull;
  gm_step_end<IN_GRAPH>(v.H, v.g, v.cs, v.sn, v.y, sc, j, m, (double)hn, loop);
}

// Resident form: one block of kResBlock threads per SM, block b owning the
// slice [b S, b S + S) of w (S a multiple of the 16-byte vector) in shared
// memory for the whole step.  w is read from global memory once (G3 wrote
// it) and V_{j+1} (and z) written once at the end; in between, projection i
// reads only V_i, already in L2 since projection i-1's dot, and V_{i+1},
// which projection i-1 prefetched into L2 before its grid barrier, so the
// barrier's wait overlaps the DRAM read.  Each thread owns the 16-byte
// chunks k = threadIdx.x + t kResBlock of the slice in every pass (so the
// slice needs no block barrier of its own) and walks them kResUnroll at a
// time, loads first, to keep that many loads in flight.  Same arithmetic per
// element as the streaming form, and the same per-thread order; only the
// partition of the dot products into partial sums differs.  (Measured on
// the 2.1 M-row Poisson matrix: 1024 threads with 2 loads in flight beat
// 1024 x 1 and 512 x 4, and a barrier-free all-gather of tagged partials
// was slower than this barrier.)
constexpr int kResBlock = 1024;
constexpr int kResUnroll = 2;

// The end of one projection in the resident kernel: the block's partial
// (the threads' v summed) goes to set[blockIdx.x]; after the grid barrier
// warp 0 adds the gridDim partials in the same order in every block (lane l:
// blocks l, l + 32, ..., then a shuffle tree), so all blocks hold the same
// total.  Two block barriers in all (the block sum, the barrier wait and the
// re-read of the partials each took their own before).  Returns false in
// every thread when a wait ran out.
__device__ __forceinline__ bool projection_total(double v, double *set, unsigned long long *count,
                                                 unsigned long long target, unsigned *err, double *out) {
  __shared__ double red[32];
  __shared__ double tot;
  __shared__ int okf;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = warp_sum(lane < nw ? red[lane] : 0.0);
    int good = 1;
    if (lane == 0) {
      set[blockIdx.x] = t;
      __threadfence();
      if (atomicAdd(count, 1ull) + 1ull < target) {
        long long spins = 0;
        while (ld_relaxed_u64(count) < target) {
          ++spins;
          if (spins > kSpinLimit || ((spins & 63) == 0 && ld_relaxed_u32(err) != 0u)) {
            atomicExch(err, 1u);
            good = 0;
            break;
          }
          __nanosleep(32);
        }
      }
      __threadfence();
    }
    good = __shfl_sync(0xffffffffu, good, 0);
    double a = 0.0;
    if (good) {
      for (int b = lane; b < (int)gridDim.x; b += 32) a += __ldcg(set + b);
      a = warp_sum(a);
    }
    if (lane == 0) {
      tot = a;
      okf = good;
    }
  }
  __syncthreads();
  *out = tot;
  return okf != 0;
}

template <typename T>
__device__ __forceinline__ void prefetch_slice_l2(const T *p, int64_t len) {
  const char *c = reinterpret_cast<const char *>(p);
  const int64_t bytes = len * (int64_t)sizeof(T);
  for (int64_t o = (int64_t)threadIdx.x * 128; o < bytes; o += (int64_t)blockDim.x * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(c + o));
}

template <typename T, bool PRE, bool IN_GRAPH>
__global__ void __launch_bounds__(kResBlock, 1) gm_arnoldi_res_kernel(GmBufs<T> v, const double *part3, int n3,
                                                                      double *part4, GmScalars *sc, int64_t S,
                                                                      cudaGraphConditionalHandle loop) {
  constexpr int W = Vec16<T>::n, U = kResUnroll;
  extern __shared__ __align__(16) unsigned char gm_dyn[];
  T *ws = reinterpret_cast<T *>(gm_dyn);
  const int phase = __ldg(&sc->phase);
  if (phase != kGmStep) {
    gm_idle<IN_GRAPH>(sc, phase, loop);
    return;
  }
  const int j = __ldg(&sc->j);
  const int m = __ldg(&sc->m), ldh = m + 1;
  const int64_t lo = (int64_t)blockIdx.x * S;
  const int64_t len = lo < v.n ? (v.n - lo < S ? v.n - lo : S) : 0;
  const int64_t nv = len / W;               // whole chunks; elements nv W .. len-1 are the tail
  const int64_t bd = blockDim.x;
  const bool stall = (int)blockIdx.x == __ldg(&sc->stall_block);
  const unsigned long long bar0 = __ldg(&sc->bar_done);
  prefetch_slice_l2(v.V + lo, len);
  if (j > 0) prefetch_slice_l2(v.V + v.ldv + lo, len);
  // w's slice into shared memory
  for (int64_t k0 = threadIdx.x; k0 < nv; k0 += U * bd) {
    T t[U][W];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (k0 + u * bd < nv) ld<W>(v.w + lo + (k0 + u * bd) * W, t[u]);
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (k0 + u * bd < nv) st<W>(ws + (k0 + u * bd) * W, t[u]);
  }
  for (int64_t e = nv * W + threadIdx.x; e < len; e += bd) ws[e] = v.w[lo + e];
  double h = block_total(part3, n3);
  for (int i = 0; i <= j; ++i) {
    if (blockIdx.x == 0 && threadIdx.x == 0) v.H[j * ldh + i] = h;
    const T hi = (T)h;
    const T *vi = v.V + (int64_t)i * v.ldv + lo;
    const T *vn = i < j ? v.V + (int64_t)(i + 1) * v.ldv + lo : nullptr;
    Acc<T> acc;
    for (int64_t k0 = threadIdx.x; k0 < nv; k0 += U * bd) {
      T a[U][W], bn[U][W];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t k = k0 + u * bd;
        if (k < nv) {
          ld<W>(vi + k * W, a[u]);
          if (vn) ld<W>(vn + k * W, bn[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t k = k0 + u * bd;
        if (k < nv) {
          T wv[W];
          ld<W>(ws + k * W, wv);
#pragma unroll
          for (int q = 0; q < W; ++q) {
            wv[q] = fma(-hi, a[u][q], wv[q]);
            acc.add(wv[q] * (vn ? bn[u][q] : wv[q]));
          }
          st<W>(ws + k * W, wv);
        }
      }
    }
    for (int64_t e = nv * W + threadIdx.x; e < len; e += bd) {
      const T wv = fma(-hi, vi[e], ws[e]);
      acc.add(wv * (vn ? vn[e] : wv));
      ws[e] = wv;
    }
    if (i + 2 <= j) prefetch_slice_l2(v.V + (int64_t)(i + 2) * v.ldv + lo, len);
    if (stall) return;  // test hook: this block never reaches the barrier
    if (!projection_total(acc.value(), part4 + (i & 1) * gridDim.x, &sc->bar_count,
                          (bar0 + (unsigned long long)i + 1ull) * gridDim.x, &sc->err, &h)) {
      gm_abort<IN_GRAPH>(sc, loop);
      return;
    }
  }
  // V_{j+1} = w / ||w||, z = P V_{j+1}
  const T hn = sqrt((T)h);
  const T inv = T(1) / hn;
  T *vj1 = v.V + (int64_t)(j + 1) * v.ldv + lo;
  for (int64_t k0 = threadIdx.x; k0 < nv; k0 += U * bd) {
    T d[U][W];
    if (PRE) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (k0 + u * bd < nv) ld<W>(v.invd + lo + (k0 + u * bd) * W, d[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t k = k0 + u * bd;
      if (k < nv) {
        T wv[W];
        ld<W>(ws + k * W, wv);
#pragma unroll
        for (int q = 0; q < W; ++q) {
          wv[q] = wv[q] * inv;
          if (PRE) d[u][q] = wv[q] * d[u][q];
        }
        st<W>(vj1 + k * W, wv);
        if (PRE) st<W>(v.z + lo + k * W, d[u]);
      }
    }
  }
  for (int64_t e = nv * W + threadIdx.x; e < len; e += bd) {
    const T wv = ws[e] * inv;
    vj1[e] = wv;
    if (PRE) v.z[lo + e] = wv * v.invd[lo + e];
  }
  if (blockIdx.x != 0) return;
  // every block read bar_done at its start, and block 0 gets here only after
  // all arrived at barrier j
  if (threadIdx.x == 0) sc->bar_done = bar0 + (unsigned long long)j + 1ull;
  gm_step_end<IN_GRAPH>(v.H, v.g, v.cs, v.sn, v.y, sc, j, m, (double)hn, loop);
}

}  // namespace b200la

using namespace b200la;

namespace b200la {

struct GmresState {
  b200la_mat A;
  b200la_ctx ctx;            // kept for destroy, which may come after A's
  b200la_solver_params prm;
  int64_t n, ldv;
  int m;
  void *V, *w, *z, *x, *bown, *invd;
  double *arrays;            // H [m][m+1], g, cs, sn, y [m+1] each
  double *part, *part3, *part4;
  GmScalars *sc, *sc_host;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int g_format, g_param;     // schedule baked into the graph
  int g_gen;                 // the matrix's schedule generation at capture
  int grid_start, grid_restart, grid_spmv, grid_ew, grid_coop;
  int grid_res;              // blocks of the resident Arnoldi kernel (0: streaming form)
  int64_t res_slice;         // elements of w per block there
};

template <typename T> static GmBufs<T> gm_bufs(const GmresState *s) {
  const int ld = s->m + 1;
  double *H = s->arrays;
  double *g = H + (size_t)s->m * ld;
  return GmBufs<T>{(T *)s->V, s->ldv, (T *)s->w, (T *)s->z, (T *)s->x, (const T *)s->bown, (const T *)s->invd,
                   H, g, g + ld, g + 2 * ld, g + 3 * ld, s->n};
}

// The Arnoldi kernel as a cooperative launch (all blocks resident, which its
// grid barrier needs), captured into the graph like any kernel node.
template <typename T, bool PRE, bool IN_GRAPH>
static int gm_launch_arnoldi(GmresState *s, cudaStream_t st, cudaGraphConditionalHandle h) {
  cudaLaunchConfig_t cfg = {};
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const GmBufs<T> v = gm_bufs<T>(s);
  if (s->grid_res > 0) {
    cfg.gridDim = dim3((unsigned)s->grid_res);
    cfg.blockDim = dim3(kResBlock);
    cfg.dynamicSmemBytes = (size_t)s->res_slice * sizeof(T);
    B_CUDA(cudaLaunchKernelEx(&cfg, gm_arnoldi_res_kernel<T, PRE, IN_GRAPH>, v, (const double *)s->part3,
                              s->grid_spmv, s->part4, s->sc, s->res_slice, h));
    return B200LA_OK;
  }
  cfg.gridDim = dim3((unsigned)s->grid_coop);
  cfg.blockDim = dim3(kBlock);
  cfg.dynamicSmemBytes = 0;
  B_CUDA(cudaLaunchKernelEx(&cfg, gm_arnoldi_kernel<T, PRE, IN_GRAPH>, v, (const double *)s->part3, s->grid_spmv,
                            s->part4, s->sc, h));
  return B200LA_OK;
}

// Sizes the resident Arnoldi kernel: one block per SM at most, each holding
// its slice of w in shared memory.  Leaves grid_res = 0 (the streaming form)
// when the slice does not fit, when a block cannot be resident, or when
// B200LA_GMRES_RESIDENT=0 is in the environment.
template <typename T, bool PRE>
static int gm_size_resident(GmresState *s) {
  s->grid_res = 0;
  s->res_slice = 0;
  const char *env = getenv("B200LA_GMRES_RESIDENT");
  if (env && env[0] == '0') return B200LA_OK;
  b200la_ctx c = s->A->ctx;
  constexpr int W = Vec16<T>::n;
  const int64_t want = (s->n + (int64_t)kResBlock * W - 1) / ((int64_t)kResBlock * W);
  const int grid = (int)(want < c->num_sms ? (want < 1 ? 1 : want) : c->num_sms);
  int64_t S = (s->n + grid - 1) / grid;
  S = (S + W - 1) / W * W;
  int optin = 0;
  B_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
  const void *kern[2] = {(const void *)gm_arnoldi_res_kernel<T, PRE, true>,
                         (const void *)gm_arnoldi_res_kernel<T, PRE, false>};
  const int64_t bytes = S * (int64_t)sizeof(T);
  for (const void *k : kern) {
    cudaFuncAttributes fa;
    B_CUDA(cudaFuncGetAttributes(&fa, k));
    if (bytes + (int64_t)fa.sharedSizeBytes > (int64_t)optin) return B200LA_OK;
  }
  for (const void *k : kern) {
    B_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    int per_sm = 0;
    B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kResBlock, (size_t)bytes));
    if (per_sm < 1) return B200LA_OK;
  }
  s->grid_res = grid;
  s->res_slice = S;
  return B200LA_OK;
}

template <typename T, bool PRE, bool IN_GRAPH>
static int gm_body_t(GmresState *s, cudaStream_t st, cudaGraphConditionalHandle h) {
  const GmBufs<T> v = gm_bufs<T>(s);
  gm_update_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->sc);
  B_TRY(with_schedule<T>(s->A, [&](auto op) -> int {
    using Op = decltype(op);
    gm_restart_kernel<Op, T, PRE><<<s->grid_restart, kBlock, 0, st>>>(op, v, s->part, s->sc);
    gm_spmv_kernel<Op, T, PRE><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part3, s->sc);
    return B200LA_OK;
  }));
  return gm_launch_arnoldi<T, PRE, IN_GRAPH>(s, st, h);
}

template <typename T, bool PRE>
static int gm_grids_t(GmresState *s) {
  b200la_ctx c = s->A->ctx;
  B_TRY(grid_for(c, (const void *)gm_update_kernel<T, PRE>, (s->n + Vec16<T>::n - 1) / Vec16<T>::n, kBlock,
                 &s->grid_ew));
  B_TRY(with_schedule<T>(s->A, [&](auto op) -> int {
    using Op = decltype(op);
    B_TRY(grid_for(c, (const void *)gm_start_kernel<Op, T>, op.work_items(), Op::kRowsPerBlock, &s->grid_start));
    B_TRY(grid_for(c, (const void *)gm_restart_kernel<Op, T, PRE>, op.work_items(), Op::kRowsPerBlock,
                   &s->grid_restart));
    B_TRY(grid_for(c, (const void *)gm_spmv_kernel<Op, T, PRE>, op.work_items(), Op::kRowsPerBlock,
                   &s->grid_spmv));
    return B200LA_OK;
  }));
  // every block of the cooperative kernel must be resident at once
  int per_sm = 0;
  B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gm_arnoldi_kernel<T, PRE, true>, kBlock, 0));
  int per_sm2 = 0;
  B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, gm_arnoldi_kernel<T, PRE, false>, kBlock, 0));
  per_sm = per_sm < per_sm2 ? per_sm : per_sm2;
  B_CHECK(per_sm >= 1, B200LA_ERR_CUDA, "gmres: the Arnoldi kernel cannot be resident");
  int64_t need = (s->n + (int64_t)kBlock * Vec16<T>::n - 1) / ((int64_t)kBlock * Vec16<T>::n);
  int64_t cap = (int64_t)c->num_sms * per_sm;
  if (cap > kMaxReduceBlocks) cap = kMaxReduceBlocks;
  s->grid_coop = (int)(need < 1 ? 1 : (need < cap ? need : cap));
  return gm_size_resident<T, PRE>(s);
}

template <typename T, bool PRE>
static int gm_build_graph_t(GmresState *s) {
  b200la_mat A = s->A;
  B_TRY((gm_grids_t<T, PRE>(s)));
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
  int rc = gm_body_t<T, PRE, true>(s, cs, h);
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

static int gm_build_graph(GmresState *s) {
  const bool pre = s->prm.precond != 0;
  if (s->A->dtype == B200LA_F64) return pre ? gm_build_graph_t<double, true>(s) : gm_build_graph_t<double, false>(s);
  return pre ? gm_build_graph_t<float, true>(s) : gm_build_graph_t<float, false>(s);
}

static int gm_fetch(GmresState *s, GmScalars *out) {
  cudaStream_t st = s->A->ctx->stream;
  B_CUDA(cudaMemcpyAsync(s->sc_host, s->sc, sizeof(GmScalars), cudaMemcpyDeviceToHost, st));
  B_CUDA(cudaStreamSynchronize(st));
  *out = *s->sc_host;
  return B200LA_OK;
}

static GmScalars gm_initial(const GmresState *s) {
  GmScalars init = {};
  init.atol = s->prm.atol;
  init.rtol = s->prm.rtol;
  init.dtol = s->prm.dtol;
  init.maxits = s->prm.maxits;
  init.m = s->m;
  init.state = B200LA_ITERATE;
  init.phase = kGmDone;
  // B200LA_TEST_STALL_BARRIER=b makes block b of the resident Arnoldi
  // kernel leave before its first grid barrier, so that the other blocks'
  // waits run out: the solve then ends with B200LA_ERR_TIMEOUT and the
  // context stays usable (the failure-path test; never set in normal use)
  const char *stall = getenv("B200LA_TEST_STALL_BARRIER");
  init.stall_block = stall && stall[0] ? atoi(stall) : -1;
  return init;
}

// Copies x, b in, resets the scalars and runs the start kernel.
template <typename T>
static int gm_begin_t(GmresState *s, const void *b_dev, const void *x_dev) {
  cudaStream_t st = s->A->ctx->stream;
  const size_t vb = (size_t)s->n * sizeof(T);
  const GmScalars init = gm_initial(s);
  B_CUDA(cudaMemcpyAsync(s->sc, &init, sizeof(init), cudaMemcpyHostToDevice, st));
  B_CUDA(cudaMemcpyAsync(s->bown, b_dev, vb, cudaMemcpyDeviceToDevice, st));
  B_CUDA(cudaMemcpyAsync(s->x, x_dev, vb, cudaMemcpyDeviceToDevice, st));
  const GmBufs<T> v = gm_bufs<T>(s);
  return with_schedule<T>(s->A, [&](auto op) -> int {
    using Op = decltype(op);
    gm_start_kernel<Op, T><<<s->grid_start, kBlock, 0, st>>>(op, v, s->part, s->sc);
    B_CUDA(cudaGetLastError());
    return B200LA_OK;
  });
}

template <typename T, bool PRE>
static int gm_host_loop_t(GmresState *s) {
  cudaStream_t st = s->A->ctx->stream;
  for (int64_t pass = 0;; pass += 16) {
    for (int k = 0; k < 16; ++k) B_TRY((gm_body_t<T, PRE, false>(s, st, 0)));
    B_CUDA(cudaGetLastError());
    GmScalars h;
    B_TRY(gm_fetch(s, &h));
    if (h.phase == kGmDone || pass > (int64_t)s->prm.maxits + 64) break;
  }
  return B200LA_OK;
}

template <typename T, bool PRE>
static int gm_profile_t(GmresState *s, const void *b_dev, const void *x_dev, int passes, double *ms) {
  cudaStream_t st = s->A->ctx->stream;
  B_TRY(gm_begin_t<T>(s, b_dev, x_dev));
  const GmBufs<T> v = gm_bufs<T>(s);
  // every pass is queued before the first wait, so the timed kernels run
  // back to back and no host launch gap falls between an event pair (the
  // first pass starts behind the start kernel)
  std::vector<cudaEvent_t> ev((size_t)(passes > 0 ? passes : 0) * 5);
  for (auto &e : ev) B_CUDA(cudaEventCreate(&e));
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  int rc = B200LA_OK;
  for (int it = 0; it < passes && rc == B200LA_OK; ++it) {
    cudaEvent_t *e = &ev[(size_t)it * 5];
    cudaEventRecord(e[0], st);
    gm_update_kernel<T, PRE><<<s->grid_ew, kBlock, 0, st>>>(v, s->sc);
    cudaEventRecord(e[1], st);
    rc = with_schedule<T>(s->A, [&](auto op) -> int {
      using Op = decltype(op);
      gm_restart_kernel<Op, T, PRE><<<s->grid_restart, kBlock, 0, st>>>(op, v, s->part, s->sc);
      cudaEventRecord(e[2], st);
      gm_spmv_kernel<Op, T, PRE><<<s->grid_spmv, kBlock, 0, st>>>(op, v, s->part3, s->sc);
      cudaEventRecord(e[3], st);
      return B200LA_OK;
    });
    if (rc == B200LA_OK) rc = gm_launch_arnoldi<T, PRE, false>(s, st, 0);
    cudaEventRecord(e[4], st);
  }
  const cudaError_t se = cudaStreamSynchronize(st);
  for (int it = 0; it < passes && rc == B200LA_OK && se == cudaSuccess; ++it)
    for (int k = 0; k < 4; ++k) {
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[(size_t)it * 5 + k], ev[(size_t)it * 5 + k + 1]);
      acc[k] += t;
    }
  for (auto &e : ev) cudaEventDestroy(e);
  B_CUDA(se);
  B_CUDA(cudaGetLastError());
  for (int k = 0; k < 4; ++k) ms[k] = passes > 0 ? acc[k] / passes : 0.0;
  return rc;
}

void gmres_destroy(GmresState *s) {
  if (!s) return;
  cudaStream_t st = s->ctx->stream;
  cudaStreamSynchronize(st);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  void *bufs[] = {s->V, s->w, s->z, s->x, s->bown, s->invd, s->arrays, s->part, s->part3, s->part4, s->sc};
  for (void *b : bufs)
    if (b) cudaFreeAsync(b, st);
  if (s->sc_host) cudaFreeHost(s->sc_host);
  delete s;
}

int gmres_create(b200la_mat A, const b200la_solver_params *prm, GmresState **out) {
  B_CHECK(prm->size_basis >= 1 && prm->size_basis <= kMaxBasis, B200LA_ERR_INVALID,
          "solver_create: GMRES basis size %d not in [1, %d]", prm->size_basis, kMaxBasis);
  b200la_ctx c = A->ctx;
  cudaStream_t st = c->stream;
  GmresState *s = new GmresState();
  s->A = A;
  s->ctx = c;
  s->prm = *prm;
  s->n = A->nrow;
  s->m = prm->size_basis < prm->maxits ? prm->size_basis : prm->maxits;
  if (s->m < 1) s->m = 1;
  const size_t es = dtype_size(A->dtype);
  const int64_t align = 256 / (int64_t)es;
  s->ldv = ((s->n > 0 ? s->n : 1) + align - 1) / align * align;
  const size_t vb = es * (size_t)s->ldv;
  auto cleanup = [&](int code) { gmres_destroy(s); return code; };
  const int ld = s->m + 1;
  if (cudaMallocAsync(&s->V, vb * (size_t)(s->m + 1), st) != cudaSuccess)
    return cleanup(fail(B200LA_ERR_NOMEM, "solver_create: GMRES basis of %d x %zu bytes does not fit", s->m + 1, vb));
  if (cudaMallocAsync(&s->w, vb, st) != cudaSuccess || cudaMallocAsync(&s->z, vb, st) != cudaSuccess ||
      cudaMallocAsync(&s->x, vb, st) != cudaSuccess || cudaMallocAsync(&s->bown, vb, st) != cudaSuccess ||
      cudaMallocAsync(&s->arrays, sizeof(double) * ((size_t)s->m * ld + 4 * (size_t)ld), st) != cudaSuccess ||
      cudaMallocAsync(&s->part, sizeof(double) * kMaxReduceBlocks, st) != cudaSuccess ||
      cudaMallocAsync(&s->part3, sizeof(double) * kMaxReduceBlocks, st) != cudaSuccess ||
      cudaMallocAsync(&s->part4, sizeof(double) * 2 * kMaxReduceBlocks, st) != cudaSuccess ||
      cudaMallocAsync(&s->sc, sizeof(GmScalars), st) != cudaSuccess ||
      cudaMallocHost(&s->sc_host, sizeof(GmScalars)) != cudaSuccess)
    return cleanup(fail(B200LA_ERR_NOMEM, "solver_create: GMRES work space allocation failed"));
  if (cudaMemsetAsync(s->arrays, 0, sizeof(double) * ((size_t)s->m * ld + 4 * (size_t)ld), st) != cudaSuccess)
    return cleanup(fail(B200LA_ERR_CUDA, "solver_create: memset failed"));
  if (prm->precond) {
    if (cudaMallocAsync(&s->invd, vb, st) != cudaSuccess)
      return cleanup(fail(B200LA_ERR_NOMEM, "solver_create: allocation of the inverse diagonal failed"));
    b200la_vec_s dv{c, s->n, A->dtype, s->invd, false};
    const int rc = b200la_mat_inv_diag(A, &dv);
    if (rc != B200LA_OK) return cleanup(rc);
  }
  if (s->n > 0) {
    const int rc = gm_build_graph(s);
    if (rc != B200LA_OK) return cleanup(rc);
  }
  *out = s;
  return B200LA_OK;
}

int gmres_solve(GmresState *s, b200la_vec b, b200la_vec x, b200la_solver_result *res) {
  b200la_mat A = s->A;
  memset(res, 0, sizeof(*res));
  if (s->n == 0) {
    res->state = B200LA_SUCCESS_ABS;
    return B200LA_OK;
  }
  cudaStream_t st = A->ctx->stream;
  const bool pre = s->prm.precond != 0;
  if (A->dtype == B200LA_F64) B_TRY(gm_begin_t<double>(s, b->d, x->d));
  else B_TRY(gm_begin_t<float>(s, b->d, x->d));
  if (A->ctx->use_graphs) {
    if (A->format != s->g_format || A->param != s->g_param || A->sched_gen != s->g_gen) B_TRY(gm_build_graph(s));
    B_CUDA(cudaGraphLaunch(s->exec, st));
  } else if (A->dtype == B200LA_F64) {
    B_TRY((pre ? gm_host_loop_t<double, true>(s) : gm_host_loop_t<double, false>(s)));
  } else {
    B_TRY((pre ? gm_host_loop_t<float, true>(s) : gm_host_loop_t<float, false>(s)));
  }
  GmScalars h;
  B_TRY(gm_fetch(s, &h));
  B_CUDA(cudaMemcpyAsync(x->d, s->x, (size_t)s->n * dtype_size(A->dtype), cudaMemcpyDeviceToDevice, st));
  B_CUDA(cudaStreamSynchronize(st));
  B_CHECK(h.err == 0, B200LA_ERR_TIMEOUT, "gmres: a wait of the Arnoldi kernel ran out");
  res->iters = h.iter;
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

int gmres_profile(GmresState *s, b200la_vec b, b200la_vec x, int passes, double *ms) {
  const bool pre = s->prm.precond != 0;
  if (s->A->dtype == B200LA_F64)
    return pre ? gm_profile_t<double, true>(s, b->d, x->d, passes, ms)
               : gm_profile_t<double, false>(s, b->d, x->d, passes, ms);
  return pre ? gm_profile_t<float, true>(s, b->d, x->d, passes, ms)
             : gm_profile_t<float, false>(s, b->d, x->d, passes, ms);
}

}  // namespace b200la
