// Helpers shared by the device solvers of krylov.cu and gmres.cu.
#pragma once

#include <type_traits>

#include "internal.cuh"

namespace b200la {

// Grid-stride loop over [0, n) in 16-byte vectors, then the ragged tail:
// f(i0, C) handles elements i0 .. i0+C-1 (C = Vec16<T>::n or 1, a
// std::integral_constant).  Work vectors start 256-byte aligned.
template <typename T, typename F>
__device__ __forceinline__ void for_each_chunk(int64_t n, F &&f) {
  constexpr int W = Vec16<T>::n;
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t i = tid; i < nv; i += stride) f(i * W, std::integral_constant<int, W>{});
  for (int64_t i = nv * W + tid; i < n; i += stride) f(i, std::integral_constant<int, 1>{});
}

template <int C, typename T> __device__ __forceinline__ void ld(const T *p, T (&a)[C]) {
  if constexpr (C == Vec16<T>::n) {
    using V = typename Vec16<T>::type;
    const V v = *reinterpret_cast<const V *>(p);
    const T *s = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int k = 0; k < C; ++k) a[k] = s[k];
  } else {
#pragma unroll
    for (int k = 0; k < C; ++k) a[k] = p[k];
  }
}

template <int C, typename T> __device__ __forceinline__ void st(T *p, const T (&a)[C]) {
  if constexpr (C == Vec16<T>::n) {
    using V = typename Vec16<T>::type;
    V v;
    T *d = reinterpret_cast<T *>(&v);
#pragma unroll
    for (int k = 0; k < C; ++k) d[k] = a[k];
    *reinterpret_cast<V *>(p) = v;
  } else {
#pragma unroll
    for (int k = 0; k < C; ++k) p[k] = a[k];
  }
}

// Bound on every spin-wait of the cooperative kernels: after kSpinLimit
// polls (a few seconds at most) a waiter gives up and reports an error.
constexpr long long kSpinLimit = 1LL << 22;

__device__ __forceinline__ unsigned ld_relaxed_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier on a monotonic 64-bit arrival counter, for kernels
// launched cooperatively that pass several barriers: every block's thread 0
// adds one and waits (relaxed loads) until the counter reaches `target` =
// gridDim.x times the barriers passed so far including this one, so the last
// arrival itself releases the waiters (no reset, no second counter).  Callers
// derive `target` from a count that all blocks read alike (e.g. kept in
// device memory by the previous launch) and zero the counter when that count
// restarts.  Waits are bounded (kSpinLimit polls, *err checked every 64);
// returns false in every thread of the block after a timeout or when *err is
// set, and the caller ends the kernel.  Must be called by every thread of
// every block.
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ bool grid_barrier_count(unsigned long long *count, unsigned long long target,
                                                   unsigned *err) {
  __shared__ bool ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    bool good = true;
    __threadfence();
    if (atomicAdd(count, 1ull) + 1ull < target) {
      long long spins = 0;
      while (ld_relaxed_u64(count) < target) {
        ++spins;
        if (spins > kSpinLimit || ((spins & 63) == 0 && ld_relaxed_u32(err) != 0u)) {
          atomicExch(err, 1u);
          good = false;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok;
}

// Restarted GMRES (gmres.cu), behind the b200la_solver_* entry points.
struct GmresState;
int gmres_create(b200la_mat A, const b200la_solver_params *prm, GmresState **out);
int gmres_solve(GmresState *s, b200la_vec b, b200la_vec x, b200la_solver_result *res);
int gmres_profile(GmresState *s, b200la_vec b, b200la_vec x, int passes, double *ms);
void gmres_destroy(GmresState *s);

}  // namespace b200la
