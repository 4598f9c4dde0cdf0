// Internal definitions shared by the b200la translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "b200la.h"

namespace b200la {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const char *fmt, ...);

#define B_CUDA(expr)                                                          \
  do {                                                                        \
    cudaError_t e_ = (expr);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return ::b200la::fail(e_ == cudaErrorMemoryAllocation ? B200LA_ERR_NOMEM \
                                                            : B200LA_ERR_CUDA, \
                            "%s:%d %s: %s", __FILE__, __LINE__, #expr,        \
                            cudaGetErrorString(e_));                          \
  } while (0)

#define B_TRY(expr)                                                           \
  do {                                                                        \
    int s_ = (expr);                                                          \
    if (s_ != B200LA_OK) return s_;                                           \
  } while (0)

#define B_CHECK(cond, code, ...)                                              \
  do {                                                                        \
    if (!(cond)) return ::b200la::fail(code, __VA_ARGS__);                    \
  } while (0)

inline size_t dtype_size(int dt) { return dt == B200LA_F64 ? 8 : 4; }
inline bool dtype_ok(int dt) { return dt == B200LA_F64 || dt == B200LA_F32; }

// ---------------------------------------------------------------- handles
constexpr int kBlock = 256;          // threads per block of every kernel here
constexpr int kMaxReduceBlocks = 4096;

// Device scratch of a context: per-block partial sums of the grid
// reductions plus the last-block tickets.
struct ReduceScratch {
  double *part;       // [4][kMaxReduceBlocks]
  unsigned *ticket;   // [16]
  double *result;     // [8]
};

}  // namespace b200la

struct b200la_ctx_s {
  int device;
  int num_sms;
  cudaStream_t own_stream;
  cudaStream_t stream;
  b200la::ReduceScratch scratch;
  double *host_result;  // pinned [8]
  // Device loops run as CUDA-graph WHILE nodes; with B200LA_GRAPHS=0 in the
  // environment the same kernels are launched from a host loop instead, so
  // a profiler can see each launch (ncu does not profile kernels inside
  // graphs with conditional nodes).
  bool use_graphs;
};

struct b200la_vec_s {
  b200la_ctx ctx;
  int64_t n;
  int dtype;
  void *d;
  bool owned;
};

constexpr int kStencilMax = 28;  // stored entries per row of the values-only copy (27 + padding)

struct SellData {
  int nslices = 0;
  int width = 0;        // values per thread per step (1, 2 or 4)
  int64_t padded = 0;   // stored entries incl. padding
  int *slice_ptr = nullptr;  // [nslices+1] offsets in entries
  int *slice_len = nullptr;  // [nslices] padded row length (multiple of width)
  int *col = nullptr;        // int32 columns (col16 == 0)
  short *col16p = nullptr;   // int16 offsets column - row (col16 == 1)
  int col16 = 0;
  void *val = nullptr;
  int *perm = nullptr;       // row of each sorted position (sigma sorting; nullptr: rows keep their order)
  int c = 32;                // rows per slice (SELL-C-sigma's C: 8, 16 or 32)
  int log2c = 5;
  int sigma = 1;             // rows per sorting window (1: no sorting)
  // values-only copy (B200LA_FMT_STENCIL): every row stores `ell` entries,
  // entry k at column row + soff[k] (clamped into [0, n); value 0 where the
  // row has no entry there); no column storage
  int stencil = 0;
  int ell = 0;
  int soff[kStencilMax] = {};
  int off_lo = 0, off_hi = 0;  // smallest and largest offset
};

struct b200la_mat_s {
  b200la_ctx ctx;
  int nrow, ncol;
  int64_t nnz;
  int dtype;
  int *rowptr;
  int *col;
  void *val;
  int *diag;          // position of the diagonal entry of each row, -1 if none
  int max_row;        // longest row
  int format;         // B200LA_FMT_CSR / B200LA_FMT_SELL
  int param;          // CSR lanes per row / SELL width
  SellData sell;
  int sched_gen;      // bumped whenever the schedule or its device data change (graphs re-capture)
};

namespace b200la {

// Host validation of a CSR structure: rowptr[0] == 0, non-decreasing,
// rowptr[nrow] == nnz, 0 <= col < ncol.  Writes the longest row length.
int validate_csr(int nrow, int ncol, int64_t nnz, const int *rowptr, const int *col, int *max_row);

// Q1 system assembly on the device (assemble.cu).
int64_t q1_rows(int dim, int n);
int64_t q1_nnz(int dim, int n);
int q1_assemble(cudaStream_t st, int num_sms, int dim, int n, uint64_t seed, double sigma, int *rowptr, int *col,
                double *val, double *b);

// Launch helpers
int grid_for(b200la_ctx ctx, const void *kernel, int64_t work_items, int items_per_block,
             int *grid);

// ---------------------------------------------------------------- device helpers
template <typename T> struct Vec16;
template <> struct Vec16<double> { using type = double2; static constexpr int n = 2; };
template <> struct Vec16<float> { using type = float4; static constexpr int n = 4; };

// Accumulator used by every reduction.  double: plain sum.  float: the
// running sum is kept in float with Neumaier compensation (Neumaier 1974,
// "Rundungsfehleranalyse einiger Verfahren zur Summation endlicher Summen"),
// so a float dot accumulates in FP32 with a compensated error term.
template <typename T> struct Acc;
template <> struct Acc<double> {
  double s = 0.0;
  __device__ __forceinline__ void add(double v) { s += v; }
  __device__ __forceinline__ double value() const { return s; }
};
template <> struct Acc<float> {
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void add(float v) {
    float t = s + v;
    if (fabsf(s) >= fabsf(v))
      c += (s - t) + v;
    else
      c += (v - t) + s;
    s = t;
  }
  __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of NV doubles; the totals end up in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem /* [NV*32] */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) smem[k * 32 + warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = lane < nwarps ? smem[k * 32 + lane] : 0.0;
      v[k] = warp_sum(t);
    }
  }
  __syncthreads();
}

// Deterministic grid reduction.  Every block stores its partial sums to
// part[k * gridDim.x + blockIdx.x]; the last block to arrive (ticket) adds
// all partials in a fixed order, so the result does not depend on block
// scheduling.  Returns true in the last block; totals are in v[] of its
// thread 0.  The ticket wraps back to 0 by itself (atomicInc modulus).
template <int NV>
__device__ __forceinline__ bool grid_sum_last(double (&v)[NV], double *part, unsigned *ticket) {
  __shared__ double smem[NV * 32];
  __shared__ bool is_last;
  block_sum<NV>(v, smem);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) part[k * gridDim.x + blockIdx.x] = v[k];
    __threadfence();
    unsigned t = atomicInc(ticket, gridDim.x - 1);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double a = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) a += __ldcg(&part[k * gridDim.x + i]);
    v[k] = a;
  }
  block_sum<NV>(v, smem);
  return true;
}

// Streaming loads for the matrix (read once per SpMV, evict first) and
// read-only cached loads for the gathered vector.
template <typename T> __device__ __forceinline__ T ld_stream(const T *p) { return __ldcs(p); }
template <typename T> __device__ __forceinline__ T ld_keep(const T *p) { return __ldg(p); }

// One row of y = A x computed by a group of G lanes of a warp (G divides 32).
// All 32 lanes must call it (the shuffles use the full mask); lanes whose row
// is out of range pass valid = false and contribute nothing.  The total is
// returned in every lane of the group.
// X is the type of x and of the sum (the stored values T are widened to it:
// FP32 values times FP64 vectors in the mixed-storage inner solve).
template <typename T, int G, typename X = T>
__device__ __forceinline__ X csr_row_group(const int *__restrict__ rowptr, const int *__restrict__ col,
                                           const T *__restrict__ val, const X *__restrict__ x, int row,
                                           bool valid) {
  const int lane = threadIdx.x & (G - 1);
  X sum = X(0);
  if (valid) {
    const int start = __ldg(rowptr + row), end = __ldg(rowptr + row + 1);
#pragma unroll 4
    for (int j = start + lane; j < end; j += G)
      sum = fma((X)ld_stream(val + j), ld_keep(x + ld_stream(col + j)), sum);
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  return sum;
}

}  // namespace b200la
