// SpMV schedules (CSR lane groups, SELL-32 slices) shared by the plain
// VectorMult entry points, the autotuner and the fused CG kernels.
//
// A schedule is an "operator" type with run(x, emit): every thread block
// walks its share of the rows (grid-stride) and calls emit(row, y_row) on
// exactly one lane per row.  The fused kernels pass emitters that also
// accumulate dot products, so the SpMV result never makes an extra trip
// through HBM.
#pragma once

#include "internal.cuh"

namespace b200la {

// ---- CSR, G lanes per row (G = 1..32) -------------------------------------
// Each warp covers 32/G consecutive rows, so a warp's loads of val/col fall
// in one contiguous span of the CSR arrays; x is gathered through L1/L2.
//
// Every schedule takes the stored value type T and the vector type X (x, y
// and the row sums; X = T except in the mixed-storage inner solve, where
// FP32 values meet FP64 vectors and each value is widened before its FMA).
template <typename T, int G, typename X = T> struct CsrOp {
  using XT = X;
  const int *__restrict__ rowptr;
  const int *__restrict__ col;
  const T *__restrict__ val;
  int n;
  static constexpr int kRowsPerBlock = kBlock / G;
  __host__ __device__ int64_t work_items() const { return n; }
  template <typename Emit> __device__ __forceinline__ void run(const X *__restrict__ x, Emit &emit) const {
    for (int base = blockIdx.x * kRowsPerBlock; base < n; base += gridDim.x * kRowsPerBlock) {
      const int row = base + (int)threadIdx.x / G;
      const bool valid = row < n;
      X y = csr_row_group<T, G, X>(rowptr, col, val, x, row, valid);
      if (valid && (threadIdx.x & (G - 1)) == 0) emit(row, y);
    }
  }
};

// ---- SELL-C-sigma ----------------------------------------------------------
// Rows are sorted by length, longest first, within windows of sigma rows
// (perm[position] = row; sigma = 1 keeps the order and perm is null), then
// cut into slices of C rows (C = 8, 16 or 32), each padded to its longest
// row rounded up to W entries.  Entry k of the row at position r of slice s
// sits at slice_ptr[s] + ((k/W)*C + r)*W + k%W: a row's W consecutive
// entries are one vector load, and the C rows of a slice read C*W contiguous
// values per step.  A warp handles 32/C slices at a time (lane = slice in
// the warp * C + r).  Padding entries hold value 0 and repeat a column the
// row already reads.  Every row's products are added in its stored order
// whatever C, sigma and W are, so all SELL variants give the same bits.
template <typename T, int W> struct VecW;
template <> struct VecW<double, 1> { using v = double; using i = int; };
template <> struct VecW<double, 2> { using v = double2; using i = int2; };
template <> struct VecW<double, 4> { using v = double4; using i = int4; };
template <> struct VecW<float, 1> { using v = float; using i = int; };
template <> struct VecW<float, 2> { using v = float2; using i = int2; };
template <> struct VecW<float, 4> { using v = float4; using i = int4; };

template <typename V, typename T, int W> __device__ __forceinline__ T lane_get(const V &v, int k) {
  return reinterpret_cast<const T *>(&v)[k];
}
template <typename I, int W> __device__ __forceinline__ int lane_geti(const I &v, int k) {
  return reinterpret_cast<const int *>(&v)[k];
}

template <typename T> __device__ __forceinline__ double4 ld_stream4(const double4 *p) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
  double2 a = __ldcs(q), b = __ldcs(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

template <typename V> __device__ __forceinline__ V ld_vec_stream(const V *p) { return __ldcs(p); }
template <> __device__ __forceinline__ double4 ld_vec_stream<double4>(const double4 *p) {
  return ld_stream4<double>(p);
}

template <typename T, int W, typename X = T> struct SellOp {
  using XT = X;
  const int *__restrict__ slice_ptr;
  const int *__restrict__ slice_len;
  const int *__restrict__ col;
  const T *__restrict__ val;
  int n, nslices;
  int log2c;                 // C = 1 << log2c rows per slice
  const int *__restrict__ perm;  // row of each position, or null (identity)
  static constexpr int kRowsPerBlock = kBlock;
  __host__ __device__ int64_t work_items() const { return n; }
  template <typename Emit> __device__ __forceinline__ void run(const X *__restrict__ x, Emit &emit) const {
    using VV = typename VecW<T, W>::v;
    using VI = typename VecW<T, W>::i;
    const int lane = threadIdx.x & 31;
    const int wpb = kBlock / 32;
    const int C = 1 << log2c, spw = 32 >> log2c;
    const int r = lane & (C - 1), sub = lane >> log2c;
    for (int s0 = (blockIdx.x * wpb + ((int)threadIdx.x >> 5)) * spw; s0 < nslices; s0 += gridDim.x * wpb * spw) {
      const int s = s0 + sub;
      const bool live = s < nslices;
      const int base = live ? __ldg(slice_ptr + s) : 0;
      const int chunks = live ? __ldg(slice_len + s) / W : 0;
      const VI *ci = reinterpret_cast<const VI *>(col + base) + r;
      const VV *vi = reinterpret_cast<const VV *>(val + base) + r;
      X sum = X(0);
#pragma unroll 4
      for (int c = 0; c < chunks; ++c) {
        VI cc = ld_vec_stream(ci + c * C);
        VV vv = ld_vec_stream(vi + c * C);
#pragma unroll
        for (int k = 0; k < W; ++k)
          sum = fma((X)lane_get<VV, T, W>(vv, k), ld_keep(x + lane_geti<VI, W>(cc, k)), sum);
      }
      const int pos = s * C + r;
      if (live && pos < n) emit(perm ? __ldg(perm + pos) : pos, sum);
    }
  }
};

// ---- SELL-32 with int16 column offsets -------------------------------------
// Same slices and value layout as SellOp; the stored column of entry k is
// (column - row) as int16, so a warp reads 2*W bytes of indices per lane and
// step instead of 4*W.  Products and their order are those of SellOp.
template <int W> struct VecS;
template <> struct VecS<1> { using i = short; };
template <> struct VecS<2> { using i = short2; };
template <> struct VecS<4> { using i = short4; };

template <typename I> __device__ __forceinline__ int lane_gets(const I &v, int k) {
  return (int)reinterpret_cast<const short *>(&v)[k];
}

template <typename T, int W, typename X = T> struct SellOp16 {
  using XT = X;
  const int *__restrict__ slice_ptr;
  const int *__restrict__ slice_len;
  const short *__restrict__ col;
  const T *__restrict__ val;
  int n, nslices;
  int log2c;                 // C = 1 << log2c rows per slice
  const int *__restrict__ perm;  // row of each position, or null (identity)
  static constexpr int kRowsPerBlock = kBlock;
  __host__ __device__ int64_t work_items() const { return n; }
  template <typename Emit> __device__ __forceinline__ void run(const X *__restrict__ x, Emit &emit) const {
    using VV = typename VecW<T, W>::v;
    using VI = typename VecS<W>::i;
    const int lane = threadIdx.x & 31;
    const int wpb = kBlock / 32;
    const int C = 1 << log2c, spw = 32 >> log2c;
    const int r = lane & (C - 1), sub = lane >> log2c;
    for (int s0 = (blockIdx.x * wpb + ((int)threadIdx.x >> 5)) * spw; s0 < nslices; s0 += gridDim.x * wpb * spw) {
      const int s = s0 + sub;
      const bool live = s < nslices;
      const int base = live ? __ldg(slice_ptr + s) : 0;
      const int chunks = live ? __ldg(slice_len + s) / W : 0;
      const VI *ci = reinterpret_cast<const VI *>(col + base) + r;
      const VV *vi = reinterpret_cast<const VV *>(val + base) + r;
      const int pos = s * C + r;
      const bool real = live && pos < n;
      // the stored offsets are relative to the row itself; padding rows
      // past n (last slice) hold offset 0 and gather x[0]
      const int row = real ? (perm ? __ldg(perm + pos) : pos) : 0;
      X sum = X(0);
#pragma unroll 4
      for (int c = 0; c < chunks; ++c) {
        VI cc = __ldcs(ci + c * C);
        VV vv = ld_vec_stream(vi + c * C);
#pragma unroll
        for (int k = 0; k < W; ++k)
          sum = fma((X)lane_get<VV, T, W>(vv, k), ld_keep(x + row + lane_gets(cc, k)), sum);
      }
      if (real) emit(row, sum);
    }
  }
};

// ---- values-only sliced ELL (a stencil of column offsets) -----------------
// Square matrices whose every row's columns are a subset of one ascending
// list of offsets (structured-grid FE matrices): 32-row slices, every row
// EP entries (the stencil, padded to a multiple of W with offset 0), entry k
// of the row at position r of slice s at s*EP*32 + ((k/W)*32 + r)*W + k%W,
// value 0 where the row has no entry.  The column of entry k is
// row + off[k] (a compile-time index into the operator's offsets, which sit
// in the kernel's parameter space); slices whose columns all fall inside
// [0, n) skip the clamp the border slices need.  No column bytes at all:
// an FP64 3D Q1 row moves 8 bytes per entry instead of 10 (SELL16) or 12.
// Products in ascending column order, the rows' stored order, so the bits
// are SELL's (absent entries add 0 * x).
template <typename T, int W, int EP, typename X = T> struct StencilOp {
  using XT = X;
  const T *__restrict__ val;
  int n, nslices;
  int lo, hi;  // smallest and largest offset
  int off[EP];
  static constexpr int kRowsPerBlock = kBlock;
  __host__ __device__ int64_t work_items() const { return n; }
  template <typename Emit> __device__ __forceinline__ void run(const X *__restrict__ x, Emit &emit) const {
    using VV = typename VecW<T, W>::v;
    const int lane = threadIdx.x & 31;
    const int wpb = kBlock / 32;
    for (int s = blockIdx.x * wpb + ((int)threadIdx.x >> 5); s < nslices; s += gridDim.x * wpb) {
      const int row = s * 32 + lane;
      const VV *vi = reinterpret_cast<const VV *>(val + (int64_t)s * EP * 32) + lane;
      X sum = X(0);
      if (s * 32 + lo >= 0 && s * 32 + 31 + hi < n) {
#pragma unroll
        for (int c = 0; c < EP / W; ++c) {
          const VV vv = ld_vec_stream(vi + c * 32);
#pragma unroll
          for (int k = 0; k < W; ++k) sum = fma((X)lane_get<VV, T, W>(vv, k), ld_keep(x + row + off[c * W + k]), sum);
        }
      } else {
#pragma unroll
        for (int c = 0; c < EP / W; ++c) {
          const VV vv = ld_vec_stream(vi + c * 32);
#pragma unroll
          for (int k = 0; k < W; ++k)
            sum = fma((X)lane_get<VV, T, W>(vv, k), ld_keep(x + min(max(row + off[c * W + k], 0), n - 1)), sum);
        }
      }
      if (row < n) emit(row, sum);
    }
  }
};

template <typename Op> Op stencil_op(const void *val, int n, const SellData &s) {
  Op op;
  op.val = (decltype(op.val))val;
  op.n = n;
  op.nslices = s.nslices;
  op.lo = s.off_lo;
  op.hi = s.off_hi;
  for (int k = 0; k < (int)(sizeof(op.off) / sizeof(int)); ++k) op.off[k] = s.soff[k];
  return op;
}

// ---- plain emitters --------------------------------------------------------
template <typename T> struct StoreEmit {
  T *__restrict__ y;
  __device__ __forceinline__ void operator()(int row, T v) { y[row] = v; }
};
template <typename T> struct AddEmit {
  T *__restrict__ y;
  __device__ __forceinline__ void operator()(int row, T v) { y[row] += v; }
};

template <typename Op, typename T, bool ADD>
__global__ void __launch_bounds__(kBlock) spmv_kernel(Op op, const T *__restrict__ x, T *__restrict__ y) {
  if (ADD) {
    AddEmit<T> e{y};
    op.run(x, e);
  } else {
    StoreEmit<T> e{y};
    op.run(x, e);
  }
}

// Calls f(op) with the schedule selected on the matrix (stored values T,
// vectors X).
template <typename T, typename X = T, typename F> int with_schedule(b200la_mat m, F &&f) {
  const T *val = (const T *)m->val;
  if (m->format == B200LA_FMT_SELL) {
    const SellData &s = m->sell;
    const T *sv = (const T *)s.val;
    switch (m->param) {
      case 1: return f(SellOp<T, 1, X>{s.slice_ptr, s.slice_len, s.col, sv, m->nrow, s.nslices, s.log2c, s.perm});
      case 2: return f(SellOp<T, 2, X>{s.slice_ptr, s.slice_len, s.col, sv, m->nrow, s.nslices, s.log2c, s.perm});
      case 4: return f(SellOp<T, 4, X>{s.slice_ptr, s.slice_len, s.col, sv, m->nrow, s.nslices, s.log2c, s.perm});
    }
    return fail(B200LA_ERR_INVALID, "SELL width %d", m->param);
  }
  if (m->format == B200LA_FMT_SELL16) {
    const SellData &s = m->sell;
    const T *sv = (const T *)s.val;
    switch (m->param) {
      case 1:
        return f(SellOp16<T, 1, X>{s.slice_ptr, s.slice_len, s.col16p, sv, m->nrow, s.nslices, s.log2c, s.perm});
      case 2:
        return f(SellOp16<T, 2, X>{s.slice_ptr, s.slice_len, s.col16p, sv, m->nrow, s.nslices, s.log2c, s.perm});
      case 4:
        return f(SellOp16<T, 4, X>{s.slice_ptr, s.slice_len, s.col16p, sv, m->nrow, s.nslices, s.log2c, s.perm});
    }
    return fail(B200LA_ERR_INVALID, "SELL16 width %d", m->param);
  }
  if (m->format == B200LA_FMT_STENCIL) {
    const SellData &s = m->sell;
    const int key = m->param * 100 + s.ell;
    switch (key) {
      case 109: return f(stencil_op<StencilOp<T, 1, 9, X>>(s.val, m->nrow, s));
      case 210: return f(stencil_op<StencilOp<T, 2, 10, X>>(s.val, m->nrow, s));
      case 412: return f(stencil_op<StencilOp<T, 4, 12, X>>(s.val, m->nrow, s));
      case 127: return f(stencil_op<StencilOp<T, 1, 27, X>>(s.val, m->nrow, s));
      case 228: return f(stencil_op<StencilOp<T, 2, 28, X>>(s.val, m->nrow, s));
      case 428: return f(stencil_op<StencilOp<T, 4, 28, X>>(s.val, m->nrow, s));
    }
    return fail(B200LA_ERR_INVALID, "STENCIL width %d with %d entries per row", m->param, s.ell);
  }
  switch (m->param) {
    case 1: return f(CsrOp<T, 1, X>{m->rowptr, m->col, val, m->nrow});
    case 2: return f(CsrOp<T, 2, X>{m->rowptr, m->col, val, m->nrow});
    case 4: return f(CsrOp<T, 4, X>{m->rowptr, m->col, val, m->nrow});
    case 8: return f(CsrOp<T, 8, X>{m->rowptr, m->col, val, m->nrow});
    case 16: return f(CsrOp<T, 16, X>{m->rowptr, m->col, val, m->nrow});
    case 32: return f(CsrOp<T, 32, X>{m->rowptr, m->col, val, m->nrow});
  }
  return fail(B200LA_ERR_INVALID, "CSR lanes per row %d", m->param);
}

int spmv_launch(b200la_mat m, const void *x, void *y, bool add, cudaStream_t s);
// y = (A - diag(A)) x from the CSR as uploaded (VectorMultNoDiag)
int spmv_nodiag_launch(b200la_mat m, const void *x, void *y, cudaStream_t s);
// Builds the sliced copy: `width` entries per vector load, int16 column
// offsets (col16), C rows per slice, rows sorted by length within windows of
// sigma rows (1 = no sorting; otherwise rounded up to a multiple of C).
int sell_build(b200la_mat m, int width, bool col16 = false, int C = 32, int sigma = 1);
// Builds the values-only copy (B200LA_FMT_STENCIL) with `width` entries per
// vector load; B200LA_ERR_UNSUPPORTED when the matrix has no stencil.
int stencil_build(b200la_mat m, int width);
inline bool is_sell(int format) { return format == B200LA_FMT_SELL || format == B200LA_FMT_SELL16; }
// any schedule with a sliced copy (rebuilt when the values change)
inline bool is_sliced(int format) { return is_sell(format) || format == B200LA_FMT_STENCIL; }
// frees the sliced copy and builds the one `format` / `param` name (C and
// sigma for SELL-C-sigma) from the CSR: after the values changed
int sliced_rebuild(b200la_mat m, int format, int param, int C, int sigma);
void sell_free(b200la_mat m);

}  // namespace b200la
