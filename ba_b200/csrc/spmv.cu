// SpMV launch, SELL-32 construction and the SpMV autotuner.
#include <algorithm>
#include <array>
#include <vector>

#include "internal.cuh"
#include "spmv.cuh"

namespace b200la {

template <typename T>
static int spmv_launch_t(b200la_mat m, const T *x, T *y, bool add, cudaStream_t s) {
  return with_schedule<T>(m, [&](auto op) -> int {
    using Op = decltype(op);
    int grid;
    if (add) {
      B_TRY(grid_for(m->ctx, (const void *)spmv_kernel<Op, T, true>, op.work_items(), Op::kRowsPerBlock, &grid));
      spmv_kernel<Op, T, true><<<grid, kBlock, 0, s>>>(op, x, y);
    } else {
      B_TRY(grid_for(m->ctx, (const void *)spmv_kernel<Op, T, false>, op.work_items(), Op::kRowsPerBlock, &grid));
      spmv_kernel<Op, T, false><<<grid, kBlock, 0, s>>>(op, x, y);
    }
    B_CUDA(cudaGetLastError());
    return B200LA_OK;
  });
}

int spmv_launch(b200la_mat m, const void *x, void *y, bool add, cudaStream_t s) {
  if (m->nrow == 0) return B200LA_OK;
  if (m->dtype == B200LA_F64) return spmv_launch_t<double>(m, (const double *)x, (double *)y, add, s);
  return spmv_launch_t<float>(m, (const float *)x, (float *)y, add, s);
}

// ---- y = (A - diag(A)) x: CPU_CSR_lMatrix::VectorMultNoDiag
// (lmp/lmatrix_csr_cpu.cc:479-493): every stored entry whose column is not
// the row, in stored order; 8 lanes per row over the CSR as uploaded (the
// stationary Jacobi path, not the PCG's hot loop).
template <typename T>
__global__ void __launch_bounds__(kBlock) spmv_nodiag_kernel(int n, const int *__restrict__ rowptr,
                                                             const int *__restrict__ col,
                                                             const T *__restrict__ val, const T *__restrict__ x,
                                                             T *__restrict__ y) {
  constexpr int G = 8;
  const int lane = threadIdx.x & (G - 1);
  for (int base = blockIdx.x * (kBlock / G); base < n; base += gridDim.x * (kBlock / G)) {
    const int row = base + (int)threadIdx.x / G;
    T sum = T(0);
    if (row < n) {
      for (int j = __ldg(rowptr + row) + lane; j < __ldg(rowptr + row + 1); j += G) {
        const int c = __ldg(col + j);
        if (c != row) sum = fma(__ldg(val + j), __ldg(x + c), sum);
      }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (row < n && lane == 0) y[row] = sum;
  }
}

int spmv_nodiag_launch(b200la_mat m, const void *x, void *y, cudaStream_t s) {
  if (m->nrow == 0) return B200LA_OK;
  int grid;
  if (m->dtype == B200LA_F64) {
    B_TRY(grid_for(m->ctx, (const void *)spmv_nodiag_kernel<double>, m->nrow, kBlock / 8, &grid));
    spmv_nodiag_kernel<double><<<grid, kBlock, 0, s>>>(m->nrow, m->rowptr, m->col, (const double *)m->val,
                                                       (const double *)x, (double *)y);
  } else {
    B_TRY(grid_for(m->ctx, (const void *)spmv_nodiag_kernel<float>, m->nrow, kBlock / 8, &grid));
    spmv_nodiag_kernel<float><<<grid, kBlock, 0, s>>>(m->nrow, m->rowptr, m->col, (const float *)m->val,
                                                      (const float *)x, (float *)y);
  }
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

// ---- SELL construction -----------------------------------------------------
__global__ void sell_len_kernel(int n, int nslices, int width, const int *__restrict__ rowptr, int *__restrict__ len) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  int mx = 0;
  for (int r = s * 32; r < min(n, s * 32 + 32); ++r) mx = max(mx, rowptr[r + 1] - rowptr[r]);
  len[s] = (mx + width - 1) / width * width;
}

template <typename T>
__global__ void sell_fill_kernel(int n, int nslices, int width, const int *__restrict__ rowptr,
                                 const int *__restrict__ col, const T *__restrict__ val,
                                 const int *__restrict__ slice_ptr, const int *__restrict__ slice_len,
                                 int *__restrict__ scol, short *__restrict__ scol16, T *__restrict__ sval) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int s = t >> 5, lane = t & 31;
  if (s >= nslices) return;
  int row = s * 32 + lane;
  int base = slice_ptr[s], L = slice_len[s];
  int start = 0, len = 0, pad_col = 0;
  if (row < n) {
    start = rowptr[row];
    len = rowptr[row + 1] - start;
    // padding repeats a column the row reads; an empty row of the int16
    // layout (square matrices only) pads with its own diagonal position
    pad_col = len > 0 ? col[start + len - 1] : (scol16 ? row : 0);
  }
  for (int k = 0; k < L; ++k) {
    int pos = base + ((k / width) * 32 + lane) * width + (k % width);
    const int c = k < len ? col[start + k] : pad_col;
    if (scol16) scol16[pos] = (short)(row < n ? c - row : 0);
    else scol[pos] = c;
    sval[pos] = k < len ? val[start + k] : T(0);
  }
}

// SELL-C-sigma fill: thread t handles position t % C of slice t / C, the
// row perm[position] (identity without sorting); same entry layout as
// sell_fill_kernel with C rows per slice.
template <typename T>
__global__ void sellcs_fill_kernel(int n, int nslices, int C, int width, const int *__restrict__ perm,
                                   const int *__restrict__ rowptr, const int *__restrict__ col,
                                   const T *__restrict__ val, const int *__restrict__ slice_ptr,
                                   const int *__restrict__ slice_len, int *__restrict__ scol,
                                   short *__restrict__ scol16, T *__restrict__ sval) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = (int)(t / C), lane = (int)(t % C);
  if (s >= nslices) return;
  const int pos = s * C + lane;
  const int row = pos < n ? (perm ? perm[pos] : pos) : -1;
  const int base = slice_ptr[s], L = slice_len[s];
  int start = 0, len = 0, pad_col = 0;
  if (row >= 0) {
    start = rowptr[row];
    len = rowptr[row + 1] - start;
    pad_col = len > 0 ? col[start + len - 1] : (scol16 ? row : 0);
  }
  for (int k = 0; k < L; ++k) {
    const int64_t p = base + ((int64_t)(k / width) * C + lane) * width + (k % width);
    const int c = k < len ? col[start + k] : pad_col;
    if (scol16) scol16[p] = (short)(row >= 0 ? c - row : 0);
    else scol[p] = c;
    sval[p] = k < len ? val[start + k] : T(0);
  }
}

// Largest |col - row| over the stored entries (atomicMax of each row's).
__global__ void offset_range_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                                    int *__restrict__ maxabs) {
  const int stride = gridDim.x * blockDim.x;
  int mx = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    for (int j = rowptr[i]; j < rowptr[i + 1]; ++j) mx = max(mx, abs(col[j] - i));
  if (mx) atomicMax(maxabs, mx);
}

void sell_free(b200la_mat m) {
  cudaStream_t s = m->ctx->stream;
  SellData &d = m->sell;
  if (d.slice_ptr) cudaFreeAsync(d.slice_ptr, s);
  if (d.slice_len) cudaFreeAsync(d.slice_len, s);
  if (d.col) cudaFreeAsync(d.col, s);
  if (d.col16p) cudaFreeAsync(d.col16p, s);
  if (d.val) cudaFreeAsync(d.val, s);
  if (d.perm) cudaFreeAsync(d.perm, s);
  d = SellData();
}

int sell_build(b200la_mat m, int width, bool col16, int C, int sigma) {
  B_CHECK(C == 8 || C == 16 || C == 32, B200LA_ERR_INVALID, "SELL: C = %d rows per slice (8, 16 or 32)", C);
  B_CHECK(sigma >= 1, B200LA_ERR_INVALID, "SELL: sigma %d (>= 1)", sigma);
  if (sigma > 1) sigma = (int)std::min<int64_t>(((int64_t)sigma + C - 1) / C * C, INT32_MAX / 2);
  if (m->sell.width == width && m->sell.col16 == (int)col16 && m->sell.c == C && m->sell.sigma == sigma &&
      (col16 ? (void *)m->sell.col16p : (void *)m->sell.col))
    return B200LA_OK;
  cudaStream_t s = m->ctx->stream;
  if (col16) {
    B_CHECK(m->nrow == m->ncol, B200LA_ERR_UNSUPPORTED, "SELL16: square matrices only (%dx%d)", m->nrow, m->ncol);
    // int16 offsets only when every stored column lies within int16 of its row
    int *d_max = nullptr, h_max = 0;
    B_CUDA(cudaMallocAsync(&d_max, sizeof(int), s));
    B_CUDA(cudaMemsetAsync(d_max, 0, sizeof(int), s));
    if (m->nrow) {
      const int grid = std::min((m->nrow + kBlock - 1) / kBlock, m->ctx->num_sms * 8);
      offset_range_kernel<<<grid, kBlock, 0, s>>>(m->nrow, m->rowptr, m->col, d_max);
    }
    B_CUDA(cudaGetLastError());
    B_CUDA(cudaMemcpyAsync(&h_max, d_max, sizeof(int), cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaFreeAsync(d_max, s));
    B_CUDA(cudaStreamSynchronize(s));
    B_CHECK(h_max <= 32767, B200LA_ERR_UNSUPPORTED, "SELL16: a column lies %d rows from its row (int16 offsets)",
            h_max);
  }
  sell_free(m);
  m->sched_gen += 1;  // graphs holding the old copy's pointers re-capture
  SellData &d = m->sell;
  d.width = width;
  d.col16 = col16 ? 1 : 0;
  d.c = C;
  d.log2c = C == 8 ? 3 : (C == 16 ? 4 : 5);
  d.sigma = sigma;
  d.nslices = (m->nrow + C - 1) / C;
  if (d.nslices == 0) return B200LA_OK;
  B_CUDA(cudaMallocAsync(&d.slice_len, sizeof(int) * d.nslices, s));
  B_CUDA(cudaMallocAsync(&d.slice_ptr, sizeof(int) * (d.nslices + 1), s));
  std::vector<int> len(d.nslices);
  std::vector<int> ptr(d.nslices + 1);
  if (C == 32 && sigma == 1) {
    sell_len_kernel<<<(d.nslices + kBlock - 1) / kBlock, kBlock, 0, s>>>(m->nrow, d.nslices, width, m->rowptr,
                                                                        d.slice_len);
    B_CUDA(cudaGetLastError());
    B_CUDA(cudaMemcpyAsync(len.data(), d.slice_len, sizeof(int) * d.nslices, cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaStreamSynchronize(s));
  } else {
    // SELL-C-sigma: the rows' lengths come to the host, each window of
    // sigma rows is ordered longest first (stable, so equal lengths keep
    // their order), and each slice takes its longest row rounded up to W
    const int n = m->nrow;
    std::vector<int> rp(n + 1);
    B_CUDA(cudaMemcpyAsync(rp.data(), m->rowptr, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaStreamSynchronize(s));
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    if (sigma > 1)
      for (int w0 = 0; w0 < n; w0 += sigma)
        std::stable_sort(perm.begin() + w0, perm.begin() + std::min(n, w0 + sigma), [&](int a, int b) {
          return rp[a + 1] - rp[a] > rp[b + 1] - rp[b];
        });
    for (int sl = 0; sl < d.nslices; ++sl) {
      int mx = 0;
      for (int r = sl * C; r < std::min(n, sl * C + C); ++r) mx = std::max(mx, rp[perm[r] + 1] - rp[perm[r]]);
      len[sl] = (mx + width - 1) / width * width;
    }
    B_CUDA(cudaMemcpyAsync(d.slice_len, len.data(), sizeof(int) * d.nslices, cudaMemcpyHostToDevice, s));
    if (sigma > 1) {
      B_CUDA(cudaMallocAsync(&d.perm, sizeof(int) * n, s));
      B_CUDA(cudaMemcpyAsync(d.perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    }
    B_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  }
  int64_t acc = 0;
  for (int i = 0; i < d.nslices; ++i) {
    ptr[i] = (int)acc;
    acc += (int64_t)len[i] * C;
    B_CHECK(acc < INT32_MAX, B200LA_ERR_UNSUPPORTED, "SELL: padded size exceeds int32 indexing");
  }
  ptr[d.nslices] = (int)acc;
  d.padded = acc;
  size_t pz = (size_t)(acc > 0 ? acc : 1);
  B_CUDA(cudaMemcpyAsync(d.slice_ptr, ptr.data(), sizeof(int) * (d.nslices + 1), cudaMemcpyHostToDevice, s));
  if (col16) B_CUDA(cudaMallocAsync(&d.col16p, sizeof(short) * pz, s));
  else B_CUDA(cudaMallocAsync(&d.col, sizeof(int) * pz, s));
  B_CUDA(cudaMallocAsync(&d.val, dtype_size(m->dtype) * pz, s));
  const int64_t threads = (int64_t)d.nslices * C;
  const int grid = (int)((threads + kBlock - 1) / kBlock);
  if (C == 32 && sigma == 1) {
    if (m->dtype == B200LA_F64)
      sell_fill_kernel<double><<<grid, kBlock, 0, s>>>(m->nrow, d.nslices, width, m->rowptr, m->col,
                                                       (const double *)m->val, d.slice_ptr, d.slice_len, d.col,
                                                       d.col16p, (double *)d.val);
    else
      sell_fill_kernel<float><<<grid, kBlock, 0, s>>>(m->nrow, d.nslices, width, m->rowptr, m->col,
                                                      (const float *)m->val, d.slice_ptr, d.slice_len, d.col,
                                                      d.col16p, (float *)d.val);
  } else if (m->dtype == B200LA_F64) {
    sellcs_fill_kernel<double><<<grid, kBlock, 0, s>>>(m->nrow, d.nslices, C, width, d.perm, m->rowptr, m->col,
                                                       (const double *)m->val, d.slice_ptr, d.slice_len, d.col,
                                                       d.col16p, (double *)d.val);
  } else {
    sellcs_fill_kernel<float><<<grid, kBlock, 0, s>>>(m->nrow, d.nslices, C, width, d.perm, m->rowptr, m->col,
                                                      (const float *)m->val, d.slice_ptr, d.slice_len, d.col,
                                                      d.col16p, (float *)d.val);
  }
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}

// ---- values-only copy (B200LA_FMT_STENCIL) ---------------------------------
struct StencilOffsets {
  int v[kStencilMax];
};

// The first row of the longest length (the stencil's source).
__global__ void longest_row_kernel(int n, const int *__restrict__ rowptr, int len, int *__restrict__ first) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    if (rowptr[i + 1] - rowptr[i] == len) atomicMin(first, i);
}

// Every row's columns strictly ascending and each column - row one of the E
// ascending offsets (a two-pointer walk); *bad = 1 otherwise.
__global__ void stencil_check_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                                     StencilOffsets off, int E, int *__restrict__ bad) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    int k = 0;
    bool ok = true;
    for (int j = rowptr[i]; j < rowptr[i + 1] && ok; ++j) {
      const int d = col[j] - i;
      while (k < E && off.v[k] < d) ++k;
      ok = k < E && off.v[k] == d;
      ++k;  // strictly ascending: the next column takes a later offset
    }
    if (!ok) *bad = 1;
  }
}

// Thread t: position t % 32 of slice t / 32 (row 32s + r); entry k of the
// row at s*EP*32 + ((k/W)*32 + r)*W + k%W, the row's value at column
// row + off[k] or 0 (rows past n: all 0).
template <typename T>
__global__ void stencil_fill_kernel(int n, int nslices, int EP, int W, const int *__restrict__ rowptr,
                                    const int *__restrict__ col, const T *__restrict__ val, StencilOffsets off,
                                    T *__restrict__ sval) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int s = (int)(t >> 5), r = (int)(t & 31);
  if (s >= nslices) return;
  const int row = s * 32 + r;
  int j = row < n ? rowptr[row] : 0;
  const int end = row < n ? rowptr[row + 1] : 0;
  T *base = sval + (int64_t)s * EP * 32;
  for (int k = 0; k < EP; ++k) {
    T v = T(0);
    if (j < end && col[j] - row == off.v[k]) v = val[j++];
    base[((k / W) * 32 + r) * W + k % W] = v;
  }
}

int stencil_build(b200la_mat m, int width) {
  B_CHECK(width == 1 || width == 2 || width == 4, B200LA_ERR_INVALID, "STENCIL: width %d (1, 2 or 4)", width);
  SellData &cur = m->sell;
  if (cur.stencil && cur.width == width && cur.val) return B200LA_OK;
  B_CHECK(m->nrow == m->ncol && m->nrow > 0, B200LA_ERR_UNSUPPORTED, "STENCIL: square matrices only (%dx%d)",
          m->nrow, m->ncol);
  const int E = m->max_row;
  B_CHECK(E == 9 || E == 27, B200LA_ERR_UNSUPPORTED, "STENCIL: longest row %d (9 or 27 entries)", E);
  cudaStream_t s = m->ctx->stream;
  const int n = m->nrow;
  // the offsets of the first longest row
  int *d_tmp = nullptr;
  B_CUDA(cudaMallocAsync(&d_tmp, sizeof(int) * 2, s));
  const int first_init = INT32_MAX;
  B_CUDA(cudaMemcpyAsync(d_tmp, &first_init, sizeof(int), cudaMemcpyHostToDevice, s));
  B_CUDA(cudaMemsetAsync(d_tmp + 1, 0, sizeof(int), s));
  const int grid = std::min((n + kBlock - 1) / kBlock, m->ctx->num_sms * 8);
  longest_row_kernel<<<grid, kBlock, 0, s>>>(n, m->rowptr, E, d_tmp);
  B_CUDA(cudaGetLastError());
  int first = 0, start = 0;
  B_CUDA(cudaMemcpyAsync(&first, d_tmp, sizeof(int), cudaMemcpyDeviceToHost, s));
  B_CUDA(cudaStreamSynchronize(s));
  int rc = B200LA_OK;
  StencilOffsets off{};
  if (first == INT32_MAX) rc = fail(B200LA_ERR_UNSUPPORTED, "STENCIL: no row of the longest length");
  if (rc == B200LA_OK) {
    int cols[kStencilMax];
    cudaError_t e = cudaMemcpyAsync(&start, m->rowptr + first, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cols, m->col + start, sizeof(int) * E, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(B200LA_ERR_CUDA, "STENCIL: %s", cudaGetErrorString(e));
    for (int k = 0; rc == B200LA_OK && k < E; ++k) {
      off.v[k] = cols[k] - first;
      if (k > 0 && off.v[k] <= off.v[k - 1])
        rc = fail(B200LA_ERR_UNSUPPORTED, "STENCIL: the columns of row %d are not strictly ascending", first);
    }
  }
  int bad = 0;
  if (rc == B200LA_OK) {
    stencil_check_kernel<<<grid, kBlock, 0, s>>>(n, m->rowptr, m->col, off, E, d_tmp + 1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_tmp + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = fail(B200LA_ERR_CUDA, "STENCIL: %s", cudaGetErrorString(e));
    else if (bad) rc = fail(B200LA_ERR_UNSUPPORTED, "STENCIL: a row's columns are not in the stencil of row %d", first);
  }
  cudaFreeAsync(d_tmp, s);
  B_TRY(rc);
  sell_free(m);
  m->sched_gen += 1;  // graphs holding the old copy's pointers re-capture
  SellData &d = m->sell;
  const int EP = (E + width - 1) / width * width;
  for (int k = E; k < EP; ++k) off.v[k] = 0;  // padding: value 0 at the row's own column
  d.stencil = 1;
  d.width = width;
  d.ell = EP;
  d.c = 32;
  d.log2c = 5;
  d.sigma = 1;
  d.nslices = (n + 31) / 32;
  d.padded = (int64_t)d.nslices * 32 * EP;
  d.off_lo = d.off_hi = 0;  // 0 included: the padding's column
  for (int k = 0; k < EP; ++k) {
    d.soff[k] = off.v[k];
    d.off_lo = std::min(d.off_lo, off.v[k]);
    d.off_hi = std::max(d.off_hi, off.v[k]);
  }
  B_CUDA(cudaMallocAsync(&d.val, dtype_size(m->dtype) * (size_t)d.padded, s));
  const int fgrid = (int)(((int64_t)d.nslices * 32 + kBlock - 1) / kBlock);
  if (m->dtype == B200LA_F64)
    stencil_fill_kernel<double><<<fgrid, kBlock, 0, s>>>(n, d.nslices, EP, width, m->rowptr, m->col,
                                                         (const double *)m->val, off, (double *)d.val);
  else
    stencil_fill_kernel<float><<<fgrid, kBlock, 0, s>>>(n, d.nslices, EP, width, m->rowptr, m->col,
                                                        (const float *)m->val, off, (float *)d.val);
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}

int sliced_rebuild(b200la_mat m, int format, int param, int C, int sigma) {
  sell_free(m);
  if (format == B200LA_FMT_STENCIL) return stencil_build(m, param);
  return sell_build(m, param, format == B200LA_FMT_SELL16, C, sigma);
}

}  // namespace b200la

using namespace b200la;

extern "C" int b200la_mat_tune(b200la_mat m, int *format, int *param, double *usec) {
  B_CHECK(m, B200LA_ERR_INVALID, "mat_tune: null matrix");
  b200la_ctx c = m->ctx;
  cudaStream_t s = c->stream;
  // candidates {format, param, C, sigma}: CSR lane groups; SELL and SELL16
  // with vector widths 1/2/4 and slice heights C = 32, 16, 8, rows in their
  // order (sigma 1) or sorted by length within windows of 1,024 rows; the
  // values-only copy with widths 1/2/4 (matrices with a stencil)
  std::vector<std::array<int, 4>> fmts = {{B200LA_FMT_CSR, 2, 0, 0},  {B200LA_FMT_CSR, 4, 0, 0},
                                          {B200LA_FMT_CSR, 8, 0, 0},  {B200LA_FMT_CSR, 16, 0, 0},
                                          {B200LA_FMT_CSR, 32, 0, 0}};
  for (int f : {B200LA_FMT_SELL, B200LA_FMT_SELL16})
    for (int sig : {1, 1024})
      for (int cc : {32, 16, 8})
        for (int w : {1, 2, 4}) fmts.push_back({f, w, cc, sig});
  for (int w : {1, 2, 4}) fmts.push_back({B200LA_FMT_STENCIL, w, 32, 1});
  size_t es = dtype_size(m->dtype);
  void *x = nullptr, *y = nullptr;
  B_CUDA(cudaMallocAsync(&x, es * (m->ncol > 0 ? m->ncol : 1), s));
  B_CUDA(cudaMallocAsync(&y, es * (m->nrow > 0 ? m->nrow : 1), s));
  B_CUDA(cudaMemsetAsync(x, 0, es * (m->ncol > 0 ? m->ncol : 1), s));
  cudaEvent_t e0, e1;
  B_CUDA(cudaEventCreate(&e0));
  B_CUDA(cudaEventCreate(&e1));
  int best_f = m->format, best_p = m->param, best_c = m->sell.c, best_sig = m->sell.sigma;
  float best = 1e30f;
  const int reps = 10;
  for (auto &fp : fmts) {
    if (is_sliced(fp[0])) {
      // sliced copies cost extra HBM; skip them when they would pad badly
      // (STENCIL: when the matrix has no stencil)
      if (fp[0] == B200LA_FMT_STENCIL) {
        if (b200la_mat_set_format(m, fp[0], fp[1]) != B200LA_OK) continue;
      } else if (b200la_mat_to_sell(m, fp[2], fp[3], fp[1], fp[0] == B200LA_FMT_SELL16) != B200LA_OK) {
        continue;
      }
      if ((double)m->sell.padded > 1.25 * (double)m->nnz + 2.0 * fp[2] * m->sell.nslices) continue;
    } else if (b200la_mat_set_format(m, fp[0], fp[1]) != B200LA_OK) {
      continue;
    }
    B_TRY(spmv_launch(m, x, y, false, s));  // warm-up
    B_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; ++r) B_TRY(spmv_launch(m, x, y, false, s));
    B_CUDA(cudaEventRecord(e1, s));
    B_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    B_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    // a sliced copy must beat the best so far by 1% to win, so C = 32
    // without sorting (listed first) is kept where the others only tie
    if (ms < (is_sliced(fp[0]) && is_sliced(best_f) ? 0.99f : 1.0f) * best) {
      best = ms;
      best_f = fp[0];
      best_p = fp[1];
      best_c = fp[2];
      best_sig = fp[3];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(x, s);
  cudaFreeAsync(y, s);
  if (is_sell(best_f)) B_TRY(b200la_mat_to_sell(m, best_c, best_sig, best_p, best_f == B200LA_FMT_SELL16));
  else B_TRY(b200la_mat_set_format(m, best_f, best_p));
  if (!is_sliced(best_f)) sell_free(m);
  if (format) *format = best_f;
  if (param) *param = best_p;
  if (usec) *usec = 1000.0 * best / reps;
  return B200LA_OK;
}
