// SpMV launch, SELL-32 construction and the SpMV autotuner.
#include <algorithm>
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

int sell_build(b200la_mat m, int width, bool col16) {
  if (m->sell.width == width && m->sell.col16 == (int)col16 && (col16 ? (void *)m->sell.col16p : (void *)m->sell.col))
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
  SellData &d = m->sell;
  d.width = width;
  d.col16 = col16 ? 1 : 0;
  d.nslices = (m->nrow + 31) / 32;
  if (d.nslices == 0) return B200LA_OK;
  B_CUDA(cudaMallocAsync(&d.slice_len, sizeof(int) * d.nslices, s));
  B_CUDA(cudaMallocAsync(&d.slice_ptr, sizeof(int) * (d.nslices + 1), s));
  sell_len_kernel<<<(d.nslices + kBlock - 1) / kBlock, kBlock, 0, s>>>(m->nrow, d.nslices, width, m->rowptr,
                                                                      d.slice_len);
  B_CUDA(cudaGetLastError());
  std::vector<int> len(d.nslices);
  std::vector<int> ptr(d.nslices + 1);
  B_CUDA(cudaMemcpyAsync(len.data(), d.slice_len, sizeof(int) * d.nslices, cudaMemcpyDeviceToHost, s));
  B_CUDA(cudaStreamSynchronize(s));
  int64_t acc = 0;
  for (int i = 0; i < d.nslices; ++i) {
    ptr[i] = (int)acc;
    acc += (int64_t)len[i] * 32;
    B_CHECK(acc < INT32_MAX, B200LA_ERR_UNSUPPORTED, "SELL: padded size exceeds int32 indexing");
  }
  ptr[d.nslices] = (int)acc;
  d.padded = acc;
  size_t pz = (size_t)(acc > 0 ? acc : 1);
  B_CUDA(cudaMemcpyAsync(d.slice_ptr, ptr.data(), sizeof(int) * (d.nslices + 1), cudaMemcpyHostToDevice, s));
  if (col16) B_CUDA(cudaMallocAsync(&d.col16p, sizeof(short) * pz, s));
  else B_CUDA(cudaMallocAsync(&d.col, sizeof(int) * pz, s));
  B_CUDA(cudaMallocAsync(&d.val, dtype_size(m->dtype) * pz, s));
  int threads = d.nslices * 32;
  int grid = (threads + kBlock - 1) / kBlock;
  if (m->dtype == B200LA_F64)
    sell_fill_kernel<double><<<grid, kBlock, 0, s>>>(m->nrow, d.nslices, width, m->rowptr, m->col,
                                                     (const double *)m->val, d.slice_ptr, d.slice_len, d.col,
                                                     d.col16p, (double *)d.val);
  else
    sell_fill_kernel<float><<<grid, kBlock, 0, s>>>(m->nrow, d.nslices, width, m->rowptr, m->col,
                                                    (const float *)m->val, d.slice_ptr, d.slice_len, d.col,
                                                    d.col16p, (float *)d.val);
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}

}  // namespace b200la

using namespace b200la;

extern "C" int b200la_mat_tune(b200la_mat m, int *format, int *param, double *usec) {
  B_CHECK(m, B200LA_ERR_INVALID, "mat_tune: null matrix");
  b200la_ctx c = m->ctx;
  cudaStream_t s = c->stream;
  const int fmts[][2] = {{B200LA_FMT_CSR, 2},    {B200LA_FMT_CSR, 4},    {B200LA_FMT_CSR, 8},
                         {B200LA_FMT_CSR, 16},   {B200LA_FMT_CSR, 32},   {B200LA_FMT_SELL, 1},
                         {B200LA_FMT_SELL, 2},   {B200LA_FMT_SELL, 4},   {B200LA_FMT_SELL16, 1},
                         {B200LA_FMT_SELL16, 2}, {B200LA_FMT_SELL16, 4}};
  size_t es = dtype_size(m->dtype);
  void *x = nullptr, *y = nullptr;
  B_CUDA(cudaMallocAsync(&x, es * (m->ncol > 0 ? m->ncol : 1), s));
  B_CUDA(cudaMallocAsync(&y, es * (m->nrow > 0 ? m->nrow : 1), s));
  B_CUDA(cudaMemsetAsync(x, 0, es * (m->ncol > 0 ? m->ncol : 1), s));
  cudaEvent_t e0, e1;
  B_CUDA(cudaEventCreate(&e0));
  B_CUDA(cudaEventCreate(&e1));
  int best_f = m->format, best_p = m->param;
  float best = 1e30f;
  const int reps = 10;
  for (auto &fp : fmts) {
    if (is_sell(fp[0])) {
      // SELL copies cost extra HBM; skip them when they would pad badly.
      if (b200la_mat_set_format(m, fp[0], fp[1]) != B200LA_OK) continue;
      if ((double)m->sell.padded > 1.25 * (double)m->nnz + 64.0 * m->sell.nslices) continue;
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
    if (ms < best) {
      best = ms;
      best_f = fp[0];
      best_p = fp[1];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(x, s);
  cudaFreeAsync(y, s);
  B_TRY(b200la_mat_set_format(m, best_f, best_p));
  if (!is_sell(best_f)) sell_free(m);
  if (format) *format = best_f;
  if (param) *param = best_p;
  if (usec) *usec = 1000.0 * best / reps;
  return B200LA_OK;
}
