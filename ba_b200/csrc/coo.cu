// COO -> CSR on the device: CPU_CSR_lMatrix::TransformFromCOO
// (lmp/lmatrix_csr_cpu.cc:883-906), i.e. coo_2_csr (lmp/lmatrix_formats.h:
// 320-452), for matrices assembled as coordinate triplets.
//
// The reference counts the entries of each row, scatters them in input order
// and then sorts every row by column with a selection sort that keeps
// duplicates (and, being a selection sort with swaps, does not keep them in
// input order).  Here the same result comes from:
//   1. a device check of every index (a bad triplet fails the upload),
//   2. a stable radix sort of the triplets by row carrying (column, input
//      position) pairs (input order kept within a row, as the reference's
//      scatter keeps it),
//   3. row offsets from the sorted rows (each row boundary writes its range),
//   4. a gather of the values from their input positions (cast to the
//      storage type), the columns coming with the sorted pairs,
//   5. the row sort, one warp per row: ranks by shuffles when the row's
//      columns are distinct (the sorted row is then unique), the
//      reference's selection sort itself when a column repeats or the row
//      is longer than 256 entries (rows above 32 entries go through a
//      worklist to a second kernel),
//   6. the diagonal positions and the longest row, as b200la_csr_upload does.
// The result is the reference's CSR bit for bit, duplicates included.
#include <cub/device/device_radix_sort.cuh>

#include <climits>
#include <cstring>

#include "internal.cuh"

namespace b200la {

// First bad triplet (smallest index), or all ones when every index is in range.
__global__ void coo_check_kernel(int64_t nnz, int nrow, int ncol, const int *__restrict__ rows,
                                 const int *__restrict__ cols, unsigned long long *bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = rows[i], c = cols[i];
    if (r < 0 || r >= nrow || c < 0 || c >= ncol) atomicMin(bad, (unsigned long long)i);
  }
}

// Sort payload of each triplet: its column in the high word and its input
// position in the low word, so that the sort carries the column along and
// the gather reads only the value from a random position.
__global__ void coo_pack_kernel(int64_t n, const int *__restrict__ cols, unsigned long long *out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = ((unsigned long long)(unsigned)cols[i] << 32) | (unsigned long long)(unsigned)i;
}

// rowptr from the rows sorted ascending: entry i starts rows prev+1 .. r.
__global__ void coo_rowptr_kernel(int64_t nnz, int nrow, const int *__restrict__ srow, int *rowptr) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const int prev = i == 0 ? -1 : srow[i - 1];
    const int r = i == nnz ? nrow : srow[i];
    for (int rr = prev + 1; rr <= r; ++rr) rowptr[rr] = (int)i;
  }
}

// The reference's per-row selection sort (lmatrix_formats.h:405-431) on
// col[b, e) / val[b, e) in place, then the first diagonal entry.
template <typename T>
__device__ void row_selection_sort(int k, int b, int e, int *col, T *val, int *diag) {
  for (int i = b; i != e; ++i) {
    int mi = i, mc = col[i];
    for (int j = i + 1; j < e; ++j)
      if (col[j] < mc) {
        mi = j;
        mc = col[j];
      }
    const int tc = col[i];
    col[i] = col[mi];
    col[mi] = tc;
    const T tv = val[i];
    val[i] = val[mi];
    val[mi] = tv;
  }
  int d = -1;
  for (int i = b; i != e; ++i)
    if (col[i] == k) {
      d = i;
      break;
    }
  diag[k] = d;
}

// Columns and values into the row-sorted order: the column comes with the
// sorted payload, the value (cast to the storage type) from its input
// position, a random read; each thread keeps kGatherUnroll of those in flight.
constexpr int kGatherUnroll = 4;

template <typename T, typename S>
__global__ void __launch_bounds__(kBlock) coo_gather_kernel(int64_t nnz, const unsigned long long *__restrict__ packed,
                                                            const S *__restrict__ vals, int *col, T *val) {
  constexpr int U = kGatherUnroll;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k0 < nnz; k0 += U * stride) {
    unsigned long long q[U];
#pragma unroll
    for (int u = 0; u < U; ++u) q[u] = k0 + u * stride < nnz ? packed[k0 + u * stride] : 0ull;
    S vv[U];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (k0 + u * stride < nnz) vv[u] = vals[(unsigned)q[u]];
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (k0 + u * stride < nnz) {
        col[k0 + u * stride] = (int)(q[u] >> 32);
        val[k0 + u * stride] = (T)vv[u];
      }
  }
}

// Row sort, one warp per row of up to 32 entries (lane l holds entry l, in
// input order as gathered).  When the row's columns are distinct the sorted
// row is unique, so each entry goes straight to b + (number of smaller
// columns), ranks taken with shuffles; that equals the reference's selection
// sort.  A row with a repeated column (found by __match_any_sync) is sorted
// by the selection sort itself (lane 0), because there the order of equal
// columns depends on its swaps.  Longer rows are appended to a worklist for
// coo_long_rows_kernel.  Also the diagonal positions and the longest row.
template <typename T>
__global__ void __launch_bounds__(kBlock) coo_rowsort_kernel(int nrow, const int *__restrict__ rowptr, int *col,
                                                             T *val, int *diag, int *max_row, int *long_rows,
                                                             int *n_long) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int longest = 0;
  for (int64_t kk = warp; kk < nrow; kk += nwarps) {
    const int k = (int)kk;
    const int b = rowptr[k], e = rowptr[k + 1], L = e - b;
    longest = L > longest ? L : longest;
    if (L > 32) {
      if (lane == 0) long_rows[atomicAdd(n_long, 1)] = k;
      continue;
    }
    const bool valid = lane < L;
    const int c = valid ? col[b + lane] : INT_MAX;  // columns are < ncol <= INT_MAX
    T v = T(0);
    if (valid) v = val[b + lane];
    const unsigned same = __match_any_sync(0xffffffffu, c);
    if (__any_sync(0xffffffffu, valid && __popc(same) > 1)) {
      if (lane == 0) row_selection_sort(k, b, e, col, val, diag);
      __syncwarp();
      continue;
    }
    int r = 0;
    for (int j = 0; j < L; ++j) r += __shfl_sync(0xffffffffu, c, j) < c ? 1 : 0;
    if (valid) {
      col[b + r] = c;
      val[b + r] = v;
    }
    // columns are distinct here, so at most one lane holds the diagonal
    const unsigned dm = __ballot_sync(0xffffffffu, valid && c == k);
    int rd = -1;
    if (dm) rd = __shfl_sync(0xffffffffu, r, __ffs(dm) - 1);
    if (lane == 0) diag[k] = dm ? b + rd : -1;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
  if (lane == 0 && longest > 0) atomicMax(max_row, longest);
}

// Rows longer than 32 entries (from coo_rowsort_kernel's worklist), one warp
// per row: lane l holds entries l, l + 32, ... (up to kMaxQ * 32 = 256) and
// the ranks come from shuffles as above; a repeated column or a longer row
// takes the selection sort (lane 0).
constexpr int kMaxQ = 8;

template <typename T>
__global__ void __launch_bounds__(kBlock) coo_long_rows_kernel(const int *__restrict__ rowptr, int *col, T *val,
                                                               int *diag, const int *__restrict__ long_rows,
                                                               const int *__restrict__ n_long) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int count = *n_long;
  for (int64_t w = warp; w < count; w += nwarps) {
    const int k = long_rows[w];
    const int b = rowptr[k], e = rowptr[k + 1], L = e - b;
    if (L > kMaxQ * 32) {
      if (lane == 0) row_selection_sort(k, b, e, col, val, diag);
      __syncwarp();
      continue;
    }
    const int nq = (L + 31) >> 5;
    int c[kMaxQ], rank[kMaxQ];
    T v[kMaxQ];
#pragma unroll
    for (int q = 0; q < kMaxQ; ++q) {
      const int i = q * 32 + lane;
      const bool ok = q < nq && i < L;
      c[q] = ok ? col[b + i] : INT_MAX;
      v[q] = ok ? val[b + i] : T(0);
      rank[q] = 0;
    }
    bool dup = false;
#pragma unroll
    for (int qj = 0; qj < kMaxQ; ++qj) {
      if (qj >= nq) break;
      const int jn = L - qj * 32 < 32 ? L - qj * 32 : 32;
      for (int jl = 0; jl < jn; ++jl) {
        const int cj = __shfl_sync(0xffffffffu, c[qj], jl);
#pragma unroll
        for (int q = 0; q < kMaxQ; ++q)
          if (q < nq && q * 32 + lane < L) {
            rank[q] += cj < c[q] ? 1 : 0;
            dup |= cj == c[q] && !(qj == q && jl == lane);
          }
      }
    }
    if (__any_sync(0xffffffffu, dup)) {
      __syncwarp();
      if (lane == 0) row_selection_sort(k, b, e, col, val, diag);
      __syncwarp();
      continue;
    }
    __syncwarp();
    int d = INT_MAX;
#pragma unroll
    for (int q = 0; q < kMaxQ; ++q) {
      const int i = q * 32 + lane;
      if (q < nq && i < L) {
        col[b + rank[q]] = c[q];
        val[b + rank[q]] = v[q];
        if (c[q] == k) d = b + rank[q];
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = min(d, __shfl_xor_sync(0xffffffffu, d, o));
    if (lane == 0) diag[k] = d == INT_MAX ? -1 : d;
  }
}

static int grid_1d(b200la_ctx c, int64_t work) {
  int64_t g = (work + kBlock - 1) / kBlock;
  const int64_t cap = (int64_t)c->num_sms * 16;
  if (g > cap) g = cap;
  return (int)(g < 1 ? 1 : g);
}

// Number of bits that hold values 0 .. n-1.
static int bits_for(int n) {
  int b = 1;
  while (b < 31 && (1LL << b) < (long long)n) ++b;
  return b;
}

}  // namespace b200la

using namespace b200la;

extern "C" int b200la_coo_upload(b200la_ctx c, int nrow, int ncol, int64_t nnz, const int *rows, const int *cols,
                                 const void *val, int val_dtype, int dtype, int device_input, b200la_mat *out) {
  B_CHECK(c && out, B200LA_ERR_INVALID, "coo_upload: null argument");
  B_CHECK(nrow >= 0 && ncol >= 0, B200LA_ERR_INVALID, "coo_upload: negative size %d x %d", nrow, ncol);
  B_CHECK(nnz >= 0 && nnz <= INT_MAX, B200LA_ERR_INVALID, "coo_upload: nnz %lld not in [0, 2^31)", (long long)nnz);
  B_CHECK(dtype == B200LA_F64 || dtype == B200LA_F32, B200LA_ERR_DTYPE, "coo_upload: dtype %d", dtype);
  B_CHECK(val_dtype == B200LA_F64 || val_dtype == B200LA_F32, B200LA_ERR_DTYPE, "coo_upload: value dtype %d",
          val_dtype);
  B_CHECK(nnz == 0 || (rows && cols && val), B200LA_ERR_INVALID, "coo_upload: null triplet arrays");
  cudaStream_t s = c->stream;
  const size_t nz = (size_t)(nnz > 0 ? nnz : 1);
  const size_t vsz = dtype_size(val_dtype);
  // scratch: device triplets (when given host arrays), sorted rows, permutation
  int *d_rows = nullptr, *d_cols = nullptr, *srow = nullptr;
  unsigned long long *idx = nullptr, *perm = nullptr;  // sort payload in and out
  void *d_vals = nullptr, *cub_tmp = nullptr;
  unsigned long long *bad = nullptr;
  int *max_row_d = nullptr, *n_long_d = nullptr, *long_rows = nullptr;
  b200la_mat m = new b200la_mat_s();
  m->ctx = c;
  m->nrow = nrow;
  m->ncol = ncol;
  m->nnz = nnz;
  m->dtype = dtype;
  int rc = B200LA_OK;
  auto cu = [&](cudaError_t e, const char *what) {
    if (e != cudaSuccess && rc == B200LA_OK)
      rc = fail(e == cudaErrorMemoryAllocation ? B200LA_ERR_NOMEM : B200LA_ERR_CUDA, "coo_upload: %s: %s", what,
                cudaGetErrorString(e));
    return rc == B200LA_OK;
  };
  do {
    if (!cu(cudaMallocAsync(&m->rowptr, sizeof(int) * ((size_t)nrow + 1), s), "allocation") ||
        !cu(cudaMallocAsync(&m->col, sizeof(int) * nz, s), "allocation") ||
        !cu(cudaMallocAsync(&m->val, dtype_size(dtype) * nz, s), "allocation") ||
        !cu(cudaMallocAsync(&m->diag, sizeof(int) * (size_t)(nrow > 0 ? nrow : 1), s), "allocation") ||
        !cu(cudaMallocAsync(&bad, sizeof(unsigned long long) + 2 * sizeof(int), s), "allocation"))
      break;
    max_row_d = reinterpret_cast<int *>(bad + 1);
    n_long_d = max_row_d + 1;
    const unsigned long long none = ~0ull;
    if (!cu(cudaMemcpyAsync(bad, &none, sizeof(none), cudaMemcpyHostToDevice, s), "copy") ||
        !cu(cudaMemsetAsync(max_row_d, 0, 2 * sizeof(int), s), "memset"))
      break;
    if (nnz == 0) {
      if (!cu(cudaMemsetAsync(m->rowptr, 0, sizeof(int) * ((size_t)nrow + 1), s), "memset")) break;
      if (nrow > 0 && !cu(cudaMemsetAsync(m->diag, 0xff, sizeof(int) * (size_t)nrow, s), "memset")) break;
      break;
    }
    const int *r_in = rows, *c_in = cols;
    const void *v_in = val;
    if (!device_input) {
      if (!cu(cudaMallocAsync(&d_rows, sizeof(int) * nz, s), "allocation") ||
          !cu(cudaMallocAsync(&d_cols, sizeof(int) * nz, s), "allocation") ||
          !cu(cudaMallocAsync(&d_vals, vsz * nz, s), "allocation") ||
          !cu(cudaMemcpyAsync(d_rows, rows, sizeof(int) * nnz, cudaMemcpyHostToDevice, s), "copy") ||
          !cu(cudaMemcpyAsync(d_cols, cols, sizeof(int) * nnz, cudaMemcpyHostToDevice, s), "copy") ||
          !cu(cudaMemcpyAsync(d_vals, val, vsz * nnz, cudaMemcpyHostToDevice, s), "copy"))
        break;
      r_in = d_rows;
      c_in = d_cols;
      v_in = d_vals;
    }
    const int g = grid_1d(c, nnz);
    coo_check_kernel<<<g, kBlock, 0, s>>>(nnz, nrow, ncol, r_in, c_in, bad);
    unsigned long long hbad = 0;
    if (!cu(cudaGetLastError(), "check") ||
        !cu(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, s), "copy") ||
        !cu(cudaStreamSynchronize(s), "check"))
      break;
    if (hbad != ~0ull) {
      rc = fail(B200LA_ERR_MATRIX, "coo_upload: triplet %llu has an index out of range", hbad);
      break;
    }
    // stable sort by row: keys rows, values input positions
    if (!cu(cudaMallocAsync(&srow, sizeof(int) * nz, s), "allocation") ||
        !cu(cudaMallocAsync(&idx, sizeof(unsigned long long) * nz, s), "allocation") ||
        !cu(cudaMallocAsync(&perm, sizeof(unsigned long long) * nz, s), "allocation"))
      break;
    coo_pack_kernel<<<g, kBlock, 0, s>>>(nnz, c_in, idx);
    size_t tmp_bytes = 0;
    const int end_bit = bits_for(nrow);
    if (!cu(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, r_in, srow, idx, perm, (int)nnz, 0, end_bit, s),
            "sort size") ||
        !cu(cudaMallocAsync(&cub_tmp, tmp_bytes > 0 ? tmp_bytes : 1, s), "allocation") ||
        !cu(cub::DeviceRadixSort::SortPairs(cub_tmp, tmp_bytes, r_in, srow, idx, perm, (int)nnz, 0, end_bit, s),
            "sort"))
      break;
    coo_rowptr_kernel<<<grid_1d(c, nnz + 1), kBlock, 0, s>>>(nnz, nrow, srow, m->rowptr);
    if (dtype == B200LA_F64) {
      if (val_dtype == B200LA_F64)
        coo_gather_kernel<double, double><<<g, kBlock, 0, s>>>(nnz, perm, (const double *)v_in, m->col,
                                                               (double *)m->val);
      else
        coo_gather_kernel<double, float><<<g, kBlock, 0, s>>>(nnz, perm, (const float *)v_in, m->col,
                                                              (double *)m->val);
    } else {
      if (val_dtype == B200LA_F64)
        coo_gather_kernel<float, double><<<g, kBlock, 0, s>>>(nnz, perm, (const double *)v_in, m->col,
                                                              (float *)m->val);
      else
        coo_gather_kernel<float, float><<<g, kBlock, 0, s>>>(nnz, perm, (const float *)v_in, m->col,
                                                             (float *)m->val);
    }
    if (nrow > 0) {
      if (!cu(cudaMallocAsync(&long_rows, sizeof(int) * (size_t)nrow, s), "allocation")) break;
      const int gr = grid_1d(c, (int64_t)nrow * 32);
      if (dtype == B200LA_F64) {
        coo_rowsort_kernel<double><<<gr, kBlock, 0, s>>>(nrow, m->rowptr, m->col, (double *)m->val, m->diag,
                                                         max_row_d, long_rows, n_long_d);
        coo_long_rows_kernel<double><<<c->num_sms * 8, kBlock, 0, s>>>(m->rowptr, m->col, (double *)m->val,
                                                                       m->diag, long_rows, n_long_d);
      } else {
        coo_rowsort_kernel<float><<<gr, kBlock, 0, s>>>(nrow, m->rowptr, m->col, (float *)m->val, m->diag,
                                                        max_row_d, long_rows, n_long_d);
        coo_long_rows_kernel<float><<<c->num_sms * 8, kBlock, 0, s>>>(m->rowptr, m->col, (float *)m->val, m->diag,
                                                                      long_rows, n_long_d);
      }
    }
    cu(cudaGetLastError(), "kernels");
  } while (false);
  int hmax = 0;
  if (rc == B200LA_OK && bad) {
    cu(cudaMemcpyAsync(&hmax, max_row_d, sizeof(int), cudaMemcpyDeviceToHost, s), "copy");
    cu(cudaStreamSynchronize(s), "sync");
  }
  void *scratch[] = {d_rows, d_cols, d_vals, srow, idx, perm, cub_tmp, bad, long_rows};
  for (void *p : scratch)
    if (p) cudaFreeAsync(p, s);
  if (rc != B200LA_OK) {
    cudaStreamSynchronize(s);
    b200la_mat_destroy(m);
    return rc;
  }
  m->max_row = hmax;
  const double avg = nrow ? (double)nnz / nrow : 0.0;
  m->format = B200LA_FMT_CSR;
  m->param = avg <= 3 ? 2 : avg <= 6 ? 4 : avg <= 14 ? 8 : avg <= 40 ? 16 : 32;
  *out = m;
  return B200LA_OK;
}

// CopyTo a host CSR: the uploaded (or built) CSR arrays as stored.
extern "C" int b200la_mat_download(b200la_mat m, int *rowptr, int *col, void *val) {
  B_CHECK(m && rowptr && (m->nnz == 0 || (col && val)), B200LA_ERR_INVALID, "mat_download: null argument");
  cudaStream_t s = m->ctx->stream;
  B_CUDA(cudaMemcpyAsync(rowptr, m->rowptr, sizeof(int) * ((size_t)m->nrow + 1), cudaMemcpyDeviceToHost, s));
  if (m->nnz) {
    B_CUDA(cudaMemcpyAsync(col, m->col, sizeof(int) * (size_t)m->nnz, cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaMemcpyAsync(val, m->val, dtype_size(m->dtype) * (size_t)m->nnz, cudaMemcpyDeviceToHost, s));
  }
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}
