// Context, vectors, matrices, BLAS-1 and SpMV of the b200la C ABI.
//
// Replaces the reference's lmp GPU backend (lmp/cuda/: lvector_gpu.cc,
// GPUblas_lvector.cu, lmatrix_csr_gpu.cc, GPUscalar_csr_lmatrix.cu,
// mem_cuda.cu).  Differences by design: every call returns a status instead
// of exit(-1); reductions are deterministic two-level grid sums instead of
// cuBLAS; ScaleAdd is one pass instead of Dscal + Daxpy
// (GPUblas_lvector.cu:341-380); the SpMV assigns a group of lanes (or a SELL
// slice) per row with coalesced streaming loads instead of one thread per
// row (cuda_spmv_kernel_csr_scalar.h:22-33).
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.cuh"
#include "spmv.cuh"

namespace b200la {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int grid_for(b200la_ctx ctx, const void *kernel, int64_t work_items, int items_per_block, int *grid) {
  int per_sm = 0;
  B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
  if (per_sm < 1) per_sm = 1;
  int64_t need = (work_items + items_per_block - 1) / items_per_block;
  int64_t cap = (int64_t)ctx->num_sms * per_sm;
  if (cap > kMaxReduceBlocks) cap = kMaxReduceBlocks;
  int64_t g = need < cap ? need : cap;
  *grid = (int)(g < 1 ? 1 : g);
  return B200LA_OK;
}

// ---------------------------------------------------------------- BLAS-1 kernels
// Element-wise kernels process 16-byte vectors (double2 / float4) with a
// grid-stride loop; the ragged tail is handled element by element.

template <typename T, typename F>
__device__ __forceinline__ void for_each_vec(int64_t n, F f) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) f.vec(i);
  for (int64_t i = nv * W + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) f.one(i);
}

template <typename T> struct AxpyF {
  T *y; const T *x; T a;
  __device__ void vec(int64_t i) {
    using V = typename Vec16<T>::type;
    V vy = reinterpret_cast<V *>(y)[i];
    V vx = reinterpret_cast<const V *>(x)[i];
    T *py = reinterpret_cast<T *>(&vy);
    const T *px = reinterpret_cast<const T *>(&vx);
#pragma unroll
    for (int k = 0; k < Vec16<T>::n; ++k) py[k] = fma(a, px[k], py[k]);
    reinterpret_cast<V *>(y)[i] = vy;
  }
  __device__ void one(int64_t i) { y[i] = fma(a, x[i], y[i]); }
};

template <typename T> struct ScaleAddF {
  T *y; const T *x; T a;
  __device__ void vec(int64_t i) {
    using V = typename Vec16<T>::type;
    V vy = reinterpret_cast<V *>(y)[i];
    V vx = reinterpret_cast<const V *>(x)[i];
    T *py = reinterpret_cast<T *>(&vy);
    const T *px = reinterpret_cast<const T *>(&vx);
#pragma unroll
    for (int k = 0; k < Vec16<T>::n; ++k) py[k] = fma(a, py[k], px[k]);
    reinterpret_cast<V *>(y)[i] = vy;
  }
  __device__ void one(int64_t i) { y[i] = fma(a, y[i], x[i]); }
};

template <typename T> struct ScaleF {
  T *y; T a;
  __device__ void vec(int64_t i) {
    using V = typename Vec16<T>::type;
    V vy = reinterpret_cast<V *>(y)[i];
    T *py = reinterpret_cast<T *>(&vy);
#pragma unroll
    for (int k = 0; k < Vec16<T>::n; ++k) py[k] *= a;
    reinterpret_cast<V *>(y)[i] = vy;
  }
  __device__ void one(int64_t i) { y[i] *= a; }
};

template <typename T> struct MulF {
  T *y; const T *x;
  __device__ void vec(int64_t i) {
    using V = typename Vec16<T>::type;
    V vy = reinterpret_cast<V *>(y)[i];
    V vx = reinterpret_cast<const V *>(x)[i];
    T *py = reinterpret_cast<T *>(&vy);
    const T *px = reinterpret_cast<const T *>(&vx);
#pragma unroll
    for (int k = 0; k < Vec16<T>::n; ++k) py[k] *= px[k];
    reinterpret_cast<V *>(y)[i] = vy;
  }
  __device__ void one(int64_t i) { y[i] *= x[i]; }
};

template <typename T, typename F>
__global__ void __launch_bounds__(kBlock) elementwise_kernel(int64_t n, F f) {
  for_each_vec<T>(n, f);
}

template <typename D, typename S>
__global__ void __launch_bounds__(kBlock) cast_kernel(int64_t n, D *__restrict__ d, const S *__restrict__ s) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) d[i] = (D)s[i];
}

// dst[i] = src[i] (add = 0) or dst[i] += w * src[i] over a sub-range at
// arbitrary offsets (no vector loads: the ranges need not be aligned)
template <typename T>
__global__ void __launch_bounds__(kBlock) range_kernel(int64_t n, T *__restrict__ dst, const T *__restrict__ src,
                                                       int add, T w) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = add ? fma(w, src[i], dst[i]) : src[i];
}

// Halo exchange of a row-partitioned vector (CoupledVector::SendBorder /
// ReceiveGhost, linear_algebra/coupled_vector.cc:890-973): gather the owned
// values peers read into a contiguous device buffer, scatter received values
// into the ghost vector.  idx is a device int32 array of n positions.
template <typename T>
__global__ void __launch_bounds__(kBlock) gather_kernel(int64_t n, const int *__restrict__ idx,
                                                        const T *__restrict__ src, T *__restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) out[k] = src[__ldg(idx + k)];
}

template <typename T>
__global__ void __launch_bounds__(kBlock) scatter_kernel(int64_t n, const int *__restrict__ idx,
                                                         const T *__restrict__ in, T *__restrict__ dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) dst[__ldg(idx + k)] = in[k];
}

// Dot product: per-thread accumulation (Acc<T>), then the deterministic grid
// sum; the last block writes the total to result[0].
template <typename T>
__global__ void __launch_bounds__(kBlock) dot_kernel(int64_t n, const T *__restrict__ a, const T *__restrict__ b,
                                                     double *part, unsigned *ticket, double *result) {
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::n;
  Acc<T> acc;
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
    V va = __ldg(reinterpret_cast<const V *>(a) + i);
    V vb = __ldg(reinterpret_cast<const V *>(b) + i);
    const T *pa = reinterpret_cast<const T *>(&va);
    const T *pb = reinterpret_cast<const T *>(&vb);
#pragma unroll
    for (int k = 0; k < W; ++k) acc.add(pa[k] * pb[k]);
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    acc.add(a[i] * b[i]);
  double v[1] = {acc.value()};
  if (grid_sum_last<1>(v, part, ticket) && threadIdx.x == 0) result[0] = v[0];
}


template <typename T>
__global__ void indexed_kernel(int n, const int *__restrict__ idx, T *__restrict__ buf, const T *vals,
                               T *out, int set) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (set) buf[idx[i]] = vals[i];
  else out[i] = buf[idx[i]];
}

// Position of the diagonal entry of each row (diag_ptr_ of
// CPU_CSR_lMatrix, set by get_diag_ptr, lmp/lmatrix_csr_cpu.cc:899-904).
__global__ void find_diag_kernel(int n, const int *__restrict__ rowptr, const int *__restrict__ col,
                                 int *__restrict__ diag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = -1;
  for (int j = rowptr[i]; j < rowptr[i + 1]; ++j)
    if (col[j] == i) { k = j; break; }
  diag[i] = k;
}

template <typename T>
__global__ void inv_diag_kernel(int n, const int *__restrict__ diag, const T *__restrict__ val, T *__restrict__ out,
                                unsigned *bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = diag[i];
  T a = k >= 0 ? val[k] : T(0);
  if (a == T(0)) {
    atomicMin(bad, (unsigned)i);
    out[i] = T(0);
  } else {
    out[i] = T(1) / a;
  }
}

template <typename T>
__global__ void zero_rows_kernel(int n, const int *__restrict__ rows, const int *__restrict__ rowptr,
                                 const int *__restrict__ col, T *__restrict__ val, T alpha) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int r = rows[i];
  for (int j = rowptr[r]; j < rowptr[r + 1]; ++j) val[j] = (col[j] == r) ? alpha : T(0);
}

template <typename T>
static int launch_dot(b200la_ctx c, int64_t n, const T *a, const T *b, double *out) {
  int grid;
  B_TRY(grid_for(c, (const void *)dot_kernel<T>, (n + Vec16<T>::n - 1) / Vec16<T>::n, kBlock, &grid));
  dot_kernel<T><<<grid, kBlock, 0, c->stream>>>(n, a, b, c->scratch.part, c->scratch.ticket, c->scratch.result);
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaMemcpyAsync(c->host_result, c->scratch.result, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  B_CUDA(cudaStreamSynchronize(c->stream));
  *out = c->host_result[0];
  return B200LA_OK;
}

template <typename T, typename F>
static int launch_ew(b200la_ctx c, int64_t n, F f) {
  if (n == 0) return B200LA_OK;
  int grid;
  B_TRY(grid_for(c, (const void *)elementwise_kernel<T, F>, (n + Vec16<T>::n - 1) / Vec16<T>::n, kBlock, &grid));
  elementwise_kernel<T, F><<<grid, kBlock, 0, c->stream>>>(n, f);
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

int validate_csr(int nrow, int ncol, int64_t nnz, const int *rowptr, const int *col, int *max_row) {
  B_CHECK(nrow >= 0 && ncol >= 0 && nnz >= 0, B200LA_ERR_MATRIX, "csr: negative dimension");
  B_CHECK(nnz < (int64_t)INT32_MAX, B200LA_ERR_MATRIX, "csr: nnz %lld exceeds int32 indexing", (long long)nnz);
  B_CHECK(rowptr, B200LA_ERR_MATRIX, "csr: rowptr is NULL");
  B_CHECK(rowptr[0] == 0, B200LA_ERR_MATRIX, "csr: rowptr[0] = %d, expected 0", rowptr[0]);
  int mr = 0;
  for (int i = 0; i < nrow; ++i) {
    int len = rowptr[i + 1] - rowptr[i];
    B_CHECK(len >= 0, B200LA_ERR_MATRIX, "csr: rowptr decreases at row %d", i);
    if (len > mr) mr = len;
  }
  B_CHECK(rowptr[nrow] == nnz, B200LA_ERR_MATRIX, "csr: rowptr[nrow] = %d != nnz %lld", rowptr[nrow], (long long)nnz);
  B_CHECK(nnz == 0 || col, B200LA_ERR_MATRIX, "csr: col is NULL");
  for (int64_t j = 0; j < nnz; ++j)
    B_CHECK(col[j] >= 0 && col[j] < ncol, B200LA_ERR_MATRIX, "csr: col[%lld] = %d out of range [0,%d)",
            (long long)j, col[j], ncol);
  *max_row = mr;
  return B200LA_OK;
}

}  // namespace b200la

using namespace b200la;

// ================================================================ C ABI
extern "C" {

const char *b200la_version(void) { return "b200la 0.1 (sm_100a)"; }
const char *b200la_last_error(void) { return g_last_error.c_str(); }

int b200la_ctx_create(int device, b200la_ctx *out) {
  B_CHECK(out, B200LA_ERR_INVALID, "ctx_create: out is NULL");
  int ndev = 0;
  B_CUDA(cudaGetDeviceCount(&ndev));
  B_CHECK(device >= 0 && device < ndev, B200LA_ERR_INVALID, "ctx_create: device %d of %d", device, ndev);
  B_CUDA(cudaSetDevice(device));
  b200la_ctx c = new b200la_ctx_s();
  c->device = device;
  B_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
  B_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
  c->stream = c->own_stream;
  {
    const char *g = getenv("B200LA_GRAPHS");
    c->use_graphs = !(g && g[0] == '0');
  }
  B_CUDA(cudaMalloc(&c->scratch.part, sizeof(double) * 4 * kMaxReduceBlocks));
  B_CUDA(cudaMalloc(&c->scratch.ticket, sizeof(unsigned) * 16));
  B_CUDA(cudaMalloc(&c->scratch.result, sizeof(double) * 8));
  B_CUDA(cudaMemset(c->scratch.ticket, 0, sizeof(unsigned) * 16));
  B_CUDA(cudaMallocHost(&c->host_result, sizeof(double) * 8));
  // Stream-ordered allocations (batch slots, tile lists, scratch) come from
  // the device's default pool.  Keep freed blocks in the pool instead of
  // returning them to the driver at every synchronisation, so adding and
  // removing systems in a loop reuses memory rather than remapping it.  The
  // attribute lives only in this process; batches trim the pool when they
  // are destroyed.
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  *out = c;
  return B200LA_OK;
}

int b200la_ctx_destroy(b200la_ctx c) {
  if (!c) return B200LA_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaFree(c->scratch.part);
  cudaFree(c->scratch.ticket);
  cudaFree(c->scratch.result);
  cudaFreeHost(c->host_result);
  cudaStreamDestroy(c->own_stream);
  delete c;
  return B200LA_OK;
}

int b200la_ctx_set_stream(b200la_ctx c, void *stream) {
  B_CHECK(c, B200LA_ERR_INVALID, "ctx_set_stream: null ctx");
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return B200LA_OK;
}

int b200la_ctx_get_stream(b200la_ctx c, void **stream) {
  B_CHECK(c && stream, B200LA_ERR_INVALID, "ctx_get_stream: null argument");
  *stream = (void *)c->stream;
  return B200LA_OK;
}

int b200la_ctx_set_graphs(b200la_ctx c, int on) {
  B_CHECK(c, B200LA_ERR_INVALID, "ctx_set_graphs: null ctx");
  c->use_graphs = on != 0;
  return B200LA_OK;
}

int b200la_ctx_synchronize(b200la_ctx c) {
  B_CHECK(c, B200LA_ERR_INVALID, "ctx_synchronize: null ctx");
  B_CUDA(cudaStreamSynchronize(c->stream));
  return B200LA_OK;
}

int b200la_ctx_num_sms(b200la_ctx c, int *out) {
  B_CHECK(c && out, B200LA_ERR_INVALID, "ctx_num_sms: null argument");
  *out = c->num_sms;
  return B200LA_OK;
}

// ---------------------------------------------------------------- vectors
int b200la_vec_create(b200la_ctx c, int64_t n, int dtype, b200la_vec *out) {
  B_CHECK(c && out, B200LA_ERR_INVALID, "vec_create: null argument");
  B_CHECK(n >= 0, B200LA_ERR_INVALID, "vec_create: negative size %lld", (long long)n);
  B_CHECK(dtype_ok(dtype), B200LA_ERR_DTYPE, "vec_create: dtype %d", dtype);
  void *d = nullptr;
  size_t bytes = (size_t)(n > 0 ? n : 1) * dtype_size(dtype);
  B_CUDA(cudaMallocAsync(&d, bytes, c->stream));
  B_CUDA(cudaMemsetAsync(d, 0, bytes, c->stream));
  b200la_vec v = new b200la_vec_s{c, n, dtype, d, true};
  *out = v;
  return B200LA_OK;
}

int b200la_vec_wrap(b200la_ctx c, int64_t n, int dtype, void *ptr, b200la_vec *out) {
  B_CHECK(c && out && (ptr || n == 0), B200LA_ERR_INVALID, "vec_wrap: null argument");
  B_CHECK(dtype_ok(dtype), B200LA_ERR_DTYPE, "vec_wrap: dtype %d", dtype);
  B_CHECK(((uintptr_t)ptr & 15) == 0, B200LA_ERR_INVALID, "vec_wrap: device pointer must be 16-byte aligned");
  *out = new b200la_vec_s{c, n, dtype, ptr, false};
  return B200LA_OK;
}

int b200la_vec_destroy(b200la_vec v) {
  if (!v) return B200LA_OK;
  if (v->owned && v->d) cudaFreeAsync(v->d, v->ctx->stream);
  delete v;
  return B200LA_OK;
}

int b200la_vec_info(b200la_vec v, int64_t *n, int *dtype, void **ptr) {
  B_CHECK(v, B200LA_ERR_INVALID, "vec_info: null vector");
  if (n) *n = v->n;
  if (dtype) *dtype = v->dtype;
  if (ptr) *ptr = v->d;
  return B200LA_OK;
}

int b200la_vec_upload(b200la_vec v, const void *host, int64_t n) {
  B_CHECK(v && (host || n == 0), B200LA_ERR_INVALID, "vec_upload: null argument");
  B_CHECK(n == v->n, B200LA_ERR_INVALID, "vec_upload: size %lld != vector size %lld", (long long)n,
          (long long)v->n);
  if (n == 0) return B200LA_OK;
  B_CUDA(cudaMemcpyAsync(v->d, host, (size_t)n * dtype_size(v->dtype), cudaMemcpyHostToDevice, v->ctx->stream));
  B_CUDA(cudaStreamSynchronize(v->ctx->stream));
  return B200LA_OK;
}

int b200la_vec_download(b200la_vec v, void *host, int64_t n) {
  B_CHECK(v && (host || n == 0), B200LA_ERR_INVALID, "vec_download: null argument");
  B_CHECK(n == v->n, B200LA_ERR_INVALID, "vec_download: size %lld != vector size %lld", (long long)n,
          (long long)v->n);
  if (n == 0) return B200LA_OK;
  B_CUDA(cudaMemcpyAsync(host, v->d, (size_t)n * dtype_size(v->dtype), cudaMemcpyDeviceToHost, v->ctx->stream));
  B_CUDA(cudaStreamSynchronize(v->ctx->stream));
  return B200LA_OK;
}

static int indexed_op(b200la_vec v, const int *index, void *values, int size, int set) {
  B_CHECK(v && (size == 0 || (index && values)), B200LA_ERR_INVALID, "vec_set/get_values: null argument");
  B_CHECK(size >= 0, B200LA_ERR_INVALID, "vec_set/get_values: negative size");
  if (size == 0) return B200LA_OK;
  for (int i = 0; i < size; ++i)
    B_CHECK(index[i] >= 0 && index[i] < v->n, B200LA_ERR_INVALID, "vec_set/get_values: index %d out of range",
            index[i]);
  cudaStream_t s = v->ctx->stream;
  size_t es = dtype_size(v->dtype);
  int *d_idx = nullptr;
  void *d_val = nullptr;
  B_CUDA(cudaMallocAsync(&d_idx, sizeof(int) * size, s));
  B_CUDA(cudaMallocAsync(&d_val, es * size, s));
  B_CUDA(cudaMemcpyAsync(d_idx, index, sizeof(int) * size, cudaMemcpyHostToDevice, s));
  if (set) B_CUDA(cudaMemcpyAsync(d_val, values, es * size, cudaMemcpyHostToDevice, s));
  int grid = (size + kBlock - 1) / kBlock;
  if (v->dtype == B200LA_F64)
    indexed_kernel<double><<<grid, kBlock, 0, s>>>(size, d_idx, (double *)v->d, (const double *)d_val,
                                                   (double *)d_val, set);
  else
    indexed_kernel<float><<<grid, kBlock, 0, s>>>(size, d_idx, (float *)v->d, (const float *)d_val,
                                                  (float *)d_val, set);
  B_CUDA(cudaGetLastError());
  if (!set) B_CUDA(cudaMemcpyAsync(values, d_val, es * size, cudaMemcpyDeviceToHost, s));
  B_CUDA(cudaFreeAsync(d_idx, s));
  B_CUDA(cudaFreeAsync(d_val, s));
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}

int b200la_vec_set_values(b200la_vec v, const int *index, const void *values, int size) {
  return indexed_op(v, index, const_cast<void *>(values), size, 1);
}

int b200la_vec_get_values(b200la_vec v, const int *index, void *values, int size) {
  return indexed_op(v, index, values, size, 0);
}

int b200la_vec_zeros(b200la_vec v) {
  B_CHECK(v, B200LA_ERR_INVALID, "vec_zeros: null vector");
  if (v->n) B_CUDA(cudaMemsetAsync(v->d, 0, (size_t)v->n * dtype_size(v->dtype), v->ctx->stream));
  return B200LA_OK;
}

static int check_pair(b200la_vec a, b200la_vec b, const char *what, bool same_dtype = true) {
  B_CHECK(a && b, B200LA_ERR_INVALID, "%s: null vector", what);
  B_CHECK(a->n == b->n, B200LA_ERR_INVALID, "%s: size mismatch %lld vs %lld", what, (long long)a->n,
          (long long)b->n);
  if (same_dtype) B_CHECK(a->dtype == b->dtype, B200LA_ERR_DTYPE, "%s: dtype mismatch", what);
  return B200LA_OK;
}

int b200la_vec_copy(b200la_vec dst, b200la_vec src) {
  B_TRY(check_pair(dst, src, "vec_copy"));
  if (dst->n && dst->d != src->d)
    B_CUDA(cudaMemcpyAsync(dst->d, src->d, (size_t)dst->n * dtype_size(dst->dtype), cudaMemcpyDeviceToDevice,
                           dst->ctx->stream));
  return B200LA_OK;
}

int b200la_vec_cast(b200la_vec dst, b200la_vec src) {
  B_TRY(check_pair(dst, src, "vec_cast", false));
  if (dst->dtype == src->dtype) return b200la_vec_copy(dst, src);
  if (!dst->n) return B200LA_OK;
  int grid;
  cudaStream_t s = dst->ctx->stream;
  if (dst->dtype == B200LA_F32) {
    B_TRY(grid_for(dst->ctx, (const void *)cast_kernel<float, double>, dst->n, kBlock, &grid));
    cast_kernel<float, double><<<grid, kBlock, 0, s>>>(dst->n, (float *)dst->d, (const double *)src->d);
  } else {
    B_TRY(grid_for(dst->ctx, (const void *)cast_kernel<double, float>, dst->n, kBlock, &grid));
    cast_kernel<double, float><<<grid, kBlock, 0, s>>>(dst->n, (double *)dst->d, (const float *)src->d);
  }
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

int b200la_vec_dot(b200la_vec a, b200la_vec b, double *out) {
  B_TRY(check_pair(a, b, "vec_dot"));
  B_CHECK(out, B200LA_ERR_INVALID, "vec_dot: out is NULL");
  if (a->n == 0) { *out = 0.0; return B200LA_OK; }
  if (a->dtype == B200LA_F64) return launch_dot<double>(a->ctx, a->n, (const double *)a->d, (const double *)b->d, out);
  return launch_dot<float>(a->ctx, a->n, (const float *)a->d, (const float *)b->d, out);
}

int b200la_vec_norm2(b200la_vec v, double *out) {
  double d = 0.0;
  B_TRY(b200la_vec_dot(v, v, &d));
  *out = sqrt(d);
  return B200LA_OK;
}

int b200la_vec_axpy(b200la_vec y, b200la_vec x, double a) {
  B_TRY(check_pair(y, x, "vec_axpy"));
  if (y->dtype == B200LA_F64) return launch_ew<double>(y->ctx, y->n, AxpyF<double>{(double *)y->d, (const double *)x->d, a});
  return launch_ew<float>(y->ctx, y->n, AxpyF<float>{(float *)y->d, (const float *)x->d, (float)a});
}

int b200la_vec_scaleadd(b200la_vec y, double a, b200la_vec x) {
  B_TRY(check_pair(y, x, "vec_scaleadd"));
  if (y->dtype == B200LA_F64)
    return launch_ew<double>(y->ctx, y->n, ScaleAddF<double>{(double *)y->d, (const double *)x->d, a});
  return launch_ew<float>(y->ctx, y->n, ScaleAddF<float>{(float *)y->d, (const float *)x->d, (float)a});
}

int b200la_vec_range_update(b200la_vec dst, int64_t dst_start, b200la_vec src, int64_t src_start, int64_t n,
                            int add, double weight) {
  B_CHECK(dst && src, B200LA_ERR_INVALID, "vec_range_update: null vector");
  B_CHECK(dst->dtype == src->dtype, B200LA_ERR_DTYPE, "vec_range_update: dtype mismatch");
  B_CHECK(n >= 0 && dst_start >= 0 && src_start >= 0 && dst_start + n <= dst->n && src_start + n <= src->n,
          B200LA_ERR_INVALID, "vec_range_update: range [%lld,+%lld) / [%lld,+%lld) outside %lld / %lld",
          (long long)dst_start, (long long)n, (long long)src_start, (long long)n, (long long)dst->n,
          (long long)src->n);
  if (n == 0) return B200LA_OK;
  b200la_ctx c = dst->ctx;
  int grid;
  if (dst->dtype == B200LA_F64) {
    B_TRY(grid_for(c, (const void *)range_kernel<double>, n, kBlock, &grid));
    range_kernel<double><<<grid, kBlock, 0, c->stream>>>(n, (double *)dst->d + dst_start,
                                                         (const double *)src->d + src_start, add, weight);
  } else {
    B_TRY(grid_for(c, (const void *)range_kernel<float>, n, kBlock, &grid));
    range_kernel<float><<<grid, kBlock, 0, c->stream>>>(n, (float *)dst->d + dst_start,
                                                        (const float *)src->d + src_start, add, (float)weight);
  }
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

int b200la_vec_gather(b200la_vec src, const int *idx, int64_t n, void *out) {
  B_CHECK(src && (n == 0 || (idx && out)) && n >= 0, B200LA_ERR_INVALID, "vec_gather: bad argument");
  if (n == 0) return B200LA_OK;
  b200la_ctx c = src->ctx;
  int grid;
  if (src->dtype == B200LA_F64) {
    B_TRY(grid_for(c, (const void *)gather_kernel<double>, n, kBlock, &grid));
    gather_kernel<double><<<grid, kBlock, 0, c->stream>>>(n, idx, (const double *)src->d, (double *)out);
  } else {
    B_TRY(grid_for(c, (const void *)gather_kernel<float>, n, kBlock, &grid));
    gather_kernel<float><<<grid, kBlock, 0, c->stream>>>(n, idx, (const float *)src->d, (float *)out);
  }
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

int b200la_vec_scatter(b200la_vec dst, const int *idx, int64_t n, const void *in) {
  B_CHECK(dst && (n == 0 || (idx && in)) && n >= 0, B200LA_ERR_INVALID, "vec_scatter: bad argument");
  if (n == 0) return B200LA_OK;
  b200la_ctx c = dst->ctx;
  int grid;
  if (dst->dtype == B200LA_F64) {
    B_TRY(grid_for(c, (const void *)scatter_kernel<double>, n, kBlock, &grid));
    scatter_kernel<double><<<grid, kBlock, 0, c->stream>>>(n, idx, (const double *)in, (double *)dst->d);
  } else {
    B_TRY(grid_for(c, (const void *)scatter_kernel<float>, n, kBlock, &grid));
    scatter_kernel<float><<<grid, kBlock, 0, c->stream>>>(n, idx, (const float *)in, (float *)dst->d);
  }
  B_CUDA(cudaGetLastError());
  return B200LA_OK;
}

int b200la_vec_scale(b200la_vec y, double a) {
  B_CHECK(y, B200LA_ERR_INVALID, "vec_scale: null vector");
  if (y->dtype == B200LA_F64) return launch_ew<double>(y->ctx, y->n, ScaleF<double>{(double *)y->d, a});
  return launch_ew<float>(y->ctx, y->n, ScaleF<float>{(float *)y->d, (float)a});
}

int b200la_vec_elementwise_mult(b200la_vec y, b200la_vec x) {
  B_TRY(check_pair(y, x, "vec_elementwise_mult"));
  if (y->dtype == B200LA_F64) return launch_ew<double>(y->ctx, y->n, MulF<double>{(double *)y->d, (const double *)x->d});
  return launch_ew<float>(y->ctx, y->n, MulF<float>{(float *)y->d, (const float *)x->d});
}

// ---------------------------------------------------------------- matrices
int b200la_csr_upload(b200la_ctx c, int nrow, int ncol, int64_t nnz, const int *rowptr, const int *col,
                      const void *val, int val_dtype, int dtype, b200la_mat *out) {
  B_CHECK(c && out, B200LA_ERR_INVALID, "csr_upload: null argument");
  B_CHECK(dtype_ok(dtype) && dtype_ok(val_dtype), B200LA_ERR_DTYPE, "csr_upload: dtype");
  B_CHECK(nnz == 0 || val, B200LA_ERR_MATRIX, "csr_upload: val is NULL");
  int max_row = 0;
  B_TRY(validate_csr(nrow, ncol, nnz, rowptr, col, &max_row));
  cudaStream_t s = c->stream;
  b200la_mat m = new b200la_mat_s();
  m->ctx = c;
  m->nrow = nrow;
  m->ncol = ncol;
  m->nnz = nnz;
  m->dtype = dtype;
  m->max_row = max_row;
  size_t nz = (size_t)(nnz > 0 ? nnz : 1);
  B_CUDA(cudaMallocAsync(&m->rowptr, sizeof(int) * (nrow + 1), s));
  B_CUDA(cudaMallocAsync(&m->col, sizeof(int) * nz, s));
  B_CUDA(cudaMallocAsync(&m->val, dtype_size(dtype) * nz, s));
  B_CUDA(cudaMallocAsync(&m->diag, sizeof(int) * (nrow > 0 ? nrow : 1), s));
  B_CUDA(cudaMemcpyAsync(m->rowptr, rowptr, sizeof(int) * (nrow + 1), cudaMemcpyHostToDevice, s));
  if (nnz) {
    B_CUDA(cudaMemcpyAsync(m->col, col, sizeof(int) * nnz, cudaMemcpyHostToDevice, s));
    if (val_dtype == dtype) {
      B_CUDA(cudaMemcpyAsync(m->val, val, dtype_size(dtype) * nnz, cudaMemcpyHostToDevice, s));
    } else {
      void *tmp = nullptr;
      B_CUDA(cudaMallocAsync(&tmp, dtype_size(val_dtype) * nnz, s));
      B_CUDA(cudaMemcpyAsync(tmp, val, dtype_size(val_dtype) * nnz, cudaMemcpyHostToDevice, s));
      int grid = (int)((nnz + kBlock - 1) / kBlock);
      if (grid > 65535 * 4) grid = 65535 * 4;
      if (dtype == B200LA_F32) cast_kernel<float, double><<<grid, kBlock, 0, s>>>(nnz, (float *)m->val, (const double *)tmp);
      else cast_kernel<double, float><<<grid, kBlock, 0, s>>>(nnz, (double *)m->val, (const float *)tmp);
      B_CUDA(cudaGetLastError());
      B_CUDA(cudaFreeAsync(tmp, s));
    }
  }
  if (nrow) {
    find_diag_kernel<<<(nrow + kBlock - 1) / kBlock, kBlock, 0, s>>>(nrow, m->rowptr, m->col, m->diag);
    B_CUDA(cudaGetLastError());
  }
  double avg = nrow ? (double)nnz / nrow : 0.0;
  m->format = B200LA_FMT_CSR;
  m->param = avg <= 3 ? 2 : avg <= 6 ? 4 : avg <= 14 ? 8 : avg <= 40 ? 16 : 32;
  B_CUDA(cudaStreamSynchronize(s));
  *out = m;
  return B200LA_OK;
}

int b200la_mat_destroy(b200la_mat m) {
  if (!m) return B200LA_OK;
  cudaStream_t s = m->ctx->stream;
  cudaFreeAsync(m->rowptr, s);
  cudaFreeAsync(m->col, s);
  cudaFreeAsync(m->val, s);
  cudaFreeAsync(m->diag, s);
  sell_free(m);
  delete m;
  return B200LA_OK;
}

int b200la_mat_info(b200la_mat m, int *nrow, int *ncol, int64_t *nnz, int *dtype) {
  B_CHECK(m, B200LA_ERR_INVALID, "mat_info: null matrix");
  if (nrow) *nrow = m->nrow;
  if (ncol) *ncol = m->ncol;
  if (nnz) *nnz = m->nnz;
  if (dtype) *dtype = m->dtype;
  return B200LA_OK;
}

int b200la_mat_cast(b200la_mat src, int dtype, b200la_mat *out) {
  B_CHECK(src && out, B200LA_ERR_INVALID, "mat_cast: null argument");
  B_CHECK(dtype_ok(dtype), B200LA_ERR_DTYPE, "mat_cast: dtype %d", dtype);
  b200la_ctx c = src->ctx;
  cudaStream_t s = c->stream;
  b200la_mat m = new b200la_mat_s();
  *m = *src;
  m->sell = SellData();
  m->dtype = dtype;
  size_t nz = (size_t)(src->nnz > 0 ? src->nnz : 1);
  B_CUDA(cudaMallocAsync(&m->rowptr, sizeof(int) * (src->nrow + 1), s));
  B_CUDA(cudaMallocAsync(&m->col, sizeof(int) * nz, s));
  B_CUDA(cudaMallocAsync(&m->val, dtype_size(dtype) * nz, s));
  B_CUDA(cudaMallocAsync(&m->diag, sizeof(int) * (src->nrow > 0 ? src->nrow : 1), s));
  B_CUDA(cudaMemcpyAsync(m->rowptr, src->rowptr, sizeof(int) * (src->nrow + 1), cudaMemcpyDeviceToDevice, s));
  B_CUDA(cudaMemcpyAsync(m->col, src->col, sizeof(int) * nz, cudaMemcpyDeviceToDevice, s));
  B_CUDA(cudaMemcpyAsync(m->diag, src->diag, sizeof(int) * (src->nrow > 0 ? src->nrow : 1), cudaMemcpyDeviceToDevice, s));
  if (src->nnz) {
    int grid = (int)((src->nnz + kBlock - 1) / kBlock);
    if (grid > 65535 * 4) grid = 65535 * 4;
    if (dtype == src->dtype)
      B_CUDA(cudaMemcpyAsync(m->val, src->val, dtype_size(dtype) * src->nnz, cudaMemcpyDeviceToDevice, s));
    else if (dtype == B200LA_F32)
      cast_kernel<float, double><<<grid, kBlock, 0, s>>>(src->nnz, (float *)m->val, (const double *)src->val);
    else
      cast_kernel<double, float><<<grid, kBlock, 0, s>>>(src->nnz, (double *)m->val, (const float *)src->val);
    B_CUDA(cudaGetLastError());
  }
  if (is_sliced(m->format)) B_TRY(sliced_rebuild(m, m->format, m->param, src->sell.c, src->sell.sigma));
  B_CUDA(cudaStreamSynchronize(s));
  *out = m;
  return B200LA_OK;
}

int b200la_mat_zero_rows(b200la_mat m, const int *rows, int size, double alpha) {
  B_CHECK(m && (size == 0 || rows), B200LA_ERR_INVALID, "mat_zero_rows: null argument");
  if (size == 0) return B200LA_OK;
  for (int i = 0; i < size; ++i)
    B_CHECK(rows[i] >= 0 && rows[i] < m->nrow, B200LA_ERR_INVALID, "mat_zero_rows: row %d out of range", rows[i]);
  cudaStream_t s = m->ctx->stream;
  int *d_rows = nullptr;
  B_CUDA(cudaMallocAsync(&d_rows, sizeof(int) * size, s));
  B_CUDA(cudaMemcpyAsync(d_rows, rows, sizeof(int) * size, cudaMemcpyHostToDevice, s));
  int grid = (size + kBlock - 1) / kBlock;
  if (m->dtype == B200LA_F64)
    zero_rows_kernel<double><<<grid, kBlock, 0, s>>>(size, d_rows, m->rowptr, m->col, (double *)m->val, alpha);
  else
    zero_rows_kernel<float><<<grid, kBlock, 0, s>>>(size, d_rows, m->rowptr, m->col, (float *)m->val, (float)alpha);
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaFreeAsync(d_rows, s));
  if (is_sliced(m->format)) {
    // the values changed: rebuild the sliced copy with the same geometry
    const int C = m->sell.c, sigma = m->sell.sigma;
    B_TRY(sliced_rebuild(m, m->format, m->param, C, sigma));
  }
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}

static int check_spmv(b200la_mat m, b200la_vec x, b200la_vec y, const char *what) {
  B_CHECK(m && x && y, B200LA_ERR_INVALID, "%s: null argument", what);
  B_CHECK(x->n == m->ncol && y->n == m->nrow, B200LA_ERR_INVALID, "%s: sizes x %lld y %lld vs %dx%d", what,
          (long long)x->n, (long long)y->n, m->nrow, m->ncol);
  B_CHECK(x->dtype == m->dtype && y->dtype == m->dtype, B200LA_ERR_DTYPE, "%s: dtype mismatch", what);
  B_CHECK(x->d != y->d, B200LA_ERR_INVALID, "%s: x and y alias", what);
  return B200LA_OK;
}

int b200la_spmv(b200la_mat m, b200la_vec x, b200la_vec y) {
  B_TRY(check_spmv(m, x, y, "spmv"));
  return spmv_launch(m, x->d, y->d, false, m->ctx->stream);
}

int b200la_spmv_add(b200la_mat m, b200la_vec x, b200la_vec y) {
  B_TRY(check_spmv(m, x, y, "spmv_add"));
  return spmv_launch(m, x->d, y->d, true, m->ctx->stream);
}

int b200la_spmv_nodiag(b200la_mat m, b200la_vec x, b200la_vec y) {
  B_TRY(check_spmv(m, x, y, "spmv_nodiag"));
  return spmv_nodiag_launch(m, x->d, y->d, m->ctx->stream);
}

int b200la_mat_inv_diag(b200la_mat m, b200la_vec out) {
  B_CHECK(m && out, B200LA_ERR_INVALID, "mat_inv_diag: null argument");
  B_CHECK(out->n == m->nrow && m->nrow == m->ncol, B200LA_ERR_INVALID, "mat_inv_diag: size mismatch");
  B_CHECK(out->dtype == m->dtype, B200LA_ERR_DTYPE, "mat_inv_diag: dtype mismatch");
  if (m->nrow == 0) return B200LA_OK;
  b200la_ctx c = m->ctx;
  unsigned *bad = c->scratch.ticket + 8;
  unsigned init = 0xffffffffu;
  B_CUDA(cudaMemcpyAsync(bad, &init, sizeof(unsigned), cudaMemcpyHostToDevice, c->stream));
  int grid = (m->nrow + kBlock - 1) / kBlock;
  if (m->dtype == B200LA_F64)
    inv_diag_kernel<double><<<grid, kBlock, 0, c->stream>>>(m->nrow, m->diag, (const double *)m->val, (double *)out->d, bad);
  else
    inv_diag_kernel<float><<<grid, kBlock, 0, c->stream>>>(m->nrow, m->diag, (const float *)m->val, (float *)out->d, bad);
  B_CUDA(cudaGetLastError());
  unsigned hb = 0;
  B_CUDA(cudaMemcpyAsync(c->host_result, bad, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  B_CUDA(cudaStreamSynchronize(c->stream));
  memcpy(&hb, c->host_result, sizeof(unsigned));
  B_CHECK(hb == 0xffffffffu, B200LA_ERR_MATRIX, "mat_inv_diag: row %u has no nonzero diagonal", hb);
  return B200LA_OK;
}

int b200la_mat_set_format(b200la_mat m, int format, int param) {
  B_CHECK(m, B200LA_ERR_INVALID, "mat_set_format: null matrix");
  if (format == B200LA_FMT_CSR) {
    B_CHECK(param == 1 || param == 2 || param == 4 || param == 8 || param == 16 || param == 32, B200LA_ERR_INVALID,
            "mat_set_format: CSR lanes per row %d (1..32, power of two)", param);
    m->format = format;
    m->param = param;
    m->sched_gen += 1;
    return B200LA_OK;
  }
  if (is_sell(format)) {
    B_CHECK(param == 1 || param == 2 || param == 4, B200LA_ERR_INVALID, "mat_set_format: SELL width %d", param);
    B_TRY(sell_build(m, param, format == B200LA_FMT_SELL16));
    m->format = format;
    m->param = param;
    m->sched_gen += 1;
    return B200LA_OK;
  }
  if (format == B200LA_FMT_STENCIL) {
    B_CHECK(param == 1 || param == 2 || param == 4, B200LA_ERR_INVALID, "mat_set_format: STENCIL width %d", param);
    B_TRY(stencil_build(m, param));
    m->format = format;
    m->param = param;
    m->sched_gen += 1;
    return B200LA_OK;
  }
  return fail(B200LA_ERR_UNSUPPORTED, "mat_set_format: format %d", format);
}

int b200la_mat_to_sell(b200la_mat m, int C, int sigma, int width, int col16) {
  B_CHECK(m, B200LA_ERR_INVALID, "mat_to_sell: null matrix");
  B_CHECK(width == 1 || width == 2 || width == 4, B200LA_ERR_INVALID, "mat_to_sell: width %d (1, 2 or 4)", width);
  B_TRY(sell_build(m, width, col16 != 0, C, sigma));
  m->format = col16 ? B200LA_FMT_SELL16 : B200LA_FMT_SELL;
  m->param = width;
  m->sched_gen += 1;
  return B200LA_OK;
}

int b200la_mat_get_sell(b200la_mat m, int *C, int *sigma, int64_t *padded) {
  B_CHECK(m && C && sigma, B200LA_ERR_INVALID, "mat_get_sell: null argument");
  B_CHECK(is_sliced(m->format), B200LA_ERR_INVALID, "mat_get_sell: the matrix's schedule is not sliced");
  *C = m->sell.c;
  *sigma = m->sell.sigma;
  if (padded) *padded = m->sell.padded;
  return B200LA_OK;
}

int b200la_mat_get_format(b200la_mat m, int *format, int *param) {
  B_CHECK(m && format && param, B200LA_ERR_INVALID, "mat_get_format: null argument");
  *format = m->format;
  *param = m->param;
  return B200LA_OK;
}

}  // extern "C"
