// Dot product that allocates nothing: b200la_dot_noalloc.
//
// Some callers cannot call cudaMalloc: cudaMalloc and cudaFree can stall
// the whole device while pipelined work is in flight (a time-stepping loop or
// a request loop that keeps solves overlapping), and host applications that
// hand all device memory to their own pool allocator, or run this library
// as a plug-in under a fixed memory quota, may not allocate outside it.  This
// entry point takes the caller's device buffers and keeps its reduction
// scratch in a file-scope __device__ array, so it never allocates.
//
// Scratch: kNoAllocBlocks partial sums plus a ticket counter and the total,
// about 32 KB, held by every GPU that loads the library until the process
// exits.  One block covers kNoAllocChunk elements, so n is limited to
// kNoAllocBlocks * kNoAllocChunk = 16,777,216 elements.
//
// All calls share the one array and it keeps the last call's contents; the
// ticket is cleared at the start of every call.  Calls whose kernels overlap
// on the GPU (several streams or host threads at once) race on the array.
#include <mutex>

#include "internal.cuh"

namespace b200la {

constexpr int kNoAllocBlocks = 4096;
constexpr int kNoAllocPerThread = 16;
constexpr int kNoAllocChunk = kBlock * kNoAllocPerThread;  // elements per block
constexpr int64_t kNoAllocMaxN = (int64_t)kNoAllocBlocks * kNoAllocChunk;
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
  double part[kNoAllocBlocks];
  unsigned ticket;
  unsigned pad;
  double total;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Host-side cache of the scratch's device address, one per device.  The
// symbol name itself is a host-side stand-in and must never reach a kernel.
static NoAllocScratch *g_noalloc_addr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mu;

template <typename T>
__global__ void __launch_bounds__(kBlock) dot_noalloc_kernel(int64_t n, const T *__restrict__ a,
                                                             const T *__restrict__ b, NoAllocScratch *scr) {
  Acc<T> acc;
  const int64_t base = (int64_t)blockIdx.x * kNoAllocChunk;
#pragma unroll
  for (int k = 0; k < kNoAllocPerThread; ++k) {
    const int64_t i = base + (int64_t)k * kBlock + threadIdx.x;
    if (i < n) acc.add(__ldg(a + i) * __ldg(b + i));
  }
  double v[1] = {acc.value()};
  if (grid_sum_last<1>(v, scr->part, &scr->ticket) && threadIdx.x == 0) scr->total = v[0];
}

// First call on a device: look up the scratch's device address with that
// device current and cache it.
static int noalloc_scratch(int device, NoAllocScratch **out) {
  B_CHECK(device >= 0 && device < kNoAllocMaxDevices, B200LA_ERR_UNSUPPORTED,
          "dot_noalloc: device %d beyond the %d supported", device, kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[device]) {
    void *p = nullptr;
    B_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    B_CHECK(p != nullptr, B200LA_ERR_CUDA, "dot_noalloc: scratch address lookup returned NULL");
    g_noalloc_addr[device] = static_cast<NoAllocScratch *>(p);
  }
  *out = g_noalloc_addr[device];
  return B200LA_OK;
}

}  // namespace b200la

using namespace b200la;

extern "C" int b200la_dot_noalloc(const void *x, const void *y, int64_t n, int dtype, void *stream,
                                  double *out) {
  B_CHECK(out && (n == 0 || (x && y)), B200LA_ERR_INVALID, "dot_noalloc: null argument");
  B_CHECK(dtype_ok(dtype), B200LA_ERR_DTYPE, "dot_noalloc: dtype %d", dtype);
  B_CHECK(n >= 0, B200LA_ERR_INVALID, "dot_noalloc: negative size %lld", (long long)n);
  B_CHECK(n <= kNoAllocMaxN, B200LA_ERR_UNSUPPORTED,
          "dot_noalloc: n = %lld exceeds the fixed scratch limit of %lld elements", (long long)n,
          (long long)kNoAllocMaxN);
  if (n == 0) {
    *out = 0.0;
    return B200LA_OK;
  }
  int device = 0;
  B_CUDA(cudaGetDevice(&device));
  NoAllocScratch *scr = nullptr;
  B_TRY(noalloc_scratch(device, &scr));
  cudaStream_t s = (cudaStream_t)stream;
  B_CUDA(cudaMemsetAsync(&scr->ticket, 0, sizeof(unsigned), s));
  const int grid = (int)((n + kNoAllocChunk - 1) / kNoAllocChunk);
  if (dtype == B200LA_F64)
    dot_noalloc_kernel<double><<<grid, kBlock, 0, s>>>(n, (const double *)x, (const double *)y, scr);
  else
    dot_noalloc_kernel<float><<<grid, kBlock, 0, s>>>(n, (const float *)x, (const float *)y, scr);
  B_CUDA(cudaGetLastError());
  B_CUDA(cudaMemcpyAsync(out, &scr->total, sizeof(double), cudaMemcpyDeviceToHost, s));
  B_CUDA(cudaStreamSynchronize(s));
  return B200LA_OK;
}
