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
#include <cuda.h>

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

// Host-side cache of the scratch's device address, one entry per device,
// tagged with the id of the CUDA context it was looked up in.  The symbol
// name itself is a host-side stand-in and must never reach a kernel.  After
// cudaDeviceReset the device gets a new primary context (a new id) in which
// the array has a new address, so a changed id triggers a new lookup.
struct NoAllocEntry {
  unsigned long long ctx_id;
  NoAllocScratch *addr;
};
static NoAllocEntry g_noalloc_addr[kNoAllocMaxDevices];
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

// Id of the context current on this thread (0 if none is current yet, or if
// the driver entry points cannot be had, in which case every call looks the
// address up again -- the lookup allocates nothing).  The driver functions
// come through the runtime's entry-point query, so the library does not link
// libcuda itself.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

static unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool tried = false;
  if (!tried) {  // called under g_noalloc_mu
    tried = true;
    void *f1 = nullptr, *f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
        cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
      get_current = (CtxGetCurrentFn)f1;
      get_id = (CtxGetIdFn)f2;
    }
  }
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Set-up on a device (its first call there, or the first after the device's
// context was replaced): look up the scratch's device address with that
// device current and cache it with the context's id.
static int noalloc_scratch(int device, NoAllocScratch **out) {
  B_CHECK(device >= 0 && device < kNoAllocMaxDevices, B200LA_ERR_UNSUPPORTED,
          "dot_noalloc: device %d beyond the %d supported", device, kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocEntry &e = g_noalloc_addr[device];
  unsigned long long id = current_ctx_id();
  if (!e.addr || id == 0 || e.ctx_id != id) {
    void *p = nullptr;
    B_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    B_CHECK(p != nullptr, B200LA_ERR_CUDA, "dot_noalloc: scratch address lookup returned NULL");
    id = current_ctx_id();  // the lookup makes the device's primary context current
    e.ctx_id = id;
    e.addr = static_cast<NoAllocScratch *>(p);
  }
  *out = e.addr;
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
