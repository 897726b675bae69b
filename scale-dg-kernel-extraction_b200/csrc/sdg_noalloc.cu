// sdg_minmax_dev_noalloc: the min/max reduction of sdg_minmax for callers
// that cannot allocate device memory.
//
// sdg_minmax reduces through scratch that its handle allocated with
// cudaMalloc.  Some callers cannot allocate device memory at the point
// where they need the diagnostic: a host time loop that runs under a fixed
// device-memory budget once set-up is over (its allocator refuses growth),
// or a caller that holds only a raw device array and no library handle.
// This entry point takes that caller's device array and device output and
// allocates nothing: its scratch is the file-scope array below, reserved in
// every GPU that loads the library until the process exits.
//
// Limits and sharing:
//   * at most kNoAllocMaxBlocks blocks of kNoAllocPerBlock values each, so
//     n <= 33,554,432 doubles (268 MB of input); larger n is rejected;
//   * every call, on every stream, uses the same scratch, which keeps the
//     last call's contents; calls that overlap on the GPU race and must be
//     serialised by the caller (one stream, or an event between them);
//   * the first call on a device looks up the scratch's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make
//     that first call before any stream capture.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "sdg_gpu.h"
#include "sdg_internal.h"

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPerThread = 32;
constexpr long long kNoAllocPerBlock = 1LL * kNoAllocThreads * kNoAllocPerThread;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr long long kNoAllocMaxN = kNoAllocPerBlock * kNoAllocMaxBlocks;
constexpr int kMaxDevices = 64;

struct NoAllocScratch {
  double partials[2 * kNoAllocMaxBlocks];  // per-block (min, max)
  unsigned int arrivals;                   // blocks finished in this call
};

// The scratch itself: 64 KB + 4 bytes per device.  Host code must not use
// this name as an address; it asks cudaGetSymbolAddress for the device one.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_noalloc_mutex;
NoAllocScratch* g_noalloc_ptr[kMaxDevices] = {};

__global__ void __launch_bounds__(kNoAllocThreads)
    minmax_noalloc_kernel(const double* __restrict__ q, long long n,
                          NoAllocScratch* scratch, double* __restrict__ out) {
  __shared__ double smin[kNoAllocThreads / 32], smax[kNoAllocThreads / 32];
  __shared__ bool last;
  const long long begin = blockIdx.x * kNoAllocPerBlock;
  const long long end = begin + kNoAllocPerBlock < n ? begin + kNoAllocPerBlock : n;
  double mn = INFINITY, mx = -INFINITY;
  for (long long x = begin + threadIdx.x; x < end; x += kNoAllocThreads) {
    const double y = q[x];
    mn = fmin(mn, y);
    mx = fmax(mx, y);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    smin[wid] = mn;
    smax[wid] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kNoAllocThreads / 32; ++w) {
      mn = fmin(mn, smin[w]);
      mx = fmax(mx, smax[w]);
    }
    scratch->partials[2 * blockIdx.x] = mn;
    scratch->partials[2 * blockIdx.x + 1] = mx;
    __threadfence();
    last = atomicAdd(&scratch->arrivals, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double a = scratch->partials[0], b = scratch->partials[1];
    for (unsigned k = 1; k < gridDim.x; ++k) {
      a = fmin(a, scratch->partials[2 * k]);
      b = fmax(b, scratch->partials[2 * k + 1]);
    }
    out[0] = a;
    out[1] = b;
    scratch->arrivals = 0u;
  }
}

// Device address of the scratch on the current device (looked up once).
int noalloc_scratch(NoAllocScratch** ptr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return sdg::fail(SDG_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return sdg::fail(SDG_ERR_CUDA, "device %d beyond the supported %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return sdg::fail(SDG_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s",
                       cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<NoAllocScratch*>(p);
  }
  *ptr = g_noalloc_ptr[dev];
  return SDG_OK;
}

}  // namespace

extern "C" int sdg_minmax_dev_noalloc(const double* q, long long n, double* out2,
                                      void* stream) {
  if (!q || !out2) return sdg::fail(SDG_ERR_ARG, "sdg_minmax_dev_noalloc: null pointer");
  if (n < 1) return sdg::fail(SDG_ERR_ARG, "sdg_minmax_dev_noalloc: n must be >= 1");
  if (n > kNoAllocMaxN)
    return sdg::fail(SDG_ERR_ARG,
                     "sdg_minmax_dev_noalloc: n = %lld exceeds the fixed scratch capacity "
                     "of %lld values (%d blocks of %lld)", n, kNoAllocMaxN,
                     kNoAllocMaxBlocks, kNoAllocPerBlock);
  NoAllocScratch* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // The arrival counter must start at zero; clear it on this stream.
  cudaError_t e = cudaMemsetAsync(&scratch->arrivals, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess)
    return sdg::fail(SDG_ERR_CUDA, "clearing the no-alloc scratch failed: %s",
                     cudaGetErrorString(e));
  const int blocks = static_cast<int>((n + kNoAllocPerBlock - 1) / kNoAllocPerBlock);
  minmax_noalloc_kernel<<<blocks, kNoAllocThreads, 0, st>>>(q, n, scratch, out2);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return sdg::fail(SDG_ERR_CUDA, "no-alloc min/max launch failed: %s", cudaGetErrorString(e));
  return SDG_OK;
}
