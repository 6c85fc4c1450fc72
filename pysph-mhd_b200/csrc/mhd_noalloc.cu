// mhd_noalloc.cu -- the timestep reduction without any allocation.
//
// Some callers cannot call cudaMalloc: code running while a CUDA graph is
// being captured, embedders whose allocator policy forbids the library from
// taking device memory on its own, and real-time loops that must not hit the
// driver's allocator.  For them mhd_timestep_noalloc computes
// dt = min_i dt_adapt_i clipped so that t + dt <= tf -- the adaptive rule of
// AdaptiveTimestep (src/equations.py:570-585) and the solver's step choice
// with its stop at tf (src/solver.py:40,61) -- with its scratch in a
// file-scope __device__ array instead of a context's workspace.
//
// The array (g_dt_scratch) holds one partial minimum per block for up to
// kNoAllocMaxBlocks blocks of kNoAllocTile elements, plus a completion
// counter: n is limited to MHD_NOALLOC_MAX_N = 67,108,864.  Every GPU that
// loads the library keeps the array (32 KiB + 8 B) until the process exits.
// A __device__ array starts zeroed when the module loads, so the counter
// needs no clearing before the first call; the last block of every call
// returns it to zero.
//
// Host code must not pass the symbol itself to a kernel: on the host it is a
// stand-in, not a device address.  The first call on each device looks up
// the real address with cudaGetSymbolAddress (that device current) and keeps
// it for the life of the process; make that first call before any stream
// capture.  After cudaDeviceReset on a device the kept address is stale and
// the entry point must not be called on that device again.  All calls share
// the one array, which keeps the last call's partials.  Calls that overlap
// on the GPU (concurrent streams on one device) race on the array and must
// be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "mhd_b200.h"
#include "mhd_common.cuh"
#include "mhd_internal.h"

namespace mhd {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocItems = 64;
constexpr int kNoAllocTile = kNoAllocThreads * kNoAllocItems;  // 16384 elements per block
constexpr int kNoAllocMaxBlocks = 4096;
static_assert((long long)kNoAllocTile * kNoAllocMaxBlocks == MHD_NOALLOC_MAX_N, "limit mismatch");

// [0, kNoAllocMaxBlocks): order-mapped block minima; [kNoAllocMaxBlocks]: counter.
static __device__ __align__(256) unsigned long long g_dt_scratch[kNoAllocMaxBlocks + 1];

__global__ void __launch_bounds__(kNoAllocThreads) k_dt_noalloc(const double* __restrict__ dt_adapt, int n, double t,
                                                                double tf, double* __restrict__ dt_out,
                                                                unsigned long long* scratch) {
  const int base = blockIdx.x * kNoAllocTile;
  double m = INFINITY;
  bool bad = false;
#pragma unroll 4
  for (int k = 0; k < kNoAllocItems; k++) {
    const int i = base + k * kNoAllocThreads + threadIdx.x;
    if (i < n) {
      const double v = dt_adapt[i];
      bad |= !(v > 0.0) || !isfinite(v);
      m = fmin(m, v);
    }
  }
  if (bad) m = -INFINITY;  // orders below every positive step: marks the result invalid
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double wmin[kNoAllocThreads / 32];
  __shared__ bool last;
  if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = wmin[0];
    for (int w = 1; w < kNoAllocThreads / 32; w++) b = fmin(b, wmin[w]);
    scratch[blockIdx.x] = dbl_order(b);
    __threadfence();
    last = atomicAdd(&scratch[kNoAllocMaxBlocks], 1ULL) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  unsigned long long lo = ~0ULL;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += kNoAllocThreads) {
    const unsigned long long v = ((volatile unsigned long long*)scratch)[b];
    lo = v < lo ? v : lo;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, lo, o);
    lo = v < lo ? v : lo;
  }
  __shared__ unsigned long long wlo[kNoAllocThreads / 32];
  if ((threadIdx.x & 31) == 0) wlo[threadIdx.x >> 5] = lo;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kNoAllocThreads / 32; w++) lo = wlo[w] < lo ? wlo[w] : lo;
    lo = wlo[0] < lo ? wlo[0] : lo;
    double dt = dbl_unorder(lo);
    if (!(dt > 0.0)) {
      dt = NAN;
    } else if (t + dt > tf) {
      dt = tf - t;
    }
    *dt_out = dt;
    scratch[kNoAllocMaxBlocks] = 0ULL;
  }
}

// Device address of g_dt_scratch for each device, looked up once (the
// array is zero from module load; nothing is cleared here).
static std::mutex g_setup_mutex;
static unsigned long long* g_scratch_addr[256] = {};

static int scratch_for_current_device(unsigned long long** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
    set_library_error("mhd_timestep_noalloc: no current CUDA device");
    return MHD_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_dt_scratch);
    if (e != cudaSuccess) {
      set_library_error(std::string("mhd_timestep_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return MHD_ERR_CUDA;
    }
    g_scratch_addr[dev] = (unsigned long long*)p;
  }
  *out = g_scratch_addr[dev];
  return MHD_OK;
}

}  // namespace mhd

extern "C" int mhd_timestep_noalloc(const double* dt_adapt, int64_t n, double t, double tf, double* dt_out,
                                    void* stream) {
  using namespace mhd;
  if (!dt_adapt || !dt_out) {
    set_library_error("mhd_timestep_noalloc: dt_adapt and dt_out must be device pointers");
    return MHD_ERR_INVALID;
  }
  if (n < 1 || n > MHD_NOALLOC_MAX_N) {
    set_library_error("mhd_timestep_noalloc: n must be in [1, MHD_NOALLOC_MAX_N = 67108864]; got " +
                      std::to_string((long long)n));
    return MHD_ERR_INVALID;
  }
  unsigned long long* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != MHD_OK) return rc;
  const int blocks = (int)((n + kNoAllocTile - 1) / kNoAllocTile);
  k_dt_noalloc<<<blocks, kNoAllocThreads, 0, (cudaStream_t)stream>>>(dt_adapt, (int)n, t, tf, dt_out, scratch);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_library_error(std::string("mhd_timestep_noalloc: launch failed: ") + cudaGetErrorString(e));
    return MHD_ERR_CUDA;
  }
  return MHD_OK;
}
