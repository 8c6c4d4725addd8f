// apirl_likelihood_noalloc: the Poisson log-likelihood reduction without any
// device allocation.
//
// apirl_likelihood allocates its per-block partial sums on every call.  Some
// callers cannot do that: a host application whose device memory is owned by
// another allocator (a framework's caching pool, a preallocated arena) and
// that must not grow it behind that allocator's back; code that runs where a
// cudaMalloc would synchronize the device or fail (inside a latency-critical
// serving loop, or while another library is capturing a stream); and embedded
// callers with a fixed memory plan.  For them this variant keeps its scratch in
// one file-scope device array, set aside when the library is loaded.
//
// Limits and rules:
//  * at most APIRL_LIKELIHOOD_NOALLOC_MAX_BINS bins per call (65,536 chunks of
//    4,096 bins; the scratch array holds one FP64 partial per chunk, 512 KiB);
//    larger calls are rejected with APIRL_ERR_INVALID;
//  * the first call on a device looks up the array's device address on that
//    device (cudaGetSymbolAddress), so make the first call on each device
//    before any stream capture;
//  * all calls share the array and every call overwrites the partials it uses
//    (nothing needs to start at zero), so calls that overlap on the GPU -- on
//    different streams, or from different threads -- race on it; serialize them.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "internal.h"
#include "../../include/apirl_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 16;
constexpr int kChunk = kThreads * kPerThread;  // bins per block
constexpr int kMaxChunks = 65536;

static __device__ __align__(256) double g_likelihood_partials[kMaxChunks];

__device__ __forceinline__ double block_sum_na(double v) {
  __shared__ double red[kThreads / 32];
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (wid == 0) {
    s = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;
}

// One chunk of kChunk bins per block; one partial per block.
__global__ void __launch_bounds__(kThreads) k_likelihood_chunks(int64_t n, const float* __restrict__ est,
                                                                const float* __restrict__ meas, int gt0,
                                                                double* __restrict__ partials) {
  const int64_t base = (int64_t)blockIdx.x * kChunk;
  double v = 0.0;
  #pragma unroll 4
  for (int c = 0; c < kPerThread; c++) {
    const int64_t i = base + (int64_t)c * kThreads + threadIdx.x;
    if (i < n) {
      const float e = est[i];
      if (gt0 ? (e > 0.f) : (e != 0.f)) v += (double)meas[i] * log((double)e) - (double)e;
    }
  }
  const double s = block_sum_na(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kThreads) k_sum_chunks(const double* __restrict__ partials, int n,
                                                         double* __restrict__ out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) v += partials[i];
  const double s = block_sum_na(v);
  if (threadIdx.x == 0) *out = s;
}

// Device address of the scratch array, looked up once per device.
constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

apirl_status scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return apirl_internal_fail(APIRL_ERR_CUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return apirl_internal_fail(APIRL_ERR_INVALID, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_likelihood_partials);
    if (e != cudaSuccess || !p) {
      char buf[160];
      snprintf(buf, sizeof buf, "cudaGetSymbolAddress of the likelihood scratch failed: %s", cudaGetErrorString(e));
      return apirl_internal_fail(APIRL_ERR_CUDA, buf);
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return APIRL_OK;
}

}  // namespace

extern "C" apirl_status apirl_likelihood_noalloc(int64_t n, const float* d_est, const float* d_meas, int gt0,
                                                 double* d_out, void* stream) {
  if (n <= 0 || !d_est || !d_meas || !d_out)
    return apirl_internal_fail(APIRL_ERR_INVALID, "apirl_likelihood_noalloc: bad arguments");
  if (n > APIRL_LIKELIHOOD_NOALLOC_MAX_BINS) {
    char buf[200];
    snprintf(buf, sizeof buf,
             "apirl_likelihood_noalloc: %lld bins exceed the fixed scratch limit of %lld bins "
             "(use apirl_likelihood)", (long long)n, (long long)APIRL_LIKELIHOOD_NOALLOC_MAX_BINS);
    return apirl_internal_fail(APIRL_ERR_INVALID, buf);
  }
  if (apirl_status pend = apirl_internal_pending()) return pend;
  double* scratch = nullptr;
  apirl_status st = scratch_for_current_device(&scratch);
  if (st != APIRL_OK) return st;
  const int chunks = (int)((n + kChunk - 1) / kChunk);
  cudaStream_t s = (cudaStream_t)stream;
  k_likelihood_chunks<<<chunks, kThreads, 0, s>>>(n, d_est, d_meas, gt0, scratch);
  k_sum_chunks<<<1, kThreads, 0, s>>>(scratch, chunks, d_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return apirl_internal_fail(APIRL_ERR_CUDA, cudaGetErrorString(e));
  return APIRL_OK;
}
