// pb_noalloc.cu -- a dot product that allocates nothing.
//
// Some callers cannot allocate device memory while they run: a solver embedded in a
// host application that has already carved up the GPU with its own memory pool, code
// running where cudaMalloc is forbidden or would synchronise the device at a bad moment
// (inside a larger asynchronous pipeline), or a caller that must not fail on a full GPU.
// parcel_b_dot_noalloc sums the same FP64 products as parcel_b_dot, in a different fixed
// order (16,384 elements per block instead of parcel_b_dot's grid), so its result is
// deterministic for a given n but may differ from parcel_b_dot's in the last bits.  Its
// scratch (one partial sum per block and the block-completion ticket) lives in a
// file-scope device array that exists for as long as the library is loaded.  It calls
// neither cudaMalloc nor cudaFree nor any allocating library routine, and it does not
// create a stream: it launches on the stream the caller passes.
//
// Limits and caveats (also in include/parcel_b.h):
//   * one partial per 16,384 elements and at most kNaMaxBlocks partials, so n may not
//     exceed kNaMaxN = 67,108,864; larger n is rejected with PARCEL_B_E_ARG;
//   * every call shares the one scratch array: calls that overlap on the GPU (on
//     different streams, or from several threads) race and must be serialised by the
//     caller;
//   * the first call on a device looks up the array's device address for that device
//     (cudaGetSymbolAddress, with that device current), so make the first call outside
//     any stream capture;
//   * the scratch keeps the previous call's contents; the ticket, which must start at
//     zero, is cleared on the stream before every launch.
#include <algorithm>
#include <mutex>

#include "pb_common.cuh"
#include "pb_device.cuh"

namespace pb {

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaPerThread = 64;
constexpr int64_t kNaPerBlock = (int64_t)kNaThreads * kNaPerThread;    // 16,384
constexpr int kNaMaxBlocks = 4096;
constexpr int64_t kNaMaxN = kNaPerBlock * kNaMaxBlocks;                 // 67,108,864
constexpr int kNaTicketSlot = kNaMaxBlocks;                             // one double slot

// Partial sums [0, kNaMaxBlocks) followed by the ticket word; the padding keeps the
// ticket on its own cache lines.  33 KiB per device.
static __device__ __align__(256) double g_noalloc_scratch[kNaMaxBlocks + 32];

constexpr int kMaxDevices = 64;
std::mutex g_na_mu;
double* g_na_ptr[kMaxDevices] = {nullptr};

__global__ void __launch_bounds__(kNaThreads) k_dot_noalloc(int64_t n, const double* __restrict__ x,
                                                            const double* __restrict__ y,
                                                            double* __restrict__ scratch,
                                                            double* __restrict__ out) {
  __shared__ double wsum[kNaThreads / 32];
  __shared__ unsigned am_last;
  unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kNaTicketSlot);
  const int64_t b0 = (int64_t)blockIdx.x * kNaPerBlock;
  double acc = 0.0;
  for (int k = 0; k < kNaPerThread; ++k) {
    const int64_t i = b0 + (int64_t)k * kNaThreads + threadIdx.x;
    if (i < n) acc += x[i] * y[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  if (lane == 0) wsum[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kNaThreads / 32; ++w) s += wsum[w];
    scratch[blockIdx.x] = s;
    __threadfence();
    am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (warp == 0) {
    double s = 0.0;
    for (unsigned b = lane; b < gridDim.x; b += 32) s += __ldcg(scratch + b);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) {
      *out = s;
      *ticket = 0u;
    }
  }
}

}  // namespace

}  // namespace pb

extern "C" int parcel_b_dot_noalloc(int64_t n, const double* x, const double* y, double* result_dev,
                                    void* stream) {
  using namespace pb;
  if (n < 0 || n > kNaMaxN) {
    set_last_error(PARCEL_B_E_ARG,
                   "parcel_b_dot_noalloc: n = %lld is outside [0, %lld], the size its fixed "
                   "scratch array covers", (long long)n, (long long)kNaMaxN);
    return PARCEL_B_E_ARG;
  }
  if (!result_dev || (n > 0 && (!x || !y))) {
    set_last_error(PARCEL_B_E_ARG, "parcel_b_dot_noalloc: NULL pointer");
    return PARCEL_B_E_ARG;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(PARCEL_B_E_CUDA, "parcel_b_dot_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
    return PARCEL_B_E_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error(PARCEL_B_E_UNSUPPORTED,
                   "parcel_b_dot_noalloc: device %d exceeds the %d devices its scratch table covers",
                   dev, kMaxDevices);
    return PARCEL_B_E_UNSUPPORTED;
  }
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
      // One-time set-up on this device (the current one): the array's device address.
      e = cudaGetSymbolAddress(reinterpret_cast<void**>(&g_na_ptr[dev]), g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_na_ptr[dev] = nullptr;
        set_last_error(PARCEL_B_E_CUDA, "parcel_b_dot_noalloc: cudaGetSymbolAddress: %s",
                       cudaGetErrorString(e));
        return PARCEL_B_E_CUDA;
      }
    }
    scratch = g_na_ptr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(scratch + kNaTicketSlot, 0, sizeof(double), st);
  if (e != cudaSuccess) {
    set_last_error(PARCEL_B_E_CUDA, "parcel_b_dot_noalloc: clearing the ticket: %s", cudaGetErrorString(e));
    return PARCEL_B_E_CUDA;
  }
  const int blocks = (int)std::max<int64_t>(1, (n + kNaPerBlock - 1) / kNaPerBlock);
  k_dot_noalloc<<<blocks, kNaThreads, 0, st>>>(n, x, y, scratch, result_dev);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_last_error(PARCEL_B_E_CUDA, "parcel_b_dot_noalloc: launch: %s", cudaGetErrorString(e));
    return PARCEL_B_E_CUDA;
  }
  return PARCEL_B_OK;
}
