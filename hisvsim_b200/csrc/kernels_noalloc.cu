// hs_norm2_noalloc: the squared norm of a state, computed without allocating
// any device memory.
//
// Who needs it: callers that cannot let the library call cudaMalloc or
// cudaFree -- a host application that hands every byte of device memory to its
// own pool and forbids other allocations, or a latency-critical loop that must
// not hit the implicit device-wide synchronisation cudaMalloc / cudaFree can
// cause.  hs_norm2 allocates a small partial-sum buffer per call; this variant
// keeps its partial sums in a fixed array that lives in the library's device
// image instead.
//
// The array: kNoAllocPartials doubles (1 MiB) plus one result slot, declared
// at file scope as a __device__ variable.  Every GPU that loads the library
// holds it until the process exits.  One partial is kept per 2^16 amplitudes,
// so states of at most kNoAllocPartials * 2^16 = 2^33 amplitudes are accepted;
// larger states are rejected with HS_E_UNSUPPORTED before anything is launched.
//
// Host code cannot use the array's name as a device address (on the host it is
// only a stand-in symbol), so the first call on each device, with that device
// current, looks the address up with cudaGetSymbolAddress and caches it; make
// that first call before any stream capture.  All calls share the array and it
// keeps the last call's contents; each call writes every partial it reads and
// the result slot before reading them, so nothing needs clearing between
// calls.  Calls that overlap on the GPU (concurrent streams or threads) race
// on the array and must be serialised by the caller.  Every call copies the
// result to the host and synchronises the given stream before it returns.
#include <mutex>

#include "internal.h"

namespace hisv {
namespace {

constexpr int kNoAllocChunkBits = 16;
constexpr int kNoAllocPartials = 1 << 17;
constexpr int kNoAllocThreads = 256;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocPartials + 1];

template <typename V>
__global__ void __launch_bounds__(kNoAllocThreads)
    k_norm_partials(const V* __restrict__ a, int chunk_bits, double* __restrict__ partial) {
  __shared__ double sh[kNoAllocThreads / 32];
  const uint64_t base = uint64_t(blockIdx.x) << chunk_bits;
  const uint64_t len = 1ull << chunk_bits;
  double s = 0;
  for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) {
    const V u = a[base + i];
    s += double(u.x) * double(u.x) + double(u.y) * double(u.y);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int w = 0; w < kNoAllocThreads / 32; ++w) r += sh[w];
    partial[blockIdx.x] = r;
  }
}

// one block adds the partials in a fixed order and writes the result slot
__global__ void __launch_bounds__(kNoAllocThreads)
    k_norm_finish(const double* __restrict__ partial, int n, double* __restrict__ result) {
  __shared__ double sh[kNoAllocThreads / 32];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int w = 0; w < kNoAllocThreads / 32; ++w) r += sh[w];
    *result = r;
  }
}

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {nullptr};

// device address of the scratch array on the current device (looked up once)
int noalloc_scratch(double** out) {
  int dev = 0;
  HS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_error(HS_E_UNSUPPORTED, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return set_error(HS_E_CUDA, "cudaGetSymbolAddress(no-alloc scratch): %s",
                       cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return HS_OK;
}

}  // namespace
}  // namespace hisv

using namespace hisv;

extern "C" int hs_norm2_noalloc(hs_state* st, double* out, void* stream) {
  if (!st || !st->amp) return set_error(HS_E_INVALID, "null or destroyed state");
  if (!out) return set_error(HS_E_INVALID, "null output pointer");
  const int chunk_bits = st->n < kNoAllocChunkBits ? st->n : kNoAllocChunkBits;
  const uint64_t nparts = 1ull << (st->n - chunk_bits);
  if (nparts > uint64_t(kNoAllocPartials))
    return set_error(HS_E_UNSUPPORTED,
                     "hs_norm2_noalloc: a state of 2^%d amplitudes needs %llu partial sums; "
                     "the fixed scratch holds %d (states of at most 2^%d amplitudes)",
                     st->n, (unsigned long long)nparts, kNoAllocPartials,
                     kNoAllocChunkBits + 17);
  double* scratch = nullptr;
  HS_TRY(noalloc_scratch(&scratch));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (st->dtype == HS_DTYPE_C128)
    k_norm_partials<double2><<<unsigned(nparts), kNoAllocThreads, 0, s>>>(
        static_cast<const double2*>(st->amp), chunk_bits, scratch);
  else
    k_norm_partials<float2><<<unsigned(nparts), kNoAllocThreads, 0, s>>>(
        static_cast<const float2*>(st->amp), chunk_bits, scratch);
  k_norm_finish<<<1, kNoAllocThreads, 0, s>>>(scratch, int(nparts), scratch + kNoAllocPartials);
  HS_CUDA(cudaGetLastError());
  HS_CUDA(cudaMemcpyAsync(out, scratch + kNoAllocPartials, sizeof(double),
                          cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaStreamSynchronize(s));
  return HS_OK;
}
