// K2 (in-place bit-swap permutation), K3 (FP64 reductions) and small
// elementwise kernels (basis-state set, dtype conversion).
#include <algorithm>
#include <vector>

#include "bounds.cuh"
#include "internal.h"

namespace hisv {
namespace {

int num_sms() { return device_sms(); }

// ---- K2 -------------------------------------------------------------------
// Replaces the MPI redistribution (gather_slots, mpi_redistributer.hpp:265-344)
// on one device.  A set of disjoint slot-bit pairs (a_i, b_i) defines the
// involution P(x) = x with bits a_i and b_i exchanged; amplitude x moves to
// P(x).  Because P is an involution the pass is in place: the thread that owns
// x < P(x) swaps the two amplitudes; fixed points are skipped.
struct SwapPairs {
  int np;
  uint64_t ma, mb;  // masks of the a and b bits
  uint8_t a[32], b[32];
};

template <typename V>
__global__ void __launch_bounds__(256) k2_bitswap(V* __restrict__ sv, uint64_t size,
                                                  const SwapPairs sp) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t x = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < size; x += stride) {
    // pairs whose two bits differ in x flip; others are unchanged
    uint64_t y = x;
#pragma unroll 4
    for (int i = 0; i < sp.np; ++i) {
      const uint64_t ba = (x >> sp.a[i]) & 1ull, bb = (x >> sp.b[i]) & 1ull;
      y ^= (ba ^ bb) * ((1ull << sp.a[i]) | (1ull << sp.b[i]));
    }
    if (x < y) {
      V u = sv[x], w = sv[y];
      sv[x] = w;
      sv[y] = u;
    }
  }
}

// ---- K3 ---------------------------------------------------------------------
// Deterministic two-stage sums in FP64: a fixed grid, a fixed per-thread
// stride, a fixed tree inside each block, then one block adds the per-block
// partials in order.  (The reference's probability() accumulates into one
// variable from all OpenMP threads, state_vector.hpp:908-914, which races.)
constexpr int kRedBlocks = 1184;  // 8 x 148
constexpr int kRedThreads = 256;

template <typename V>
__device__ __forceinline__ double2 ld2(const V* p, uint64_t i) {
  V v = p[i];
  return make_double2(double(v.x), double(v.y));
}

__device__ __forceinline__ double block_sum(double x, double* sh) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = x;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < int(blockDim.x >> 5); ++i) r += sh[i];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double block_max(double x, double* sh) {
  for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = x;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < int(blockDim.x >> 5); ++i) r = fmax(r, sh[i]);
  __syncthreads();
  return r;
}

enum RedKind { RED_NORM = 0, RED_PROB0 = 1, RED_ZZ = 2, RED_INNER = 3, RED_MAXDIFF = 4 };

// partial[k * gridDim.x + blockIdx.x] for k < nout
template <typename V>
__global__ void __launch_bounds__(kRedThreads) k3_reduce(const V* __restrict__ a,
                                                         const V* __restrict__ b, uint64_t size,
                                                         int kind, uint64_t m1, uint64_t m2,
                                                         double* __restrict__ partial) {
  __shared__ double sh[kRedThreads / 32];
  double s0 = 0, s1 = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < size; i += stride) {
    const double2 u = ld2(a, i);
    if (kind == RED_NORM) {
      s0 += u.x * u.x + u.y * u.y;
    } else if (kind == RED_PROB0) {
      if (!(i & m1)) s0 += u.x * u.x + u.y * u.y;
    } else if (kind == RED_ZZ) {
      const double p = u.x * u.x + u.y * u.y;
      const bool odd = (__popcll(i & m1) + __popcll(i & m2)) & 1;
      s0 += odd ? -p : p;
    } else if (kind == RED_INNER) {
      const double2 w = ld2(b, i);  // conj(u) * w
      s0 += u.x * w.x + u.y * w.y;
      s1 += u.x * w.y - u.y * w.x;
    } else {
      const double2 w = ld2(b, i);
      const double dx = u.x - w.x, dy = u.y - w.y;
      s0 = fmax(s0, sqrt(dx * dx + dy * dy));
    }
  }
  if (kind == RED_MAXDIFF) {
    const double r = block_max(s0, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = r;
  } else {
    const double r0 = block_sum(s0, sh);
    const double r1 = block_sum(s1, sh);
    if (threadIdx.x == 0) {
      partial[blockIdx.x] = r0;
      partial[gridDim.x + blockIdx.x] = r1;
    }
  }
}

__global__ void k3_finish(const double* __restrict__ partial, int nblocks, int kind,
                          double* __restrict__ out) {
  __shared__ double sh[kRedThreads / 32];
  for (int k = 0; k < 2; ++k) {
    double s = kind == RED_MAXDIFF ? 0.0 : 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
      const double v = partial[k * nblocks + i];
      s = kind == RED_MAXDIFF ? fmax(s, v) : s + v;
    }
    const double r = kind == RED_MAXDIFF ? block_max(s, sh) : block_sum(s, sh);
    if (threadIdx.x == 0) out[k] = r;
    if (kind == RED_MAXDIFF) break;
  }
}

template <typename V>
int run_reduce(const void* a, const void* b, int n, int kind, uint64_t m1, uint64_t m2,
               double out[2], cudaStream_t s) {
  const uint64_t size = 1ull << n;
  const int blocks = int(std::min<uint64_t>(kRedBlocks, (size + kRedThreads - 1) / kRedThreads));
  double* scratch = nullptr;  // [2*blocks partials | 2 results]
  HS_CUDA(cudaMallocAsync(&scratch, sizeof(double) * (2 * blocks + 2), s));
  k3_reduce<V><<<blocks, kRedThreads, 0, s>>>(static_cast<const V*>(a),
                                               static_cast<const V*>(b), size, kind, m1, m2,
                                               scratch);
  k3_finish<<<1, kRedThreads, 0, s>>>(scratch, blocks, kind, scratch + 2 * blocks);
  cudaError_t e1 = cudaGetLastError();
  double host[2] = {0, 0};
  cudaError_t e2 = cudaMemcpyAsync(host, scratch + 2 * blocks, sizeof(host),
                                   cudaMemcpyDeviceToHost, s);
  cudaError_t e3 = cudaFreeAsync(scratch, s);
  cudaError_t e4 = cudaStreamSynchronize(s);
  for (cudaError_t e : {e1, e2, e3, e4})
    if (e != cudaSuccess)
      return set_error(HS_E_CUDA, "reduction: %s", cudaGetErrorString(e));
  out[0] = host[0];
  out[1] = host[1];
  return HS_OK;
}

int reduce_any(const void* a, const void* b, int dtype, int n, int kind, uint64_t m1,
               uint64_t m2, double out[2], cudaStream_t s) {
  if (dtype == HS_DTYPE_C128) return run_reduce<double2>(a, b, n, kind, m1, m2, out, s);
  return run_reduce<float2>(a, b, n, kind, m1, m2, out, s);
}

// per-chunk probability mass: block b sums |a_i|^2 over chunk b (fixed order)
template <typename V>
__global__ void __launch_bounds__(kRedThreads) k3_chunks(const V* __restrict__ a, int chunk_bits,
                                                         double* __restrict__ out) {
  __shared__ double sh[kRedThreads / 32];
  const uint64_t base = uint64_t(blockIdx.x) << chunk_bits;
  const uint64_t len = 1ull << chunk_bits;
  double s = 0;
  for (uint64_t i = threadIdx.x; i < len; i += blockDim.x) {
    const double2 u = ld2(a, base + i);
    s += u.x * u.x + u.y * u.y;
  }
  const double r = block_sum(s, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = r;
}

template <typename V>
__global__ void k_set_basis(V* __restrict__ sv, uint64_t size, uint64_t index) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < size; i += stride) {
    V v;
    v.x = i == index ? 1 : 0;
    v.y = 0;
    sv[i] = v;
  }
}

template <typename A, typename B>
__global__ void k_convert(const A* __restrict__ src, B* __restrict__ dst, uint64_t count) {
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    A a = src[i];
    B b;
    b.x = decltype(b.x)(a.x);
    b.y = decltype(b.y)(a.y);
    dst[i] = b;
  }
}

int grid_for(uint64_t size, int threads) {
  const uint64_t want = uint64_t(num_sms()) * 8;
  const uint64_t need = (size + threads - 1) / threads;
  return int(std::max<uint64_t>(1, std::min(want, need)));
}

// <a|b>, max|a-b| and <b|b> over two states of possibly different precision
template <typename VA, typename VB>
__global__ void __launch_bounds__(kRedThreads) k3_compare(const VA* __restrict__ a,
                                                          const VB* __restrict__ b, uint64_t size,
                                                          double* __restrict__ partial) {
  __shared__ double sh[kRedThreads / 32];
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < size; i += stride) {
    const double2 u = ld2(a, i), w = ld2(b, i);
    s0 += u.x * w.x + u.y * w.y;
    s1 += u.x * w.y - u.y * w.x;
    const double dx = u.x - w.x, dy = u.y - w.y;
    s2 = fmax(s2, sqrt(dx * dx + dy * dy));
    s3 += w.x * w.x + w.y * w.y;
  }
  const double r0 = block_sum(s0, sh), r1 = block_sum(s1, sh), r3 = block_sum(s3, sh);
  const double r2 = block_max(s2, sh);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = r0;
    partial[gridDim.x + blockIdx.x] = r1;
    partial[2 * gridDim.x + blockIdx.x] = r2;
    partial[3 * gridDim.x + blockIdx.x] = r3;
  }
}

__global__ void k3_compare_finish(const double* __restrict__ partial, int nblocks,
                                  double* __restrict__ out) {
  __shared__ double sh[kRedThreads / 32];
  for (int k = 0; k < 4; ++k) {
    double s = 0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
      const double v = partial[k * nblocks + i];
      s = k == 2 ? fmax(s, v) : s + v;
    }
    const double r = k == 2 ? block_max(s, sh) : block_sum(s, sh);
    if (threadIdx.x == 0) out[k] = r;
  }
}

template <typename VA, typename VB>
int run_compare(const void* a, const void* b, uint64_t size, double out[4], cudaStream_t s) {
  const int blocks = int(std::min<uint64_t>(kRedBlocks, (size + kRedThreads - 1) / kRedThreads));
  double* scratch = nullptr;
  HS_CUDA(cudaMallocAsync(&scratch, sizeof(double) * (4 * blocks + 4), s));
  k3_compare<VA, VB><<<blocks, kRedThreads, 0, s>>>(static_cast<const VA*>(a),
                                                    static_cast<const VB*>(b), size, scratch);
  k3_compare_finish<<<1, kRedThreads, 0, s>>>(scratch, blocks, scratch + 4 * blocks);
  cudaError_t e1 = cudaGetLastError();
  cudaError_t e2 = cudaMemcpyAsync(out, scratch + 4 * blocks, 4 * sizeof(double),
                                   cudaMemcpyDeviceToHost, s);
  cudaError_t e3 = cudaFreeAsync(scratch, s);
  cudaError_t e4 = cudaStreamSynchronize(s);
  for (cudaError_t e : {e1, e2, e3, e4})
    if (e != cudaSuccess) return set_error(HS_E_CUDA, "compare: %s", cudaGetErrorString(e));
  return HS_OK;
}

}  // namespace

int reduce_compare(const void* a, int adtype, const void* b, int bdtype, int n, double out[4],
                   cudaStream_t s) {
  return reduce_compare_count(a, adtype, b, bdtype, 1ull << n, out, s);
}

int reduce_compare_count(const void* a, int adtype, const void* b, int bdtype, uint64_t count,
                         double out[4], cudaStream_t s) {
  if (adtype == HS_DTYPE_C128 && bdtype == HS_DTYPE_C128)
    return run_compare<double2, double2>(a, b, count, out, s);
  if (adtype == HS_DTYPE_C128 && bdtype == HS_DTYPE_C64)
    return run_compare<double2, float2>(a, b, count, out, s);
  if (adtype == HS_DTYPE_C64 && bdtype == HS_DTYPE_C128)
    return run_compare<float2, double2>(a, b, count, out, s);
  return run_compare<float2, float2>(a, b, count, out, s);
}

int reduce_chunks(const void* amp, int dtype, int n, int chunk_bits, double* host_out,
                  cudaStream_t s) {
  const uint64_t nchunks = 1ull << (n - chunk_bits);
  double* scratch = nullptr;
  HS_CUDA(cudaMallocAsync(&scratch, sizeof(double) * nchunks, s));
  if (dtype == HS_DTYPE_C128)
    k3_chunks<double2><<<unsigned(nchunks), kRedThreads, 0, s>>>(
        static_cast<const double2*>(amp), chunk_bits, scratch);
  else
    k3_chunks<float2><<<unsigned(nchunks), kRedThreads, 0, s>>>(
        static_cast<const float2*>(amp), chunk_bits, scratch);
  cudaError_t e1 = cudaGetLastError();
  cudaError_t e2 = cudaMemcpyAsync(host_out, scratch, sizeof(double) * nchunks,
                                   cudaMemcpyDeviceToHost, s);
  cudaError_t e3 = cudaFreeAsync(scratch, s);
  cudaError_t e4 = cudaStreamSynchronize(s);
  for (cudaError_t e : {e1, e2, e3, e4})
    if (e != cudaSuccess) return set_error(HS_E_CUDA, "chunk sums: %s", cudaGetErrorString(e));
  return HS_OK;
}

namespace {
// Tiled form of K2: the tile holds every bit of the pass's pairs plus the
// lowest other slots, so the permutation maps each tile onto itself.  A CTA
// loads a tile (cp.async, double-buffered), then writes every element of it
// back in global order, reading shared memory at the permuted position: one
// coalesced read and one coalesced write of every amplitude.
constexpr int kK2Threads = 256;
constexpr int kK2MaxTileBits = 12;

struct TilePerm {
  Runs tile, outer;
  int32_t m, np;
  uint64_t ntiles;
  uint8_t pa[8], pb[8];  // tile-bit positions of each pair
};

__device__ __forceinline__ uint64_t dep_runs(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i) out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}

template <int BYTES>
__device__ __forceinline__ void cp_async_el(uint32_t saddr, const void* g) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr), "l"(g) : "memory");
}

template <typename V>
__global__ void __launch_bounds__(kK2Threads) k2_tile(V* __restrict__ sv, const __grid_constant__ TilePerm P) {
  extern __shared__ __align__(16) unsigned char smem_k2[];
  const int t = threadIdx.x;
  const int T = 1 << P.m;
  const int per = T > kK2Threads ? T / kK2Threads : 1;
  V* bufs = reinterpret_cast<V*>(smem_k2);
  uint64_t* gk = reinterpret_cast<uint64_t*>(smem_k2 + 2 * size_t(T) * sizeof(V));
  for (int k = t; k < per; k += kK2Threads) gk[k] = dep_runs(uint64_t(k) * kK2Threads, P.tile);
  __syncthreads();
  const bool active = t < T;
  const uint64_t gt = dep_runs(uint64_t(t), P.tile);
  const uint32_t sb = uint32_t(__cvta_generic_to_shared(bufs));
  const uint64_t size = P.ntiles << P.m;  // amplitudes of the state (bounds checks)
  auto issue = [&](uint64_t tile, int b) {
    if (!active) return;
    const uint64_t gb = dep_runs(tile, P.outer) + gt;
    for (int k = 0; k < per; ++k) {
      const uint32_t j = uint32_t(t + k * kK2Threads);
      if (HS_IN_BOUNDS(gb + gk[k] < size && j < uint32_t(T), kBoundsK2))
        cp_async_el<sizeof(V)>(sb + uint32_t((b * T + j) * sizeof(V)), sv + gb + gk[k]);
    }
  };
  uint64_t tile = blockIdx.x;
  if (tile < P.ntiles) issue(tile, 0);
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int it = 0; tile < P.ntiles; ++it, tile += gridDim.x) {
    const uint64_t next = tile + gridDim.x;
    if (next < P.ntiles) issue(next, (it + 1) & 1);
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 1;" ::: "memory");
    __syncthreads();
    const V* cur = bufs + (it & 1) * T;
    if (active) {
      const uint64_t gb = dep_runs(tile, P.outer) + gt;
      for (int k = 0; k < per; ++k) {
        uint32_t j = uint32_t(t + k * kK2Threads);
        // element j receives the amplitude from the exchanged position
        for (int i = 0; i < P.np; ++i) {
          const uint32_t d = ((j >> P.pa[i]) ^ (j >> P.pb[i])) & 1u;
          j ^= d * ((1u << P.pa[i]) | (1u << P.pb[i]));
        }
        if (HS_IN_BOUNDS(gb + gk[k] < size && j < uint32_t(T), kBoundsK2))
          __stcs(sv + gb + gk[k], cur[j]);
      }
    }
    __syncthreads();  // this buffer is refilled by the prefetch issued next iteration
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

void runs_from(const std::vector<int>& dst, Runs* r) {
  r->n = 0;
  size_t i = 0;
  while (i < dst.size()) {
    size_t j = i + 1;
    while (j < dst.size() && dst[j] == dst[j - 1] + 1) ++j;
    r->src[r->n] = uint8_t(i);
    r->len[r->n] = uint8_t(j - i);
    r->dst[r->n] = uint8_t(dst[i]);
    ++r->n;
    i = j;
  }
}

template <typename V>
int launch_tile_perm(V* amp, int n, const int32_t* pairs, int np, int max_bits, cudaStream_t s) {
  std::vector<int> tile;
  for (int i = 0; i < np; ++i) {
    tile.push_back(pairs[2 * i]);
    tile.push_back(pairs[2 * i + 1]);
  }
  const int m = std::min(n, max_bits);
  for (int sl = 0; sl < n && int(tile.size()) < m; ++sl)
    if (std::find(tile.begin(), tile.end(), sl) == tile.end()) tile.push_back(sl);
  std::sort(tile.begin(), tile.end());
  TilePerm P{};
  P.m = int(tile.size());
  P.np = np;
  P.ntiles = 1ull << (n - P.m);
  runs_from(tile, &P.tile);
  std::vector<int> outer;
  for (int sl = 0; sl < n; ++sl)
    if (std::find(tile.begin(), tile.end(), sl) == tile.end()) outer.push_back(sl);
  runs_from(outer, &P.outer);
  if (P.tile.n > kMaxRuns || P.outer.n > kMaxRuns)
    return set_error(HS_E_UNSUPPORTED, "bit-swap tile has too many runs");
  for (int i = 0; i < np; ++i) {
    P.pa[i] = uint8_t(std::find(tile.begin(), tile.end(), pairs[2 * i]) - tile.begin());
    P.pb[i] = uint8_t(std::find(tile.begin(), tile.end(), pairs[2 * i + 1]) - tile.begin());
  }
  const int T = 1 << P.m;
  const int per = T > kK2Threads ? T / kK2Threads : 1;
  const size_t smem = 2 * size_t(T) * sizeof(V) + size_t(per) * 8;
  HS_TRY(smem_optin(reinterpret_cast<const void*>(k2_tile<V>)));
  int per_sm = 1;
  HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2_tile<V>, kK2Threads, smem));
  const uint64_t want = uint64_t(num_sms()) * uint64_t(std::max(per_sm, 1));
  const int grid = int(P.ntiles < want ? P.ntiles : want);
  k2_tile<V><<<grid, kK2Threads, smem, s>>>(amp, P);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}
}  // namespace

#ifdef HS_BOUNDS
HS_BOUNDS_TAKE(bounds_take_misc)
#endif

int launch_permute(void* amp, int dtype, int n, const int32_t* pairs, int npairs,
                   cudaStream_t s) {
  if (npairs <= 0) return HS_OK;
  if (npairs > 32) return set_error(HS_E_INVALID, "at most 32 bit pairs per pass");
  // pairs commute (they are disjoint): apply them in tiled passes of at most
  // five pairs, each tile keeping at least one more low slot for contiguity
  const int max_bits = dtype == HS_DTYPE_C128 ? 11 : kK2MaxTileBits;
  const int chunk = std::min(5, std::max(1, (std::min(n, max_bits) - 1) / 2));
  for (int first = 0; first < npairs; first += chunk) {
    const int np = std::min(chunk, npairs - first);
    if (dtype == HS_DTYPE_C128)
      HS_TRY(launch_tile_perm(static_cast<double2*>(amp), n, pairs + 2 * first, np, max_bits, s));
    else
      HS_TRY(launch_tile_perm(static_cast<float2*>(amp), n, pairs + 2 * first, np, max_bits, s));
  }
  return HS_OK;
}

int reduce_norm2(const void* amp, int dtype, int n, double* out, cudaStream_t s) {
  double r[2];
  HS_TRY(reduce_any(amp, amp, dtype, n, RED_NORM, 0, 0, r, s));
  *out = r[0];
  return HS_OK;
}

int reduce_inner(const void* a, const void* b, int dtype, int n, double out[2],
                 cudaStream_t s) {
  return reduce_any(a, b, dtype, n, RED_INNER, 0, 0, out, s);
}

int reduce_maxdiff(const void* a, const void* b, int dtype, int n, double* out,
                   cudaStream_t s) {
  double r[2];
  HS_TRY(reduce_any(a, b, dtype, n, RED_MAXDIFF, 0, 0, r, s));
  *out = r[0];
  return HS_OK;
}

int reduce_prob0(const void* amp, int dtype, int n, int slot, double* out, cudaStream_t s) {
  double r[2];
  HS_TRY(reduce_any(amp, amp, dtype, n, RED_PROB0, 1ull << slot, 0, r, s));
  *out = r[0];
  return HS_OK;
}

int reduce_zz(const void* amp, int dtype, int n, const int32_t* slot_pairs, int npairs,
              double* out, cudaStream_t s) {
  for (int i = 0; i < npairs; ++i) {
    double r[2];
    HS_TRY(reduce_any(amp, amp, dtype, n, RED_ZZ, 1ull << slot_pairs[2 * i],
                      1ull << slot_pairs[2 * i + 1], r, s));
    out[i] = r[0];
  }
  return HS_OK;
}

namespace {
struct ProjectMap {
  int32_t nbits;
  uint8_t slot[40];  // old slot of each bit of the projected index
};

template <typename T>
__global__ void k_project(const T* __restrict__ in, T* __restrict__ out, uint64_t count,
                          ProjectMap map, uint64_t offset) {
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count;
       j += uint64_t(gridDim.x) * blockDim.x) {
    uint64_t src = offset;
    for (int b = 0; b < map.nbits; ++b) src |= ((j >> b) & 1ull) << map.slot[b];
    out[j] = in[src];
  }
}

template <typename T>
__global__ void k_scale(T* __restrict__ a, uint64_t count, double f) {
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < count;
       j += uint64_t(gridDim.x) * blockDim.x) {
    T v = a[j];
    v.x = decltype(v.x)(v.x * f);
    v.y = decltype(v.y)(v.y * f);
    a[j] = v;
  }
}
}  // namespace

int project_kernel(const void* in, void* out, int dtype, int out_bits, const int* old_slots,
                   uint64_t offset, cudaStream_t s) {
  ProjectMap map{};
  map.nbits = out_bits;
  for (int b = 0; b < out_bits; ++b) map.slot[b] = uint8_t(old_slots[b]);
  const uint64_t count = 1ull << out_bits;
  const int g = grid_for(count, 256);
  if (dtype == HS_DTYPE_C128)
    k_project<double2><<<g, 256, 0, s>>>(static_cast<const double2*>(in),
                                         static_cast<double2*>(out), count, map, offset);
  else
    k_project<float2><<<g, 256, 0, s>>>(static_cast<const float2*>(in),
                                        static_cast<float2*>(out), count, map, offset);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int scale_kernel(void* amp, int dtype, int n, double f, cudaStream_t s) {
  const uint64_t count = 1ull << n;
  const int g = grid_for(count, 256);
  if (dtype == HS_DTYPE_C128)
    k_scale<double2><<<g, 256, 0, s>>>(static_cast<double2*>(amp), count, f);
  else
    k_scale<float2><<<g, 256, 0, s>>>(static_cast<float2*>(amp), count, f);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

namespace {
// FP64 FMA throughput probe: 8 independent chains per thread
__global__ void k_fma_probe(double* out, double a, double b, int iters) {
  double r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = double(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fma(r[k], a, b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 12345.678) out[0] = s;  // keeps the chains live; never true in practice
}
}  // namespace

int fp64_probe(double* tflops) {
  int dev = 0, sms = 148;
  HS_CUDA(cudaGetDevice(&dev));
  HS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* d = nullptr;
  HS_CUDA(cudaMalloc(&d, sizeof(double)));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0);
    k_fma_probe<<<blocks, threads>>>(d, 0.999999, 1e-7, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  const cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return set_error(HS_E_CUDA, "fp64 probe: %s", cudaGetErrorString(e));
  *tflops = 2.0 * 8.0 * double(iters) * blocks * threads / (double(best) * 1e-3) / 1e12;
  return HS_OK;
}

int set_basis_kernel(void* amp, int dtype, int n, uint64_t index, cudaStream_t s) {
  const uint64_t size = 1ull << n;
  if (dtype == HS_DTYPE_C128)
    k_set_basis<double2><<<grid_for(size, 256), 256, 0, s>>>(static_cast<double2*>(amp), size,
                                                             index);
  else
    k_set_basis<float2><<<grid_for(size, 256), 256, 0, s>>>(static_cast<float2*>(amp), size,
                                                            index);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int convert_kernel(const void* src, int sdtype, void* dst, int ddtype, uint64_t count,
                   cudaStream_t s) {
  const int g = grid_for(count, 256);
  if (sdtype == HS_DTYPE_C128 && ddtype == HS_DTYPE_C64)
    k_convert<double2, float2><<<g, 256, 0, s>>>(static_cast<const double2*>(src),
                                                 static_cast<float2*>(dst), count);
  else if (sdtype == HS_DTYPE_C64 && ddtype == HS_DTYPE_C128)
    k_convert<float2, double2><<<g, 256, 0, s>>>(static_cast<const float2*>(src),
                                                 static_cast<double2*>(dst), count);
  else if (sdtype == HS_DTYPE_C128)
    k_convert<double2, double2><<<g, 256, 0, s>>>(static_cast<const double2*>(src),
                                                  static_cast<double2*>(dst), count);
  else
    k_convert<float2, float2><<<g, 256, 0, s>>>(static_cast<const float2*>(src),
                                                static_cast<float2*>(dst), count);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace hisv
