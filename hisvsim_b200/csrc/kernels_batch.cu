// K6: the batching form.  Many QAOA MaxCut instances of different qubit counts
// are advanced by ONE persistent launch: CTAs take work items (instance, step,
// tile) from a global queue in step order; a step of an instance is one pass
// over its complex64 state (the first pass of a round applies the cost phase
// e^{i gamma/2 (2 cut(x) - |E|)} = prod_E RZZ(gamma), every pass applies the
// mixer RX(2 beta) to its share of the qubits).  A tile of step k waits for all
// tiles of step k-1 of the same instance through a completion counter; items
// are dequeued in step order, so the earliest unfinished item never waits and
// the queue always drains.  Waits are bounded: a timeout sets an error flag.
#include "internal.h"

namespace hisv {
namespace {

__device__ __forceinline__ uint64_t bdep(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i) out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}

// tile position of tile index i (pairs of amplitudes stay adjacent)
__device__ __forceinline__ uint32_t bswz(uint32_t i) {
  return i ^ ((((i >> 4) ^ (i >> 7) ^ (i >> 10)) & 7u) << 1);
}

__device__ __forceinline__ void cp16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}

// cut(x) = number of edges whose endpoints differ in x
__device__ __forceinline__ int cut_full(uint64_t x, const BatchInstance& I) {
  int c = 0;
  for (int e = 0; e < I.nedges; ++e) c += int(((x >> I.edge_a[e]) ^ (x >> I.edge_b[e])) & 1ull);
  return c;
}

// cut(xb | S) for the 16 subsets S of four qubits q[0..3] (all 0 in xb):
// edges with exactly one endpoint among q flip when that endpoint is set,
// edges between two of them flip when exactly one of the two is set
__device__ __forceinline__ void cut_table(uint64_t xb, const uint8_t (&q)[4], const BatchInstance& I,
                                          int (&out)[16]) {
  int d[4] = {0, 0, 0, 0};
  int rr[6];
  int nrr = 0;
  int c0 = 0;
  for (int e = 0; e < I.nedges; ++e) {
    const int a = I.edge_a[e], b = I.edge_b[e];
    const int ba = int((xb >> a) & 1ull), bb = int((xb >> b) & 1ull);
    c0 += ba ^ bb;
    int ja = -1, jb = -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (q[j] == a) ja = j;
      if (q[j] == b) jb = j;
    }
    if (ja >= 0 && jb >= 0) {
      if (nrr < 6) rr[nrr++] = (1 << ja) | (1 << jb);
    } else if (ja >= 0) {
      d[ja] += 1 - 2 * (ba ^ bb);
    } else if (jb >= 0) {
      d[jb] += 1 - 2 * (ba ^ bb);
    }
  }
#pragma unroll
  for (int S = 0; S < 16; ++S) {
    int c = c0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if ((S >> j) & 1) c += d[j];
    for (int k = 0; k < nrr; ++k) {
      const int w = S & rr[k];
      c += (w != 0 && w != rr[k]) ? 1 : 0;
    }
    out[S] = c;
  }
}

constexpr uint32_t kDepLimit = 1u << 24;  // polls (with ~0.1 us sleeps) before giving up

__global__ void __launch_bounds__(kBatchThreads, 3)
    k6_batch(const BatchInstance* __restrict__ insts, const BatchParams* __restrict__ pars,
             const BatchItem* __restrict__ groups, int ngroups, uint64_t total,
             uint32_t* __restrict__ counters, unsigned long long* __restrict__ head,
             int* __restrict__ err) {
  __shared__ __align__(16) float2 tile[4096];
  __shared__ float2 s_phase[kBatchMaxEdges + 1];
  __shared__ unsigned long long s_item;
  __shared__ int s_abort;
  const int t = threadIdx.x;
  const uint32_t tile_s = uint32_t(__cvta_generic_to_shared(tile));
  for (;;) {
    if (t == 0) s_item = atomicAdd(head, 1ull);
    __syncthreads();
    const uint64_t item = s_item;
    if (item >= total) break;
    // the item's (instance, step) group: last group with first <= item
    int lo = 0, hi = ngroups - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (groups[mid].first <= item) lo = mid; else hi = mid - 1;
    }
    const BatchItem G = groups[lo];
    const BatchInstance& I = insts[G.inst];
    const int k = G.step;
    const int round = k / I.npasses, pj = k - round * I.npasses;
    const BatchPass& P = I.pass[pj];
    const uint64_t tix = item - G.first;
    // dependency on the previous step of this instance
    if (t == 0) {
      s_abort = 0;
      if (k > 0) {
        const BatchPass& Pp = I.pass[(k - 1) % I.npasses];
        const uint32_t need = uint32_t(1ull << (I.n - Pp.m));
        const uint32_t* cnt = counters + I.step_base + (k - 1);
        uint32_t polls = 0;
        uint32_t seen;
        do {
          asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(cnt) : "memory");
          if (seen >= need) break;
          __nanosleep(100);
        } while (++polls < kDepLimit);
        if (seen < need) {
          s_abort = 1;
          atomicExch(err, 1);
        }
      }
    }
    if (t < kBatchMaxEdges + 1) s_phase[t] = pars[G.inst].phase[round][t];
    __syncthreads();
    if (s_abort) break;
    const int m = P.m, T = 1 << m;
    const uint64_t gbase = bdep(tix, P.outer);
    float2* amp = I.amp;
    // load: 16-byte chunks of two amplitudes (tile bit 0 is slot 0)
    for (int c = t; c < T / 2; c += kBatchThreads)
      cp16(tile_s + bswz(2u * uint32_t(c)) * 8u, amp + gbase + bdep(2ull * c, P.tile));
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const float2 rx = pars[G.inst].rx[round][0];  // (cos beta, sin beta)
    const bool active = t < (T >> 4);
    for (int g = 0; g < P.ngroups; ++g) {
      if (active) {
        // thread bits: the tile bits not held in registers, ascending
        uint32_t thr = 0;
        {
          uint32_t rmask = 0;
          for (int j = 0; j < 4; ++j) rmask |= 1u << P.group_bits[g][j];
          int src = 0;
          for (int b = 0; b < m; ++b)
            if (!((rmask >> b) & 1u)) thr |= uint32_t((t >> src++) & 1) << b;
        }
        uint32_t rb[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) rb[j] = 1u << P.group_bits[g][j];
        float2 v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          uint32_t idx = thr;
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if ((e >> j) & 1) idx |= rb[j];
          v[e] = tile[bswz(idx)];
        }
        if (g == 0 && P.phase) {
          uint8_t q[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) q[j] = P.tile_slot[P.group_bits[0][j]];
          int cut[16];
          cut_table(gbase | bdep(thr, P.tile), q, I, cut);
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const float2 ph = s_phase[cut[e]];
            const float2 a = v[e];
            v[e] = make_float2(ph.x * a.x - ph.y * a.y, ph.x * a.y + ph.y * a.x);
          }
        }
        // mixer RX(2 beta) = [[c, -i s], [-i s, c]] on the group's target bits
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (!((P.group_rx[g] >> j) & 1)) continue;
#pragma unroll
          for (int e0 = 0; e0 < 16; ++e0) {
            if ((e0 >> j) & 1) continue;
            const int e1 = e0 | (1 << j);
            const float2 a = v[e0], b = v[e1];
            v[e0] = make_float2(rx.x * a.x + rx.y * b.y, rx.x * a.y - rx.y * b.x);
            v[e1] = make_float2(rx.y * a.y + rx.x * b.x, -rx.y * a.x + rx.x * b.y);
          }
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          uint32_t idx = thr;
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if ((e >> j) & 1) idx |= rb[j];
          tile[bswz(idx)] = v[e];
        }
      }
      __syncthreads();
    }
    for (int c = t; c < T / 2; c += kBatchThreads) {
      const uint4 d = *reinterpret_cast<const uint4*>(&tile[bswz(2u * uint32_t(c))]);
      *reinterpret_cast<uint4*>(amp + gbase + bdep(2ull * c, P.tile)) = d;
    }
    __threadfence();
    __syncthreads();
    if (t == 0) atomicAdd(counters + I.step_base + k, 1u);
  }
}

// |+>^n: every amplitude 2^(-n/2)
__global__ void k6_init(const BatchInstance* __restrict__ insts) {
  const BatchInstance& I = insts[blockIdx.y];
  const uint64_t size = 1ull << I.n;
  const float a = float(exp2(-0.5 * double(I.n)));
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < size;
       i += uint64_t(gridDim.x) * blockDim.x)
    I.amp[i] = make_float2(a, 0.f);
}

// <H_C> = sum_x |a_x|^2 cut(x) in FP64: block (chunk, instance) sums 2^16
// consecutive amplitudes (16 per thread, cut by table), then one block per
// instance adds its chunk partials in order
constexpr int kChunkBits = 16;

__global__ void __launch_bounds__(256) k6_expect(const BatchInstance* __restrict__ insts,
                                                 double* __restrict__ partial, int max_chunks) {
  __shared__ double sh[8];
  const BatchInstance& I = insts[blockIdx.y];
  const int cb = I.n < kChunkBits ? I.n : kChunkBits;
  const uint64_t nchunks = 1ull << (I.n - cb);
  if (blockIdx.x >= nchunks) return;
  const uint64_t base = uint64_t(blockIdx.x) << cb;
  double s = 0;
  const uint8_t q[4] = {0, 1, 2, 3};
  for (uint64_t i = uint64_t(threadIdx.x) * 16; i < (1ull << cb); i += 256ull * 16) {
    int cut[16];
    cut_table(base + i, q, I, cut);
#pragma unroll
    for (int e = 0; e < 16; ++e) {
      const float2 a = I.amp[base + i + e];
      s += (double(a.x) * a.x + double(a.y) * a.y) * double(cut[e]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0;
    for (int w = 0; w < 8; ++w) r += sh[w];
    partial[size_t(blockIdx.y) * max_chunks + blockIdx.x] = r;
  }
}

__global__ void k6_expect_finish(const BatchInstance* __restrict__ insts,
                                 const double* __restrict__ partial, int max_chunks,
                                 double* __restrict__ out) {
  const BatchInstance& I = insts[blockIdx.x];
  if (threadIdx.x != 0) return;
  const int cb = I.n < kChunkBits ? I.n : kChunkBits;
  const uint64_t nchunks = 1ull << (I.n - cb);
  double s = 0;
  for (uint64_t c = 0; c < nchunks; ++c) s += partial[size_t(blockIdx.x) * max_chunks + c];
  out[blockIdx.x] = s;
}

}  // namespace

int launch_batch(const BatchInstance* d_inst, const BatchParams* d_par, const BatchItem* d_items,
                 int ngroups, uint64_t total_items, uint32_t* d_counters,
                 unsigned long long* d_head, int* d_err, int grid, cudaStream_t s) {
  k6_batch<<<grid, kBatchThreads, 0, s>>>(d_inst, d_par, d_items, ngroups, total_items,
                                          d_counters, d_head, d_err);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_batch_init(const BatchInstance* d_inst, int ninst, cudaStream_t s) {
  k6_init<<<dim3(64, ninst), 256, 0, s>>>(d_inst);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_batch_expect(const BatchInstance* d_inst, int ninst, int max_n, double* d_partial,
                        double* d_out, cudaStream_t s) {
  const int max_chunks = 1 << (max_n > kChunkBits ? max_n - kChunkBits : 0);
  k6_expect<<<dim3(max_chunks, ninst), 256, 0, s>>>(d_inst, d_partial, max_chunks);
  k6_expect_finish<<<ninst, 32, 0, s>>>(d_inst, d_partial, max_chunks, d_out);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace hisv
