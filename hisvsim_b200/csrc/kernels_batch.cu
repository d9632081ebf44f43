// K6: the batching form.  Many QAOA MaxCut instances of different qubit counts
// are advanced by ONE persistent launch.  A step of an instance is one pass
// over its complex64 state: a pass applies the mixer RX(2 beta) to its share
// of the qubits, and the pass that ends round r also applies the cost phase
// e^{i gamma/2 (2 cut(x) - |E|)} = prod_E RZZ(gamma) of round r+1 and round
// r+1's RX on the same qubits (the rounds run their passes in alternating
// order, so the pass that ends one round starts the next; the planner's
// descriptors say what each register-group visit applies).  The tiles of a step are cut
// into chunks; CTAs take chunks from a global queue in step order and stream
// their tiles through two shared-memory buffers (the next tile loads while
// the current one is processed).  A chunk of step k waits until every chunk
// of step k-1 of its instance is done (a completion counter); chunks are
// dequeued in step order, so the earliest unfinished chunk never waits and
// the queue always drains.  Waits are bounded: a timeout sets an error flag.
//
// cut(x) in a phase pass: with the outer bits fixed, cut(x) = cut_table[i] +
// C + sum_b w_b i_b over the tile bits b, where cut_table counts the edges
// with both ends in the tile (a table per phase pass), C the edges outside it
// plus the crossing edges whose outer end is 1, and w_b = (#crossing edges
// at tile bit b whose outer end is 0) - (#those whose outer end is 1).
#include "bounds.cuh"
#include "internal.h"

namespace hisv {
namespace {

// a CTA of NT threads holds tiles of up to 16 NT amplitudes (16 per thread)
// default polls (with ~0.1 us sleeps) of a dependency wait before it gives
// up; the batch keeps its own limit in device memory (hs_batch_set_wait_limit)
constexpr uint32_t kDepLimit = 1u << 24;

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
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int NT>
struct Shared {
  alignas(16) uint8_t cut[16 * NT];
  BatchPass pass;  // the item's pass, copied once per item
  float2 phase[kBatchMaxEdges + 1];
  uint8_t ea[kBatchMaxEdges], eb[kBatchMaxEdges];
  uint64_t gk[8];  // global offset of chunk k * NT
  uint32_t gro[4];  // last group: global offset of each register bit
  float2 rx[2];     // (cos beta, sin beta) of rounds ra and rb
  int w[2][16];  // per tile buffer: warp 0 prepares the next tile's weights
  int c[2];      // while the other warps may still read the current ones
  int group;
  int abort;
  unsigned long long item;
};

// (C, w) of the tile whose outer bits are gbase (warp 0 only): tbit[q] is the
// tile bit of qubit q or -1; an edge with one end in the tile at bit b adds
// i_b (outer end 0) or 1 - i_b (outer end 1), one with both ends outside adds
// its fixed value, and edges inside the tile are in the pass's cut table
template <class Sh>
__device__ __forceinline__ void cross_weights(Sh& S, int nedges, const int8_t* tbit, uint64_t gbase,
                                              int buf) {
  const int lane = threadIdx.x & 31;
  int* w = S.w[buf];
  if (lane < 16) w[lane] = 0;
  __syncwarp();
  int c = 0;
  for (int e = lane; e < nedges; e += 32) {
    const int a = S.ea[e], b = S.eb[e];
    const int ta = tbit[a], tb = tbit[b];
    const int xa = int((gbase >> a) & 1ull), xb = int((gbase >> b) & 1ull);
    if (ta < 0 && tb < 0) {
      c += xa ^ xb;
    } else if (ta >= 0 && tb < 0) {
      c += xb;
      atomicAdd(&w[ta], xb ? -1 : 1);
    } else if (ta < 0 && tb >= 0) {
      c += xa;
      atomicAdd(&w[tb], xa ? -1 : 1);
    }
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) S.c[buf] = c;
}

template <int NT>
__global__ void __launch_bounds__(NT, NT == 128 ? 6 : 3)
    k6_batch(const BatchInstance* __restrict__ insts, const BatchParams* __restrict__ pars,
             const BatchItem* __restrict__ groups, int ngroups, uint64_t total,
             uint32_t* __restrict__ counters, unsigned long long* __restrict__ head,
             int* __restrict__ err, const uint32_t* __restrict__ wait_limit) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kTileMax = 16 * NT;
  constexpr int kBatchThreads = NT;
  float2* tiles = reinterpret_cast<float2*>(smem_raw);  // two buffers of kTileMax
  Shared<NT>& S = *reinterpret_cast<Shared<NT>*>(smem_raw + 2 * kTileMax * sizeof(float2));
  const int t = threadIdx.x;
  const uint32_t tiles_s = uint32_t(__cvta_generic_to_shared(tiles));
  const uint32_t limit = *wait_limit;
  for (;;) {
    if (t == 0) {
      const unsigned long long item = atomicAdd(head, 1ull);
      S.item = item;
      S.abort = 0;
      if (item < total) {
        // the item's (instance, step) group: last group with first <= item
        int lo = 0, hi = ngroups - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (groups[mid].first <= item) lo = mid; else hi = mid - 1;
        }
        S.group = lo;
        const BatchItem& G = groups[lo];
        if (G.step > 0) {  // every chunk of the previous step of this instance
          const uint32_t* cnt = counters + insts[G.inst].step_base + (G.step - 1);
          uint32_t polls = 0, seen;
          do {
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(seen) : "l"(cnt) : "memory");
            if (seen >= G.need) break;
            __nanosleep(100);
          } while (++polls < limit);
          if (seen < G.need) {
            S.abort = 1;
            atomicExch(err, 1);
          }
        }
      }
    }
    __syncthreads();
    const unsigned long long item = S.item;
    if (item >= total || S.abort) break;
    const BatchItem G = groups[S.group];
    const BatchInstance& I = insts[G.inst];
    const int k = G.step;
    {
      // the pass descriptor is read many times per tile: keep it in shared memory
      static_assert(sizeof(BatchPass) % 4 == 0, "BatchPass words");
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&I.pass[k]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&S.pass);
      for (int w = t; w < int(sizeof(BatchPass) / 4); w += kBatchThreads) dst[w] = src[w];
    }
    __syncthreads();
    const BatchPass& P = S.pass;
    const int m = P.m, T = 1 << m, ngr = P.ngroups, nv = P.nvisits, nedges = I.nedges;
    const bool phase = P.phase != 0;
    const uint32_t t_begin = uint32_t(item - G.first) * G.chunk;
    const uint32_t t_end = min(G.ntiles, t_begin + G.chunk);
    float2* amp = I.amp;
    if (phase) {
      if (t < nedges + 1) S.phase[t] = pars[G.inst].phase[P.rb][t];
      if (t < nedges) {
        S.ea[t] = I.edge_a[t];
        S.eb[t] = I.edge_b[t];
      }
      const uint4* cs = reinterpret_cast<const uint4*>(I.cut + P.cut_off);
      uint4* cd = reinterpret_cast<uint4*>(S.cut);
      for (int i = t; i < (T + 15) / 16; i += kBatchThreads) cd[i] = cs[i];
    }
    if (t == 0) {
      S.rx[0] = pars[G.inst].rx[P.ra][0];  // (cos beta, sin beta) of round ra
      S.rx[1] = pars[G.inst].rx[P.rb][0];  // and of round rb
    }
    const bool active = t < (T >> 4);
    // 16-byte chunk c = t + k * threads covers tile indices 2c, 2c + 1; the
    // bits of t and of k * threads are disjoint, so its global offset is
    // bdep(2t) + bdep(2k * threads)
    const int nck = (T / 2 + kBatchThreads - 1) / kBatchThreads;
    if (t < nck) S.gk[t] = bdep(2ull * uint64_t(t) * kBatchThreads, P.tile);
    const uint64_t gt = bdep(2ull * t, P.tile);
    // thread bits of each register group: the tile bits not held in registers;
    // bswz is linear over GF(2), so a register element's slot is
    // bswz(thread part) ^ (XOR of bswz(register bit))
    // (the thread part of group g, recomputed where the phase needs it)
    auto thread_part = [&](int g) {
      uint32_t rmask = 0, thr = 0;
      for (int j = 0; j < 4; ++j) rmask |= 1u << P.group_bits[g][j];
      int src = 0;
      for (int b = 0; b < m; ++b)
        if (!((rmask >> b) & 1u)) thr |= uint32_t((t >> src++) & 1) << b;
      return thr;
    };
    uint32_t sbase[3] = {0, 0, 0};
    for (int g = 0; g < ngr; ++g) sbase[g] = bswz(thread_part(g));
    // the last visit writes its registers straight to global memory: the
    // thread part's offset and each register bit's offset (disjoint bits add)
    // (instances have at most 30 qubits, so offsets within a state fit 32 bits)
    const int glast = P.visit_group[nv - 1];
    const uint32_t gl_base = uint32_t(bdep(thread_part(glast), P.tile));
    if (t < 4) S.gro[t] = uint32_t(bdep(1ull << P.group_bits[glast][t], P.tile));
    __syncthreads();  // S.gk, S.gro, S.rx
    // prologue: first tile into buffer 0
    {
      const uint64_t gb = bdep(t_begin, P.outer) + gt;
      for (int k = 0, c = t; c < T / 2; ++k, c += kBatchThreads)
        if (HS_IN_BOUNDS(gb + S.gk[k] + 2 <= (1ull << I.n) && bswz(2u * uint32_t(c)) + 2 <= uint32_t(T),
                         kBoundsK6))
          cp16(tiles_s + bswz(2u * uint32_t(c)) * 8u, amp + gb + S.gk[k]);
      cp_commit();
    }
    for (uint32_t ti = t_begin; ti < t_end; ++ti) {
      const int buf = int(ti - t_begin) & 1;
      float2* tile = tiles + buf * kTileMax;
      const uint64_t gbase = bdep(ti, P.outer);
      cp_wait<0>();  // this tile's copies (the only ones in flight)
      if (phase && t < 32) cross_weights(S, nedges, P.tbit, gbase, buf);
      // one barrier per tile: every thread's copies and the weights are
      // visible, and every thread is past the previous tile's last visit,
      // so the other buffer may be refilled
      __syncthreads();
      if (ti + 1 < t_end) {
        const uint64_t nb = bdep(ti + 1, P.outer) + gt;
        const uint32_t ns = tiles_s + uint32_t((buf ^ 1) * kTileMax * 8);
        for (int k = 0, c = t; c < T / 2; ++k, c += kBatchThreads)
          if (HS_IN_BOUNDS(nb + S.gk[k] + 2 <= (1ull << I.n) && bswz(2u * uint32_t(c)) + 2 <= uint32_t(T),
                           kBoundsK6))
            cp16(ns + bswz(2u * uint32_t(c)) * 8u, amp + nb + S.gk[k]);
        cp_commit();
      }
      for (int vi = 0; vi < nv; ++vi) {
        const int g = P.visit_group[vi];
        const uint32_t sbg = sbase[g];
        if (active) {
          uint32_t so[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) so[j] = bswz(1u << P.group_bits[g][j]);
          float2 v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            uint32_t a = sbg;
#pragma unroll
            for (int j = 0; j < 4; ++j)
              if ((e >> j) & 1) a ^= so[j];
            if (HS_IN_BOUNDS(a < uint32_t(T), kBoundsK6)) v[e] = tile[a];
          }
          // mixer RX(2 beta) = [[c, -i s], [-i s, c]] on register bit j
          auto rx_bit = [&](int j, float2 rx) {
#pragma unroll
            for (int e0 = 0; e0 < 16; ++e0) {
              if ((e0 >> j) & 1) continue;
              const int e1 = e0 | (1 << j);
              const float2 a = v[e0], b = v[e1];
              v[e0] = make_float2(rx.x * a.x + rx.y * b.y, rx.x * a.y - rx.y * b.x);
              v[e1] = make_float2(rx.y * a.y + rx.x * b.x, -rx.y * a.x + rx.x * b.y);
            }
          };
          auto rx_mask = [&](int gm, float2 rx) {
            if (gm == 15) {  // the common case: all four register bits are targets
              rx_bit(0, rx);
              rx_bit(1, rx);
              rx_bit(2, rx);
              rx_bit(3, rx);
            } else {
              if (gm & 1) rx_bit(0, rx);
              if (gm & 2) rx_bit(1, rx);
              if (gm & 4) rx_bit(2, rx);
              if (gm & 8) rx_bit(3, rx);
            }
          };
          // RX of round ra, then the cost phase and RX of round rb: one copy
          // of the RX code for both
#pragma unroll 1
          for (int h = 0; h < 2; ++h) {
            if (h == 1 && P.ph[vi]) {
              // cut = cut_table[i] + C + sum_b w_b i_b over the tile bits b
              const uint32_t thr = thread_part(g);
              const int* wt = S.w[buf];
              int dthr = S.c[buf];
              for (int b = 0; b < m; ++b)
                if ((thr >> b) & 1u) dthr += wt[b];
              int wr[4];
              uint32_t rb[4];
#pragma unroll
              for (int j = 0; j < 4; ++j) {
                wr[j] = wt[P.group_bits[g][j]];
                rb[j] = 1u << P.group_bits[g][j];
              }
#pragma unroll
              for (int e = 0; e < 16; ++e) {
                uint32_t idx = thr;
                int cc = dthr;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                  if ((e >> j) & 1) {
                    idx |= rb[j];
                    cc += wr[j];
                  }
                if (!HS_IN_BOUNDS(idx < uint32_t(T) && int(S.cut[idx]) + cc >= 0 &&
                                      int(S.cut[idx]) + cc <= nedges,
                                  kBoundsK6))
                  continue;
                const float2 ph = S.phase[int(S.cut[idx]) + cc];
                const float2 a = v[e];
                v[e] = make_float2(ph.x * a.x - ph.y * a.y, ph.x * a.y + ph.y * a.x);
              }
            }
            const int gm = h ? P.rx_b[vi] : P.rx_a[vi];
            if (gm) rx_mask(gm, S.rx[h]);
          }
          if (vi == nv - 1) {
            // last visit: registers straight to global memory (the lanes run
            // over the low, contiguous tile bits, so the stores coalesce)
            float2* base = amp + gbase + gl_base;
            uint32_t ro[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) ro[j] = S.gro[j];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              uint32_t off = 0;
#pragma unroll
              for (int j = 0; j < 4; ++j)
                if ((e >> j) & 1) off += ro[j];
              if (HS_IN_BOUNDS(gbase + gl_base + off < (1ull << I.n), kBoundsK6)) base[off] = v[e];
            }
          } else {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              uint32_t a = sbg;
#pragma unroll
              for (int j = 0; j < 4; ++j)
                if ((e >> j) & 1) a ^= so[j];
              if (HS_IN_BOUNDS(a < uint32_t(T), kBoundsK6)) tile[a] = v[e];
            }
          }
        }
        // the next visit reads what this one wrote; after the last visit the
        // next tile's first barrier protects the buffer
        if (vi < nv - 1) __syncthreads();
      }
    }
    __threadfence();
    __syncthreads();
    if (t == 0) atomicAdd(counters + I.step_base + k, 1u);
  }
}

template <int NT>
constexpr size_t batch_smem() {
  return 2 * 16 * NT * sizeof(float2) + sizeof(Shared<NT>);
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

// <H_C> = sum_x |a_x|^2 cut(x) in FP64.  Block (b, instance) takes ranges of
// 2^m amplitudes (m = the first phase pass's tile bits, so its cut table applies) r = b,
// b + gridDim.x, ...; per range warp 0 derives C and w_q as in K6, then every
// thread sums its amplitudes.  Per-block partials, added in order by
// k6_expect_finish: the result does not depend on timing.
constexpr int kExpectBlocks = 256;

__global__ void __launch_bounds__(256) k6_expect(const BatchInstance* __restrict__ insts,
                                                 double* __restrict__ partial) {
  __shared__ Shared<256> S;  // cut table for tiles of up to 2^12
  __shared__ double sh[8];
  const BatchInstance& I = insts[blockIdx.y];
  const int m = I.pass[0].m, nedges = I.nedges, t = threadIdx.x;
  const uint64_t nranges = 1ull << (I.n - m);
  // step 0 is the first phase pass: its tile is qubits [0, m), its cut table
  // comes first
  for (int i = t; i < (1 << m); i += 256) S.cut[i] = I.cut[I.pass[0].cut_off + i];
  if (t < nedges) {
    S.ea[t] = I.edge_a[t];
    S.eb[t] = I.edge_b[t];
  }
  double s = 0;
  for (uint64_t r = blockIdx.x; r < nranges; r += gridDim.x) {
    __syncthreads();
    if (t < 32) cross_weights(S, nedges, I.pass[0].tbit, r << m, 0);
    __syncthreads();
    const float2* a = I.amp + (r << m);
    for (int i = t; i < (1 << m); i += 256) {
      int c = S.c[0] + int(S.cut[i]);
      for (int b = 0; b < m; ++b)
        if ((i >> b) & 1) c += S.w[0][b];
      const float2 v = a[i];
      s += (double(v.x) * v.x + double(v.y) * v.y) * double(c);
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((t & 31) == 0) sh[t >> 5] = s;
  __syncthreads();
  if (t == 0) {
    double r = 0;
    for (int w = 0; w < 8; ++w) r += sh[w];
    partial[size_t(blockIdx.y) * kExpectBlocks + blockIdx.x] = r;
  }
}

__global__ void k6_expect_finish(const double* __restrict__ partial, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0;
  for (int b = 0; b < kExpectBlocks; ++b) s += partial[size_t(blockIdx.x) * kExpectBlocks + b];
  out[blockIdx.x] = s;
}

}  // namespace

namespace {
template <int NT>
int max_ctas() {
  int n = 0;
  if (cudaFuncSetAttribute(k6_batch<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(batch_smem<NT>())) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k6_batch<NT>, NT, batch_smem<NT>()) !=
          cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return n < 1 ? 1 : n;
}
}  // namespace

#ifdef HS_BOUNDS
HS_BOUNDS_TAKE(bounds_take_batch)
#endif

int batch_max_ctas_per_sm(int threads) {
  return threads == 256 ? max_ctas<256>() : max_ctas<128>();
}

int launch_batch(const BatchInstance* d_inst, const BatchParams* d_par, const BatchItem* d_items,
                 int ngroups, uint64_t total_items, uint32_t* d_counters,
                 unsigned long long* d_head, int* d_err, const uint32_t* d_limit, int grid,
                 int threads, cudaStream_t s) {
  if (threads == 256) {
    HS_CUDA(cudaFuncSetAttribute(k6_batch<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(batch_smem<256>())));
    k6_batch<256><<<grid, 256, batch_smem<256>(), s>>>(d_inst, d_par, d_items, ngroups,
                                                        total_items, d_counters, d_head, d_err, d_limit);
  } else {
    HS_CUDA(cudaFuncSetAttribute(k6_batch<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(batch_smem<128>())));
    k6_batch<128><<<grid, 128, batch_smem<128>(), s>>>(d_inst, d_par, d_items, ngroups,
                                                        total_items, d_counters, d_head, d_err, d_limit);
  }
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_batch_init(const BatchInstance* d_inst, int ninst, cudaStream_t s) {
  k6_init<<<dim3(64, ninst), 256, 0, s>>>(d_inst);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

// d_partial: ninst x kExpectBlocks doubles
int launch_batch_expect(const BatchInstance* d_inst, int ninst, int max_n, double* d_partial,
                        double* d_out, cudaStream_t s) {
  (void)max_n;
  k6_expect<<<dim3(kExpectBlocks, ninst), 256, 0, s>>>(d_inst, d_partial);
  k6_expect_finish<<<ninst, 32, 0, s>>>(d_partial, d_out);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace hisv
