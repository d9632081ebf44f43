// Precision form: each part (<= 6 qubits) is fused into a 64x64 complex
// unitary composed in FP64 (K5) and applied to a complex64 state on the
// tcgen05 tensor cores (K4) as a real GEMM with split-BF16 operands and FP32
// accumulation.
//
// Complex product Y = U X as one real product with (re, im) interleaved:
//     Y[2p + c] = sum_k A[2p + c][k] X[k],  A[2po+co][2pi+ci] = the 2x2 real
//     block [[Re, -Im], [Im, Re]] of U(po, pi)   (A: 128 x 128, B: 128 x N)
// with X the tile viewed as 64 (part index) x N (other tile bits).  Each FP32
// operand x is split as hi = bf16(x), lo = bf16(x - hi) and the product is
// Ah*Bh + Ah*Bl + Al*Bh (the Al*Bl term, ~2^-16 relative, is dropped).
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>

#include "bounds.cuh"
#include "internal.h"
#include "tcgen05.cuh"

namespace hisv {
namespace {

// The real form with (re, im) interleaved: row r = 2*po + co, column
// k = 2*pi + ci holds Re U (co = ci), -Im U (co=0, ci=1) or Im U (co=1, ci=0)
// of U(po, pi); stored as BF16 hi / lo in the K-major operand layout.  Thread
// j of 64 handles every 64th element.
__device__ void pack_real_form(const double2* __restrict__ U, uint8_t* __restrict__ ao, int j) {
  for (int e = j; e < 128 * 128; e += kFusedDim) {
    const int r = e >> 7, c = e & 127;
    const double2 u = U[(r >> 1) * kFusedDim + (c >> 1)];
    const int co = r & 1, ci = c & 1;
    const double x = co == ci ? u.x : (co == 0 ? -u.y : u.y);
    const __nv_bfloat16 hi = __double2bfloat16(x);
    const __nv_bfloat16 lo = __double2bfloat16(x - double(__bfloat162float(hi)));
    const uint32_t off = tc::kmajor_off(uint32_t(r), uint32_t(c), 2048u);
    *reinterpret_cast<__nv_bfloat16*>(ao + off) = hi;
    *reinterpret_cast<__nv_bfloat16*>(ao + kFusedABytes / 2 + off) = lo;
  }
}

// ---- K5: compose each part's unitary in FP64 --------------------------------
// One CTA per part, thread j owns column j of U (the image of basis state j);
// U lives row-major in shared memory so that a warp's accesses are contiguous.
__global__ void __launch_bounds__(64) k5_compose(const FusedGate* __restrict__ gates,
                                                 const int32_t* __restrict__ offs,
                                                 double2* __restrict__ u_out,
                                                 uint8_t* __restrict__ a_out) {
  extern __shared__ __align__(16) double2 U[];  // [64][64]
  const int part = blockIdx.x;
  const int j = threadIdx.x;
  for (int i = 0; i < kFusedDim; ++i) U[i * kFusedDim + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  for (int g = offs[part]; g < offs[part + 1]; ++g) {
    const FusedGate& G = gates[g];
    if (G.nt == 1) {
      const int t = 1 << G.t0;
      for (int i = 0; i < kFusedDim; ++i) {
        if ((i & t) || (i & G.cmask) != G.cmask) continue;
        const double2 a = U[i * kFusedDim + j], b = U[(i | t) * kFusedDim + j];
        const double2 m0 = G.m[0], m1 = G.m[1], m2 = G.m[2], m3 = G.m[3];
        U[i * kFusedDim + j] = make_double2(m0.x * a.x - m0.y * a.y + m1.x * b.x - m1.y * b.y,
                                            m0.x * a.y + m0.y * a.x + m1.x * b.y + m1.y * b.x);
        U[(i | t) * kFusedDim + j] =
            make_double2(m2.x * a.x - m2.y * a.y + m3.x * b.x - m3.y * b.y,
                         m2.x * a.y + m2.y * a.x + m3.x * b.y + m3.y * b.x);
      }
    } else {
      const int b0 = 1 << G.t0, b1 = 1 << G.t1;
      for (int i = 0; i < kFusedDim; ++i) {
        if ((i & (b0 | b1)) || (i & G.cmask) != G.cmask) continue;
        const int idx[4] = {i, i | b1, i | b0, i | b0 | b1};  // reference index 2*b(t0)+b(t1)
        double2 in[4];
        for (int q = 0; q < 4; ++q) in[q] = U[idx[q] * kFusedDim + j];
        for (int r = 0; r < 4; ++r) {
          double re = 0, im = 0;
          for (int q = 0; q < 4; ++q) {
            const double2 c = G.m[4 * r + q];
            re += c.x * in[q].x - c.y * in[q].y;
            im += c.x * in[q].y + c.y * in[q].x;
          }
          U[idx[r] * kFusedDim + j] = make_double2(re, im);
        }
      }
    }
  }
  __syncthreads();
  if (u_out) {
    double2* uo = u_out + size_t(part) * kFusedDim * kFusedDim;
    for (int i = 0; i < kFusedDim; ++i) uo[i * kFusedDim + j] = U[i * kFusedDim + j];
  }
  pack_real_form(U, a_out + size_t(part) * kFusedABytes, j);
}

// A user-supplied unitary (row-major 64 x 64 per part) packed the same way
__global__ void __launch_bounds__(64) k5_pack(const double2* __restrict__ u,
                                              uint8_t* __restrict__ a_out) {
  pack_real_form(u + size_t(blockIdx.x) * kFusedDim * kFusedDim,
                 a_out + size_t(blockIdx.x) * kFusedABytes, threadIdx.x);
}

// ---- K4: apply fused unitaries to complex64 tiles on the tensor cores --------
constexpr int kK4Threads = 256;
constexpr uint32_t kK4TmemCols = 64;     // FP32 accumulator: 128 lanes x N <= 64 columns
constexpr uint32_t kK4DirectCols = 128;  // the direct form: N <= 128 columns, two accumulators
constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before giving up

__device__ __forceinline__ uint64_t dep(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i) out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}

// tile buffer position of tile index i: bits 1..3 XOR a fold of bits >= 4, so
// that accesses spread over the banks; bit 0 is kept so that the two
// amplitudes of a 16-byte chunk stay adjacent
__device__ __forceinline__ uint32_t tswz(uint32_t i) {
  return i ^ ((((i >> 4) ^ (i >> 7) ^ (i >> 10)) & 7u) << 1);
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared memory: [A: nops x 64 KiB][B hi | B lo: N x 256 B each]
//                [tile buffers: 2 x 2^m complex64][tables][mbarrier][TMEM address]
// The next tile streams into the second buffer (cp.async, 16-byte chunks of two
// amplitudes) while the current one is processed.
__global__ void __launch_bounds__(kK4Threads, 2)
    k4_fused(float2* __restrict__ sv, const __grid_constant__ FusedPass P,
             const uint8_t* __restrict__ a_all, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m = P.m;
  const int T = 1 << m;            // tile amplitudes
  const int N = T >> kFusedBits;   // GEMM columns
  const int lgN = m - kFusedBits;
  const uint32_t bk = uint32_t(N) * 16u;  // B: bytes between K-blocks of 8
  uint8_t* sA = sm;
  uint8_t* sBh = sA + P.nops * kFusedABytes;
  uint8_t* sBl = sBh + N * 256;
  float* buf0 = reinterpret_cast<float*>(sBl + N * 256);  // interleaved (re, im)
  float* buf1 = buf0 + 2 * T;
  uint16_t* dp = reinterpret_cast<uint16_t*>(buf1 + 2 * T);  // [nops][64]
  uint16_t* dn = dp + P.nops * 64;                            // [nops][N]
  uint64_t* gk = reinterpret_cast<uint64_t*>(
      (reinterpret_cast<uintptr_t>(dn + P.nops * N) + 7) & ~uintptr_t(7));  // chunk-row offsets
  uint64_t* mbar = gk + 8;
  uint32_t* tmem_base = reinterpret_cast<uint32_t*>(mbar + 1);

  for (int o = 0; o < P.nops; ++o) {
    const uint4* src = reinterpret_cast<const uint4*>(a_all + size_t(P.part[o]) * kFusedABytes);
    uint4* dst = reinterpret_cast<uint4*>(sA + o * kFusedABytes);
    for (int i = t; i < kFusedABytes / 16; i += kK4Threads) dst[i] = src[i];
  }
  for (int o = 0; o < P.nops; ++o) {
    uint32_t pmask = 0;
    for (int b = 0; b < kFusedBits; ++b) pmask |= 1u << P.pbits[o][b];
    for (int p = t; p < 64; p += kK4Threads) {
      uint32_t x = 0;
      for (int b = 0; b < kFusedBits; ++b) x |= uint32_t((p >> b) & 1) << P.pbits[o][b];
      dp[o * 64 + p] = uint16_t(tswz(x));
    }
    for (int nn = t; nn < N; nn += kK4Threads) {
      uint32_t x = 0, bit = 0;
      for (int b = 0; b < m; ++b)
        if (!((pmask >> b) & 1)) x |= uint32_t((nn >> bit++) & 1) << b;
      dn[o * N + nn] = uint16_t(tswz(x));
    }
  }
  // chunk c = t + r*256 holds tile indices 2c, 2c+1 (tile bit 0 is slot 0);
  // its global index is dep(2t) + dep(2*r*256)
  const int chunks = T / 2, rows = chunks / kK4Threads;
  for (int r = t; r < rows; r += kK4Threads) gk[r] = dep(uint64_t(r) * kK4Threads * 2, P.tile);
  if (t == 0) tc::mbar_init(mbar, 1);
  if (warp == 0) {
    tc::tmem_alloc(tmem_base, kK4TmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_base;
  const uint64_t gt = dep(uint64_t(t) * 2, P.tile);
  const uint32_t idesc = tc::idesc_bf16_f32(128, uint32_t(N));
  const uint32_t sb[2] = {tc::smem_u32(buf0), tc::smem_u32(buf1)};
  uint32_t phase = 0;
  bool failed = false;

  auto issue_load = [&](uint64_t tl, uint32_t dst) {
    const uint64_t gb = dep(tl, P.outer);
    for (int r = 0; r < rows; ++r)
      cp_async16(dst + tswz(2u * uint32_t(t + r * kK4Threads)) * 8u, sv + gb + gt + gk[r]);
    (void)0;
  };
  uint64_t tile = blockIdx.x;
  if (tile < P.ntiles) issue_load(tile, sb[0]);
  cp_async_commit();
  for (int it = 0; tile < P.ntiles; ++it, tile += gridDim.x) {
    const uint64_t next = tile + gridDim.x;
    if (next < P.ntiles) issue_load(next, sb[(it + 1) & 1]);
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    float* X = (it & 1) ? buf1 : buf0;
    const uint64_t gbase = dep(tile, P.outer);
    for (int o = 0; o < P.nops; ++o) {
      // B (N x 128, K-major), k = 2p + c: Re (c=0) / Im (c=1) of part index p.
      // Item (kb, nn): K-block kb (part indices 4kb..4kb+3) of column nn; lanes
      // run over consecutive columns, i.e. over the low tile bits.
      for (int item = t; item < N * 16; item += kK4Threads) {
        const int kb = item >> lgN, nn = item & (N - 1);
        const uint32_t col = dn[o * N + nn];
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 x = *reinterpret_cast<const float2*>(X + 2 * (dp[o * 64 + 4 * kb + q] ^ col));
          const __nv_bfloat162 h = __floats2bfloat162_rn(x.x, x.y);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(x.x - hf.x, x.y - hf.y);
          hw[q] = *reinterpret_cast<const uint32_t*>(&h);
          lw[q] = *reinterpret_cast<const uint32_t*>(&l);
        }
        const uint32_t off = tc::kmajor_off(uint32_t(nn), uint32_t(kb * 8), bk);
        *reinterpret_cast<uint4*>(sBh + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(sBl + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
      }
      tc::fence_proxy_async_smem();
      __syncthreads();
      if (t == 0) {
        tc::tc_fence_after();
        const uint32_t a0 = tc::smem_u32(sA + o * kFusedABytes);
        const uint32_t bh = tc::smem_u32(sBh), bl = tc::smem_u32(sBl);
        const int nprod = P.precision == 1 ? 1 : 3;
        uint32_t acc = 0;
        for (int prod = 0; prod < nprod; ++prod) {
          const uint32_t abase = a0 + (prod == 2 ? uint32_t(kFusedABytes / 2) : 0u);  // Al: third
          const uint32_t bbase = prod == 1 ? bl : bh;                                 // Bl: second
          for (int s = 0; s < 8; ++s) {  // K = 128 in steps of 16 (two 8-wide blocks)
            const uint64_t ad = tc::smem_desc(abase + uint32_t(s) * 2u * 2048u, 2048u, 128u);
            const uint64_t bd = tc::smem_desc(bbase + uint32_t(s) * 2u * bk, bk, 128u);
            tc::mma_bf16(tmem, ad, bd, idesc, acc);
            acc = 1;
          }
        }
        tc::mma_commit(mbar);
      }
      const bool ok = tc::mbar_wait(mbar, phase, kWaitLimit);
      if (__syncthreads_or(!ok)) {  // block-uniform decision
        failed = true;
        if (t == 0) atomicExch(err, 1);
        tc::mbar_wait(mbar, phase, kWaitLimit);  // give the MMAs a last bounded chance
        break;
      }
      phase ^= 1u;
      tc::tc_fence_after();
      {
        // D row r = 2p + c (TMEM lane r): Re (c=0) / Im (c=1) of part index p.
        // Warp w reads lanes 32*(w%4).. and half of the columns, 16 at a time
        // (with N = 16 the second half-group idles).
        const int quad = warp & 3, half = warp >> 2;
        const int r = quad * 32 + lane;
        const int comp = r & 1;
        const uint32_t prow = dp[o * 64 + (r >> 1)];
        const int per_half = N / 2 < 16 ? 16 : N / 2;
        const int c_begin = half * per_half;
        const int c_end = c_begin + per_half < N ? c_begin + per_half : N;
        for (int c0 = c_begin; c0 + 16 <= c_end; c0 += 16) {
          float d[16];
          tc::tmem_ld16(tmem + (uint32_t(quad * 32) << 16) + uint32_t(c0), d);
          // the 16 column positions are the same for every lane: read them as
          // eight broadcast 32-bit words
          const uint32_t* cw = reinterpret_cast<const uint32_t*>(dn + o * N + c0);
#pragma unroll
          for (int j = 0; j < 16; j += 2) {
            const uint32_t w = cw[j >> 1];
            X[2 * (prow ^ (w & 0xffffu)) + comp] = d[j];
            X[2 * (prow ^ (w >> 16)) + comp] = d[j + 1];
          }
        }
      }
      tc::tc_fence_before();
      __syncthreads();
    }
    if (failed) break;
    // write the tile back: 16-byte chunks, coalesced
    for (int r = 0; r < rows; ++r) {
      const uint4 d = *reinterpret_cast<const uint4*>(X + 2 * tswz(2u * uint32_t(t + r * kK4Threads)));
      __stcs(reinterpret_cast<uint4*>(sv + gbase + gt + gk[r]), d);
    }
    __syncthreads();  // this buffer is refilled by the prefetch issued next iteration
  }
  cp_async_wait0();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kK4TmemCols);
}

// ---- K4, one unitary per pass, operands straight from and to HBM ------------
// The tile never sits in shared memory as complex64: each thread loads its
// amplitudes from global memory (coalesced over the tile's columns), splits
// them into the BF16 hi / lo B operands, and the epilogue moves results from
// TMEM to global memory directly (re / im paired by a lane shuffle).  Only A
// (64 KiB) and two B buffers live in shared memory, so tiles can be 2^13
// amplitudes (N = 128 columns, half the tensor-core operand reads per
// amplitude of N = 64).  Tile i's MMAs run while tile i+1's loads are in flight
// and tile i-1 drains; two TMEM accumulators and two B buffers alternate.
// Shared memory: [A][B0 hi|lo][B1 hi|lo][gp: 64 x u64][gn: N x u64][2 mbarriers][TMEM address]
constexpr int kK4DirectThreads = 512;  // 16 warps: four per TMEM lane quadrant
constexpr int kK4DirectItems = 4;      // B items per thread (N * 16 / 512 for N = 128)

__global__ void __launch_bounds__(kK4DirectThreads, 1)
    k4_direct(float2* __restrict__ sv, const __grid_constant__ FusedPass P,
              const uint8_t* __restrict__ a_all, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m = P.m;
  const int N = 1 << (m - kFusedBits);
  const int lgN = m - kFusedBits;
  const uint32_t bk = uint32_t(N) * 16u;
  const uint32_t bbytes = uint32_t(N) * 256u;
  uint8_t* sA = sm;
  uint8_t* sB = sA + kFusedABytes;  // [2][hi|lo]
  uint64_t* gp = reinterpret_cast<uint64_t*>(sB + 4 * bbytes);  // part index -> global offset
  uint64_t* gn = gp + 64;                                        // column -> global offset
  uint64_t* mbar = gn + N;                                       // [2]
  uint32_t* tmem_base = reinterpret_cast<uint32_t*>(mbar + 2);

  {
    const uint4* src = reinterpret_cast<const uint4*>(a_all + size_t(P.part[0]) * kFusedABytes);
    uint4* dst = reinterpret_cast<uint4*>(sA);
    for (int i = t; i < kFusedABytes / 16; i += kK4DirectThreads) dst[i] = src[i];
  }
  uint32_t pmask = 0;
  for (int b = 0; b < kFusedBits; ++b) pmask |= 1u << P.pbits[0][b];
  for (int p = t; p < 64; p += kK4DirectThreads) {
    uint64_t x = 0;
    for (int b = 0; b < kFusedBits; ++b) x |= uint64_t((p >> b) & 1) << P.pbits[0][b];
    gp[p] = dep(x, P.tile);
  }
  for (int nn = t; nn < N; nn += kK4DirectThreads) {
    uint64_t x = 0;
    int bit = 0;
    for (int b = 0; b < m; ++b)
      if (!((pmask >> b) & 1)) x |= uint64_t((nn >> bit++) & 1) << b;
    gn[nn] = dep(x, P.tile);
  }
  if (t == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_base, 2 * kK4DirectCols);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_base;
  const uint32_t idesc = tc::idesc_bf16_f32(128, uint32_t(N));
  const int nprod = P.precision == 1 ? 1 : 3;
  const int nitems = (N * 16 + kK4DirectThreads - 1) / kK4DirectThreads;  // 1..4
  const bool pairs = (gn[1] == 1);  // column bit 0 is global slot 0: columns pair up in 16 B
  uint32_t phase[2] = {0, 0};
  bool pend[2] = {false, false};
  bool failed = false;
  const uint64_t cnt =
      blockIdx.x < P.ntiles ? (P.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto tile_of = [&](uint64_t i) { return blockIdx.x + i * gridDim.x; };

  // this thread's B items: item = t + k * 256 -> (kb, nn)
  float2 L[kK4DirectItems][4];
  auto load_tile = [&](uint64_t i) {
    const float2* base = sv + dep(tile_of(i), P.outer);
#pragma unroll
    for (int k = 0; k < kK4DirectItems; ++k) {
      if (k >= nitems) break;
      const int item = t + k * kK4DirectThreads;
      if (item >= N * 16) break;
      const int kb = item >> lgN, nn = item & (N - 1);
      const float2* col = base + gn[nn];
#pragma unroll
      for (int q = 0; q < 4; ++q) L[k][q] = __ldcs(col + gp[4 * kb + q]);
    }
  };
  auto build_b = [&](uint64_t i) {
    uint8_t* bh = sB + (i & 1) * 2 * bbytes;
    uint8_t* bl = bh + bbytes;
#pragma unroll
    for (int k = 0; k < kK4DirectItems; ++k) {
      if (k >= nitems) break;
      const int item = t + k * kK4DirectThreads;
      if (item >= N * 16) break;
      const int kb = item >> lgN, nn = item & (N - 1);
      uint32_t hw[4], lw[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const float2 x = L[k][q];
        const __nv_bfloat162 h = __floats2bfloat162_rn(x.x, x.y);
        const float2 hf = __bfloat1622float2(h);
        const __nv_bfloat162 l = __floats2bfloat162_rn(x.x - hf.x, x.y - hf.y);
        hw[q] = *reinterpret_cast<const uint32_t*>(&h);
        lw[q] = *reinterpret_cast<const uint32_t*>(&l);
      }
      const uint32_t off = tc::kmajor_off(uint32_t(nn), uint32_t(kb * 8), bk);
      *reinterpret_cast<uint4*>(bh + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
      *reinterpret_cast<uint4*>(bl + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
  };
  // TMEM accumulator of tile j -> global memory
  auto drain = [&](uint64_t j) -> bool {
    const int b = int(j & 1);
    const bool ok = tc::mbar_wait(&mbar[b], phase[b], kWaitLimit);
    if (__syncthreads_or(!ok)) return false;
    phase[b] ^= 1u;
    pend[b] = false;
    tc::tc_fence_after();
    // warp w reads TMEM lanes 32 (w % 4) ..; the four warps of a lane quadrant
    // split the columns
    const int quad = warp & 3, part_of_quad = warp >> 2;
    const int r = quad * 32 + lane;  // TMEM lane = D row = 2 p + c
    const int comp = r & 1;
    float2* base = sv + dep(tile_of(j), P.outer) + gp[r >> 1];
    const int per = N / 4 < 16 ? 16 : N / 4;
    const int c_begin = part_of_quad * per;
    const int c_end = c_begin + per < N ? c_begin + per : N;
    for (int c0 = c_begin; c0 + 16 <= c_end; c0 += 16) {
      float d[16];
      tc::tmem_ld16(tmem + uint32_t(b) * kK4DirectCols + (uint32_t(quad * 32) << 16) + uint32_t(c0), d);
      // pair re / im with the neighbouring lane: the even lane keeps columns
      // c0..c0+7, the odd lane c0+8..c0+15
      float o[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) o[k] = __shfl_xor_sync(0xffffffffu, comp ? d[k] : d[8 + k], 1);
      const int cb = c0 + (comp ? 8 : 0);
      if (pairs) {
#pragma unroll
        for (int k = 0; k < 8; k += 2) {
          const float4 v = comp ? make_float4(o[k], d[8 + k], o[k + 1], d[9 + k])
                                : make_float4(d[k], o[k], d[k + 1], o[k + 1]);
          __stcs(reinterpret_cast<float4*>(base + gn[cb + k]), v);
        }
      } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float2 v = comp ? make_float2(o[k], d[8 + k]) : make_float2(d[k], o[k]);
          __stcs(base + gn[cb + k], v);
        }
      }
    }
    tc::tc_fence_before();
    return true;
  };

  if (cnt > 0) load_tile(0);
  for (uint64_t i = 0; i < cnt; ++i) {
    build_b(i);  // B(i%2) was last read by the MMAs of tile i-2, drained before
    tc::fence_proxy_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    if (t == 0) {
      tc::tc_fence_after();
      const uint32_t a0 = tc::smem_u32(sA);
      const uint32_t bhs = tc::smem_u32(sB + (i & 1) * 2 * bbytes), bls = bhs + bbytes;
      const uint32_t d = tmem + uint32_t(i & 1) * kK4DirectCols;
      uint32_t acc = 0;
      for (int prod = 0; prod < nprod; ++prod) {
        const uint32_t abase = a0 + (prod == 2 ? uint32_t(kFusedABytes / 2) : 0u);
        const uint32_t bbase = prod == 1 ? bls : bhs;
        for (int s = 0; s < 8; ++s) {
          const uint64_t ad = tc::smem_desc(abase + uint32_t(s) * 2u * 2048u, 2048u, 128u);
          const uint64_t bd = tc::smem_desc(bbase + uint32_t(s) * 2u * bk, bk, 128u);
          tc::mma_bf16(d, ad, bd, idesc, acc);
          acc = 1;
        }
      }
      tc::mma_commit(&mbar[i & 1]);
    }
    pend[i & 1] = true;
    if (i + 1 < cnt) load_tile(i + 1);  // in flight while tile i multiplies and i-1 drains
    if (i > 0 && !drain(i - 1)) {
      failed = true;
      break;
    }
  }
  if (!failed && cnt > 0 && !drain(cnt - 1)) failed = true;
  if (failed) {
    if (t == 0) atomicExch(err, 1);
    for (int b = 0; b < 2; ++b)
      if (pend[b]) tc::mbar_wait(&mbar[b], phase[b], kWaitLimit);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 2 * kK4DirectCols);
}

// ---- K4, one unitary per pass, warp-specialised ---------------------------------
// Three roles run concurrently on one CTA per SM, handing tiles over through
// mbarriers instead of CTA-wide barriers:
//   warps 0-7   producers: load tile i from HBM into registers, split into
//               BF16 hi / lo, write B(i%2), arrive on bfull(i%2);
//   warp 16     one thread issues tile i's MMAs into TMEM accumulator i%2
//               and commits them to mdone(i%2);
//   warps 8-15  epilogue: wait mdone(i%2), move the accumulator from TMEM to
//               HBM, arrive on tfree(i%2).
// B(b) is rewritten only after mdone(b) of the tile two back, and
// accumulator b only after tfree(b) of the tile two back, so loads, MMAs and
// stores of three consecutive tiles overlap.  Every wait is bounded; a
// timeout sets the error flag and the shared abort word, and the other roles
// leave at their next wait.
constexpr int kWsProducers = 256;
constexpr int kWsThreads = 544;  // 8 producer warps, 8 epilogue warps, 1 MMA warp
constexpr int kWsItems = 8;      // B items per producer thread (N * 16 / 256, N <= 128)

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(kWsThreads, 1)
    k4_ws(float2* __restrict__ sv, const __grid_constant__ FusedPass P,
          const uint8_t* __restrict__ a_all, int* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m = P.m;
  const int N = 1 << (m - kFusedBits);
  const int lgN = m - kFusedBits;
  const uint32_t bk = uint32_t(N) * 16u;
  const uint32_t bbytes = uint32_t(N) * 256u;
  uint8_t* sA = sm;
  uint8_t* sB = sA + kFusedABytes;  // [2][hi|lo]
  uint64_t* gp = reinterpret_cast<uint64_t*>(sB + 4 * bbytes);
  uint64_t* gn = gp + 64;
  uint64_t* bfull = gn + N;   // [2]
  uint64_t* mdone = bfull + 2;  // [2]
  uint64_t* tfree = mdone + 2;  // [2]
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tfree + 2);
  uint32_t* tmem_base = reinterpret_cast<uint32_t*>(tfree + 3);

  {
    const uint4* src = reinterpret_cast<const uint4*>(a_all + size_t(P.part[0]) * kFusedABytes);
    uint4* dst = reinterpret_cast<uint4*>(sA);
    for (int i = t; i < kFusedABytes / 16; i += kWsThreads) dst[i] = src[i];
  }
  uint32_t pmask = 0;
  for (int b = 0; b < kFusedBits; ++b) pmask |= 1u << P.pbits[0][b];
  for (int p = t; p < 64; p += kWsThreads) {
    uint64_t x = 0;
    for (int b = 0; b < kFusedBits; ++b) x |= uint64_t((p >> b) & 1) << P.pbits[0][b];
    gp[p] = dep(x, P.tile);
  }
  for (int nn = t; nn < N; nn += kWsThreads) {
    uint64_t x = 0;
    int bit = 0;
    for (int b = 0; b < m; ++b)
      if (!((pmask >> b) & 1)) x |= uint64_t((nn >> bit++) & 1) << b;
    gn[nn] = dep(x, P.tile);
  }
  if (t == 0) {
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&bfull[b], kWsProducers);
      tc::mbar_init(&mdone[b], 1);
      tc::mbar_init(&tfree[b], kWsProducers);  // the epilogue has as many threads
    }
    *abort_flag = 0;
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_base, 2 * kK4DirectCols);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_base;
  const uint64_t cnt =
      blockIdx.x < P.ntiles ? (P.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto tile_of = [&](uint64_t i) { return blockIdx.x + i * gridDim.x; };
  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };

  if (warp < 8) {
    // ---- producers
    const int nitems = (N * 16) / kWsProducers;  // 1..8
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & 1);
      float2 L[kWsItems][4];
      const float2* base = sv + dep(tile_of(i), P.outer);
#pragma unroll
      for (int k = 0; k < kWsItems; ++k) {
        if (k >= nitems) break;
        const int item = t + k * kWsProducers;
        const int kb = item >> lgN, nn = item & (N - 1);
        const float2* col = base + gn[nn];
#pragma unroll
        for (int q = 0; q < 4; ++q) L[k][q] = __ldcs(col + gp[4 * kb + q]);
      }
      if (i >= 2 && !tc::mbar_wait(&mdone[b], uint32_t((i - 2) >> 1) & 1u, kWaitLimit)) {
        fail();
        break;
      }
      uint8_t* bh = sB + b * 2 * bbytes;
      uint8_t* bl = bh + bbytes;
#pragma unroll
      for (int k = 0; k < kWsItems; ++k) {
        if (k >= nitems) break;
        const int item = t + k * kWsProducers;
        const int kb = item >> lgN, nn = item & (N - 1);
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float2 x = L[k][q];
          const __nv_bfloat162 h = __floats2bfloat162_rn(x.x, x.y);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(x.x - hf.x, x.y - hf.y);
          hw[q] = *reinterpret_cast<const uint32_t*>(&h);
          lw[q] = *reinterpret_cast<const uint32_t*>(&l);
        }
        const uint32_t off = tc::kmajor_off(uint32_t(nn), uint32_t(kb * 8), bk);
        *reinterpret_cast<uint4*>(bh + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(bl + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
      }
      tc::fence_proxy_async_smem();  // the B writes become visible to the tensor cores
      mbar_arrive(&bfull[b]);
    }
  } else if (warp < 16) {
    // ---- epilogue: TMEM accumulator -> HBM
    const int quad = warp & 3, half = (warp - 8) >> 2;
    const int r = quad * 32 + lane;
    const int comp = r & 1;
    const bool pairs = (gn[1] == 1);
    const int per = N / 2 < 16 ? 16 : N / 2;
    const int c_begin = half * per;
    const int c_end = c_begin + per < N ? c_begin + per : N;
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & 1);
      if (!tc::mbar_wait(&mdone[b], uint32_t(i >> 1) & 1u, kWaitLimit)) {
        fail();
        break;
      }
      tc::tc_fence_after();
      float2* base = sv + dep(tile_of(i), P.outer) + gp[r >> 1];
      for (int c0 = c_begin; c0 + 16 <= c_end; c0 += 16) {
        float d[16];
        tc::tmem_ld16(tmem + uint32_t(b) * kK4DirectCols + (uint32_t(quad * 32) << 16) + uint32_t(c0), d);
        float o[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) o[k] = __shfl_xor_sync(0xffffffffu, comp ? d[k] : d[8 + k], 1);
        const int cb = c0 + (comp ? 8 : 0);
        if (pairs) {
#pragma unroll
          for (int k = 0; k < 8; k += 2) {
            const float4 v = comp ? make_float4(o[k], d[8 + k], o[k + 1], d[9 + k])
                                  : make_float4(d[k], o[k], d[k + 1], o[k + 1]);
            __stcs(reinterpret_cast<float4*>(base + gn[cb + k]), v);
          }
        } else {
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            const float2 v = comp ? make_float2(o[k], d[8 + k]) : make_float2(d[k], o[k]);
            __stcs(base + gn[cb + k], v);
          }
        }
      }
      tc::tc_fence_before();
      mbar_arrive(&tfree[b]);
    }
  } else if (lane == 0) {
    // ---- MMA issue
    const uint32_t idesc = tc::idesc_bf16_f32(128, uint32_t(N));
    const int nprod = P.precision == 1 ? 1 : 3;
    const uint32_t a0 = tc::smem_u32(sA);
    uint64_t issued = 0;
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & 1);
      if (!tc::mbar_wait(&bfull[b], uint32_t(i >> 1) & 1u, kWaitLimit) ||
          (i >= 2 && !tc::mbar_wait(&tfree[b], uint32_t((i - 2) >> 1) & 1u, kWaitLimit))) {
        fail();
        break;
      }
      tc::tc_fence_after();
      const uint32_t bhs = tc::smem_u32(sB + b * 2 * bbytes), bls = bhs + bbytes;
      const uint32_t d = tmem + uint32_t(b) * kK4DirectCols;
      uint32_t acc = 0;
      for (int prod = 0; prod < nprod; ++prod) {
        const uint32_t abase = a0 + (prod == 2 ? uint32_t(kFusedABytes / 2) : 0u);
        const uint32_t bbase = prod == 1 ? bls : bhs;
        for (int s = 0; s < 8; ++s) {
          const uint64_t ad = tc::smem_desc(abase + uint32_t(s) * 2u * 2048u, 2048u, 128u);
          const uint64_t bd = tc::smem_desc(bbase + uint32_t(s) * 2u * bk, bk, 128u);
          tc::mma_bf16(d, ad, bd, idesc, acc);
          acc = 1;
        }
      }
      tc::mma_commit(&mdone[b]);
      issued = i + 1;
    }
    // the last committed MMAs complete before TMEM is released
    if (issued > 0) {
      const uint64_t j = issued - 1;
      tc::mbar_wait(&mdone[j & 1], uint32_t(j >> 1) & 1u, kWaitLimit);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 2 * kK4DirectCols);
}

// ---- K4, one unitary per pass, bulk-loaded ----------------------------------------
// The warp-specialised pipeline with a fourth role: a loader warp brings
// whole tiles into shared memory with bulk copies (cp.async.bulk, completing
// on an mbarrier with a byte count), so the HBM reads in flight are not
// bounded by the producers' registers or per-thread load slots.  A raw
// complex64 tile and its BF16 hi / lo B operand have the same size, so each
// of the four buffers holds tile i first raw, then as B:
//   warp 17     loader: for tile i, once the MMAs of tile i-NB have read
//               buffer i%NB (bfree), arm rfull(i%NB) with the tile's byte count
//               and copy the tile's contiguous runs (the lowest run of tile
//               bits, slots 0..L0-1) in tile-index order;
//   warps 0-7   producers: wait rfull(i%NB), read their raw amplitudes into
//               registers, meet at a named barrier (every raw read precedes
//               every B write), write the BF16 hi / lo rows, arrive on
//               bfull(i%NB);
//   warp 16     MMA issue (commits to mdone(i%2) and bfree(i%NB));
//   warps 8-15  epilogue: TMEM -> registers -> a per-warp shared-memory
//               transpose -> 16-byte stores, each lane writing two amplitudes
//               that are adjacent in memory, the lanes of a store covering
//               contiguous runs.
// With tiles of 2^12 amplitudes the ring has four buffers (three tiles in
// flight while one is converted); tiles of 2^13 (contiguous runs twice as
// long) fit two.
constexpr int kBulkThreads = 576;  // 8 producer, 8 epilogue, 1 MMA, 1 loader warps
constexpr int kBulkItems = 8;      // B items per producer thread (N * 16 / 256, N <= 128)
constexpr int kBulkBuffers = 4;    // ring buffers at most (2^(lgb) used)
constexpr int kBulkMaxChunkBits = 9;  // bulk copies of at most 2^9 amplitudes (4 KiB)
constexpr int kBulkStageFloats = 512;  // per epilogue warp: 16 p x 16 columns x (re, im)

__global__ void __launch_bounds__(kBulkThreads, 1)
    k4_bulk(float2* __restrict__ sv, const __grid_constant__ FusedPass P,
            const uint8_t* __restrict__ a_all, int* __restrict__ err, int chunk_bits, int lgb) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m = P.m, T = 1 << m;
  const int N = 1 << (m - kFusedBits);
  const int lgN = m - kFusedBits;
  const uint32_t bk = uint32_t(N) * 16u;
  const uint32_t bbytes = uint32_t(N) * 256u;
  const int nchunks = T >> chunk_bits;
  const uint32_t chunk_bytes = 8u << chunk_bits;
  const uint64_t bmask = (1u << lgb) - 1u;  // ring buffer of tile i: i & bmask
  uint8_t* sA = sm;
  uint8_t* sB = sA + kFusedABytes;  // [kBulkBuffers][T * 8 bytes]: raw tile, then hi | lo
  uint64_t* gp = reinterpret_cast<uint64_t*>(sB + (size_t(T) * 8 << lgb));
  uint64_t* gn = gp + 64;
  uint64_t* gc = gn + N;                                     // global offset of chunk c
  uint32_t* tq = reinterpret_cast<uint32_t*>(gc + nchunks);  // tile index of part index p
  uint32_t* tn = tq + 64;                                    // tile index of column n
  uint64_t* bars = reinterpret_cast<uint64_t*>(tn + N);
  uint64_t* rfull = bars;                  // [kBulkBuffers]
  uint64_t* bfull = rfull + kBulkBuffers;  // [kBulkBuffers]
  uint64_t* bfree = bfull + kBulkBuffers;  // [kBulkBuffers]
  uint64_t* mdone = bfree + kBulkBuffers;  // [2]
  uint64_t* tfree = mdone + 2;             // [2]
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tfree + 2);
  uint32_t* tmem_base = reinterpret_cast<uint32_t*>(tfree + 3);
  float* stage = reinterpret_cast<float*>(tfree + 4);  // [8 warps][kBulkStageFloats]

  {
    const uint4* src = reinterpret_cast<const uint4*>(a_all + size_t(P.part[0]) * kFusedABytes);
    uint4* dst = reinterpret_cast<uint4*>(sA);
    for (int i = t; i < kFusedABytes / 16; i += kBulkThreads) dst[i] = src[i];
  }
  uint32_t pmask = 0;
  for (int b = 0; b < kFusedBits; ++b) pmask |= 1u << P.pbits[0][b];
  for (int p = t; p < 64; p += kBulkThreads) {
    uint32_t x = 0;
    for (int b = 0; b < kFusedBits; ++b) x |= uint32_t((p >> b) & 1) << P.pbits[0][b];
    tq[p] = x;
    gp[p] = dep(x, P.tile);
  }
  for (int nn = t; nn < N; nn += kBulkThreads) {
    uint32_t x = 0;
    int bit = 0;
    for (int b = 0; b < m; ++b)
      if (!((pmask >> b) & 1)) x |= uint32_t((nn >> bit++) & 1) << b;
    tn[nn] = x;
    gn[nn] = dep(x, P.tile);
  }
  for (int c = t; c < nchunks; c += kBulkThreads) gc[c] = dep(uint64_t(c) << chunk_bits, P.tile);
  if (t == 0) {
    for (int b = 0; b < kBulkBuffers; ++b) {
      tc::mbar_init(&rfull[b], 1);
      tc::mbar_init(&bfull[b], kWsProducers);
      tc::mbar_init(&bfree[b], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&mdone[b], 1);
      tc::mbar_init(&tfree[b], kWsProducers);  // the epilogue has as many threads
    }
    *abort_flag = 0;
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_base, 2 * kK4DirectCols);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_base;
  const uint64_t cnt =
      blockIdx.x < P.ntiles ? (P.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto tile_of = [&](uint64_t i) { return blockIdx.x + i * gridDim.x; };
  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };

  if (warp == 17) {
    // ---- loader
    uint64_t issued = 0;
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & bmask);
      if ((i >> lgb) > 0 && !tc::mbar_wait(&bfree[b], uint32_t((i >> lgb) - 1) & 1u, kWaitLimit)) {
        fail();
        break;
      }
      if (lane == 0) tc::mbar_arrive_expect_tx(&rfull[b], uint32_t(T) * 8u);
      __syncwarp();
      const float2* base = sv + dep(tile_of(i), P.outer);
      const uint32_t dst = tc::smem_u32(sB + size_t(b) * T * 8);
      const uint64_t tb0 = dep(tile_of(i), P.outer);
      for (int c = lane; c < nchunks; c += 32)
        if (HS_IN_BOUNDS(tb0 + gc[c] + (chunk_bytes >> 3) <= (1ull << P.n) &&
                             uint64_t(c + 1) * chunk_bytes <= uint64_t(T) * 8u,
                         kBoundsK4))
          tc::bulk_load(dst + uint32_t(c) * chunk_bytes, base + gc[c], chunk_bytes, &rfull[b]);
      issued = i + 1;
    }
    // no copy may still be landing when the CTA leaves: wait for the last
    // tile of each buffer (its phase is that buffer's latest)
    for (uint64_t j = issued > bmask + 1 ? issued - bmask - 1 : 0; j < issued; ++j)
      tc::mbar_wait(&rfull[j & bmask], uint32_t(j >> lgb) & 1u, kWaitLimit);
  } else if (warp < 8) {
    // ---- producers: item k is amplitudes p = 4kb..4kb+3 of column nn
    const int nitems = (N * 16) / kWsProducers;  // 1..8
    for (uint64_t i = 0; i < cnt; ++i) {
      const int b = int(i & bmask);
      const bool ok =
          !*abort_flag && tc::mbar_wait(&rfull[b], uint32_t(i >> lgb) & 1u, kWaitLimit);
      if (!ok) fail();
      uint8_t* buf = sB + size_t(b) * T * 8;
      float2 x[kBulkItems][4];
#pragma unroll
      for (int k = 0; k < kBulkItems; ++k) {
        if (k >= nitems) break;
        const int item = t + k * kWsProducers;
        const int kb = item >> lgN, nn = item & (N - 1);
        const uint32_t tcol = tn[nn];
        const uint4 tp = *reinterpret_cast<const uint4*>(tq + 4 * kb);  // p = 4kb..4kb+3
        if (!HS_IN_BOUNDS(((tp.x | tp.y | tp.z | tp.w) | tcol) < uint32_t(T), kBoundsK4)) continue;
        x[k][0] = *reinterpret_cast<const float2*>(buf + size_t(tp.x | tcol) * 8);
        x[k][1] = *reinterpret_cast<const float2*>(buf + size_t(tp.y | tcol) * 8);
        x[k][2] = *reinterpret_cast<const float2*>(buf + size_t(tp.z | tcol) * 8);
        x[k][3] = *reinterpret_cast<const float2*>(buf + size_t(tp.w | tcol) * 8);
      }
      // every raw read precedes every B write; the producers leave together
      // (a vote at the same named barrier) when any of them saw a timeout or
      // the abort word
      uint32_t stop;
      asm volatile(
          "{\n .reg .pred p, q;\n setp.eq.u32 p, %1, 0;\n"
          " bar.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
          : "=r"(stop)
          : "r"(uint32_t(ok)), "n"(kWsProducers)
          : "memory");
      if (stop) break;
      uint8_t* bl = buf + bbytes;
#pragma unroll
      for (int k = 0; k < kBulkItems; ++k) {
        if (k >= nitems) break;
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(x[k][q].x, x[k][q].y);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(x[k][q].x - hf.x, x[k][q].y - hf.y);
          hw[q] = *reinterpret_cast<const uint32_t*>(&h);
          lw[q] = *reinterpret_cast<const uint32_t*>(&l);
        }
        const int item = t + k * kWsProducers;
        const uint32_t boff = tc::kmajor_off(uint32_t(item & (N - 1)), uint32_t((item >> lgN) * 8), bk);
        *reinterpret_cast<uint4*>(buf + boff) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(bl + boff) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
      }
      tc::fence_proxy_async_smem();  // the B writes become visible to the tensor cores
      mbar_arrive(&bfull[b]);
    }
  } else if (warp < 16) {
    // ---- epilogue: TMEM accumulator -> shared-memory transpose -> HBM.
    // Thread (quad, lane) holds real-form row r = 32 quad + lane, i.e. the
    // re (lane even) or im part of part index p = 16 quad + lane / 2.  Per
    // chunk of 16 columns the warp writes its 16 p x 16 columns x (re, im)
    // to its staging block (column pairs XOR-swizzled by p, so the writes
    // spread over the banks and a column pair stays one 16-byte slot), then
    // stores two memory-adjacent amplitudes per lane: (p; c, c+1) when
    // column bit 0 is slot 0, else (p, p+1; c) (part bit 0 is slot 0).
    const int quad = warp & 3, half = (warp - 8) >> 2;
    const int comp = lane & 1, pl = lane >> 1;
    const bool pairs = (gn[1] == 1);
    const int per = N / 2 < 16 ? 16 : N / 2;
    const int c_begin = half * per;
    const int c_end = c_begin + per < N ? c_begin + per : N;
    float* stg = stage + (warp - 8) * kBulkStageFloats;
    // column c of part row p sits at word 2 (c ^ f(p)), f(p) = 2 (p mod 8) +
    // (p div 8): the 16 rows x (re, im) of one column hit 32 distinct banks;
    // a column pair (c, c + 1), c even, stays one 16-byte slot (spair), in
    // reversed order for rows p >= 8 (odd f)
    auto fsw = [](int p) { return ((p & 7) << 1) | ((p >> 3) & 1); };
    auto sidx = [&](int p, int c) { return p * 32 + ((c ^ fsw(p)) << 1); };
    auto spair = [&](int p, int c) { return p * 32 + (((c ^ fsw(p)) & ~1) << 1); };
    const uint64_t* gpq = gp + quad * 16;
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & 1);
      if (!tc::mbar_wait(&mdone[b], uint32_t(i >> 1) & 1u, kWaitLimit)) {
        fail();
        break;
      }
      tc::tc_fence_after();
      float2* tb = sv + dep(tile_of(i), P.outer);
      for (int c0 = c_begin; c0 + 16 <= c_end; c0 += 16) {
        float d[16];
        tc::tmem_ld16(tmem + uint32_t(b) * kK4DirectCols + (uint32_t(quad * 32) << 16) + uint32_t(c0), d);
        __syncwarp();  // the previous chunk's staging reads are done
#pragma unroll
        for (int c = 0; c < 16; ++c) stg[sidx(pl, c) + comp] = d[c];
        __syncwarp();
        if (pairs) {
#pragma unroll
          for (int s4 = 0; s4 < 4; ++s4) {
            const int p = (lane >> 3) + 4 * s4, c = 2 * (lane & 7);
            float4 v = *reinterpret_cast<const float4*>(stg + spair(p, c));
            if (s4 >= 2) v = make_float4(v.z, v.w, v.x, v.y);  // p >= 8
            if (HS_IN_BOUNDS(uint64_t(tb - sv) + gpq[p] + gn[c0 + c] + 2 <= (1ull << P.n), kBoundsK4))
              __stcs(reinterpret_cast<float4*>(tb + gpq[p] + gn[c0 + c]), v);
          }
        } else {
#pragma unroll
          for (int s4 = 0; s4 < 4; ++s4) {
            const int p = 2 * ((lane >> 4) + 2 * s4), c = lane & 15;
            const float2 lo = *reinterpret_cast<const float2*>(stg + sidx(p, c));
            const float2 hi = *reinterpret_cast<const float2*>(stg + sidx(p + 1, c));
            if (HS_IN_BOUNDS(uint64_t(tb - sv) + gpq[p] + gn[c0 + c] + 2 <= (1ull << P.n), kBoundsK4))
              __stcs(reinterpret_cast<float4*>(tb + gpq[p] + gn[c0 + c]),
                     make_float4(lo.x, lo.y, hi.x, hi.y));
          }
        }
      }
      tc::tc_fence_before();
      mbar_arrive(&tfree[b]);
    }
  } else if (warp == 16 && lane == 0) {
    // ---- MMA issue
    const uint32_t idesc = tc::idesc_bf16_f32(128, uint32_t(N));
    const int nprod = P.precision == 1 ? 1 : 3;
    const uint32_t a0 = tc::smem_u32(sA);
    uint64_t issued = 0;
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & 1);
      const int bb = int(i & bmask);
      if (!tc::mbar_wait(&bfull[bb], uint32_t(i >> lgb) & 1u, kWaitLimit) ||
          (i >= 2 && !tc::mbar_wait(&tfree[b], uint32_t((i - 2) >> 1) & 1u, kWaitLimit))) {
        fail();
        break;
      }
      tc::tc_fence_after();
      const uint32_t bhs = tc::smem_u32(sB + size_t(bb) * T * 8), bls = bhs + bbytes;
      const uint32_t d = tmem + uint32_t(b) * kK4DirectCols;
      uint32_t acc = 0;
      for (int prod = 0; prod < nprod; ++prod) {
        const uint32_t abase = a0 + (prod == 2 ? uint32_t(kFusedABytes / 2) : 0u);
        const uint32_t bbase = prod == 1 ? bls : bhs;
        for (int s = 0; s < 8; ++s) {
          const uint64_t ad = tc::smem_desc(abase + uint32_t(s) * 2u * 2048u, 2048u, 128u);
          const uint64_t bd = tc::smem_desc(bbase + uint32_t(s) * 2u * bk, bk, 128u);
          tc::mma_bf16(d, ad, bd, idesc, acc);
          acc = 1;
        }
      }
      tc::mma_commit(&mdone[b]);
      tc::mma_commit(&bfree[bb]);  // buffer bb may take tile i + NB
      issued = i + 1;
    }
    // the last committed MMAs complete before TMEM is released
    if (issued > 0) {
      const uint64_t j = issued - 1;
      tc::mbar_wait(&mdone[j & 1], uint32_t(j >> 1) & 1u, kWaitLimit);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 2 * kK4DirectCols);
}

// ---- K4, two unitaries per pass, bulk-loaded --------------------------------------
// The bulk-loaded pipeline applied twice to each tile before it leaves the
// SM: the first product's accumulator goes back into the tile's shared
// buffer as complex64 (in tile-index order, like the loaded tile), is split
// again into the BF16 operand of the second unitary (whose six bits are
// other tile bits) and only the second product is stored to HBM.  Tiles of
// 2^12 amplitudes; both 128 x 128 real-form operands A1, A2 stay in shared
// memory; two ring buffers; four TMEM accumulators (stage x tile parity).
// Each role runs its steps in a skewed order, every step waiting only on
// earlier steps of the other roles:
//   loader      L(i)  waits bfree(i-2)  (the second MMA of tile i-2 read its buffer)
//   producers   P1(i) waits rfull(i);   P2(i-1) waits rmid(i-1)
//   MMA         M1(i) waits bfull1(i), tfree1(i-2);  M2(i-1) waits bfull2(i-1), tfree2(i-3)
//   epilogue    MID(i) waits mdone1(i) and writes the buffer (rmid);
//               FIN(i-1) waits mdone2(i-1) and stores to HBM
// Every wait is bounded; a timeout sets the error flag and the abort word.
constexpr int kBulk2Threads = 576;     // 8 producer, 8 epilogue, 1 MMA, 1 loader warps
constexpr int kBulk2MaxTileBits = 12;  // N <= 64 columns
constexpr int kBulk2Items = 4;         // B items per producer thread (N * 16 / 256)

__global__ void __launch_bounds__(kBulk2Threads, 1)
    k4_bulk2(float2* __restrict__ sv, const __grid_constant__ FusedPass P,
             const uint8_t* __restrict__ a_all, int* __restrict__ err, int chunk_bits) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int m = P.m, T = 1 << m;
  const int N = 1 << (m - kFusedBits);
  const int lgN = m - kFusedBits;
  const uint32_t bk = uint32_t(N) * 16u;
  const uint32_t bbytes = uint32_t(N) * 256u;
  const int nchunks = T >> chunk_bits;
  const uint32_t chunk_bytes = 8u << chunk_bits;
  uint8_t* sA = sm;                       // [2][kFusedABytes]
  uint8_t* sB = sA + 2 * kFusedABytes;    // [2][T * 8]: raw tile / B operand
  uint64_t* gc = reinterpret_cast<uint64_t*>(sB + size_t(T) * 16);  // global offset of chunk c
  uint64_t* gp2 = gc + nchunks;           // global offset of stage-2 part index p
  uint64_t* gn2 = gp2 + 64;               // global offset of stage-2 column n
  uint32_t* tq = reinterpret_cast<uint32_t*>(gn2 + N);  // [2][64]: tile index of part index p
  uint32_t* tn = tq + 128;                // [2][N]: tile index of column n
  uint64_t* bars = reinterpret_cast<uint64_t*>(tn + 2 * N + (N & 1));
  uint64_t* rfull = bars;        // [2] loader -> producers
  uint64_t* bfull1 = bars + 2;   // [2] producers (stage 1) -> MMA
  uint64_t* rmid = bars + 4;     // [2] epilogue (stage 1 result in the buffer) -> producers
  uint64_t* bfull2 = bars + 6;   // [2] producers (stage 2) -> MMA
  uint64_t* bfree = bars + 8;    // [2] MMA (stage 2 read the buffer) -> loader
  uint64_t* mdone = bars + 10;   // [2 stages][2] MMA -> epilogue
  uint64_t* tfree = bars + 14;   // [2 stages][2] epilogue -> MMA
  volatile int* abort_flag = reinterpret_cast<volatile int*>(bars + 18);
  uint32_t* tmem_base = reinterpret_cast<uint32_t*>(bars + 19);
  float* stage = reinterpret_cast<float*>(bars + 20);  // [8 warps][kBulkStageFloats]

  for (int s2 = 0; s2 < 2; ++s2) {
    const uint4* src = reinterpret_cast<const uint4*>(a_all + size_t(P.part[s2]) * kFusedABytes);
    uint4* dst = reinterpret_cast<uint4*>(sA + size_t(s2) * kFusedABytes);
    for (int i = t; i < kFusedABytes / 16; i += kBulk2Threads) dst[i] = src[i];
  }
  for (int s2 = 0; s2 < 2; ++s2) {
    uint32_t pmask = 0;
    for (int b = 0; b < kFusedBits; ++b) pmask |= 1u << P.pbits[s2][b];
    for (int p = t; p < 64; p += kBulk2Threads) {
      uint32_t x = 0;
      for (int b = 0; b < kFusedBits; ++b) x |= uint32_t((p >> b) & 1) << P.pbits[s2][b];
      tq[s2 * 64 + p] = x;
      if (s2 == 1) gp2[p] = dep(x, P.tile);
    }
    for (int nn = t; nn < N; nn += kBulk2Threads) {
      uint32_t x = 0;
      int bit = 0;
      for (int b = 0; b < m; ++b)
        if (!((pmask >> b) & 1)) x |= uint32_t((nn >> bit++) & 1) << b;
      tn[s2 * N + nn] = x;
      if (s2 == 1) gn2[nn] = dep(x, P.tile);
    }
  }
  for (int c = t; c < nchunks; c += kBulk2Threads) gc[c] = dep(uint64_t(c) << chunk_bits, P.tile);
  if (t == 0) {
    for (int b = 0; b < 2; ++b) {
      // short runs: one cp.async arrival per loader lane; long runs: one
      // arrival with the tile's byte count
      tc::mbar_init(&rfull[b], (8u << chunk_bits) < 1024u ? 32 : 1);
      tc::mbar_init(&bfull1[b], kWsProducers);
      tc::mbar_init(&rmid[b], kWsProducers);  // the epilogue has as many threads
      tc::mbar_init(&bfull2[b], kWsProducers);
      tc::mbar_init(&bfree[b], 1);
    }
    for (int b = 0; b < 4; ++b) {
      tc::mbar_init(&mdone[b], 1);
      tc::mbar_init(&tfree[b], kWsProducers);
    }
    *abort_flag = 0;
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_base, 4 * 64);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_base;
  // accumulator of stage s (0, 1) for tile parity b
  auto acc = [&](int s, int b) { return tmem + uint32_t(2 * s + b) * 64u; };
  const uint64_t cnt =
      blockIdx.x < P.ntiles ? (P.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto tile_of = [&](uint64_t i) { return blockIdx.x + i * gridDim.x; };
  auto fail = [&]() {
    *abort_flag = 1;
    atomicExch(err, 1);
  };
  auto ph = [](uint64_t i) { return uint32_t(i >> 1) & 1u; };  // phase parity of tile i's barriers

  if (warp == 17) {
    // ---- loader: runs of 1 KiB or more as bulk copies (complete_tx on
    // rfull); shorter runs as 16-byte cp.async copies, each lane's completing
    // on rfull through cp.async.mbarrier.arrive (rfull then counts the lanes)
    const bool small = chunk_bytes < 1024u;
    uint64_t issued = 0;
    for (uint64_t i = 0; i < cnt && !*abort_flag; ++i) {
      const int b = int(i & 1);
      if (i >= 2 && !tc::mbar_wait(&bfree[b], ph(i - 2), kWaitLimit)) {
        fail();
        break;
      }
      const float2* base = sv + dep(tile_of(i), P.outer);
      const uint32_t dst = tc::smem_u32(sB + size_t(b) * T * 8);
      if (small) {
        const int per_chunk = int(chunk_bytes >> 4);  // 16-byte pieces per run
        for (int u = lane; u < (T >> 1); u += 32) {
          const int c = u / per_chunk, w = u - c * per_chunk;
          if (HS_IN_BOUNDS(dep(tile_of(i), P.outer) + gc[c] + 2 * w + 2 <= (1ull << P.n),
                           kBoundsK4))
            cp_async16(dst + uint32_t(u) * 16u, base + gc[c] + 2 * w);
        }
        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(
                         tc::smem_u32(&rfull[b]))
                     : "memory");
      } else {
        if (lane == 0) tc::mbar_arrive_expect_tx(&rfull[b], uint32_t(T) * 8u);
        __syncwarp();
        const uint64_t tb0 = dep(tile_of(i), P.outer);
        for (int c = lane; c < nchunks; c += 32)
          if (HS_IN_BOUNDS(tb0 + gc[c] + (chunk_bytes >> 3) <= (1ull << P.n) &&
                               uint64_t(c + 1) * chunk_bytes <= uint64_t(T) * 8u,
                           kBoundsK4))
            tc::bulk_load(dst + uint32_t(c) * chunk_bytes, base + gc[c], chunk_bytes, &rfull[b]);
      }
      issued = i + 1;
    }
    for (uint64_t j = issued > 2 ? issued - 2 : 0; j < issued; ++j)
      tc::mbar_wait(&rfull[j & 1], ph(j), kWaitLimit);
    if (small) cp_async_wait0();
  } else if (warp < 8) {
    // ---- producers: stage s of tile i reads the raw tile (s = 0: as loaded,
    // s = 1: the first product) and writes stage s's BF16 hi / lo operand
    const int nitems = (N * 16) / kWsProducers;  // 1..4
    auto produce = [&](int s2, uint64_t i) -> bool {
      const int b = int(i & 1);
      uint64_t* wait_bar = s2 == 0 ? &rfull[b] : &rmid[b];
      const bool ok = !*abort_flag && tc::mbar_wait(wait_bar, ph(i), kWaitLimit);
      if (!ok) fail();
      uint8_t* buf = sB + size_t(b) * T * 8;
      const uint32_t* tqs = tq + s2 * 64;
      const uint32_t* tns = tn + s2 * N;
      float2 x[kBulk2Items][4];
#pragma unroll
      for (int k = 0; k < kBulk2Items; ++k) {
        if (k >= nitems) break;
        const int item = t + k * kWsProducers;
        const int kb = item >> lgN, nn = item & (N - 1);
        const uint32_t tcol = tns[nn];
        const uint4 tp = *reinterpret_cast<const uint4*>(tqs + 4 * kb);
        if (!HS_IN_BOUNDS(((tp.x | tp.y | tp.z | tp.w) | tcol) < uint32_t(T), kBoundsK4)) continue;
        x[k][0] = *reinterpret_cast<const float2*>(buf + size_t(tp.x | tcol) * 8);
        x[k][1] = *reinterpret_cast<const float2*>(buf + size_t(tp.y | tcol) * 8);
        x[k][2] = *reinterpret_cast<const float2*>(buf + size_t(tp.z | tcol) * 8);
        x[k][3] = *reinterpret_cast<const float2*>(buf + size_t(tp.w | tcol) * 8);
      }
      uint32_t stop;
      asm volatile(
          "{\n .reg .pred p, q;\n setp.eq.u32 p, %1, 0;\n"
          " bar.red.or.pred q, 1, %2, p;\n selp.u32 %0, 1, 0, q;\n}\n"
          : "=r"(stop)
          : "r"(uint32_t(ok)), "n"(kWsProducers)
          : "memory");
      if (stop) return false;
      uint8_t* bl = buf + bbytes;
#pragma unroll
      for (int k = 0; k < kBulk2Items; ++k) {
        if (k >= nitems) break;
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const __nv_bfloat162 h = __floats2bfloat162_rn(x[k][q].x, x[k][q].y);
          const float2 hf = __bfloat1622float2(h);
          const __nv_bfloat162 l = __floats2bfloat162_rn(x[k][q].x - hf.x, x[k][q].y - hf.y);
          hw[q] = *reinterpret_cast<const uint32_t*>(&h);
          lw[q] = *reinterpret_cast<const uint32_t*>(&l);
        }
        const int item = t + k * kWsProducers;
        const uint32_t boff = tc::kmajor_off(uint32_t(item & (N - 1)), uint32_t((item >> lgN) * 8), bk);
        *reinterpret_cast<uint4*>(buf + boff) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(bl + boff) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
      }
      tc::fence_proxy_async_smem();
      mbar_arrive(s2 == 0 ? &bfull1[b] : &bfull2[b]);
      return true;
    };
    bool go = true;
    for (uint64_t i = 0; i < cnt && go; ++i) {
      go = produce(0, i);
      if (go && i >= 1) go = produce(1, i - 1);
    }
    if (go && cnt > 0) produce(1, cnt - 1);
  } else if (warp < 16) {
    // ---- epilogue: stage 0's accumulator back into the tile buffer (in tile
    // index order), stage 1's to HBM; both through the per-warp staging
    // transpose of k4_bulk (two memory-adjacent amplitudes per lane)
    const int quad = warp & 3, half = (warp - 8) >> 2;
    const int comp = lane & 1, pl = lane >> 1;
    const int per = N / 2 < 16 ? 16 : N / 2;
    const int c_begin = half * per;
    const int c_end = c_begin + per < N ? c_begin + per : N;
    float* stg = stage + (warp - 8) * kBulkStageFloats;
    // column c of part row p sits at word 2 (c ^ f(p)), f(p) = 2 (p mod 8) +
    // (p div 8): the 16 rows x (re, im) of one column hit 32 distinct banks;
    // a column pair (c, c + 1), c even, stays one 16-byte slot (spair), in
    // reversed order for rows p >= 8 (odd f)
    auto fsw = [](int p) { return ((p & 7) << 1) | ((p >> 3) & 1); };
    auto sidx = [&](int p, int c) { return p * 32 + ((c ^ fsw(p)) << 1); };
    auto spair = [&](int p, int c) { return p * 32 + (((c ^ fsw(p)) & ~1) << 1); };
    auto drain = [&](int s2, uint64_t i) -> bool {
      const int b = int(i & 1);
      if (!tc::mbar_wait(&mdone[2 * s2 + b], ph(i), kWaitLimit)) {
        fail();
        return false;
      }
      tc::tc_fence_after();
      // destination of amplitude (p, c): global offset (stage 1) or the tile
      // index in the buffer (stage 0)
      const bool to_smem = s2 == 0;
      const uint32_t* tqs = tq + quad * 16;            // stage 0 rows
      const uint32_t* tns = tn;                        // stage 0 columns
      const uint64_t* gpq = gp2 + quad * 16;           // stage 1 rows
      const bool pairs = to_smem ? (tn[1] == 1) : (gn2[1] == 1);
      float2* tb = sv + dep(tile_of(i), P.outer);
      float2* sbuf = reinterpret_cast<float2*>(sB + size_t(b) * T * 8);
      for (int c0 = c_begin; c0 + 16 <= c_end; c0 += 16) {
        float d[16];
        tc::tmem_ld16(acc(s2, b) + (uint32_t(quad * 32) << 16) + uint32_t(c0), d);
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 16; ++c) stg[sidx(pl, c) + comp] = d[c];
        __syncwarp();
#pragma unroll
        for (int s4 = 0; s4 < 4; ++s4) {
          int p, c;
          float4 v;
          if (pairs) {
            p = (lane >> 3) + 4 * s4;
            c = 2 * (lane & 7);
            v = *reinterpret_cast<const float4*>(stg + spair(p, c));
            if (s4 >= 2) v = make_float4(v.z, v.w, v.x, v.y);  // p >= 8
          } else {
            p = 2 * ((lane >> 4) + 2 * s4);
            c = lane & 15;
            const float2 lo = *reinterpret_cast<const float2*>(stg + sidx(p, c));
            const float2 hi = *reinterpret_cast<const float2*>(stg + sidx(p + 1, c));
            v = make_float4(lo.x, lo.y, hi.x, hi.y);
          }
          if (to_smem) {
            if (HS_IN_BOUNDS((tqs[p] | tns[c0 + c]) + 2u <= uint32_t(T), kBoundsK4))
              *reinterpret_cast<float4*>(sbuf + (tqs[p] | tns[c0 + c])) = v;
          } else if (HS_IN_BOUNDS(uint64_t(tb - sv) + gpq[p] + gn2[c0 + c] + 2 <= (1ull << P.n),
                                  kBoundsK4)) {
            __stcs(reinterpret_cast<float4*>(tb + gpq[p] + gn2[c0 + c]), v);
          }
        }
      }
      tc::tc_fence_before();
      mbar_arrive(&tfree[2 * s2 + b]);
      if (to_smem) mbar_arrive(&rmid[b]);  // release: the buffer writes precede it
      return true;
    };
    bool go = true;
    for (uint64_t i = 0; i < cnt && go && !*abort_flag; ++i) {
      go = drain(0, i);
      if (go && i >= 1) go = drain(1, i - 1);
    }
    if (go && cnt > 0 && !*abort_flag) drain(1, cnt - 1);
  } else if (warp == 16 && lane == 0) {
    // ---- MMA issue
    const uint32_t idesc = tc::idesc_bf16_f32(128, uint32_t(N));
    const int nprod = P.precision == 1 ? 1 : 3;
    uint64_t last2 = 0;
    bool any2 = false;
    auto issue = [&](int s2, uint64_t i) -> bool {
      const int b = int(i & 1);
      uint64_t* full = s2 == 0 ? &bfull1[b] : &bfull2[b];
      if (!tc::mbar_wait(full, ph(i), kWaitLimit) ||
          (i >= 2 && !tc::mbar_wait(&tfree[2 * s2 + b], ph(i - 2), kWaitLimit))) {
        fail();
        return false;
      }
      tc::tc_fence_after();
      const uint32_t a0 = tc::smem_u32(sA + size_t(s2) * kFusedABytes);
      const uint32_t bhs = tc::smem_u32(sB + size_t(b) * T * 8), bls = bhs + bbytes;
      const uint32_t d = acc(s2, b);
      uint32_t accum = 0;
      for (int prod = 0; prod < nprod; ++prod) {
        const uint32_t abase = a0 + (prod == 2 ? uint32_t(kFusedABytes / 2) : 0u);
        const uint32_t bbase = prod == 1 ? bls : bhs;
        for (int k = 0; k < 8; ++k) {
          const uint64_t ad = tc::smem_desc(abase + uint32_t(k) * 2u * 2048u, 2048u, 128u);
          const uint64_t bd = tc::smem_desc(bbase + uint32_t(k) * 2u * bk, bk, 128u);
          tc::mma_bf16(d, ad, bd, idesc, accum);
          accum = 1;
        }
      }
      tc::mma_commit(&mdone[2 * s2 + b]);
      if (s2 == 1) {
        tc::mma_commit(&bfree[b]);  // buffer b may take tile i + 2
        last2 = i;
        any2 = true;
      }
      return true;
    };
    bool go = true;
    for (uint64_t i = 0; i < cnt && go && !*abort_flag; ++i) {
      go = issue(0, i);
      if (go && i >= 1) go = issue(1, i - 1);
    }
    if (go && cnt > 0 && !*abort_flag) issue(1, cnt - 1);
    // the last committed MMAs complete before TMEM is released
    if (any2) tc::mbar_wait(&mdone[2 + int(last2 & 1)], ph(last2), kWaitLimit);
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, 4 * 64);
}

}  // namespace

#ifdef HS_BOUNDS
HS_BOUNDS_TAKE(bounds_take_fused)
#endif

// one unitary per pass: 0 direct, 1 warp-specialised, 2 bulk-loaded (default)
std::atomic<int> g_k4_variant{2};

int set_k4_variant(int v) { return g_k4_variant.exchange(v); }

int launch_compose(const FusedGate* d_gates, const int32_t* d_offs, int nparts, double2* d_u,
                   void* d_a, cudaStream_t s) {
  if (nparts <= 0) return HS_OK;
  HS_TRY(smem_optin(reinterpret_cast<const void*>(k5_compose)));
  k5_compose<<<nparts, kFusedDim, sizeof(double2) * kFusedDim * kFusedDim, s>>>(
      d_gates, d_offs, d_u, static_cast<uint8_t*>(d_a));
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_pack(const double2* d_u, int nparts, void* d_a, cudaStream_t s) {
  if (nparts <= 0) return HS_OK;
  k5_pack<<<nparts, kFusedDim, 0, s>>>(d_u, static_cast<uint8_t*>(d_a));
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

int launch_fused(void* amp, const FusedPass& P, const void* d_a, int* d_err, cudaStream_t s) {
  HS_TRY(smem_optin(reinterpret_cast<const void*>(k4_fused)));
  const int T = 1 << P.m, N = T >> kFusedBits;
  const int variant = g_k4_variant.load();
  // the bulk form copies the lowest run of tile bits (slot 0 upward) and
  // stores two memory-adjacent amplitudes per lane: slot 0 must be tile bit
  // 0 and, when it belongs to the part, its local bit 0
  bool bulk = P.nops == 1 && variant == 2 && P.m <= 13 && P.tile.n > 0 && P.tile.src[0] == 0 &&
              P.tile.dst[0] == 0 && P.tile.len[0] >= 2;
  for (int j = 1; j < kFusedBits; ++j) bulk = bulk && P.pbits[0][j] != 0;
  if (bulk) {
    // A, four raw / B buffers, offset tables, sixteen mbarriers, the abort
    // word, the TMEM address and the epilogue's staging blocks
    HS_TRY(smem_optin(reinterpret_cast<const void*>(k4_bulk)));
    const int chunk_bits = std::min<int>(P.tile.len[0], kBulkMaxChunkBits);
    const int nchunks = T >> chunk_bits;
    const int lgb = P.m <= 12 ? 2 : 1;  // ring of four buffers, or two for 2^13 tiles
    const size_t bsmem = size_t(kFusedABytes) + (size_t(T) * 8 << lgb) + 64 * 8 + size_t(N) * 8 +
                         size_t(nchunks) * 8 + 64 * 4 + size_t(N) * 4 + 20 * 8 +
                         8 * kBulkStageFloats * 4;
    if (bsmem > 227 * 1024) return set_error(HS_E_UNSUPPORTED, "K4 bulk pass needs %zu B", bsmem);
    const int bsms = device_sms();
    const int bgrid = int(P.ntiles < uint64_t(bsms) ? P.ntiles : uint64_t(bsms));
    k4_bulk<<<bgrid, kBulkThreads, bsmem, s>>>(static_cast<float2*>(amp), P,
                                               static_cast<const uint8_t*>(d_a), d_err, chunk_bits,
                                               lgb);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
  }
  // two unitaries per pass on 2^12 tiles: both parts must meet the bulk
  // form's conditions (slot 0 is tile bit 0, and a part holding it has it as
  // local bit 0)
  bool bulk2 = P.nops == 2 && P.m <= kBulk2MaxTileBits && P.m >= kFusedBits + 4 && P.tile.n > 0 &&
               P.tile.src[0] == 0 && P.tile.dst[0] == 0 && P.tile.len[0] >= 2 &&
               g_k4_variant.load() == 2;
  for (int o = 0; o < 2; ++o)
    for (int j = 1; j < kFusedBits; ++j) bulk2 = bulk2 && P.pbits[o][j] != 0;
  if (bulk2) {
    HS_TRY(smem_optin(reinterpret_cast<const void*>(k4_bulk2)));
    const int chunk_bits = std::min<int>(P.tile.len[0], kBulkMaxChunkBits);
    const int nchunks = T >> chunk_bits;
    const size_t smem2 = 2 * size_t(kFusedABytes) + size_t(T) * 16 + size_t(nchunks) * 8 +
                         64 * 8 + size_t(N) * 8 + 128 * 4 + size_t(2 * N + (N & 1)) * 4 +
                         20 * 8 + 8 * kBulkStageFloats * 4;
    if (smem2 > 227 * 1024) return set_error(HS_E_UNSUPPORTED, "K4 two-unitary pass needs %zu B", smem2);
    const int sms = device_sms();
    const int grid2 = int(P.ntiles < uint64_t(sms) ? P.ntiles : uint64_t(sms));
    k4_bulk2<<<grid2, kBulk2Threads, smem2, s>>>(static_cast<float2*>(amp), P,
                                                 static_cast<const uint8_t*>(d_a), d_err, chunk_bits);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
  }
  if (P.nops == 1 && variant >= 1) {
    // warp-specialised form: A, two B buffers, offset tables, six mbarriers
    HS_TRY(smem_optin(reinterpret_cast<const void*>(k4_ws)));
    if (P.m > 13) return set_error(HS_E_UNSUPPORTED, "K4 tiles up to 2^13");
    const size_t wsmem = size_t(kFusedABytes) + size_t(N) * 1024 + 64 * 8 + size_t(N) * 8 +
                         6 * 8 + 8 + 16;
    const int wsms = device_sms();
    const int wgrid = int(P.ntiles < uint64_t(wsms) ? P.ntiles : uint64_t(wsms));
    k4_ws<<<wgrid, kWsThreads, wsmem, s>>>(static_cast<float2*>(amp), P,
                                           static_cast<const uint8_t*>(d_a), d_err);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
  }
  if (P.nops == 1) {
    // direct form: A, two B buffers, offset tables, barriers
    HS_TRY(smem_optin(reinterpret_cast<const void*>(k4_direct)));
    const size_t dsmem = size_t(kFusedABytes) + size_t(N) * 1024 + 64 * 8 + size_t(N) * 8 + 16 + 16;
    if (P.m > 13) return set_error(HS_E_UNSUPPORTED, "K4 tiles up to 2^13");
    const int dsms = device_sms();
    const int dgrid = int(P.ntiles < uint64_t(dsms) ? P.ntiles : uint64_t(dsms));
    k4_direct<<<dgrid, kK4DirectThreads, dsmem, s>>>(static_cast<float2*>(amp), P,
                                               static_cast<const uint8_t*>(d_a), d_err);
    HS_CUDA(cudaGetLastError());
    return HS_OK;
  }
  // A operands, B hi/lo, two tile buffers, the dp/dn tables, chunk offsets
  // (8-byte aligned), mbarrier, TMEM address
  const size_t tables = (size_t(P.nops) * (64 + N) * 2 + 7) & ~size_t(7);
  const size_t smem = size_t(P.nops) * kFusedABytes + size_t(N) * 512 + size_t(T) * 16 + tables +
                      8 * 8 + 8 + 8 + 16;
  if (smem > 227 * 1024) return set_error(HS_E_UNSUPPORTED, "K4 pass needs %zu B of shared memory", smem);
  const int sms = device_sms();
  int per_sm = 1;
  HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k4_fused, kK4Threads, smem));
  if (per_sm < 1) return set_error(HS_E_UNSUPPORTED, "K4 pass does not fit an SM");
  const uint64_t want = uint64_t(sms) * uint64_t(per_sm);
  const int grid = int(P.ntiles < want ? P.ntiles : want);
  k4_fused<<<grid, kK4Threads, smem, s>>>(static_cast<float2*>(amp), P,
                                          static_cast<const uint8_t*>(d_a), d_err);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace hisv
