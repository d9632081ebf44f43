// K1: the part kernel.  One CTA holds one 2^m-amplitude tile of the state at a
// time (grid-stride over the 2^(n-m) tiles); every gate of the part is applied
// to the tile on chip and the tile is written back once.
//
// Replaces the per-part gather -> execute_on -> scatter of
// gather_and_execute_on_multi (execute.hpp:318-470) and the OpenMP loop nest
// that drives it (loop.hpp:468-962, state_vector.hpp:310-342).
//
// Layout on chip: thread t of the CTA holds E = 2^R amplitudes v[e]; the tile
// index of v[e] is deposit(t -> the group's thread bits) | deposit(e -> the
// group's register bits).  A gate targets register bits only, so it runs on
// registers with compile-time indices.  Between groups the tile goes through
// shared memory (XOR-swizzled 16-byte slots) to re-assign the register bits.
// The first group loads straight from global memory and the last group stores
// straight to it.
#include "internal.h"

namespace hisv {
namespace {

template <typename V>
struct Scalar;
template <>
struct Scalar<double2> {
  using T = double;
};
template <>
struct Scalar<float2> {
  using T = float;
};

template <typename V>
__device__ __forceinline__ V mk(typename Scalar<V>::T x, typename Scalar<V>::T y) {
  V r;
  r.x = x;
  r.y = y;
  return r;
}

// c * a + d * b with complex operands (coefficients in double, cast to T)
template <typename V>
__device__ __forceinline__ V cmac2(double2 c, V a, double2 d, V b) {
  using T = typename Scalar<V>::T;
  const T cr = T(c.x), ci = T(c.y), dr = T(d.x), di = T(d.y);
  T re = cr * a.x;
  re = fma(-ci, a.y, re);
  re = fma(dr, b.x, re);
  re = fma(-di, b.y, re);
  T im = cr * a.y;
  im = fma(ci, a.x, im);
  im = fma(dr, b.y, im);
  im = fma(di, b.x, im);
  return mk<V>(re, im);
}

template <typename V>
__device__ __forceinline__ V cmul(double2 c, V a) {
  using T = typename Scalar<V>::T;
  const T cr = T(c.x), ci = T(c.y);
  return mk<V>(fma(-ci, a.y, cr * a.x), fma(ci, a.x, cr * a.y));
}

__device__ __forceinline__ uint64_t deposit(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i)
    out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}

// shared-memory slot of tile index i: XOR the 16-byte slot within a 128-byte
// row with a fold of the higher bits, so that lanes differing in any three
// bits with distinct residues mod 3 hit distinct bank groups
__device__ __forceinline__ uint32_t swz(uint32_t i) {
  return i ^ (((i >> 3) ^ (i >> 6) ^ (i >> 9) ^ (i >> 12)) & 7u);
}

// ---- gate bodies on registers ------------------------------------------------
// Each thread holds its amplitudes in one of two register arrays.  Uncontrolled
// dense gates write the other array (all of its elements), so no register is
// copied back after a gate; the op interpreter is a two-state machine that
// tracks which array holds the data.  Controlled dense gates and diagonal
// gates update the current array in place; sign flips and phases are
// specialized by their register mask so only the affected elements are
// touched.

__host__ __device__ constexpr int lowest_bit(int e) {
  return (e & 1) ? 0 : (e & 2) ? 1 : (e & 4) ? 2 : (e & 8) ? 3 : (e & 16) ? 4 : 5;
}

template <int J>
__device__ __forceinline__ constexpr int ins0(int p) {  // insert a 0 bit at J
  return ((p >> J) << (J + 1)) | (p & ((1 << J) - 1));
}

__device__ __forceinline__ double flip_sign(double x, uint32_t sm) {
  return __hiloint2double(__double2hiint(x) ^ int(sm), __double2loint(x));
}
__device__ __forceinline__ float flip_sign(float x, uint32_t sm) {
  return __int_as_float(__float_as_int(x) ^ int(sm));
}

// dense 2x2 on register bit J, src -> dst
template <int R, int J, typename V>
__device__ __forceinline__ void d1x(const V (&s)[1 << R], V (&d)[1 << R], const double2* __restrict__ c) {
  constexpr int E = 1 << R;
  const double2 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
#pragma unroll
  for (int p = 0; p < E / 2; ++p) {
    const int e0 = ins0<J>(p), e1 = e0 | (1 << J);
    d[e0] = cmac2(c0, s[e0], c1, s[e1]);
    d[e1] = cmac2(c2, s[e0], c3, s[e1]);
  }
}

// dense 2x2 with a real top-left coefficient on register bit J, in place
template <int R, int J, typename V>
__device__ __forceinline__ void d1r(V (&v)[1 << R], const double2* __restrict__ c) {
  using T = typename Scalar<V>::T;
  constexpr int E = 1 << R;
  const T c0 = T(c[0].x), c1r = T(c[1].x), c1i = T(c[1].y);
  const double2 c2 = c[2], c3 = c[3];
#pragma unroll
  for (int p = 0; p < E / 2; ++p) {
    const int e0 = ins0<J>(p), e1 = e0 | (1 << J);
    const V a = v[e0], b = v[e1];
    T re = c0 * a.x;
    re = fma(c1r, b.x, re);
    re = fma(-c1i, b.y, re);
    T im = c0 * a.y;
    im = fma(c1r, b.y, im);
    im = fma(c1i, b.x, im);
    v[e0] = mk<V>(re, im);
    v[e1] = cmac2(c2, a, c3, b);
  }
}

// dense 2x2 on register bit J, in place, for pairs whose controls hold
template <int R, int J, typename V>
__device__ __forceinline__ void d1c(V (&v)[1 << R], const double2* __restrict__ c, uint32_t creg,
                                    bool ok) {
  constexpr int E = 1 << R;
  const double2 c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
#pragma unroll
  for (int p = 0; p < E / 2; ++p) {
    const int e0 = ins0<J>(p), e1 = e0 | (1 << J);
    if (!ok || (uint32_t(e0) & creg) != creg) continue;
    const V a = v[e0], b = v[e1];
    v[e0] = cmac2(c0, a, c1, b);
    v[e1] = cmac2(c2, a, c3, b);
  }
}

// sign flip of the elements whose register bits cover mask M (sm = 0 or sign bit)
template <int R, int M, typename V>
__device__ __forceinline__ void dneg(V (&v)[1 << R], uint32_t sm) {
  constexpr int E = 1 << R;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if ((e & M) == M) {
      v[e].x = flip_sign(v[e].x, sm);
      v[e].y = flip_sign(v[e].y, sm);
    }
}

// multiply the elements whose register bits cover mask M by f (in place)
template <int R, int M, typename V>
__device__ __forceinline__ void dphase(V (&v)[1 << R], double2 f) {
  using T = typename Scalar<V>::T;
  constexpr int E = 1 << R;
  const T fx = T(f.x), fy = T(f.y);
#pragma unroll
  for (int e = 0; e < E; ++e)
    if ((e & M) == M) {
      const T a = fy * v[e].y, b = fy * v[e].x;
      v[e].x = fma(fx, v[e].x, -a);
      v[e].y = fma(fx, v[e].y, b);
    }
}

// general diagonal: coefficient c[b0 | b1 << 1] with its target bits read from
// register, thread or outer bits (in place)
template <int R, typename V>
__device__ __forceinline__ void ddiag(V (&v)[1 << R], const DevOp& op, const double2* __restrict__ c,
                                      uint32_t thr, uint64_t gbase, bool ok) {
  constexpr int E = 1 << R;
  const uint32_t creg = ok ? uint32_t(op.creg) : 0xffffffffu;
  auto fixed = [&](uint8_t w, uint8_t pos) -> uint32_t {
    return w == TW_THR ? ((thr >> pos) & 1u) : w == TW_OUT ? uint32_t((gbase >> pos) & 1ull) : 0u;
  };
  const uint32_t f0 = fixed(op.t0w, op.t0p), f1 = fixed(op.t1w, op.t1p) << 1;
  const bool r0 = op.t0w == TW_REG, r1 = op.t1w == TW_REG;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    if ((uint32_t(e) & creg) != creg) continue;
    const uint32_t q0 = r0 ? ((uint32_t(e) >> op.t0p) & 1u) : f0;
    const uint32_t q1 = r1 ? (((uint32_t(e) >> op.t1p) & 1u) << 1) : f1;
    v[e] = cmul(c[q0 | q1], v[e]);
  }
}

// dense 4x4 on register bits JA < JB, src -> dst
template <int R, int JA, int JB, typename V>
__device__ __forceinline__ void d2x(const V (&s)[1 << R], V (&d)[1 << R], const double2* __restrict__ c) {
  constexpr int E = 1 << R;
#pragma unroll
  for (int p = 0; p < E / 4; ++p) {
    const int x = ins0<JB>(ins0<JA>(p));
    const int e[4] = {x, x | (1 << JA), x | (1 << JB), x | (1 << JA) | (1 << JB)};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const V t0 = cmac2(c[4 * r], s[e[0]], c[4 * r + 1], s[e[1]]);
      const V t1 = cmac2(c[4 * r + 2], s[e[2]], c[4 * r + 3], s[e[3]]);
      d[e[r]] = mk<V>(t0.x + t1.x, t0.y + t1.y);
    }
  }
}

// 4x4 dense (controlled) or swap, in place
template <int R, int JA, int JB, bool SWAP, typename V>
__device__ __forceinline__ void d2c(V (&v)[1 << R], const double2* __restrict__ c, uint32_t creg,
                                    bool ok) {
  constexpr int E = 1 << R;
#pragma unroll
  for (int p = 0; p < E / 4; ++p) {
    const int x = ins0<JB>(ins0<JA>(p));
    const int e[4] = {x, x | (1 << JA), x | (1 << JB), x | (1 << JA) | (1 << JB)};
    if (!ok || (uint32_t(x) & creg) != creg) continue;
    if (SWAP) {
      const V t = v[e[1]];
      v[e[1]] = v[e[2]];
      v[e[2]] = t;
    } else {
      const V a[4] = {v[e[0]], v[e[1]], v[e[2]], v[e[3]]};
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const V t0 = cmac2(c[4 * r], a[0], c[4 * r + 1], a[1]);
        const V t1 = cmac2(c[4 * r + 2], a[2], c[4 * r + 3], a[3]);
        v[e[r]] = mk<V>(t0.x + t1.x, t0.y + t1.y);
      }
    }
  }
}

// HS_K1_PINGPONG=1: uncontrolled dense gates write the second register array
// (two-state interpreter); 0: every gate updates one array in place.
#ifndef HS_K1_PINGPONG
#define HS_K1_PINGPONG 0
#endif

template <bool FULL>
__device__ __forceinline__ bool is_xfer(int code) {
  return HS_K1_PINGPONG && (code < 4 || (FULL && code >= 64 && code < 70));
}

template <int R, bool FULL, typename V>
__device__ __forceinline__ void op_xfer(const V (&s)[1 << R], V (&d)[1 << R], int code,
                                        const double2* c) {
#define X1(J) \
  case (J): if constexpr ((J) < R) d1x<R, J>(s, d, c); break;
#define X2(P, JA, JB) \
  case 64 + (P): if constexpr (FULL && (JB) < R) d2x<R, JA, JB>(s, d, c); break;
  switch (code) {
    X1(0) X1(1) X1(2) X1(3)
    X2(0, 0, 1) X2(1, 0, 2) X2(2, 0, 3) X2(3, 1, 2) X2(4, 1, 3) X2(5, 2, 3)
    default: break;
  }
#undef X1
#undef X2
}

// A per-thread sign that commutes with every op of a group: sign flips whose
// mask lies wholly in thread / outer bits negate all of a thread's
// amplitudes, so they are collected and applied once when the group ends.
template <typename V>
struct Deferred {
  uint32_t sign = 0;   // 0 or the sign bit
  bool any = false;    // warp-uniform: a sign was deferred in this group
};

template <int R, typename V>
__device__ __forceinline__ void apply_deferred(V (&v)[1 << R], const Deferred<V>& d) {
  constexpr int E = 1 << R;
  if (!d.any) return;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    v[e].x = flip_sign(v[e].x, d.sign);
    v[e].y = flip_sign(v[e].y, d.sign);
  }
}

template <int R, bool FULL, typename V>
__device__ __forceinline__ void op_inplace(V (&v)[1 << R], const DevOp& op, const double2* c,
                                           uint32_t thr, uint64_t gbase, Deferred<V>& dfr) {
  // thread and outer part of the controls (register part is in the code /
  // creg); evaluated only by the ops that have such controls
  auto ok = [&]() {
    return ((thr & op.cthr) == op.cthr) && ((gbase & op.couter) == op.couter);
  };
#define C1(J) \
  case 4 + (J): if constexpr ((J) < R) d1c<R, J>(v, c, op.creg, ok()); break;
#define NEG(M) \
  case 16 + (M): if constexpr ((M) < (1 << R)) dneg<R, M>(v, ok() ? 0x80000000u : 0u); break;
#define PH(M) \
  case 32 + (M): if constexpr ((M) < (1 << R)) dphase<R, M>(v, ok() ? c[0] : make_double2(1.0, 0.0)); break;
#define C2(P, JA, JB) \
  case 72 + (P): if constexpr (FULL && (JB) < R) d2c<R, JA, JB, false>(v, c, op.creg, ok()); break;
#define SW(P, JA, JB) \
  case 80 + (P): if constexpr (FULL && (JB) < R) d2c<R, JA, JB, true>(v, c, op.creg, ok()); break;
#define D1(J) \
  case (J): if constexpr ((J) < R) d1c<R, J>(v, c, 0u, true); break;
#define D2(P, JA, JB) \
  case 64 + (P): if constexpr (FULL && (JB) < R) d2c<R, JA, JB, false>(v, c, 0u, true); break;
#define DR(J) \
  case 88 + (J): if constexpr ((J) < R) d1r<R, J>(v, c); break;
  // the most frequent ops first (uncontrolled dense one-qubit gates, with a
  // real top-left coefficient or general), so that their dispatch takes two
  // short tests instead of a search over every code
  const int code = op.code;
  if (code >= 88) {
    switch (code) {
      DR(0) DR(1) DR(2) DR(3)
      default: break;
    }
    return;
  }
  if (code < 4) {
    switch (code) {
      D1(0) D1(1) D1(2) D1(3)
      default: break;
    }
    return;
  }
  switch (code) {
    D2(0, 0, 1) D2(1, 0, 2) D2(2, 0, 3) D2(3, 1, 2) D2(4, 1, 3) D2(5, 2, 3)
    C1(0) C1(1) C1(2) C1(3)
    case 16:  // sign flip of every element of the thread (mask outside the registers)
      dfr.sign ^= ok() ? 0x80000000u : 0u;
      dfr.any = true;
      break;
    NEG(1) NEG(2) NEG(3) NEG(4) NEG(5) NEG(6) NEG(7)
    NEG(8) NEG(9) NEG(10) NEG(11) NEG(12) NEG(13) NEG(14) NEG(15)
    PH(0) PH(1) PH(2) PH(3) PH(4) PH(5) PH(6) PH(7)
    PH(8) PH(9) PH(10) PH(11) PH(12) PH(13) PH(14) PH(15)
    case 48: ddiag<R>(v, op, c, thr, gbase, ok()); break;
    C2(0, 0, 1) C2(1, 0, 2) C2(2, 0, 3) C2(3, 1, 2) C2(4, 1, 3) C2(5, 2, 3)
    SW(0, 0, 1) SW(1, 0, 2) SW(2, 0, 3) SW(3, 1, 2) SW(4, 1, 3) SW(5, 2, 3)
    default: break;
  }
#undef D1
#undef D2
#undef DR
#undef C1
#undef NEG
#undef PH
#undef C2
#undef SW
}

}  // namespace

namespace {

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared-memory byte offset of tile index i: 16-byte slots hold 1 (complex128)
// or 2 (complex64) amplitudes; slots are XOR-swizzled (swz is linear over
// GF(2), so the offset of thr | reg(e) is built from per-bit parts).
template <typename V>
struct SmemMap {
  static constexpr int SH = sizeof(V) == 8 ? 1 : 0;  // amplitudes per slot = 2^SH
  __device__ __forceinline__ static uint32_t off(uint32_t i) {
    return (swz(i >> SH) << 4) | ((i & ((1u << SH) - 1u)) * uint32_t(sizeof(V)));
  }
};

// Issue the asynchronous copy of one tile into a shared buffer: 16-byte
// chunks, chunk c covering tile indices [c*2^SH, (c+1)*2^SH) that are
// contiguous in global memory (tile bit 0 is always global slot 0 when SH=1).
template <int R, typename V>
__device__ __forceinline__ void issue_tile_load(const V* __restrict__ sv, uint32_t sbuf,
                                                uint64_t gbase, const uint64_t* __restrict__ gchunk,
                                                uint64_t gt, int nchunk_per_thr) {
  using M = SmemMap<V>;
  const uint32_t t = threadIdx.x;
  for (int k = 0; k < nchunk_per_thr; ++k) {
    const uint32_t c = t + uint32_t(k) * blockDim.x;
    const uint64_t g = gbase + gt + gchunk[k];
    cp_async16(sbuf + (swz(c) << 4), sv + g);
  }
  (void)M::SH;
}

// complex64 tiles are at most 2^12 amplitudes: 2^(12-R) = 256 threads, one
// CTA per SM bound; complex128 tiles at most 2^11: 128 threads of 16
// amplitudes (R = 4) or 256 threads of 8 (R = 3), and the register bound
// leaves room for three CTAs per SM (FP64-heavy passes need the extra warps
// to hide latency; with two-qubit dense ops, R = 3 takes two CTAs of 256
// threads so that the 4x4 bodies do not spill)
constexpr int kThrCache = 4;  // groups whose thread parts are tabulated per launch

template <typename V, int R, bool FULL>
struct K1Threads {
  static constexpr int value = 256;
  static constexpr int min_blocks = 1;
};
template <int R, bool FULL>
struct K1Threads<double2, R, FULL> {
  static constexpr int value = R == 3 ? 256 : 128;
  static constexpr int min_blocks = (R == 3 && FULL) ? 2 : 3;
};

template <int R, bool FULL, typename V>
__global__ void __launch_bounds__(K1Threads<V, R, FULL>::value, K1Threads<V, R, FULL>::min_blocks)
    k1_part(V* __restrict__ sv, const __grid_constant__ PartProgram P) {
  using M = SmemMap<V>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int E = 1 << R;
  const uint32_t t = threadIdx.x;
  const uint32_t nthr = blockDim.x;
  const uint32_t tile_bytes = uint32_t(sizeof(V)) << P.m;
  unsigned char* buf[2] = {smem_raw, smem_raw + tile_bytes};
  uint64_t* s_gchunk = reinterpret_cast<uint64_t*>(smem_raw + 2 * tile_bytes);
  // chunk c = t + k*nthr; its first tile index is c << SH.  The bits of t and
  // of k*nthr are disjoint, so deposit(c << SH) = deposit(t << SH) + deposit(k*nthr << SH).
  const int nchunk = (1 << P.m) >> M::SH;
  const int per_thr = nchunk / int(nthr);
  // the last group writes its registers straight to global memory: the global
  // offset of each of its register bits and of each thread's thread part
  // (after the chunk table; kept in shared memory to spare registers)
  uint64_t* s_glreg = s_gchunk + per_thr;
  uint64_t* s_glthr = s_glreg + R;
  // the thread part (tile index bits held by this thread) of the first
  // kThrCache groups, the same in every tile
  uint32_t* s_thr = reinterpret_cast<uint32_t*>(s_glthr + nthr);
  const GroupDesc& GL = P.groups[P.ngroups - 1];
  for (int k = t; k < per_thr; k += nthr)
    s_gchunk[k] = deposit(uint64_t(k) * nthr << M::SH, P.tile);
  for (int j = int(t); j < R; j += int(nthr)) s_glreg[j] = deposit(1ull << GL.reg_tbit[j], P.tile);
  // (the last group's lanes run over the lowest tile bits, so the direct
  // stores coalesce)
  s_glthr[t] = deposit(deposit(t, GL.thr), P.tile);
  for (int g = 0; g < P.ngroups && g < kThrCache; ++g)
    s_thr[g * nthr + t] = uint32_t(deposit(t, P.groups[g].thr));
  __syncthreads();
  const uint64_t gt = deposit(uint64_t(t) << M::SH, P.tile);
  const uint32_t sb0 = uint32_t(__cvta_generic_to_shared(buf[0]));
  const uint32_t sb1 = uint32_t(__cvta_generic_to_shared(buf[1]));

  uint64_t tile = blockIdx.x;
  if (tile < P.ntiles)
    issue_tile_load<R, V>(sv, sb0, deposit(tile, P.outer), s_gchunk, gt, per_thr);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  V v[E], w[E];
  for (int it = 0; tile < P.ntiles; ++it, tile += gridDim.x) {
    // this tile has landed and every thread is past the previous one (the
    // barrier that ends the previous tile's last group), so the previous
    // tile's buffer may take the next tile
    const uint64_t next = tile + gridDim.x;
    if (next < P.ntiles) {
      issue_tile_load<R, V>(sv, (it & 1) ? sb0 : sb1, deposit(next, P.outer), s_gchunk, gt,
                            per_thr);
      cp_async_commit();
    }
    unsigned char* A = buf[it & 1];
    const uint64_t gbase = deposit(tile, P.outer);
    for (int g = 0; g < P.ngroups; ++g) {
      const GroupDesc& G = P.groups[g];
      const bool last = g == P.ngroups - 1;
      const uint32_t thr = g < kThrCache ? s_thr[g * nthr + t] : uint32_t(deposit(t, G.thr));
      // per register bit: the offset change of setting that bit (swizzled slot
      // part and in-slot part occupy disjoint bits, so they combine by XOR and
      // so do the bits of an element index)
      uint32_t dx[R];
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const uint32_t b = 1u << G.reg_tbit[j];
        dx[j] = (swz(b >> M::SH) << 4) ^ ((b & ((1u << M::SH) - 1u)) * uint32_t(sizeof(V)));
      }
      const uint32_t sthr = M::off(thr);
      // offsets of the E elements, each one XOR from an earlier one
      auto offsets = [&](uint32_t (&a)[E]) {
        a[0] = sthr;
#pragma unroll
        for (int e = 1; e < E; ++e) a[e] = a[e & (e - 1)] ^ dx[lowest_bit(e)];
      };
      // the group's result: to shared memory for the next group, or (last
      // group) straight to global memory, each element's offset a sum of
      // disjoint bit parts
      auto finish = [&](const V (&x)[E]) {
        if (last) {
          // elements in Gray-code order: each address is the previous one
          // plus or minus one register bit's offset (one live pointer)
          V* p = sv + gbase + s_glthr[t];
#pragma unroll
          for (int i = 0; i < E; ++i) {
            const int e = i ^ (i >> 1);
            if (i > 0) {
              const int j = lowest_bit(i);
              if ((e >> j) & 1) p += s_glreg[j]; else p -= s_glreg[j];
            }
            __stcs(p, x[e]);
          }
        } else {
          uint32_t a[E];
          offsets(a);
#pragma unroll
          for (int e = 0; e < E; ++e) *reinterpret_cast<V*>(A + a[e]) = x[e];
        }
      };
      {
        uint32_t a[E];
        offsets(a);
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = *reinterpret_cast<const V*>(A + a[e]);
      }
      // op descriptors and coefficients are read from the (warp-uniform)
      // parameter space, so every dispatch below is a uniform branch
      int o = G.first_op;
      const int o_end = G.first_op + G.num_ops;
      Deferred<V> dfr;
    in_v:
      while (o < o_end) {
        const DevOp& op = P.ops[o++];
        if (is_xfer<FULL>(op.code)) {
          op_xfer<R, FULL>(v, w, op.code, P.coef + op.coef);
          goto in_w;
        }
        op_inplace<R, FULL>(v, op, P.coef + op.coef, thr, gbase, dfr);
      }
      apply_deferred<R>(v, dfr);
      finish(v);
      goto group_done;
    in_w:
      while (o < o_end) {
        const DevOp& op = P.ops[o++];
        if (is_xfer<FULL>(op.code)) {
          op_xfer<R, FULL>(w, v, op.code, P.coef + op.coef);
          goto in_v;
        }
        op_inplace<R, FULL>(w, op, P.coef + op.coef, thr, gbase, dfr);
      }
      apply_deferred<R>(w, dfr);
      finish(w);
    group_done:
      // the group's writes precede the next group's reads; after the last
      // group the next tile's copies (the only ones in flight) must have
      // landed and every thread must be done with this tile's buffer
      if (last) cp_async_wait<0>();
      __syncthreads();
    }
  }
  cp_async_wait<0>();
}

struct LaunchCfg {
  int threads;
  size_t smem;
  int grid;
};

int g_num_sms = 0;

template <int R, bool FULL, typename V>
int launch_k1(V* sv, const PartProgram& P, cudaStream_t s) {
  static bool attr_set[64] = {false};
  int dev = 0;
  HS_CUDA(cudaGetDevice(&dev));
  if (!attr_set[dev & 63]) {
    HS_CUDA(cudaFuncSetAttribute(k1_part<R, FULL, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 227 * 1024));
    attr_set[dev & 63] = true;
  }
  if (g_num_sms == 0) HS_CUDA(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 1 << (P.m - R);
  const int per_thr = ((1 << P.m) * int(sizeof(V)) / 16) / threads;
  const size_t smem = 2 * (sizeof(V) << P.m) + sizeof(uint64_t) * (per_thr + R + threads) +
                      sizeof(uint32_t) * kThrCache * threads;
  if (smem > 227 * 1024) return set_error(HS_E_UNSUPPORTED, "K1 tile of 2^%d needs %zu B", P.m, smem);
  int per_sm = 0;
  HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k1_part<R, FULL, V>, threads, smem));
  if (per_sm < 1) return set_error(HS_E_UNSUPPORTED, "K1 tile does not fit an SM (m=%d)", P.m);
  const uint64_t want = uint64_t(g_num_sms) * uint64_t(per_sm);
  const int grid = int(P.ntiles < want ? P.ntiles : want);
  k1_part<R, FULL, V><<<grid, threads, smem, s>>>(sv, P);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace

template <typename V>
int launch_typed(V* a, const PartProgram& P, cudaStream_t s) {
  bool full = false;
  for (int i = 0; i < P.nops; ++i) full |= P.ops[i].kind == OP2_DENSE || P.ops[i].kind == OP2_SWAP;
  const int R = P.rbits;
  if (full) {
    switch (R) {
      case 1: return launch_k1<1, true>(a, P, s);
      case 2: return launch_k1<2, true>(a, P, s);
      case 3: return launch_k1<3, true>(a, P, s);
      default: return launch_k1<4, true>(a, P, s);
    }
  }
  switch (R) {
    case 1: return launch_k1<1, false>(a, P, s);
    case 2: return launch_k1<2, false>(a, P, s);
    case 3: return launch_k1<3, false>(a, P, s);
    default: return launch_k1<4, false>(a, P, s);
  }
}

int launch_part(void* amp, int dtype, const PartProgram& P, cudaStream_t s) {
  if (P.ngroups < 1 || P.nops < 1) return HS_OK;
  if (dtype == HS_DTYPE_C128) return launch_typed(static_cast<double2*>(amp), P, s);
  return launch_typed(static_cast<float2*>(amp), P, s);
}

}  // namespace hisv
