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
// The first group loads from the tile buffer that cp.async filled while the
// previous tile was processed; the last group stores straight to global memory.
//
// Op dispatch: every op carries one dense code (K1Code), so the switch below
// is a jump table; op descriptors are read from the (warp-uniform) parameter
// space, coefficients from a shared-memory copy (one 16-byte load each).
#include "bounds.cuh"
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

__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
  return make_double2(fma(-a.y, b.y, a.x * b.x), fma(a.y, b.x, a.x * b.y));
}

__device__ __forceinline__ uint64_t deposit(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i)
    out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}

// shared-memory slot of 16-byte slot s: s XOR the program's fold of its bits
// (a move within the 128-byte row, chosen by the planner so that every
// register group's lanes hit distinct banks)
__device__ __forceinline__ uint32_t swz(const PartProgram& P, uint32_t s) {
  uint32_t r = s;
  for (int k = 0; s >> k; ++k)
    if ((s >> k) & 1u) r ^= P.fold[k];
  return r;
}

// ---- gate bodies on registers (in place) -------------------------------------

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

// Rotation on register bit J, every step an in-place shear x += t y (so no
// register is copied): with Z, the phase e^{i beta} turns the (re, im) plane
// of the pair's second amplitude B by the three shears (cz = (tan(beta/2),
// sin(beta))); then the (A.re, B.re) and (A.im, B.im) planes take the real
// shears of cy = (t, s) in the given form: 0 = A += tB; B += sA; A += tB
// (an exact plane rotation), 1 = the first two, 2 = the last two (the
// planner carries the scale these leave).  9 FMA per amplitude pair (7 in
// forms 1 and 2), 6 (4) without the phase.  The form is warp-uniform.
template <int R, int J, bool Z, typename V>
__device__ __forceinline__ void rot(V (&v)[1 << R], const double2 cy, const double2 cz,
                                    uint32_t form) {
  using T = typename Scalar<V>::T;
  constexpr int NP = (1 << R) / 2;
  const T t = T(cy.x), s = T(cy.y), tz = T(cz.x), sz = T(cz.y);
  // one shear at a time across all pairs: NP-fold independent FMAs per step
#define A(p) v[ins0<J>(p)]
#define B(p) v[ins0<J>(p) | (1 << J)]
  if constexpr (Z) {
#pragma unroll
    for (int p = 0; p < NP; ++p) B(p).x = fma(-tz, B(p).y, B(p).x);
#pragma unroll
    for (int p = 0; p < NP; ++p) B(p).y = fma(sz, B(p).x, B(p).y);
#pragma unroll
    for (int p = 0; p < NP; ++p) B(p).x = fma(-tz, B(p).y, B(p).x);
  }
  if (!(form & 2u)) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      A(p).x = fma(t, B(p).x, A(p).x);
      A(p).y = fma(t, B(p).y, A(p).y);
    }
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    B(p).x = fma(s, A(p).x, B(p).x);
    B(p).y = fma(s, A(p).y, B(p).y);
  }
  if (!(form & 1u)) {
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      A(p).x = fma(t, B(p).x, A(p).x);
      A(p).y = fma(t, B(p).y, A(p).y);
    }
  }
#undef A
#undef B
}

// dense 2x2 on register bit J for pairs whose controls hold
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

// multiply the elements whose register bits cover mask M by f
template <int R, int M, typename V>
__device__ __forceinline__ void dphase(V (&v)[1 << R], double2 f) {
  constexpr int E = 1 << R;
#pragma unroll
  for (int e = 0; e < E; ++e)
    if ((e & M) == M) v[e] = cmul(f, v[e]);
}

// general diagonal: coefficient c[b0 | b1 << 1] with its target bits read from
// register, thread or outer bits
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

// 4x4 dense (optionally controlled) or swap on register bits JA < JB
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

// A per-thread sign that commutes with every op of a group: sign flips whose
// mask lies wholly in thread / outer bits negate all of a thread's
// amplitudes, so they are collected and applied once when the group ends.
struct Deferred {
  uint32_t sign = 0;   // 0 or the sign bit
  bool any = false;    // warp-uniform: a sign was deferred in this group
};

template <int R, typename V>
__device__ __forceinline__ void apply_deferred(V (&v)[1 << R], const Deferred& d) {
  constexpr int E = 1 << R;
  if (!d.any) return;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    v[e].x = flip_sign(v[e].x, d.sign);
    v[e].y = flip_sign(v[e].y, d.sign);
  }
}

// One non-rotation op on a thread's registers.  `op` lives in the parameter
// space (its fields are warp-uniform), `c` in shared memory.  Sign flips
// update registers in place and come first.  With FAST the other kinds are
// limited to phases and the frame flush: a program goes to the FAST
// instantiation when it holds nothing else, because a switch over every op
// kind in the loop makes the compiler reconcile the register copies of all
// cases at its join (measured: ~50 register moves per op and 160 instead of
// ~110 registers per thread).
template <int R, bool FULL, bool FAST, typename V>
__device__ __forceinline__ void run_op(V (&v)[1 << R], const DevOp& op, const double2* s_coef,
                                       uint32_t thr, uint64_t gbase, Deferred& dfr,
                                       const PartProgram& P) {
  constexpr int E = 1 << R;
  // the op's first 24 bytes in three 8-byte loads: code (byte 1), coefficient
  // index (bytes 8-9), thread mask (bytes 12-15), outer mask (bytes 16-23)
  const uint64_t* ow = reinterpret_cast<const uint64_t*>(&op);
  const uint64_t w0 = ow[0], w1 = ow[1], w2 = ow[2];
  const int code = int(w0 >> 8) & 255;
  const double2* c = s_coef + (uint32_t(w1) & 0xffffu);
  if (!HS_IN_BOUNDS((uint32_t(w1) & 0xffffu) <= uint32_t(P.ncoef), kBoundsK1)) return;
  const uint32_t cthr = uint32_t(w1 >> 32);
  // thread and outer part of the controls (the register part is in the code /
  // creg); evaluated only by the ops that have such controls
  auto ok = [&]() { return ((thr & cthr) == cthr) && ((gbase & w2) == w2); };
  if (code >= kc_neg && code < kc_ph) {  // sign flips (CZ and other -1 phases)
    const uint32_t sm = ok() ? 0x80000000u : 0u;
#define NEG(M) \
  case kc_neg + (M): if constexpr ((M) < (1 << R)) dneg<R, M>(v, sm); break;
    switch (code) {
      case kc_neg:  // every element of the thread (mask outside the registers): deferred
        dfr.sign ^= sm;
        dfr.any = true;
        break;
      NEG(1) NEG(2) NEG(3) NEG(4) NEG(5) NEG(6) NEG(7)
      NEG(8) NEG(9) NEG(10) NEG(11) NEG(12) NEG(13) NEG(14) NEG(15)
      default: break;
    }
#undef NEG
    return;
  }
  if (code == kc_flush) {
    // G times the factors of the listed thread / outer bits that are set
    double2 f = c[0];
    const int f0 = op.fl_first, nf = op.fl_n;
    for (int i = 0; i < nf; ++i) {
      const uint32_t wh = P.flw[f0 + i], pos = P.flp[f0 + i];
      const uint32_t bit = wh == TW_THR ? (thr >> pos) & 1u : uint32_t(gbase >> pos) & 1u;
      if (bit) f = cmul_d(c[1 + i], f);
    }
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cmul(f, v[e]);
    return;
  }
#define PH(M) \
  case kc_ph + (M): if constexpr ((M) < (1 << R)) dphase<R, M>(v, ok() ? c[0] : make_double2(1.0, 0.0)); break;
#define D1(J) \
  case kc_d1 + (J): if constexpr (!FAST && (J) < R) d1c<R, J>(v, c, 0u, true); break;
#define C1(J) \
  case kc_c1 + (J): if constexpr (!FAST && (J) < R) d1c<R, J>(v, c, op.creg, ok()); break;
#define D2(P_, JA, JB) \
  case kc_d2 + (P_): if constexpr (!FAST && FULL && (JB) < R) d2c<R, JA, JB, false>(v, c, 0u, true); break;
#define C2(P_, JA, JB) \
  case kc_c2 + (P_): if constexpr (!FAST && FULL && (JB) < R) d2c<R, JA, JB, false>(v, c, op.creg, ok()); break;
#define SW(P_, JA, JB) \
  case kc_sw + (P_): if constexpr (!FAST && FULL && (JB) < R) d2c<R, JA, JB, true>(v, c, op.creg, ok()); break;
#define PAIRS(X) X(0, 0, 1) X(1, 0, 2) X(2, 0, 3) X(3, 1, 2) X(4, 1, 3) X(5, 2, 3)
  switch (code) {
    PH(0) PH(1) PH(2) PH(3) PH(4) PH(5) PH(6) PH(7)
    PH(8) PH(9) PH(10) PH(11) PH(12) PH(13) PH(14) PH(15)
    D1(0) D1(1) D1(2) D1(3)
    C1(0) C1(1) C1(2) C1(3)
    case kc_diag: if constexpr (!FAST) ddiag<R>(v, op, c, thr, gbase, ok()); break;
    PAIRS(D2) PAIRS(C2) PAIRS(SW)
    default: break;
  }
#undef PH
#undef D1
#undef C1
#undef D2
#undef C2
#undef SW
#undef PAIRS
}

__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(saddr), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Shared-memory byte offset of tile index i: 16-byte slots hold 1 (complex128)
// or 2 (complex64) amplitudes; slots are moved by the program's fold (linear
// over GF(2), so the offset of thr | reg(e) is built from per-bit parts).
template <typename V>
struct SmemMap {
  static constexpr int SH = sizeof(V) == 8 ? 1 : 0;  // amplitudes per slot = 2^SH
  __device__ __forceinline__ static uint32_t off(const PartProgram& P, uint32_t i) {
    return (swz(P, i >> SH) << 4) | ((i & ((1u << SH) - 1u)) * uint32_t(sizeof(V)));
  }
};

// Issue the asynchronous copy of one tile into the shared buffer: 16-byte
// chunks, chunk c = t + k*nthr covering tile indices [c*2^SH, (c+1)*2^SH)
// that are contiguous in global memory (tile bit 0 is always global slot 0
// when SH=1); its shared slot is swz(t) ^ swz(k*nthr) (disjoint bits).
template <typename V>
__device__ __forceinline__ void issue_tile_load(const V* __restrict__ sv, uint32_t sbuf,
                                                uint64_t gbase, const uint64_t* __restrict__ gchunk,
                                                const uint32_t* __restrict__ cswz, uint32_t tswz,
                                                uint64_t gt, int nchunk_per_thr, uint64_t size,
                                                uint32_t tile_bytes) {
  const V* base = sv + gbase + gt;
  for (int k = 0; k < nchunk_per_thr; ++k)
    if (HS_IN_BOUNDS(gbase + gt + gchunk[k] + 16 / sizeof(V) <= size &&
                         (tswz ^ cswz[k]) + 16u <= tile_bytes,
                     kBoundsK1))
      cp_async16(sbuf + (tswz ^ cswz[k]), base + gchunk[k]);
  (void)size;
  (void)tile_bytes;
}

// CTA shapes: 2^(m-R) threads.  Complex128 with 16 amplitudes per thread:
// 2^10 tiles in CTAs of 64 threads or 2^11 tiles in CTAs of 128, one tile
// buffer each.  8 amplitudes per thread (R = 3): up to 256 threads.
// Complex64: 2^12 tiles, 256 threads.
constexpr int kThrCache = 8;  // groups whose thread parts are tabulated per launch

template <typename V, int R, bool FULL, bool FAST, bool WIDE>
struct K1Threads {
  static constexpr int value = 256;
  // complex64 with 4x4 ops: room for the coefficient loads
  static constexpr int min_blocks = (R >= 3 && FULL) ? 1 : 2;
};
// complex128, 16 amplitudes per thread: the frequent-op instantiation is held
// to ~100 registers so that five CTAs of 128 (ten of 64) share an SM, the
// general ones get ~168; WIDE (2^12 tiles, 256 threads) is held to 128
template <int R, bool FULL, bool FAST, bool WIDE>
struct K1Threads<double2, R, FULL, FAST, WIDE> {
  static constexpr int value = (WIDE || R < 4) ? 256 : 128;
  static constexpr int min_blocks = WIDE ? (FAST ? 2 : 1) : R >= 4 ? (FAST ? 5 : 3) : 2;
};

template <int R, bool FULL, bool FAST, bool WIDE, typename V>
__global__ void __launch_bounds__(K1Threads<V, R, FULL, FAST, WIDE>::value, K1Threads<V, R, FULL, FAST, WIDE>::min_blocks)
    k1_part(V* __restrict__ sv, const __grid_constant__ PartProgram P) {
  using M = SmemMap<V>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int E = 1 << R;
  const uint32_t t = threadIdx.x;
  const uint32_t nthr = blockDim.x;
  const uint32_t tile_bytes = uint32_t(sizeof(V)) << P.m;
  const uint64_t size = 1ull << P.n;  // amplitudes of the state (bounds checks)
  double2* s_coef = reinterpret_cast<double2*>(smem_raw + tile_bytes);
  uint64_t* s_gchunk = reinterpret_cast<uint64_t*>(s_coef + P.ncoef);
  // chunk c = t + k*nthr; its first tile index is c << SH.  The bits of t and
  // of k*nthr are disjoint, so deposit(c << SH) = deposit(t << SH) + deposit(k*nthr << SH).
  const int nchunk = (1 << P.m) >> M::SH;
  const int per_thr = nchunk / int(nthr);
  // the last group writes its registers straight to global memory: the global
  // offset of each of its register bits and of each thread's thread part
  uint64_t* s_glreg = s_gchunk + per_thr;
  uint64_t* s_glthr = s_glreg + R;
  // the thread part (tile index bits held by this thread) of the first
  // kThrCache groups and its shared-memory offset, the same in every tile
  uint32_t* s_thr = reinterpret_cast<uint32_t*>(s_glthr + nthr);
  uint32_t* s_a0 = s_thr + kThrCache * nthr;
  // shared slot part of chunk k*nthr (the copy of a tile)
  uint32_t* s_cswz = s_a0 + kThrCache * nthr;
  const GroupDesc& GL = P.groups[P.ngroups - 1];
  for (int i = int(t); i < P.ncoef; i += int(nthr)) s_coef[i] = P.coef[i];
  for (int k = int(t); k < per_thr; k += int(nthr)) {
    s_gchunk[k] = deposit(uint64_t(k) * nthr << M::SH, P.tile);
    s_cswz[k] = swz(P, uint32_t(k) * nthr) << 4;
  }
  for (int j = int(t); j < R; j += int(nthr)) s_glreg[j] = deposit(1ull << GL.reg_tbit[j], P.tile);
  // (the last group's lanes run over the lowest free tile bits, so the direct
  // stores coalesce)
  s_glthr[t] = deposit(deposit(t, GL.thr), P.tile);
  for (int g = 0; g < P.ngroups && g < kThrCache; ++g) {
    const uint32_t thr = uint32_t(deposit(t, P.groups[g].thr));
    s_thr[g * nthr + t] = thr;
    s_a0[g * nthr + t] = M::off(P, thr);
  }
  const uint32_t tswz = swz(P, t) << 4;
  __syncthreads();
  const uint64_t gt = deposit(uint64_t(t) << M::SH, P.tile);
  const uint32_t sb0 = uint32_t(__cvta_generic_to_shared(smem_raw));

  uint64_t tile = blockIdx.x;
  // global offset of the tile being processed (computed when its copy is issued)
  uint64_t gbase = tile < P.ntiles ? deposit(tile, P.outer) : 0;
  // the next tile's offset by an addition in the scattered outer bits: with
  // every other bit set the carries run through the gaps, so
  // deposit(t + G) = ((deposit(t) | ~mask) + deposit(G)) & mask
  const uint64_t omask = deposit(P.ntiles - 1, P.outer);
  const uint64_t ostep = deposit(uint64_t(gridDim.x), P.outer);
  if (tile < P.ntiles) issue_tile_load<V>(sv, sb0, gbase, s_gchunk, s_cswz, tswz, gt, per_thr, size, tile_bytes);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  V v[E];
  for (; tile < P.ntiles; tile += gridDim.x) {
    const uint64_t next = tile + gridDim.x;
    const uint64_t gnext = next < P.ntiles ? (((gbase | ~omask) + ostep) & omask) : 0;
    for (int g = 0; g < P.ngroups; ++g) {
      const GroupDesc& G = P.groups[g];
      const bool last = g == P.ngroups - 1;
      const uint32_t thr = g < kThrCache ? s_thr[g * nthr + t] : uint32_t(deposit(t, G.thr));
      // offset of element e: the thread's slot XOR the (warp-uniform) change
      // of e's register bits, whose per-bit parts come from the planner
      const uint32_t a0 = g < kThrCache ? s_a0[g * nthr + t] : M::off(P, thr);
      auto ux = [&](int e) {
        uint32_t d = 0;
#pragma unroll
        for (int j = 0; j < R; ++j)
          if ((e >> j) & 1) d ^= G.dx[j];
        return d;
      };
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (HS_IN_BOUNDS((a0 ^ ux(e)) + sizeof(V) <= tile_bytes, kBoundsK1))
          v[e] = *reinterpret_cast<const V*>(smem_raw + (a0 ^ ux(e)));
      if (last) {
        // every thread holds its registers of the last group: the buffer
        // takes the next tile while this one is finished and stored (one
        // tile buffer per CTA leaves room for more CTAs per SM)
        __syncthreads();
        if (next < P.ntiles) {
          issue_tile_load<V>(sv, sb0, gnext, s_gchunk, s_cswz, tswz, gt, per_thr, size, tile_bytes);
          cp_async_commit();
        }
      }
      // the group's rounds: one rotation per register bit in a fixed order
      // (uniform tests, no dispatch), then the round's other ops
      Deferred dfr;
      for (int r = G.first_round, r_end = G.first_round + G.num_rounds; r < r_end; ++r) {
        const uint64_t rw = P.rounds[r];
        const uint32_t zmask = uint32_t(rw) & 15u;
#define SLOT(J)                                                             \
  if constexpr ((J) < R) {                                                  \
    const uint32_t sw = uint32_t(rw >> (20 + 11 * (J))) & 2047u;            \
    if (sw & 511u) {                                                        \
      const uint32_t ci = (sw & 511u) * 2u;                                 \
      if (!HS_IN_BOUNDS(ci + 2u <= uint32_t(P.ncoef), kBoundsK1)) continue; \
      const double2* c = s_coef + ci;                                       \
      if (zmask & (1u << (J)))                                              \
        rot<R, (J), true>(v, c[0], c[1], sw >> 9);                          \
      else                                                                  \
        rot<R, (J), false>(v, c[0], c[0], sw >> 9);                         \
    }                                                                       \
  }
        SLOT(0) SLOT(1) SLOT(2) SLOT(3)
#undef SLOT
        // the round's sign flips: register mask and at most one condition bit
        if (const uint64_t sgw = P.signs[r]) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint32_t f = uint32_t(sgw >> (16 * q)) & 0xffffu;
            if (f == 0u) break;  // entries are packed from the low end
            const uint32_t kind = (f >> 4) & 3u, pos = (f >> 6) & 63u;
            const uint32_t bit = kind == 1u   ? (thr >> pos) & 1u
                                 : kind == 2u ? uint32_t(gbase >> pos) & 1u
                                              : 1u;
            const uint32_t sm = bit ? 0x80000000u : 0u;
#define SNEG(M) \
  case (M): if constexpr ((M) < (1 << R)) dneg<R, M>(v, sm); break;
            switch (f & 15u) {
              SNEG(1) SNEG(2) SNEG(3) SNEG(4) SNEG(5) SNEG(6) SNEG(7)
              SNEG(8) SNEG(9) SNEG(10) SNEG(11) SNEG(12) SNEG(13) SNEG(14) SNEG(15)
              default: break;
            }
#undef SNEG
          }
        }
        const int k0 = int(rw >> 12) & 255, k1 = k0 + (int(rw >> 4) & 255);
        for (int k = k0; k < k1; ++k) {
          run_op<R, FULL, FAST>(v, P.ops[P.others[k]], s_coef, thr, gbase, dfr, P);
        }
      }
      apply_deferred<R>(v, dfr);
      if (last) {
        // elements in Gray-code order: each address is the previous one plus
        // or minus one register bit's offset (one live pointer)
        V* p = sv + gbase + s_glthr[t];
#pragma unroll
        for (int i = 0; i < E; ++i) {
          const int e = i ^ (i >> 1);
          if (i > 0) {
            const int j = lowest_bit(i);
            if ((e >> j) & 1) p += s_glreg[j]; else p -= s_glreg[j];
          }
          if (HS_IN_BOUNDS(uint64_t(p - sv) < size, kBoundsK1)) __stcs(p, v[e]);
        }
        // the next tile's copies (the only ones in flight) must have landed
        cp_async_wait<0>();
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (HS_IN_BOUNDS((a0 ^ ux(e)) + sizeof(V) <= tile_bytes, kBoundsK1))
            *reinterpret_cast<V*>(smem_raw + (a0 ^ ux(e))) = v[e];
      }
      __syncthreads();
    }
    gbase = gnext;
  }
  cp_async_wait<0>();
}

template <int R, bool FULL, bool FAST, bool WIDE, typename V>
int launch_k1(V* sv, const PartProgram& P, cudaStream_t s) {
  HS_TRY(smem_optin(reinterpret_cast<const void*>(k1_part<R, FULL, FAST, WIDE, V>)));
  const int threads = 1 << (P.m - R);
  const int per_thr = ((1 << P.m) * int(sizeof(V)) / 16) / threads;
  const size_t smem = (sizeof(V) << P.m) + sizeof(double2) * P.ncoef +
                      sizeof(uint64_t) * (per_thr + R + threads) +
                      sizeof(uint32_t) * (2 * kThrCache * threads + per_thr);
  if (smem > 227 * 1024) return set_error(HS_E_UNSUPPORTED, "K1 tile of 2^%d needs %zu B", P.m, smem);
  int per_sm = 0;
  HS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k1_part<R, FULL, FAST, WIDE, V>, threads, smem));
  if (per_sm < 1) return set_error(HS_E_UNSUPPORTED, "K1 tile does not fit an SM (m=%d)", P.m);
  const uint64_t want = uint64_t(device_sms()) * uint64_t(per_sm);
  const int grid = int(P.ntiles < want ? P.ntiles : want);
  k1_part<R, FULL, FAST, WIDE, V><<<grid, threads, smem, s>>>(sv, P);
  HS_CUDA(cudaGetLastError());
  return HS_OK;
}

}  // namespace

// rotations, sign flips, phases and flushes only: the FAST instantiation
bool fast_program(const PartProgram& P) {
  for (int i = 0; i < P.nops; ++i) {
    const int c = P.ops[i].code;
    if (!(c < kc_d1 || (c >= kc_neg && c < kc_diag) || c == kc_flush)) return false;
  }
  return true;
}

template <bool WIDE, typename V>
int launch_shape(V* a, const PartProgram& P, cudaStream_t s) {
  bool full = false;
  for (int i = 0; i < P.nops; ++i) full |= P.ops[i].kind == OP2_DENSE || P.ops[i].kind == OP2_SWAP;
  const int R = P.rbits;
  if (fast_program(P)) {
    switch (R) {
      case 1: return launch_k1<1, false, true, WIDE>(a, P, s);
      case 2: return launch_k1<2, false, true, WIDE>(a, P, s);
      case 3: return launch_k1<3, false, true, WIDE>(a, P, s);
      default: return launch_k1<4, false, true, WIDE>(a, P, s);
    }
  }
  if (full) {
    switch (R) {
      case 1: return launch_k1<1, true, false, WIDE>(a, P, s);
      case 2: return launch_k1<2, true, false, WIDE>(a, P, s);
      case 3: return launch_k1<3, true, false, WIDE>(a, P, s);
      default: return launch_k1<4, true, false, WIDE>(a, P, s);
    }
  }
  switch (R) {
    case 1: return launch_k1<1, false, false, WIDE>(a, P, s);
    case 2: return launch_k1<2, false, false, WIDE>(a, P, s);
    case 3: return launch_k1<3, false, false, WIDE>(a, P, s);
    default: return launch_k1<4, false, false, WIDE>(a, P, s);
  }
}

// complex128 programs whose CTAs exceed 128 threads (2^12 tiles at 16
// amplitudes per thread) run the WIDE instantiation; complex64 has one shape
template <typename V>
int launch_typed(V* a, const PartProgram& P, cudaStream_t s) {
  if (sizeof(V) == 16 && (P.m - P.rbits) > 7) return launch_shape<true>(a, P, s);
  return launch_shape<false>(a, P, s);
}

#ifdef HS_BOUNDS
HS_BOUNDS_TAKE(bounds_take_part)
#endif

int launch_part(void* amp, int dtype, const PartProgram& P, cudaStream_t s) {
  if (P.ngroups < 1 || P.nops < 1) return HS_OK;
  if (dtype == HS_DTYPE_C128) return launch_typed(static_cast<double2*>(amp), P, s);
  return launch_typed(static_cast<float2*>(amp), P, s);
}

}  // namespace hisv
