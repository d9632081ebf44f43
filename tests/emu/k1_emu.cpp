// Host emulator of K1 programs -- TEST INFRASTRUCTURE ONLY.
//
// Runs the library's own planner (plan.cpp, gatemath.cpp, compiled into this
// test library) and executes the programs it produces on a host array the way
// the K1 kernel does: per tile, the cp.async chunk placement into an
// XOR-swizzled shared buffer, per register group the loads at
// (thread slot ^ planner offset), the op codes on 2^R registers, the stores
// back (or, for the last group, the Gray-code walk of direct global stores).
// The CPU tests compare its result with the oracle, which checks the planner's
// gate rewriting and the kernel's addressing without a GPU.  Nothing in the
// product loads this file.
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <algorithm>
#include <vector>

#include "internal.h"

namespace hisv {
static char g_err[512];
int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}
static int g_rbits = 4;
int k1_reg_bits(int) { return g_rbits; }
int current_tile_hint() { return 0; }
}  // namespace hisv

using namespace hisv;
using C = std::complex<double>;

namespace {

uint64_t deposit(uint64_t x, const Runs& r) {
  uint64_t out = 0;
  for (int i = 0; i < r.n; ++i) out |= ((x >> r.src[i]) & ((1ull << r.len[i]) - 1ull)) << r.dst[i];
  return out;
}
uint32_t swz(const PartProgram& P, uint32_t s) {
  uint32_t r = s;
  for (int k = 0; (s >> k) != 0; ++k)
    if ((s >> k) & 1u) r ^= P.fold[k];
  return r;
}
int lowest_bit(int e) { return __builtin_ctz(unsigned(e)); }
C cc(const double2& d) { return C(d.x, d.y); }

struct Emu {
  const PartProgram& P;
  int R, E, SH, ab;
  std::vector<unsigned char> buf;
  uint32_t off(uint32_t i) const {
    return (swz(P, i >> SH) << 4) | ((i & ((1u << SH) - 1u)) * uint32_t(ab));
  }
  C ld(uint32_t o) const {
    if (ab == 16) {
      double d[2];
      std::memcpy(d, &buf[o], 16);
      return C(d[0], d[1]);
    }
    float f[2];
    std::memcpy(f, &buf[o], 8);
    return C(f[0], f[1]);
  }
  void st(uint32_t o, C x) {
    if (ab == 16) {
      double d[2] = {x.real(), x.imag()};
      std::memcpy(&buf[o], d, 16);
    } else {
      float f[2] = {float(x.real()), float(x.imag())};
      std::memcpy(&buf[o], f, 8);
    }
  }
};

C rnd(C x, int ab) { return ab == 16 ? x : C(float(x.real()), float(x.imag())); }

// the kernel's op semantics on a thread's registers (complex64 rounds after each op)
void run_op(std::vector<C>& v, int R, const PartProgram& P, const DevOp& op, const double2* c,
            uint32_t thr, uint64_t gbase, uint32_t& dsign, int ab) {
  const int E = 1 << R;
  const bool ok = ((thr & op.cthr) == op.cthr) && ((gbase & op.couter) == op.couter);
  const int code = op.code;
  auto pairs = [&](int J, auto&& f) {
    for (int e0 = 0; e0 < E; ++e0)
      if (!((e0 >> J) & 1)) f(e0, e0 | (1 << J));
  };
  if (code < kc_d1) {
    const bool z = code < kc_y;
    const int J = code % 4;
    // phase shears on B, then the real shears of form op.form
    const double t = c[0].x, s = c[0].y, tz = z ? c[1].x : 0.0, sz = z ? c[1].y : 0.0;
    const bool first = !(op.form & 2u), third = !(op.form & 1u);
    pairs(J, [&](int e0, int e1) {
      double ax = v[e0].real(), ay = v[e0].imag(), bx = v[e1].real(), by = v[e1].imag();
      if (z) {
        bx = std::fma(-tz, by, bx);
        by = std::fma(sz, bx, by);
        bx = std::fma(-tz, by, bx);
      }
      if (first) {
        ax = std::fma(t, bx, ax);
        ay = std::fma(t, by, ay);
      }
      bx = std::fma(s, ax, bx);
      by = std::fma(s, ay, by);
      if (third) {
        ax = std::fma(t, bx, ax);
        ay = std::fma(t, by, ay);
      }
      v[e0] = C(ax, ay);
      v[e1] = C(bx, by);
    });
  } else if (code < kc_neg) {
    const bool ctl = code >= kc_c1;
    const int J = (code - kc_d1) % 4;
    const uint32_t creg = ctl ? op.creg : 0u;
    if (!ctl || ok)
      pairs(J, [&](int e0, int e1) {
        if ((uint32_t(e0) & creg) != creg) return;
        const C a = v[e0], b = v[e1];
        v[e0] = cc(c[0]) * a + cc(c[1]) * b;
        v[e1] = cc(c[2]) * a + cc(c[3]) * b;
      });
  } else if (code < kc_ph) {
    const int M = code - kc_neg;
    if (M == 0) {
      if (ok) dsign ^= 1u;
    } else if (ok) {
      for (int e = 0; e < E; ++e)
        if ((e & M) == M) v[e] = -v[e];
    }
  } else if (code < kc_diag) {
    const int M = code - kc_ph;
    if (ok)
      for (int e = 0; e < E; ++e)
        if ((e & M) == M) v[e] *= cc(c[0]);
  } else if (code == kc_diag) {
    auto fixed = [&](uint8_t w, uint8_t pos) -> uint32_t {
      return w == TW_THR ? ((thr >> pos) & 1u) : w == TW_OUT ? uint32_t((gbase >> pos) & 1ull) : 0u;
    };
    const uint32_t creg = ok ? uint32_t(op.creg) : 0xffffffffu;
    for (int e = 0; e < E; ++e) {
      if ((uint32_t(e) & creg) != creg) continue;
      const uint32_t q0 = op.t0w == TW_REG ? ((uint32_t(e) >> op.t0p) & 1u) : fixed(op.t0w, op.t0p);
      const uint32_t q1 =
          op.t1w == TW_REG ? ((uint32_t(e) >> op.t1p) & 1u) : fixed(op.t1w, op.t1p);
      v[e] *= cc(c[q0 | (q1 << 1)]);
    }
  } else if (code < kc_flush) {
    static const int pj[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
    const int kind = (code - kc_d2) / 6, pi = (code - kc_d2) % 6;
    const int JA = pj[pi][0], JB = pj[pi][1];
    const bool ctl = kind >= 1;
    const uint32_t creg = ctl ? op.creg : 0u;
    if (!ctl || ok)
      for (int x = 0; x < E; ++x) {
        if (((x >> JA) & 1) || ((x >> JB) & 1)) continue;
        if ((uint32_t(x) & creg) != creg) continue;
        const int e[4] = {x, x | (1 << JA), x | (1 << JB), x | (1 << JA) | (1 << JB)};
        if (kind == 2) {
          std::swap(v[e[1]], v[e[2]]);
        } else {
          const C a[4] = {v[e[0]], v[e[1]], v[e[2]], v[e[3]]};
          for (int r = 0; r < 4; ++r) {
            C s = 0;
            for (int k = 0; k < 4; ++k) s += cc(c[4 * r + k]) * a[k];
            v[e[r]] = s;
          }
        }
      }
  } else if (code == kc_flush) {
    C f = cc(c[0]);
    for (int i = 0; i < op.fl_n; ++i) {
      const uint32_t w = P.flw[op.fl_first + i], pos = P.flp[op.fl_first + i];
      const uint32_t bit = w == TW_THR ? (thr >> pos) & 1u : uint32_t(gbase >> pos) & 1u;
      if (bit) f = cc(c[1 + i]) * f;
    }
    for (int e = 0; e < E; ++e) v[e] *= f;
  }
  for (int e = 0; e < E; ++e) v[e] = rnd(v[e], ab);
}

int64_t wave_total = 0, wave_ideal = 0;

void run_program(const PartProgram& P, int ab, std::vector<C>& sv) {
  const int R = P.rbits, E = 1 << R, m = P.m;
  const int nthr = 1 << (m - R);
  Emu em{P, R, E, ab == 8 ? 1 : 0, ab, {}};
  em.buf.assign(size_t(ab) << m, 0);
  const int SH = em.SH;
  const int nchunk = (1 << m) >> SH, per_thr = nchunk / nthr;
  const GroupDesc& GL = P.groups[P.ngroups - 1];
  std::vector<uint64_t> glreg(R), glthr(nthr), gchunk(per_thr);
  for (int k = 0; k < per_thr; ++k) gchunk[k] = deposit(uint64_t(k) * nthr << SH, P.tile);
  for (int j = 0; j < R; ++j) glreg[j] = deposit(1ull << GL.reg_tbit[j], P.tile);
  for (int t = 0; t < nthr; ++t) glthr[t] = deposit(deposit(t, GL.thr), P.tile);
  std::vector<std::vector<C>> regs(nthr, std::vector<C>(E));
  for (uint64_t tile = 0; tile < P.ntiles; ++tile) {
    const uint64_t gbase = deposit(tile, P.outer);
    // cp.async placement: chunk c of thread t (c = t + k*nthr) holds tile
    // indices [c << SH, (c + 1) << SH), contiguous from global gbase + gt + gchunk[k]
    for (int t = 0; t < nthr; ++t) {
      const uint64_t gt = deposit(uint64_t(t) << SH, P.tile);
      for (int k = 0; k < per_thr; ++k) {
        const uint32_t cix = uint32_t(t + k * nthr);
        const uint64_t g = gbase + gt + gchunk[k];
        for (int s = 0; s < (1 << SH); ++s) em.st((swz(P, cix) << 4) + s * ab, sv[g + s]);
      }
    }
    if (tile == 0)
      for (int g = 0; g < P.ngroups; ++g) {
        const GroupDesc& G = P.groups[g];
        const int plen = ab == 16 ? 8 : 16;
        for (int t0 = 0; t0 < nthr; t0 += plen) {
          int cnt[16] = {0};
          int worst = 0;
          uint32_t halves = 0;
          for (int t = t0; t < t0 + plen && t < nthr; ++t) {
            const uint32_t a = em.off(uint32_t(deposit(t, G.thr)));
            const int key = ab == 16 ? int((a >> 4) & 7u) : int((a >> 3) & 15u);
            worst = std::max(worst, ++cnt[key]);
            halves |= 1u << ((a >> 3) & 1u);
          }
          wave_total += worst;
          // lower bound: 8-byte lanes that all sit in the same half of their
          // 16-byte slots reach only 8 distinct bank pairs
          wave_ideal += (ab == 8 && halves != 3u) ? 2 : 1;
        }
      }
    for (int g = 0; g < P.ngroups; ++g) {
      const GroupDesc& G = P.groups[g];
      const bool last = g == P.ngroups - 1;
      for (int t = 0; t < nthr; ++t) {
        const uint32_t thr = uint32_t(deposit(t, G.thr));
        const uint32_t a0 = em.off(thr);
        auto ux = [&](int e) {
          uint32_t d = 0;
          for (int j = 0; j < R; ++j)
            if ((e >> j) & 1) d ^= G.dx[j];
          return d;
        };
        std::vector<C>& v = regs[t];
        for (int e = 0; e < E; ++e) v[e] = em.ld(a0 ^ ux(e));
        uint32_t dsign = 0;
        for (int r = G.first_round; r < G.first_round + G.num_rounds; ++r) {
          const uint64_t rw = P.rounds[r];
          const uint32_t zmask = uint32_t(rw) & 15u;
          for (int j = 0; j < R; ++j) {
            const uint32_t sw = uint32_t(rw >> (20 + 11 * j)) & 2047u;
            if (!(sw & 511u)) continue;
            DevOp rop;
            std::memset(&rop, 0, sizeof(rop));
            rop.code = uint8_t((((zmask >> j) & 1) ? kc_zy : kc_y) + j);
            rop.form = sw >> 9;
            const uint32_t ci = (sw & 511u) * 2u;
            if (ci + 2 > uint32_t(P.ncoef)) throw std::runtime_error("rotation coefficients out of range");
            run_op(v, R, P, rop, P.coef + ci, thr, gbase, dsign, ab);
          }
          // the round's sign word: register mask M, at most one condition bit
          for (int q = 0; q < 4; ++q) {
            const uint32_t f = uint32_t(P.signs[r] >> (16 * q)) & 0xffffu;
            if (!f) break;
            const uint32_t kind = (f >> 4) & 3u, pos = (f >> 6) & 63u;
            const uint32_t bit = kind == 1u ? (thr >> pos) & 1u
                                 : kind == 2u ? uint32_t(gbase >> pos) & 1u : 1u;
            const int M = int(f & 15u);
            if (bit)
              for (int e = 0; e < E; ++e)
                if ((e & M) == M) v[e] = -v[e];
          }
          const int k0 = int(rw >> 12) & 255, k1 = k0 + (int(rw >> 4) & 255);
          for (int k = k0; k < k1; ++k) {
            const DevOp& op = P.ops[P.others[k]];
            run_op(v, R, P, op, P.coef + op.coef, thr, gbase, dsign, ab);
          }
        }
        if (dsign)
          for (int e = 0; e < E; ++e) v[e] = -v[e];
        if (last) {
          uint64_t p = gbase + glthr[t];
          for (int i = 0; i < E; ++i) {
            const int e = i ^ (i >> 1);
            if (i > 0) {
              const int j = lowest_bit(i);
              if ((e >> j) & 1) p += glreg[j]; else p -= glreg[j];
            }
            sv[p] = v[e];
          }
        } else {
          for (int e = 0; e < E; ++e) em.st(a0 ^ ux(e), v[e]);
        }
      }
    }
  }
}

}  // namespace

extern "C" {

const char* emu_last_error() { return g_err; }

// Lower, plan (frames carried across parts, flushed by the last one; with
// per_part != 0 every part is planned on its own and flushed) and execute on
// `amps` (2^n interleaved complex128, in/out).  dtype HS_DTYPE_C64 rounds the
// amplitudes to complex64 as the kernel would.  stats: {passes, groups, ops,
// rotation ops, max tile bits, rounds, shared-memory wavefronts of the group
// loads of one tile (summed over programs), the conflict-free count, rotation
// ops in a two-shear form}.
int emu_parts_run(int n, int dtype, const hs_gate* gates, const int32_t* offs, int nparts,
                  int rbits, int tile_hint, int per_part, double* amps, int32_t* stats) {
  g_rbits = rbits;
  std::vector<C> sv(size_t(1) << n);
  for (size_t i = 0; i < sv.size(); ++i) sv[i] = rnd(C(amps[2 * i], amps[2 * i + 1]), amp_bytes(dtype));
  std::vector<int> q2s(n);
  for (int q = 0; q < n; ++q) q2s[q] = q;
  Frames fr;
  fr.reset(n);
  int32_t st[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  wave_total = wave_ideal = 0;
  for (int p = 0; p < nparts; ++p) {
    std::vector<LoweredGate> lg(offs[p + 1] - offs[p]);
    for (int i = offs[p]; i < offs[p + 1]; ++i) {
      int rc = lower_gate(gates[i], n, &lg[i - offs[p]]);
      if (rc != HS_OK) return rc;
    }
    std::vector<PartProgram> progs;
    int rc = per_part ? plan_part(n, q2s, lg, tile_hint, dtype, &progs)
                      : plan_gates(n, q2s, lg, &fr, p == nparts - 1, tile_hint, dtype, &progs);
    if (rc != HS_OK) return rc;
    for (const auto& P : progs) {
      if (P.ngroups < 1 || P.nops < 1) continue;
      try {
        run_program(P, int(amp_bytes(dtype)), sv);
      } catch (const std::exception& e) {
        std::snprintf(g_err, sizeof(g_err), "%s", e.what());
        return HS_E_INVALID;
      }
      st[0] += 1;
      st[1] += P.ngroups;
      st[2] += P.nops;
      for (int i = 0; i < P.nops; ++i) {
        st[3] += P.ops[i].kind == OP1_ROT;
        st[8] += P.ops[i].kind == OP1_ROT && P.ops[i].form != 0;
      }
      st[4] = std::max(st[4], P.m);
      st[5] += P.nrounds;
    }
  }
  for (size_t i = 0; i < sv.size(); ++i) {
    amps[2 * i] = sv[i].real();
    amps[2 * i + 1] = sv[i].imag();
  }
  st[6] = int32_t(wave_total);
  st[7] = int32_t(wave_ideal);
  if (stats) std::memcpy(stats, st, sizeof(st));
  return HS_OK;
}
}
