// Host-side gate construction: the coefficient arithmetic of the reference's
// BasicGates constructors (basic_gates.hpp:99-1408, scalar branches),
// restated over std::complex<double>, and the lowering of each gate to a 2x2
// or 4x4 matrix that the K1 kernel applies.
#include <cmath>
#include <cstring>

#include "internal.h"

namespace hisv {
namespace {

constexpr double kPi = 3.14159265358979323846;        // types.hpp:19
constexpr double kPiBy2 = 1.57079632679489661923;     // types.hpp:20
constexpr double kInvSqrt2 = 0.707106781186547524401;  // types.hpp:23
const cplx kI(0.0, 1.0);

cplx param(const hs_gate& g, int i) { return cplx(g.params[2 * i], g.params[2 * i + 1]); }

// 2x2 matrices in row-major order, v_out[r] = sum_c M[r][c] v_in[c].
void set2(cplx* m, cplx a, cplx b, cplx c, cplx d) {
  m[0] = a;
  m[1] = b;
  m[2] = c;
  m[3] = d;
}

// RX(theta): cos(theta/2), i sin(theta/2) -> [[c, -is], [-is, c]] (basic_gates.hpp:343-363)
void rx(cplx th, cplx* m) {
  cplx c = std::cos(th / cplx(2)), is = kI * std::sin(th / cplx(2));
  set2(m, c, -is, -is, c);
}
// RY(theta) -> [[c, -s], [s, c]] (basic_gates.hpp:401-422)
void ry(cplx th, cplx* m) {
  cplx c = std::cos(th / cplx(2)), s = std::sin(th / cplx(2));
  set2(m, c, -s, s, c);
}
// RI(theta) -> exp(-i theta/2) * I (basic_gates.hpp:460-478)
void ri(cplx th, cplx* m) {
  cplx e = std::exp(-kI * th / cplx(2));
  set2(m, e, 0.0, 0.0, e);
}
// RZ(theta) == U1 -> diag(exp(-i theta/2), exp(i theta/2)) (basic_gates.hpp:515-535,571)
void rz(cplx th, cplx* m) {
  set2(m, std::exp(-kI * th / cplx(2)), 0.0, 0.0, std::exp(kI * th / cplx(2)));
}
// *Frac(numerator, power): -pi * numerator / 2^(power-1) with unsigned
// arithmetic (basic_gates.hpp:732-733; power-1 wraps for power == 0).
double frac_angle(uint32_t num, uint32_t power) {
  return -kPi * double(num) / std::pow(2.0, double(uint32_t(power - 1u)));
}
void mul2(const cplx* a, const cplx* b, cplx* out) {  // out = a * b
  cplx r[4];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) r[2 * i + j] = a[2 * i] * b[j] + a[2 * i + 1] * b[2 + j];
  std::memcpy(out, r, sizeof(r));
}

// 4-amplitude register for composing the 2-target sequences; index
// i = 2*b(target0) + b(target1), so "+ (1 << slots[1])" is +1 and
// "+ (1 << slots[0])" is +2 (basic_gates.hpp:580-583).
struct Quad {
  cplx w[4];
  void one(const cplx* m, int base, int stride) {
    cplx a = w[base], b = w[base + stride];
    w[base] = m[0] * a + m[1] * b;
    w[base + stride] = m[2] * a + m[3] * b;
  }
  void swap(int a, int b) { std::swap(w[a], w[b]); }
};

// Compose the 4x4 matrix of a 2-target gate by running its reference sequence
// on each basis vector.  `seq` receives a Quad and mutates it.
template <typename F>
void compose4(cplx* m, F&& seq) {
  for (int c = 0; c < 4; ++c) {
    Quad q;
    for (int r = 0; r < 4; ++r) q.w[r] = (r == c) ? cplx(1.0) : cplx(0.0);
    seq(q);
    for (int r = 0; r < 4; ++r) m[4 * r + c] = q.w[r];
  }
}

}  // namespace

int lower_gate(const hs_gate& g, int num_qubits, LoweredGate* out) {
  LoweredGate L;
  if (g.num_controls < 0 || g.num_controls > HS_MAX_CONTROLS)
    return set_error(HS_E_INVALID, "gate has %d controls (max %d)", g.num_controls,
                     HS_MAX_CONTROLS);
  if (g.num_targets < 1 || g.num_targets > HS_MAX_TARGETS)
    return set_error(HS_E_INVALID, "gate has %d targets", g.num_targets);
  const bool two = g.type == HS_GATE_SWAP || g.type == HS_GATE_C2 || g.type == HS_GATE_RXX ||
                   g.type == HS_GATE_RYY || g.type == HS_GATE_RZZ;
  const int want = two ? 2 : 1;
  if (g.num_targets != want)
    return set_error(HS_E_INVALID, "gate type %d takes %d target(s), got %d", g.type, want,
                     g.num_targets);
  // every qubit in range and distinct (state_vector.hpp:413-426)
  int seen[64] = {0};
  for (int i = 0; i < g.num_targets + g.num_controls; ++i) {
    int q = i < g.num_targets ? g.targets[i] : g.controls[i - g.num_targets];
    if (q < 0 || q >= num_qubits)
      return set_error(HS_E_INVALID, "operation on an unallocated qubit %d", q);
    if (seen[q]++) return set_error(HS_E_INVALID, "qubit %d used twice by one gate", q);
  }
  L.nt = want;
  for (int i = 0; i < want; ++i) L.targets[i] = g.targets[i];
  L.nc = g.num_controls;
  for (int i = 0; i < g.num_controls; ++i) L.controls[i] = g.controls[i];
  cplx* m = L.m;
  const cplx th = param(g, 0);
  switch (g.type) {
    case HS_GATE_I: L.nt = 0; break;                                   // no-op (:99-106)
    case HS_GATE_X: set2(m, 0.0, 1.0, 1.0, 0.0); break;                // :120
    case HS_GATE_Y: set2(m, 0.0, -kI, kI, 0.0); break;                 // :142-145
    case HS_GATE_Z: set2(m, 1.0, 0.0, 0.0, -1.0); break;               // :230
    case HS_GATE_H: set2(m, kInvSqrt2, kInvSqrt2, kInvSqrt2, -kInvSqrt2); break;  // :186-189
    case HS_GATE_S: set2(m, 1.0, 0.0, 0.0, kI); break;                 // :262
    case HS_GATE_T: set2(m, 1.0, 0.0, 0.0, std::sqrt(kI)); break;      // :297
    case HS_GATE_SDG: set2(m, 1.0, 0.0, 0.0, -kI); break;              // :1379
    case HS_GATE_TDG: set2(m, 1.0, 0.0, 0.0, kInvSqrt2 * (1.0 - kI)); break;  // :1338
    case HS_GATE_RX: rx(th, m); break;
    case HS_GATE_RY: ry(th, m); break;
    case HS_GATE_RI: ri(th, m); break;
    case HS_GATE_RZ:
    case HS_GATE_U1: rz(th, m); break;
    case HS_GATE_R1: {  // rz_{theta} then ri_{-theta} (basic_gates.hpp:718-724)
      cplx a[4], b[4];
      rz(th, a);
      ri(-th, b);
      mul2(b, a, m);
      break;
    }
    case HS_GATE_RXFRAC: rx(frac_angle(g.frac_num, g.frac_pow), m); break;
    case HS_GATE_RYFRAC: ry(frac_angle(g.frac_num, g.frac_pow), m); break;
    case HS_GATE_RZFRAC: rz(frac_angle(g.frac_num, g.frac_pow), m); break;
    case HS_GATE_RIFRAC: ri(frac_angle(g.frac_num, g.frac_pow), m); break;
    case HS_GATE_R1FRAC: {  // rzf_{-numerator, power+1}, rif_{numerator, power+1} (:785-791)
      cplx a[4], b[4];
      rz(frac_angle(0u - g.frac_num, g.frac_pow + 1u), a);
      ri(frac_angle(g.frac_num, g.frac_pow + 1u), b);
      mul2(b, a, m);
      break;
    }
    case HS_GATE_C1: set2(m, param(g, 0), param(g, 1), param(g, 2), param(g, 3)); break;
    case HS_GATE_U2: {  // basic_gates.hpp:1025-1029
      cplx phi = param(g, 0), lam = param(g, 1);
      set2(m, cplx(kInvSqrt2, 0.0), -kInvSqrt2 * (std::cos(lam) + kI * std::sin(lam)),
           kInvSqrt2 * (std::cos(phi) + kI * std::sin(phi)),
           kInvSqrt2 * (std::cos(phi + lam) + kI * std::sin(phi + lam)));
      break;
    }
    case HS_GATE_U3: {  // basic_gates.hpp:1044-1052
      cplx t = param(g, 0), p = param(g, 1), l = param(g, 2);
      cplx c = std::cos(t / 2.0), s = std::sin(t / 2.0);
      set2(m, c * std::cos((-p - l) / 2.0) + kI * c * std::sin((-p - l) / 2.0),
           -s * std::cos((-p + l) / 2.0) + kI * -s * std::sin((-p + l) / 2.0),
           s * std::cos((p - l) / 2.0) + kI * s * std::sin((p - l) / 2.0),
           c * std::cos((p + l) / 2.0) + kI * c * std::sin((p + l) / 2.0));
      break;
    }
    case HS_GATE_SWAP:  // swap base[1<<s0] <-> base[1<<s1]: i=2 <-> i=1 (:804-805)
      compose4(m, [](Quad& q) { q.swap(2, 1); });
      break;
    case HS_GATE_C2: {  // the constructor copies c_r0 across row r (:972-987)
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) m[4 * r + c] = param(g, 4 * r);
      break;
    }
    case HS_GATE_RXX: {  // H/H/H(x2 on one half)/swap/RZ/swap/H/H sequence (:587-599)
      cplx h[4], z[4];
      set2(h, kInvSqrt2, kInvSqrt2, kInvSqrt2, -kInvSqrt2);
      rz(th, z);
      compose4(m, [&](Quad& q) {
        q.one(h, 0, 2);
        q.one(h, 1, 2);
        q.one(h, 0, 1);
        q.one(h, 2, 1);
        q.one(h, 0, 1);
        q.swap(2, 3);
        q.one(z, 0, 1);
        q.one(z, 2, 1);
        q.swap(2, 3);
        q.one(h, 0, 1);
        q.one(h, 2, 1);
        q.one(h, 0, 2);
        q.one(h, 1, 2);
      });
      break;
    }
    case HS_GATE_RYY: {  // rx(pi/2) x4, swap, rz, swap, rx(-pi/2) x4 (:1108-1120)
      cplx a[4], b[4], z[4];
      rx(cplx(kPiBy2), a);
      rx(cplx(-kPiBy2), b);
      rz(th, z);
      compose4(m, [&](Quad& q) {
        q.one(a, 0, 2);
        q.one(a, 1, 2);
        q.one(a, 0, 1);
        q.one(a, 2, 1);
        q.swap(2, 3);
        q.one(z, 0, 1);
        q.one(z, 2, 1);
        q.swap(2, 3);
        q.one(b, 0, 2);
        q.one(b, 1, 2);
        q.one(b, 0, 1);
        q.one(b, 2, 1);
      });
      break;
    }
    case HS_GATE_RZZ: {  // swap, rz on target1 (both halves), swap (:1249-1252)
      cplx z[4];
      rz(th, z);
      compose4(m, [&](Quad& q) {
        q.swap(2, 3);
        q.one(z, 0, 1);
        q.one(z, 2, 1);
        q.swap(2, 3);
      });
      break;
    }
    case HS_GATE_ALLOC:
    case HS_GATE_FREE:
      // The factories reach NOT_IMPLEMENTED for these (basic_gates.hpp:1573-1574).
      return set_error(HS_E_UNSUPPORTED, "ALLOC/FREE gates are not constructible");
    default:
      return set_error(HS_E_INVALID, "invalid gate type %d", g.type);
  }
  *out = L;
  return HS_OK;
}

}  // namespace hisv
