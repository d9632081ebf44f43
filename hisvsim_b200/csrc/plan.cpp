// Host planner for K1: turns a gate sequence (one part, or the parts of one
// call) into tile programs.
//
// The reference runs a part by gathering, for each assignment of the outer
// qubits, the 2^k amplitudes of the part's qubits into an inner state vector,
// applying every gate there and scattering back (execute.hpp:318-470,
// state_vector.hpp:617-673; the loop nest of loop.hpp:468-962).  Here a tile
// is the same gather, widened by the three lowest slots so that every global
// access moves whole 128-byte lines of complex128 (the GPU form of opt_slots,
// execute.hpp:184-199).
// Each tile is held by one CTA: 2^R amplitudes per thread in registers, where
// R tile bits are "register bits".  A non-diagonal gate's targets must be
// register bits; consecutive gates whose targets fit in R bits form a group,
// and between groups the tile is exchanged through shared memory so that the
// next group's targets become register bits.  Diagonal gates (Z, S, T, RZ,
// controlled phases, RZZ, ...) only scale amplitudes by a phase chosen from
// index bits, so they run in any layout and their qubits need not be in the
// tile at all.  Controls are index predicates wherever their bits are, as
// control_offset is in StateVector::apply (state_vector.hpp:410-417).
//
// Before that, the gate sequence is rewritten (Frames, internal.h): an
// uncontrolled one-qubit gate U on qubit q, preceded by the pending diagonal
// diag(1, r_q), is factored (Z-Y-Z Euler form) as
//     U diag(1, r_q) = diag(a0, a1) * RY(theta) * diag(1, e^{i beta}),
// with |beta| <= pi/2 (otherwise Z = diag(1, -1) moves to the left factor:
// RY(theta) Z = Z RY(-theta)).  RY(theta) diag(1, e^{i beta}) is applied as
// exact plane rotations, each written as three in-place shears (x -= t y;
// y += s x; x -= t y, with t = tan(angle/2), s = sin(angle)): the phase turns
// the (re, im) plane of the pair's second amplitude by beta, RY the (first,
// second) plane of the pair's real and of its imaginary parts by theta/2.
// 9 FP64 FMA per amplitude pair (6 without the phase), every one updating a
// register in place, so the kernel's op dispatch needs no register moves.
// For complex128 states the RY part is instead written, when cos(theta/2) >=
// 0.4, as two shears and a real diagonal scale that joins the pending factor
// (factor_rotation): 7 FMA per pair.  diag(a0, a1) (times that scale) joins
// the pending diagonal, which commutes with every diagonal gate (CZ, phases)
// and is absorbed by the next one-qubit gate on q.
// Diagonal one-qubit gates (S, T, RZ, ...) only update the pending diagonal.
// Whatever is pending at the end of a call is applied by one flush op.  The
// result is the reference's state up to rounding.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <functional>

#include "internal.h"

namespace hisv {

bool Frames::identity() const {
  if (G != cplx(1.0, 0.0)) return false;
  for (const auto& x : r)
    if (x != cplx(1.0, 0.0)) return false;
  return true;
}

namespace {

void build_runs(const std::vector<int>& dst_of_src, Runs* r) {
  // dst_of_src[i] = destination bit of source bit i; merge consecutive bits.
  r->n = 0;
  int i = 0;
  const int len = int(dst_of_src.size());
  while (i < len) {
    int j = i + 1;
    while (j < len && dst_of_src[j] == dst_of_src[j - 1] + 1) ++j;
    r->src[r->n] = uint8_t(i);
    r->len[r->n] = uint8_t(j - i);
    r->dst[r->n] = uint8_t(dst_of_src[i]);
    ++r->n;
    i = j;
  }
}

bool exact(cplx a, double re, double im = 0.0) { return a.real() == re && a.imag() == im; }

bool is_diagonal(const LoweredGate& g) {
  const int d = g.nt == 1 ? 2 : 4;
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c)
      if (r != c && !exact(g.m[d * r + c], 0)) return false;
  return true;
}

// ---- the factored rotation ---------------------------------------------------
// Applied to the stored pair (A, B) = (amplitude with the qubit 0, with it 1):
// first the phase b1 = e^{i beta} on B as the three shears of its (re, im)
// plane (tan(beta/2), sin(beta)), then real shears on the (A.re, B.re) and
// (A.im, B.im) planes with one coefficient pair (t, s):
//   form 0:  A += t B;  B += s A;  A += t B
//   form 1:  A += t B;  B += s A
//   form 2:             B += s A;  A += t B
// and the left diagonal diag(g0, g1) joins the pending factors.
struct Rot {
  bool has_z;        // phase part present (beta != 0)
  double tz, sz;     // shears of the phase: tan(beta/2), sin(beta)
  int form;
  double t, s;
  cplx g0, g1;       // left diagonal
};

// Two-shear forms are used when cos(theta/2) >= kShearPivot: their
// coefficients stay below ~3 and the pending scale of a qubit within
// [kShearPivot^2, kShearPivot^-2].
constexpr double kShearPivot = 0.4;

// W = U diag(1, r): U unitary, r the qubit's pending factor, so W's first
// column is a unit vector and its second |r| = rho times one.  With
// Wn = W diag(1, 1/rho) = diag(a0, a1) RY diag(1, b1) (Z-Y-Z; RY = [[c, -sg],
// [sg, c]], c = cos(theta/2) >= 0, |arg b1| <= pi/2):
//   W = diag(a0, a1) M diag(1, b1),  M = RY diag(1, rho) = [[c, -sg rho], [sg, c rho]],
// and M is written as shears times a left diagonal:
//   form 0 (exact rotation): M = diag(1, rho) S3, S3 the three shears with
//     t = -rho tan(theta/4), s = sg / rho (rho never changes);
//   form 1 (scaled, rho <= 1): M = diag(c, rho / c) [[1, 0], [s, 1]] [[1, t], [0, 1]],
//     t = -sg rho / c, s = sg c / rho (rho grows to rho / c^2);
//   form 2 (scaled, rho > 1): M = diag(1 / c, c rho) [[1, t], [0, 1]] [[1, 0], [s, 1]],
//     s = sg / (c rho), t = -sg c rho (rho shrinks to c^2 rho).
// Forms 1 and 2 take 4 FMA per pair instead of 6 and leave a real scale on
// the qubit's two values, which complex128 frames carry (`scaled`);
// complex64 states keep form 0.  False when W is not of the form above to
// 1e-12 (custom C1 matrices need not be).
bool factor_rotation(const cplx* W, bool scaled, Rot* R) {
  const double c = std::abs(W[0]), s = std::abs(W[2]);
  const double rho = std::hypot(std::abs(W[1]), std::abs(W[3]));
  const double tol = 1e-12;
  if (!(rho > 0.0) || !std::isfinite(rho)) return false;
  const cplx w1 = W[1] / rho, w3 = W[3] / rho;
  const double c1 = std::abs(w3), s1 = std::abs(w1);
  if (std::fabs(c * c + s * s - 1.0) > tol || std::fabs(c1 * c1 + s1 * s1 - 1.0) > tol ||
      std::abs(std::conj(W[0]) * w1 + std::conj(W[2]) * w3) > tol)
    return false;
  cplx a0, a1, b1;
  double cc = c, ss = s;
  if (c > 0.0 && s > 0.0) {
    a0 = W[0] / c;
    a1 = W[2] / s;
    b1 = c >= s ? w3 / (a1 * c) : -w1 / (a0 * s);
    b1 /= std::abs(b1);
  } else if (c == 0.0) {  // anti-diagonal
    a0 = -w1;
    a1 = W[2];
    b1 = 1.0;
    cc = 0.0;
    ss = 1.0;
  } else {
    return false;  // diagonal: handled by the caller
  }
  // the norms of the rows are 1 to 1e-12; keep the phases unit-modulus
  a0 /= std::abs(a0);
  a1 /= std::abs(a1);
  const double nrm = std::hypot(cc, ss);
  cc /= nrm;
  ss /= nrm;
  double sign = 1.0;
  if (b1.real() < 0.0) {
    // RY(theta) diag(1, b1) = Z RY(-theta) diag(1, -b1): |arg(-b1)| <= pi/2
    b1 = -b1;
    a1 = -a1;
    sign = -1.0;
  }
  const double sg = sign * ss;
  double g0 = 1.0, g1 = rho;
  if (scaled && cc >= kShearPivot) {
    if (rho <= 1.0) {
      R->form = 1;
      R->t = -sg * rho / cc;
      R->s = sg * cc / rho;
      g0 = cc;
      g1 = rho / cc;
    } else {
      R->form = 2;
      R->s = sg / (cc * rho);
      R->t = -sg * cc * rho;
      g0 = 1.0 / cc;
      g1 = cc * rho;
    }
  } else {
    // tan(theta/4) = s / (1 + c) (half-angle formula for theta/2, c >= 0)
    R->form = 0;
    R->t = -rho * sg / (1.0 + cc);
    R->s = sg / rho;
  }
  R->g0 = a0 * g0;
  R->g1 = a1 * g1;
  R->has_z = !(b1.real() == 1.0 && b1.imag() == 0.0);
  // tan(beta/2) = sin(beta) / (1 + cos(beta)), cos(beta) >= 0
  R->tz = R->has_z ? b1.imag() / (1.0 + b1.real()) : 0.0;
  R->sz = R->has_z ? b1.imag() : 0.0;
  return true;
}

// ---- rewritten gates -----------------------------------------------------------
enum RKind { RK_MATRIX = 0, RK_ROT = 1, RK_FLUSH = 2 };

struct RGate {
  RKind kind = RK_MATRIX;
  LoweredGate g;              // targets / controls (and the matrix for RK_MATRIX)
  Rot rot;                    // RK_ROT
  std::vector<int> flq;       // RK_FLUSH: qubits
  std::vector<cplx> flr;      //           their factors r_q (applied where the bit is 1)
  cplx flG{1.0, 0.0};         //           global factor
};

bool is_swap4(const cplx* m) {
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      const bool one = (r == 0 && c == 0) || (r == 3 && c == 3) || (r == 1 && c == 2) ||
                       (r == 2 && c == 1);
      if (!exact(m[4 * r + c], one ? 1.0 : 0.0)) return false;
    }
  return true;
}

// phase r on the |1> of qubit q, as a diagonal one-qubit gate
RGate phase_gate(int q, cplx r) {
  RGate x;
  x.g.nt = 1;
  x.g.targets[0] = q;
  x.g.nc = 0;
  x.g.m[0] = 1.0;
  x.g.m[1] = x.g.m[2] = 0.0;
  x.g.m[3] = r;
  return x;
}

RGate flush_gate(Frames* F) {
  RGate x;
  x.kind = RK_FLUSH;
  x.g.nt = 0;
  x.g.nc = 0;
  for (int q = 0; q < int(F->r.size()); ++q)
    if (F->r[q] != cplx(1.0, 0.0)) {
      x.flq.push_back(q);
      x.flr.push_back(F->r[q]);
      F->r[q] = 1.0;
    }
  x.flG = F->G;
  F->G = 1.0;
  return x;
}

// `scaled`: rotations may leave real scales in the frames (complex128);
// `lim`: the global factor's scale is flushed once it leaves 2^+-lim.
void rewrite(const std::vector<LoweredGate>& in, Frames* F, bool scaled, double lim,
             std::vector<RGate>* out) {
  for (const auto& g : in) {
    if (g.nt == 0) continue;
    const bool diag = is_diagonal(g);
    if (g.nt == 1 && g.nc == 0) {
      const int q = g.targets[0];
      const cplx rq = F->r[q];
      if (diag) {
        if (g.m[0] != cplx(0.0, 0.0)) {  // joins the pending diagonal
          F->G *= g.m[0];
          F->r[q] = g.m[3] * rq / g.m[0];
        } else {  // degenerate (custom C1): applied with the pending factor
          RGate x;
          x.g = g;
          x.g.m[3] *= rq;
          F->r[q] = 1.0;
          out->push_back(x);
        }
        continue;
      }
      cplx W[4] = {g.m[0], g.m[1] * rq, g.m[2], g.m[3] * rq};
      RGate x;
      x.g = g;
      if (factor_rotation(W, scaled, &x.rot)) {
        x.kind = RK_ROT;
        F->G *= x.rot.g0;
        F->r[q] = x.rot.g1 / x.rot.g0;
      } else {
        for (int k = 0; k < 4; ++k) x.g.m[k] = W[k];
        F->r[q] = 1.0;
      }
      out->push_back(x);
      if (std::fabs(std::log2(std::abs(F->G))) > lim) {
        // bring the stored amplitudes' scale back (one multiply of the state)
        Frames sc;
        sc.G = std::abs(F->G);
        out->push_back(flush_gate(&sc));
        F->G /= std::abs(F->G);
      }
      continue;
    }
    if (diag) {  // controlled or two-qubit diagonal: commutes with the pending diagonal
      RGate x;
      x.g = g;
      out->push_back(x);
      continue;
    }
    if (g.nt == 2 && g.nc == 0) {
      const int t0 = g.targets[0], t1 = g.targets[1];
      RGate x;
      x.g = g;
      if (is_swap4(g.m)) {
        std::swap(F->r[t0], F->r[t1]);
      } else {
        // absorb diag(1, r_t0) (x) diag(1, r_t1); reference index i = 2*b(t0) + b(t1)
        for (int c = 0; c < 4; ++c) {
          cplx d = 1.0;
          if (c & 2) d *= F->r[t0];
          if (c & 1) d *= F->r[t1];
          for (int r = 0; r < 4; ++r) x.g.m[4 * r + c] *= d;
        }
        F->r[t0] = F->r[t1] = 1.0;
      }
      out->push_back(x);
      continue;
    }
    // controlled non-diagonal gate: apply the pending factors of its targets first
    for (int i = 0; i < g.nt; ++i) {
      const int t = g.targets[i];
      if (F->r[t] != cplx(1.0, 0.0)) {
        out->push_back(phase_gate(t, F->r[t]));
        F->r[t] = 1.0;
      }
    }
    RGate x;
    x.g = g;
    out->push_back(x);
  }
}

// ---- slot view -------------------------------------------------------------------
struct SlotGate {
  const RGate* rg;
  bool diag;
  int nt;
  int ts[2];                 // non-diagonal target slots
  std::vector<int> slots;    // every slot the gate touches (dependencies)
};

int coef_count(const SlotGate& sg) {
  const RGate& r = *sg.rg;
  if (r.kind == RK_ROT) return 4;  // a pair, aligned, after the two reserved entries
  if (r.kind == RK_FLUSH) return 1 + int(r.flq.size());
  if (sg.diag) return 4;
  return r.g.nt == 1 ? 4 : 16;
}

struct Layout {
  const std::vector<int>* tbit_of_slot;  // slot -> tile bit or -1
  int regpos_of_tbit[kMaxTileBits];      // tile bit -> register position or -1
};

// where a slot's bit sits for the group: register / thread / outer
void locate(const Layout& L, int slot, uint8_t* where, uint8_t* pos) {
  const int tb = (*L.tbit_of_slot)[slot];
  if (tb < 0) {
    *where = TW_OUT;
    *pos = uint8_t(slot);
  } else if (L.regpos_of_tbit[tb] >= 0) {
    *where = TW_REG;
    *pos = uint8_t(L.regpos_of_tbit[tb]);
  } else {
    *where = TW_THR;
    *pos = uint8_t(tb);
  }
}

void add_mask_bit(const Layout& L, int slot, DevOp* op) {
  uint8_t w, p;
  locate(L, slot, &w, &p);
  if (w == TW_OUT)
    op->couter |= 1ull << p;
  else if (w == TW_REG)
    op->creg |= uint16_t(1u << p);
  else
    op->cthr |= 1u << p;
}

struct Emitter {
  PartProgram* P;
  const std::vector<int>* q2s;
  void push(cplx c) {
    P->coef[P->ncoef].x = c.real();
    P->coef[P->ncoef].y = c.imag();
    ++P->ncoef;
  }
  void add(const DevOp& op) { P->ops[P->nops++] = op; }
  DevOp blank() {
    DevOp op;
    std::memset(&op, 0, sizeof(op));
    op.coef = uint16_t(P->ncoef);
    return op;
  }
};

void emit_matrix(const SlotGate& sg, const Layout& L, Emitter& E) {
  const LoweredGate& g = sg.rg->g;
  DevOp op = E.blank();
  for (int i = 0; i < g.nc; ++i) add_mask_bit(L, (*E.q2s)[g.controls[i]], &op);
  const cplx* m = g.m;
  const bool ctrl = op.creg != 0 || op.cthr != 0 || op.couter != 0;
  if (sg.diag) {
    const int s0 = (*E.q2s)[g.targets[0]];
    if (g.nt == 1 && exact(m[0], 1)) {
      // phase on the |1> of the target: a mask over controls + target
      add_mask_bit(L, s0, &op);
      if (exact(m[3], -1)) {
        op.kind = OPD_NEG;
        op.code = uint8_t(kc_neg + op.creg);
      } else {
        op.kind = OPD_PHASE;
        op.code = uint8_t(kc_ph + op.creg);
        E.push(m[3]);
      }
    } else {
      op.kind = OPD_DIAG;
      op.code = kc_diag;
      locate(L, s0, &op.t0w, &op.t0p);
      if (g.nt == 1) {
        E.push(m[0]);
        E.push(m[3]);
      } else {
        // device index q = b(t0) | b(t1) << 1; reference index i = 2*b(t0) + b(t1)
        locate(L, (*E.q2s)[g.targets[1]], &op.t1w, &op.t1p);
        E.push(m[0]);   // q=0: i=0
        E.push(m[10]);  // q=1: b0=1,b1=0 -> i=2
        E.push(m[5]);   // q=2: b0=0,b1=1 -> i=1
        E.push(m[15]);  // q=3: i=3
      }
    }
  } else if (g.nt == 1) {
    uint8_t w;
    locate(L, sg.ts[0], &w, &op.ja);
    op.kind = OP1_DENSE;
    for (int k = 0; k < 4; ++k) E.push(m[k]);
    op.code = uint8_t((ctrl ? kc_c1 : kc_d1) + op.ja);
  } else {
    uint8_t w, p0, p1;
    locate(L, sg.ts[0], &w, &p0);
    locate(L, sg.ts[1], &w, &p1);
    op.ja = std::min(p0, p1);
    op.jb = std::max(p0, p1);
    // device index q = b(ja) | b(jb) << 1; reference index i = 2*b(t0) + b(t1)
    auto ref_index = [&](int q) { return p0 < p1 ? (((q & 1) << 1) | (q >> 1)) : q; };
    cplx md[16];
    for (int qo = 0; qo < 4; ++qo)
      for (int qi = 0; qi < 4; ++qi) md[4 * qo + qi] = m[4 * ref_index(qo) + ref_index(qi)];
    static const int pair_index[4][4] = {{-1, 0, 1, 2}, {-1, -1, 3, 4}, {-1, -1, -1, 5},
                                         {-1, -1, -1, -1}};
    const int pi = pair_index[op.ja][op.jb];
    if (is_swap4(md)) {
      op.kind = OP2_SWAP;
      op.code = uint8_t(kc_sw + pi);
    } else {
      op.kind = OP2_DENSE;
      for (int k = 0; k < 16; ++k) E.push(md[k]);
      op.code = uint8_t((ctrl ? kc_c2 : kc_d2) + pi);
    }
  }
  E.add(op);
}

void emit_rot(const SlotGate& sg, const Layout& L, Emitter& E) {
  DevOp op = E.blank();
  uint8_t w;
  locate(L, sg.ts[0], &w, &op.ja);
  const Rot& r = sg.rg->rot;
  op.kind = OP1_ROT;
  op.code = uint8_t((r.has_z ? kc_zy : kc_y) + op.ja);
  op.form = uint32_t(r.form);
  // coefficient pairs start at even indices >= 2 (pair 0 marks "none")
  while (E.P->ncoef < 2 || (E.P->ncoef & 1)) E.push(0.0);
  op.coef = uint16_t(E.P->ncoef);
  E.push(cplx(r.t, r.s));
  E.push(r.has_z ? cplx(r.tz, r.sz) : cplx(0.0, 0.0));
  E.add(op);
}

// register-bit factors become phase ops; thread / outer ones and G one flush op
int emit_flush(const SlotGate& sg, const Layout& L, Emitter& E) {
  const RGate& r = *sg.rg;
  std::vector<int> rest;
  for (size_t i = 0; i < r.flq.size(); ++i) {
    uint8_t w, p;
    locate(L, (*E.q2s)[r.flq[i]], &w, &p);
    if (w == TW_REG) {
      DevOp op = E.blank();
      op.kind = OPD_PHASE;
      op.creg = uint16_t(1u << p);
      op.code = uint8_t(kc_ph + op.creg);
      E.push(r.flr[i]);
      E.add(op);
    } else {
      rest.push_back(int(i));
    }
  }
  if (rest.empty() && r.flG == cplx(1.0, 0.0)) return HS_OK;
  PartProgram* P = E.P;
  if (P->nfl + int(rest.size()) > kMaxFlush)
    return set_error(HS_E_UNSUPPORTED, "frame flush of %d entries exceeds %d", int(rest.size()),
                     kMaxFlush);
  DevOp op = E.blank();
  op.kind = OPD_FLUSH;
  op.code = kc_flush;
  op.fl_first = uint16_t(P->nfl);
  op.fl_n = uint16_t(rest.size());
  E.push(r.flG);
  for (int i : rest) {
    uint8_t w, p;
    locate(L, (*E.q2s)[r.flq[i]], &w, &p);
    P->flw[P->nfl] = w;
    P->flp[P->nfl] = p;
    ++P->nfl;
    E.push(r.flr[i]);
  }
  E.add(op);
  return HS_OK;
}

// does op x act on register bit j (target, control or mask)?
bool touches_reg(const DevOp& x, int j) {
  if (x.kind == OP1_ROT || x.kind == OP1_DENSE) {
    if (x.ja == j) return true;
  } else if (x.kind == OP2_DENSE || x.kind == OP2_SWAP) {
    if (x.ja == j || x.jb == j) return true;
  } else if (x.kind == OPD_DIAG) {
    if ((x.t0w == TW_REG && x.t0p == j) || (x.t1w == TW_REG && x.t1p == j)) return true;
  }
  return ((x.creg >> j) & 1) != 0;
}

bool diagonal_op(const DevOp& x) { return x.kind >= OPD_PHASE; }

// the sign word entry of a sign flip on register elements (mask creg) whose
// thread / outer condition is at most one bit
bool sign_entry(const DevOp& x, uint32_t* entry) {
  if (x.kind != OPD_NEG || x.creg == 0 || x.creg > 15) return false;
  const int nthr = __builtin_popcount(x.cthr), nout = __builtin_popcountll(x.couter);
  if (nthr + nout > 1) return false;
  uint32_t kind = 0, pos = 0;
  if (nthr) {
    kind = 1;
    pos = uint32_t(__builtin_ctz(x.cthr));
  } else if (nout) {
    kind = 2;
    pos = uint32_t(__builtin_ctzll(x.couter));
  }
  *entry = uint32_t(x.creg) | kind << 4 | pos << 6;
  return true;
}

// Pack the group's ops into rounds (RoundDesc) by list scheduling: op b must
// follow an earlier op a only when both act on a common register bit and not
// both are diagonal (ops act non-diagonally on register bits alone, so
// anything else commutes).  Each round takes, per register bit, the first
// rotation whose predecessors are all in earlier rounds, then every other op
// whose predecessors are scheduled (this round's rotations included), in
// program order.
void build_rounds(PartProgram* P, GroupDesc* gd) {
  gd->first_round = uint16_t(P->nrounds);
  const int o0 = gd->first_op, n = gd->num_ops;
  std::vector<uint16_t> regs(n, 0);  // register bits each op acts on
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < kRegBits; ++j)
      if (touches_reg(P->ops[o0 + i], j)) regs[i] |= uint16_t(1u << j);
  std::vector<std::vector<int>> preds(n);
  for (int b = 0; b < n; ++b)
    for (int a = 0; a < b; ++a)
      if ((regs[a] & regs[b]) && !(diagonal_op(P->ops[o0 + a]) && diagonal_op(P->ops[o0 + b])))
        preds[b].push_back(a);
  // 0: unscheduled, 1: in an earlier round, 2: in this round
  std::vector<int> state(n, 0);
  int left = n;
  auto ready = [&](int b, int need) {
    for (int a : preds[b])
      if (state[a] == 0 || state[a] > need) return false;
    return true;
  };
  while (left > 0) {
    uint32_t mask = 0, zmask = 0, pair[4] = {0, 0, 0, 0}, form[4] = {0, 0, 0, 0};
    const uint32_t first_other = uint32_t(P->nothers);
    uint32_t num_other = 0;
    for (int b = 0; b < n; ++b) {
      const DevOp& x = P->ops[o0 + b];
      if (state[b] || x.kind != OP1_ROT || ((mask >> x.ja) & 1) || !ready(b, 1)) continue;
      // an earlier unscheduled rotation on the same bit goes first
      bool first = true;
      for (int a = 0; a < b; ++a)
        if (!state[a] && P->ops[o0 + a].kind == OP1_ROT && P->ops[o0 + a].ja == x.ja) first = false;
      if (!first) continue;
      mask |= 1u << x.ja;
      if (x.code < kc_y) zmask |= 1u << x.ja;
      pair[x.ja] = x.coef / 2u;
      form[x.ja] = x.form;
      state[b] = 2;
      --left;
    }
    // sign flips on register elements with at most one thread / outer
    // condition go to the round's sign word (applied before its other ops:
    // valid while every other op placed before them is diagonal)
    uint64_t signs = 0;
    int nsign = 0;
    bool others_diag = true;
    for (bool grew = true; grew;) {
      grew = false;
      for (int b = 0; b < n; ++b) {
        const DevOp& x = P->ops[o0 + b];
        if (state[b] || x.kind == OP1_ROT || !ready(b, 2)) continue;
        uint32_t entry = 0;
        if (others_diag && nsign < 4 && sign_entry(x, &entry)) {
          signs |= uint64_t(entry) << (16 * nsign++);
        } else {
          P->others[P->nothers++] = uint8_t(o0 + b);
          ++num_other;
          if (!diagonal_op(x)) others_diag = false;
        }
        state[b] = 2;
        --left;
        grew = true;
      }
    }
    P->signs[P->nrounds] = signs;
    P->rounds[P->nrounds++] = round_pack(zmask, first_other, num_other, pair, form);
    for (int b = 0; b < n; ++b)
      if (state[b] == 2) state[b] = 1;
  }
  gd->num_rounds = uint16_t(P->nrounds - gd->first_round);
}

// ---- shared-memory layout ----------------------------------------------------
// Slot s of the tile (16 bytes) sits at s ^ fold(s), fold(s) = XOR over the
// set bits k of s of fold[k] (3 bits: a move within the 128-byte row).
uint32_t fold_of(const PartProgram& P, uint32_t s) {
  uint32_t r = 0;
  for (int k = 0; k < 16; ++k)
    if ((s >> k) & 1u) r ^= P.fold[k];
  return r;
}

// Byte offset change of setting tile bit tbit (the map is linear over GF(2)).
uint32_t smem_dx(const PartProgram& P, int tbit, int dtype) {
  const int sh = dtype == HS_DTYPE_C64 ? 1 : 0;
  const uint32_t b = 1u << tbit;
  const uint32_t slot = b >> sh;
  return ((slot ^ fold_of(P, slot)) << 4) ^ ((b & ((1u << sh) - 1u)) * uint32_t(amp_bytes(dtype)));
}

// Pick fold so that, in every register group, the lanes of one access phase
// (8 lanes of 16 bytes for complex128, 16 of 8 bytes for complex64) hit
// distinct banks: the lanes differ in the group's lowest thread tile bits,
// whose images (slot bits 0..2 after the fold, plus the in-slot bit for
// complex64) must be linearly independent.  Slot bits 0..2 keep fold 0, so
// the chunked tile copy (lanes over consecutive slots) is conflict-free too.
// Small backtracking search, the fixed fold of the earlier layout (bit k >= 3
// onto bit k mod 3) first; kept when no assignment is found.
void choose_fold(PartProgram* P, int dtype) {
  const int sh = dtype == HS_DTYPE_C64 ? 1 : 0;
  const int nslot = P->m - sh;
  const int lane_bits = std::min(dtype == HS_DTYPE_C64 ? 4 : 3, P->m - P->rbits);
  std::memset(P->fold, 0, sizeof(P->fold));
  for (int k = 3; k < nslot; ++k) P->fold[k] = uint8_t(1u << (k % 3));
  if (lane_bits < 1 || nslot <= 3) return;
  // constraints: the lane tile bits of each group
  std::vector<std::vector<int>> cons;
  for (int g = 0; g < P->ngroups; ++g) {
    std::vector<int> lb;
    for (int b = 0; b < P->m && int(lb.size()) < lane_bits; ++b) {
      bool reg = false;
      for (int j = 0; j < P->rbits; ++j) reg |= P->groups[g].reg_tbit[j] == b;
      if (!reg) lb.push_back(b);
    }
    cons.push_back(lb);
  }
  auto vec = [&](const uint8_t* F, int tbit) -> uint32_t {
    if (tbit < sh) return 8u << tbit;  // in-slot bit: its own dimension
    const int k = tbit - sh;
    return (k < 3 ? (1u << k) : 0u) ^ F[k];
  };
  // the lanes' images must have full rank: min(lanes, 3 slot bits + the
  // in-slot bit when a lane bit is one) -- complex64 lanes that share the
  // in-slot half can at best hit every bank pair twice
  auto independent = [&](const uint8_t* F, const std::vector<int>& lb) {
    int dims = 3;
    for (int b : lb) dims += b < sh;
    const int want = std::min(int(lb.size()), dims);
    uint32_t basis[8];
    int rank = 0;
    for (int b : lb) {
      uint32_t x = vec(F, b);
      for (int i = 0; i < rank; ++i) x = std::min(x, x ^ basis[i]);
      if (x) basis[rank++] = x;
      for (int i = rank - 1; i > 0 && basis[i] > basis[i - 1]; --i) std::swap(basis[i], basis[i - 1]);
    }
    return rank >= want;
  };
  // the highest slot bit each constraint involves (checked once it is set)
  auto top = [&](const std::vector<int>& lb) {
    int t = -1;
    for (int b : lb) t = std::max(t, b - sh);
    return t;
  };
  uint8_t F[16];
  std::memcpy(F, P->fold, sizeof(F));
  bool ok = true;
  for (const auto& c : cons)
    if (!independent(F, c)) ok = false;
  if (ok) return;
  int budget = 20000;
  std::function<bool(int)> dfs = [&](int k) -> bool {
    if (--budget < 0) return false;
    if (k >= nslot) return true;
    const uint8_t first = uint8_t(1u << (k % 3));
    for (int i = 0; i < 8; ++i) {
      const uint8_t cand = uint8_t(i == 0 ? first : (i == first ? 0 : i));
      F[k] = cand;
      bool good = true;
      for (const auto& c : cons)
        if (top(c) == k && !independent(F, c)) {
          good = false;
          break;
        }
      if (good && dfs(k + 1)) return true;
    }
    F[k] = first;
    return false;
  };
  // constraints that involve only slot bits 0..2 do not depend on fold
  if (dfs(3)) std::memcpy(P->fold, F, sizeof(F));
}

void finish_layout(PartProgram* P, int dtype) {
  choose_fold(P, dtype);
  for (int g = 0; g < P->ngroups; ++g)
    for (int j = 0; j < P->rbits; ++j) P->groups[g].dx[j] = smem_dx(*P, P->groups[g].reg_tbit[j], dtype);
}

}  // namespace

int plan_gates(int n, const std::vector<int>& q2s, const std::vector<LoweredGate>& gates,
               Frames* fr, bool flush, int tile_bits_hint, int dtype,
               std::vector<PartProgram>* programs) {
  programs->clear();
  if (n < 1 || n > 63) return set_error(HS_E_INVALID, "bad qubit count %d", n);
  if (int(fr->r.size()) != n) fr->reset(n);
  std::vector<RGate> rg;
  rg.reserve(gates.size() + 2);
  // keep the carried scale within a few dozen binary orders (it moves with
  // the scaled rotation forms and non-unitary diagonal gates)
  const double lim = dtype == HS_DTYPE_C64 ? 24.0 : 48.0;
  rewrite(gates, fr, dtype == HS_DTYPE_C128, lim, &rg);
  if (flush) {
    if (!fr->identity()) rg.push_back(flush_gate(fr));
  } else if (std::fabs(std::log2(std::abs(fr->G))) > lim) {
    Frames scale;
    scale.G = std::abs(fr->G);
    rg.push_back(flush_gate(&scale));
    fr->G /= std::abs(fr->G);
  }
  // one tile buffer per CTA: up to 2^12 amplitudes (64 KiB of complex128)
  const int max_tile = std::min(n, max_tile_bits(dtype));
  const int rbits = k1_reg_bits(dtype);
  // automatic size: complex128 tiles of 2^10 (CTAs of 64 threads x 16
  // amplitudes, ten per SM), complex64 tiles of 2^12
  const int auto_m = dtype == HS_DTYPE_C128 ? 10 : max_tile;
  const int m_target = std::min(max_tile, tile_bits_hint > 0 ? tile_bits_hint : auto_m);
  // keep the three lowest slots in the tile where they fit, so that global
  // accesses come in contiguous runs of at least 8 amplitudes (128 bytes of
  // complex128: whole L2 lines; with 64-byte runs the other half of each
  // line is fetched as well and often evicted before its own tile reads it
  // -- 3.7% slower at 33 qubits)
  const int low_min = std::min(n, 3);
  std::vector<SlotGate> sgs;
  sgs.reserve(rg.size());
  for (const auto& r : rg) {
    SlotGate s;
    s.rg = &r;
    s.nt = 0;
    if (r.kind == RK_FLUSH) {
      s.diag = true;
      for (int q : r.flq) s.slots.push_back(q2s[q]);
    } else {
      s.diag = r.kind == RK_MATRIX && is_diagonal(r.g);
      for (int i = 0; i < r.g.nt; ++i) {
        s.slots.push_back(q2s[r.g.targets[i]]);
        if (!s.diag) s.ts[s.nt++] = q2s[r.g.targets[i]];
      }
      for (int i = 0; i < r.g.nc; ++i) s.slots.push_back(q2s[r.g.controls[i]]);
    }
    sgs.push_back(std::move(s));
  }
  auto low_union_size = [&](const std::vector<int>& t, int lows) {
    int extra = 0;
    for (int s = 0; s < lows; ++s)
      if (std::find(t.begin(), t.end(), s) == t.end()) ++extra;
    return int(t.size()) + extra;
  };
  // a chunk only needs the low slots the 16-byte chunk copy requires (slot 0
  // for complex64); where the targets leave room the tile takes all three:
  // shorter runs cost less than another pass
  const int low_need = std::min(n, dtype == HS_DTYPE_C64 ? 1 : 0);
  size_t gi = 0;
  while (gi < sgs.size()) {
    // ---- chunk: gates whose non-diagonal target slots (+ low slots) fit one tile
    std::vector<int> tset;
    size_t gend = gi;
    int ops = 0, coefs = 0, fls = 0;
    while (gend < sgs.size()) {
      std::vector<int> t2 = tset;
      for (int i = 0; i < sgs[gend].nt; ++i)
        if (std::find(t2.begin(), t2.end(), sgs[gend].ts[i]) == t2.end())
          t2.push_back(sgs[gend].ts[i]);
      const int cc = coef_count(sgs[gend]);
      const int nops_g = sgs[gend].rg->kind == RK_FLUSH ? 1 + int(sgs[gend].rg->flq.size()) : 1;
      const int nfl_g = sgs[gend].rg->kind == RK_FLUSH ? int(sgs[gend].rg->flq.size()) : 0;
      if (low_union_size(t2, low_need) > max_tile || ops + nops_g > kMaxOps || coefs + cc > kMaxCoef ||
          fls + nfl_g > kMaxFlush)
        break;
      tset = t2;
      ops += nops_g;
      coefs += cc;
      fls += nfl_g;
      ++gend;
    }
    if (gend == gi) return set_error(HS_E_INVALID, "gate does not fit a tile");
    // ---- tile: non-diagonal target slots + lowest slots up to the target size
    std::vector<int> tile = tset;
    const int m = std::min(max_tile, std::max(m_target, low_union_size(tset, low_min)));
    for (int s = 0; s < n && int(tile.size()) < m; ++s)
      if (std::find(tile.begin(), tile.end(), s) == tile.end()) tile.push_back(s);
    std::sort(tile.begin(), tile.end());
    const int R = std::min(rbits, m);
    std::vector<int> tbit_of_slot(n, -1);
    for (int i = 0; i < m; ++i) tbit_of_slot[tile[i]] = i;
    PartProgram* P = nullptr;
    auto new_program = [&]() {
      programs->emplace_back();
      P = &programs->back();
      std::memset(P, 0, sizeof(*P));
      P->n = n;
      P->m = m;
      P->ntiles = 1ull << (n - m);
      P->rbits = R;
      build_runs(tile, &P->tile);
      for (int b = 0; b < m; ++b) P->tile_slot[b] = uint8_t(tile[b]);
      std::vector<int> outer;
      for (int s = 0; s < n; ++s)
        if (tbit_of_slot[s] < 0) outer.push_back(s);
      build_runs(outer, &P->outer);
    };
    new_program();
    // ---- groups: a second-level acyclic partition of the chunk.  Each group
    // takes, in circuit order, every remaining gate whose non-diagonal targets
    // fit the R register bits and none of whose qubits is held by a gate left
    // for a later group (so every gate still follows all gates it depends on).
    std::vector<size_t> remaining;
    for (size_t x = gi; x < gend; ++x) remaining.push_back(x);
    while (!remaining.empty()) {
      std::vector<int> regs;
      std::vector<size_t> members, rest;
      std::vector<int> blocked;  // slots held back by a deferred gate
      auto touches = [&](const SlotGate& g) {
        for (int s : g.slots)
          if (std::find(blocked.begin(), blocked.end(), s) != blocked.end()) return true;
        return false;
      };
      auto block = [&](const SlotGate& g) {
        for (int s : g.slots) blocked.push_back(s);
      };
      for (size_t x : remaining) {
        const SlotGate& g = sgs[x];
        if (touches(g)) {
          block(g);
          rest.push_back(x);
          continue;
        }
        if (!g.diag) {
          std::vector<int> r2 = regs;
          for (int i = 0; i < g.nt; ++i) {
            const int tb = tbit_of_slot[g.ts[i]];
            if (std::find(r2.begin(), r2.end(), tb) == r2.end()) r2.push_back(tb);
          }
          if (int(r2.size()) > R) {
            block(g);
            rest.push_back(x);
            continue;
          }
          regs = r2;
        }
        members.push_back(x);
      }
      if (P->ngroups == kMaxGroups) new_program();  // a new pass (rare)
      GroupDesc& gd = P->groups[P->ngroups++];
      std::memset(&gd, 0, sizeof(gd));
      // fill the register set with the highest unused tile bits so that the
      // thread (lane) bits stay on the low, contiguous slots
      for (int b = m - 1; b >= 0 && int(regs.size()) < R; --b)
        if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
      std::sort(regs.begin(), regs.end());
      for (int j = 0; j < R; ++j) gd.reg_tbit[j] = uint8_t(regs[j]);
      std::vector<int> thr;
      for (int b = 0; b < m; ++b)
        if (std::find(regs.begin(), regs.end(), b) == regs.end()) thr.push_back(b);
      build_runs(thr, &gd.thr);
      Layout L;
      L.tbit_of_slot = &tbit_of_slot;
      for (int b = 0; b < kMaxTileBits; ++b) L.regpos_of_tbit[b] = -1;
      for (int j = 0; j < R; ++j) L.regpos_of_tbit[regs[j]] = j;
      gd.first_op = uint16_t(P->nops);
      Emitter E{P, &q2s};
      for (size_t x : members) {
        const SlotGate& sg = sgs[x];
        if (sg.rg->kind == RK_ROT)
          emit_rot(sg, L, E);
        else if (sg.rg->kind == RK_FLUSH)
          HS_TRY(emit_flush(sg, L, E));
        else
          emit_matrix(sg, L, E);
      }
      gd.num_ops = uint16_t(P->nops - gd.first_op);
      build_rounds(P, &gd);
      remaining = rest;
    }
    gi = gend;
  }
  for (auto& P : *programs) finish_layout(&P, dtype);
  return HS_OK;
}

int plan_part(int n, const std::vector<int>& q2s, const std::vector<LoweredGate>& gates,
              int tile_bits_hint, int dtype, std::vector<PartProgram>* programs) {
  Frames fr;
  fr.reset(n);
  return plan_gates(n, q2s, gates, &fr, true, tile_bits_hint, dtype, programs);
}

}  // namespace hisv
