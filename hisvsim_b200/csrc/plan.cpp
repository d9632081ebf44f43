// Host planner for K1: turns one part (a gate sequence) into tile programs.
//
// The reference runs a part by gathering, for each assignment of the outer
// qubits, the 2^k amplitudes of the part's qubits into an inner state vector,
// applying every gate there and scattering back (execute.hpp:318-470,
// state_vector.hpp:617-673; the loop nest of loop.hpp:468-962).  Here a tile
// is the same gather, widened by the lowest slots so that every global access
// moves whole 32-byte sectors (the GPU form of opt_slots, execute.hpp:184-199).
// Each tile is held by one CTA: 2^R amplitudes per thread in registers, where
// R tile bits are "register bits".  A non-diagonal gate's targets must be
// register bits; consecutive gates whose targets fit in R bits form a group,
// and between groups the tile is exchanged through shared memory so that the
// next group's targets become register bits.  Diagonal gates (Z, S, T, RZ,
// controlled phases, RZZ, ...) only scale amplitudes by a phase chosen from
// index bits, so they run in any layout and their qubits need not be in the
// tile at all.  Controls are index predicates wherever their bits are, as
// control_offset is in StateVector::apply (state_vector.hpp:410-417).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>

#include "internal.h"

namespace hisv {
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

struct SlotGate {
  const LoweredGate* g;
  bool diag;
  int ts[2];  // target slots
  int nc;
  int cs[HS_MAX_CONTROLS];
};

int coef_count(const SlotGate& sg) {
  if (sg.diag) return 4;
  return sg.g->nt == 1 ? 4 : 16;
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

void emit_op(const SlotGate& sg, const Layout& L, PartProgram* P) {
  DevOp op;
  std::memset(&op, 0, sizeof(op));
  for (int i = 0; i < sg.nc; ++i) add_mask_bit(L, sg.cs[i], &op);
  const cplx* m = sg.g->m;
  int base = P->ncoef;  // coefficients are appended in op order
  auto push = [&](cplx c) {
    P->coef[base].x = c.real();
    P->coef[base].y = c.imag();
    ++base;
  };
  op.coef = uint16_t(base);
  const bool ctrl = op.creg != 0 || op.cthr != 0 || op.couter != 0;
  if (sg.diag) {
    if (sg.g->nt == 1 && exact(m[0], 1)) {
      // phase on the |1> of the target: a mask over controls + target
      add_mask_bit(L, sg.ts[0], &op);
      if (exact(m[3], -1)) {
        op.kind = OPD_NEG;
      } else {
        op.kind = OPD_PHASE;
        push(m[3]);
      }
    } else {
      op.kind = OPD_DIAG;
      locate(L, sg.ts[0], &op.t0w, &op.t0p);
      if (sg.g->nt == 1) {
        push(m[0]);
        push(m[3]);
      } else {
        // device index q = b(t0) | b(t1) << 1; reference index i = 2*b(t0) + b(t1)
        locate(L, sg.ts[1], &op.t1w, &op.t1p);
        push(m[0]);   // q=0: i=0
        push(m[10]);  // q=1: b0=1,b1=0 -> i=2
        push(m[5]);   // q=2: b0=0,b1=1 -> i=1
        push(m[15]);  // q=3: i=3
      }
    }
    if (op.kind == OPD_NEG)
      op.code = uint8_t(16 + op.creg);
    else if (op.kind == OPD_PHASE)
      op.code = uint8_t(32 + op.creg);
    else
      op.code = 48;
  } else if (sg.g->nt == 1) {
    uint8_t w;
    locate(L, sg.ts[0], &w, &op.ja);
    // every non-diagonal one-target gate runs as a dense 2x2 (X, Y and H
    // included: multiplying by 0 and +-1 is exact, H differs from
    // s*(a+b) by at most one rounding)
    op.kind = OP1_DENSE;
    for (int k = 0; k < 4; ++k) push(m[k]);
    op.code = uint8_t((ctrl ? 4 : 0) + op.ja);
  } else {
    uint8_t w;
    uint8_t p0, p1;
    locate(L, sg.ts[0], &w, &p0);
    locate(L, sg.ts[1], &w, &p1);
    op.ja = std::min(p0, p1);
    op.jb = std::max(p0, p1);
    // device index q = b(ja) | b(jb) << 1; reference index i = 2*b(t0) + b(t1)
    auto ref_index = [&](int q) { return p0 < p1 ? (((q & 1) << 1) | (q >> 1)) : q; };
    cplx md[16];
    for (int qo = 0; qo < 4; ++qo)
      for (int qi = 0; qi < 4; ++qi) md[4 * qo + qi] = m[4 * ref_index(qo) + ref_index(qi)];
    bool swap = true;
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        const bool one = (r == 0 && c == 0) || (r == 3 && c == 3) || (r == 1 && c == 2) ||
                         (r == 2 && c == 1);
        if (!exact(md[4 * r + c], one ? 1.0 : 0.0)) swap = false;
      }
    if (swap) {
      op.kind = OP2_SWAP;
    } else {
      op.kind = OP2_DENSE;
      for (int k = 0; k < 16; ++k) push(md[k]);
    }
    static const int pair_index[4][4] = {{-1, 0, 1, 2}, {-1, -1, 3, 4}, {-1, -1, -1, 5},
                                         {-1, -1, -1, -1}};
    op.code = uint8_t((op.kind == OP2_SWAP ? 80 : (ctrl ? 72 : 64)) + pair_index[op.ja][op.jb]);
  }
  P->ncoef = base;
  P->ops[P->nops++] = op;
}

}  // namespace

// Uncontrolled dense one-qubit ops run with a real top-left coefficient
// (code 88 + j: two FP64 instructions fewer per amplitude pair): op U becomes
// e^{-ia} U with a = arg U00, and the program's last uncontrolled dense op,
// which keeps the general form, absorbs the product of the removed phases (a
// global phase commutes with every op).  Ops with U00 = 0 keep the general
// form.
void factor_phases(PartProgram* P) {
  int last = -1;
  for (int i = 0; i < P->nops; ++i)
    if (P->ops[i].kind == OP1_DENSE && P->ops[i].code < 4) last = i;
  if (last < 0) return;
  std::complex<double> g(1.0, 0.0);
  for (int i = 0; i < last; ++i) {
    DevOp& op = P->ops[i];
    if (op.kind != OP1_DENSE || op.code >= 4) continue;
    double2* c = P->coef + op.coef;
    const double r = std::hypot(c[0].x, c[0].y);
    if (!(r > 0.0)) continue;
    const std::complex<double> f(c[0].x / r, -c[0].y / r);  // e^{-ia}
    for (int k = 1; k < 4; ++k) {
      const std::complex<double> v = std::complex<double>(c[k].x, c[k].y) * f;
      c[k].x = v.real();
      c[k].y = v.imag();
    }
    c[0].x = r;
    c[0].y = 0.0;
    g *= std::conj(f);
    op.code = uint8_t(88 + op.ja);
  }
  double2* c = P->coef + P->ops[last].coef;
  for (int k = 0; k < 4; ++k) {
    const std::complex<double> v = std::complex<double>(c[k].x, c[k].y) * g;
    c[k].x = v.real();
    c[k].y = v.imag();
  }
}

int plan_part(int n, const std::vector<int>& q2s, const std::vector<LoweredGate>& gates,
              int tile_bits_hint, int dtype, std::vector<PartProgram>* programs) {
  programs->clear();
  if (n < 1 || n > 63) return set_error(HS_E_INVALID, "bad qubit count %d", n);
  // two tile buffers must fit in shared memory: 2^12 complex128 / 2^13 complex64
  const int max_tile = std::min(n, max_tile_bits(dtype));
  // automatic size: the largest tile, except complex128 with 8 amplitudes per
  // thread, whose 2^10 tiles (CTAs of 128 threads, six per SM) hide FP64
  // latency better than 2^11 (measured)
  const int auto_m = (dtype == HS_DTYPE_C128 && k1_reg_bits(dtype) == 3) ? 10 : max_tile;
  const int m_target = std::min(max_tile, tile_bits_hint > 0 ? tile_bits_hint : auto_m);
  // keep the lowest slots in the tile so that global accesses come in
  // contiguous runs of at least 64 bytes (complex64 tiles also need slot 0 for
  // their 16-byte chunks)
  const int low_min = std::min(n, dtype == HS_DTYPE_C64 ? 3 : 2);
  std::vector<SlotGate> sgs;
  for (const auto& g : gates) {
    if (g.nt == 0) continue;
    SlotGate s;
    s.g = &g;
    s.diag = is_diagonal(g);
    for (int i = 0; i < g.nt; ++i) s.ts[i] = q2s[g.targets[i]];
    s.nc = g.nc;
    for (int i = 0; i < g.nc; ++i) s.cs[i] = q2s[g.controls[i]];
    sgs.push_back(s);
  }
  auto low_union_size = [&](const std::vector<int>& t) {
    int extra = 0;
    for (int s = 0; s < low_min; ++s)
      if (std::find(t.begin(), t.end(), s) == t.end()) ++extra;
    return int(t.size()) + extra;
  };
  size_t gi = 0;
  while (gi < sgs.size()) {
    // ---- chunk: gates whose non-diagonal target slots (+ low slots) fit one tile
    std::vector<int> tset;
    size_t gend = gi;
    int ops = 0, coefs = 0;
    while (gend < sgs.size()) {
      std::vector<int> t2 = tset;
      if (!sgs[gend].diag)
        for (int i = 0; i < sgs[gend].g->nt; ++i)
          if (std::find(t2.begin(), t2.end(), sgs[gend].ts[i]) == t2.end())
            t2.push_back(sgs[gend].ts[i]);
      const int cc = coef_count(sgs[gend]);
      if (low_union_size(t2) > max_tile || ops + 1 > kMaxOps || coefs + cc > kMaxCoef) break;
      tset = t2;
      ++ops;
      coefs += cc;
      ++gend;
    }
    if (gend == gi) return set_error(HS_E_INVALID, "gate does not fit a tile");
    // ---- tile: non-diagonal target slots + lowest slots up to the target size
    std::vector<int> tile = tset;
    const int m = std::min(max_tile, std::max(m_target, low_union_size(tset)));
    for (int s = 0; s < n && int(tile.size()) < m; ++s)
      if (std::find(tile.begin(), tile.end(), s) == tile.end()) tile.push_back(s);
    std::sort(tile.begin(), tile.end());
    const int R = std::min(k1_reg_bits(dtype), m);
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
      auto touches = [&](const SlotGate& g, const std::vector<int>& set) {
        for (int i = 0; i < g.g->nt; ++i)
          if (std::find(set.begin(), set.end(), g.ts[i]) != set.end()) return true;
        for (int i = 0; i < g.nc; ++i)
          if (std::find(set.begin(), set.end(), g.cs[i]) != set.end()) return true;
        return false;
      };
      auto block = [&](const SlotGate& g) {
        for (int i = 0; i < g.g->nt; ++i) blocked.push_back(g.ts[i]);
        for (int i = 0; i < g.nc; ++i) blocked.push_back(g.cs[i]);
      };
      for (size_t x : remaining) {
        const SlotGate& g = sgs[x];
        if (touches(g, blocked)) {
          block(g);
          rest.push_back(x);
          continue;
        }
        if (!g.diag) {
          std::vector<int> r2 = regs;
          for (int i = 0; i < g.g->nt; ++i) {
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
      for (size_t x : members) emit_op(sgs[x], L, P);
      gd.num_ops = uint16_t(P->nops - gd.first_op);
      remaining = rest;
    }
    gi = gend;
  }
  for (auto& P : *programs) factor_phases(&P);
  return HS_OK;
}

}  // namespace hisv
