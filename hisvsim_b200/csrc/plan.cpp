// Host planner for K1: turns one part (a gate sequence) into tile programs.
//
// The reference runs a part by gathering, for each assignment of the outer
// qubits, the 2^k amplitudes of the part's qubits into an inner state vector,
// applying every gate there and scattering back (execute.hpp:318-470,
// state_vector.hpp:617-673; the loop nest of loop.hpp:468-962).  Here a tile
// is the same gather, widened by the lowest slots so that every global access
// moves whole 32-byte sectors (the GPU form of opt_slots, execute.hpp:184-199).
// Each tile is held by one CTA: 2^R amplitudes per thread in registers, where
// R tile bits are "register bits"; a gate's targets must be register bits.
// Consecutive gates whose targets fit in R bits form a group; between groups
// the tile is exchanged through shared memory so that the next group's targets
// become register bits.  Controls are predicates (register, thread or outer
// bits), as control_offset is in StateVector::apply (state_vector.hpp:410-417).
#include <algorithm>
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

struct SlotGate {
  const LoweredGate* g;
  int ts[2];   // target slots
  int nc;
  int cs[HS_MAX_CONTROLS];
};

int coef_count(const LoweredGate& g) {
  const cplx* m = g.m;
  if (g.nt == 1) {
    if (exact(m[1], 0) && exact(m[2], 0)) {
      if (exact(m[0], 1)) return exact(m[3], -1) ? 0 : 1;
      return 2;
    }
    return 4;  // upper bound (X/H/Y use none)
  }
  bool diag = true;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c)
      if (r != c && !exact(m[4 * r + c], 0)) diag = false;
  return diag ? 4 : 16;
}

// Fill the op for gate sg in group gd of a program whose tile maps slot ->
// tile bit via tbit_of_slot (-1 outside the tile).
void emit_op(const SlotGate& sg, const GroupDesc& gd, int R, const std::vector<int>& tbit_of_slot,
             PartProgram* P) {
  DevOp op;
  std::memset(&op, 0, sizeof(op));
  int regpos_of_tbit[kMaxTileBits];
  for (int b = 0; b < kMaxTileBits; ++b) regpos_of_tbit[b] = -1;
  for (int j = 0; j < R; ++j) regpos_of_tbit[gd.reg_tbit[j]] = j;
  for (int i = 0; i < sg.nc; ++i) {
    int s = sg.cs[i];
    int tb = tbit_of_slot[s];
    if (tb < 0)
      op.couter |= 1ull << s;
    else if (regpos_of_tbit[tb] >= 0)
      op.creg |= uint16_t(1u << regpos_of_tbit[tb]);
    else
      op.cthr |= 1u << tb;
  }
  const cplx* m = sg.g->m;
  int base = P->ncoef;  // coefficients are appended in op order
  auto push = [&](cplx c) {
    P->coef[base].x = c.real();
    P->coef[base].y = c.imag();
    ++base;
  };
  op.coef = uint16_t(base);
  if (sg.g->nt == 1) {
    op.ja = uint8_t(regpos_of_tbit[tbit_of_slot[sg.ts[0]]]);
    const double s = 0.707106781186547524401;
    if (exact(m[1], 0) && exact(m[2], 0)) {
      if (exact(m[0], 1)) {
        if (exact(m[3], -1)) {
          op.kind = OP1_NEG;
        } else {
          op.kind = OP1_PHASE;
          push(m[3]);
        }
      } else {
        op.kind = OP1_DIAG;
        push(m[0]);
        push(m[3]);
      }
    } else if (exact(m[0], 0) && exact(m[3], 0) && exact(m[1], 1) && exact(m[2], 1)) {
      op.kind = OP1_X;
    } else if (exact(m[0], s) && exact(m[1], s) && exact(m[2], s) && exact(m[3], -s)) {
      op.kind = OP1_H;
    } else if (exact(m[0], 0) && exact(m[3], 0) && exact(m[1], 0, -1) && exact(m[2], 0, 1)) {
      op.kind = OP1_Y;
    } else {
      op.kind = OP1_DENSE;
      for (int k = 0; k < 4; ++k) push(m[k]);
    }
  } else {
    int p0 = regpos_of_tbit[tbit_of_slot[sg.ts[0]]];
    int p1 = regpos_of_tbit[tbit_of_slot[sg.ts[1]]];
    op.ja = uint8_t(std::min(p0, p1));
    op.jb = uint8_t(std::max(p0, p1));
    // device index q = b(ja) | b(jb) << 1; reference index i = 2*b(t0) + b(t1)
    auto ref_index = [&](int q) { return p0 < p1 ? (((q & 1) << 1) | (q >> 1)) : q; };
    cplx md[16];
    for (int qo = 0; qo < 4; ++qo)
      for (int qi = 0; qi < 4; ++qi) md[4 * qo + qi] = m[4 * ref_index(qo) + ref_index(qi)];
    bool diag = true, swap = true;
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        if (r != c && !exact(md[4 * r + c], 0)) diag = false;
        const bool one = (r == 0 && c == 0) || (r == 3 && c == 3) || (r == 1 && c == 2) ||
                         (r == 2 && c == 1);
        if (!exact(md[4 * r + c], one ? 1.0 : 0.0)) swap = false;
      }
    if (swap) {
      op.kind = OP2_SWAP;
    } else if (diag) {
      op.kind = OP2_DIAG;
      for (int k = 0; k < 4; ++k) push(md[5 * k]);
    } else {
      op.kind = OP2_DENSE;
      for (int k = 0; k < 16; ++k) push(md[k]);
    }
  }
  P->ncoef = base;
  P->ops[P->nops++] = op;
}

}  // namespace

int plan_part(int n, const std::vector<int>& q2s, const std::vector<LoweredGate>& gates,
              int tile_bits_hint, std::vector<PartProgram>* programs) {
  programs->clear();
  if (n < 1 || n > 63) return set_error(HS_E_INVALID, "bad qubit count %d", n);
  const int max_tile = std::min(n, kMaxTileBits);
  const int m_target = std::min(n, tile_bits_hint > 0 ? std::min(tile_bits_hint, kMaxTileBits)
                                                      : 12);
  const int low_min = std::min(n, 3);
  std::vector<SlotGate> sgs;
  for (const auto& g : gates) {
    if (g.nt == 0) continue;
    SlotGate s;
    s.g = &g;
    for (int i = 0; i < g.nt; ++i) s.ts[i] = q2s[g.targets[i]];
    s.nc = g.nc;
    for (int i = 0; i < g.nc; ++i) s.cs[i] = q2s[g.controls[i]];
    sgs.push_back(s);
  }
  size_t gi = 0;
  while (gi < sgs.size()) {
    // ---- chunk: gates whose target slots (plus the low slots) fit one tile
    std::vector<int> tset;  // target slots in the chunk
    auto low_union_size = [&](const std::vector<int>& t) {
      int extra = 0;
      for (int s = 0; s < low_min; ++s)
        if (std::find(t.begin(), t.end(), s) == t.end()) ++extra;
      return int(t.size()) + extra;
    };
    size_t gend = gi;
    int ops = 0, coefs = 0;
    while (gend < sgs.size()) {
      std::vector<int> t2 = tset;
      for (int i = 0; i < sgs[gend].g->nt; ++i)
        if (std::find(t2.begin(), t2.end(), sgs[gend].ts[i]) == t2.end())
          t2.push_back(sgs[gend].ts[i]);
      const int cc = coef_count(*sgs[gend].g);
      if (low_union_size(t2) > max_tile || ops + 1 > kMaxOps || coefs + cc > kMaxCoef) break;
      tset = t2;
      ++ops;
      coefs += cc;
      ++gend;
    }
    if (gend == gi) return set_error(HS_E_INVALID, "gate does not fit a tile");
    // ---- tile: target slots + lowest slots up to the target size
    std::vector<int> tile = tset;
    const int m = std::max(m_target, low_union_size(tset));
    for (int s = 0; s < n && int(tile.size()) < m; ++s)
      if (std::find(tile.begin(), tile.end(), s) == tile.end()) tile.push_back(s);
    std::sort(tile.begin(), tile.end());
    const int R = std::min(kRegBits, m);
    std::vector<int> tbit_of_slot(n, -1);
    for (int i = 0; i < m; ++i) tbit_of_slot[tile[i]] = i;
    // ---- groups over [gi, gend)
    PartProgram* P = nullptr;
    size_t k = gi;
    auto new_program = [&]() {
      programs->emplace_back();
      P = &programs->back();
      std::memset(P, 0, sizeof(*P));
      P->n = n;
      P->m = m;
      P->ntiles = 1ull << (n - m);
      build_runs(tile, &P->tile);
      std::vector<int> outer;
      for (int s = 0; s < n; ++s)
        if (tbit_of_slot[s] < 0) outer.push_back(s);
      build_runs(outer, &P->outer);
    };
    new_program();
    while (k < gend) {
      std::vector<int> regs;  // tile bits needed in registers
      size_t e = k;
      while (e < gend) {
        std::vector<int> r2 = regs;
        for (int i = 0; i < sgs[e].g->nt; ++i) {
          int tb = tbit_of_slot[sgs[e].ts[i]];
          if (std::find(r2.begin(), r2.end(), tb) == r2.end()) r2.push_back(tb);
        }
        if (int(r2.size()) > R) break;
        regs = r2;
        ++e;
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
      gd.first_op = uint16_t(P->nops);
      for (size_t x = k; x < e; ++x) emit_op(sgs[x], gd, R, tbit_of_slot, P);
      gd.num_ops = uint16_t(P->nops - gd.first_op);
      k = e;
    }
    gi = gend;
  }
  return HS_OK;
}

}  // namespace hisv
