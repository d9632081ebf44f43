// Part features for the learned cost model: what a part looks like to K1
// (its qubits, strides, gate mix and the planner's own pass/group/op counts),
// for explicit parts or for every contiguous segment of a topological order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace hisv;

namespace {

constexpr int kTypeLo = HS_GATE_I, kTypeHi = HS_GATE_SDG;
constexpr int kNumFeatures = 15 + (kTypeHi - kTypeLo + 1);

bool is_diagonal(const LoweredGate& g) {
  const int d = g.nt == 2 ? 4 : 2;
  for (int r = 0; r < d; ++r)
    for (int c = 0; c < d; ++c)
      if (r != c && std::abs(g.m[r * d + c]) != 0.0) return false;
  return true;
}

struct Lowered {
  std::vector<hs_gate> raw;
  std::vector<LoweredGate> lg;
  std::vector<uint64_t> qmask, ndmask;  // all qubits; non-diagonal targets
  std::vector<uint8_t> twoq, ctrl;
};

int lower_all(int n, const hs_gate* gates, int ng, Lowered* L) {
  L->raw.assign(gates, gates + ng);
  L->lg.resize(ng);
  L->qmask.assign(ng, 0);
  L->ndmask.assign(ng, 0);
  L->twoq.assign(ng, 0);
  L->ctrl.assign(ng, 0);
  for (int i = 0; i < ng; ++i) {
    HS_TRY(lower_gate(gates[i], n, &L->lg[i]));
    const LoweredGate& g = L->lg[i];
    uint64_t q = 0, t = 0;
    for (int k = 0; k < g.nt; ++k) t |= 1ull << g.targets[k];
    for (int k = 0; k < g.nc; ++k) q |= 1ull << g.controls[k];
    q |= t;
    // identity gates still occupy their qubits in the reference's parts
    for (int k = 0; k < gates[i].num_targets; ++k) q |= 1ull << gates[i].targets[k];
    L->qmask[i] = q;
    L->ndmask[i] = (g.nt > 0 && !is_diagonal(g)) ? t : 0;
    L->twoq[i] = __builtin_popcountll(q) >= 2;
    L->ctrl[i] = g.nc > 0;
  }
  return HS_OK;
}

int features_of(int n, int dtype, const Lowered& L, const int32_t* idx, int len,
                const std::vector<int>& q2s, float* f) {
  std::memset(f, 0, sizeof(float) * kNumFeatures);
  uint64_t q = 0, nd = 0;
  int twoq = 0, ctrl = 0;
  std::vector<LoweredGate> part;
  part.reserve(len);
  for (int i = 0; i < len; ++i) {
    const int g = idx[i];
    q |= L.qmask[g];
    nd |= L.ndmask[g];
    twoq += L.twoq[g];
    ctrl += L.ctrl[g];
    const int t = L.raw[g].type;
    if (t >= kTypeLo && t <= kTypeHi) f[15 + t - kTypeLo] += 1.f / 16.f;
    if (L.lg[g].nt > 0) part.push_back(L.lg[g]);
  }
  int high = 0, maxs = 0, minnd = n;
  for (int b = 0; b < n; ++b) {
    if (!((q >> b) & 1ull)) continue;
    const int s = q2s[b];
    high += s >= 10;
    maxs = std::max(maxs, s);
    if ((nd >> b) & 1ull) minnd = std::min(minnd, s);
  }
  f[0] = float(n) / 32.f;
  f[1] = float(__builtin_popcountll(q)) / 12.f;
  f[2] = float(len) / 32.f;
  f[3] = float(__builtin_popcountll(nd)) / 12.f;
  f[4] = float(high) / 12.f;
  f[5] = float(maxs) / float(n);
  f[6] = nd ? float(minnd) / float(n) : 0.f;
  f[7] = len ? float(twoq) / float(len) : 0.f;
  f[8] = float(ctrl) / 32.f;
  if (!part.empty()) {
    std::vector<PartProgram> progs;
    HS_TRY(plan_part(n, q2s, part, current_tile_hint(), dtype, &progs));
    int groups = 0, ops = 0, diag = 0, dense = 0, m = 0;
    for (const auto& p : progs) {
      groups += p.ngroups;
      ops += p.nops;
      m = std::max(m, int(p.m));
      for (int i = 0; i < p.nops; ++i) {
        diag += p.ops[i].kind >= OPD_PHASE;
        dense += p.ops[i].kind == OP1_ROT || p.ops[i].kind == OP1_DENSE ||
                 p.ops[i].kind == OP2_DENSE;
      }
    }
    f[9] = float(progs.size()) / 4.f;
    f[10] = float(groups) / 16.f;
    f[11] = float(ops) / 64.f;
    f[12] = float(dense) / 64.f;
    f[13] = float(diag) / 64.f;
    f[14] = float(m) / 12.f;
  }
  return HS_OK;
}

int check_args(int n, int dtype, const hs_gate* gates, int ng) {
  if (n < 1 || n > 40) return set_error(HS_E_INVALID, "bad qubit count");
  if (dtype != HS_DTYPE_C128 && dtype != HS_DTYPE_C64) return set_error(HS_E_INVALID, "bad dtype");
  if (ng < 0 || (ng > 0 && !gates)) return set_error(HS_E_INVALID, "bad gate list");
  return HS_OK;
}

}  // namespace

extern "C" {

int hs_num_part_features(void) { return kNumFeatures; }

int hs_part_features(int num_qubits, int dtype, const hs_gate* gates, int num_gates,
                     const int32_t* part_gates, const int32_t* part_offsets, int num_parts,
                     float* feats) {
  HS_TRY(check_args(num_qubits, dtype, gates, num_gates));
  Lowered L;
  HS_TRY(lower_all(num_qubits, gates, num_gates, &L));
  std::vector<int> q2s(num_qubits);
  for (int b = 0; b < num_qubits; ++b) q2s[b] = b;
  for (int p = 0; p < num_parts; ++p) {
    const int a = part_offsets[p], e = part_offsets[p + 1];
    for (int i = a; i < e; ++i)
      if (part_gates[i] < 0 || part_gates[i] >= num_gates)
        return set_error(HS_E_INVALID, "gate index out of range");
    HS_TRY(features_of(num_qubits, dtype, L, part_gates + a, e - a, q2s,
                       feats + size_t(p) * kNumFeatures));
  }
  return HS_OK;
}

int hs_order_segments(int num_qubits, int dtype, const hs_gate* gates, int num_gates,
                      const int32_t* order, int max_qubits, int max_len, int capacity,
                      int32_t* seg_start, int32_t* seg_len, float* feats, int32_t* count) {
  HS_TRY(check_args(num_qubits, dtype, gates, num_gates));
  if (!order || !count || max_qubits < 1 || max_len < 1 || capacity < 0)
    return set_error(HS_E_INVALID, "bad arguments");
  Lowered L;
  HS_TRY(lower_all(num_qubits, gates, num_gates, &L));
  std::vector<int> q2s(num_qubits);
  for (int b = 0; b < num_qubits; ++b) q2s[b] = b;
  int c = 0;
  for (int i = 0; i < num_gates; ++i) {
    uint64_t q = 0;
    for (int j = i; j < num_gates && j - i < max_len; ++j) {
      if (order[j] < 0 || order[j] >= num_gates)
        return set_error(HS_E_INVALID, "order index out of range");
      q |= L.qmask[order[j]];
      if (__builtin_popcountll(q) > max_qubits) break;
      if (c < capacity) {
        seg_start[c] = i;
        seg_len[c] = j - i + 1;
        if (feats)
          HS_TRY(features_of(num_qubits, dtype, L, order + i, j - i + 1, q2s,
                             feats + size_t(c) * kNumFeatures));
      }
      ++c;
    }
  }
  *count = c;
  if (c > capacity) return set_error(HS_E_INVALID, "%d segments exceed capacity %d", c, capacity);
  return HS_OK;
}

}  // extern "C"
