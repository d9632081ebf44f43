// Host side of the precision form (hs_fused_*): fuse each part into a 64x64
// unitary in FP64 (K5) and apply the unitaries to a complex64 state on the
// tensor cores (K4), several per state pass.  Also the mixed-precision state
// comparison used to report fidelity loss.
#include <algorithm>
#include <cstring>
#include <vector>

#include <atomic>

#include "internal.h"

namespace hisv {
namespace {

cudaStream_t S(void* stream) { return static_cast<cudaStream_t>(stream); }

struct PartLocal {
  int qubits[kFusedBits];  // qubit of local bit j (ascending slot)
  std::vector<FusedGate> gates;
};

// Lower one part to local bits.  The part's qubits are padded to six with the
// qubits in the lowest other slots; local bit j is the j-th lowest slot.
int localize(const hs_gate* gates, int ng, int n, const std::vector<int>& q2s,
             const std::vector<int>& s2q, PartLocal* out) {
  std::vector<LoweredGate> lg(ng);
  std::vector<int> qs;
  for (int i = 0; i < ng; ++i) {
    HS_TRY(lower_gate(gates[i], n, &lg[i]));
    for (int k = 0; k < lg[i].nt; ++k) qs.push_back(lg[i].targets[k]);
    for (int k = 0; k < lg[i].nc; ++k) qs.push_back(lg[i].controls[k]);
  }
  std::sort(qs.begin(), qs.end());
  qs.erase(std::unique(qs.begin(), qs.end()), qs.end());
  if (int(qs.size()) > kFusedBits)
    return set_error(HS_E_INVALID, "a fused part touches %zu qubits (max %d)", qs.size(), kFusedBits);
  for (int s = 0; s < n && int(qs.size()) < kFusedBits; ++s)
    if (std::find(qs.begin(), qs.end(), s2q[s]) == qs.end()) qs.push_back(s2q[s]);
  std::sort(qs.begin(), qs.end(), [&](int a, int b) { return q2s[a] < q2s[b]; });
  int local[64];
  for (int j = 0; j < kFusedBits; ++j) {
    out->qubits[j] = qs[j];
    local[qs[j]] = j;
  }
  out->gates.clear();
  for (const auto& g : lg) {
    if (g.nt == 0) continue;
    FusedGate f;
    std::memset(&f, 0, sizeof(f));
    f.nt = g.nt;
    f.t0 = local[g.targets[0]];
    f.t1 = g.nt > 1 ? local[g.targets[1]] : 0;
    for (int k = 0; k < g.nc; ++k) f.cmask |= 1 << local[g.controls[k]];
    const int d = g.nt == 1 ? 4 : 16;
    for (int k = 0; k < d; ++k) f.m[k] = make_double2(g.m[k].real(), g.m[k].imag());
    out->gates.push_back(f);
  }
  return HS_OK;
}

struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
};

int compose_all(int n, const std::vector<int>& q2s, const std::vector<int>& s2q,
                const hs_gate* gates, const int32_t* offs, int nparts, cudaStream_t s,
                std::vector<PartLocal>* parts, DevBuf* d_a, DevBuf* d_u) {
  parts->resize(nparts);
  std::vector<FusedGate> flat;
  std::vector<int32_t> foffs(nparts + 1, 0);
  for (int p = 0; p < nparts; ++p) {
    HS_TRY(localize(gates + offs[p], offs[p + 1] - offs[p], n, q2s, s2q, &(*parts)[p]));
    flat.insert(flat.end(), (*parts)[p].gates.begin(), (*parts)[p].gates.end());
    foffs[p + 1] = int32_t(flat.size());
  }
  DevBuf d_g, d_o;
  d_g.s = d_o.s = d_a->s = s;
  if (d_u) d_u->s = s;
  HS_CUDA(cudaMallocAsync(&d_g.p, sizeof(FusedGate) * std::max<size_t>(1, flat.size()), s));
  HS_CUDA(cudaMallocAsync(&d_o.p, sizeof(int32_t) * foffs.size(), s));
  HS_CUDA(cudaMallocAsync(&d_a->p, size_t(kFusedABytes) * nparts, s));
  if (d_u) HS_CUDA(cudaMallocAsync(&d_u->p, sizeof(double2) * kFusedDim * kFusedDim * nparts, s));
  if (!flat.empty())
    HS_CUDA(cudaMemcpyAsync(d_g.p, flat.data(), sizeof(FusedGate) * flat.size(),
                            cudaMemcpyHostToDevice, s));
  HS_CUDA(cudaMemcpyAsync(d_o.p, foffs.data(), sizeof(int32_t) * foffs.size(),
                          cudaMemcpyHostToDevice, s));
  HS_TRY(launch_compose(static_cast<FusedGate*>(d_g.p), static_cast<int32_t*>(d_o.p), nparts,
                        d_u ? static_cast<double2*>(d_u->p) : nullptr, d_a->p, s));
  // host vectors must outlive the async copies: wait here (the copies are tiny)
  HS_CUDA(cudaStreamSynchronize(s));
  return HS_OK;
}

void runs_of(const std::vector<int>& dst, Runs* r) {
  r->n = 0;
  size_t i = 0;
  while (i < dst.size()) {
    size_t j = i + 1;
    while (j < dst.size() && dst[j] == dst[j - 1] + 1) ++j;
    r->src[r->n] = uint8_t(i);
    r->len[r->n] = uint8_t(j - i);
    r->dst[r->n] = uint8_t(dst[i]);
    ++r->n;
    i = j;
  }
}

}  // namespace

// passes for the fused unitaries: consecutive parts whose slots (plus the two
// lowest slots) fit a tile of 2^12 amplitudes, at most kFusedMaxOps per pass
// pass shape: unitaries per state pass and tile bits (hs_set_fused_shape)
std::atomic<int> g_fused_ops{1}, g_fused_bits{13};

int plan_fused(int n, const std::vector<int>& q2s, const std::vector<PartLocal>& parts,
               int precision, std::vector<FusedPass>* out) {
  out->clear();
  const int mmax = std::min(n, g_fused_bits.load());
  const int max_ops = g_fused_ops.load();
  size_t p = 0;
  while (p < parts.size()) {
    std::vector<int> slots = {0, 1};
    size_t e = p;
    while (e < parts.size() && int(e - p) < max_ops) {
      std::vector<int> s2 = slots;
      for (int j = 0; j < kFusedBits; ++j) {
        const int sl = q2s[parts[e].qubits[j]];
        if (std::find(s2.begin(), s2.end(), sl) == s2.end()) s2.push_back(sl);
      }
      if (int(s2.size()) > mmax) break;
      slots = s2;
      ++e;
    }
    if (e == p) return set_error(HS_E_INVALID, "a fused part does not fit a tile");
    for (int sl = 2; sl < n && int(slots.size()) < mmax; ++sl)
      if (std::find(slots.begin(), slots.end(), sl) == slots.end()) slots.push_back(sl);
    std::sort(slots.begin(), slots.end());
    FusedPass P;
    std::memset(&P, 0, sizeof(P));
    P.n = n;
    P.m = int(slots.size());
    P.ntiles = 1ull << (n - P.m);
    P.precision = precision;
    runs_of(slots, &P.tile);
    std::vector<int> outer;
    for (int sl = 0; sl < n; ++sl)
      if (std::find(slots.begin(), slots.end(), sl) == slots.end()) outer.push_back(sl);
    runs_of(outer, &P.outer);
    P.nops = int(e - p);
    for (size_t k = p; k < e; ++k) {
      P.part[k - p] = int32_t(k);
      for (int j = 0; j < kFusedBits; ++j) {
        const int sl = q2s[parts[k].qubits[j]];
        P.pbits[k - p][j] = uint8_t(std::find(slots.begin(), slots.end(), sl) - slots.begin());
      }
    }
    out->push_back(P);
    p = e;
  }
  return HS_OK;
}

}  // namespace hisv

using namespace hisv;

extern "C" {

int hs_fused_parts_run(hs_state* st, const hs_gate* gates, const int32_t* part_offsets,
                       int num_parts, int precision, void* stream) {
  if (!st || !st->amp) return set_error(HS_E_INVALID, "null or destroyed state");
  if (st->dtype != HS_DTYPE_C64)
    return set_error(HS_E_UNSUPPORTED, "the fused form runs on complex64 states");
  if (st->n < 10) return set_error(HS_E_UNSUPPORTED, "the fused form needs at least 10 qubits");
  if (precision != HS_FUSED_BF16X3 && precision != HS_FUSED_BF16X1)
    return set_error(HS_E_INVALID, "unknown precision %d", precision);
  if (num_parts <= 0) return HS_OK;
  cudaStream_t s = S(stream);
  std::vector<PartLocal> parts;
  DevBuf d_a;
  HS_TRY(compose_all(st->n, st->q2s, st->s2q, gates, part_offsets, num_parts, s, &parts, &d_a,
                     nullptr));
  std::vector<FusedPass> passes;
  HS_TRY(plan_fused(st->n, st->q2s, parts, precision, &passes));
  DevBuf d_err;
  d_err.s = s;
  HS_CUDA(cudaMallocAsync(&d_err.p, sizeof(int), s));
  HS_CUDA(cudaMemsetAsync(d_err.p, 0, sizeof(int), s));
  {
    TimedRegion tr(s);
    for (const auto& P : passes) {
      HS_TRY(launch_fused(st->amp, P, d_a.p, static_cast<int*>(d_err.p), s));
      count_pass(P.nops);
    }
  }
  int err = 0;
  HS_CUDA(cudaMemcpyAsync(&err, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaStreamSynchronize(s));
  if (err) return set_error(HS_E_TIMEOUT, "a tensor-core wait in K4 timed out");
  return HS_OK;
}

int hs_fused_apply(hs_state* st, const double* u, const int32_t* qubits, int precision,
                   void* stream) {
  if (!st || !st->amp) return set_error(HS_E_INVALID, "null or destroyed state");
  if (st->dtype != HS_DTYPE_C64)
    return set_error(HS_E_UNSUPPORTED, "the fused form runs on complex64 states");
  if (st->n < 10) return set_error(HS_E_UNSUPPORTED, "the fused form needs at least 10 qubits");
  if (!u || !qubits) return set_error(HS_E_INVALID, "null unitary or qubit list");
  if (precision != HS_FUSED_BF16X3 && precision != HS_FUSED_BF16X1)
    return set_error(HS_E_INVALID, "unknown precision %d", precision);
  std::vector<PartLocal> parts(1);
  for (int j = 0; j < kFusedBits; ++j) {
    const int q = qubits[j];
    if (q < 0 || q >= st->n) return set_error(HS_E_INVALID, "qubit %d out of range", q);
    for (int k = 0; k < j; ++k)
      if (qubits[k] == q) return set_error(HS_E_INVALID, "qubit %d repeated", q);
    parts[0].qubits[j] = q;
  }
  const cudaStream_t s = S(stream);
  DevBuf d_u, d_a, d_err;
  d_u.s = d_a.s = d_err.s = s;
  HS_CUDA(cudaMallocAsync(&d_u.p, sizeof(double2) * kFusedDim * kFusedDim, s));
  HS_CUDA(cudaMallocAsync(&d_a.p, kFusedABytes, s));
  HS_CUDA(cudaMallocAsync(&d_err.p, sizeof(int), s));
  HS_CUDA(cudaMemcpyAsync(d_u.p, u, sizeof(double2) * kFusedDim * kFusedDim,
                          cudaMemcpyHostToDevice, s));
  HS_CUDA(cudaMemsetAsync(d_err.p, 0, sizeof(int), s));
  HS_TRY(launch_pack(static_cast<const double2*>(d_u.p), 1, d_a.p, s));
  std::vector<FusedPass> passes;
  HS_TRY(plan_fused(st->n, st->q2s, parts, precision, &passes));
  {
    TimedRegion tr(s);
    for (const auto& P : passes) {
      HS_TRY(launch_fused(st->amp, P, d_a.p, static_cast<int*>(d_err.p), s));
      count_pass(P.nops);
    }
  }
  int err = 0;
  HS_CUDA(cudaMemcpyAsync(&err, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  HS_CUDA(cudaStreamSynchronize(s));
  if (err) return set_error(HS_E_TIMEOUT, "a tensor-core wait in K4 timed out");
  return HS_OK;
}

int hs_set_k4_variant(int variant) {
  if (variant < 0 || variant > 2) return set_error(HS_E_INVALID, "K4 variant 0, 1 or 2");
  return set_k4_variant(variant);
}

int hs_set_fused_shape(int max_ops_per_pass, int tile_bits) {
  if (max_ops_per_pass < 1 || max_ops_per_pass > kFusedMaxOps || tile_bits < 10 ||
      tile_bits > (max_ops_per_pass == 1 ? 13 : 12))
    return set_error(HS_E_INVALID, "1 unitary per pass with 10..13 tile bits, or 2 with 10..12");
  const int prev = g_fused_ops.exchange(max_ops_per_pass) * 100 + g_fused_bits.exchange(tile_bits);
  return prev;
}

int hs_fused_compose(int num_qubits, const hs_gate* gates, const int32_t* part_offsets,
                     int num_parts, double* out_u, int32_t* out_qubits) {
  if (num_qubits < kFusedBits || num_qubits > 40)
    return set_error(HS_E_INVALID, "need 6..40 qubits");
  std::vector<int> q2s(num_qubits);
  for (int q = 0; q < num_qubits; ++q) q2s[q] = q;
  std::vector<PartLocal> parts;
  DevBuf d_a, d_u;
  HS_TRY(compose_all(num_qubits, q2s, q2s, gates, part_offsets, num_parts, nullptr, &parts, &d_a,
                     &d_u));
  HS_CUDA(cudaMemcpy(out_u, d_u.p, sizeof(double2) * kFusedDim * kFusedDim * num_parts,
                     cudaMemcpyDeviceToHost));
  for (int p = 0; p < num_parts; ++p)
    for (int j = 0; j < kFusedBits; ++j) out_qubits[p * kFusedBits + j] = parts[p].qubits[j];
  return HS_OK;
}

int hs_compare(hs_state* a, hs_state* b, double out[4]) {
  if (!a || !b || !a->amp || !b->amp) return set_error(HS_E_INVALID, "null state");
  if (a->n != b->n) return set_error(HS_E_INVALID, "qubit counts differ");
  if (a->q2s != b->q2s) {
    HS_TRY(hs_state_canonicalize(a, nullptr));
    HS_TRY(hs_state_canonicalize(b, nullptr));
  }
  return reduce_compare(a->amp, a->dtype, b->amp, b->dtype, a->n, out, nullptr);
}

int hs_compare_host(hs_state* a, const void* host_b, int bdtype, double out[4]) {
  if (!a || !a->amp || !host_b || !out) return set_error(HS_E_INVALID, "null argument");
  if (bdtype != HS_DTYPE_C128 && bdtype != HS_DTYPE_C64) return set_error(HS_E_INVALID, "bad dtype");
  HS_TRY(hs_state_canonicalize(a, nullptr));
  const uint64_t size = 1ull << a->n;
  const size_t bb = amp_bytes(bdtype), ab = amp_bytes(a->dtype);
  const uint64_t chunk = std::min<uint64_t>(size, 1ull << 26);
  DevBuf stage;
  HS_CUDA(cudaMallocAsync(&stage.p, chunk * bb, nullptr));
  double acc[4] = {0, 0, 0, 0};
  for (uint64_t first = 0; first < size; first += chunk) {
    HS_CUDA(cudaMemcpy(stage.p, static_cast<const char*>(host_b) + first * bb, chunk * bb,
                       cudaMemcpyHostToDevice));
    double part[4];
    HS_TRY(reduce_compare_count(static_cast<const char*>(a->amp) + first * ab, a->dtype, stage.p,
                                bdtype, chunk, part, nullptr));
    acc[0] += part[0];
    acc[1] += part[1];
    acc[2] = std::max(acc[2], part[2]);
    acc[3] += part[3];
  }
  for (int k = 0; k < 4; ++k) out[k] = acc[k];
  return HS_OK;
}

}  // extern "C"
