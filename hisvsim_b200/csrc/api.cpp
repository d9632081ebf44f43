// C ABI of libhisv (include/hisv.h): state management, the plain-form entry
// points, redistribution and reductions.  Every function returns a status and
// never aborts; messages are kept per calling thread.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <random>
#include <set>

#include "bounds.cuh"
#include "internal.h"

namespace hisv {

static thread_local char g_err[512] = "";

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

static std::atomic<long long> g_gates{0}, g_passes{0}, g_param_bytes{0};
static std::atomic<int> g_tile_hint{0};
int current_tile_hint() { return g_tile_hint.load(); }
static std::atomic<int> g_k1_rbits{4};
int k1_reg_bits(int dtype) { return dtype == HS_DTYPE_C128 ? g_k1_rbits.load() : kRegBits; }

// device-time accounting of K1/K2 launches: event pairs resolved when read
static std::mutex g_ev_mu;
static std::vector<std::pair<cudaEvent_t, cudaEvent_t>> g_events;
static std::atomic<long long> g_apply_us{0};
static std::atomic<int> g_timing{0};

int device_sms() {
  static std::mutex mu;
  static int cache[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  std::lock_guard<std::mutex> lk(mu);
  int& v = cache[dev & 63];
  if (v <= 0 && (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                 v <= 0))
    v = 148;
  return v;
}

int smem_optin(const void* func) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  HS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, func})) return HS_OK;
  HS_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  done.insert({dev, func});
  return HS_OK;
}

void count_pass(long long gates) {
  g_passes += 1;
  g_gates += gates;
}

TimedRegion::TimedRegion(cudaStream_t s_) : s(s_) {
  if (g_timing.load()) {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s);
  }
}

TimedRegion::~TimedRegion() {
  if (a) {
    cudaEventRecord(b, s);
    std::lock_guard<std::mutex> lk(g_ev_mu);
    g_events.emplace_back(a, b);
  }
}

namespace {

cudaStream_t S(void* stream) { return static_cast<cudaStream_t>(stream); }

int check_state(const hs_state* st) {
  if (!st || !st->amp) return set_error(HS_E_INVALID, "null or destroyed state");
  return HS_OK;
}

// Apply a permutation of bit positions to the data: the bit at position p
// moves to position pi[p].  Done as two in-place involution passes of K2:
// every cycle (c0 -> c1 -> ... ) is the product of two reflections.
int permute_positions(hs_state* st, const std::vector<int>& pi, cudaStream_t s) {
  const int n = st->n;
  std::vector<int> t1(n), t2(n);
  for (int p = 0; p < n; ++p) t1[p] = t2[p] = p;
  std::vector<bool> seen(n, false);
  for (int p = 0; p < n; ++p) {
    if (seen[p]) continue;
    std::vector<int> cyc;
    for (int q = p; !seen[q]; q = pi[q]) {
      seen[q] = true;
      cyc.push_back(q);
    }
    const int k = int(cyc.size());
    if (k < 2) continue;
    for (int i = 0; i < k; ++i) {
      t1[cyc[i]] = cyc[(k - i) % k];
      t2[cyc[i]] = cyc[(k + 1 - i) % k];
    }
  }
  for (const auto* t : {&t1, &t2}) {
    std::vector<int32_t> pairs;
    for (int p = 0; p < n; ++p)
      if ((*t)[p] > p) {
        pairs.push_back(p);
        pairs.push_back((*t)[p]);
      }
    if (pairs.empty()) continue;
    HS_TRY(launch_permute(st->amp, st->dtype, n, pairs.data(), int(pairs.size() / 2), s));
    count_pass(0);
  }
  std::vector<int> s2q(n);
  for (int p = 0; p < n; ++p) s2q[pi[p]] = st->s2q[p];
  st->s2q = s2q;
  for (int p = 0; p < n; ++p) st->q2s[s2q[p]] = p;
  return HS_OK;
}

int run_lowered(hs_state* st, const std::vector<LoweredGate>& lg, long long ngates,
                cudaStream_t s) {
  std::vector<PartProgram> progs;
  HS_TRY(plan_part(st->n, st->q2s, lg, g_tile_hint.load(), st->dtype, &progs));
  TimedRegion tr(s);
  for (const auto& p : progs) {
    HS_TRY(launch_part(st->amp, st->dtype, p, s));
    count_pass(p.nops);
    g_param_bytes += (long long)sizeof(PartProgram);
  }
  (void)ngates;
  return HS_OK;
}

int lower_all(const hs_state* st, const hs_gate* gates, int num, std::vector<LoweredGate>* out) {
  out->resize(num);
  for (int i = 0; i < num; ++i) HS_TRY(lower_gate(gates[i], st->n, &(*out)[i]));
  return HS_OK;
}

}  // namespace
}  // namespace hisv

using namespace hisv;

extern "C" {

const char* hs_last_error(void) { return g_err; }
int hs_version(void) { return 1; }

int hs_device_count(int* count) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) c = 0;
  if (count) *count = c;
  return HS_OK;
}

int hs_device_set(int device) {
  HS_CUDA(cudaSetDevice(device));
  return HS_OK;
}

int hs_device_synchronize(void) {
  HS_CUDA(cudaDeviceSynchronize());
  return HS_OK;
}

int hs_event_create(void** ev) {
  cudaEvent_t e;
  HS_CUDA(cudaEventCreate(&e));
  *ev = e;
  return HS_OK;
}

int hs_event_record(void* ev, void* stream) {
  HS_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(ev), S(stream)));
  return HS_OK;
}

int hs_event_elapsed_ms(void* start, void* stop, float* ms) {
  HS_CUDA(cudaEventSynchronize(static_cast<cudaEvent_t>(stop)));
  HS_CUDA(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start),
                               static_cast<cudaEvent_t>(stop)));
  return HS_OK;
}

int hs_event_destroy(void* ev) {
  if (ev) cudaEventDestroy(static_cast<cudaEvent_t>(ev));
  return HS_OK;
}

int hs_state_create(int num_qubits, int dtype, hs_state** out) {
  if (!out) return set_error(HS_E_INVALID, "null output pointer");
  *out = nullptr;
  if (num_qubits < 1 || num_qubits > 40)
    return set_error(HS_E_INVALID, "qubit count %d outside 1..40", num_qubits);
  if (dtype != HS_DTYPE_C128 && dtype != HS_DTYPE_C64)
    return set_error(HS_E_INVALID, "unknown dtype %d", dtype);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(HS_E_NODEVICE, "no CUDA device visible");
  }
  auto* st = new hs_state;
  st->n = num_qubits;
  st->dtype = dtype;
  const size_t bytes = amp_bytes(dtype) << num_qubits;
  cudaError_t e = cudaMalloc(&st->amp, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete st;
    return set_error(HS_E_NOMEM, "cudaMalloc of %zu bytes failed: %s", bytes,
                     cudaGetErrorString(e));
  }
  st->q2s.resize(num_qubits);
  st->s2q.resize(num_qubits);
  for (int q = 0; q < num_qubits; ++q) st->q2s[q] = st->s2q[q] = q;
  int rc = set_basis_kernel(st->amp, dtype, num_qubits, 0, nullptr);
  if (rc == HS_OK) {
    e = cudaStreamSynchronize(nullptr);
    if (e != cudaSuccess) rc = set_error(HS_E_CUDA, "init: %s", cudaGetErrorString(e));
  }
  if (rc != HS_OK) {
    cudaFree(st->amp);
    delete st;
    return rc;
  }
  *out = st;
  return HS_OK;
}

int hs_state_destroy(hs_state* st) {
  if (!st) return HS_OK;
  if (st->amp) cudaFree(st->amp);
  st->amp = nullptr;
  delete st;
  return HS_OK;
}

int hs_state_num_qubits(const hs_state* st, int* n) {
  HS_TRY(check_state(st));
  *n = st->n;
  return HS_OK;
}

int hs_state_dtype(const hs_state* st, int* dtype) {
  HS_TRY(check_state(st));
  *dtype = st->dtype;
  return HS_OK;
}

int hs_state_device_ptr(const hs_state* st, void** dptr) {
  HS_TRY(check_state(st));
  *dptr = st->amp;
  return HS_OK;
}

int hs_state_qubit_to_slot(const hs_state* st, int32_t* q2s) {
  HS_TRY(check_state(st));
  for (int q = 0; q < st->n; ++q) q2s[q] = st->q2s[q];
  return HS_OK;
}

int hs_state_set_basis(hs_state* st, uint64_t x, void* stream) {
  HS_TRY(check_state(st));
  if (st->n < 64 && (x >> st->n)) return set_error(HS_E_INVALID, "basis index out of range");
  for (int q = 0; q < st->n; ++q) st->q2s[q] = st->s2q[q] = q;
  return set_basis_kernel(st->amp, st->dtype, st->n, x, S(stream));
}

int hs_state_copy_to_host(hs_state* st, void* host, uint64_t first, uint64_t count,
                          void* stream) {
  HS_TRY(check_state(st));
  const uint64_t size = 1ull << st->n;
  if (first > size || count > size - first) return set_error(HS_E_INVALID, "range outside state");
  const size_t b = amp_bytes(st->dtype);
  HS_CUDA(cudaMemcpyAsync(host, static_cast<char*>(st->amp) + first * b, count * b,
                          cudaMemcpyDeviceToHost, S(stream)));
  HS_CUDA(cudaStreamSynchronize(S(stream)));
  return HS_OK;
}

int hs_state_copy_from_host(hs_state* st, const void* host, uint64_t first, uint64_t count,
                            void* stream) {
  HS_TRY(check_state(st));
  const uint64_t size = 1ull << st->n;
  if (first > size || count > size - first) return set_error(HS_E_INVALID, "range outside state");
  const size_t b = amp_bytes(st->dtype);
  HS_CUDA(cudaMemcpyAsync(static_cast<char*>(st->amp) + first * b, host, count * b,
                          cudaMemcpyHostToDevice, S(stream)));
  HS_CUDA(cudaStreamSynchronize(S(stream)));
  return HS_OK;
}

int hs_state_canonicalize(hs_state* st, void* stream) {
  HS_TRY(check_state(st));
  // the bit at slot p belongs to qubit s2q[p]; it must move to slot s2q[p]
  std::vector<int> pi(st->s2q.begin(), st->s2q.end());
  bool ident = true;
  for (int p = 0; p < st->n; ++p) ident &= pi[p] == p;
  if (ident) return HS_OK;
  return permute_positions(st, pi, S(stream));
}

int hs_state_convert(const hs_state* src, hs_state* dst, void* stream) {
  HS_TRY(check_state(src));
  HS_TRY(check_state(dst));
  if (src->n != dst->n) return set_error(HS_E_INVALID, "qubit counts differ");
  HS_TRY(convert_kernel(src->amp, src->dtype, dst->amp, dst->dtype, 1ull << src->n,
                        S(stream)));
  dst->q2s = src->q2s;
  dst->s2q = src->s2q;
  return HS_OK;
}

int hs_gate_apply(hs_state* st, const hs_gate* gate, void* stream) {
  HS_TRY(check_state(st));
  if (!gate) return set_error(HS_E_INVALID, "null gate");
  std::vector<LoweredGate> lg;
  HS_TRY(lower_all(st, gate, 1, &lg));
  return run_lowered(st, lg, 1, S(stream));
}

int hs_part_run(hs_state* st, const hs_gate* gates, int num_gates, void* stream) {
  HS_TRY(check_state(st));
  if (num_gates < 0 || (num_gates > 0 && !gates)) return set_error(HS_E_INVALID, "bad gate list");
  if (num_gates == 0) return HS_OK;
  std::vector<LoweredGate> lg;
  HS_TRY(lower_all(st, gates, num_gates, &lg));
  return run_lowered(st, lg, num_gates, S(stream));
}

int hs_frames_create(int num_qubits, hs_frames** out) {
  if (!out) return set_error(HS_E_INVALID, "null output pointer");
  if (num_qubits < 1 || num_qubits > 63) return set_error(HS_E_INVALID, "bad qubit count %d", num_qubits);
  hs_frames* f = new (std::nothrow) hs_frames;
  if (!f) return set_error(HS_E_NOMEM, "frames");
  f->n = num_qubits;
  f->fr.reset(num_qubits);
  *out = f;
  return HS_OK;
}

int hs_frames_destroy(hs_frames* fr) {
  delete fr;
  return HS_OK;
}

int hs_frames_pending(const hs_frames* fr, int* pending) {
  if (!fr || !pending) return set_error(HS_E_INVALID, "null argument");
  *pending = fr->fr.identity() ? 0 : 1;
  return HS_OK;
}

int hs_part_run_carry(hs_state* st, hs_frames* fr, const hs_gate* gates, int num_gates,
                      void* stream) {
  HS_TRY(check_state(st));
  if (!fr || fr->n != st->n) return set_error(HS_E_INVALID, "frames missing or of another size");
  if (num_gates < 0 || (num_gates > 0 && !gates)) return set_error(HS_E_INVALID, "bad gate list");
  if (num_gates == 0) return HS_OK;
  std::vector<LoweredGate> lg;
  HS_TRY(lower_all(st, gates, num_gates, &lg));
  std::vector<PartProgram> progs;
  HS_TRY(plan_gates(st->n, st->q2s, lg, &fr->fr, false, g_tile_hint.load(), st->dtype, &progs));
  TimedRegion tr(S(stream));
  for (const auto& pr : progs) {
    HS_TRY(launch_part(st->amp, st->dtype, pr, S(stream)));
    count_pass(pr.nops);
    g_param_bytes += (long long)sizeof(PartProgram);
  }
  return HS_OK;
}

int hs_frames_flush(hs_state* st, hs_frames* fr, void* stream) {
  HS_TRY(check_state(st));
  if (!fr || fr->n != st->n) return set_error(HS_E_INVALID, "frames missing or of another size");
  if (fr->fr.identity()) return HS_OK;
  std::vector<PartProgram> progs;
  HS_TRY(plan_gates(st->n, st->q2s, {}, &fr->fr, true, g_tile_hint.load(), st->dtype, &progs));
  TimedRegion tr(S(stream));
  for (const auto& pr : progs) {
    HS_TRY(launch_part(st->amp, st->dtype, pr, S(stream)));
    count_pass(pr.nops);
    g_param_bytes += (long long)sizeof(PartProgram);
  }
  return HS_OK;
}

int hs_parts_run(hs_state* st, const hs_gate* gates, const int32_t* part_offsets,
                 int num_parts, void* stream) {
  HS_TRY(check_state(st));
  if (num_parts < 0 || (num_parts > 0 && (!gates || !part_offsets)))
    return set_error(HS_E_INVALID, "bad part list");
  for (int p = 0; p < num_parts; ++p) {
    if (part_offsets[p + 1] < part_offsets[p] || part_offsets[p] < 0)
      return set_error(HS_E_INVALID, "part offsets must be non-decreasing");
  }
  // lower everything first so that a bad gate leaves the state untouched
  std::vector<std::vector<LoweredGate>> all(num_parts);
  for (int p = 0; p < num_parts; ++p)
    HS_TRY(lower_all(st, gates + part_offsets[p], part_offsets[p + 1] - part_offsets[p],
                     &all[p]));
  // one pass (or more) per part; the pending diagonal of the factored
  // rotations is carried from part to part and applied by the last one
  Frames fr;
  fr.reset(st->n);
  std::vector<PartProgram> progs;
  for (int p = 0; p < num_parts; ++p) {
    HS_TRY(plan_gates(st->n, st->q2s, all[p], &fr, p == num_parts - 1, g_tile_hint.load(),
                      st->dtype, &progs));
    TimedRegion tr(S(stream));
    for (const auto& pr : progs) {
      HS_TRY(launch_part(st->amp, st->dtype, pr, S(stream)));
      count_pass(pr.nops);
      g_param_bytes += (long long)sizeof(PartProgram);
    }
  }
  return HS_OK;
}

int hs_parts_run_timed(hs_state* st, const hs_gate* gates, const int32_t* part_offsets,
                       int num_parts, float* part_ms, void* stream) {
  HS_TRY(check_state(st));
  if (num_parts < 0 || (num_parts > 0 && (!gates || !part_offsets || !part_ms)))
    return set_error(HS_E_INVALID, "bad part list");
  for (int p = 0; p < num_parts; ++p)
    if (part_offsets[p + 1] < part_offsets[p] || part_offsets[p] < 0)
      return set_error(HS_E_INVALID, "part offsets must be non-decreasing");
  // plan every part before the first launch, so that the device never waits
  // for the host between two parts and each event pair brackets one part only
  std::vector<std::vector<PartProgram>> progs(num_parts);
  Frames fr;
  fr.reset(st->n);
  for (int p = 0; p < num_parts; ++p) {
    std::vector<LoweredGate> lg;
    HS_TRY(lower_all(st, gates + part_offsets[p], part_offsets[p + 1] - part_offsets[p], &lg));
    HS_TRY(plan_gates(st->n, st->q2s, lg, &fr, p == num_parts - 1, g_tile_hint.load(),
                      st->dtype, &progs[p]));
  }
  std::vector<cudaEvent_t> ev(num_parts + 1, nullptr);
  int rc = HS_OK;
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) rc = set_error(HS_E_CUDA, "event create");
  const cudaStream_t s = S(stream);
  if (rc == HS_OK && cudaEventRecord(ev[0], s) != cudaSuccess)
    rc = set_error(HS_E_CUDA, "event record");
  for (int p = 0; p < num_parts && rc == HS_OK; ++p) {
    for (const auto& pr : progs[p]) {
      if ((rc = launch_part(st->amp, st->dtype, pr, s)) != HS_OK) break;
      count_pass(pr.nops);
    }
    if (rc == HS_OK && cudaEventRecord(ev[p + 1], s) != cudaSuccess)
      rc = set_error(HS_E_CUDA, "event record");
  }
  if (rc == HS_OK && cudaStreamSynchronize(s) != cudaSuccess)
    rc = set_error(HS_E_CUDA, "synchronize");
  for (int p = 0; p < num_parts && rc == HS_OK; ++p)
    if (cudaEventElapsedTime(&part_ms[p], ev[p], ev[p + 1]) != cudaSuccess)
      rc = set_error(HS_E_CUDA, "elapsed time");
  for (auto& e : ev)
    if (e) cudaEventDestroy(e);
  return rc;
}

int hs_plan_stats(int num_qubits, int dtype, const hs_gate* gates, int num_gates,
                  int32_t* stats) {
  if (num_qubits < 1 || num_qubits > 40) return set_error(HS_E_INVALID, "bad qubit count");
  if (dtype != HS_DTYPE_C128 && dtype != HS_DTYPE_C64) return set_error(HS_E_INVALID, "bad dtype");
  std::vector<LoweredGate> lg(num_gates);
  for (int i = 0; i < num_gates; ++i) HS_TRY(lower_gate(gates[i], num_qubits, &lg[i]));
  std::vector<int> q2s(num_qubits);
  for (int q = 0; q < num_qubits; ++q) q2s[q] = q;
  std::vector<PartProgram> progs;
  HS_TRY(plan_part(num_qubits, q2s, lg, g_tile_hint.load(), dtype, &progs));
  int32_t groups = 0, ops = 0, diag = 0, dense = 0, m = 0;
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
  stats[0] = int32_t(progs.size());
  stats[1] = groups;
  stats[2] = ops;
  stats[3] = dense;
  stats[4] = diag;
  stats[5] = m;
  return HS_OK;
}

int hs_set_tile_qubits(int m) {
  if (m < 0 || m > kMaxTileBits) return set_error(HS_E_INVALID, "tile bits must be 0..%d",
                                                  kMaxTileBits);
  return g_tile_hint.exchange(m);
}

int hs_set_k1_reg_bits(int r) {
  if (r != 3 && r != 4) return set_error(HS_E_INVALID, "K1 register bits must be 3 or 4");
  return g_k1_rbits.exchange(r);
}

int hs_permute_bits(hs_state* st, const int32_t* pairs, int num_pairs, void* stream) {
  HS_TRY(check_state(st));
  std::vector<int> pi(st->n);
  for (int p = 0; p < st->n; ++p) pi[p] = p;
  for (int i = 0; i < num_pairs; ++i) {
    const int a = pairs[2 * i], b = pairs[2 * i + 1];
    if (a < 0 || b < 0 || a >= st->n || b >= st->n || a == b || pi[a] != a || pi[b] != b)
      return set_error(HS_E_INVALID, "bit pairs must be distinct, disjoint slots");
    pi[a] = b;
    pi[b] = a;
  }
  if (num_pairs == 0) return HS_OK;
  TimedRegion tr(S(stream));
  HS_TRY(launch_permute(st->amp, st->dtype, st->n, pairs, num_pairs, S(stream)));
  count_pass(0);
  std::vector<int> s2q(st->n);
  for (int p = 0; p < st->n; ++p) s2q[pi[p]] = st->s2q[p];
  st->s2q = s2q;
  for (int p = 0; p < st->n; ++p) st->q2s[s2q[p]] = p;
  return HS_OK;
}

int hs_gather_qubits(hs_state* st, const int32_t* proc_qubits, int num, void* stream) {
  HS_TRY(check_state(st));
  std::vector<bool> is_proc(st->n, false);
  for (int i = 0; i < num; ++i) {
    const int q = proc_qubits[i];
    if (q < 0 || q >= st->n || is_proc[q]) return set_error(HS_E_INVALID, "bad proc qubit set");
    is_proc[q] = true;
  }
  // new slot order (svsim-mpi.hpp:141-152): non-proc qubits in slot order,
  // then the proc qubits in slot order
  std::vector<int> order;
  for (int p = 0; p < st->n; ++p)
    if (!is_proc[st->s2q[p]]) order.push_back(p);
  for (int p = 0; p < st->n; ++p)
    if (is_proc[st->s2q[p]]) order.push_back(p);
  std::vector<int> pi(st->n);
  for (int j = 0; j < st->n; ++j) pi[order[j]] = j;
  TimedRegion tr(S(stream));
  return permute_positions(st, pi, S(stream));
}

int hs_project(hs_state* st, const int32_t* qubits, const int32_t* values, int count,
               int norm_mode, hs_state** out, double* prob_out, void* stream) {
  HS_TRY(check_state(st));
  if (!out) return set_error(HS_E_INVALID, "null output pointer");
  *out = nullptr;
  if (count < 1 || count >= st->n || !qubits)
    return set_error(HS_E_INVALID, "project 1..%d of %d qubits", st->n - 1, st->n);
  if (norm_mode < 0 || norm_mode > 2) return set_error(HS_E_INVALID, "norm mode 0, 1 or 2");
  std::vector<char> used(st->n, 0);
  uint64_t offset = 0;
  for (int i = 0; i < count; ++i) {
    const int q = qubits[i], v = values ? values[i] : 0;
    if (q < 0 || q >= st->n || used[q]) return set_error(HS_E_INVALID, "bad or repeated qubit");
    if (v != 0 && v != 1) return set_error(HS_E_INVALID, "values must be 0 or 1");
    used[q] = 1;
    offset |= uint64_t(v) << st->q2s[q];
  }
  std::vector<int> slots;
  for (int q = 0; q < st->n; ++q)
    if (!used[q]) slots.push_back(st->q2s[q]);
  hs_state* ns = nullptr;
  HS_TRY(hs_state_create(st->n - count, st->dtype, &ns));
  const cudaStream_t s = S(stream);
  double p = 0;
  int rc = project_kernel(st->amp, ns->amp, st->dtype, ns->n, slots.data(), offset, s);
  if (rc == HS_OK) rc = reduce_norm2(ns->amp, ns->dtype, ns->n, &p, s);
  // the reference divides by p (state_vector.hpp:867-882) and skips p <= 1e-12
  if (rc == HS_OK && norm_mode != 2 && p > 1e-12)
    rc = scale_kernel(ns->amp, ns->dtype, ns->n, norm_mode == 0 ? 1.0 / std::sqrt(p) : 1.0 / p,
                      s);
  if (rc == HS_OK && cudaStreamSynchronize(s) != cudaSuccess)
    rc = set_error(HS_E_CUDA, "project: synchronize");
  if (rc != HS_OK) {
    hs_state_destroy(ns);
    return rc;
  }
  if (prob_out) *prob_out = p;
  *out = ns;
  return HS_OK;
}

int hs_bounds_status(uint32_t* flags, int reset) {
  if (!flags) return set_error(HS_E_INVALID, "null output");
  *flags = 0;
#ifdef HS_BOUNDS
  HS_CUDA(cudaDeviceSynchronize());
  *flags = bounds_take_part(reset) | bounds_take_misc(reset) | bounds_take_fused(reset) |
           bounds_take_batch(reset);
  return HS_OK;
#else
  (void)reset;
  return set_error(HS_E_UNSUPPORTED, "this library was built without index checks");
#endif
}

int hs_fp64_peak(double* tflops) {
  if (!tflops) return set_error(HS_E_INVALID, "null output");
  return fp64_probe(tflops);
}

int hs_norm2(hs_state* st, double* out) {
  HS_TRY(check_state(st));
  return reduce_norm2(st->amp, st->dtype, st->n, out, nullptr);
}

static int align_maps(hs_state* a, hs_state* b) {
  HS_TRY(check_state(a));
  HS_TRY(check_state(b));
  if (a->n != b->n || a->dtype != b->dtype)
    return set_error(HS_E_INVALID, "states differ in qubit count or dtype");
  if (a->q2s != b->q2s) {
    // move b's bits to a's layout: the bit of qubit q goes from b->q2s[q] to a->q2s[q]
    std::vector<int> pi(b->n);
    for (int q = 0; q < b->n; ++q) pi[b->q2s[q]] = a->q2s[q];
    HS_TRY(permute_positions(b, pi, nullptr));
  }
  return HS_OK;
}

int hs_inner(hs_state* a, hs_state* b, double out[2]) {
  HS_TRY(align_maps(a, b));
  return reduce_inner(a->amp, b->amp, a->dtype, a->n, out, nullptr);
}

int hs_max_abs_diff(hs_state* a, hs_state* b, double* out) {
  HS_TRY(align_maps(a, b));
  return reduce_maxdiff(a->amp, b->amp, a->dtype, a->n, out, nullptr);
}

int hs_probability(hs_state* st, int qubit, int value, double* out) {
  HS_TRY(check_state(st));
  if (qubit < 0 || qubit >= st->n) return set_error(HS_E_INVALID, "operation on an unallocated qubit");
  if (value != 0 && value != 1) return set_error(HS_E_INVALID, "value must be 0 or 1");
  double p0 = 0;
  HS_TRY(reduce_prob0(st->amp, st->dtype, st->n, st->q2s[qubit], &p0, nullptr));
  *out = value == 0 ? p0 : 1.0 - p0;  // state_vector.hpp:918-922
  return HS_OK;
}

int hs_expect_zz(hs_state* st, const int32_t* pairs, int num_pairs, double* out) {
  HS_TRY(check_state(st));
  std::vector<int32_t> sp(2 * num_pairs);
  for (int i = 0; i < 2 * num_pairs; ++i) {
    if (pairs[i] < 0 || pairs[i] >= st->n) return set_error(HS_E_INVALID, "bad qubit");
    sp[i] = st->q2s[pairs[i]];
  }
  return reduce_zz(st->amp, st->dtype, st->n, sp.data(), num_pairs, out, nullptr);
}

int hs_measure(hs_state* st, const int32_t* qubits, int num_qubits, uint32_t num_samples,
               uint64_t seed, int32_t* out) {
  HS_TRY(check_state(st));
  if (num_samples == 0) return HS_OK;
  std::vector<int> slots(num_qubits);
  for (int j = 0; j < num_qubits; ++j) {
    if (qubits[j] < 0 || qubits[j] >= st->n)
      return set_error(HS_E_INVALID, "operation on an unallocated qubit");
    slots[j] = st->q2s[qubits[j]];
  }
  // sorted uniform samples walked against the cumulative distribution in
  // slot order, as measure() does (state_vector.hpp:935-967)
  std::mt19937 gen(uint32_t(seed ^ (seed >> 32)));
  std::uniform_real_distribution<> dis(0.0, 1.0);
  std::vector<double> u(num_samples);
  for (auto& x : u) x = dis(gen);
  std::sort(u.begin(), u.end());
  const int cb = std::min(st->n, 16);
  std::vector<double> chunk(size_t(1) << (st->n - cb));
  HS_TRY(reduce_chunks(st->amp, st->dtype, st->n, cb, chunk.data(), nullptr));
  const size_t b = amp_bytes(st->dtype);
  std::vector<char> host((size_t(1) << cb) * b);
  uint32_t k = 0;
  double cum = 0;
  auto emit = [&](uint64_t pos) {
    for (int j = 0; j < num_qubits; ++j) out[size_t(k) * num_qubits + j] = int32_t((pos >> slots[j]) & 1);
    ++k;
  };
  for (size_t c = 0; c < chunk.size() && k < num_samples; ++c) {
    if (u[k] >= cum + chunk[c]) {
      cum += chunk[c];
      continue;
    }
    const uint64_t first = uint64_t(c) << cb;
    HS_CUDA(cudaMemcpy(host.data(), static_cast<char*>(st->amp) + first * b, host.size(),
                       cudaMemcpyDeviceToHost));
    for (uint64_t i = 0; i < (1ull << cb) && k < num_samples; ++i) {
      double re, im;
      if (st->dtype == HS_DTYPE_C128) {
        re = reinterpret_cast<double*>(host.data())[2 * i];
        im = reinterpret_cast<double*>(host.data())[2 * i + 1];
      } else {
        re = reinterpret_cast<float*>(host.data())[2 * i];
        im = reinterpret_cast<float*>(host.data())[2 * i + 1];
      }
      const double p = re * re + im * im;
      while (k < num_samples && u[k] < cum + p) emit(first + i);
      cum += p;
    }
  }
  // samples beyond the accumulated mass read as all ones (state_vector.hpp:969-978)
  for (; k < num_samples; ++k)
    for (int j = 0; j < num_qubits; ++j) out[size_t(k) * num_qubits + j] = 1;
  return HS_OK;
}

int hs_counters(long long* apply_us, long long* gate_count, long long* pass_count) {
  {
    std::lock_guard<std::mutex> lk(g_ev_mu);
    for (auto& ev : g_events) {
      float ms = 0;
      if (cudaEventSynchronize(ev.second) == cudaSuccess &&
          cudaEventElapsedTime(&ms, ev.first, ev.second) == cudaSuccess)
        g_apply_us += (long long)(ms * 1000.0f);
      cudaEventDestroy(ev.first);
      cudaEventDestroy(ev.second);
    }
    g_events.clear();
  }
  if (apply_us) *apply_us = g_apply_us.load();
  if (gate_count) *gate_count = g_gates.load();
  if (pass_count) *pass_count = g_passes.load();
  return HS_OK;
}

int hs_counters_reset(void) {
  long long dummy;
  hs_counters(&dummy, nullptr, nullptr);
  g_apply_us = 0;
  g_gates = 0;
  g_passes = 0;
  g_param_bytes = 0;
  return HS_OK;
}

int hs_launch_bytes(long long* bytes) {
  if (bytes) *bytes = g_param_bytes.load();
  return HS_OK;
}

int hs_set_timing(int on) { return g_timing.exchange(on ? 1 : 0); }

}  // extern "C"
