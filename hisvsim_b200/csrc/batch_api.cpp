// Host side of the batching form (hs_batch_*): instance layout, pass planning,
// the work queue, CUDA-graph capture of one whole batch run, and the
// autotuner that picks the tile size and the CTA count by timing.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace hisv;

struct hs_batch {
  int ninst = 0, p = 0, max_n = 0;
  std::vector<int> n;
  std::vector<std::vector<std::pair<int, int>>> edges;
  std::vector<double> gammas, betas;
  int tile_cap = 11, ctas_per_sm = 16, chunk = 8;
  int threads = 128;  // CTA size of the plan: 256 once some tile has 2^12 amplitudes
  int low_keep = 3;  // lowest qubits kept in every later pass's tile (contiguous runs)
  int cap_of_n[kBatchMaxQubits + 1] = {};  // per qubit count; 0 = tile_cap
  void* pool = nullptr;
  std::vector<uint64_t> offset;  // amplitude offset of each instance in the pool
  BatchInstance* d_inst = nullptr;
  BatchParams* d_par = nullptr;
  BatchItem* d_items = nullptr;
  uint32_t* d_counters = nullptr;
  uint8_t* d_cut = nullptr;
  unsigned long long* d_head = nullptr;
  int* d_err = nullptr;
  uint32_t* d_limit = nullptr;   // polls of a dependency wait before it gives up
  std::vector<BatchItem> items;  // the planned work items (host copy)
  double* d_partial = nullptr;
  double* d_expect = nullptr;
  double* h_expect = nullptr;
  int* h_err = nullptr;
  int ngroups = 0;
  uint64_t total = 0, ncounters = 0, pass_bytes = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

void free_plan(hs_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  for (void* p : {(void*)b->d_inst, (void*)b->d_items, (void*)b->d_counters, (void*)b->d_partial,
                  (void*)b->d_cut})
    if (p) cudaFree(p);
  b->d_cut = nullptr;
  b->d_inst = nullptr;
  b->d_items = nullptr;
  b->d_counters = nullptr;
  b->d_partial = nullptr;
}

void runs(const std::vector<int>& dst, Runs* r) {
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

// Passes of one round for n qubits with tiles of at most `cap` bits: pass 0
// takes qubits [0, cap) (its RX targets); later passes keep the `low` lowest
// qubits for contiguity and mix the next cap-low qubits.
void round_passes(int n, int cap, int low, std::vector<std::vector<int>>* tiles,
                  std::vector<std::vector<int>>* targets) {
  tiles->clear();
  targets->clear();
  if (n <= cap) {
    std::vector<int> all;
    for (int q = 0; q < n; ++q) all.push_back(q);
    tiles->push_back(all);
    targets->push_back(all);
    return;
  }
  std::vector<int> t0;
  for (int q = 0; q < cap; ++q) t0.push_back(q);
  tiles->push_back(t0);
  targets->push_back(t0);
  int covered = cap;
  while (covered < n) {
    const int nw = std::min(cap - low, n - covered);
    std::vector<int> tl, tg;
    for (int q = 0; q < low; ++q) tl.push_back(q);
    for (int q = covered; q < covered + nw; ++q) {
      tl.push_back(q);
      tg.push_back(q);
    }
    // widen the tile with the next-lowest qubits (no gate on them in this
    // pass): fewer, larger tiles and longer contiguous runs
    for (int q = low; q < n && int(tl.size()) < cap; ++q)
      if (std::find(tl.begin(), tl.end(), q) == tl.end()) tl.push_back(q);
    std::sort(tl.begin(), tl.end());
    tiles->push_back(tl);
    targets->push_back(tg);
    covered += nw;
  }
}

// cut of the edges with both ends in the tile, for every tile index x < 2^m
// (tile bit b is qubit tl[b])
void cut_table(const std::vector<std::pair<int, int>>& edges, const std::vector<int>& tl,
               uint8_t* out) {
  std::vector<std::pair<int, int>> in;
  auto bit_of = [&](int q) { return int(std::find(tl.begin(), tl.end(), q) - tl.begin()); };
  for (const auto& e : edges) {
    const int a = bit_of(e.first), b = bit_of(e.second);
    if (a < int(tl.size()) && b < int(tl.size())) in.push_back({a, b});
  }
  for (uint32_t x = 0; x < (1u << tl.size()); ++x) {
    int c = 0;
    for (const auto& e : in) c += int(((x >> e.first) ^ (x >> e.second)) & 1u);
    out[x] = uint8_t(c);
  }
}

// kinds of pass: the first of the circuit (phase, then RX of its round), a
// plain mixer pass, and a pass that ends one round and starts the next
enum StepKind { kFirst, kMix, kJoin };

// All steps of an instance: p rounds of the round's passes.  Round r+1 runs
// the passes in the opposite order of round r, so the pass that ends round
// r is also the one that starts round r+1, and the two share one state pass
// (RX of round r, cost phase and RX of round r+1 in one visit of the tile):
// np + (p-1)(np-1) steps instead of p np.  With a single pass per round every
// step is phase + RX of its round.
int plan_steps(int n, int cap, int low, int p, const std::vector<std::pair<int, int>>& edges,
               BatchInstance* I, std::vector<uint8_t>* cut) {
  std::vector<std::vector<int>> tiles, targets;
  round_passes(n, cap, low, &tiles, &targets);
  const int np = int(tiles.size());
  if (np > kBatchMaxPasses)
    return set_error(HS_E_UNSUPPORTED, "%d qubits need %d passes with %d-qubit tiles (max %d)", n, np,
                     cap, kBatchMaxPasses);
  struct Step {
    int pass, kind, ra, rb;
  };
  std::vector<Step> steps;
  if (np == 1) {
    for (int r = 0; r < p; ++r) steps.push_back({0, kFirst, r, r});
  } else {
    std::vector<int> order(np);
    for (int j = 0; j < np; ++j) order[j] = j;
    steps.push_back({order[0], kFirst, 0, 0});
    for (int r = 0; r < p; ++r) {
      for (int j = 1; j < np - 1; ++j) steps.push_back({order[j], kMix, r, r});
      if (r + 1 < p) {
        steps.push_back({order[np - 1], kJoin, r, r + 1});
        std::reverse(order.begin(), order.end());
      } else {
        steps.push_back({order[np - 1], kMix, r, r});
      }
    }
  }
  if (int(steps.size()) > kBatchMaxSteps)
    return set_error(HS_E_UNSUPPORTED, "%d qubits x %d rounds need %d passes (max %d)", n, p,
                     int(steps.size()), kBatchMaxSteps);
  I->nsteps = int(steps.size());
  cut->clear();
  for (int k = 0; k < I->nsteps; ++k) {
    const Step& st = steps[k];
    BatchPass& P = I->pass[k];
    std::memset(&P, 0, sizeof(P));
    const std::vector<int>& tl = tiles[st.pass];
    P.m = int(tl.size());
    runs(tl, &P.tile);
    for (int b = 0; b < P.m; ++b) P.tile_slot[b] = uint8_t(tl[b]);
    for (int q = 0; q < kBatchMaxQubits; ++q) P.tbit[q] = -1;
    for (int b = 0; b < P.m; ++b) P.tbit[tl[b]] = int8_t(b);
    std::vector<int> outer;
    for (int q = 0; q < n; ++q)
      if (std::find(tl.begin(), tl.end(), q) == tl.end()) outer.push_back(q);
    runs(outer, &P.outer);
    std::vector<int> tb;  // target tile bits
    for (int q : targets[st.pass]) tb.push_back(int(std::find(tl.begin(), tl.end(), q) - tl.begin()));
    P.ngroups = int((tb.size() + 3) / 4);
    uint8_t gmask[3] = {0, 0, 0};
    for (int g = 0; g < P.ngroups; ++g) {
      std::vector<int> regs;
      for (size_t x = 4 * g; x < tb.size() && regs.size() < 4; ++x) regs.push_back(tb[x]);
      gmask[g] = uint8_t((1 << regs.size()) - 1);
      for (int b = P.m - 1; b >= 0 && regs.size() < 4; --b)
        if (std::find(regs.begin(), regs.end(), b) == regs.end()) regs.push_back(b);
      for (int j = 0; j < 4; ++j) P.group_bits[g][j] = uint8_t(regs[j]);
    }
    P.ra = uint8_t(st.ra);
    P.rb = uint8_t(st.rb);
    const int G = P.ngroups;
    auto visit = [&](int g, uint8_t a, uint8_t ph, uint8_t b) {
      const int v = P.nvisits++;
      P.visit_group[v] = uint8_t(g);
      P.rx_a[v] = a;
      P.ph[v] = ph;
      P.rx_b[v] = b;
    };
    if (st.kind == kFirst) {
      for (int g = 0; g < G; ++g) visit(g, 0, g == 0, gmask[g]);
    } else if (st.kind == kMix) {
      for (int g = 0; g < G; ++g) visit(g, gmask[g], 0, 0);
    } else {
      for (int g = 0; g < G - 1; ++g) visit(g, gmask[g], 0, 0);
      visit(G - 1, gmask[G - 1], 1, gmask[G - 1]);
      for (int g = G - 2; g >= 0; --g) visit(g, 0, 0, gmask[g]);
    }
    P.phase = st.kind != kMix;
    if (P.phase) {
      cut->resize((cut->size() + 15) & ~size_t(15));  // 16-byte aligned tables
      P.cut_off = uint32_t(cut->size());
      cut->resize(cut->size() + (size_t(1) << P.m));
      cut_table(edges, tl, cut->data() + P.cut_off);
    }
  }
  return HS_OK;
}

int upload_params(hs_batch* b) {
  std::vector<BatchParams> par(b->ninst);
  std::memset(par.data(), 0, sizeof(BatchParams) * par.size());
  for (int i = 0; i < b->ninst; ++i) {
    const int ne = int(b->edges[i].size());
    for (int r = 0; r < b->p; ++r) {
      const double beta = b->betas[size_t(i) * b->p + r], gamma = b->gammas[size_t(i) * b->p + r];
      // RX(2 beta): cos(beta), -i sin(beta); RZZ(gamma) on every edge
      par[i].rx[r][0] = make_float2(float(std::cos(beta)), float(std::sin(beta)));
      for (int c = 0; c <= ne; ++c) {
        const double ang = 0.5 * gamma * (2.0 * c - ne);
        par[i].phase[r][c] = make_float2(float(std::cos(ang)), float(std::sin(ang)));
      }
    }
  }
  HS_CUDA(cudaMemcpy(b->d_par, par.data(), sizeof(BatchParams) * par.size(),
                     cudaMemcpyHostToDevice));
  return HS_OK;
}

int build_plan(hs_batch* b) {
  free_plan(b);
  std::vector<BatchInstance> inst(b->ninst);
  std::memset(inst.data(), 0, sizeof(BatchInstance) * inst.size());
  uint64_t nc = 0;
  int maxsteps = 0;
  b->pass_bytes = 0;
  std::vector<size_t> cut_off(b->ninst);
  std::vector<uint8_t> cut, icut;
  int max_m = 0;
  for (int i = 0; i < b->ninst; ++i) {
    BatchInstance& I = inst[i];
    I.amp = static_cast<float2*>(b->pool) + b->offset[i];
    I.n = b->n[i];
    I.p = b->p;
    I.nedges = int(b->edges[i].size());
    for (int e = 0; e < I.nedges; ++e) {
      I.edge_a[e] = uint8_t(b->edges[i][e].first);
      I.edge_b[e] = uint8_t(b->edges[i][e].second);
    }
    HS_TRY(plan_steps(I.n, b->cap_of_n[I.n] ? b->cap_of_n[I.n] : b->tile_cap, b->low_keep, b->p,
                      b->edges[i], &I, &icut));
    for (int j = 0; j < I.nsteps; ++j) max_m = std::max(max_m, int(I.pass[j].m));
    I.step_base = nc;
    const int steps = I.nsteps;
    nc += uint64_t(steps);
    maxsteps = std::max(maxsteps, steps);
    for (int k = 0; k < steps; ++k) b->pass_bytes += 2ull * (8ull << I.n);
    // 16-byte aligned tables (the kernel stages them with 16-byte loads)
    cut_off[i] = cut.size();
    cut.insert(cut.end(), icut.begin(), icut.end());
    cut.resize((cut.size() + 15) & ~size_t(15));
  }
  b->threads = max_m > 11 ? 256 : 128;
  HS_CUDA(cudaMalloc(&b->d_cut, cut.size()));
  HS_CUDA(cudaMemcpy(b->d_cut, cut.data(), cut.size(), cudaMemcpyHostToDevice));
  for (int i = 0; i < b->ninst; ++i) inst[i].cut = b->d_cut + cut_off[i];
  // work items: per step level, per instance, the step's tiles in chunks
  std::vector<BatchItem> items;
  std::vector<uint32_t> prev_chunks(b->ninst, 0);
  uint64_t total = 0;
  for (int k = 0; k < maxsteps; ++k)
    for (int i = 0; i < b->ninst; ++i) {
      const BatchInstance& I = inst[i];
      if (k >= I.nsteps) continue;
      BatchItem it;
      it.first = total;
      it.inst = i;
      it.step = k;
      it.ntiles = uint32_t(1ull << (I.n - I.pass[k].m));
      it.chunk = std::min<uint32_t>(uint32_t(b->chunk), it.ntiles);
      it.need = prev_chunks[i];
      const uint32_t nchunks = (it.ntiles + it.chunk - 1) / it.chunk;
      prev_chunks[i] = nchunks;
      items.push_back(it);
      total += nchunks;
    }
  b->ngroups = int(items.size());
  b->items = items;
  b->total = total;
  b->ncounters = nc;
  HS_CUDA(cudaMalloc(&b->d_inst, sizeof(BatchInstance) * inst.size()));
  HS_CUDA(cudaMalloc(&b->d_items, sizeof(BatchItem) * items.size()));
  HS_CUDA(cudaMalloc(&b->d_counters, sizeof(uint32_t) * nc));
  HS_CUDA(cudaMalloc(&b->d_partial, sizeof(double) * size_t(b->ninst) * 256));
  HS_CUDA(cudaMemcpy(b->d_inst, inst.data(), sizeof(BatchInstance) * inst.size(),
                     cudaMemcpyHostToDevice));
  HS_CUDA(cudaMemcpy(b->d_items, items.data(), sizeof(BatchItem) * items.size(),
                     cudaMemcpyHostToDevice));
  // one whole run as a CUDA graph: reset the queue, |+>^n, the persistent
  // launch, <H_C>, and the read-back of results and error flag
  int dev = 0, sms = 148;
  HS_CUDA(cudaGetDevice(&dev));
  HS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  HS_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  cudaMemsetAsync(b->d_head, 0, sizeof(unsigned long long), b->stream);
  cudaMemsetAsync(b->d_counters, 0, sizeof(uint32_t) * nc, b->stream);
  cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream);
  int rc = launch_batch_init(b->d_inst, b->ninst, b->stream);
  if (rc == HS_OK)
    rc = launch_batch(b->d_inst, b->d_par, b->d_items, b->ngroups, b->total, b->d_counters,
                      b->d_head, b->d_err, b->d_limit,
                      sms * std::min(b->ctas_per_sm, batch_max_ctas_per_sm(b->threads)),
                      b->threads, b->stream);
  if (rc == HS_OK)
    rc = launch_batch_expect(b->d_inst, b->ninst, b->max_n, b->d_partial, b->d_expect, b->stream);
  cudaMemcpyAsync(b->h_expect, b->d_expect, sizeof(double) * b->ninst, cudaMemcpyDeviceToHost,
                  b->stream);
  cudaMemcpyAsync(b->h_err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc != HS_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return set_error(HS_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
  b->graph = g;
  HS_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
  return HS_OK;
}

int run_once(hs_batch* b, double* ms) {
  if (!b->exec) return set_error(HS_E_INVALID, "batch has no plan");
  HS_CUDA(cudaEventRecord(b->ev0, b->stream));
  HS_CUDA(cudaGraphLaunch(b->exec, b->stream));
  HS_CUDA(cudaEventRecord(b->ev1, b->stream));
  HS_CUDA(cudaStreamSynchronize(b->stream));
  if (ms) {
    float f = 0;
    HS_CUDA(cudaEventElapsedTime(&f, b->ev0, b->ev1));
    *ms = f;
  }
  if (*b->h_err) return set_error(HS_E_TIMEOUT, "a batch dependency wait timed out");
  return HS_OK;
}

}  // namespace

extern "C" {

int hs_batch_create_qaoa(int num_instances, const int32_t* num_qubits, const int32_t* edge_offsets,
                         const int32_t* edges, int p, const double* gammas, const double* betas,
                         hs_batch** out) {
  if (!out) return set_error(HS_E_INVALID, "null output");
  *out = nullptr;
  if (num_instances < 1 || p < 1 || p > kBatchMaxRounds)
    return set_error(HS_E_INVALID, "need >= 1 instance and 1..%d rounds", kBatchMaxRounds);
  auto* b = new hs_batch;
  b->ninst = num_instances;
  b->p = p;
  b->n.assign(num_qubits, num_qubits + num_instances);
  b->edges.resize(num_instances);
  uint64_t amps = 0;
  for (int i = 0; i < num_instances; ++i) {
    const int n = b->n[i];
    if (n < 4 || n > kBatchMaxQubits) {
      delete b;
      return set_error(HS_E_INVALID, "instance %d: %d qubits outside 4..%d", i, n, kBatchMaxQubits);
    }
    const int ne = edge_offsets[i + 1] - edge_offsets[i];
    if (ne < 0 || ne > kBatchMaxEdges) {
      delete b;
      return set_error(HS_E_INVALID, "instance %d: %d edges (max %d)", i, ne, kBatchMaxEdges);
    }
    for (int e = edge_offsets[i]; e < edge_offsets[i + 1]; ++e) {
      const int a = edges[2 * e], c = edges[2 * e + 1];
      if (a < 0 || c < 0 || a >= n || c >= n || a == c) {
        delete b;
        return set_error(HS_E_INVALID, "instance %d: bad edge (%d, %d)", i, a, c);
      }
      b->edges[i].push_back({a, c});
    }
    b->offset.push_back(amps);
    amps += 1ull << n;
    b->max_n = std::max(b->max_n, n);
  }
  b->gammas.assign(gammas, gammas + size_t(num_instances) * p);
  b->betas.assign(betas, betas + size_t(num_instances) * p);
  int rc = HS_OK;
  auto fail = [&](int code) {
    hs_batch_destroy(b);
    return code;
  };
  if (cudaMalloc(&b->pool, amps * sizeof(float2)) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    return set_error(HS_E_NOMEM, "batch states: %llu amplitudes", (unsigned long long)amps);
  }
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
      cudaMalloc(&b->d_par, sizeof(BatchParams) * num_instances) != cudaSuccess ||
      cudaMalloc(&b->d_head, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->d_err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&b->d_limit, sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&b->d_expect, sizeof(double) * num_instances) != cudaSuccess ||
      cudaMallocHost(&b->h_expect, sizeof(double) * num_instances) != cudaSuccess ||
      cudaMallocHost(&b->h_err, sizeof(int)) != cudaSuccess)
    return fail(set_error(HS_E_NOMEM, "batch buffers"));
  {
    const uint32_t lim = kBatchDefaultWaitLimit;
    if (cudaMemcpy(b->d_limit, &lim, sizeof(lim), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(set_error(HS_E_CUDA, "batch wait limit"));
  }
  if ((rc = upload_params(b)) != HS_OK) return fail(rc);
  if ((rc = build_plan(b)) != HS_OK) return fail(rc);
  *out = b;
  return HS_OK;
}

int hs_batch_set_params(hs_batch* b, const double* gammas, const double* betas) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  b->gammas.assign(gammas, gammas + size_t(b->ninst) * b->p);
  b->betas.assign(betas, betas + size_t(b->ninst) * b->p);
  return upload_params(b);
}

int hs_batch_set_chunk(hs_batch* b, int tiles_per_item) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  if (tiles_per_item < 1 || tiles_per_item > 4096)
    return set_error(HS_E_INVALID, "tiles per work item 1..4096");
  b->chunk = tiles_per_item;
  return build_plan(b);
}

int hs_batch_set_low_keep(hs_batch* b, int low) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  if (low < 2 || low > 3) return set_error(HS_E_INVALID, "keep 2 or 3 low qubits");
  const int old = b->low_keep;
  b->low_keep = low;
  const int rc = build_plan(b);
  if (rc != HS_OK) {
    b->low_keep = old;
    build_plan(b);
  }
  return rc;
}

int hs_batch_configure(hs_batch* b, int tile_cap, int ctas_per_sm) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  if (tile_cap < 6 || tile_cap > kBatchMaxTileBits || ctas_per_sm < 1 || ctas_per_sm > 16)
    return set_error(HS_E_INVALID, "tile cap 6..%d, 1..16 CTAs per SM", kBatchMaxTileBits);
  const int old_cap = b->tile_cap, old_ctas = b->ctas_per_sm;
  b->tile_cap = tile_cap;
  b->ctas_per_sm = ctas_per_sm;
  std::fill(std::begin(b->cap_of_n), std::end(b->cap_of_n), 0);
  const int rc = build_plan(b);
  if (rc != HS_OK) {  // keep the previous schedule usable
    b->tile_cap = old_cap;
    b->ctas_per_sm = old_ctas;
    if (build_plan(b) != HS_OK) return rc;
  }
  return rc;
}

int hs_batch_set_wait_limit(hs_batch* b, uint32_t polls) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  if (polls < 1) return set_error(HS_E_INVALID, "the wait limit is at least one poll");
  HS_CUDA(cudaStreamSynchronize(b->stream));
  HS_CUDA(cudaMemcpy(b->d_limit, &polls, sizeof(polls), cudaMemcpyHostToDevice));
  return HS_OK;
}

int hs_batch_block_step(hs_batch* b, int instance, int step, int block) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  for (size_t g = 0; g < b->items.size(); ++g) {
    const BatchItem& it = b->items[g];
    if (it.inst != instance || it.step != step) continue;
    if (step < 1) return set_error(HS_E_INVALID, "the first step has no dependency");
    // the device copy of the item: its need field alone
    const uint32_t need = block ? 0xffffffffu : it.need;
    HS_CUDA(cudaStreamSynchronize(b->stream));
    HS_CUDA(cudaMemcpy(reinterpret_cast<char*>(b->d_items + g) + offsetof(BatchItem, need), &need,
                       sizeof(need), cudaMemcpyHostToDevice));
    return HS_OK;
  }
  return set_error(HS_E_INVALID, "instance %d has no step %d", instance, step);
}

int hs_batch_run(hs_batch* b, double* expect_out, double* ms) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  HS_TRY(run_once(b, ms));
  if (expect_out) std::memcpy(expect_out, b->h_expect, sizeof(double) * b->ninst);
  return HS_OK;
}

int hs_batch_tune(hs_batch* b, int32_t* best_cap, int32_t* best_ctas, double* best_ms) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  auto timed = [&](double* best) -> int {  // best of two graph replays after a warm one
    double a = 0, c = 0;
    HS_TRY(run_once(b, nullptr));
    HS_TRY(run_once(b, &a));
    HS_TRY(run_once(b, &c));
    *best = std::min(a, c);
    return HS_OK;
  };
  // 1) one tile cap for every instance x CTAs per SM (up to the occupancy
  // limit) x tiles per work item
  double best = 1e300;
  const int maxc = 16;  // clamped to what fits an SM at launch
  int bc = b->tile_cap, bt = b->ctas_per_sm, bk = b->chunk;
  int bl = b->low_keep;
  for (int cap : {9, 10, 11, 12})
    for (int low : {2, 3})
      for (int chunk : {4, 16}) {
        b->chunk = chunk;
        b->low_keep = low;
        if (hs_batch_configure(b, cap, maxc) != HS_OK) continue;
        double ms = 0;
        HS_TRY(timed(&ms));
        if (ms < best) {
          best = ms;
          bc = cap;
          bt = maxc;
          bk = chunk;
          bl = low;
        }
      }
  b->chunk = bk;
  b->low_keep = bl;
  HS_TRY(hs_batch_configure(b, bc, bt));
  // 2) per qubit count, largest states first: try the other caps, keep a
  // change only if the whole batch gets at least 1% faster
  std::vector<int> ns(b->n.begin(), b->n.end());
  std::sort(ns.begin(), ns.end());
  ns.erase(std::unique(ns.begin(), ns.end()), ns.end());
  std::reverse(ns.begin(), ns.end());
  for (int n : ns) {
    if (n <= 9) continue;  // one pass whatever the cap
    const int keep = b->cap_of_n[n];
    int chosen = keep;
    for (int cap : {9, 10, 11, 12}) {
      if (cap == (keep ? keep : bc)) continue;
      b->cap_of_n[n] = cap;
      if (build_plan(b) != HS_OK) continue;
      double ms = 0;
      HS_TRY(timed(&ms));
      if (ms < 0.99 * best) {
        best = ms;
        chosen = cap;
      }
    }
    b->cap_of_n[n] = chosen;
  }
  HS_TRY(build_plan(b));
  if (best_cap) *best_cap = bc;
  if (best_ctas) *best_ctas = bt;
  if (best_ms) *best_ms = best;
  return HS_OK;
}

int hs_batch_tile_caps(hs_batch* b, int32_t* caps) {
  if (!b || !caps) return set_error(HS_E_INVALID, "null argument");
  for (int i = 0; i < b->ninst; ++i)
    caps[i] = b->cap_of_n[b->n[i]] ? b->cap_of_n[b->n[i]] : b->tile_cap;
  return HS_OK;
}

int hs_batch_stats(hs_batch* b, int64_t* stats) {
  if (!b) return set_error(HS_E_INVALID, "null batch");
  stats[0] = int64_t(b->total);
  stats[1] = int64_t(b->ncounters);
  stats[2] = int64_t(b->pass_bytes);
  stats[3] = b->tile_cap;
  stats[4] = std::min(b->ctas_per_sm, batch_max_ctas_per_sm(b->threads));
  stats[5] = b->chunk;
  stats[6] = b->low_keep;
  stats[7] = b->threads;
  return HS_OK;
}

int hs_batch_state(hs_batch* b, int instance, void* host_out) {
  if (!b || instance < 0 || instance >= b->ninst) return set_error(HS_E_INVALID, "bad instance");
  HS_CUDA(cudaMemcpy(host_out, static_cast<float2*>(b->pool) + b->offset[instance],
                     sizeof(float2) << b->n[instance], cudaMemcpyDeviceToHost));
  return HS_OK;
}

int hs_batch_destroy(hs_batch* b) {
  if (!b) return HS_OK;
  free_plan(b);
  for (void* p : {b->pool, (void*)b->d_par, (void*)b->d_head, (void*)b->d_err, (void*)b->d_expect,
                  (void*)b->d_limit})
    if (p) cudaFree(p);
  if (b->h_expect) cudaFreeHost(b->h_expect);
  if (b->h_err) cudaFreeHost(b->h_err);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return HS_OK;
}

}  // extern "C"
