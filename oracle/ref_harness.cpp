// Oracle harness over the reference's own C++ headers.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled (by oracle/Makefile) against
// the unmodified reference headers state_vector.hpp / execute.hpp /
// basic_gates.hpp / loop.hpp / types.hpp where they lie in the reference
// checkout, into oracle/_ref/libhisv_ref.so.  Only tests/, the smoke check and
// bench.py's CPU-baseline / reference arm load it — as the checker and the
// timed CPU baseline, never as the product path.
//
// It exposes two drivers of the reference's CPU path:
//   mode 0: BoundGate::apply per gate            (state_vector.hpp:1349)
//   mode 1: gather_and_execute_on_multi per part (execute.hpp:318-470), the
//           live form of the part path; the exported gather_and_execute_on
//           (execute.hpp:171) has its gather/execute/scatter commented out
//           (execute.hpp:270,276,283) and would leave the state unchanged.
// Gates arrive as hs_gate records (include/hisv.h) and are turned into
// AggregateGate_* / AggregateGateFactory / BoundGate objects by GateType, the
// way py_wrapper.cpp:101-154 builds them from Python.
#include <omp.h>

#include <cstring>
#include <iostream>
#include <sstream>
#include <vector>

#include "execute.hpp"
#include "hisv.h"
#include "state_vector.hpp"

using namespace SvSim;

namespace {

Type P(const hs_gate& g, int i) { return Type(g.params[2 * i], g.params[2 * i + 1]); }

// Returns false for gate types the reference's factories reject
// (basic_gates.hpp:1570-1575 etc. end in UNREACHABLE / NOT_IMPLEMENTED).
bool make_factory(const hs_gate& g, AggregateGateFactory** out) {
  GateType t = static_cast<GateType>(g.type);
  switch (t) {
    case GateType::I:
    case GateType::X:
    case GateType::Y:
    case GateType::Z:
    case GateType::H:
    case GateType::S:
    case GateType::T:
    case GateType::SWAP:
    case GateType::TDG:
    case GateType::SDG:
      *out = new AggregateGateFactory(AggregateGate_0(t));
      return true;
    case GateType::RX:
    case GateType::RY:
    case GateType::RZ:
    case GateType::RI:
    case GateType::R1:
    case GateType::U1:
    case GateType::RXX:
    case GateType::RYY:
    case GateType::RZZ:
      *out = new AggregateGateFactory(AggregateGate_1(t, P(g, 0)));
      return true;
    case GateType::U2:
      *out = new AggregateGateFactory(AggregateGate_2(t, P(g, 0), P(g, 1)));
      return true;
    case GateType::U3:
      *out = new AggregateGateFactory(AggregateGate_3(t, P(g, 0), P(g, 1), P(g, 2)));
      return true;
    case GateType::C1:
      *out = new AggregateGateFactory(
          AggregateGate_C1(t, P(g, 0), P(g, 1), P(g, 2), P(g, 3)));
      return true;
    case GateType::C2:
      *out = new AggregateGateFactory(AggregateGate_C2(
          t, P(g, 0), P(g, 1), P(g, 2), P(g, 3), P(g, 4), P(g, 5), P(g, 6), P(g, 7),
          P(g, 8), P(g, 9), P(g, 10), P(g, 11), P(g, 12), P(g, 13), P(g, 14), P(g, 15)));
      return true;
    case GateType::RXFrac:
    case GateType::RYFrac:
    case GateType::RZFrac:
    case GateType::RIFrac:
    case GateType::R1Frac:
      *out = new AggregateGateFactory(AggregateGate_Frac(t, g.frac_num, g.frac_pow));
      return true;
    default:
      return false;
  }
}

bool make_bound(const hs_gate& g, std::vector<BoundGate>* out) {
  AggregateGateFactory* f = nullptr;
  if (!make_factory(g, &f)) return false;
  if (g.num_controls < 0 || g.num_controls > 5 || g.num_targets < 1 || g.num_targets > 5) {
    delete f;
    return false;
  }
  std::vector<Qubit> c(g.controls, g.controls + g.num_controls);
  std::vector<Qubit> t(g.targets, g.targets + g.num_targets);
  out->push_back(BoundGate(*f, c, t));
  delete f;
  return true;
}

struct QuietCout {
  std::stringstream sink;
  std::streambuf* old;
  QuietCout() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~QuietCout() { std::cout.rdbuf(old); }
};

}  // namespace

extern "C" {

int ref_hs_gate_size(void) { return (int)sizeof(hs_gate); }

// Runs `gates` on an n-qubit reference StateVector.
//   state: 2^n interleaved complex128 in/out (qubit order == slot order: the
//          reference never permutes slots on one node).  If init == 0 the
//          input is ignored and the run starts from |0...0>.
//   mode 0: per-gate BoundGate::apply.  mode 1: parts through
//          gather_and_execute_on_multi, part i = gates[offs[i]..offs[i+1]).
// Returns 0, or -1 for a gate the reference cannot build.
int ref_run(int n, const hs_gate* gates, int num_gates, const int32_t* offs,
            int num_parts, int mode, int opt_slots, int threads, int init,
            double* state) {
  if (n < 1 || n > 40) return -1;
  QuietCout quiet;
  set_num_threads(threads);
  set_init_num_threads(threads);
  set_opt_slots(opt_slots);
  std::vector<BoundGate> bound;
  bound.reserve(num_gates);
  for (int i = 0; i < num_gates; ++i)
    if (!make_bound(gates[i], &bound)) return -1;
  StateVector sv(n, 0);
  const size_t size = size_t(1) << n;
  Type* amp = sv.state();
  if (init) std::memcpy(amp, state, size * sizeof(Type));
  if (mode == 0) {
    for (auto& b : bound) b.apply(sv);
  } else {
    // execute_on has no case for GateType::I (execute.hpp:56 is commented
    // out) and would abort on it; I is the identity, so parts drop it.
    for (int p = 0; p < num_parts; ++p) {
      std::vector<BoundGate> part;
      for (int i = offs[p]; i < offs[p + 1]; ++i)
        if (gates[i].type != HS_GATE_I) part.push_back(bound[i]);
      if (part.empty()) continue;
      gather_and_execute_on_multi(sv, part, {}, 16);
    }
  }
  std::memcpy(state, amp, size * sizeof(Type));
  free(amp);  // allocated with posix_memalign (state_vector.hpp:211)
  return 0;
}

// probability(qubit, value) of the reference (state_vector.hpp:897-923) on a
// given state, single-threaded (the reference's accumulation races when run
// with more than one thread).
double ref_probability(int n, const double* state, int qubit, int value) {
  QuietCout quiet;
  set_num_threads(1);
  set_init_num_threads(1);
  StateVector sv(n, 0);
  std::memcpy(sv.state(), state, (size_t(1) << n) * sizeof(Type));
  double p = sv.probability(qubit, value);
  free(sv.state());
  return p;
}

// StateVector::project(qubits, values, renormalize) of the reference
// (state_vector.hpp:829-894) on a given state: out receives the projected
// state over the remaining 2^(n-k) indices, in the order of the reference's
// own loop over the remaining qubits (qubit_loop, trip_count).
int ref_project(int n, const double* state, const int32_t* qubits, const int32_t* values, int k,
                int renormalize, double* out) {
  if (n < 2 || k < 1 || k >= n) return -1;
  QuietCout quiet;
  set_num_threads(1);
  set_init_num_threads(1);
  StateVector sv(n, 0);
  Type* before = sv.state();
  std::memcpy(before, state, (size_t(1) << n) * sizeof(Type));
  std::vector<Qubit> q(qubits, qubits + k);
  std::vector<int> v(values, values + k);
  sv.project(q, v, renormalize != 0);
  Type* after = sv.state();
  std::memcpy(out, after, (size_t(1) << (n - k)) * sizeof(Type));
  free(after);
  free(before);
  return 0;
}

}  // extern "C"
