// pybind11 module `svsimulator_py_wrapper`: the reference's Python API
// (py_wrapper.cpp:15-177 of pnnl/hisvsim) bound onto the C ABI of libhisv.
//
// Same class and function names, constructor arguments and call order as the
// reference, so that qasm_assembler_standalone.py-style drivers run unchanged:
//   AggregateGate_0/_1/_2/_3/_C1/_C2/_Frac, AggregateGateFactory,
//   StateVector(n, numa), BoundGate(factory, controls, targets).apply(sv),
//   gather_and_execute_on(sv, [BoundGate]), obtain_*, set_*.
// Differences, all toward errors instead of aborts:
//   * a gate name the reference cannot construct raises ValueError (the
//     reference reaches UNREACHABLE / NOT_IMPLEMENTED, i.e. assert(0));
//   * gather_and_execute_on really executes the part (the reference's exported
//     function has its gather/execute/scatter commented out,
//     execute.hpp:270,276,283; here it has the semantics of the live
//     gather_and_execute_on_multi, execute.hpp:318-470);
//   * measure() draws from a seeded generator (set_seed) instead of
//     std::random_device and does not print.
#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/operators.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <bitset>
#include <cctype>
#include <chrono>
#include <complex>
#include <cstring>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "hisv.h"

namespace py = pybind11;
using Type = std::complex<double>;

namespace {

void check(int rc) {
  if (rc != HS_OK) {
    std::string msg = hs_last_error();
    if (rc == HS_E_INVALID || rc == HS_E_UNSUPPORTED) throw py::value_error(msg);
    if (rc == HS_E_NOMEM) throw std::bad_alloc();
    throw std::runtime_error("hisv error " + std::to_string(rc) + ": " + msg);
  }
}

// gate_name_to_type (basic_gates.hpp:1487-1522): the name is upper-cased and
// compared with the table, whose *Frac entries are mixed-case and so never
// match -- the reference cannot build Frac gates by name.
int gate_name_to_type(std::string name) {
  for (auto& c : name) c = char(::toupper(c));
  static const std::pair<const char*, int> table[] = {
      {"I", HS_GATE_I},       {"ALLOC", HS_GATE_ALLOC}, {"FREE", HS_GATE_FREE},
      {"X", HS_GATE_X},       {"Y", HS_GATE_Y},         {"Z", HS_GATE_Z},
      {"H", HS_GATE_H},       {"S", HS_GATE_S},         {"T", HS_GATE_T},
      {"RX", HS_GATE_RX},     {"RY", HS_GATE_RY},       {"RZ", HS_GATE_RZ},
      {"RI", HS_GATE_RI},     {"R1", HS_GATE_R1},       {"RXFrac", HS_GATE_RXFRAC},
      {"RYFrac", HS_GATE_RYFRAC}, {"RZFrac", HS_GATE_RZFRAC}, {"RIFrac", HS_GATE_RIFRAC},
      {"R1Frac", HS_GATE_R1FRAC}, {"SWAP", HS_GATE_SWAP}, {"C1", HS_GATE_C1},
      {"C2", HS_GATE_C2},     {"U1", HS_GATE_U1},       {"U2", HS_GATE_U2},
      {"U3", HS_GATE_U3},     {"RXX", HS_GATE_RXX},     {"RYY", HS_GATE_RYY},
      {"RZZ", HS_GATE_RZZ},   {"TDG", HS_GATE_TDG},     {"SDG", HS_GATE_SDG}};
  for (const auto& e : table)
    if (name == e.first) return e.second;
  return HS_GATE_INVALID;
}

struct AG {  // common body of the AggregateGate_* classes
  hs_gate rec;
  AG() { std::memset(&rec, 0, sizeof(rec)); }
  void set_params(std::initializer_list<Type> ps) {
    int i = 0;
    for (const Type& p : ps) {
      rec.params[2 * i] = p.real();
      rec.params[2 * i + 1] = p.imag();
      ++i;
    }
  }
  // family check of the AggregateGate_* constructors (basic_gates.hpp:1538-1776)
  void require(const std::string& name, std::initializer_list<int> allowed, const char* cls) {
    rec.type = gate_name_to_type(name);
    if (rec.type == HS_GATE_INVALID)
      throw py::value_error("unknown gate name '" + name + "' (" + cls + ")");
    if (std::find(allowed.begin(), allowed.end(), rec.type) == allowed.end())
      throw py::value_error("gate '" + name + "' is not a " + cls + " gate");
  }
};

struct AG0 : AG {
  explicit AG0(const std::string& n) {
    require(n, {HS_GATE_I, HS_GATE_X, HS_GATE_Y, HS_GATE_Z, HS_GATE_H, HS_GATE_S, HS_GATE_T,
                HS_GATE_SWAP, HS_GATE_TDG, HS_GATE_SDG},
            "AggregateGate_0");
  }
};
struct AG1 : AG {
  AG1(const std::string& n, Type t) {
    require(n, {HS_GATE_RI, HS_GATE_RX, HS_GATE_RY, HS_GATE_RZ, HS_GATE_R1, HS_GATE_RXX,
                HS_GATE_RZZ, HS_GATE_RYY, HS_GATE_U1},
            "AggregateGate_1");
    set_params({t});
  }
};
struct AG2 : AG {
  AG2(const std::string& n, Type phi, Type lambda) {
    require(n, {HS_GATE_U2}, "AggregateGate_2");
    set_params({phi, lambda});
  }
};
struct AG3 : AG {
  AG3(const std::string& n, Type theta, Type phi, Type lambda) {
    require(n, {HS_GATE_U3}, "AggregateGate_3");
    set_params({theta, phi, lambda});
  }
};
struct AGC1 : AG {
  AGC1(const std::string& n, Type a, Type b, Type c, Type d) {
    require(n, {HS_GATE_C1}, "AggregateGate_C1");
    set_params({a, b, c, d});
  }
};
struct AGC2 : AG {
  AGC2(const std::string& n, Type c00, Type c01, Type c02, Type c03, Type c10, Type c11,
       Type c12, Type c13, Type c20, Type c21, Type c22, Type c23, Type c30, Type c31,
       Type c32, Type c33) {
    require(n, {HS_GATE_C2}, "AggregateGate_C2");
    set_params({c00, c01, c02, c03, c10, c11, c12, c13, c20, c21, c22, c23, c30, c31, c32, c33});
  }
};
struct AGFrac : AG {
  AGFrac(const std::string& n, unsigned num, unsigned pow) {
    require(n, {HS_GATE_RIFRAC, HS_GATE_R1FRAC, HS_GATE_RXFRAC, HS_GATE_RYFRAC,
                HS_GATE_RZFRAC},
            "AggregateGate_Frac");
    rec.frac_num = num;
    rec.frac_pow = pow;
  }
};

struct Factory {  // AggregateGateFactory (basic_gates.hpp:1779-1845)
  hs_gate rec;
  explicit Factory(const AG& ag) : rec(ag.rec) {}
};

// process-wide counters and settings (the reference's globals)
int g_num_threads = 1, g_init_threads = 1, g_opt_slots = 0;
long long g_gather_us = 0;
std::mt19937_64 g_seed_gen(std::random_device{}());

struct SV {  // StateVector
  hs_state* st = nullptr;
  // factors that gather_and_execute_on / BoundGate.apply leave pending
  // (hs_part_run_carry); every method that reads or writes the amplitudes
  // applies them first (settle), so the object behaves as the reference's
  // StateVector after each call
  hs_frames* fr = nullptr;
  int n = 0;
  SV(int num_qubits, int numa) {
    (void)numa;  // allocation policy of host memory; the state lives in HBM
    py::gil_scoped_release nogil;
    check(hs_state_create(num_qubits, HS_DTYPE_C128, &st));
    n = num_qubits;
    const int rc = hs_frames_create(num_qubits, &fr);
    if (rc != HS_OK) {
      hs_state_destroy(st);
      st = nullptr;
      check(rc);
    }
  }
  ~SV() {
    if (fr) hs_frames_destroy(fr);
    if (st) hs_state_destroy(st);
  }
  void settle() { check(hs_frames_flush(st, fr, nullptr)); }
  std::vector<int> qubits() const {
    std::vector<int> q(n);
    for (int i = 0; i < n; ++i) q[i] = i;
    return q;
  }
  py::array_t<std::complex<double>> amplitudes() {
    py::array_t<std::complex<double>> out(size_t(1) << n);
    {
      py::gil_scoped_release nogil;
      settle();
      check(hs_state_canonicalize(st, nullptr));
    }
    check(hs_state_copy_to_host(st, out.mutable_data(), 0, uint64_t(1) << n, nullptr));
    return out;
  }
  void load(py::array_t<std::complex<double>, py::array::c_style | py::array::forcecast> a) {
    if (size_t(a.size()) != (size_t(1) << n)) throw py::value_error("need 2^n amplitudes");
    settle();  // (the pending factors then reset; the amplitudes are overwritten)
    check(hs_state_set_basis(st, 0, nullptr));
    check(hs_state_copy_from_host(st, a.data(), 0, uint64_t(1) << n, nullptr));
  }
  std::vector<std::vector<int>> measure(const std::vector<int>& qs, unsigned nsamples) {
    std::vector<int32_t> out(size_t(nsamples) * qs.size());
    std::vector<int32_t> q(qs.begin(), qs.end());
    {
      py::gil_scoped_release nogil;
      settle();
      check(hs_measure(st, q.data(), int(q.size()), nsamples, g_seed_gen(), out.data()));
    }
    std::vector<std::vector<int>> r(nsamples, std::vector<int>(qs.size()));
    for (size_t s = 0; s < nsamples; ++s)
      for (size_t j = 0; j < qs.size(); ++j) r[s][j] = out[s * qs.size() + j];
    return r;
  }
  double max_abs_diff(SV& o) {
    double d = 0;
    py::gil_scoped_release nogil;
    settle();
    o.settle();
    check(hs_max_abs_diff(st, o.st, &d));
    return d;
  }
  // state_equal (state_vector.hpp:1003-1010): |a_i - b_i| <= 1e-10 for all i
  bool state_equal(SV& o) {
    if (o.n != n) return false;
    return max_abs_diff(o) <= 1e-10;
  }
  // dump_state_new (state_vector.hpp:135-140): "bitset<16>(i): (re,im)" lines
  void dump_state() {
    auto a = amplitudes();
    auto p = a.unchecked<1>();
    std::ostringstream os;
    for (py::ssize_t i = 0; i < p.shape(0); ++i)
      os << std::bitset<16>(size_t(i)) << ": " << p(i) << "\n";
    py::print(os.str(), py::arg("end") = "");
  }
  double norm() {
    double s = 0;
    py::gil_scoped_release nogil;
    settle();
    check(hs_norm2(st, &s));
    return s;
  }
  double probability(int q, int v) {
    double p = 0;
    py::gil_scoped_release nogil;
    settle();
    check(hs_probability(st, q, v, &p));
    return p;
  }
};

struct Bound {  // BoundGate (state_vector.hpp:1332-1379)
  hs_gate rec;
  Bound(Factory& f, const std::vector<int>& controls, const std::vector<int>& targets) : rec(f.rec) {
    if (controls.size() > HS_MAX_CONTROLS || targets.size() > HS_MAX_TARGETS || targets.empty())
      throw py::value_error("BoundGate takes at most 5 controls and 1..5 targets");
    rec.num_controls = int(controls.size());
    rec.num_targets = int(targets.size());
    for (size_t i = 0; i < controls.size(); ++i) rec.controls[i] = controls[i];
    for (size_t i = 0; i < targets.size(); ++i) rec.targets[i] = targets[i];
  }
  void apply(SV& sv) {
    py::gil_scoped_release nogil;
    check(hs_part_run_carry(sv.st, sv.fr, &rec, 1, nullptr));
  }
};

std::vector<hs_gate> records(const std::vector<Bound*>& gates) {
  std::vector<hs_gate> r;
  r.reserve(gates.size());
  for (auto* g : gates) r.push_back(g->rec);
  return r;
}

void gather_and_execute_on(SV& sv, std::vector<Bound*> gates) {
  auto recs = records(gates);
  auto t0 = std::chrono::steady_clock::now();
  {
    py::gil_scoped_release nogil;
    check(hs_part_run_carry(sv.st, sv.fr, recs.data(), int(recs.size()), nullptr));
  }
  g_gather_us += std::chrono::duration_cast<std::chrono::microseconds>(
                     std::chrono::steady_clock::now() - t0).count();
}

// The proc qubits of one top-level part of the MPI drivers: the qubits the
// part's gates do not touch, after padding the touched set with the lowest
// other qubits up to nlocal when opt_slots is set (execute.hpp:565-571,
// 815-821).
std::vector<int32_t> proc_qubits(int n, int nlocal, const std::vector<hs_gate>& recs) {
  std::vector<int> needed;
  for (auto& r : recs) {
    for (int i = 0; i < r.num_targets; ++i) needed.push_back(r.targets[i]);
    for (int i = 0; i < r.num_controls; ++i) needed.push_back(r.controls[i]);
  }
  std::sort(needed.begin(), needed.end());
  needed.erase(std::unique(needed.begin(), needed.end()), needed.end());
  if (int(needed.size()) > nlocal)
    throw py::value_error("a part touches more qubits than num_local_qubits");
  if (g_opt_slots == 1)
    for (int q = 0; q < n && int(needed.size()) < nlocal; ++q)
      if (std::find(needed.begin(), needed.end(), q) == needed.end()) needed.push_back(q);
  std::vector<int32_t> proc;
  for (int q = 0; q < n; ++q)
    if (std::find(needed.begin(), needed.end(), q) == needed.end()) proc.push_back(q);
  return proc;
}

// Single-device form of gather_and_execute_on_mpi (execute.hpp:542-728): the
// state's top slots play the MPI rank bits; before every part but the first,
// the part's proc qubits become those top slots through the in-HBM
// permutation (SvSimMPI::gather_qubits, svsim-mpi.hpp:123-173); then the part
// runs.  Returns the final StateVector.
SV* gather_and_execute_on_mpi(int n, int nlocal, std::vector<std::vector<Bound*>> parts) {
  if (nlocal < 1 || nlocal > n) throw py::value_error("need 1 <= num_local_qubits <= n");
  auto sv = std::make_unique<SV>(n, 0);
  for (size_t p = 0; p < parts.size(); ++p) {
    auto recs = records(parts[p]);
    const std::vector<int32_t> proc = proc_qubits(n, nlocal, recs);
    py::gil_scoped_release nogil;
    if (p > 0 && !proc.empty())
      check(hs_gather_qubits(sv->st, proc.data(), int(proc.size()), nullptr));
    // the pending factors belong to qubits: they follow the gather
    check(hs_part_run_carry(sv->st, sv->fr, recs.data(), int(recs.size()), nullptr));
  }
  return sv.release();
}

// Single-device form of gather_and_execute_multilevel_on_mpi
// (execute.hpp:730-900): multi_parts[p][0] lists every gate of top-level part
// p and decides its proc qubits (gathered to the top slots before every top
// part but the first); multi_parts[p][1..] are its second-level parts, run in
// order (the reference runs each with gather_and_execute_on_multi,
// execute.hpp:867).  Here the second-level parts of one top part go to the
// device as one hs_parts_run call.  Returns the final StateVector.
SV* gather_and_execute_multilevel_on_mpi(int n, int nlocal,
                                         std::vector<std::vector<std::vector<Bound*>>> multi) {
  if (nlocal < 1 || nlocal > n) throw py::value_error("need 1 <= num_local_qubits <= n");
  auto sv = std::make_unique<SV>(n, 0);
  for (size_t p = 0; p < multi.size(); ++p) {
    if (multi[p].empty()) throw py::value_error("a top-level part needs its gate list first");
    const std::vector<int32_t> proc = proc_qubits(n, nlocal, records(multi[p][0]));
    std::vector<hs_gate> flat;
    std::vector<int32_t> offs{0};
    for (size_t i = 1; i < multi[p].size(); ++i) {
      auto r = records(multi[p][i]);
      flat.insert(flat.end(), r.begin(), r.end());
      offs.push_back(int32_t(flat.size()));
    }
    py::gil_scoped_release nogil;
    if (p > 0 && !proc.empty())
      check(hs_gather_qubits(sv->st, proc.data(), int(proc.size()), nullptr));
    if (offs.size() > 1)
      check(hs_parts_run(sv->st, flat.data(), offs.data(), int(offs.size()) - 1, nullptr));
  }
  return sv.release();
}

}  // namespace

PYBIND11_MODULE(svsimulator_py_wrapper, m) {
  m.doc() = "B200-native hierarchical state-vector simulator (reference API of pnnl/hisvsim)";
  py::class_<AG>(m, "_AggregateGate");
  py::class_<AG0, AG>(m, "AggregateGate_0").def(py::init<const std::string&>());
  py::class_<AG1, AG>(m, "AggregateGate_1").def(py::init<const std::string&, Type>());
  py::class_<AG2, AG>(m, "AggregateGate_2").def(py::init<const std::string&, Type, Type>());
  py::class_<AG3, AG>(m, "AggregateGate_3")
      .def(py::init<const std::string&, Type, Type, Type>());
  py::class_<AGC1, AG>(m, "AggregateGate_C1")
      .def(py::init<const std::string&, Type, Type, Type, Type>());
  py::class_<AGC2, AG>(m, "AggregateGate_C2")
      .def(py::init<const std::string&, Type, Type, Type, Type, Type, Type, Type, Type, Type,
                    Type, Type, Type, Type, Type, Type, Type>());
  py::class_<AGFrac, AG>(m, "AggregateGate_Frac")
      .def(py::init<const std::string&, unsigned, unsigned>());
  py::class_<Factory>(m, "AggregateGateFactory")
      .def(py::init<AG0&>())
      .def(py::init<AG1&>())
      .def(py::init<AG2&>())
      .def(py::init<AG3&>())
      .def(py::init<AGFrac&>())
      .def(py::init<AGC1&>())
      .def(py::init<AGC2&>());
  py::class_<SV>(m, "StateVector")
      .def(py::init<int, int>(), py::arg("n"), py::arg("numa") = 1)
      .def("qubits", &SV::qubits)
      .def("measure", &SV::measure, py::arg("qubits"), py::arg("num_samples") = 1)
      .def("state_equal", &SV::state_equal)
      .def("dump_state", &SV::dump_state)
      .def("__eq__", [](SV& a, SV& b) { return a.n == b.n && a.max_abs_diff(b) <= 1e-10; })
      // additions: amplitude readback and FP64 reductions
      .def("amplitudes", &SV::amplitudes)
      .def("load", &SV::load)
      .def("norm", &SV::norm)
      .def("probability", &SV::probability, py::arg("qubit"), py::arg("value") = 0)
      .def("max_abs_diff", &SV::max_abs_diff)
      .def_property_readonly("num_qubits", [](const SV& s) { return s.n; });
  py::class_<Bound>(m, "BoundGate")
      .def(py::init<Factory&, const std::vector<int>&, const std::vector<int>&>())
      .def("apply", &Bound::apply);
  m.def("gather_and_execute_on", &gather_and_execute_on);
  m.def("gather_and_execute_on_mpi", &gather_and_execute_on_mpi,
        py::return_value_policy::take_ownership);
  m.def("gather_and_execute_multilevel_on_mpi", &gather_and_execute_multilevel_on_mpi,
        py::return_value_policy::take_ownership);
  m.def("obtain_apply_time", []() {
    long long us = 0;
    hs_counters(&us, nullptr, nullptr);
    return us;
  });
  m.def("obtain_gate_counter", []() {
    long long g = 0;
    hs_counters(nullptr, &g, nullptr);
    return g;
  });
  m.def("obtain_move_counter", []() {
    long long p = 0;
    hs_counters(nullptr, nullptr, &p);
    return p;
  });
  m.def("obtain_gather_time", []() { return g_gather_us; });
  m.def("set_num_threads", [](int t) { g_num_threads = t; });
  m.def("set_init_num_threads", [](int t) { g_init_threads = t; });
  m.def("set_opt_slots", [](int o) { g_opt_slots = o; });
  m.def("set_seed", [](unsigned long long s) { g_seed_gen.seed(s); });
  m.def("set_timing", [](int on) { return hs_set_timing(on); });
}
