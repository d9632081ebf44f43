"""The drop-in: the reference's Python API (py_wrapper.cpp) driving the GPU,
used the way qasm_assembler_standalone.py uses it (:1768-2018)."""
import numpy as np
import pytest

from hisvsim_b200 import circuits, partition
from hisvsim_b200.gates import NOPARAM, ONEPARAM, to_records

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def svsim():
    from hisvsim_b200 import svsimulator_py_wrapper

    return svsimulator_py_wrapper


def bound(svsim, g):
    p = g.params
    if g.name in NOPARAM:
        ag = svsim.AggregateGate_0(g.name)
    elif g.name in ONEPARAM:
        ag = svsim.AggregateGate_1(g.name, p[0])
    elif g.name == "U2":
        ag = svsim.AggregateGate_2(g.name, p[0], p[1])
    elif g.name == "U3":
        ag = svsim.AggregateGate_3(g.name, p[0], p[1], p[2])
    elif g.name == "C1":
        ag = svsim.AggregateGate_C1(g.name, *p)
    else:
        ag = svsim.AggregateGate_C2(g.name, *p)
    return svsim.BoundGate(svsim.AggregateGateFactory(ag), list(g.controls), list(g.targets))


def test_part_driver_matches_reference(svsim, ref):
    n = 18
    gates = circuits.random_layered(n, 12, 21)
    parts = partition.partition_acyclic(gates, 9)
    sim = svsim.StateVector(n, 0)
    for p in parts:
        svsim.gather_and_execute_on(sim, [bound(svsim, gates[i]) for i in p])
    want = ref.run(n, to_records(gates))
    assert np.abs(sim.amplitudes() - want).max() <= 1e-12
    assert svsim.obtain_gate_counter() > 0


def test_per_gate_driver(svsim, port):
    n = 12
    gates = circuits.random_layered(n, 5, 2)
    sim = svsim.StateVector(n, 1)
    for g in gates:
        bound(svsim, g).apply(sim)
    want = port.run(n, to_records(gates))
    assert np.abs(sim.amplitudes() - want).max() <= 1e-12


def test_equality_and_measure(svsim):
    a, b = svsim.StateVector(6, 0), svsim.StateVector(6, 0)
    assert a.state_equal(b) and a == b
    bound(svsim, circuits.Gate("H", (2,))).apply(a)
    assert not a.state_equal(b) and not (a == b)
    assert abs(a.probability(2, 0) - 0.5) <= 1e-12
    svsim.set_seed(5)
    r = a.measure([2, 0], 7)
    assert len(r) == 7 and all(len(x) == 2 and x[1] == 0 for x in r)
    assert a.qubits() == list(range(6))


def test_dump_state_format(svsim, capsys):
    a = svsim.StateVector(1, 0)
    a.dump_state()
    out = capsys.readouterr().out.splitlines()
    assert out == ["0000000000000000: (1,0)", "0000000000000001: (0,0)"]


def test_mpi_driver_emulation(svsim, port):
    """gather_and_execute_on_mpi on one device (redistribution by K2)."""
    n, nlocal = 14, 10
    gates = circuits.random_layered(n, 6, 13)
    parts = partition.partition_acyclic(gates, 6)
    lists = [[bound(svsim, gates[i]) for i in p] for p in parts]
    sim = svsim.gather_and_execute_on_mpi(n, nlocal, lists)
    want = port.run(n, to_records(gates))
    assert np.abs(sim.amplitudes() - want).max() <= 1e-12


@pytest.mark.parametrize("opt_slots", [0, 1])
def test_multilevel_mpi_driver_matches_reference(svsim, ref, opt_slots):
    """gather_and_execute_multilevel_on_mpi (py_wrapper.cpp:158-161,
    execute.hpp:730-900) on one device: top-level parts of <= 8 qubits, each
    split into second-level parts of <= 4 qubits; every top part after the
    first gathers its proc qubits to the top slots (K2), its second-level
    parts run through K1.  Compared with the reference's own per-gate path."""
    n, nlocal = 13, 9
    gates = circuits.random_layered(n, 6, 29)
    top = partition.partition_acyclic(gates, 8)
    multi = []
    for p in top:
        sub_gates = [gates[i] for i in p]
        second = partition.partition_acyclic(sub_gates, 4)
        multi.append([[bound(svsim, g) for g in sub_gates]] +
                     [[bound(svsim, sub_gates[i]) for i in s] for s in second])
    svsim.set_opt_slots(opt_slots)
    try:
        sim = svsim.gather_and_execute_multilevel_on_mpi(n, nlocal, multi)
    finally:
        svsim.set_opt_slots(0)
    want = ref.run(n, to_records(gates), mode=0)
    assert np.abs(sim.amplitudes() - want).max() <= 1e-12
    with pytest.raises(ValueError):
        svsim.gather_and_execute_multilevel_on_mpi(n, 3, multi)  # parts wider than nlocal
