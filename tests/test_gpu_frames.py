"""Deferred factors between part calls (hs_part_run_carry / hs_frames_flush):
parts run one call at a time with their pending phase and scale factors
carried equal the same parts run by hs_parts_run and by the oracle, also
with qubit permutations in between; the pybind StateVector, which defers
them, reads back the reference's amplitudes."""
import numpy as np
import pytest

from hisvsim_b200 import abi, circuits, partition
from hisvsim_b200.gates import part_offsets, to_records

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("n,k,seed", [(14, 7, 1), (17, 9, 2)])
def test_carried_parts_match_parts_run_and_oracle(port, n, k, seed):
    gates = circuits.random_u3_cz(n, 10, seed)
    parts = partition.partition_frontier(gates, k)
    want = port.run(n, to_records(gates))
    st = abi.State(n, abi.C128)
    fr = abi.Frames(n)
    for p in parts:
        st.run_part_carry(fr, [gates[i] for i in p])
    assert fr.pending
    st.flush(fr)
    assert not fr.pending
    assert np.abs(st.amplitudes() - want).max() <= TOL
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st2 = abi.State(n, abi.C128)
    st2.run_parts(rec, offs)
    assert np.abs(st2.amplitudes() - want).max() <= TOL
    # flushing with nothing pending is a no-op
    st.flush(fr)
    assert np.abs(st.amplitudes() - want).max() <= TOL


def test_carried_factors_follow_qubit_permutations(port):
    n = 15
    gates = circuits.random_layered(n, 6, 4)
    parts = partition.partition_acyclic(gates, 6)
    want = port.run(n, to_records(gates))
    st = abi.State(n, abi.C128)
    fr = abi.Frames(n)
    for i, p in enumerate(parts):
        if i % 3 == 1:
            st.permute_bits([(0, n - 1), (2, n - 3)])
        st.run_part_carry(fr, [gates[j] for j in p])
    st.flush(fr)
    assert np.abs(st.amplitudes() - want).max() <= TOL * max(1.0, np.abs(want).max())


def test_frames_reject_wrong_size():
    st = abi.State(8, abi.C128)
    fr = abi.Frames(9)
    with pytest.raises(abi.HisvError) as e:
        st.flush(fr)
    assert e.value.code == abi.HS_E_INVALID


def test_pywrapper_defers_and_settles(port):
    from hisvsim_b200 import svsimulator_py_wrapper as sv
    from hisvsim_b200.gates import NOPARAM

    n = 13
    gates = circuits.random_u3_cz(n, 8, 9)
    parts = partition.partition_frontier(gates, 7)

    def bound(g):
        ag = sv.AggregateGate_0(g.name) if g.name in NOPARAM else sv.AggregateGate_3(g.name, *g.params)
        return sv.BoundGate(sv.AggregateGateFactory(ag), list(g.controls), list(g.targets))

    s = sv.StateVector(n, 0)
    half = len(parts) // 2
    for p in parts[:half]:
        sv.gather_and_execute_on(s, [bound(gates[i]) for i in p])
    # a read in between applies the pending factors
    assert abs(s.norm() - 1.0) <= 1e-12
    for p in parts[half:]:
        for i in p:
            bound(gates[i]).apply(s)
    want = port.run(n, to_records(gates))
    assert np.abs(s.amplitudes() - want).max() <= TOL
    assert abs(s.probability(0, 1) - np.sum(np.abs(want[1::2]) ** 2)) <= 1e-12
