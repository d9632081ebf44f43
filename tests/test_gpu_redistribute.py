"""K2 permutations (the single-device redistribution) and K3 reductions,
against the oracle's restatement of gather_slots / probability."""
import numpy as np
import pytest

from hisvsim_b200 import abi, circuits
from hisvsim_b200.gates import to_records

pytestmark = pytest.mark.gpu


def prepared(n, seed=3):
    st = abi.State(n)
    st.run_part(circuits.random_layered(n, 3, seed))
    return st


def swapbits(x, pairs):
    y = x.copy()
    for a, b in pairs:
        ba = (x >> a) & 1
        bb = (x >> b) & 1
        y ^= (ba ^ bb) * ((1 << a) | (1 << b))
    return y


@pytest.mark.parametrize("pairs", [[(0, 1)], [(0, 13)], [(2, 9), (4, 11)], [(12, 13)],
                                   [(0, 7), (1, 8), (2, 9), (3, 10), (4, 11)]])
def test_permute_bits(pairs):
    n = 14
    st = prepared(n)
    base = st.raw()
    st.permute_bits([v for p in pairs for v in p])
    x = np.arange(1 << n)
    assert np.array_equal(st.raw()[swapbits(x, pairs)], base[x])
    st.canonicalize()
    assert np.array_equal(st.raw(), base)


@pytest.mark.parametrize("proc", [[0], [13], [2, 5, 7], [0, 1, 2, 3], [9, 3, 11, 6, 1]])
def test_gather_qubits(port, proc):
    n = 14
    st = prepared(n, 4)
    base = st.raw()
    st.gather_qubits(proc)
    assert np.array_equal(st.raw(), port.gather_slots(base, n, proc))
    # state semantics unchanged: gates still act on the right qubits
    g = circuits.random_layered(n, 2, 9)
    st.run_part(g)
    want = port.run(n, to_records(g), init_state=base)
    assert np.abs(st.amplitudes() - want).max() <= 1e-12


def test_parts_after_redistribution_match(port):
    n = 16
    gates = circuits.random_layered(n, 6, 2)
    want = port.run(n, to_records(gates))
    st = abi.State(n)
    st.gather_qubits([0, 1, 2, 3])
    st.run_part(gates[:40])
    st.gather_qubits([10, 4])
    st.permute_bits([0, 15, 3, 7])
    st.run_part(gates[40:])
    assert np.abs(st.amplitudes() - want).max() <= 1e-12


def test_reductions(port, ref):
    n = 16
    st = prepared(n, 6)
    a = st.amplitudes()
    assert abs(st.norm2() - port.norm2(n, a)) <= 1e-13
    for q in (0, 5, 15):
        for v in (0, 1):
            assert abs(st.probability(q, v) - ref.probability(n, a, q, v)) <= 1e-13
    zz = st.expect_zz([0, 1, 3, 9])
    p = np.abs(a) ** 2
    x = np.arange(1 << n)
    for k, (i, j) in enumerate([(0, 1), (3, 9)]):
        s = 1 - 2 * (((x >> i) ^ (x >> j)) & 1)
        assert abs(zz[k] - (p * s).sum()) <= 1e-12
    other = prepared(n, 7)
    b = other.amplitudes()
    ip = st.inner(other)
    assert abs(ip - np.vdot(a, b)) <= 1e-12
    assert abs(st.max_abs_diff(other) - np.abs(a - b).max()) <= 1e-15


def test_inner_aligns_slot_maps():
    n = 12
    a, b = prepared(n, 1), prepared(n, 1)
    b.gather_qubits([3, 4])
    assert abs(a.inner(b) - 1) <= 1e-12
    assert a.max_abs_diff(b) <= 1e-15


def test_reductions_deterministic():
    st = prepared(20, 2)
    vals = {st.norm2() for _ in range(5)}
    assert len(vals) == 1


def test_measure_distribution():
    n = 10
    st = prepared(n, 8)
    p = np.abs(st.amplitudes()) ** 2
    s = st.measure(list(range(n)), 20000, 1234)
    idx = (s * (1 << np.arange(n))).sum(axis=1)
    counts = np.bincount(idx, minlength=1 << n) / len(idx)
    assert np.abs(counts - p).max() < 0.02
    assert np.array_equal(st.measure([0, 3], 50, 99), st.measure([0, 3], 50, 99))
