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
                                   [(0, 7), (1, 8), (2, 9), (3, 10), (4, 11)],
                                   [(0, 13), (1, 12), (2, 11), (3, 10), (4, 9), (5, 8), (6, 7)]])
@pytest.mark.parametrize("dtype", [abi.C128, abi.C64])
def test_permute_bits(pairs, dtype):
    n = 14
    st = abi.State(n, dtype)
    st.run_part(circuits.random_layered(n, 3, 3))
    base = st.raw()
    st.permute_bits([v for p in pairs for v in p])
    x = np.arange(1 << n)
    assert np.array_equal(st.raw()[swapbits(x, pairs)], base[x])
    st.canonicalize()
    assert np.array_equal(st.raw(), base)


@pytest.mark.parametrize("n,pairs", [(3, [(0, 2)]), (5, [(0, 4), (1, 3)]), (22, [(0, 21), (3, 17)])])
def test_permute_small_and_large_states(n, pairs):
    st = prepared(n)
    base = st.raw()
    st.permute_bits([v for p in pairs for v in p])
    x = np.arange(1 << n)
    assert np.array_equal(st.raw()[swapbits(x, pairs)], base[x])


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


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("dtype", [abi.C128, abi.C64])
def test_project_matches_numpy(mode, dtype):
    """hs_project (state_vector.hpp:829-894) against a numpy restatement, on a
    state whose slots are permuted (qubit q not at slot q)."""
    n = 9
    gates = circuits.random_u3_cz(n, 6, 31)
    st = abi.State(n, dtype)
    st.set_basis(0)
    for g in gates:
        st.apply(g)
    st.permute_bits([(0, 7), (2, 5)])
    full = st.amplitudes().astype(np.complex128)
    st.permute_bits([(0, 7), (2, 5)])
    qubits, values = [6, 1, 3], [1, 0, 1]
    sub, p = st.project(qubits, values, mode)
    idx = np.arange(1 << n)
    keep = np.ones(1 << n, dtype=bool)
    for q, v in zip(qubits, values):
        keep &= ((idx >> q) & 1) == v
    want = full[keep]  # remaining qubits in increasing order = ascending index
    wp = float(np.sum(np.abs(want) ** 2))
    tol = 1e-12 if dtype == abi.C128 else 1e-5
    assert p == pytest.approx(wp, rel=tol, abs=tol)
    assert wp > 1e-3  # a generic state: the projected part is not empty
    want = want / (np.sqrt(wp) if mode == 0 else wp if mode == 1 else 1.0)
    assert sub.n == n - 3
    assert np.abs(sub.amplitudes() - want).max() <= tol * max(1.0, np.abs(want).max())
    if mode == 0:
        assert sub.norm2() == pytest.approx(1.0, abs=tol)


def test_project_of_an_empty_part_is_left_unnormalised():
    st = abi.State(5)
    st.set_basis(0b00101)
    sub, p = st.project([0], [0])  # qubit 0 is 1 with certainty
    assert p == 0.0 and np.abs(sub.amplitudes()).max() == 0.0


def test_project_rejects_bad_arguments():
    st = abi.State(4)
    for q, v in ([[0, 0], [0, 1]], [[5], [0]], [[1], [2]], [[0, 1, 2, 3], None]):
        with pytest.raises(abi.HisvError):
            st.project(q, v)


@pytest.mark.parametrize("renormalize", [True, False])
@pytest.mark.parametrize("permuted", [False, True])
def test_project_matches_reference_project(ref, renormalize, permuted):
    """hs_project with the reference's normalisation (mode 1: divide by p;
    mode 2: renormalize=false) against StateVector::project itself
    (state_vector.hpp:829-894, through the oracle harness) on the same state,
    at 1e-12; the device state's slots are permuted in one case."""
    from hisvsim_b200.gates import to_records

    n = 10
    gates = circuits.random_layered(n, 5, 41)
    full = ref.run(n, to_records(gates))
    st = abi.State(n, abi.C128)
    st.load(full)
    if permuted:
        st.permute_bits([(1, 8), (3, 6)])
    for qubits, values in (([4], [1]), ([7, 0, 2], [0, 1, 1]), ([9, 5], [1, 1])):
        sub, p = st.project(qubits, values, 1 if renormalize else 2)
        want = ref.project(n, full, qubits, values, renormalize)
        assert np.abs(sub.amplitudes() - want).max() <= 1e-12
        sub.close()
