"""Parity of the plain form (K1/K2/K3 through the C ABI) against the oracle.

Tolerance: max |amplitude difference| <= 1e-12 for complex128 (the plain
form's contract), 1e-5 for complex64 states."""
import math

import numpy as np
import pytest

from conftest import golden_names, load_golden
from hisvsim_b200 import abi, circuits, partition
from hisvsim_b200.gates import Gate, part_offsets, to_records

pytestmark = pytest.mark.gpu
TOL = 1e-12


def all_gates(n, ng, seed):
    import tests.golden.make_golden as mg  # the same mix the golden vectors use

    return mg.all_gate_circuit(n, ng, seed)


def state_from(n, x=0, dtype=abi.C128):
    st = abi.State(n, dtype)
    st.set_basis(x)
    return st


@pytest.mark.parametrize("name", golden_names())
def test_golden_vectors(name):
    n, rec, offs, x, amps = load_golden(name)
    st = state_from(n, x)
    st.run_parts(rec, offs)
    assert np.abs(st.amplitudes() - amps).max() <= TOL


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 9, 12, 13, 14, 16])
def test_all_gates_per_gate_part_parts(port, n):
    gates = all_gates(n, 150, 1000 + n)
    want = port.run(n, to_records(gates))
    a = abi.State(n)
    for g in gates:
        a.apply(g)
    assert np.abs(a.amplitudes() - want).max() <= TOL
    b = abi.State(n)
    b.run_part(gates)
    assert np.abs(b.amplitudes() - want).max() <= TOL
    if n >= 2:
        parts = partition.partition_acyclic(gates, min(n, 5))
        rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
        c = abi.State(n)
        c.run_parts(rec, offs)
        assert np.abs(c.amplitudes() - want).max() <= TOL


@pytest.mark.parametrize("m", [4, 6, 8, 10, 11, 12, 13])
def test_tile_sizes(port, m):
    n = 15
    gates = all_gates(n, 120, 7)
    want = port.run(n, to_records(gates))
    prev = abi.set_tile_qubits(m)
    try:
        st = abi.State(n)
        st.run_part(gates)
        assert np.abs(st.amplitudes() - want).max() <= TOL
    finally:
        abi.set_tile_qubits(prev)


@pytest.mark.parametrize("r,m", [(3, 3), (3, 5), (3, 9), (3, 11), (4, 4), (4, 9), (4, 11)])
def test_amplitudes_per_thread(port, r, m):
    """complex128 passes with 8 (r = 3, the default) or 16 (r = 4) amplitudes
    per thread give the oracle's result, with and without two-qubit dense ops."""
    n = 14
    gates = all_gates(n, 140, 31 + m)
    want = port.run(n, to_records(gates))
    prev_m = abi.set_tile_qubits(m)
    prev_r = abi.set_k1_reg_bits(r)
    try:
        st = abi.State(n)
        st.run_part(gates)
        assert np.abs(st.amplitudes() - want).max() <= TOL
        u3 = circuits.random_u3_cz(n, 6, 5)
        parts = partition.partition_dfs(u3, 9)
        rec, offs = part_offsets(partition.parts_to_gates(u3, parts))
        st.set_basis(0)
        st.run_parts(rec, offs)
        assert np.abs(st.amplitudes() - port.run(n, to_records(u3))).max() <= TOL
    finally:
        abi.set_tile_qubits(prev_m)
        abi.set_k1_reg_bits(prev_r)


def test_config0_20q_against_reference(ref):
    """20 qubits, 20 random layers, acyclic parts of <= 10 qubits."""
    gates = circuits.random_layered(20, 20, 0)
    parts = partition.partition_acyclic(gates, 10)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = ref.run(20, rec, offs, mode=1, opt_slots=1)
    st = abi.State(20)
    st.run_parts(rec, offs)
    assert np.abs(st.amplitudes() - want).max() <= TOL


def test_qft_22q_against_port(port):
    gates, x = circuits.qft(22, 3)
    parts = partition.partition_acyclic(gates, 7)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    init = np.zeros(1 << 22, complex)
    init[x] = 1
    want = port.run(22, to_records(gates), init_state=init)
    st = state_from(22, x)
    st.run_parts(rec, offs)
    assert np.abs(st.amplitudes() - want).max() <= TOL


def qft_expected(n, x, ks):
    """QFT|x> amplitude at index k (textbook phases, bit-reversed by the final swaps)."""
    N = 1 << n
    frac = (np.uint64(x) * np.asarray(ks, dtype=np.uint64)) % np.uint64(N)  # exact x*k mod N
    return np.exp(2j * math.pi * frac.astype(np.float64) / N) / math.sqrt(N)


@pytest.mark.parametrize("k", [6, 8])
def test_qft_30q_full_size_analytic(k):
    """Full-size config: 30-qubit QFT on a random basis state; sampled
    amplitudes equal the closed form and the norm stays 1."""
    n = 30
    gates, x = circuits.qft(n, 2)
    parts = partition.partition_acyclic(gates, k)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st = state_from(n, x)
    st.run_parts(rec, offs)
    assert abs(st.norm2() - 1) <= 1e-12
    st.canonicalize()
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(1 << n, 64, replace=False))
    got = np.array([st.raw(int(i), 1)[0] for i in idx])
    want = qft_expected(n, x, idx)
    assert np.abs(got - want).max() <= 1e-12


def test_forward_inverse_identity_28q():
    """verify_compute's property (qasm_assembler_standalone.py:716-1198): a
    circuit followed by its inverse returns |0..0>."""
    n = 28
    rng = np.random.default_rng(5)
    fwd = []
    for _ in range(6):
        for q in range(n):
            fwd.append(Gate("U3", (q,), params=tuple(rng.uniform(0, 2 * np.pi, 3))))
        for a, b in rng.permutation(n).reshape(-1, 2):
            fwd.append(Gate("Z", (int(b),), (int(a),)))
    inv = []
    for g in reversed(fwd):
        if g.name == "U3":
            t, p, l = (v.real for v in g.params)
            inv.append(Gate("U3", g.targets, params=(-t, -l, -p)))  # U3(t,p,l)^-1 = U3(-t,-l,-p)
        else:
            inv.append(g)
    gates = fwd + inv
    parts = partition.partition_acyclic(gates, 8)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st = abi.State(n)
    st.run_parts(rec, offs)
    a0 = st.raw(0, 4)
    assert abs(a0[0] - 1) <= 1e-12 and np.abs(a0[1:]).max() <= 1e-12
    assert abs(st.norm2() - 1) <= 1e-12


def test_c64_state(port):
    n = 14
    gates = circuits.random_layered(n, 10, 3)
    want = port.run(n, to_records(gates))
    st = abi.State(n, abi.C64)
    parts = partition.partition_acyclic(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st.run_parts(rec, offs)
    got = st.amplitudes().astype(complex)
    assert np.abs(got - want).max() <= 1e-5


def test_bad_gates_raise_and_leave_state():
    st = abi.State(4)
    st.apply(Gate("H", (0,)))
    before = st.amplitudes()
    with pytest.raises(abi.HisvError):
        st.apply(Gate("X", (7,)))  # unallocated qubit
    with pytest.raises(abi.HisvError):
        st.apply(Gate("X", (1,), (1,)))  # control == target
    with pytest.raises(abi.HisvError):
        st.run_parts(to_records([Gate("H", (1,)), Gate("ALLOC", (2,))]), np.array([0, 1, 2]))
    assert np.abs(st.amplitudes() - before).max() == 0


def test_empty_part_and_identity():
    st = abi.State(5)
    st.run_part([])
    st.run_part([Gate("I", (3,))])
    a = st.amplitudes()
    assert a[0] == 1 and np.abs(a[1:]).max() == 0


def _host_available():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return float(line.split()[1]) * 1024
    except OSError:
        pass
    return 0.0


def test_qft_30q_against_reference_all_amplitudes(ref):
    """Config 1 in full: the 30-qubit QFT on a random basis state |x> through
    the GPU plain path (DFS-order parts of <= 7 qubits; the final swaps and the
    controlled phases included) against the reference's own per-gate path on
    the host cores (|x> prepared by X gates), every one of the 2^30 amplitudes
    to 1e-12, compared in 2^26-amplitude chunks."""
    n = 30
    if _host_available() < 40 * 2 ** 30:
        pytest.skip("needs ~40 GiB of host memory for the reference's 16 GiB state and its copy")
    gates, x = circuits.qft(n, 3)
    prep = [Gate("X", (q,)) for q in range(n) if (x >> q) & 1]
    want = ref.run(n, to_records(prep + gates), mode=0)
    parts = partition.partition_dfs(gates, 7)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st = abi.State(n, abi.C128)
    st.set_basis(x)
    st.run_parts(rec, offs)
    st.canonicalize()
    worst = 0.0
    step = 1 << 26
    for first in range(0, 1 << n, step):
        worst = max(worst, float(np.abs(st.raw(first, step) - want[first:first + step]).max()))
    st.close()
    assert worst <= 1e-12, worst
