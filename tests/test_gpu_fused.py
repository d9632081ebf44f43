"""Precision form: FP64-composed 64x64 unitaries (K5) applied to complex64
states on the tensor cores with split-BF16 operands (K4).

Tolerances: composed unitaries match the oracle to 1e-12; the complex64
result keeps fidelity loss 1 - |<psi_fp64|psi>|^2 <= 1e-6 (the precision
form's bound) and max amplitude error <= 1e-5 against complex128."""
import numpy as np
import pytest

from hisvsim_b200 import abi, circuits, partition
from hisvsim_b200.gates import Gate, part_offsets, to_records

pytestmark = pytest.mark.gpu


def fid(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def test_compose_matches_oracle(port):
    n = 8
    gates = circuits.random_layered(n, 4, 3) + [Gate("RXX", (1, 4), params=(0.4,)),
                                                Gate("SWAP", (2, 5), (0,))]
    parts = partition.partition_acyclic(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    U, Q = abi.fused_compose(n, rec, offs)
    for p in range(len(parts)):
        pg = to_records([gates[i] for i in parts[p]])
        place = lambda j: sum(((j >> b) & 1) << int(Q[p][b]) for b in range(6))
        for j in range(64):
            init = np.zeros(1 << n, complex)
            init[place(j)] = 1
            out = port.run(n, pg, init_state=init)
            col = np.array([out[place(i)] for i in range(64)])
            assert np.abs(col - U[p][:, j]).max() <= 1e-12


@pytest.mark.parametrize("n", [10, 11, 12, 14, 16])
def test_fused_against_oracle(port, n):
    gates = circuits.random_u3_cz(n, 6, 5)
    parts = partition.partition_acyclic(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    st = abi.State(n, abi.C64)
    st.run_fused(rec, offs, 0)  # three BF16 products
    got = st.amplitudes().astype(complex)
    assert 1 - fid(want, got) <= 1e-8
    assert np.abs(got - want).max() <= 1e-5


def test_fused_all_gate_kinds(port):
    n = 12
    import tests.golden.make_golden as mg

    gates = [g for g in mg.all_gate_circuit(n, 120, 77) if len(set(g.qubits)) <= 6]
    parts = partition.partition_acyclic(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    st = abi.State(n, abi.C64)
    st.run_fused(rec, offs)
    got = st.amplitudes().astype(complex)
    # the all-gate mix is not unitary (C1 / C2 with arbitrary entries): compare
    # directions and relative error
    assert 1 - fid(want, got) <= 1e-8
    assert np.abs(got - want).max() <= 1e-5 * max(1.0, np.abs(want).max())


def test_single_product_is_coarser(port):
    n = 12
    gates = circuits.random_u3_cz(n, 6, 6)
    parts = partition.partition_acyclic(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    st = abi.State(n, abi.C64)
    st.run_fused(rec, offs, 1)
    loss = 1 - fid(want, st.amplitudes().astype(complex))
    assert 1e-9 < loss <= 1e-3


def test_fused_28q_against_plain_complex128():
    n = 28
    gates = circuits.random_u3_cz(n, 10, 1)
    fparts = partition.partition_acyclic(gates, 6)
    frec, foffs = part_offsets(partition.parts_to_gates(gates, fparts))
    pparts = partition.partition_acyclic(gates, 9)
    prec, poffs = part_offsets(partition.parts_to_gates(gates, pparts))
    f = abi.State(n, abi.C64)
    f.run_fused(frec, foffs)
    p = abi.State(n, abi.C128)
    p.run_parts(prec, poffs)
    c = p.compare(f)
    assert 1 - c["fidelity"] <= 1e-6
    assert c["max_abs_diff"] <= 1e-5
    h = p.compare_host(f.raw())
    assert abs(h["fidelity"] - c["fidelity"]) <= 1e-12


def test_fused_errors():
    with pytest.raises(abi.HisvError):
        abi.State(12, abi.C128).run_fused(to_records([Gate("H", (0,))]), np.array([0, 1]))
    with pytest.raises(abi.HisvError):
        abi.State(8, abi.C64).run_fused(to_records([Gate("H", (0,))]), np.array([0, 1]))
    big = [Gate("X", (q,)) for q in range(7)]
    with pytest.raises(abi.HisvError):
        abi.State(12, abi.C64).run_fused(to_records(big), np.array([0, 7]))


@pytest.mark.parametrize("shape", [(1, 10), (1, 11), (1, 12), (1, 13), (2, 11), (2, 12)])
def test_fused_pass_shapes(port, shape):
    """Every pass shape (unitaries per pass, tile bits) gives the same result
    (one unitary per pass: operands straight from and to HBM)."""
    n = 15
    gates = circuits.random_u3_cz(n, 8, 17)
    parts = partition.partition_acyclic(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    prev = abi.set_fused_shape(*shape)
    try:
        st = abi.State(n, abi.C64)
        st.run_fused(rec, offs, 0)
        got = st.amplitudes().astype(complex)
    finally:
        abi.set_fused_shape(prev // 100, prev % 100)
    assert 1 - fid(want, got) <= 1e-8
    assert np.abs(got - want).max() <= 1e-5


@pytest.mark.parametrize("variant,bits", [(1, 13), (2, 12), (2, 13)])
@pytest.mark.parametrize("qubits", [[11, 0, 5, 3, 9, 7], [0, 11, 5, 3, 9, 7], [12, 2, 5, 3, 9, 7],
                                    [1, 2, 3, 4, 5, 6]])
def test_fused_apply_given_unitary(variant, bits, qubits):
    """hs_fused_apply with a random 64x64 unitary on scattered qubits, against
    numpy on the complex128 amplitudes: slot 0 as a later local bit (the
    bulk-loaded kernel hands such passes to the warp-specialised one), as
    local bit 0, outside the unitary, and a unitary on slots 1-6."""
    n = 13
    rng = np.random.default_rng(4)
    z = rng.normal(size=(64, 64)) + 1j * rng.normal(size=(64, 64))
    u, _ = np.linalg.qr(z)
    prev = abi.set_k4_variant(variant)
    shape = abi.set_fused_shape(1, bits)
    try:
        _apply_and_check(n, u, qubits)
    finally:
        abi.set_k4_variant(prev)
        abi.set_fused_shape(shape // 100, shape % 100)


def _apply_and_check(n, u, qubits):
    st = abi.State(n, abi.C64)
    gates = circuits.random_u3_cz(n, 3, 8)
    for g in gates:
        st.apply(g)
    before = st.amplitudes().astype(complex)
    st.fused_apply(u, qubits)
    got = st.amplitudes().astype(complex)
    # numpy: axis for qubit q of a C-ordered reshape is n-1-q
    psi = before.reshape([2] * n)
    axes = [n - 1 - q for q in qubits][::-1]  # U index bit 5 first
    moved = np.moveaxis(psi, axes, range(6)).reshape(64, -1)
    out = (u @ moved).reshape([2] * 6 + [2] * (n - 6))
    want = np.moveaxis(out, range(6), axes).reshape(-1)
    assert 1 - fid(want, got) <= 1e-8
    assert np.abs(got - want).max() <= 1e-5


@pytest.mark.parametrize("variant,bits", [(0, 13), (1, 13), (1, 12), (2, 10), (2, 11), (2, 12),
                                          (2, 13)])
@pytest.mark.parametrize("n", [10, 13, 17])
def test_k4_variants(port, variant, bits, n):
    """The one-unitary-per-pass kernels (direct, warp-specialised,
    bulk-loaded) agree with the oracle, including states with fewer tiles
    than SMs."""
    gates = circuits.random_u3_cz(n, 6, 23)
    parts = partition.partition_dfs(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    prev = abi.set_k4_variant(variant)
    shape = abi.set_fused_shape(1, bits)
    try:
        st = abi.State(n, abi.C64)
        st.run_fused(rec, offs, 0)
        got = st.amplitudes().astype(complex)
    finally:
        abi.set_k4_variant(prev)
        abi.set_fused_shape(shape // 100, shape % 100)
    assert 1 - fid(want, got) <= 1e-8
    assert np.abs(got - want).max() <= 1e-5


@pytest.mark.parametrize("n", [12, 14, 17, 20])
def test_two_unitaries_per_pass(port, n):
    """Two fused unitaries per state pass on 2^12 tiles (the first product
    goes back to the tile's shared buffer and feeds the second on chip):
    DFS-order parts of a U3 + CZ circuit against the oracle."""
    gates = circuits.random_u3_cz(n, 10, 300 + n)
    parts = partition.partition_dfs(gates, 6)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    prev = abi.set_fused_shape(2, 12)
    try:
        st = abi.State(n, abi.C64)
        st.run_fused(rec, offs, 0)
        got = st.amplitudes().astype(complex)
    finally:
        abi.set_fused_shape(prev // 100, prev % 100)
    assert 1 - fid(want, got) <= 1e-8
    assert np.abs(got - want).max() <= 1e-5
