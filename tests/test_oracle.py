"""The oracle, pinned: known answers from the reference's own doctest block
(state_vector.hpp:1404-1738, restated as facts) and the golden vectors the
reference produced (tests/golden/make_golden.py), checked against both the
reference harness and the C restatement (oracle/port.c)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden
from hisvsim_b200 import circuits, partition
from hisvsim_b200.gates import Gate, part_offsets, to_records

S2 = 0.707106781186547524401


def run1(oracle, n, gates, init):
    return oracle.run(n, to_records(gates), init_state=np.asarray(init, dtype=complex))


@pytest.fixture(params=["ref", "port"])
def oracle(request):
    return request.getfixturevalue(request.param)


# single-qubit truth tables (state_vector.hpp:1439-1503)
KAT1 = [
    ("I", [1, 0], [1, 0]), ("I", [0, 1], [0, 1]),
    ("X", [1, 0], [0, 1]), ("X", [0, 1], [1, 0]),
    ("Y", [1, 0], [0, 1j]), ("Y", [0, 1], [-1j, 0]),
    ("Z", [1, 0], [1, 0]), ("Z", [0, 1], [0, -1]),
    ("H", [1, 0], [S2, S2]), ("H", [0, 1], [S2, -S2]),
    ("S", [1, 0], [1, 0]), ("S", [0, 1], [0, 1j]),
    ("T", [1, 0], [1, 0]), ("T", [0, 1], [0, np.sqrt(1j)]),
]


@pytest.mark.parametrize("name,inp,out", KAT1)
def test_single_qubit_kat(oracle, name, inp, out):
    got = run1(oracle, 1, [Gate(name, (0,))], inp)
    assert np.abs(got - np.asarray(out)).max() <= 1e-10


@pytest.mark.parametrize("inv,fwd", [("SDG", "S"), ("TDG", "T")])
@pytest.mark.parametrize("inp", [[1, 0], [0, 1]])
def test_inverse_pairs(oracle, inv, fwd, inp):
    got = run1(oracle, 1, [Gate(inv, (0,)), Gate(fwd, (0,))], inp)
    assert np.abs(got - np.asarray(inp)).max() <= 1e-10


BASIS2 = [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]]


@pytest.mark.parametrize("i,o", [(0, 0), (1, 2), (2, 1), (3, 3)])
def test_swap_kat(oracle, i, o):  # state_vector.hpp:1506-1531
    got = run1(oracle, 2, [Gate("SWAP", (0, 1))], BASIS2[i])
    assert np.abs(got - np.asarray(BASIS2[o])).max() <= 1e-10


@pytest.mark.parametrize("i,o", [(0, 0), (1, 1), (2, 3), (3, 2)])
def test_cx_kat(oracle, i, o):  # control qubit 1, target 0 (state_vector.hpp:1533-1565)
    got = run1(oracle, 2, [Gate("X", (0,), (1,))], BASIS2[i])
    assert np.abs(got - np.asarray(BASIS2[o])).max() <= 1e-10


@pytest.mark.parametrize("i", range(4))
def test_cy_is_s_cx_sdg(oracle, i):  # state_vector.hpp:1567-1602
    a = run1(oracle, 2, [Gate("Y", (1,), (0,))], BASIS2[i])
    b = run1(oracle, 2, [Gate("SDG", (1,)), Gate("X", (1,), (0,)), Gate("S", (1,))], BASIS2[i])
    assert np.abs(a - b).max() <= 1e-10


@pytest.mark.parametrize("i", range(4))
def test_cz_is_h_cx_h(oracle, i):  # state_vector.hpp:1604-1639
    a = run1(oracle, 2, [Gate("Z", (1,), (0,))], BASIS2[i])
    b = run1(oracle, 2, [Gate("H", (1,)), Gate("X", (1,), (0,)), Gate("H", (1,))], BASIS2[i])
    assert np.abs(a - b).max() <= 1e-10


@pytest.mark.parametrize("i,o", [(0, [1, 0, 0, 0]), (1, [0, 1, 0, 0]), (2, [0, 0, S2, S2]),
                                 (3, [0, 0, S2, -S2])])
def test_ch_kat(oracle, i, o):  # state_vector.hpp:1641-1667
    got = run1(oracle, 2, [Gate("H", (0,), (1,))], BASIS2[i])
    assert np.abs(got - np.asarray(o)).max() <= 1e-10


def test_probability_after_h(ref, port):  # state_vector.hpp:1711-1737
    st = run1(port, 1, [Gate("H", (0,))], [1, 0])
    for p in (ref.probability(1, st, 0, 0), port.probability(1, st, 0, 0)):
        assert abs(p - 0.5) <= 1e-10
    st = run1(port, 1, [Gate("X", (0,))], [1, 0])
    assert abs(ref.probability(1, st, 0, 1) - 1.0) <= 1e-10
    assert abs(port.probability(1, st, 0, 1) - 1.0) <= 1e-10


@pytest.mark.parametrize("name", golden_names())
def test_golden_port(port, name):
    n, rec, offs, x, amps = load_golden(name)
    init = np.zeros(1 << n, complex)
    init[x] = 1
    mode = 1 if len(offs) > 2 else 0
    got = port.run(n, rec, offs, mode=mode, opt_slots=1, init_state=init)
    assert np.abs(got - amps).max() <= 1e-12


@pytest.mark.parametrize("name", golden_names())
def test_golden_ref_reproducible(ref, name):
    n, rec, offs, x, amps = load_golden(name)
    init = np.zeros(1 << n, complex)
    init[x] = 1
    got = ref.run(n, rec, init_state=init, threads=2)  # per-gate path
    assert np.abs(got - amps).max() <= 1e-12


def test_part_path_equals_per_gate(ref, port):
    gates = circuits.random_layered(16, 6, 3)
    parts = partition.partition_acyclic(gates, 8)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    a = ref.run(16, to_records(gates), threads=4)
    b = ref.run(16, rec, offs, mode=1, opt_slots=1, threads=4)
    c = port.run(16, rec, offs, mode=1, opt_slots=0)
    assert np.abs(a - b).max() <= 1e-12 and np.abs(a - c).max() <= 1e-12


def test_gather_slots_semantics(port):
    # SvSimMPI::gather_qubits order: non-proc slots in order, then proc slots
    n = 6
    st = np.arange(1 << n).astype(complex)
    out = port.gather_slots(st, n, [1, 4])
    src = [0, 2, 3, 5, 1, 4]
    for x in range(1 << n):
        y = sum(((x >> s) & 1) << j for j, s in enumerate(src))
        assert out[y] == st[x]


def test_reference_rejects_alloc(ref):
    with pytest.raises(ValueError):
        ref.run(2, to_records([Gate("ALLOC", (0,))]))


# ---- the cost model's network (oracle/mlp.py), pinned by finite differences


def test_mlp_oracle_gradient_matches_finite_differences():
    from oracle import mlp

    rng = np.random.default_rng(3)
    d = 7
    p = rng.normal(0, 0.3, mlp.num_params(d))
    x = rng.normal(0, 1, (19, d))
    y = rng.normal(0, 1, 19)
    loss, g = mlp.loss_and_grad(p, x, y)
    idx = rng.choice(p.size, 60, replace=False)
    idx = np.concatenate([idx, [p.size - 1, mlp.num_params(d) - 65]])  # b4 and a w4 entry
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        fd = (mlp.loss_and_grad(p + e, x, y)[0] - mlp.loss_and_grad(p - e, x, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
    assert loss == pytest.approx(np.mean((mlp.forward(p, x)[0] - y) ** 2))


def test_mlp_oracle_adam_known_step():
    from oracle import mlp

    p = np.array([1.0, -2.0, 0.5])
    g = np.array([0.1, -0.3, 0.0])
    m = np.zeros(3)
    v = np.zeros(3)
    mlp.adam_step(p, g, m, v, 1, 0.01)
    # first bias-corrected step moves each coordinate by lr * sign(g) (g != 0)
    assert p == pytest.approx([0.99, -1.99, 0.5], abs=1e-7)
