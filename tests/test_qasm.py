"""QASM front end (hisvsim_b200/qasm.py) against the reference driver's own
parser, parameter conversion, BoundGate lowering and DAG writer, recorded in
tests/golden/qasm_golden.json by tests/golden/make_qasm_golden.py."""
import json
import math
import os

import pytest

from conftest import ROOT
from hisvsim_b200 import qasm

GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLD, "qasm_golden.json")) as f:
        return json.load(f)


def program(name, params="reference"):
    return qasm.load(os.path.join(GOLD, "qasm", name), params)


def test_reference_param_conversion(golden):
    for text, want in golden["params"]:
        assert qasm.convert_param_reference(text) == want, text


def test_exact_params_fix_the_reference_conversion():
    p = program("params.qasm", "exact")
    got = [op.params for op in p.ops]
    assert got[0] == (1e-3,) and got[1] == (math.pi,)
    assert got[2] == pytest.approx((3 * math.pi / 4,))
    assert got[3] == pytest.approx((2 / math.pi,)) and got[4] == pytest.approx((-math.pi / 2,))
    assert got[6] == pytest.approx((math.pi / 2, 2.5, -0.75))
    assert got[7] == pytest.approx((-2 * math.pi,))


@pytest.mark.parametrize("name", ["basic.qasm", "registers.qasm", "custom.qasm", "params.qasm"])
def test_ordered_ops_match_reference_parser(golden, name):
    g = golden["files"][name]
    p = program(name)
    assert p.num_qubits == len(g["qubits"])
    assert len(p.ops) == len(g["ops"])
    for op, want in zip(p.ops, g["ops"]):
        assert op.name == want["gate"]
        assert op.line - 1 == want["line"]
        assert list(op.params) == pytest.approx(want["params"])
        if op.name == "measure":
            assert p.qubit_name(op.qubits[0]) == want["qubits"][0]
        else:
            assert [g["qubits"][p.qubit_name(q)] for q in op.qubits] == \
                [g["qubits"][q] for q in want["qubits"]]


@pytest.mark.parametrize("name", ["basic.qasm", "registers.qasm", "custom.qasm", "params.qasm"])
def test_lowering_matches_reference_bound_gates(golden, name):
    g = golden["files"][name]
    gates = program(name).circuit()
    assert len(gates) == len(g["bound"])
    for gate, want in zip(gates, g["bound"]):
        assert gate.name == want["name"]
        assert list(gate.controls) == want["controls"]
        got = [x for c in gate.params for x in (c.real, c.imag)]
        assert got == pytest.approx([x for pair in want["params"] for x in pair])
        if gate.name == "SWAP" and not gate.controls:
            # the reference binds a bare swap with no qubits; here it acts on both
            assert want["targets"] == [] and len(gate.targets) == 2
        else:
            assert list(gate.targets) == want["targets"]


@pytest.mark.parametrize("name", ["basic.qasm", "registers.qasm", "custom.qasm", "params.qasm"])
def test_dag_matches_reference_dot_graphs(golden, name, tmp_path):
    g = golden["files"][name]
    p = program(name)
    graphs = qasm.dag_graphs(p)
    assert len(graphs) == len(g["dot"])
    for (nodes, edges), want in zip(graphs, g["dot"]):
        assert nodes == want["nodes"]
        assert sorted([list(e) for e in edges]) == want["edges"]
    paths = qasm.write_dot(p, str(tmp_path / "circ"))
    assert len(paths) == len(graphs)
    for path, (nodes, edges) in zip(paths, graphs):
        rn, re_ = qasm.read_dot(path)
        assert rn == nodes and sorted(re_) == sorted(edges)


def test_extensions_parameterised_gates_broadcast_one_line():
    src = """OPENQASM 2.0; qreg a[2]; qreg b[2]; creg c[2];
    gate rot(t, u) x, y { rz(t) x; cx x, y; ry(u / 2) y; }
    rot(pi/2, 0.4) a[0], b[1]; cx a, b; measure b -> c; // comment
    """
    p = qasm.parse(src)
    names = [(op.name, op.qubits) for op in p.ops]
    assert names == [("rz", (0,)), ("cx", (0, 3)), ("ry", (3,)), ("cx", (0, 2)), ("cx", (1, 3)),
                     ("measure", (2,)), ("measure", (3,))]
    assert p.ops[0].params == pytest.approx((math.pi / 2,))
    assert p.ops[2].params == pytest.approx((0.2,))
    assert p.measured_qubits() == [2, 3]


@pytest.mark.parametrize("src,msg", [
    ("qreg q[2]; foo q[0];", "unknown gate"),
    ("qreg q[2]; cx q[0];", "takes 2 qubits"),
    ("qreg q[2]; rx q[0];", "takes 1 parameters"),
    ("qreg q[2]; h q[2];", "out of range"),
    ("qreg q[2]; cx q[0],q[0];", "twice"),
    ("qreg q[2]; creg c[2]; if (c==1) x q[0];", "classically"),
    ("qreg q[2]; opaque g a;", "opaque"),
    ("qreg q[2]; gate g a { g a; } g q[0];", "nest"),
    ("qreg q[2]; rx(1/0) q[0];", "division"),
    ("qreg q[2]; rx(foo) q[0];", "unknown symbol"),
    ("qreg q[3]; qreg r[2]; cx q, r;", "do not match"),
])
def test_errors(src, msg):
    with pytest.raises(qasm.QasmError, match=msg):
        qasm.parse(src)


def test_part_file_parts_skip_measurements(tmp_path):
    p = program("registers.qasm")
    lines = [f"{i + 1} n{i} {0 if i < 8 else 1}" for i in range(len(p.ops))]
    path = tmp_path / "parts"
    path.write_text("\n".join(lines) + "\n")
    parts = qasm.parts_from_file(p, str(path))
    assert sum(len(x) for x in parts) == len(p.circuit())
    assert p.ops[7].name == "measure"
    assert parts[0] == list(range(7))  # ops 0..7: seven gates and a measurement
