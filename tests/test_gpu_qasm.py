"""QASM programs through the GPU path: the front end's gate lists run in
parts (acyclic, and from a part file) and gate by gate, against the oracle
on the same gate list (complex128, 1e-12)."""
import os

import numpy as np
import pytest

from conftest import ROOT
from hisvsim_b200 import abi, qasm
from hisvsim_b200.gates import to_records

pytestmark = pytest.mark.gpu
GOLD = os.path.join(ROOT, "tests", "golden", "qasm")


@pytest.mark.parametrize("name", ["basic.qasm", "registers.qasm", "custom.qasm", "params.qasm"])
@pytest.mark.parametrize("params", ["exact", "reference"])
def test_qasm_programs_match_oracle(port, name, params):
    p = qasm.load(os.path.join(GOLD, name), params)
    gates = p.circuit()
    want = port.run(p.num_qubits, to_records(gates))
    for k in (3, 4, p.num_qubits):  # ccx / cswap touch three qubits
        st = qasm.simulate(p, max_qubits=k)
        assert np.abs(st.amplitudes() - want).max() <= 1e-12
    one = abi.State(p.num_qubits)
    for g in gates:
        one.apply(g)
    assert np.abs(one.amplitudes() - want).max() <= 1e-12


def test_qasm_with_part_file(port, tmp_path):
    p = qasm.load(os.path.join(GOLD, "registers.qasm"))
    path = tmp_path / "registers.qasm_part_nat"
    path.write_text("".join(f"{i + 1} n{i} {i // 4}\n" for i in range(len(p.ops))))
    parts = qasm.parts_from_file(p, str(path))
    st = qasm.simulate(p, parts=parts)
    want = port.run(p.num_qubits, to_records(p.circuit()))
    assert np.abs(st.amplitudes() - want).max() <= 1e-12
