"""Generate tests/golden/qasm_golden.json from the reference's own Python.

Runs (in the build container only; the reference is not present elsewhere)
the reference driver's QASM_parser, convert_param, produce_dot_file and the
QASM-to-BoundGate lowering of verify_compute, taken from
qasm_assembler_standalone.py by AST extraction (the module itself imports
mpi4py and the compiled simulator, which are absent), on the .qasm files of
tests/golden/qasm/ (circuits written for these tests).  The compiled simulator
is replaced by a recorder of the AggregateGate / BoundGate constructor calls.

    python tests/golden/make_qasm_golden.py [path/to/reference]
"""
import ast
import collections
import copy
import json
import math
import os
import re
import sys
from datetime import datetime

HERE = os.path.dirname(os.path.abspath(__file__))
REF = (sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HISV_REFERENCE")
       or os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                       "reference"))
SRC = os.path.join(REF, "qasm_assembler_standalone.py")

PARAM_CASES = ["0.5", "-0.75", "3", "1e-3", "0.25e1", "pi", "-pi", "pi/2", "-pi/2", "pi/8",
               "2/pi", "pi*2", "2*pi", "-2*pi", "3*pi/4", "0.1"]


class Recorder:
    """Stands in for svsimulator_py_wrapper: records what the driver binds."""

    def __init__(self):
        self.bound = []

    def _ag(kind):
        def make(self, name, *params):
            return ("ag", kind, name, [complex(p) if not isinstance(p, int) else p for p in params])
        return make

    AggregateGate_0 = _ag("0")
    AggregateGate_1 = _ag("1")
    AggregateGate_2 = _ag("2")
    AggregateGate_3 = _ag("3")
    AggregateGate_C1 = _ag("C1")
    AggregateGate_C2 = _ag("C2")
    AggregateGate_Frac = _ag("Frac")

    def AggregateGateFactory(self, ag):
        return ag

    def BoundGate(self, factory, controls, targets):
        rec = self

        class BG:
            def apply(self, sim):
                rec.bound.append({"name": factory[2], "params": [[p.real, p.imag] for p in factory[3]],
                                  "controls": list(controls), "targets": list(targets)})
        return BG()

    def StateVector(self, n, alloc):
        class SV:
            def __eq__(self, other):
                return True
        return SV()


def extract(names):
    tree = ast.parse(open(SRC).read())
    keep = []
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names:
            keep.append(node)
        elif isinstance(node, ast.Assign) and any(
                isinstance(t, ast.Name) and t.id in names for t in node.targets):
            keep.append(node)
    return ast.Module(body=keep, type_ignores=[])


def main():
    import networkx as nx

    rec = Recorder()
    captured = []
    ns = {"re": re, "math": math, "collections": collections, "copy": copy, "nx": nx,
          "datetime": datetime, "svsim": rec, "allocation_scheme": 0, "acc_timer": 0,
          "start_timer": 0, "print": lambda *a, **k: None}
    names = {"gates", "GATE_NOPARAM", "GATE_ONEPARAM", "GATE_TWOPARAM", "GATE_THREEPARAM",
             "GATE_C1", "GATE_C2", "GATE_FRAC", "measure_op", "TargetGate", "QASM_parser",
             "convert_param", "handle_pi", "generate_void_vertex", "get_unique_name",
             "add_input_node_pass", "produce_dot_file"}
    exec(compile(extract(names), SRC, "exec"), ns)
    nx.drawing.nx_pydot.write_dot = lambda G, path: captured.append(G.copy())

    out = {"params": [[v, ns["convert_param"](v)] for v in PARAM_CASES], "files": {}}
    for fname in sorted(os.listdir(os.path.join(HERE, "qasm"))):
        path = os.path.join(HERE, "qasm", fname)
        p = ns["QASM_parser"](path)
        p.identify_qubit_allocation()
        p.identify_custom_gate_pass()
        p.identify_gate_pass()
        p.order_gate_list()
        p.expand_qubit()
        uq = p.create_universal_qubit()
        ops = [{"gate": op.get_gate(), "params": list(op.get_params()), "qubits": op.get_qubits(),
                "line": op.get_index()} for op in p.ordered_gate_list]
        rec.bound = []
        p.verify_compute()
        nforward = sum(1 for op in p.ordered_gate_list if op.get_gate() != "measure")
        captured.clear()
        ns["measure_op"].clear()
        ns["produce_dot_file"](p.ordered_gate_list, path, "out")
        graphs = [{"nodes": {str(n): {k: v for k, v in d.items()} for n, d in G.nodes(data=True)},
                   "edges": sorted([str(u), str(v), d["label"]] for u, v, d in G.edges(data=True))}
                  for G in captured]
        out["files"][fname] = {"qubits": uq, "ops": ops, "bound": rec.bound[:nforward],
                               "dot": graphs}
    with open(os.path.join(HERE, "qasm_golden.json"), "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print("wrote", os.path.join(HERE, "qasm_golden.json"))


if __name__ == "__main__":
    main()
