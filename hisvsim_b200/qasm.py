"""OpenQASM 2 front end: circuit text -> the gate list the C ABI and the
pybind module take.

It keeps the reference driver's semantics (``QASM_parser``,
qasm_assembler_standalone.py:64-408, and the QASM-to-BoundGate lowering of its
part runners, e.g. :741-952 and :1802-2010):

* registers are numbered in declaration order, qubit ``r[i]`` of the k-th
  register gets index ``sum(sizes of earlier registers) + i``
  (``create_universal_qubit``, :3569-3575);
* a one-qubit gate applied to a whole register is applied to each of its
  qubits (``expand_qubit``, :285-298); user-defined ``gate`` blocks are
  expanded in place (``order_gate_list``, :209-282);
* ``measure`` stays in the ordered operation list (part files count it,
  :1795-1801) but applies nothing; ``barrier`` is dropped; ``reset`` and
  ``id`` lower to the identity gate ``I`` (an unknown basic gate lowers to
  ``AggregateGate_0("I")``, :771-772);
* ``cx/cy/cz/ch/crx/cry/crz/cu1/cu3`` become X/Y/Z/H/RX/RY/RZ/U1/U3 with one
  control, ``ccx/c3x/c4x`` X with 2/3/4 controls, ``cswap`` SWAP with one
  control, ``rxx/ryy/rzz`` two-target gates.

Differences, all where the reference fails or is wrong:

* parameters are evaluated as expressions (``pi``, numbers with exponents,
  ``+ - * / ^``, parentheses, sin/cos/tan/exp/ln/sqrt).  The reference's
  ``convert_param`` (:3581-3617) returns 1.0 for any literal containing an
  ``e`` (so ``1e-3`` -> 1.0), 0.0 for a bare ``pi``, and mis-evaluates
  ``3*pi/4`` as 3*pi.  ``params="reference"`` reproduces that behaviour;
* ``swap a,b`` acts on both qubits (the reference binds it with empty control
  and target lists, :770-952 has no two-qubit SWAP case);
* parameterised ``gate`` definitions, several statements per line, one-line
  gate bodies and register broadcasts of multi-qubit gates are accepted.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

from .gates import Gate

# The reference's accepted gate names (qasm_assembler_standalone.py:19) and
# the ones its lowering handles but its parse list lacks.
REFERENCE_GATES = ("u3", "u2", "u1", "id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "rx",
                   "ry", "rz", "cz", "cx", "cy", "ch", "ccx", "crz", "cu1", "cu3", "reset",
                   "swap", "rxx", "ryy", "rzz", "cswap")
EXTRA_GATES = ("crx", "cry", "c3x", "c4x")

# name -> (basic gate, controls, targets, parameter count)
_LOWER = {
    "u3": ("U3", 0, 1, 3), "u2": ("U2", 0, 1, 2), "u1": ("U1", 0, 1, 1),
    "id": ("I", 0, 1, 0), "reset": ("I", 0, 1, 0),
    "x": ("X", 0, 1, 0), "y": ("Y", 0, 1, 0), "z": ("Z", 0, 1, 0), "h": ("H", 0, 1, 0),
    "s": ("S", 0, 1, 0), "sdg": ("SDG", 0, 1, 0), "t": ("T", 0, 1, 0), "tdg": ("TDG", 0, 1, 0),
    "rx": ("RX", 0, 1, 1), "ry": ("RY", 0, 1, 1), "rz": ("RZ", 0, 1, 1),
    "cx": ("X", 1, 1, 0), "cy": ("Y", 1, 1, 0), "cz": ("Z", 1, 1, 0), "ch": ("H", 1, 1, 0),
    "crx": ("RX", 1, 1, 1), "cry": ("RY", 1, 1, 1), "crz": ("RZ", 1, 1, 1),
    "cu1": ("U1", 1, 1, 1), "cu3": ("U3", 1, 1, 3),
    "ccx": ("X", 2, 1, 0), "c3x": ("X", 3, 1, 0), "c4x": ("X", 4, 1, 0),
    "swap": ("SWAP", 0, 2, 0), "cswap": ("SWAP", 1, 2, 0),
    "rxx": ("RXX", 0, 2, 1), "ryy": ("RYY", 0, 2, 1), "rzz": ("RZZ", 0, 2, 1),
}


class QasmError(ValueError):
    """A QASM program this front end cannot lower (with the line number)."""


# ---- the reference's parameter conversion (for parity checks) ---------------


def convert_param_reference(val: str) -> float:
    """The reference's ``convert_param``/``handle_pi`` (qasm_assembler_standalone.py:3581-3617),
    quirks included: 'e' anywhere -> 1.0, bare 'pi' -> 0.0, 'a/pi' -> a/pi,
    a '*' term overrides a '/' term, a leading '-pi' negates."""
    if "pi" in val:
        ret = 0.0
        if "/" in val:
            a, b = val.split("/")
            if "pi" in a:
                ret = math.pi / float(b)
            elif "pi" in b:
                ret = float(a) / math.pi
            else:
                raise QasmError(f"no pi in {val!r}")
        if "*" in val:
            a, b = val.split("*")
            if "pi" in a:
                ret = math.pi * float(b)
            elif "pi" in b:
                ret = float(a) * math.pi
            else:
                raise QasmError(f"no pi in {val!r}")
        if "-pi" in val:
            ret = -ret
        return ret
    if "e" in val:
        return 1.0
    return float(val)


# ---- tokens and expressions ---------------------------------------------------

_TOKEN = re.compile(r"""
    (?P<ws>\s+) | (?P<comment>//[^\n]*) |
    (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?) |
    (?P<id>[A-Za-z_][A-Za-z0-9_]*) |
    (?P<str>"[^"]*") |
    (?P<op>->|==|[()\[\]{},;+\-*/^])
""", re.X)

_FUNCS = {"sin": math.sin, "cos": math.cos, "tan": math.tan, "exp": math.exp,
          "ln": math.log, "sqrt": math.sqrt}


@dataclass
class _Tok:
    kind: str
    text: str
    line: int
    pos: int


def _tokenize(src: str) -> List[_Tok]:
    out, pos, line = [], 0, 1
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise QasmError(f"line {line}: unexpected character {src[pos]!r}")
        kind = m.lastgroup
        text = m.group()
        if kind not in ("ws", "comment"):
            out.append(_Tok(kind, text, line, pos))
        line += text.count("\n")
        pos = m.end()
    return out


class _Expr:
    """Recursive-descent evaluation of a parameter expression."""

    def __init__(self, toks: List[_Tok], env: Dict[str, float]):
        self.t, self.i, self.env = toks, 0, env

    def peek(self):
        return self.t[self.i].text if self.i < len(self.t) else None

    def take(self, text=None):
        if self.i >= len(self.t):
            raise QasmError("unexpected end of expression")
        tok = self.t[self.i]
        if text is not None and tok.text != text:
            raise QasmError(f"line {tok.line}: expected {text!r}, got {tok.text!r}")
        self.i += 1
        return tok

    def parse(self) -> float:
        v = self.sum()
        if self.i != len(self.t):
            tok = self.t[self.i]
            raise QasmError(f"line {tok.line}: unexpected {tok.text!r} in expression")
        return v

    def sum(self):
        v = self.product()
        while self.peek() in ("+", "-"):
            v = v + self.product() if self.take().text == "+" else v - self.product()
        return v

    def product(self):
        v = self.unary()
        while self.peek() in ("*", "/"):
            if self.take().text == "*":
                v = v * self.unary()
            else:
                d = self.unary()
                if d == 0:
                    raise QasmError("division by zero in a parameter")
                v = v / d
        return v

    def unary(self):
        if self.peek() == "-":
            self.take()
            return -self.unary()
        if self.peek() == "+":
            self.take()
            return self.unary()
        return self.power()

    def power(self):
        v = self.atom()
        if self.peek() == "^":
            self.take()
            return v ** self.unary()
        return v

    def atom(self):
        tok = self.take()
        if tok.kind == "num":
            return float(tok.text)
        if tok.text == "(":
            v = self.sum()
            self.take(")")
            return v
        if tok.kind == "id":
            if tok.text == "pi":
                return math.pi
            if tok.text in _FUNCS and self.peek() == "(":
                self.take("(")
                v = self.sum()
                self.take(")")
                return _FUNCS[tok.text](v)
            if tok.text in self.env:
                return self.env[tok.text]
        raise QasmError(f"line {tok.line}: unknown symbol {tok.text!r} in expression")


# ---- program -------------------------------------------------------------------


@dataclass
class Op:
    """One entry of the ordered operation list (the reference's
    ``ordered_gate_list``): a basic QASM gate or a measurement."""

    name: str                      # lower-case QASM name ("measure" included)
    params: Tuple[float, ...]
    qubits: Tuple[int, ...]        # universal qubit indices
    line: int                      # 1-based source line
    clbits: Tuple[int, ...] = ()   # measure: classical bit indices


@dataclass
class Program:
    qregs: Dict[str, int] = field(default_factory=dict)
    cregs: Dict[str, int] = field(default_factory=dict)
    ops: List[Op] = field(default_factory=list)

    @property
    def num_qubits(self) -> int:
        return sum(self.qregs.values())

    def qubit_name(self, q: int) -> str:
        for name, size in self.qregs.items():
            if q < size:
                return f"{name}[{q}]"
            q -= size
        raise IndexError(q)

    def lower(self, op: Op) -> Optional[Gate]:
        """The bound gate of one operation (None for a measurement)."""
        if op.name == "measure":
            return None
        base, nc, nt, npar = _LOWER[op.name]
        return Gate(base, targets=op.qubits[nc:nc + nt], controls=op.qubits[:nc],
                    params=op.params[:npar])

    def gates(self) -> List[Optional[Gate]]:
        """Bound gates aligned with ``ops`` (None where ``ops`` measures)."""
        return [self.lower(op) for op in self.ops]

    def circuit(self) -> List[Gate]:
        """The bound gates in order, measurements left out."""
        return [g for g in self.gates() if g is not None]

    def measured_qubits(self) -> List[int]:
        return [op.qubits[0] for op in self.ops if op.name == "measure"]


@dataclass
class _GateDef:
    params: List[str]
    args: List[str]
    body: List[_Tok]


class _Parser:
    def __init__(self, src: str, params: str):
        if params not in ("exact", "reference"):
            raise ValueError("params must be 'exact' or 'reference'")
        self.src = src
        self.mode = params
        self.t = _tokenize(src)
        self.i = 0
        self.prog = Program()
        self.defs: Dict[str, _GateDef] = {}

    # -- token helpers
    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else None

    def take(self, text=None, kind=None) -> _Tok:
        tok = self.peek()
        if tok is None:
            raise QasmError("unexpected end of program")
        if (text is not None and tok.text != text) or (kind is not None and tok.kind != kind):
            raise QasmError(f"line {tok.line}: expected {text or kind!r}, got {tok.text!r}")
        self.i += 1
        return tok

    def until(self, text) -> List[_Tok]:
        out = []
        while self.peek() is not None and self.peek().text != text:
            out.append(self.take())
        self.take(text)
        return out

    # -- statements
    def parse(self) -> Program:
        while self.peek() is not None:
            tok = self.peek()
            if tok.text == "OPENQASM":
                self.until(";")
            elif tok.text == "include":
                self.until(";")
            elif tok.text in ("qreg", "creg"):
                self.take()
                name = self.take(kind="id").text
                self.take("[")
                size = int(self.take(kind="num").text)
                self.take("]")
                self.take(";")
                regs = self.prog.qregs if tok.text == "qreg" else self.prog.cregs
                if name in self.prog.qregs or name in self.prog.cregs:
                    raise QasmError(f"line {tok.line}: register {name} declared twice")
                regs[name] = size
            elif tok.text == "gate":
                self.gate_def()
            elif tok.text == "opaque":
                raise QasmError(f"line {tok.line}: opaque gates have no definition to run")
            elif tok.text == "if":
                raise QasmError(f"line {tok.line}: classically controlled gates are not supported")
            elif tok.text == "barrier":
                self.until(";")
            elif tok.text == "measure":
                self.measure()
            else:
                self.call(self.until(";"), {}, None, tok.line)
        return self.prog

    def gate_def(self):
        self.take("gate")
        name = self.take(kind="id").text
        params: List[str] = []
        if self.peek().text == "(":
            self.take("(")
            while self.peek().text != ")":
                params.append(self.take(kind="id").text)
                if self.peek().text == ",":
                    self.take(",")
            self.take(")")
        args = []
        while self.peek().text != "{":
            tok = self.take()
            if tok.kind == "id":
                args.append(tok.text)
        self.take("{")
        body, depth = [], 1
        while True:
            tok = self.take()
            depth += tok.text == "{"
            depth -= tok.text == "}"
            if depth == 0:
                break
            body.append(tok)
        self.defs[name] = _GateDef(params, args, body)

    def reg_bits(self, toks: List[_Tok], regs: Dict[str, int], offset_of) -> List[List[int]]:
        """Comma-separated register arguments -> per argument its bit list."""
        out, j = [], 0
        while j < len(toks):
            name = toks[j].text
            if name not in regs:
                raise QasmError(f"line {toks[j].line}: unknown register {name}")
            if j + 1 < len(toks) and toks[j + 1].text == "[":
                idx = int(toks[j + 2].text)
                if idx >= regs[name]:
                    raise QasmError(f"line {toks[j].line}: {name}[{idx}] out of range")
                out.append([offset_of(name) + idx])
                j += 4
            else:
                out.append([offset_of(name) + k for k in range(regs[name])])
                j += 1
            if j < len(toks):
                if toks[j].text != ",":
                    raise QasmError(f"line {toks[j].line}: expected ','")
                j += 1
        return out

    def offset(self, regs: Dict[str, int]):
        def f(name):
            o = 0
            for r, size in regs.items():
                if r == name:
                    return o
                o += size
            raise KeyError(name)
        return f

    def measure(self):
        line = self.take("measure").line
        toks = self.until(";")
        arrow = next((k for k, t in enumerate(toks) if t.text == "->"), None)
        if arrow is None:
            raise QasmError(f"line {line}: measure needs '->'")
        qs = self.reg_bits(toks[:arrow], self.prog.qregs, self.offset(self.prog.qregs))
        cs = self.reg_bits(toks[arrow + 1:], self.prog.cregs, self.offset(self.prog.cregs))
        if len(qs) != 1 or len(cs) != 1 or len(qs[0]) != len(cs[0]):
            raise QasmError(f"line {line}: measure arguments do not match")
        for q, c in zip(qs[0], cs[0]):
            self.prog.ops.append(Op("measure", (), (q,), line, (c,)))

    # -- gate calls
    def params_of(self, toks: List[_Tok], env: Dict[str, float]) -> Tuple[List[float], int]:
        """Parameters of a call starting at toks[1] == '(' -> (values, index after ')')."""
        depth, j, groups, cur = 0, 1, [], []
        while True:
            if j >= len(toks):
                raise QasmError(f"line {toks[0].line}: unbalanced parentheses")
            tok = toks[j]
            if tok.text == "(":
                depth += 1
                if depth > 1:
                    cur.append(tok)
            elif tok.text == ")":
                depth -= 1
                if depth == 0:
                    break
                cur.append(tok)
            elif tok.text == "," and depth == 1:
                groups.append(cur)
                cur = []
            else:
                cur.append(tok)
            j += 1
        if cur or groups:
            groups.append(cur)
        if self.mode == "reference":
            # the reference takes the text between the first '(' and the first
            # ')' of the statement and converts each comma-separated piece
            start = toks[1].pos + 1
            raw = self.src[start:self.src.index(")", start)]
            try:
                return [convert_param_reference(v) for v in raw.split(",")], j + 1
            except ValueError as ex:
                raise QasmError(f"line {toks[0].line}: {ex}") from None
        return [_Expr(g, env).parse() for g in groups], j + 1

    def call(self, toks: List[_Tok], env: Dict[str, float], qmap: Optional[Dict[str, int]],
             line: int, depth: int = 0):
        if not toks:
            return
        if depth > 64:
            raise QasmError(f"line {line}: gate definitions nest too deeply")
        head = toks[0]
        name = head.text
        if name == "barrier":
            return
        if head.kind != "id":
            raise QasmError(f"line {head.line}: expected a gate name, got {name!r}")
        params: List[float] = []
        j = 1
        if len(toks) > 1 and toks[1].text == "(":
            params, j = self.params_of(toks, env)
        argt = toks[j:]
        if qmap is None:
            args = self.reg_bits(argt, self.prog.qregs, self.offset(self.prog.qregs))
        else:
            args = []
            for k, tok in enumerate(argt):
                if k % 2 == 1:
                    if tok.text != ",":
                        raise QasmError(f"line {tok.line}: expected ','")
                    continue
                if tok.text not in qmap:
                    raise QasmError(f"line {tok.line}: {tok.text} is not an argument of the gate")
                args.append([qmap[tok.text]])
        if not args:
            raise QasmError(f"line {head.line}: {name} has no qubit arguments")
        width = max(len(a) for a in args)
        if any(len(a) not in (1, width) for a in args):
            raise QasmError(f"line {head.line}: register sizes of {name} do not match")
        for k in range(width):
            qubits = tuple(a[k] if len(a) > 1 else a[0] for a in args)
            if len(set(qubits)) != len(qubits):
                raise QasmError(f"line {head.line}: {name} uses a qubit twice")
            if name in _LOWER:
                _, nc, nt, npar = _LOWER[name]
                if len(qubits) != nc + nt:
                    raise QasmError(f"line {head.line}: {name} takes {nc + nt} qubits")
                if len(params) != npar:
                    raise QasmError(f"line {head.line}: {name} takes {npar} parameters")
                self.prog.ops.append(Op(name, tuple(params), qubits, head.line))
            elif name in self.defs:
                d = self.defs[name]
                if len(d.args) != len(qubits) or len(d.params) != len(params):
                    raise QasmError(f"line {head.line}: {name} takes {len(d.params)} parameters "
                                    f"and {len(d.args)} qubits")
                sub_env = dict(zip(d.params, params))
                sub_q = dict(zip(d.args, qubits))
                stmt: List[_Tok] = []
                for tok in d.body:
                    if tok.text == ";":
                        self.call(stmt, sub_env, sub_q, tok.line, depth + 1)
                        stmt = []
                    else:
                        stmt.append(tok)
                if stmt:
                    raise QasmError(f"line {stmt[0].line}: missing ';' in gate {name}")
            elif name == "measure":
                raise QasmError(f"line {head.line}: measure inside a gate definition")
            else:
                raise QasmError(f"line {head.line}: unknown gate {name}")


def parse(text: str, params: str = "exact") -> Program:
    """Parse OpenQASM 2 text.  params: "exact" (expressions evaluated) or
    "reference" (the reference's convert_param, quirks included)."""
    return _Parser(text, params).parse()


def load(path: str, params: str = "exact") -> Program:
    with open(path) as f:
        return parse(f.read(), params)


# ---- DAG files -------------------------------------------------------------------


def dag_graphs(program: Program):
    """The gate DAGs the reference's ``produce_dot_file`` writes
    (qasm_assembler_standalone.py:3688-3764), one per measurement-separated
    segment: nodes {name: attrs} and edges [(u, v, qubit label)].  Gate nodes
    are ``<gate>_<counter>`` (label = QASM name, line = 0-based source line,
    order = 1-based position in the operation list); every wire ends in an
    ``exit`` node and starts at an input node named after the qubit
    (``add_input_node_pass``, :3625-3686)."""
    graphs = []
    nodes: Dict[str, dict] = {}
    edges: List[Tuple[str, str, str]] = []
    open_end: Dict[str, Tuple[str, str]] = {}  # qubit label -> (last gate, its exit node)
    counter = 0
    exit_order = len(program.ops) + 8192

    def close():
        # input nodes for wires that start inside this segment
        heads: List[Tuple[str, str]] = []
        has_in = {(v, lab) for (_, v, lab) in edges}
        for u, v, lab in edges:
            if not nodes[u]["label"] == "exit" and (u, lab) not in has_in and \
                    nodes[u].get("order", 0) != 0 and (lab, u) not in heads:
                heads.append((lab, u))
        for lab, u in heads:
            nodes.setdefault(lab, {"label": lab, "order": 0})
            edges.append((lab, u, lab))
        graphs.append((dict(nodes), list(edges)))

    for order, op in enumerate(program.ops):
        if op.name == "measure":
            if not nodes:
                continue
            close()
            nodes, edges, open_end = {}, [], {}
            continue
        gname = f"{op.name}_{counter}"
        counter += 1
        nodes[gname] = {"label": op.name, "line": op.line - 1, "order": order + 1}
        labels = [program.qubit_name(q).replace("[", "").replace("]", "") for q in op.qubits]
        for lab in labels:
            void = f"{lab}_exit_{counter}"
            counter += 1
            if lab in open_end:  # reconnect the wire: previous gate -> this gate
                prev, prev_void = open_end[lab]
                edges.remove((prev, prev_void, lab))
                del nodes[prev_void]
                edges.append((prev, gname, lab))
            nodes[void] = {"label": "exit", "order": exit_order}
            edges.append((gname, void, lab))
            open_end[lab] = (gname, void)
    if nodes:
        close()
    return graphs


def _dot_attr(v):
    return str(v) if isinstance(v, int) else '"' + str(v).replace('"', '\\"') + '"'


def write_dot(program: Program, prefix: str) -> List[str]:
    """Write ``<prefix>_PART_<k>.dot`` per DAG segment (DOT written directly;
    the reference goes through networkx + pydot)."""
    paths = []
    for k, (nodes, edges) in enumerate(dag_graphs(program)):
        path = f"{prefix}_PART_{k}.dot"
        with open(path, "w") as f:
            f.write("digraph {\n")
            for name, attrs in nodes.items():
                a = ", ".join(f"{key}={_dot_attr(val)}" for key, val in attrs.items())
                f.write(f'"{name}" [{a}];\n')
            keys: Dict[Tuple[str, str], int] = {}
            for u, v, lab in edges:
                kk = keys.get((u, v), 0)
                keys[(u, v)] = kk + 1
                f.write(f'"{u}" -> "{v}" [key={kk}, label={_dot_attr(lab)}];\n')
            f.write("}\n")
        paths.append(path)
    return paths


def read_dot(path: str):
    """Nodes and edges of a DOT file written by ``write_dot``."""
    nodes, edges = {}, []
    node_re = re.compile(r'^"([^"]+)" \[(.*)\];$')
    edge_re = re.compile(r'^"([^"]+)" -> "([^"]+)" \[key=\d+, label="([^"]*)"\];$')
    with open(path) as f:
        for line in f:
            line = line.strip()
            m = edge_re.match(line)
            if m:
                edges.append((m.group(1), m.group(2), m.group(3)))
                continue
            m = node_re.match(line)
            if m:
                attrs = {}
                for kv in re.findall(r'(\w+)=("[^"]*"|\d+)', m.group(2)):
                    attrs[kv[0]] = kv[1].strip('"') if kv[1].startswith('"') else int(kv[1])
                nodes[m.group(1)] = attrs
    return nodes, edges


# ---- running -----------------------------------------------------------------


def parts_from_file(program: Program, path: str) -> List[List[int]]:
    """A part file (``order_id node part_id`` lines, qasm_assembler_standalone.py:3549-3567)
    as lists of gate indices into ``program.circuit()`` (measurements drop out)."""
    from . import partition

    op_parts = partition.read_part_file(path, len(program.ops))
    gate_index, k = {}, 0
    for i, op in enumerate(program.ops):
        if op.name != "measure":
            gate_index[i] = k
            k += 1
    return [[gate_index[i] for i in p if i in gate_index] for p in op_parts]


def simulate(program: Program, parts: Optional[Sequence[Sequence[int]]] = None, dtype: int = 0,
             max_qubits: int = 10, state=None):
    """Run the program's gates on the GPU from |0...0> (or on ``state``) in
    ``parts`` (gate index lists into ``program.circuit()``; default: the
    frontier partitioner with ``max_qubits``, the fewest parts).  Returns the
    ``abi.State``."""
    from . import abi, partition
    from .gates import part_offsets

    gates = program.circuit()
    if parts is None:
        parts = partition.partition_frontier(gates, max_qubits) if gates else []
    if state is None:
        state = abi.State(program.num_qubits, dtype)
        state.set_basis(0)
    if parts:
        rec, offs = part_offsets([[gates[i] for i in p] for p in parts])
        state.run_parts(rec, offs)
    return state
