"""Circuit partitioners and the reference's part-file format.

The reference ships no partitioner: parts come from the external dagP tool
(README.md:3-5) as three-column files ``order_id node part_id`` that
``parse_parts_file`` (qasm_assembler_standalone.py:3549-3567) reads; order ids
are 1-based gate positions, id 0 and ids past the gate list are skipped
(qasm_assembler_standalone.py:1786-1791).  Three strategies ship as outputs
(``*_part_smart`` = acyclic, ``*_part_dfs``, ``*_part_nat``); this module
implements the same three strategies under a qubit limit:

* ``partition_acyclic`` -- greedy acyclic parts: each part takes every
  remaining gate (in circuit order) whose qubits fit in the part and none of
  whose predecessors is still unplaced.  Parts run in order form a valid
  topological order of the gate DAG.
* ``partition_natural`` -- consecutive runs of the gate list.
* ``partition_dfs``     -- consecutive runs of a depth-first order of the
  gate DAG.

One more strategy, not among the reference's outputs, aims at the fewest
parts (every part is one state pass, so passes dominate the run time):

* ``partition_frontier`` -- parts grown from the DAG's ready frontier with a
  lookahead (fewest parts on layered circuits: 123 against 154 DFS-order
  parts of <= 6 qubits, 71 against 93 of <= 9 qubits, for 33 qubits x 40
  layers of U3 + CZ).
"""
from __future__ import annotations

from collections import OrderedDict
from typing import Dict, List, Sequence

from .gates import DIAGONAL, Gate


def _check(max_qubits: int, gates: Sequence[Gate]):
    if max_qubits < 1:
        raise ValueError("max_qubits must be >= 1")
    for g in gates:
        if len(set(g.qubits)) > max_qubits:
            raise ValueError(f"gate {g} touches more than {max_qubits} qubits")


def partition_acyclic(gates: Sequence[Gate], max_qubits: int) -> List[List[int]]:
    """Greedy acyclic partition; returns parts as lists of gate indices."""
    _check(max_qubits, gates)
    remaining = list(range(len(gates)))
    parts: List[List[int]] = []
    while remaining:
        part: List[int] = []
        qubits: set = set()
        blocked: set = set()
        rest: List[int] = []
        for i in remaining:
            gq = set(gates[i].qubits)
            if gq & blocked or len(qubits | gq) > max_qubits:
                # this gate waits; everything after it on its qubits waits too
                blocked |= gq
                rest.append(i)
                continue
            part.append(i)
            qubits |= gq
        parts.append(part)
        remaining = rest
    return parts


def partition_natural(gates: Sequence[Gate], max_qubits: int) -> List[List[int]]:
    """Consecutive runs of the gate list with at most max_qubits qubits each."""
    _check(max_qubits, gates)
    parts: List[List[int]] = []
    cur: List[int] = []
    qubits: set = set()
    for i, g in enumerate(gates):
        gq = set(g.qubits)
        if cur and len(qubits | gq) > max_qubits:
            parts.append(cur)
            cur, qubits = [], set()
        cur.append(i)
        qubits |= gq
    if cur:
        parts.append(cur)
    return parts


def dag_successors(gates: Sequence[Gate]) -> List[List[int]]:
    """Edges of the gate DAG: gate i -> the next gate on each of its qubits."""
    last: Dict[int, int] = {}
    succ: List[List[int]] = [[] for _ in gates]
    for i, g in enumerate(gates):
        for q in g.qubits:
            if q in last and i not in succ[last[q]]:
                succ[last[q]].append(i)
            last[q] = i
    return succ


def dfs_order(gates: Sequence[Gate]) -> List[int]:
    """A depth-first topological order of the gate DAG (reverse postorder)."""
    succ = dag_successors(gates)
    indeg = [0] * len(gates)
    for s in succ:
        for j in s:
            indeg[j] += 1
    seen = [False] * len(gates)
    post: List[int] = []
    for root in range(len(gates)):
        if indeg[root] or seen[root]:
            continue
        stack = [(root, 0)]
        seen[root] = True
        while stack:
            v, k = stack[-1]
            if k < len(succ[v]):
                stack[-1] = (v, k + 1)
                w = succ[v][k]
                if not seen[w]:
                    seen[w] = True
                    stack.append((w, 0))
            else:
                post.append(v)
                stack.pop()
    return post[::-1]


def partition_dfs(gates: Sequence[Gate], max_qubits: int) -> List[List[int]]:
    """Consecutive runs (under the qubit limit) of a DFS topological order."""
    order = dfs_order(gates)
    reordered = [gates[i] for i in order]
    return [[order[j] for j in part] for part in partition_natural(reordered, max_qubits)]


def parts_to_gates(gates: Sequence[Gate], parts: Sequence[Sequence[int]]) -> List[List[Gate]]:
    return [[gates[i] for i in p] for p in parts]


def is_valid_partition(gates: Sequence[Gate], parts: Sequence[Sequence[int]]) -> bool:
    """Every gate once, and parts in order respect every DAG edge."""
    pos = {}
    for pi, p in enumerate(parts):
        for k, i in enumerate(p):
            if i in pos:
                return False
            pos[i] = (pi, k)
    if sorted(pos) != list(range(len(gates))):
        return False
    for i, s in enumerate(dag_successors(gates)):
        for j in s:
            if pos[i] >= pos[j]:
                return False
    return True


# ---- the reference's part-file format ------------------------------------

def write_part_file(path: str, gates: Sequence[Gate], parts: Sequence[Sequence[int]]):
    """Write ``order_id node part_id`` lines (order_id = 1-based gate index)."""
    with open(path, "w") as f:
        for pi, p in enumerate(parts):
            for i in p:
                f.write(f"{i + 1} {gates[i].name.lower()}{i + 1} {pi}\n")


def read_part_file(path: str, num_gates: int) -> List[List[int]]:
    """Read a part file the way parse_parts_file does (qasm_assembler_standalone.py:3549-3567).

    Parts are ordered by part id; order id 0 and ids beyond the gate list are
    skipped (:1786-1791); ids are 1-based.
    """
    parts: "OrderedDict[int, List[int]]" = OrderedDict()
    with open(path) as f:
        for line in f:
            line = line.rstrip("\n")
            if not line:
                continue
            items = line.split(" ")
            if len(items) != 3:
                raise ValueError(f"bad part-file line: {line!r}")
            order_id, part_id = int(items[0]), int(items[2])
            parts.setdefault(part_id, []).append(order_id)
    out: List[List[int]] = []
    for pid in sorted(parts):
        ids = [o - 1 for o in parts[pid] if o != 0 and 1 <= o <= num_gates]
        out.append(ids)
    return out


def _absorbable(qset, ready, indeg, succ, qubits) -> int:
    """Gates that could run inside qubit set qset from the current frontier:
    the ready gates within qset and, transitively, their successors within it."""
    left: Dict[int, int] = {}
    stack = [i for i in ready if qubits[i] <= qset]
    seen = set(stack)
    count = 0
    while stack:
        i = stack.pop()
        count += 1
        for j in succ[i]:
            d = left.get(j, indeg[j]) - 1
            left[j] = d
            if d == 0 and j not in seen and qubits[j] <= qset:
                seen.add(j)
                stack.append(j)
    return count


def partition_frontier(gates: Sequence[Gate], max_qubits: int, age_weight: float = 1.0,
                       free_diagonal: bool = False) -> List[List[int]]:
    """Acyclic parts grown from the ready frontier of the gate DAG.

    A part starts with an empty qubit set S and repeats: absorb every ready
    gate whose qubits lie in S (which readies its successors); then, among the
    ready gates that would keep |S| <= max_qubits, add the qubits of the one
    that lets the most gates run inside the enlarged set per qubit added
    (``_absorbable``), preferring earlier gates (``age_weight`` * index / N)
    and then fewer new qubits.  The part closes when no ready gate fits.
    Gates are taken only when ready, so the parts in order are a topological
    order of the DAG.

    With ``free_diagonal`` the limit counts only the targets of non-diagonal
    gates: the part kernel holds those in its tile, while diagonal gates and
    controls act on index bits wherever they are, so CZ partners and controls
    cost nothing (for the plain form's K1; a fused unitary needs every qubit
    its gates touch)."""
    _check(max_qubits, gates)
    n = len(gates)
    succ = dag_successors(gates)
    if free_diagonal:
        qubits = [frozenset() if g.name in DIAGONAL else frozenset(g.targets) for g in gates]
    else:
        qubits = [frozenset(g.qubits) for g in gates]
    indeg = [0] * n
    for s in succ:
        for j in s:
            indeg[j] += 1
    ready = {i for i in range(n) if indeg[i] == 0}
    parts: List[List[int]] = []
    done = 0
    while done < n:
        qset: frozenset = frozenset()
        part: List[int] = []
        while True:
            grew = True
            while grew:
                grew = False
                for i in sorted(ready):
                    if qubits[i] <= qset:
                        ready.remove(i)
                        part.append(i)
                        done += 1
                        grew = True
                        for j in succ[i]:
                            indeg[j] -= 1
                            if indeg[j] == 0:
                                ready.add(j)
            best = None
            for i in ready:
                grown = qset | qubits[i]
                if len(grown) > max_qubits:
                    continue
                added = len(grown) - len(qset)
                score = _absorbable(grown, ready, indeg, succ, qubits)
                key = (score / max(1, added) - age_weight * i / n, -added, -i)
                if best is None or key > best[0]:
                    best = (key, grown)
            if best is None:
                break
            qset = best[1]
        parts.append(part)
    return parts
