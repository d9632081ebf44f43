"""Seeded synthetic circuits for the benchmark and parity workloads.

The reference measures on QASMBench circuits; these generators stand in for
them with the shapes the workloads name:

* ``random_layered``  -- layers of one random gate per qubit from
  {H, X, S, T, RZ(t), U3(t,p,l)} (angles U[0, 2pi)) followed by CX or CZ on a
  random perfect matching (the plain-form parity workload, 20 qubits).
* ``random_u3_cz``    -- layers of U3 with uniform angles on every qubit, then
  CZ on a random matching (one qubit idles per layer when n is odd) (the
  33-qubit precision / plain workload).
* ``qft``             -- full QFT: H plus controlled phase 2pi/2^m on all pairs,
  then the bit-reversal swaps, on a seeded random basis state.  The
  controlled phase is C1(1, 0, 0, e^{i phi}) with one control, i.e. the
  textbook phase gate (the reference's CU1 lowering would be a controlled RZ,
  qasm_assembler_standalone.py:1918-1925).
* ``qaoa_maxcut``     -- p rounds of RZZ(gamma) on every edge of a random
  3-regular graph and RX(2 beta) on every qubit, from |+>^n.

Gate semantics follow the reference's lowering of QASM gates to BoundGates
(qasm_assembler_standalone.py:1831-2010): CX -> X with one control, CZ -> Z
with one control.
"""
from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .gates import Gate

TWO_PI = 2.0 * math.pi


def _matching(rng: np.random.Generator, n: int) -> List[Tuple[int, int]]:
    perm = rng.permutation(n)
    return [(int(perm[2 * i]), int(perm[2 * i + 1])) for i in range(n // 2)]


def random_layered(n: int, layers: int, seed: int) -> List[Gate]:
    """Random layered circuit over {H, X, S, T, RZ, U3} + CX/CZ matchings."""
    rng = np.random.default_rng(seed)
    out: List[Gate] = []
    names = ["H", "X", "S", "T", "RZ", "U3"]
    for _ in range(layers):
        for q in range(n):
            name = names[int(rng.integers(len(names)))]
            if name == "RZ":
                out.append(Gate("RZ", (q,), params=(rng.uniform(0, TWO_PI),)))
            elif name == "U3":
                out.append(Gate("U3", (q,), params=tuple(rng.uniform(0, TWO_PI, 3))))
            else:
                out.append(Gate(name, (q,)))
        for a, b in _matching(rng, n):
            # per-pair choice of CNOT or CZ, control a, target b
            if rng.integers(2) == 0:
                out.append(Gate("X", (b,), (a,)))
            else:
                out.append(Gate("Z", (b,), (a,)))
    return out


def random_u3_cz(n: int, layers: int, seed: int) -> List[Gate]:
    """Layers of U3 (uniform angles) on every qubit + CZ on a random matching."""
    rng = np.random.default_rng(seed)
    out: List[Gate] = []
    for _ in range(layers):
        for q in range(n):
            out.append(Gate("U3", (q,), params=tuple(rng.uniform(0, TWO_PI, 3))))
        for a, b in _matching(rng, n):
            out.append(Gate("Z", (b,), (a,)))
    return out


def qft(n: int, seed: int) -> Tuple[List[Gate], int]:
    """Full QFT; returns (gates, x) where |x> is the seeded initial basis state."""
    rng = np.random.default_rng(seed)
    x = int(rng.integers(0, 1 << min(n, 62))) if n <= 62 else 0
    out: List[Gate] = []
    for i in range(n - 1, -1, -1):
        out.append(Gate("H", (i,)))
        for j in range(i - 1, -1, -1):
            m = i - j + 1
            phi = TWO_PI / (1 << m)
            out.append(Gate("C1", (i,), (j,), params=(1.0, 0.0, 0.0, complex(math.cos(phi), math.sin(phi)))))
    for i in range(n // 2):
        out.append(Gate("SWAP", (i, n - 1 - i)))
    return out, x


def random_regular3(n: int, rng: np.random.Generator, tries: int = 1000) -> List[Tuple[int, int]]:
    """Random simple 3-regular graph on n (even) vertices by the pairing model."""
    if n % 2 or n < 4:
        raise ValueError("a 3-regular graph needs an even n >= 4")
    for _ in range(tries):
        stubs = rng.permutation(np.repeat(np.arange(n), 3))
        edges = set()
        ok = True
        for k in range(0, len(stubs), 2):
            a, b = int(stubs[k]), int(stubs[k + 1])
            if a == b or (min(a, b), max(a, b)) in edges:
                ok = False
                break
            edges.add((min(a, b), max(a, b)))
        if ok:
            return sorted(edges)
    raise RuntimeError("could not draw a simple 3-regular graph")


def random_maxcut_graph(n: int, rng: np.random.Generator, tries: int = 1000) -> List[Tuple[int, int]]:
    """Random simple 3-regular graph for even n; for odd n (no 3-regular graph
    exists) the same pairing model with one vertex of degree 2, so every qubit
    stays coupled and |E| = (3n - 1) / 2."""
    if n % 2 == 0:
        return random_regular3(n, rng, tries)
    if n < 5:
        raise ValueError("need n >= 5 for an odd near-3-regular graph")
    for _ in range(tries):
        deg = np.full(n, 3)
        deg[int(rng.integers(n))] = 2
        stubs = rng.permutation(np.repeat(np.arange(n), deg))
        edges = set()
        ok = True
        for k in range(0, len(stubs), 2):
            a, b = int(stubs[k]), int(stubs[k + 1])
            if a == b or (min(a, b), max(a, b)) in edges:
                ok = False
                break
            edges.add((min(a, b), max(a, b)))
        if ok:
            return sorted(edges)
    raise RuntimeError("could not draw a simple near-3-regular graph")


def qaoa_maxcut(n: int, p: int, seed: int):
    """QAOA MaxCut on a random 3-regular graph (near-3-regular for odd n).

    Returns (gates, edges, gammas, betas); gates start with H on every qubit
    (|+>^n), then per round RZZ(gamma) on each edge and RX(2 beta) on each qubit.
    """
    rng = np.random.default_rng(seed)
    edges = random_maxcut_graph(n, rng)
    gammas = rng.uniform(0, math.pi, p)
    betas = rng.uniform(0, math.pi / 2, p)
    out: List[Gate] = [Gate("H", (q,)) for q in range(n)]
    for r in range(p):
        for a, b in edges:
            out.append(Gate("RZZ", (a, b), params=(gammas[r],)))
        for q in range(n):
            out.append(Gate("RX", (q,), params=(2 * betas[r],)))
    return out, edges, gammas, betas
