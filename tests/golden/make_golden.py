"""Generate the golden vectors in tests/golden/ from the reference itself.

Each fixture is a seeded circuit (stored as hs_gate records, so the fixture
does not depend on the generators staying unchanged) and the final amplitudes
computed by the reference's own C++ path (oracle/_ref/libhisv_ref.so:
BoundGate::apply per gate, state_vector.hpp:1349, and
gather_and_execute_on_multi per part, execute.hpp:318-470).

Run from the repository root after ``make -C oracle``:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from hisvsim_b200 import circuits, partition  # noqa: E402
from hisvsim_b200.gates import Gate, part_offsets, to_records  # noqa: E402
from oracle.oracle import RefOracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def all_gate_circuit(n, ng, seed):
    """Every constructible gate type, random controls (0-2)."""
    rng = np.random.default_rng(seed)
    names1 = ["I", "X", "Y", "Z", "H", "S", "T", "TDG", "SDG"]
    out = []
    for _ in range(ng):
        kind = int(rng.integers(8))
        qs = rng.permutation(n)
        nc = int(rng.integers(0, min(3, n - 1))) if n > 2 else 0
        ctl = tuple(int(q) for q in qs[2:2 + nc])
        t0, t1 = int(qs[0]), int(qs[1 % n])
        if kind in (5, 6) and n < 2:
            kind = 0
        if kind == 0:
            out.append(Gate(names1[rng.integers(len(names1))], (t0,), ctl))
        elif kind == 1:
            out.append(Gate(["RX", "RY", "RZ", "RI", "R1", "U1"][rng.integers(6)], (t0,), ctl,
                            params=(rng.uniform(0, 2 * np.pi),)))
        elif kind == 2:
            out.append(Gate("U2", (t0,), ctl, params=tuple(rng.uniform(0, 2 * np.pi, 2))))
        elif kind == 3:
            out.append(Gate("U3", (t0,), ctl, params=tuple(rng.uniform(0, 2 * np.pi, 3))))
        elif kind == 4:
            out.append(Gate("C1", (t0,), ctl, params=tuple(np.exp(1j * rng.uniform(0, 6, 4)) / 2)))
        elif kind == 5:
            out.append(Gate(["RXX", "RYY", "RZZ"][rng.integers(3)], (t0, t1), ctl,
                            params=(rng.uniform(0, 2 * np.pi),)))
        elif kind == 6:
            out.append(Gate("SWAP", (t0, t1), ctl))
        elif kind == 7:
            out.append(Gate(["RXFRAC", "RYFRAC", "RZFRAC", "RIFRAC", "R1FRAC"][rng.integers(5)],
                            (t0,), ctl, frac=(int(rng.integers(1, 9)), int(rng.integers(1, 6)))))
    return out


def c2_circuit(n, seed):
    rng = np.random.default_rng(seed)
    out = [Gate("H", (q,)) for q in range(n)]
    for _ in range(6):
        a, b = (int(x) for x in rng.permutation(n)[:2])
        out.append(Gate("C2", (a, b), params=tuple(rng.normal(size=16) / 4)))
    return out


def main():
    ref = RefOracle()
    fixtures = {}
    for n in (1, 2, 3, 5, 8, 10):
        fixtures[f"allgates_n{n}"] = (n, all_gate_circuit(n, 120, 100 + n), None, 0)
    fixtures["c2_n6"] = (6, c2_circuit(6, 7), None, 0)
    fixtures["layered_n12"] = (12, circuits.random_layered(12, 8, 11), None, 0)
    g, x = circuits.qft(10, 5)
    fixtures["qft_n10"] = (10, g, None, x)
    g = circuits.random_layered(14, 6, 12)
    fixtures["parts_n14"] = (14, g, partition.partition_acyclic(g, 6), 0)
    g, _, _, _ = circuits.qaoa_maxcut(10, 2, 3)
    fixtures["qaoa_n10"] = (10, g, None, 0)
    for name, (n, gates, parts, x) in fixtures.items():
        init = np.zeros(1 << n, dtype=np.complex128)
        init[x] = 1.0
        if parts is None:
            rec = to_records(gates)
            offs = np.array([0, len(rec)], dtype=np.int32)
            amps = ref.run(n, rec, mode=0, threads=4, init_state=init)
        else:
            rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
            amps = ref.run(n, rec, offs, mode=1, opt_slots=1, threads=4, init_state=init)
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), n=n, records=rec, offsets=offs,
                            basis=x, amplitudes=amps)
        print(name, n, len(rec), "gates", np.linalg.norm(amps))


if __name__ == "__main__":
    main()
