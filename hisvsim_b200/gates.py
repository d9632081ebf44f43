"""Gate records of the C ABI (include/hisv.h ``hs_gate``) and their Python form.

A ``Gate`` is the Python-side equivalent of the reference's ``BoundGate``
(state_vector.hpp:1332-1379): a gate type from ``SvSim::GateType``
(basic_gates.hpp:12-44), its constructor parameters, and the control / target
qubits.  ``to_records`` packs a gate list into the 320-byte ``hs_gate``
structs the C ABI takes.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, Sequence, Tuple

import numpy as np

# SvSim::GateType numbering (basic_gates.hpp:12-44)
GATE_TYPES = {
    "INVALID": 0, "ALLOC": 1, "FREE": 2, "I": 3, "X": 4, "Y": 5, "Z": 6, "H": 7, "S": 8,
    "T": 9, "RX": 10, "RY": 11, "RZ": 12, "RI": 13, "R1": 14, "RXFRAC": 15, "RYFRAC": 16,
    "RZFRAC": 17, "RIFRAC": 18, "R1FRAC": 19, "SWAP": 20, "C1": 21, "C2": 22, "U1": 23,
    "U2": 24, "U3": 25, "RXX": 26, "RYY": 27, "RZZ": 28, "TDG": 29, "SDG": 30,
}
TYPE_NAMES = {v: k for k, v in GATE_TYPES.items()}

# Parameter arity per constructor family (AggregateGate_0/1/2/3/C1/C2/Frac,
# basic_gates.hpp:1527-1776).
NOPARAM = {"I", "X", "Y", "Z", "H", "S", "T", "SWAP", "TDG", "SDG"}
ONEPARAM = {"RX", "RY", "RZ", "RI", "R1", "U1", "RXX", "RYY", "RZZ"}
TWOPARAM = {"U2"}
THREEPARAM = {"U3"}
FRAC = {"RXFRAC", "RYFRAC", "RZFRAC", "RIFRAC", "R1FRAC"}
TWO_TARGET = {"SWAP", "C2", "RXX", "RYY", "RZZ"}
# Gates whose matrix is diagonal in the computational basis.
DIAGONAL = {"I", "Z", "S", "T", "TDG", "SDG", "RZ", "U1", "RI", "R1", "RZFRAC", "RIFRAC",
            "R1FRAC", "RZZ"}

HS_GATE_DTYPE = np.dtype([
    ("type", "<i4"), ("num_controls", "<i4"), ("num_targets", "<i4"),
    ("controls", "<i4", (5,)), ("targets", "<i4", (5,)),
    ("frac_num", "<u4"), ("frac_pow", "<u4"), ("reserved", "<i4"),
    ("params", "<f8", (32,)),
], align=True)
assert HS_GATE_DTYPE.itemsize == 320


@dataclass(frozen=True)
class Gate:
    """One bound gate: name, params, controls, targets (qubit indices)."""

    name: str
    targets: Tuple[int, ...]
    controls: Tuple[int, ...] = ()
    params: Tuple[complex, ...] = ()
    frac: Tuple[int, int] = (0, 0)

    def __post_init__(self):
        object.__setattr__(self, "name", self.name.upper())
        object.__setattr__(self, "targets", tuple(int(t) for t in self.targets))
        object.__setattr__(self, "controls", tuple(int(c) for c in self.controls))
        object.__setattr__(self, "params", tuple(complex(p) for p in self.params))
        if self.name not in GATE_TYPES:
            raise ValueError(f"unknown gate {self.name}")

    @property
    def type(self) -> int:
        return GATE_TYPES[self.name]

    @property
    def qubits(self) -> Tuple[int, ...]:
        return self.controls + self.targets


def to_records(gates: Sequence[Gate]) -> np.ndarray:
    """Pack gates into an array of ``hs_gate`` structs."""
    rec = np.zeros(len(gates), dtype=HS_GATE_DTYPE)
    for i, g in enumerate(gates):
        if len(g.controls) > 5 or not 1 <= len(g.targets) <= 5:
            raise ValueError(f"gate {g}: at most 5 controls and 1..5 targets")
        if len(g.params) > 16:
            raise ValueError(f"gate {g}: at most 16 complex parameters")
        r = rec[i]
        r["type"] = g.type
        r["num_controls"] = len(g.controls)
        r["num_targets"] = len(g.targets)
        r["controls"][: len(g.controls)] = g.controls
        r["targets"][: len(g.targets)] = g.targets
        r["frac_num"], r["frac_pow"] = g.frac
        for j, p in enumerate(g.params):
            r["params"][2 * j] = p.real
            r["params"][2 * j + 1] = p.imag
    return rec


def part_offsets(parts: Sequence[Sequence[Gate]]) -> Tuple[np.ndarray, np.ndarray]:
    """Flatten a list of parts into (records, int32 offsets[len(parts)+1])."""
    flat = [g for p in parts for g in p]
    offs = np.zeros(len(parts) + 1, dtype=np.int32)
    np.cumsum([len(p) for p in parts], out=offs[1:])
    return to_records(flat), offs


def gate_qubit_set(gates: Iterable[Gate]) -> set:
    s = set()
    for g in gates:
        s.update(g.qubits)
    return s
