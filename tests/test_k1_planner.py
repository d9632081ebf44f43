"""K1 planner and addressing on the CPU: the library's own planner (plan.cpp,
gatemath.cpp) compiled with the host emulator tests/emu/k1_emu.cpp, which
executes the planned programs the way the K1 kernel does (tile chunk
placement, swizzled shared-memory offsets, register groups, rounds, op codes,
Gray-code direct stores).  Compared with the oracle (port.c, pinned to the
reference) at <= 1e-12, for carried frames across parts and for
self-contained parts, 8 and 16 amplitudes per thread, and complex64 rounding.
No GPU needed; the GPU parity tests check the kernel itself.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_names, load_golden
from hisvsim_b200 import circuits, partition
from hisvsim_b200.gates import Gate, part_offsets, to_records

CSRC = os.path.join(ROOT, "hisvsim_b200", "csrc")
SRCS = [os.path.join(ROOT, "tests", "emu", "k1_emu.cpp"), os.path.join(CSRC, "plan.cpp"),
        os.path.join(CSRC, "gatemath.cpp")]


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("emu") / "libk1emu.so")
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I/usr/local/cuda/include",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC] + SRCS + ["-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail("emulator build failed:\n" + r.stderr[-3000:])
    lib = ctypes.CDLL(out)
    P = ctypes.c_void_p
    lib.emu_parts_run.argtypes = [ctypes.c_int, ctypes.c_int, P, P, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_int, P, P]
    lib.emu_last_error.restype = ctypes.c_char_p

    def run(n, rec, offs, dtype=0, rbits=4, hint=0, per_part=False, init=None):
        a = np.zeros(1 << n, complex)
        if init is None:
            a[0] = 1
        else:
            a[:] = init
        st = np.zeros(9, np.int32)
        rc = lib.emu_parts_run(n, dtype, rec.ctypes.data, offs.ctypes.data, len(offs) - 1, rbits,
                               hint, int(per_part), a.ctypes.data, st.ctypes.data)
        if rc:
            raise RuntimeError(lib.emu_last_error().decode())
        return a, dict(zip(["passes", "groups", "ops", "rotations", "tile_bits", "rounds",
                            "wavefronts", "wavefronts_ideal", "two_shear"], st.tolist()))
    return run


def _circuit(kind, n, seed):
    if kind == "layered":
        return circuits.random_layered(n, 8, seed)
    if kind == "u3cz":
        return circuits.random_u3_cz(n, 8, seed)
    g, _ = circuits.qft(n, seed)
    return g


@pytest.mark.parametrize("kind,n,k", [("layered", 13, 7), ("u3cz", 14, 9), ("qft", 12, 6),
                                      ("u3cz", 11, 10)])
@pytest.mark.parametrize("rbits", [3, 4])
@pytest.mark.parametrize("per_part", [False, True])
def test_planned_programs_match_oracle(emu, port, kind, n, k, rbits, per_part):
    gates = _circuit(kind, n, 5)
    parts = partition.partition_dfs(gates, k)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    got, st = emu(n, rec, offs, rbits=rbits, per_part=per_part)
    want = port.run(n, to_records(gates))
    assert np.abs(got - want).max() <= 1e-12
    assert st["rotations"] > 0 or kind == "qft"


def test_rotations_pack_into_rounds(emu):
    """U3 + CZ layers: rotations on distinct register bits share a round."""
    gates = circuits.random_u3_cz(14, 8, 1)
    parts = partition.partition_dfs(gates, 9)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    _, st = emu(14, rec, offs)
    assert st["rotations"] == 14 * 8
    assert st["rounds"] < st["rotations"]


def test_complex64_rounding(emu, port):
    gates = circuits.random_u3_cz(12, 6, 3)
    parts = partition.partition_dfs(gates, 8)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    got, _ = emu(12, rec, offs, dtype=1)
    want = port.run(12, to_records(gates))
    assert np.abs(got - want).max() <= 1e-5


@pytest.mark.parametrize("name", golden_names())
def test_golden_fixtures(emu, name):
    n, rec, offs, basis, amps = load_golden(name)
    init = np.zeros(1 << n, complex)
    init[basis] = 1
    got, _ = emu(n, rec, offs, init=init)
    assert np.abs(got - amps).max() <= 1e-12


def test_every_gate_kind_with_frames(emu, port):
    """Every gate family next to rotations, so the pending diagonal meets
    controlled gates (flushed), two-qubit gates (absorbed), swaps (exchanged),
    diagonal gates (merged) and non-unitary custom matrices (applied as is)."""
    rng = np.random.default_rng(11)
    n = 7
    g = []
    for _ in range(6):
        for q in range(n):
            g.append(Gate("U3", (q,), params=tuple(rng.uniform(0, 2 * np.pi, 3))))
        g += [Gate("X", (1,), (0,)), Gate("RZ", (2,), params=(0.3,)), Gate("SWAP", (3, 4)),
              Gate("RXX", (5, 6), params=(0.7,)), Gate("H", (6,), (2, 3)), Gate("T", (0,)),
              Gate("C1", (4,), params=(1.5, 0.2j, 0.1, 0.9)), Gate("U1", (5,), (1,), params=(0.4,)),
              Gate("RZZ", (0, 3), params=(1.1,)), Gate("Y", (2,)), Gate("S", (5,)),
              Gate("C2", (1, 6), params=tuple(rng.normal(size=16) + 1j * rng.normal(size=16)))]
    for k in (3, 5, 7):
        parts = partition.partition_acyclic(g, k)
        rec, offs = part_offsets(partition.parts_to_gates(g, parts))
        want = port.run(n, to_records(g))
        for per_part in (False, True):
            got, _ = emu(n, rec, offs, per_part=per_part)
            assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("dtype", [0, 1])
def test_group_loads_are_conflict_free(emu, dtype):
    """The per-program shared-memory fold puts the lanes of every register
    group's loads on distinct banks (U3 + CZ layers, parts of <= 9 qubits)."""
    gates = circuits.random_u3_cz(16, 12, 2)
    parts = partition.partition_dfs(gates, 9)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    _, st = emu(16, rec, offs, dtype=dtype)
    assert st["wavefronts"] == st["wavefronts_ideal"]


def test_two_shear_forms_and_scaled_frames(emu, port):
    """Complex128 programs write most rotations as two shears plus a real
    scale carried in the frames (complex64 keeps the exact three-shear form);
    a long circuit, whose frames carry those scales across many parts and
    calls of the global renormalisation, still matches the oracle."""
    n = 12
    gates = circuits.random_u3_cz(n, 60, 21)
    parts = partition.partition_dfs(gates, 7)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    got, st = emu(n, rec, offs)
    assert st["two_shear"] > 0.6 * st["rotations"]
    assert np.abs(got - want).max() <= 1e-12
    got64, st64 = emu(n, rec, offs, dtype=1)
    assert st64["two_shear"] == 0
    assert np.abs(got64 - want).max() <= 1e-5


def test_targets_filling_the_tile_leave_out_low_slots(emu, port):
    """A part whose non-diagonal targets fill the largest tile (12 qubits, none
    of them low) runs as one pass without the low slots (shorter contiguous
    runs rather than a second pass); complex64 keeps slot 0 (its 16-byte
    chunks), so there it takes two."""
    rng = np.random.default_rng(5)
    n = 16
    qs = list(range(3, 15))
    gates = [Gate("U3", (q,), params=tuple(rng.uniform(0, 2 * np.pi, 3))) for q in qs]
    gates += [Gate("Z", (qs[i + 1],), (qs[i],)) for i in range(0, 12, 2)]
    rec, offs = part_offsets([gates])
    want = port.run(n, to_records(gates))
    got, st = emu(n, rec, offs)
    assert st["passes"] == 1 and st["tile_bits"] == 12
    assert np.abs(got - want).max() <= 1e-12
    got64, st64 = emu(n, rec, offs, dtype=1)
    assert st64["passes"] == 2
    assert np.abs(got64 - want).max() <= 1e-5


@pytest.mark.parametrize("kind,n,k", [("u3cz", 16, 7), ("u3cz", 17, 9), ("layered", 14, 5),
                                      ("qft", 13, 6)])
def test_parts_with_free_diagonal_gates(emu, port, kind, n, k):
    """Frontier parts whose qubit limit counts only non-diagonal targets (CZ
    partners and controls act on index bits anywhere): fewer parts, one pass
    each, the oracle's amplitudes."""
    gates = _circuit(kind, n, 5)
    parts = partition.partition_frontier(gates, k, free_diagonal=True)
    assert partition.is_valid_partition(gates, parts)
    assert len(parts) < len(partition.partition_frontier(gates, k))
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    want = port.run(n, to_records(gates))
    for per_part in (False, True):
        got, st = emu(n, rec, offs, per_part=per_part)
        assert st["passes"] == len(parts)
        assert np.abs(got - want).max() <= 1e-12


def test_long_part_splits_into_programs(emu, port):
    """A part with more ops than one program holds (7 rotated qubits, 170
    controlled phases and sign flips on 12 qubits: one free-diagonal part)
    runs as two passes with the frames carried between them."""
    rng = np.random.default_rng(3)
    n = 12
    g = [Gate("U3", (q,), params=tuple(rng.uniform(0, 2 * np.pi, 3))) for q in range(7)]
    for i in range(170):
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        g.append(Gate("U1", (a,), (b,), params=(float(rng.uniform(0, 2 * np.pi)),)) if i % 2
                 else Gate("Z", (a,), (b,)))
    g += [Gate("U3", (q,), params=tuple(rng.uniform(0, 2 * np.pi, 3))) for q in range(7)]
    parts = partition.partition_frontier(g, 7, free_diagonal=True)
    assert len(parts) == 1
    rec, offs = part_offsets(partition.parts_to_gates(g, parts))
    want = port.run(n, to_records(g))
    for per_part in (False, True):
        got, st = emu(n, rec, offs, per_part=per_part)
        assert st["passes"] == 2
        assert np.abs(got - want).max() <= 1e-12
