"""ctypes front of the oracle libraries.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference arm, as the checker; the product
(hisvsim_b200) never imports it.

Two oracles share one contract (``run``):
  * ``RefOracle``  -- oracle/_ref/libhisv_ref.so: the reference's own C++
    headers driven by ref_harness.cpp (BoundGate::apply per gate,
    state_vector.hpp:1349; gather_and_execute_on_multi per part,
    execute.hpp:318-470).
  * ``PortOracle`` -- oracle/_build/libhisv_port.so: port.c, the plain-C
    restatement of the same path, plus the redistribution permutation
    (svsim-mpi.hpp:123-173) and the reductions.
Both are built by oracle/Makefile (``make -C oracle``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libhisv_ref.so")
PORT_LIB = os.path.join(HERE, "_build", "libhisv_port.so")

_c_int = ctypes.c_int
_p = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _prep(n, gates, offsets, init_state):
    gates = np.ascontiguousarray(gates)
    if offsets is None:
        offsets = np.array([0, len(gates)], dtype=np.int32)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    if init_state is None:
        state = np.zeros(1 << n, dtype=np.complex128)
        init = 0
    else:
        state = np.array(init_state, dtype=np.complex128, copy=True)
        if state.size != (1 << n):
            raise ValueError("init_state must have 2^n amplitudes")
        init = 1
    return gates, offsets, state, init


class RefOracle:
    """The reference's CPU path, compiled from its own headers."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        self.lib = ctypes.CDLL(path)
        self.lib.ref_run.argtypes = [_c_int, _p, _c_int, _p, _c_int, _c_int, _c_int, _c_int,
                                     _c_int, _p]
        self.lib.ref_run.restype = _c_int
        self.lib.ref_probability.argtypes = [_c_int, _p, _c_int, _c_int]
        self.lib.ref_probability.restype = ctypes.c_double
        self.lib.ref_project.argtypes = [_c_int, _p, _p, _p, _c_int, _c_int, _p]
        self.lib.ref_project.restype = _c_int
        self.gate_size = self.lib.ref_hs_gate_size()

    def run(self, n, gates, offsets=None, mode=0, opt_slots=0, threads=None,
            init_state=None):
        """mode 0: per-gate sweeps; mode 1: parts (gate records split by offsets)."""
        threads = threads or os.cpu_count() or 1
        gates, offsets, state, init = _prep(n, gates, offsets, init_state)
        rc = self.lib.ref_run(n, _ptr(gates), len(gates), _ptr(offsets), len(offsets) - 1,
                              mode, opt_slots, threads, init, _ptr(state))
        if rc != 0:
            raise ValueError("reference rejected the circuit")
        return state

    def probability(self, n, state, qubit, value=0):
        state = np.ascontiguousarray(state, dtype=np.complex128)
        return self.lib.ref_probability(n, _ptr(state), qubit, value)

    def project(self, n, state, qubits, values, renormalize=True):
        """StateVector::project (state_vector.hpp:829-894): the reference's
        projected state over the remaining qubits (it divides by p)."""
        state = np.ascontiguousarray(state, dtype=np.complex128)
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.int32)
        out = np.zeros(1 << (n - len(q)), dtype=np.complex128)
        rc = self.lib.ref_project(n, _ptr(state), _ptr(q), _ptr(v), len(q), int(renormalize),
                                  _ptr(out))
        if rc != 0:
            raise ValueError("reference rejected the projection")
        return out


class PortOracle:
    """port.c: the plain-C restatement of the reference path."""

    def __init__(self, path: str = PORT_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle port`")
        self.lib = ctypes.CDLL(path)
        self.lib.port_run.argtypes = [_c_int, _p, _c_int, _p, _c_int, _c_int, _c_int, _c_int, _p]
        self.lib.port_run.restype = _c_int
        self.lib.port_gather_slots.argtypes = [_p, _p, _c_int, _p, _c_int]
        self.lib.port_gather_slots.restype = _c_int
        self.lib.port_probability.argtypes = [_c_int, _p, _c_int, _c_int]
        self.lib.port_probability.restype = ctypes.c_double
        self.lib.port_norm2.argtypes = [_c_int, _p]
        self.lib.port_norm2.restype = ctypes.c_double
        self.lib.port_construct.argtypes = [_p, _p]
        self.lib.port_construct.restype = _c_int
        self.gate_size = self.lib.port_hs_gate_size()

    def run(self, n, gates, offsets=None, mode=0, opt_slots=0, threads=None,
            init_state=None):
        gates, offsets, state, init = _prep(n, gates, offsets, init_state)
        rc = self.lib.port_run(n, _ptr(gates), len(gates), _ptr(offsets), len(offsets) - 1,
                               mode, opt_slots, init, _ptr(state))
        if rc != 0:
            raise ValueError("port rejected the circuit")
        return state

    def construct(self, gate_record):
        rec = np.ascontiguousarray(np.atleast_1d(gate_record))
        out = np.zeros(16, dtype=np.complex128)
        if self.lib.port_construct(_ptr(rec), _ptr(out)) != 0:
            raise ValueError("port rejected the gate")
        return out

    def gather_slots(self, state, n, proc_slots):
        state = np.ascontiguousarray(state, dtype=np.complex128)
        out = np.empty_like(state)
        ps = np.ascontiguousarray(proc_slots, dtype=np.int32)
        if self.lib.port_gather_slots(_ptr(state), _ptr(out), n, _ptr(ps), len(ps)) != 0:
            raise ValueError("bad slot set")
        return out

    def probability(self, n, state, slot, value=0):
        state = np.ascontiguousarray(state, dtype=np.complex128)
        return self.lib.port_probability(n, _ptr(state), slot, value)

    def norm2(self, n, state):
        state = np.ascontiguousarray(state, dtype=np.complex128)
        return self.lib.port_norm2(n, _ptr(state))
