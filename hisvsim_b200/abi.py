"""ctypes binding of the C ABI in include/hisv.h (libhisv.so).

This is the thin Python view of the drop-in boundary used by the tests, the
benchmark and the Python-level helpers; the pybind11 module
``svsimulator_py_wrapper`` binds the same library with the reference's class
names.  There is no CPU fallback: if libhisv.so is missing, or a call needs a
GPU and none is visible, an error is raised.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from .gates import HS_GATE_DTYPE, Gate, to_records

HERE = os.path.dirname(os.path.abspath(__file__))
# HISV_LIB selects another build of the same library (the index-checked
# libhisv_bounds.so next to it); the default is the normal build
LIB_PATH = os.environ.get("HISV_LIB") or os.path.join(HERE, "libhisv.so")

HS_OK = 0
HS_E_INVALID = -1
HS_E_NOMEM = -2
HS_E_CUDA = -3
HS_E_UNSUPPORTED = -4
HS_E_TIMEOUT = -5
HS_E_NODEVICE = -6
C128 = 0
C64 = 1

_vp = ctypes.c_void_p
_i = ctypes.c_int
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_dp = ctypes.POINTER(ctypes.c_double)
_llp = ctypes.POINTER(ctypes.c_longlong)

# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "hs_last_error": [],
    "hs_version": [],
    "hs_device_count": [ctypes.POINTER(_i)],
    "hs_device_set": [_i],
    "hs_device_synchronize": [],
    "hs_event_create": [ctypes.POINTER(_vp)],
    "hs_event_record": [_vp, _vp],
    "hs_event_elapsed_ms": [_vp, _vp, ctypes.POINTER(ctypes.c_float)],
    "hs_event_destroy": [_vp],
    "hs_launch_bytes": [_llp],
    "hs_state_create": [_i, _i, ctypes.POINTER(_vp)],
    "hs_state_destroy": [_vp],
    "hs_state_num_qubits": [_vp, ctypes.POINTER(_i)],
    "hs_state_dtype": [_vp, ctypes.POINTER(_i)],
    "hs_state_device_ptr": [_vp, ctypes.POINTER(_vp)],
    "hs_state_qubit_to_slot": [_vp, _vp],
    "hs_state_set_basis": [_vp, _u64, _vp],
    "hs_state_copy_to_host": [_vp, _vp, _u64, _u64, _vp],
    "hs_state_copy_from_host": [_vp, _vp, _u64, _u64, _vp],
    "hs_state_canonicalize": [_vp, _vp],
    "hs_state_convert": [_vp, _vp, _vp],
    "hs_gate_apply": [_vp, _vp, _vp],
    "hs_part_run": [_vp, _vp, _i, _vp],
    "hs_frames_create": [_i, ctypes.POINTER(_vp)],
    "hs_frames_destroy": [_vp],
    "hs_frames_pending": [_vp, ctypes.POINTER(_i)],
    "hs_part_run_carry": [_vp, _vp, _vp, _i, _vp],
    "hs_frames_flush": [_vp, _vp, _vp],
    "hs_parts_run": [_vp, _vp, _vp, _i, _vp],
    "hs_set_tile_qubits": [_i],
    "hs_set_k1_reg_bits": [_i],
    "hs_plan_stats": [_i, _i, _vp, _i, _vp],
    "hs_fused_parts_run": [_vp, _vp, _vp, _i, _i, _vp],
    "hs_fused_compose": [_i, _vp, _vp, _i, _vp, _vp],
    "hs_compare": [_vp, _vp, _dp],
    "hs_compare_host": [_vp, _vp, _i, _dp],
    "hs_batch_create_qaoa": [_i, _vp, _vp, _vp, _i, _vp, _vp, ctypes.POINTER(_vp)],
    "hs_batch_set_params": [_vp, _vp, _vp],
    "hs_batch_configure": [_vp, _i, _i],
    "hs_batch_tune": [_vp, _vp, _vp, _dp],
    "hs_batch_run": [_vp, _vp, _dp],
    "hs_batch_stats": [_vp, _vp],
    "hs_batch_set_chunk": [_vp, _i],
    "hs_batch_set_low_keep": [_vp, _i],
    "hs_batch_tile_caps": [_vp, _vp],
    "hs_batch_state": [_vp, _i, _vp],
    "hs_batch_set_wait_limit": [_vp, _u32],
    "hs_bounds_status": [_vp, _i],
    "hs_batch_block_step": [_vp, _i, _i, _i],
    "hs_batch_destroy": [_vp],
    "hs_mlp_create": [_i, ctypes.c_uint64, ctypes.POINTER(_vp)],
    "hs_mlp_num_params": [_vp],
    "hs_mlp_get_params": [_vp, _vp],
    "hs_mlp_set_params": [_vp, _vp],
    "hs_mlp_predict": [_vp, _vp, _i, _vp],
    "hs_mlp_gradients": [_vp, _vp, _vp, _i, _vp, _vp],
    "hs_mlp_train": [_vp, _vp, _vp, _i, _i, _i, ctypes.c_float, ctypes.c_uint64, _vp],
    "hs_mlp_destroy": [_vp],
    "hs_num_part_features": [],
    "hs_part_features": [_i, _i, _vp, _i, _vp, _vp, _i, _vp],
    "hs_order_segments": [_i, _i, _vp, _i, _vp, _i, _i, _i, _vp, _vp, _vp, _vp],
    "hs_parts_run_timed": [_vp, _vp, _vp, _i, _vp, _vp],
    "hs_project": [_vp, _vp, _vp, _i, _i, ctypes.POINTER(_vp), _dp, _vp],
    "hs_fp64_peak": [_dp],
    "hs_set_fused_shape": [_i, _i],
    "hs_set_k4_variant": [_i],
    "hs_fused_apply": [_vp, _vp, _vp, _i, _vp],
    "hs_permute_bits": [_vp, _vp, _i, _vp],
    "hs_gather_qubits": [_vp, _vp, _i, _vp],
    "hs_norm2": [_vp, _dp],
    "hs_norm2_noalloc": [_vp, _dp, _vp],
    "hs_inner": [_vp, _vp, _dp],
    "hs_max_abs_diff": [_vp, _vp, _dp],
    "hs_probability": [_vp, _i, _i, _dp],
    "hs_expect_zz": [_vp, _vp, _i, _dp],
    "hs_measure": [_vp, _vp, _i, _u32, _u64, _vp],
    "hs_counters": [_llp, _llp, _llp],
    "hs_counters_reset": [],
    "hs_set_timing": [_i],
}
_RESTYPE = {"hs_last_error": ctypes.c_char_p}


class HisvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hisv error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Load libhisv.so once (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built: run `python -m hisvsim_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def check(rc: int):
    if rc != HS_OK:
        raise HisvError(rc, lib().hs_last_error().decode(errors="replace"))
    return rc


def device_count() -> int:
    c = _i(0)
    check(lib().hs_device_count(ctypes.byref(c)))
    return c.value


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_vp)


def _records(gates) -> np.ndarray:
    if isinstance(gates, np.ndarray) and gates.dtype == HS_GATE_DTYPE:
        return np.ascontiguousarray(gates)
    return to_records(list(gates))


class State:
    """A device-resident state vector (hs_state)."""

    def __init__(self, n: int, dtype: int = C128):
        h = _vp()
        check(lib().hs_state_create(n, dtype, ctypes.byref(h)))
        self.h = h
        self.n = n
        self.dtype = dtype

    def close(self):
        if getattr(self, "h", None):
            lib().hs_state_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def np_dtype(self):
        return np.complex128 if self.dtype == C128 else np.complex64

    def set_basis(self, x: int, stream=None):
        check(lib().hs_state_set_basis(self.h, x, stream))

    @classmethod
    def _wrap(cls, handle, n: int, dtype: int) -> "State":
        st = cls.__new__(cls)
        st.h, st.n, st.dtype = handle, n, dtype
        return st

    def project(self, qubits, values=None, norm_mode: int = 0):
        """hs_project: (new state over the remaining qubits, probability)."""
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        v = None if values is None else np.ascontiguousarray(values, dtype=np.int32)
        h = _vp()
        p = ctypes.c_double()
        check(lib().hs_project(self.h, _ptr(q), _ptr(v), len(q), norm_mode, ctypes.byref(h),
                               ctypes.byref(p), None))
        return State._wrap(h, self.n - len(q), self.dtype), p.value

    def qubit_to_slot(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int32)
        check(lib().hs_state_qubit_to_slot(self.h, _ptr(out)))
        return out

    def raw(self, first: int = 0, count: Optional[int] = None) -> np.ndarray:
        """Slot-ordered amplitudes [first, first+count)."""
        count = (1 << self.n) - first if count is None else count
        out = np.empty(count, dtype=self.np_dtype)
        check(lib().hs_state_copy_to_host(self.h, _ptr(out), first, count, None))
        return out

    def load(self, amps: np.ndarray, first: int = 0):
        a = np.ascontiguousarray(amps, dtype=self.np_dtype)
        check(lib().hs_state_copy_from_host(self.h, _ptr(a), first, a.size, None))

    def canonicalize(self, stream=None):
        check(lib().hs_state_canonicalize(self.h, stream))

    def amplitudes(self) -> np.ndarray:
        """Amplitudes in qubit order (canonicalizes the slot map first)."""
        self.canonicalize()
        return self.raw()

    def apply(self, gate, stream=None):
        rec = _records([gate] if isinstance(gate, Gate) else gate)
        check(lib().hs_gate_apply(self.h, _ptr(rec), stream))

    def run_part(self, gates, stream=None):
        rec = _records(gates)
        check(lib().hs_part_run(self.h, _ptr(rec), len(rec), stream))

    def run_part_carry(self, frames: "Frames", gates, stream=None):
        """hs_part_run_carry: the part's pending factors stay in `frames`."""
        rec = _records(gates)
        check(lib().hs_part_run_carry(self.h, frames.h, _ptr(rec), len(rec), stream))

    def flush(self, frames: "Frames", stream=None):
        check(lib().hs_frames_flush(self.h, frames.h, stream))

    def run_parts(self, records: np.ndarray, offsets: np.ndarray, stream=None):
        records = _records(records)
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        check(lib().hs_parts_run(self.h, _ptr(records), _ptr(offsets), len(offsets) - 1, stream))

    def run_parts_timed(self, records: np.ndarray, offsets: np.ndarray, stream=None) -> np.ndarray:
        """run_parts with per-part device times (ms)."""
        records = _records(records)
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        ms = np.zeros(len(offsets) - 1, dtype=np.float32)
        check(lib().hs_parts_run_timed(self.h, _ptr(records), _ptr(offsets), len(offsets) - 1,
                                       _ptr(ms), stream))
        return ms

    def run_fused(self, records: np.ndarray, offsets: np.ndarray, precision: int = 0,
                  stream=None):
        """Precision form: one fused unitary per part, tensor-core GEMMs (complex64)."""
        records = _records(records)
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        check(lib().hs_fused_parts_run(self.h, _ptr(records), _ptr(offsets), len(offsets) - 1,
                                       precision, stream))

    def fused_apply(self, u, qubits, precision: int = 0, stream=None):
        """hs_fused_apply: a 64x64 unitary on six qubits (bit j of the index = qubits[j])."""
        u = np.ascontiguousarray(u, dtype=np.complex128).reshape(64, 64)
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        check(lib().hs_fused_apply(self.h, _ptr(u), _ptr(q), precision, stream))

    def compare(self, other: "State") -> dict:
        """<self|other>, max |self - other|, <other|other> and the fidelity."""
        out = np.zeros(4)
        check(lib().hs_compare(self.h, other.h, out.ctypes.data_as(_dp)))
        ip = complex(out[0], out[1])
        na = self.norm2()
        return {"inner": ip, "max_abs_diff": out[2], "norm_other": out[3],
                "fidelity": abs(ip) ** 2 / (na * out[3]) if na * out[3] > 0 else 0.0}

    def compare_host(self, host: np.ndarray) -> dict:
        """compare() against amplitudes held in host memory (qubit order)."""
        host = np.ascontiguousarray(host)
        dt = C128 if host.dtype == np.complex128 else C64
        out = np.zeros(4)
        check(lib().hs_compare_host(self.h, _ptr(host), dt, out.ctypes.data_as(_dp)))
        ip = complex(out[0], out[1])
        na = self.norm2()
        return {"inner": ip, "max_abs_diff": out[2], "norm_other": out[3],
                "fidelity": abs(ip) ** 2 / (na * out[3]) if na * out[3] > 0 else 0.0}

    def permute_bits(self, pairs: Sequence[int], stream=None):
        p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1)
        check(lib().hs_permute_bits(self.h, _ptr(p), len(p) // 2, stream))

    def gather_qubits(self, proc_qubits: Sequence[int], stream=None):
        p = np.ascontiguousarray(proc_qubits, dtype=np.int32)
        check(lib().hs_gather_qubits(self.h, _ptr(p), len(p), stream))

    def norm2(self) -> float:
        out = ctypes.c_double()
        check(lib().hs_norm2(self.h, ctypes.byref(out)))
        return out.value

    def inner(self, other: "State") -> complex:
        out = (ctypes.c_double * 2)()
        check(lib().hs_inner(self.h, other.h, out))
        return complex(out[0], out[1])

    def max_abs_diff(self, other: "State") -> float:
        out = ctypes.c_double()
        check(lib().hs_max_abs_diff(self.h, other.h, ctypes.byref(out)))
        return out.value

    def probability(self, qubit: int, value: int = 0) -> float:
        out = ctypes.c_double()
        check(lib().hs_probability(self.h, qubit, value, ctypes.byref(out)))
        return out.value

    def expect_zz(self, pairs) -> np.ndarray:
        p = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1)
        out = np.zeros(len(p) // 2)
        check(lib().hs_expect_zz(self.h, _ptr(p), len(p) // 2,
                                 out.ctypes.data_as(_dp)))
        return out

    def measure(self, qubits: Sequence[int], nsamples: int, seed: int) -> np.ndarray:
        q = np.ascontiguousarray(qubits, dtype=np.int32)
        out = np.zeros((nsamples, len(q)), dtype=np.int32)
        check(lib().hs_measure(self.h, _ptr(q), len(q), nsamples, seed, _ptr(out)))
        return out


def plan_stats(n: int, gates, dtype: int = C128) -> dict:
    """Host-only K1 planning statistics of one part (no GPU needed)."""
    rec = _records(gates)
    out = np.zeros(6, dtype=np.int32)
    check(lib().hs_plan_stats(n, dtype, _ptr(rec), len(rec), _ptr(out)))
    return dict(zip(["passes", "groups", "ops", "dense", "diag", "tile_bits"], out.tolist()))


def num_part_features() -> int:
    return lib().hs_num_part_features()


def part_features(n: int, gates, parts, dtype: int = C64) -> np.ndarray:
    """Cost-model features (host only) of parts given as gate index lists."""
    rec = _records(gates)
    offs = np.zeros(len(parts) + 1, dtype=np.int32)
    np.cumsum([len(p) for p in parts], out=offs[1:])
    idx = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int32) for p in parts])
                               if parts else np.zeros(0, dtype=np.int32), dtype=np.int32)
    out = np.zeros((len(parts), num_part_features()), dtype=np.float32)
    check(lib().hs_part_features(n, dtype, _ptr(rec), len(rec), _ptr(idx), _ptr(offs), len(parts),
                                 _ptr(out)))
    return out


def order_segments(n: int, gates, order, max_qubits: int, max_len: int, dtype: int = C64):
    """All contiguous segments of a topological order under the limits:
    (start, length, features)."""
    rec = _records(gates)
    order = np.ascontiguousarray(order, dtype=np.int32)
    cap = len(order) * max_len
    st = np.zeros(cap, dtype=np.int32)
    ln = np.zeros(cap, dtype=np.int32)
    ft = np.zeros((cap, num_part_features()), dtype=np.float32)
    cnt = ctypes.c_int32()
    check(lib().hs_order_segments(n, dtype, _ptr(rec), len(rec), _ptr(order), max_qubits, max_len,
                                  cap, _ptr(st), _ptr(ln), _ptr(ft), ctypes.byref(cnt)))
    c = cnt.value
    return st[:c], ln[:c], ft[:c]


def fused_compose(n: int, records: np.ndarray, offsets: np.ndarray):
    """K5 only: FP64 unitaries (parts x 64 x 64) and the qubit of each local bit."""
    records = _records(records)
    offsets = np.ascontiguousarray(offsets, dtype=np.int32)
    nparts = len(offsets) - 1
    u = np.zeros((nparts, 64, 64), dtype=np.complex128)
    q = np.zeros((nparts, 6), dtype=np.int32)
    check(lib().hs_fused_compose(n, _ptr(records), _ptr(offsets), nparts, _ptr(u), _ptr(q)))
    return u, q


def set_device(d: int):
    check(lib().hs_device_set(d))


def synchronize():
    check(lib().hs_device_synchronize())


class Frames:
    """Pending per-qubit factors carried between part calls (hs_frames)."""

    def __init__(self, n: int):
        self.h = _vp()
        check(lib().hs_frames_create(n, ctypes.byref(self.h)))

    @property
    def pending(self) -> bool:
        p = _i()
        check(lib().hs_frames_pending(self.h, ctypes.byref(p)))
        return bool(p.value)

    def close(self):
        if self.h:
            lib().hs_frames_destroy(self.h)
            self.h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Event:
    """A CUDA event recorded on the library's stream (NULL = legacy default)."""

    def __init__(self):
        h = _vp()
        check(lib().hs_event_create(ctypes.byref(h)))
        self.h = h

    def record(self, stream=None):
        check(lib().hs_event_record(self.h, stream))

    def elapsed_ms(self, end: "Event") -> float:
        ms = ctypes.c_float()
        check(lib().hs_event_elapsed_ms(self.h, end.h, ctypes.byref(ms)))
        return ms.value

    def __del__(self):
        try:
            lib().hs_event_destroy(self.h)
        except Exception:
            pass


def launch_bytes() -> int:
    b = ctypes.c_longlong()
    check(lib().hs_launch_bytes(ctypes.byref(b)))
    return b.value


def set_timing(on: bool) -> int:
    return lib().hs_set_timing(1 if on else 0)


class Mlp:
    """Learned cost model: in_dim -> 64 -> 64 -> 64 -> 1 (ReLU, FP32) on the GPU."""

    def __init__(self, in_dim: int, seed: int = 0):
        h = _vp()
        check(lib().hs_mlp_create(in_dim, seed, ctypes.byref(h)))
        self.h = h
        self.in_dim = in_dim
        self.num_params = lib().hs_mlp_num_params(h)

    @staticmethod
    def _f32(a, shape=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        return a if shape is None else a.reshape(shape)

    def params(self) -> np.ndarray:
        out = np.empty(self.num_params, dtype=np.float32)
        check(lib().hs_mlp_get_params(self.h, _ptr(out)))
        return out

    def set_params(self, p):
        p = self._f32(p, (self.num_params,))
        check(lib().hs_mlp_set_params(self.h, _ptr(p)))

    def predict(self, x) -> np.ndarray:
        x = self._f32(x, (-1, self.in_dim))
        out = np.empty(len(x), dtype=np.float32)
        check(lib().hs_mlp_predict(self.h, _ptr(x), len(x), _ptr(out)))
        return out

    def gradients(self, x, y):
        x = self._f32(x, (-1, self.in_dim))
        y = self._f32(y, (-1,))
        g = np.empty(self.num_params, dtype=np.float32)
        loss = ctypes.c_float()
        check(lib().hs_mlp_gradients(self.h, _ptr(x), _ptr(y), len(x), _ptr(g),
                                     ctypes.byref(loss)))
        return loss.value, g

    def train(self, x, y, epochs: int, batch: int = 256, lr: float = 1e-3, seed: int = 0):
        x = self._f32(x, (-1, self.in_dim))
        y = self._f32(y, (-1,))
        losses = np.zeros(max(epochs, 1), dtype=np.float32)
        check(lib().hs_mlp_train(self.h, _ptr(x), _ptr(y), len(x), epochs, batch, lr, seed,
                                 _ptr(losses)))
        return losses[:epochs]

    def close(self):
        if getattr(self, "h", None):
            lib().hs_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class QaoaBatch:
    """Batching form: many QAOA MaxCut instances in one persistent launch."""

    def __init__(self, instances, p: int):
        """instances: list of (n, edges, gammas[p], betas[p])."""
        self.n = np.array([int(i[0]) for i in instances], dtype=np.int32)
        offs = np.zeros(len(instances) + 1, dtype=np.int32)
        np.cumsum([len(i[1]) for i in instances], out=offs[1:])
        edges = np.array([e for i in instances for e in i[1]], dtype=np.int32).reshape(-1)
        g = np.array([i[2] for i in instances], dtype=np.float64).reshape(-1)
        b = np.array([i[3] for i in instances], dtype=np.float64).reshape(-1)
        h = _vp()
        check(lib().hs_batch_create_qaoa(len(instances), _ptr(self.n), _ptr(offs), _ptr(edges), p,
                                         _ptr(g), _ptr(b), ctypes.byref(h)))
        self.h = h
        self.p = p
        self.count = len(instances)

    def set_params(self, gammas, betas):
        g = np.ascontiguousarray(gammas, dtype=np.float64).reshape(-1)
        b = np.ascontiguousarray(betas, dtype=np.float64).reshape(-1)
        check(lib().hs_batch_set_params(self.h, _ptr(g), _ptr(b)))

    def configure(self, tile_cap: int, ctas_per_sm: int):
        check(lib().hs_batch_configure(self.h, tile_cap, ctas_per_sm))

    def set_chunk(self, tiles_per_item: int):
        check(lib().hs_batch_set_chunk(self.h, tiles_per_item))

    def set_low_keep(self, low: int):
        check(lib().hs_batch_set_low_keep(self.h, low))

    def set_wait_limit(self, polls: int):
        """Polls a work item's dependency wait makes before it gives up."""
        check(lib().hs_batch_set_wait_limit(self.h, polls))

    def block_step(self, instance: int, step: int, block: bool = True):
        """Make (or stop making) the wait of one step unreachable (failure tests)."""
        check(lib().hs_batch_block_step(self.h, instance, step, int(block)))

    def tune(self):
        cap, ctas, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        check(lib().hs_batch_tune(self.h, ctypes.byref(cap), ctypes.byref(ctas), ctypes.byref(ms)))
        return cap.value, ctas.value, ms.value

    def run(self):
        out = np.zeros(self.count)
        ms = ctypes.c_double()
        check(lib().hs_batch_run(self.h, out.ctypes.data_as(_dp), ctypes.byref(ms)))
        return out, ms.value

    def stats(self):
        s = np.zeros(8, dtype=np.int64)
        check(lib().hs_batch_stats(self.h, _ptr(s)))
        return dict(zip(["items", "steps", "bytes_per_run", "tile_cap", "ctas_per_sm",
                         "tiles_per_item", "low_keep", "threads"], s.tolist()))

    def tile_caps(self) -> np.ndarray:
        caps = np.zeros(self.count, dtype=np.int32)
        check(lib().hs_batch_tile_caps(self.h, _ptr(caps)))
        return caps

    def state(self, i: int) -> np.ndarray:
        out = np.empty(1 << int(self.n[i]), dtype=np.complex64)
        check(lib().hs_batch_state(self.h, i, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().hs_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_fused_shape(max_ops_per_pass: int, tile_bits: int) -> int:
    r = lib().hs_set_fused_shape(max_ops_per_pass, tile_bits)
    if r < 0:
        check(r)
    return r


def set_k4_variant(variant: int) -> int:
    r = lib().hs_set_k4_variant(variant)
    if r < 0:
        check(r)
    return r


def fp64_peak_tflops() -> float:
    """Measured FP64 FMA throughput of the current device (TFLOP/s)."""
    out = ctypes.c_double()
    check(lib().hs_fp64_peak(ctypes.byref(out)))
    return out.value


def set_tile_qubits(m: int) -> int:
    rc = lib().hs_set_tile_qubits(m)
    if rc < 0:
        check(rc)
    return rc


def set_k1_reg_bits(r: int) -> int:
    """Amplitudes per thread (2^r, r = 3 or 4) of complex128 part passes."""
    rc = lib().hs_set_k1_reg_bits(r)
    if rc < 0:
        check(rc)
    return rc


def bounds_status(reset: bool = False) -> int:
    """Kernel bits whose index checks failed (index-checked build only)."""
    f = _u32(0)
    check(lib().hs_bounds_status(ctypes.byref(f), int(reset)))
    return f.value


def counters():
    a, g, p = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    check(lib().hs_counters(ctypes.byref(a), ctypes.byref(g), ctypes.byref(p)))
    return {"apply_us": a.value, "gates": g.value, "passes": p.value}


def counters_reset():
    check(lib().hs_counters_reset())
