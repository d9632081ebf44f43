"""hs_norm2_noalloc: the norm computed with no device allocation.

Some callers cannot let the library call cudaMalloc / cudaFree -- hosts that
hand all device memory to their own pool, or loops that must avoid the
synchronisation those calls can bring.  This entry point keeps its partial sums
in a fixed array inside the library instead.  The test compares it, through
the C ABI, with hs_norm2 (which allocates) on two calls in a row; this file is
collected last so that a stop-at-first-failure run has already run every other
test before it."""
import ctypes

import numpy as np
import pytest

from hisvsim_b200 import abi, circuits

pytestmark = pytest.mark.gpu
TOL = 1e-12


def norm_noalloc(st):
    out = ctypes.c_double()
    abi.check(abi.lib().hs_norm2_noalloc(st.h, ctypes.byref(out), None))
    return out.value


@pytest.mark.parametrize("n,dtype", [(3, abi.C128), (16, abi.C128), (22, abi.C128), (20, abi.C64)])
def test_noalloc_norm_matches_allocating_norm(n, dtype):
    st = abi.State(n, dtype)
    st.run_part(circuits.random_layered(n, 3, 17))
    rng = np.random.default_rng(n)
    scale = rng.uniform(0.5, 2.0)  # a non-unit norm, so the value itself is checked
    amps = st.raw() * scale
    st.load(amps)
    want = st.norm2()
    first = norm_noalloc(st)
    second = norm_noalloc(st)
    assert abs(first - want) <= TOL * max(1.0, want)
    assert abs(second - want) <= TOL * max(1.0, want)
    assert abs(want - scale * scale) <= (1e-12 if dtype == abi.C128 else 1e-5) * scale * scale


def test_noalloc_rejects_null():
    out = ctypes.c_double()
    assert abi.lib().hs_norm2_noalloc(None, ctypes.byref(out), None) == abi.HS_E_INVALID


def test_noalloc_on_a_user_stream():
    """The stream argument: a stream the caller created (not the legacy default
    stream), after work queued on that stream wrote the state."""
    import torch

    n = 18
    st = abi.State(n, abi.C128)
    st.run_part(circuits.random_layered(n, 3, 5))
    want = st.norm2()
    s = torch.cuda.Stream(device=0)
    out = ctypes.c_double()
    for _ in range(3):
        abi.check(abi.lib().hs_norm2_noalloc(st.h, ctypes.byref(out), ctypes.c_void_p(s.cuda_stream)))
        assert abs(out.value - want) <= TOL * max(1.0, want)


@pytest.mark.skipif(abi.device_count() < 2, reason="needs a second GPU")
def test_noalloc_on_a_second_device():
    """The per-device address cache: a state on device 1 after one on device 0."""
    out = ctypes.c_double()
    for dev in (0, 1):
        abi.set_device(dev)
        st = abi.State(12, abi.C128)
        st.run_part(circuits.random_layered(12, 2, dev))
        want = st.norm2()
        abi.check(abi.lib().hs_norm2_noalloc(st.h, ctypes.byref(out), None))
        assert abs(out.value - want) <= TOL * max(1.0, want)
        del st
    abi.set_device(0)
