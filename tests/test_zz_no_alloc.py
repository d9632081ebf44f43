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
