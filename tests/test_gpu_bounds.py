"""The index-checked build (libhisv_bounds.so, compiled with -DHS_BOUNDS):
every global and shared-memory access of the part (K1), bit-swap (K2), fused
(K4) and batch (K6) kernels checks its index, and a failed check skips the
access and sets the kernel's bit.  The small parity cases of those kernels
run against it in a fresh process (HISV_LIB selects the build) and must give
the oracle's results with every bit clear.  This stands in for a device
memory checker."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

SCRIPT = r'''
import numpy as np
from hisvsim_b200 import abi, circuits, partition
from hisvsim_b200.gates import Gate, part_offsets, to_records
from oracle.oracle import PortOracle

assert abi.LIB_PATH.endswith("libhisv_bounds.so"), abi.LIB_PATH
port = PortOracle()
abi.set_device(0)
abi.bounds_status(reset=True)

def fid(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)

# K1: layered circuits with every gate family, U3 + CZ, QFT; 8 and 16
# amplitudes per thread; complex128 and complex64
cases = [(circuits.random_layered(13, 6, 3), 13, 7), (circuits.random_u3_cz(15, 8, 4), 15, 9),
         (circuits.qft(12, 5)[0], 12, 6), (circuits.random_u3_cz(17, 6, 8), 17, 10)]
for rb in (4, 3):
    abi.set_k1_reg_bits(rb)
    for gates, n, k in cases:
        parts = partition.partition_dfs(gates, k)
        rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
        want = port.run(n, to_records(gates))
        st = abi.State(n, abi.C128)
        st.run_parts(rec, offs)
        assert np.abs(st.amplitudes() - want).max() <= 1e-12, ("K1", rb, n)
        s64 = abi.State(n, abi.C64)
        s64.run_parts(rec, offs)
        assert np.abs(s64.amplitudes() - want).max() <= 1e-5, ("K1 c64", rb, n)
abi.set_k1_reg_bits(4)

# K2: bit-swap passes and the return to the identity map
n = 16
gates = circuits.random_layered(n, 3, 9)
want = port.run(n, to_records(gates))
st = abi.State(n, abi.C128)
st.load(want)
st.permute_bits([(0, 15), (3, 9), (5, 12)])
st.permute_bits([(1, 14), (2, 7)])
st.canonicalize()
assert np.abs(st.amplitudes() - want).max() == 0.0, "K2"

# K4: one unitary per pass (bulk-loaded, warp-specialised) and two per pass
n = 16
gates = circuits.random_u3_cz(n, 8, 17)
parts = partition.partition_dfs(gates, 6)
rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
want = port.run(n, to_records(gates))
for variant, shape in ((2, (1, 13)), (2, (1, 12)), (1, (1, 13)), (2, (2, 12))):
    pv = abi.set_k4_variant(variant)
    ps = abi.set_fused_shape(*shape)
    st = abi.State(n, abi.C64)
    st.run_fused(rec, offs, 0)
    got = st.amplitudes().astype(complex)
    abi.set_fused_shape(ps // 100, ps % 100)
    abi.set_k4_variant(pv)
    assert 1 - fid(want, got) <= 1e-8, ("K4", variant, shape)

# K6: a small batch against complex128 plain runs
insts = []
for i, nq in enumerate([8, 11, 13, 16]):
    g, e, gam, bet = circuits.qaoa_maxcut(nq, 3, 40 + i)
    insts.append((nq, e, gam, bet, g))
b = abi.QaoaBatch([(nq, e, gm, bt) for nq, e, gm, bt, _ in insts], 3)
for cap in (9, 12):
    b.configure(cap, 4)
    hc, _ = b.run()
    for i, (nq, e, _, _, g) in enumerate(insts):
        w = port.run(nq, to_records(g))
        assert np.abs(b.state(i) - w).max() <= 1e-5, ("K6", cap, i)
b.close()

flags = abi.bounds_status()
print("BOUNDS_FLAGS", flags)
assert flags == 0, flags
'''


def test_kernels_under_index_checks():
    lib = os.path.join(ROOT, "hisvsim_b200", "libhisv_bounds.so")
    assert os.path.exists(lib), "build the index-checked library (hisvsim_b200.build)"
    env = dict(os.environ, HISV_LIB=lib, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", SCRIPT], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "BOUNDS_FLAGS 0" in r.stdout
