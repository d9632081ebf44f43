"""Host-side checks that need no GPU: the C ABI library and its exports, the
pybind11 module's API surface and error behaviour, partitioners and the
part-file format, circuit generators."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from hisvsim_b200 import abi, circuits, partition
from hisvsim_b200.gates import HS_GATE_DTYPE, Gate, to_records


def header_functions():
    txt = open(os.path.join(ROOT, "include", "hisv.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hs_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = abi.lib()
    names = header_functions()
    assert len(names) >= 29
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_signatures_cover_header():
    assert set(header_functions()) <= set(abi.SIGNATURES)


def test_gate_record_layout(port):
    assert HS_GATE_DTYPE.itemsize == 320 == port.gate_size


def test_version_and_errors_without_device():
    assert abi.lib().hs_version() >= 1
    if abi.device_count() == 0:
        with pytest.raises(abi.HisvError) as e:
            abi.State(4)
        assert e.value.code == abi.HS_E_NODEVICE


def test_null_state_is_an_error():
    rc = abi.lib().hs_norm2(None, ctypes.byref(ctypes.c_double()))
    assert rc == abi.HS_E_INVALID
    assert b"null" in abi.lib().hs_last_error()


def test_tile_hint_bounds():
    assert abi.lib().hs_set_tile_qubits(99) == abi.HS_E_INVALID
    prev = abi.set_tile_qubits(11)
    assert abi.set_tile_qubits(prev) == 11
    assert abi.lib().hs_set_k1_reg_bits(2) == abi.HS_E_INVALID
    prev = abi.set_k1_reg_bits(3)
    assert prev == 4  # the default
    assert abi.set_k1_reg_bits(prev) == 3


def test_fused_knob_bounds():
    """K4 variant and fused pass shape: defaults (bulk-loaded, one unitary
    per pass on 2^13 tiles) and the rejected values."""
    assert abi.lib().hs_set_k4_variant(3) == abi.HS_E_INVALID
    assert abi.lib().hs_set_k4_variant(-1) == abi.HS_E_INVALID
    prev = abi.set_k4_variant(1)
    assert prev == 2
    assert abi.set_k4_variant(prev) == 1
    assert abi.lib().hs_set_fused_shape(1, 14) == abi.HS_E_INVALID
    assert abi.lib().hs_set_fused_shape(2, 13) == abi.HS_E_INVALID
    prev = abi.set_fused_shape(2, 12)
    assert prev == 113
    assert abi.set_fused_shape(prev // 100, prev % 100) == 212


def test_pymod_surface():
    from hisvsim_b200 import svsimulator_py_wrapper as sv

    for name in ["AggregateGate_0", "AggregateGate_1", "AggregateGate_2", "AggregateGate_3",
                 "AggregateGate_C1", "AggregateGate_C2", "AggregateGate_Frac",
                 "AggregateGateFactory", "StateVector", "BoundGate", "gather_and_execute_on",
                 "gather_and_execute_on_mpi", "gather_and_execute_multilevel_on_mpi",
                 "obtain_apply_time", "obtain_gate_counter", "obtain_move_counter",
                 "obtain_gather_time", "set_num_threads", "set_init_num_threads",
                 "set_opt_slots"]:
        assert hasattr(sv, name), name
    ag = sv.AggregateGate_3("u3", 0.1, 0.2, 0.3)
    b = sv.BoundGate(sv.AggregateGateFactory(ag), [1], [0])
    assert b is not None
    # names the reference cannot build raise instead of aborting
    with pytest.raises(ValueError):
        sv.AggregateGate_0("RX")
    with pytest.raises(ValueError):
        sv.AggregateGate_1("NOPE", 1.0)
    with pytest.raises(ValueError):
        sv.AggregateGate_Frac("RZFrac", 1, 2)  # mixed-case table entry never matches
    with pytest.raises(ValueError):
        sv.BoundGate(sv.AggregateGateFactory(sv.AggregateGate_0("X")), [1, 2, 3, 4, 5, 6], [0])


@pytest.mark.parametrize("strategy", [partition.partition_acyclic, partition.partition_natural,
                                      partition.partition_dfs])
@pytest.mark.parametrize("k", [2, 4, 7])
def test_partitions_valid(strategy, k):
    gates = circuits.random_layered(12, 5, 4)
    parts = strategy(gates, k)
    assert partition.is_valid_partition(gates, parts)
    for p in parts:
        assert len({q for i in p for q in gates[i].qubits}) <= k


def test_acyclic_beats_natural():
    gates = circuits.random_u3_cz(20, 10, 1)
    a = partition.partition_acyclic(gates, 6)
    b = partition.partition_natural(gates, 6)
    assert len(a) <= len(b)


def test_part_file_roundtrip(tmp_path):
    gates = circuits.random_layered(8, 3, 2)
    parts = partition.partition_acyclic(gates, 4)
    f = tmp_path / "c_part_smart"
    partition.write_part_file(str(f), gates, parts)
    assert partition.read_part_file(str(f), len(gates)) == parts
    # order id 0 and ids beyond the gate list are skipped (parse rules of the reference driver)
    with open(f, "a") as fh:
        fh.write(f"0 start 0\n{len(gates) + 2000} exit 1\n")
    assert partition.read_part_file(str(f), len(gates)) == parts


def test_partition_rejects_oversized_gate():
    with pytest.raises(ValueError):
        partition.partition_acyclic([Gate("X", (0,), (1, 2))], 2)


def test_generators_shapes():
    g = circuits.random_layered(20, 20, 0)
    assert len(g) == 20 * (20 + 10)
    g2 = circuits.random_u3_cz(33, 40, 0)
    assert len(g2) == 40 * (33 + 16)
    q, x = circuits.qft(30, 1)
    assert len(q) == 30 + 30 * 29 // 2 + 15 and 0 <= x < 2 ** 30
    qa, edges, gam, bet = circuits.qaoa_maxcut(16, 4, 9)
    assert len(edges) == 24 and all(d == 3 for d in np.bincount(np.ravel(edges)))
    assert circuits.random_layered(10, 3, 5) == circuits.random_layered(10, 3, 5)


def test_records_roundtrip():
    gates = [Gate("U3", (3,), (1, 2), params=(0.1, 0.2, 0.3)), Gate("R1FRAC", (0,), frac=(3, 4))]
    r = to_records(gates)
    assert r["type"].tolist() == [25, 19]
    assert r["controls"][0][:2].tolist() == [1, 2]
    assert r["frac_num"][1] == 3 and r["frac_pow"][1] == 4


def test_odd_qubit_counts_use_near_regular_graphs():
    for n in (17, 21, 25):
        edges = circuits.random_maxcut_graph(n, np.random.default_rng(n))
        deg = np.bincount(np.array(edges).reshape(-1), minlength=n)
        assert sorted(deg.tolist()) == [2] + [3] * (n - 1)
        assert len(edges) == (3 * n - 1) // 2
    assert len(circuits.random_maxcut_graph(16, np.random.default_rng(0))) == 24


@pytest.mark.parametrize("bad", ["small_n", "big_n", "self_loop", "edge_range", "rounds"])
def test_batch_rejects_bad_instances(bad):
    n, edges, p = 8, [(0, 1), (2, 3)], 2
    if bad == "small_n":
        n = 3
        edges = [(0, 1)]
    elif bad == "big_n":
        n = 31
    elif bad == "self_loop":
        edges = [(2, 2)]
    elif bad == "edge_range":
        edges = [(0, 8)]
    elif bad == "rounds":
        p = 9
    with pytest.raises(abi.HisvError) as e:
        abi.QaoaBatch([(n, edges, [0.1] * p, [0.2] * p)], p)
    assert e.value.code == abi.HS_E_INVALID


class _PassCountModel:
    """Stand-in cost model (no GPU): one unit per K1 pass plus a little per gate."""

    trained = True

    def predict_ms(self, X, n):
        return X[:, 9] * 4.0 + X[:, 2] * 0.05


def test_part_features_layout():
    from hisvsim_b200 import learned  # noqa: F401  (imports without a GPU)

    gates = circuits.random_u3_cz(12, 4, 2)
    parts = partition.partition_acyclic(gates, 5)
    f = abi.part_features(12, gates, parts)
    assert f.shape == (len(parts), abi.num_part_features()) == (len(parts), 43)
    assert np.all(f[:, 0] == np.float32(12 / 32))
    for p, row in zip(parts, f):
        assert row[2] == pytest.approx(len(p) / 32)
        qs = {q for i in p for q in gates[i].controls + gates[i].targets}
        assert row[1] == pytest.approx(len(qs) / 12)
        st = abi.plan_stats(12, [gates[i] for i in p], abi.C64)
        assert row[9] == pytest.approx(st["passes"] / 4) and row[14] == pytest.approx(st["tile_bits"] / 12)
        assert row[15:].sum() == pytest.approx(len(p) / 16)


def test_order_segments_are_convex_parts():
    gates = circuits.random_layered(10, 5, 4)
    order = partition.dfs_order(gates)
    st, ln, ft = abi.order_segments(10, gates, order, 6, 20)
    assert len(st) == len(ln) == len(ft) > 0
    assert (ln >= 1).all() and (ln <= 20).all()
    for a, l in list(zip(st, ln))[::37]:
        seg = [order[i] for i in range(a, a + l)]
        qs = {q for i in seg for q in gates[i].controls + gates[i].targets}
        assert len(qs) <= 6
    rc = abi.lib().hs_order_segments(10, 1, None, 0, None, 6, 20, 0, None, None, None, None)
    assert rc == abi.HS_E_INVALID


def test_proposer_dp_and_fallback():
    from hisvsim_b200 import learned

    gates = circuits.random_u3_cz(14, 6, 9)
    fb = learned.propose(gates, 14, None, default_k=7)
    assert fb["method"].startswith("acyclic k=7")
    assert fb["parts"] == partition.partition_acyclic(gates, 7)
    prop = learned.propose(gates, 14, _PassCountModel(), ks=(5, 7, 9))
    assert partition.is_valid_partition(gates, prop["parts"])
    best_acyclic = min(v for k, v in prop["candidates"].items() if k.startswith("acyclic"))
    assert prop["predicted_ms"] <= best_acyclic + 1e-9
    # the dynamic program is exact: no segmentation of its order is cheaper
    cuts, total = learned._dp(np.array([0, 0, 1, 2]), np.array([1, 3, 2, 1]),
                              np.array([1.0, 2.5, 1.0, 1.0]), 3)
    assert cuts == [(0, 1), (1, 2)] and total == 2.0


def test_index_checks_only_in_the_checked_build():
    """The normal build has no index checks (hs_bounds_status says so); the
    index-checked build exports the same C ABI."""
    with pytest.raises(abi.HisvError) as e:
        abi.bounds_status()
    assert e.value.code == abi.HS_E_UNSUPPORTED
    path = os.path.join(ROOT, "hisvsim_b200", "libhisv_bounds.so")
    assert os.path.exists(path)
    L = ctypes.CDLL(path)
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.parametrize("k", [3, 6, 9])
def test_frontier_partition_valid_and_fewer(k):
    """The frontier partitioner gives valid acyclic parts under the qubit
    limit, and fewer than the DFS-order runs on layered circuits."""
    for gates in (circuits.random_u3_cz(16, 12, k), circuits.random_layered(12, 6, k)):
        parts = partition.partition_frontier(gates, k)
        assert partition.is_valid_partition(gates, parts)
        for p in parts:
            assert len({q for i in p for q in gates[i].qubits}) <= k
    g = circuits.random_u3_cz(33, 40, 2024)
    assert len(partition.partition_frontier(g, k)) < 0.9 * len(partition.partition_dfs(g, k))
    with pytest.raises(ValueError):
        partition.partition_frontier([Gate("X", (0,), (1, 2))], 2)


def test_frames_handles_without_device():
    """The deferred-factor handle is host-only: created, queried, destroyed;
    bad sizes are rejected."""
    fr = abi.Frames(12)
    assert not fr.pending
    fr.close()
    h = ctypes.c_void_p()
    assert abi.lib().hs_frames_create(0, ctypes.byref(h)) == abi.HS_E_INVALID
    assert abi.lib().hs_frames_create(64, ctypes.byref(h)) == abi.HS_E_INVALID
    assert abi.lib().hs_frames_pending(None, None) == abi.HS_E_INVALID
    assert abi.lib().hs_part_run_carry(None, None, None, 0, None) == abi.HS_E_INVALID


def test_proposer_segmentation_margin():
    """A dynamic-programming segmentation replaces the best whole-partition
    candidate only when predicted faster by more than the margin: with the
    margin at 1 it never does, with 0 the cheapest prediction wins."""
    from hisvsim_b200 import learned

    gates = circuits.random_u3_cz(14, 6, 9)
    strict = learned.propose(gates, 14, _PassCountModel(), ks=(5, 7, 9), dp_margin=1.0)
    assert not strict["method"].startswith("dp over")
    loose = learned.propose(gates, 14, _PassCountModel(), ks=(5, 7, 9), dp_margin=0.0)
    assert loose["predicted_ms"] == pytest.approx(min(loose["candidates"].values()))
    assert strict["predicted_ms"] >= loose["predicted_ms"]


def test_bench_partitions(monkeypatch):
    """The benchmark's part choices: the plain form's frontier parts bound only
    non-diagonal targets, the precision form's and the reference path's every
    touched qubit; all are valid partitions of the workload."""
    import sys

    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setattr(sys, "argv", ["bench.py"])
    args = bench.parse()
    gates, parts, rec, offs = bench.workload(20, 6, 1, 9, bench.plain_partitioner(args))
    assert partition.is_valid_partition(gates, parts) and int(offs[-1]) == len(gates)
    bounded = bench.partitioner(args)(gates, 9)
    assert partition.is_valid_partition(gates, bounded)
    assert len(parts) < len(bounded)
    for p in bounded:
        assert len({q for i in p for q in gates[i].qubits}) <= 9
    fused = bench.partitioner(args)(gates, 6)
    assert all(len({q for i in p for q in gates[i].qubits}) <= 6 for p in fused)
