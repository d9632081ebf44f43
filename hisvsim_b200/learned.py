"""Learned form: a cost model of parts and a proposer of part sizes and cut points.

The network (``abi.Mlp``: 43 features -> 64 -> 64 -> 64 -> 1, ReLU, FP32,
trained by the library's own K7 kernels) predicts the log device time of one
part, scaled to a 30-qubit state, from the part's features
(``abi.part_features``: its qubits, strides, gate mix and the K1 planner's own
pass/group/op counts).  Training data are part timings the simulator measures
on itself (``harvest``: ``hs_parts_run_timed`` over seeded random circuits).

``propose`` chooses a partition of a circuit:
  * for every part size k, the acyclic partitioner's parts (the method without
    the network: ``partition.partition_acyclic``, the role of the reference's
    dagP/acyclic part files) and the frontier partitioner's
    (``partition.partition_frontier``), scored by the network;
  * for several topological orders (DFS, the acyclic partitioner's own order
    at its best k, the frontier partition's order at its best k, the listed
    order), a dynamic program over cut points: every contiguous
    segment of the order with at most ``max_qubits`` qubits is a valid acyclic
    part, the network prices each, and the cheapest segmentation wins.
The acyclic partitioner is the fallback: without a model, or when no
candidate is predicted to be faster than its best k, its parts are returned.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import abi, circuits, partition
from .gates import Gate, part_offsets, to_records

REF_QUBITS = 30
LN2 = math.log(2.0)


def target_from_ms(ms, n):
    """Training target: log of the part's time scaled to a 30-qubit state."""
    return np.log(np.asarray(ms, dtype=np.float64)) - (np.asarray(n) - REF_QUBITS) * LN2


def ms_from_target(y, n):
    return np.exp(np.asarray(y, dtype=np.float64) + (np.asarray(n) - REF_QUBITS) * LN2)


def acyclic_order(gates: Sequence[Gate], k: int) -> List[int]:
    return [i for p in partition.partition_acyclic(gates, k) for i in p]


def _circuit(n: int, layers: int, seed: int) -> List[Gate]:
    if seed % 2 == 0:
        return circuits.random_u3_cz(n, layers, seed)
    return circuits.random_layered(n, layers, seed)


def sample_parts(gates: Sequence[Gate], rng: np.random.Generator, count: int,
                 max_qubits: int = 13) -> List[List[int]]:
    """Parts like those the proposer will price: acyclic and frontier parts of
    random k and random contiguous segments of DFS / acyclic / frontier orders
    under random qubit caps."""
    orders = [partition.dfs_order(gates)]
    orders += [acyclic_order(gates, int(k)) for k in rng.choice(np.arange(4, 13), 2, replace=False)]
    front = partition.partition_frontier(gates, int(rng.integers(4, 13)))
    orders.append([i for p in front for i in p])
    qm = [set(g.controls) | set(g.targets) for g in gates]
    out: List[List[int]] = []
    acyc = partition.partition_acyclic(gates, int(rng.integers(4, 13)))
    out += [list(p) for p in acyc[: count // 8]]
    out += [list(p) for p in front[: count // 8]]
    while len(out) < count:
        order = orders[int(rng.integers(len(orders)))]
        cap = int(rng.integers(2, max_qubits + 1))
        i = int(rng.integers(len(order)))
        qs: set = set()
        seg: List[int] = []
        limit = int(rng.integers(1, 80))
        for j in range(i, len(order)):
            nq = qs | qm[order[j]]
            if len(nq) > cap or len(seg) >= limit:
                break
            qs = nq
            seg.append(order[j])
        if seg:
            out.append(seg)
    return out[:count]


def harvest(counts: Dict[int, int], seed: int = 0, dtype: int = abi.C64, layers: int = 40,
            chunk: int = 256):
    """Time parts on the GPU.  counts: {qubits: number of parts}.  Returns
    (features [N x 43], targets [N], qubits [N], ms [N])."""
    feats, ys, ns, mss = [], [], [], []
    rng = np.random.default_rng(seed)
    for n, cnt in sorted(counts.items()):
        st = abi.State(n, dtype)
        st.set_basis(0)
        done = 0
        c = 0
        while done < cnt:
            gates = _circuit(n, layers, seed * 100003 + n * 1009 + c)
            c += 1
            take = min(chunk, cnt - done)
            parts = sample_parts(gates, rng, take)
            # the first part runs twice; its first time (launch from idle) is dropped
            plist = [parts[0]] + parts
            rec, offs = part_offsets([[gates[i] for i in p] for p in plist])
            ms = st.run_parts_timed(rec, offs)[1:]
            x = abi.part_features(n, gates, parts, dtype)
            keep = ms > 0
            feats.append(x[keep])
            mss.append(ms[keep])
            ns.append(np.full(int(keep.sum()), n))
            done += take
        st.close()
    X = np.concatenate(feats).astype(np.float32)
    n_all = np.concatenate(ns)
    ms_all = np.concatenate(mss).astype(np.float64)
    return X, target_from_ms(ms_all, n_all).astype(np.float32), n_all, ms_all


class CostModel:
    """The MLP with the target scaling; ``predict_ms`` prices parts at n qubits."""

    def __init__(self, seed: int = 0):
        self.mlp = abi.Mlp(abi.num_part_features(), seed)
        self.trained = False
        self.floor = -np.inf

    def fit(self, X, y, epochs: int = 150, batch: int = 256, lr: float = 2e-3, seed: int = 0):
        losses = self.mlp.train(X, y, epochs, batch, lr, seed)
        self.trained = True
        # no part runs faster than the fastest pass measured (a pass streams
        # the whole state): predictions are held above the smallest training
        # target
        self.floor = float(np.min(np.asarray(y, dtype=np.float64)))
        return losses

    def predict_target(self, X) -> np.ndarray:
        return np.maximum(self.mlp.predict(X).astype(np.float64), self.floor)

    def predict_ms(self, X, n) -> np.ndarray:
        return ms_from_target(self.predict_target(X), n)

    def close(self):
        self.mlp.close()


def _dp(starts: np.ndarray, lens: np.ndarray, cost: np.ndarray, total: int):
    """Cheapest segmentation of [0, total) into the given segments."""
    best = np.full(total + 1, np.inf)
    arg = np.full(total + 1, -1, dtype=np.int64)
    best[0] = 0.0
    order = np.argsort(starts, kind="stable")
    for s in order:  # segments ending at i all start before i: best[i] is final
        i = int(starts[s])
        if not np.isfinite(best[i]):
            continue
        j = i + int(lens[s])
        v = best[i] + cost[s]
        if v < best[j]:
            best[j] = v
            arg[j] = s
    if not np.isfinite(best[total]):
        return None, np.inf
    cuts = []
    j = total
    while j > 0:
        s = int(arg[j])
        cuts.append((int(starts[s]), int(lens[s])))
        j = int(starts[s])
    return cuts[::-1], float(best[total])


def propose(gates: Sequence[Gate], n: int, model: Optional[CostModel], dtype: int = abi.C64,
            ks: Sequence[int] = tuple(range(4, 13)), default_k: int = 9, max_qubits: int = 12,
            max_len: int = 64, dp_margin: float = 0.10) -> dict:
    """Choose part sizes and cut points.  Returns {"parts", "method",
    "predicted_ms", "candidates"}; the fallback is partition_acyclic(default_k).

    A dynamic-programming segmentation is taken over the best partitioner
    candidate only when its predicted time is lower by more than
    ``dp_margin``: the minimum over many segments' noisy predictions is
    biased low (each segment is picked where the network errs low): measured,
    such segmentations predicted 3% faster than the best partitioner came
    out up to 6% slower."""
    if model is None or not model.trained:
        return {"parts": partition.partition_acyclic(gates, default_k),
                "method": f"acyclic k={default_k} (no model)", "predicted_ms": None,
                "candidates": {}}
    cands = {}
    best_k, best_k_ms = default_k, np.inf
    best_f, best_f_ms, best_f_parts = default_k, np.inf, None
    for k in ks:
        parts = partition.partition_acyclic(gates, k)
        ms = float(model.predict_ms(abi.part_features(n, gates, parts, dtype), n).sum())
        cands[f"acyclic k={k}"] = (ms, parts)
        if ms < best_k_ms:
            best_k, best_k_ms = k, ms
        fparts = partition.partition_frontier(gates, k)
        fms = float(model.predict_ms(abi.part_features(n, gates, fparts, dtype), n).sum())
        cands[f"frontier k={k}"] = (fms, fparts)
        if fms < best_f_ms:
            best_f, best_f_ms, best_f_parts = k, fms, fparts
    orders = {"dfs": partition.dfs_order(gates),
              f"acyclic-order k={best_k}": acyclic_order(gates, best_k),
              f"frontier-order k={best_f}": [i for p in best_f_parts for i in p],
              "listed": list(range(len(gates)))}
    for name, order in orders.items():
        st, ln, ft = abi.order_segments(n, gates, order, max_qubits, max_len, dtype)
        cost = model.predict_ms(ft, n)
        cuts, total = _dp(st, ln, cost, len(order))
        if cuts is None:
            continue
        parts = [[order[i] for i in range(a, a + l)] for a, l in cuts]
        cands[f"dp over {name} order"] = (total, parts)
    name = min(cands, key=lambda c: cands[c][0])
    base = min((c for c in cands if not c.startswith("dp over")), key=lambda c: cands[c][0])
    if name.startswith("dp over") and cands[name][0] > (1.0 - dp_margin) * cands[base][0]:
        name = base
    if cands[name][0] >= cands[f"acyclic k={best_k}"][0]:
        name = f"acyclic k={best_k}"
    return {"parts": cands[name][1], "method": name, "predicted_ms": cands[name][0],
            "candidates": {c: v[0] for c, v in cands.items()}}


def propose_fewest(gates: Sequence[Gate], n: int, dtype: int = abi.C64, max_qubits: int = 12,
                   max_len: int = 64) -> dict:
    """The proposer's dynamic program with a trivial cost (every segment costs
    1: the fewest parts) over the same orders and segment limits: the method
    without the network, for measuring what the network adds."""
    best = None
    orders = {"dfs": partition.dfs_order(gates), "listed": list(range(len(gates))),
              "frontier": [i for p in partition.partition_frontier(gates, max_qubits) for i in p]}
    for name, order in orders.items():
        st, ln, _ = abi.order_segments(n, gates, order, max_qubits, max_len, dtype)
        cuts, total = _dp(st, ln, np.ones(len(st)), len(order))
        if cuts is None:
            continue
        parts = [[order[i] for i in range(a, a + l)] for a, l in cuts]
        if best is None or total < best[0]:
            best = (total, parts, f"fewest parts over {name} order")
    return {"parts": best[1], "method": best[2], "num_parts": int(best[0])}


def measure(st: "abi.State", gates: Sequence[Gate], parts, reps: int = 3, warmup: int = 1) -> float:
    """Device time (s) of one run of the circuit in the given parts (median)."""
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    times = []
    for r in range(warmup + reps):
        st.set_basis(0)
        a, b = abi.Event(), abi.Event()
        abi.synchronize()
        a.record()
        st.run_parts(rec, offs)
        b.record()
        abi.synchronize()
        if r >= warmup:
            times.append(a.elapsed_ms(b) / 1e3)
    return float(np.median(times))
