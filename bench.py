"""Benchmark: a 33-qubit, 40-layer random circuit on one B200.

Workload (seeded synthetic stand-in for the reference's QASMBench-style
circuits): 40 layers of U3 with uniform angles on every qubit followed by CZ
on a random matching (33 is odd: one qubit idles per layer), 1960 gates,
state |0...0>, acyclic parts of <= k qubits from hisvsim_b200.partition
(grown from the DAG's ready frontier by default, the fewest parts; for the
plain form's part kernel the limit counts only non-diagonal targets, since
CZ partners and controls act on index bits wherever they are;
--partitioner dfs / acyclic select DFS-order runs or the greedy acyclic
partitioner).

A step simulates the whole circuit once.  `value` is the plain complex128
form's throughput in amplitude updates per second (sum over gates of 2^n,
divided by the circuit's device time); the circuit seconds and the HBM GB/s
of the K1 passes ride along in the same line.  The state (128 GiB) is far
larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hisv|reference]

Multi-GPU: replicas only (the path does not shard in this build); every rank
simulates its own circuit, timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "33q circuit sec & HBM GB/s; fused FP32 vs plain FP64 GPU at 1-F≤1e-6"
UNIT = "amp-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hisv", choices=["hisv", "reference"])
    ap.add_argument("--qubits", type=int, default=33)
    ap.add_argument("--layers", type=int, default=40)
    ap.add_argument("--part-qubits", type=int, default=9)
    ap.add_argument("--partitioner", default="frontier", choices=["frontier", "dfs", "acyclic"],
                    help="acyclic parts grown from the DAG's ready frontier (default, fewest "
                         "parts), consecutive runs of a DFS topological order, or the greedy "
                         "acyclic partitioner")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-qubits", type=int, default=26, help="size of the CPU sample")
    ap.add_argument("--cpu-layers", type=int, default=8)
    ap.add_argument("--cpu-full-qubits", type=int, default=30,
                    help="state size of the full-size CPU rate (16 GiB at 30)")
    ap.add_argument("--cpu-full-layers", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--tile-qubits", type=int, default=0, help="K1 tile bits (0 = automatic)")
    ap.add_argument("--no-fused", action="store_true", help="skip the precision form")
    ap.add_argument("--fused-shape", default="",
                    help="unitaries per pass and tile bits of the precision form, e.g. 2,12")
    ap.add_argument("--no-fidelity", action="store_true", help="skip the 1-F check")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching form")
    ap.add_argument("--batch-instances", type=int, default=512)
    ap.add_argument("--batch-check", type=int, default=512,
                    help="instances whose <H_C> is checked against complex128 plain runs")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned form")
    ap.add_argument("--no-config1", action="store_true", help="skip the 30-qubit QFT section")
    ap.add_argument("--config1-qubits", type=int, default=30)
    ap.add_argument("--learned-qubits", type=int, default=34)
    ap.add_argument("--learned-parts", type=int, default=20000, help="part timings harvested")
    return ap.parse_args()


# ---- distributed plumbing (replicas) ------------------------------------------

def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def dist_max(pg, x):
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ---- clocks --------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, nme in enumerate(names):
                if len(r) > 4 + i and r[4 + i].lower().startswith("active"):
                    reasons.add(nme)
        loaded = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


# ---- workload ------------------------------------------------------------------

def partitioner(args):
    from hisvsim_b200 import partition

    return {"frontier": partition.partition_frontier, "dfs": partition.partition_dfs,
            "acyclic": partition.partition_acyclic}[args.partitioner]


def plain_partitioner(args):
    """Parts for the plain form's part kernel.  With the frontier partitioner
    the limit counts only the targets of non-diagonal gates: the kernel's
    tile holds those, while CZ partners and controls act on index bits
    wherever they are (48 instead of 74 parts of 9 qubits at 33 qubits).
    The precision form and the reference's part path keep parts bounded by
    every qubit a gate touches (their unitaries / gathered states need them)."""
    from hisvsim_b200 import partition

    if args.partitioner == "frontier":
        return lambda gates, k: partition.partition_frontier(gates, k, free_diagonal=True)
    return partitioner(args)


def workload(n, layers, seed, k, split=None):
    from hisvsim_b200 import circuits, partition
    from hisvsim_b200.gates import part_offsets

    gates = circuits.random_u3_cz(n, layers, seed)
    parts = (split or partition.partition_acyclic)(gates, k)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    return gates, parts, rec, offs


def cpu_sample(args, threads, full_size=False):
    """The reference's own CPU path (oracle/_ref: its headers compiled here) on
    a bounded sample of the workload, through both of its live entry points on
    the same circuit and parts the GPU runs: per-gate BoundGate::apply
    (state_vector.hpp:1349) and the part path gather_and_execute_on_multi
    (execute.hpp:318-470) with opt_slots=1.  With full_size, also the
    per-gate path on a --cpu-full-qubits state (a few layers)."""
    from oracle.oracle import RefOracle

    from hisvsim_b200.gates import to_records

    n, layers = args.cpu_qubits, args.cpu_layers
    gates, parts, rec, offs = workload(n, layers, args.seed, min(args.part_qubits, n),
                                       partitioner(args))
    ref = RefOracle()
    upd = len(gates) * float(1 << n)
    t = time.perf_counter()
    ref.run(n, to_records(gates), mode=0, threads=threads)
    t_gate = time.perf_counter() - t
    t = time.perf_counter()
    ref.run(n, rec, offs, mode=1, opt_slots=1, threads=threads)
    t_part = time.perf_counter() - t
    # the baseline is the faster of the reference's two live paths
    faster = "parts" if t_part < t_gate else "per_gate"
    out = {"value": upd / min(t_gate, t_part), "unit": UNIT, "cores": threads,
           "kind": "reference",
           "sample": f"{n} qubits x {layers} layers of the same circuit family ({len(gates)} gates, "
                     f"{len(parts)} parts of <= {args.part_qubits} qubits), all host threads; "
                     f"value = the faster of the two live paths ({faster})",
           "seconds": min(t_gate, t_part), "path": faster,
           "per_gate": {"entry": "BoundGate::apply (state_vector.hpp:1349)", "seconds": t_gate,
                        "value": upd / t_gate},
           "parts": {"entry": "gather_and_execute_on_multi, opt_slots=1 (execute.hpp:318-470)",
                     "seconds": t_part, "value": upd / t_part, "parts": len(parts)}}
    if full_size:
        nf, lf = args.cpu_full_qubits, args.cpu_full_layers
        fg = workload(nf, lf, args.seed, min(args.part_qubits, nf), partitioner(args))[0]
        t = time.perf_counter()
        ref.run(nf, to_records(fg), mode=0, threads=threads)
        t_full = time.perf_counter() - t
        out["full_size"] = {"entry": "BoundGate::apply", "qubits": nf, "layers": lf,
                            "gates": len(fg), "seconds": t_full,
                            "value": len(fg) * float(1 << nf) / t_full,
                            "state_bytes": (1 << nf) * 16}
    return out


def run_reference_arm(args):
    # a CPU-only arm: rank 0 alone times the reference; other ranks exit at once
    if int(os.environ.get("RANK", "0")) != 0:
        return
    threads = os.cpu_count() or 1
    gate_vals, parts_vals = [], []
    r = None
    for i in range(args.warmup + args.steps):
        r = cpu_sample(args, threads)
        if i >= args.warmup:
            gate_vals.append(r["per_gate"]["value"])
            parts_vals.append(r["parts"]["value"])
    # the faster of the reference's two live paths, averaged over the steps
    g_mean, p_mean = statistics.mean(gate_vals), statistics.mean(parts_vals)
    v = max(g_mean, p_mean)
    faster = "gather_and_execute_on_multi" if p_mean > g_mean else "BoundGate::apply"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"random U3+CZ circuit, CPU sample {args.cpu_qubits}q x "
                                   f"{args.cpu_layers} layers (33q x 40 layers needs 128 GiB "
                                   f"and ~2 h of CPU per step)",
                       "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": r["sample"].split("; value")[0] +
                                       f"; value = {faster}, the faster of the reference's "
                                       "two live paths"},
            "per_gate_path": {"entry": r["per_gate"]["entry"], "value": g_mean, "unit": UNIT},
            "parts_path": {"entry": r["parts"]["entry"], "value": p_mean, "unit": UNIT},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def host_available_bytes() -> float:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return float(line.split()[1]) * 1024
    except OSError:
        pass
    return 0.0


def fidelity_small(args, abi, n):
    """1-F and max |d| of the precision form against a complex128 plain run of
    the same circuit family at n qubits, both on the device."""
    from hisvsim_b200 import partition
    from hisvsim_b200.gates import part_offsets

    gates, parts, rec, offs = workload(n, args.layers, args.seed, args.part_qubits,
                                       partitioner(args))
    fparts = partitioner(args)(gates, 6)
    frec, foffs = part_offsets(partition.parts_to_gates(gates, fparts))
    a = abi.State(n, abi.C64)
    a.set_basis(0)
    a.run_fused(frec, foffs, 0)
    b = abi.State(n, abi.C128)
    b.set_basis(0)
    b.run_parts(rec, offs)
    cm = a.compare(b)
    a.close()
    b.close()
    return {"qubits": n, "fidelity_loss": 1.0 - cm["fidelity"], "max_abs_err": cm["max_abs_diff"]}


def batch_form(args, abi, peak_gbs, pg, device):
    """Batching form: QAOA MaxCut instances (qubit counts uniform in 16..26,
    p = 4, seeded random 3-regular graphs, near-3-regular for odd counts) in one
    persistent launch per run, replayed as a CUDA graph after autotuning.  Each
    instance's <H_C> is compared with a complex128 plain run of its circuit."""
    import numpy as np

    from hisvsim_b200 import circuits, partition
    from hisvsim_b200.gates import part_offsets

    p = 4
    rng = np.random.default_rng(args.seed)
    ns = rng.integers(16, 27, args.batch_instances)
    insts = [circuits.qaoa_maxcut(int(n), p, args.seed * 1000 + i) for i, n in enumerate(ns)]
    b = abi.QaoaBatch([(int(n), e, g, bt) for n, (_, e, g, bt) in zip(ns, insts)], p)
    cap, ctas, tune_ms = b.tune()
    for _ in range(args.warmup):
        b.run()
    barrier(pg)
    ms = []
    with ClockSampler(device) as clk:
        for _ in range(args.steps):
            hc, t = b.run()
            ms.append(t)
    t_run = dist_max(pg, float(np.mean(ms)) / 1e3)
    st = b.stats()
    upd = sum((n + p * (len(e) + n)) * float(1 << int(n)) for n, (_, e, _, _) in zip(ns, insts))
    # complex128 plain runs of the same circuits: the <H_C> check, and the
    # time the same circuits take one after another through the plain form
    check = min(args.batch_check, len(insts))
    worst = 0.0
    t_plain = 0.0
    for i in range(check):
        n = int(ns[i])
        gates, edges = insts[i][0], insts[i][1]
        parts = partition.partition_acyclic(gates, 10)
        rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
        s = abi.State(n, abi.C128)
        s.set_basis(0)
        abi.synchronize()
        t0 = time.perf_counter()
        s.run_parts(rec, offs)
        zz = s.expect_zz(edges)
        t_plain += time.perf_counter() - t0
        want = float(np.sum((1.0 - zz) / 2.0))
        worst = max(worst, abs(hc[i] - want) / len(edges))
        s.close()
    caps = b.tile_caps()
    b.close()
    return {"instances": len(insts), "p": p, "qubits": "uniform 16..26",
            "run_ms": t_run * 1e3, "circuits_per_s": len(insts) / t_run,
            "value": upd / t_run, "unit": UNIT,
            "hbm_GBps": st["bytes_per_run"] / t_run / 1e9,
            "hbm_frac": st["bytes_per_run"] / t_run / 1e9 / peak_gbs,
            "bytes_per_run": st["bytes_per_run"], "work_items": st["items"],
            "tuned": {"tile_cap": cap, "ctas_per_sm": ctas, "best_ms": tune_ms,
                      "tiles_per_item": st["tiles_per_item"], "low_keep": st["low_keep"],
                      "threads_per_cta": st["threads"], "ctas_per_sm_used": st["ctas_per_sm"],
                      "caps_by_qubits": {int(n): int(c) for n, c in zip(ns, caps)}},
            "max_hc_err_per_edge": worst, "checked_instances": check,
            "plain_c128_sequential_s": t_plain,
            "dtype": "c64 states, fp64 <H_C>", "clocks": clk.summary()}


def learned_form(args, abi, pg, device):
    """Learned form: harvest part timings (complex64, random circuits of
    24-32 qubits), train the cost model with the library's K7 kernels, let it
    propose part sizes and cut points for a complex64 random circuit
    (``--learned-qubits`` qubits x 40 layers, U3 + CZ), and time that against
    the acyclic partitioner (the fallback) at its default and best part size."""
    import numpy as np

    from hisvsim_b200 import circuits, learned, partition

    weights = {24: 4000, 25: 3500, 26: 3000, 27: 2500, 28: 2500, 29: 1800, 30: 1400, 31: 800,
               32: 500}
    total_w = sum(weights.values())
    counts = {n: max(50, int(w * args.learned_parts / total_w)) for n, w in weights.items()}
    t0 = time.perf_counter()
    X, y, ns, _ = learned.harvest(counts, seed=args.seed)
    t_h = time.perf_counter() - t0
    rng = np.random.default_rng(args.seed)
    perm = rng.permutation(len(y))
    ntr = int(0.9 * len(y))
    model = learned.CostModel(seed=args.seed)
    t0 = time.perf_counter()
    losses = model.fit(X[perm[:ntr]], y[perm[:ntr]], epochs=150, batch=256, lr=2e-3)
    t_t = time.perf_counter() - t0
    te = perm[ntr:]
    rel = float(np.mean(np.abs(np.exp(model.predict_target(X[te]) - y[te]) - 1)))
    n = args.learned_qubits
    gates = circuits.random_u3_cz(n, 40, args.seed + 34)
    t0 = time.perf_counter()
    prop = learned.propose(gates, n, model)
    t_p = time.perf_counter() - t0
    st = abi.State(n, abi.C64)
    ks = [9] + [k for k in (7, 8, 10) if f"acyclic k={k}" in prop["candidates"]]
    res = {}
    with ClockSampler(device) as clk:
        t_learned = learned.measure(st, gates, prop["parts"], reps=1, warmup=0)
        for k in ks:
            res[k] = learned.measure(st, gates, partition.partition_acyclic(gates, k), reps=1,
                                     warmup=0)
        # the method without the network: the same DP with a trivial cost
        # (fewest parts), DFS-order and frontier parts at every size (best measured)
        fewest = learned.propose_fewest(gates, n)
        t_fewest = learned.measure(st, gates, fewest["parts"], reps=1, warmup=0)
        t_dfs = {k: learned.measure(st, gates, partition.partition_dfs(gates, k), reps=1, warmup=0)
                 for k in (8, 9, 10, 11, 12)}
        t_front = {k: learned.measure(st, gates, partition.partition_frontier(gates, k), reps=1,
                                      warmup=0)
                   for k in (8, 9, 10, 11, 12)}
    st.close()
    model.close()
    best_k = min(res, key=res.get)
    best_dfs = min(t_dfs, key=t_dfs.get)
    best_front = min(t_front, key=t_front.get)
    nonlearned = {"dp_fewest_parts_s": t_fewest, "dfs_s": {str(k): v for k, v in t_dfs.items()},
                  "best_dfs_k": best_dfs,
                  "frontier_s": {str(k): v for k, v in t_front.items()},
                  "best_frontier_k": best_front, f"acyclic_best_k{best_k}_s": res[best_k]}
    best_nonlearned = min(t_fewest, t_dfs[best_dfs], t_front[best_front], res[best_k])
    return {"harvest_parts": int(len(y)), "harvest_qubits": "24..32", "harvest_s": t_h,
            "train_s": t_t, "final_train_mse": float(losses[-1]), "holdout_mean_rel_err": rel,
            "eval": f"random U3+CZ circuit {n} qubits x 40 layers, complex64",
            "proposal": prop["method"], "proposal_parts": len(prop["parts"]),
            "propose_s": t_p, "learned_s": t_learned,
            "acyclic_s": {str(k): v for k, v in res.items()},
            "gain_vs_acyclic_k9": res[9] / t_learned,
            "gain_vs_best_acyclic": res[best_k] / t_learned, "best_acyclic_k": best_k,
            "nonlearned": nonlearned,
            "gain_vs_best_nonlearned": best_nonlearned / t_learned,
            "clocks": clk.summary()}


def config1_form(args, abi, peak_gbs, pg, device):
    """Config 1: the 30-qubit QFT (H, controlled phases 2 pi / 2^m on every
    pair, final swaps) on a seeded random basis state, complex128, frontier
    parts of <= 7 qubits: circuit time, passes and the K1 pass roofline.  And
    the choice the plain path makes for parts on high qubits: a part whose
    qubits are the top ones runs on strided tiles in one pass; the
    alternative, a K2 bit-swap pass that brings those qubits to the low
    slots followed by the part on contiguous tiles, is timed beside it."""
    import numpy as np

    from hisvsim_b200 import circuits, partition
    from hisvsim_b200.gates import Gate, part_offsets, to_records

    n = args.config1_qubits
    gates, x = circuits.qft(n, args.seed)
    parts = partition.partition_frontier(gates, 7, free_diagonal=True)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st = abi.State(n, abi.C128)

    def step():
        st.set_basis(x)
        st.run_parts(rec, offs)

    t, c, clk = timed_steps(abi, step, max(1, args.warmup), max(1, args.steps), pg, device)
    passes = c["passes"] / max(1, args.steps)
    k1_ms = c["apply_us"] / 1e3 / max(1, c["passes"])
    bpp = 2.0 * (1 << n) * 16
    # a 7-qubit part of dense gates on the top qubits vs the same part on the
    # lowest qubits after a bit-swap pass
    rng = np.random.default_rng(7)
    def part_on(qs):
        g = []
        for _ in range(2):
            for q in qs:
                g.append(Gate("U3", (q,), params=tuple(rng.uniform(0, 2 * np.pi, 3))))
            for a, b in zip(qs[::2], qs[1::2]):
                g.append(Gate("Z", (b,), (a,)))
        return to_records(g)
    hi = list(range(n - 7, n))
    lo = list(range(2, 9))
    r_hi, r_lo = part_on(hi), part_on(lo)
    def dev_ms(fn, reps=5):
        fn()
        abi.synchronize()
        a, b = abi.Event(), abi.Event()
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        return a.elapsed_ms(b) / reps
    ms_hi = dev_ms(lambda: st.run_part(r_hi))
    ms_lo = dev_ms(lambda: st.run_part(r_lo))
    pairs = [(hi[i], lo[i]) for i in range(7)]
    ms_swap = dev_ms(lambda: st.permute_bits(pairs[:5]), reps=4)
    st.close()
    return {"workload": f"QFT {n} qubits on a random basis state, {len(gates)} gates, "
                        f"{len(parts)} frontier parts of <= 7 non-diagonal target qubits, "
                        f"complex128",
            "circuit_s": t, "passes_per_step": passes, "value": len(gates) * float(1 << n) / t,
            "unit": UNIT,
            "roofline": {"bound": "hbm", "kernel": "k1_part", "avg_launch_ms": k1_ms,
                         "achieved": bpp / (k1_ms / 1e3) / 1e9, "peak": peak_gbs, "unit": "GB/s",
                         "frac": bpp / (k1_ms / 1e3) / 1e9 / peak_gbs},
            "high_qubit_parts": {"part_on_top_qubits_ms": ms_hi, "part_on_low_qubits_ms": ms_lo,
                                 "bitswap_pass_5_pairs_ms": ms_swap,
                                 "strided_tile_wins_by_ms": ms_lo + ms_swap - ms_hi},
            "clocks": clk}


def timed_steps(abi, step, warmup, steps, pg, device):
    """W untimed steps, then K steps between events on the library stream."""
    for _ in range(warmup):
        step()
    abi.synchronize()
    abi.counters_reset()
    abi.set_timing(True)
    barrier(pg)
    start, stop = abi.Event(), abi.Event()
    with ClockSampler(device) as clk:
        abi.synchronize()
        start.record()
        for _ in range(steps):
            step()
        stop.record()
        ms = start.elapsed_ms(stop)
    abi.set_timing(False)
    c = abi.counters()
    return dist_max(pg, ms / 1e3 / steps), c, clk.summary()


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    rank, world, local, pg = dist_setup(args.gpus)
    import numpy as np

    from hisvsim_b200 import abi, partition
    from hisvsim_b200.gates import part_offsets

    abi.set_device(local)
    if args.tile_qubits:
        abi.set_tile_qubits(args.tile_qubits)
    n = args.qubits
    gates, parts, rec, offs = workload(n, args.layers, args.seed + rank, args.part_qubits,
                                       plain_partitioner(args))
    upd = len(gates) * float(1 << n)
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak_gbs, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak_gbs, peak_src = 6650.0, "fallback"

    # ---- precision form: complex64 state, one 64x64 unitary per part of <= 6
    # qubits, split-BF16 tensor-core GEMMs (timed first; its result is kept in
    # host memory for the fidelity check against the complex128 run)
    fused = None
    fused_host = None
    if not args.no_fused:
        if args.fused_shape:
            abi.set_fused_shape(*[int(x) for x in args.fused_shape.split(",")])
        fparts = partitioner(args)(gates, 6)
        frec, foffs = part_offsets(partition.parts_to_gates(gates, fparts))
        stf = abi.State(n, abi.C64)

        def fstep():
            stf.set_basis(0)
            stf.run_fused(frec, foffs, 0)

        t_f, cf, clk_f = timed_steps(abi, fstep, args.warmup, args.steps, pg, local)
        fpasses = cf["passes"] / args.steps
        fbytes = 2.0 * (1 << n) * 8
        k4_ms = cf["apply_us"] / 1e3 / max(1, cf["passes"])
        shape = abi.set_fused_shape(1, 13)
        abi.set_fused_shape(shape // 100, shape % 100)
        variant = abi.set_k4_variant(2)
        abi.set_k4_variant(variant)
        kname = ({0: "k4_direct", 1: "k4_ws", 2: "k4_bulk"}[variant] if shape // 100 == 1
                 else "k4_fused")
        # tensor work: three BF16 products of a 128 x 128 real GEMM per amplitude column
        tflops = 3 * 8.0 * 64 * (1 << n) * fpasses / t_f / 1e12
        fused = {"circuit_s": t_f, "parts": len(fparts), "passes_per_step": fpasses,
                 "shape": {"unitaries_per_pass": shape // 100, "tile_bits": shape % 100},
                 "value": world * upd / t_f, "unit": UNIT,
                 "hbm_GBps": fpasses * fbytes / t_f / 1e9,
                 "roofline": {"bound": "hbm", "kernel": kname, "avg_launch_ms": k4_ms,
                              "achieved": fbytes / (k4_ms / 1e3) / 1e9 if k4_ms else None,
                              "peak": peak_gbs, "unit": "GB/s",
                              "frac": fbytes / (k4_ms / 1e3) / 1e9 / peak_gbs if k4_ms else None,
                              "tensor_tflops": tflops},
                 "dtype": "c64 state, bf16x3 split operands, fp32 accumulate, fp64 unitaries",
                 "clocks": clk_f}
        if rank == 0 and not args.no_fidelity:
            # the full-size check stages the complex64 result in host memory
            # (2^n x 8 bytes) while the complex128 run holds the device
            need = (1 << n) * 8 * 1.25
            if host_available_bytes() > need:
                fused_host = stf.raw()
            else:
                fused["fidelity_full_size"] = (f"skipped: {host_available_bytes() / 2**30:.0f} GiB "
                                               f"of host memory available, {need / 2**30:.0f} "
                                               f"GiB needed")
            fused["fidelity_28q"] = fidelity_small(args, abi, min(n, 28))
        stf.close()
        del stf

    # ---- plain form (the drop-in): complex128, K1 passes
    st = abi.State(n, abi.C128)

    def step():
        st.set_basis(0)
        st.run_parts(rec, offs)

    t_step, c, clk = timed_steps(abi, step, args.warmup, args.steps, pg, local)
    pbytes = abi.launch_bytes()
    # the same circuit in parts bounded by every qubit a gate touches (the
    # reference's part semantics): more, lighter passes
    alt = None
    if args.partitioner == "frontier":
        g_b, p_b, rec_b, offs_b = workload(n, args.layers, args.seed + rank, args.part_qubits,
                                           partition.partition_frontier)

        def step_b():
            st.set_basis(0)
            st.run_parts(rec_b, offs_b)

        t_b, c_b, _ = timed_steps(abi, step_b, 1, 1, pg, local)
        ms_b = c_b["apply_us"] / 1e3 / max(1, c_b["passes"])
        alt = {"partition": f"frontier, <= {args.part_qubits} qubits touched per part",
               "parts": len(p_b), "circuit_s": t_b, "value": world * upd / t_b,
               "passes_per_step": c_b["passes"], "avg_launch_ms": ms_b,
               "k1_frac": 2.0 * (1 << n) * 16 / (ms_b / 1e3) / 1e9 / peak_gbs}
    passes = c["passes"] / args.steps
    k1_avg_ms = c["apply_us"] / 1e3 / max(1, c["passes"])
    bytes_per_pass = 2.0 * (1 << n) * 16
    norm = st.norm2()
    k1_gbs = bytes_per_pass / (k1_avg_ms / 1e3) / 1e9
    if fused is not None:
        fused["speedup_vs_plain"] = t_step / fused["circuit_s"]
        if fused_host is not None:
            cmpd = st.compare_host(fused_host)
            fused["fidelity_loss"] = 1.0 - cmpd["fidelity"]
            fused["max_abs_err"] = cmpd["max_abs_diff"]
            fused["fidelity_ref"] = f"complex128 plain run of the same {n}-qubit circuit"
            del fused_host
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "k1_traffic.json")))
        traffic = tr.get("bytes_per_launch_scaled")
    except Exception:
        pass
    # FP64 work of the plain pass: every U3 runs as a rotation, per amplitude
    # pair 3 FMA for the phase of the pair's second amplitude and 2 x 2 real
    # shears for RY when |cos(theta/2)| >= 0.4 (the planner's two-shear form,
    # its scale carried in the frames), else 2 x 3; the CZ sign flips take none
    fma_pair = sum(3 + (4 if abs(math.cos(complex(g.params[0]).real / 2)) >= 0.4 else 6)
                   for g in gates if g.name == "U3")
    dense = sum(1 for g in gates if g.name == "U3")
    fma_step = fma_pair * 0.5 * float(1 << n)
    fp64_peak = abi.fp64_peak_tflops()
    k1_total_s = c["apply_us"] / 1e6 / args.steps
    fp64 = {"fma_per_step": fma_step, "achieved_tflops": 2 * fma_step / k1_total_s / 1e12,
            "peak_tflops": fp64_peak, "source": "hs_fp64_peak (measured FP64 FMA probe)",
            "frac": 2 * fma_step / k1_total_s / 1e12 / fp64_peak}
    # K2: one in-place bit-swap pass over the same state (the redistribution
    # kernel), timed by CUDA events; half the amplitudes move
    k2 = None
    try:
        pairs = [(0, n - 1), (1, n - 2), (2, n - 3)]
        st.permute_bits(pairs)
        abi.synchronize()
        a, b = abi.Event(), abi.Event()
        a.record()
        for _ in range(3):
            st.permute_bits(pairs)
        b.record()
        abi.synchronize()
        k2_ms = a.elapsed_ms(b) / 3
        moved = (1 << n) * 16 * (1 - 0.5 ** len(pairs))  # amplitudes whose index changes
        k2 = {"kernel": "k2_bitswap", "pairs": len(pairs), "avg_launch_ms": k2_ms,
              "algorithmic_bytes_per_launch": 2 * moved,
              "achieved_GBps": 2 * moved / (k2_ms / 1e3) / 1e9,
              "frac": 2 * moved / (k2_ms / 1e3) / 1e9 / peak_gbs}
    except Exception as ex:  # keep the headline if the extra measurement fails
        k2 = {"error": str(ex)}
    st.close()
    del st

    # end to end through the public API (pybind module): allocate, run every
    # part from host gate lists, read back the norm
    e2e = None
    if not args.no_e2e:
        from hisvsim_b200 import svsimulator_py_wrapper as svsim
        from hisvsim_b200.gates import NOPARAM

        def bound(g):
            if g.name in NOPARAM:
                ag = svsim.AggregateGate_0(g.name)
            else:
                ag = svsim.AggregateGate_3(g.name, *g.params)
            return svsim.BoundGate(svsim.AggregateGateFactory(ag), list(g.controls),
                                   list(g.targets))

        lists = [[bound(gates[i]) for i in p] for p in parts]
        e2e_steps = max(1, min(args.steps, 2))
        abi.counters_reset()
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            sim = svsim.StateVector(n, 0)
            for bl in lists:
                svsim.gather_and_execute_on(sim, bl)
            _ = sim.norm()
            del sim
        t_e2e = dist_max(pg, (time.perf_counter() - t0) / e2e_steps)
        e2e = {"value": world * upd / t_e2e, "unit": UNIT,
               "h2d_bytes_per_step": abi.launch_bytes() // e2e_steps,
               "d2h_bytes_per_step": 16, "circuit_s": t_e2e,
               "path": "svsimulator_py_wrapper: StateVector -> gather_and_execute_on per part "
                       "-> norm readback (gate programs travel as kernel parameters; the "
                       "initial state |0..0> is created on the device, as StateVector does)"}

    config1 = None
    if not args.no_config1:
        config1 = config1_form(args, abi, peak_gbs, pg, local)

    batch = None
    if not args.no_batch:
        batch = batch_form(args, abi, peak_gbs, pg, local)

    learned_res = None
    if not args.no_learned and rank == 0:
        learned_res = learned_form(args, abi, pg, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_sample(args, os.cpu_count() or 1,
                             full_size=host_available_bytes() > (1 << args.cpu_full_qubits) * 16 * 1.5)
        except Exception as ex:  # the oracle library may be missing
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                   "sample": f"unavailable: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": world * upd / t_step, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic",
            "config": {"workload": f"random circuit {n} qubits x {args.layers} layers "
                                   f"(U3 all qubits + CZ random matching), plain complex128",
                       "gates": len(gates), "parts": len(parts),
                       "part_qubits": args.part_qubits,
                       "partitioner": args.partitioner + (
                           " (limit on non-diagonal targets)" if args.partitioner == "frontier"
                           else ""),
                       "tile_qubits": args.tile_qubits or "automatic (2^10 tiles, 16 amplitudes "
                                                          "per thread for complex128)",
                       "passes_per_step": passes, "state_bytes": (1 << n) * 16,
                       "l2": "state >> L2 (126 MB), no flush", "parallelism": f"replicas{world}"},
            "circuit_s": t_step, "hbm_GBps": passes * bytes_per_pass / t_step / 1e9,
            "hbm_frac": passes * bytes_per_pass / t_step / 1e9 / peak_gbs,
            "norm": norm,
            "roofline": {"bound": "hbm", "achieved": k1_gbs, "peak": peak_gbs, "unit": "GB/s",
                         "frac": k1_gbs / peak_gbs, "traffic": traffic, "peak_source": peak_src,
                         "kernel": "k1_part", "algorithmic_bytes_per_launch": bytes_per_pass,
                         "avg_launch_ms": k1_avg_ms, "fp64": fp64},
            "qubit_bounded_parts": alt,
            "fused": fused,
            "redistribution": k2,
            "config1": config1,
            "batch": batch,
            "learned": learned_res,
            "gpu_launches": int(c["passes"] + args.steps),
            "launch_param_bytes_per_step": pbytes / args.steps,
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
