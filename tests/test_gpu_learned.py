"""Learned form on the GPU: the K7 network kernels against the numpy oracle
(oracle/mlp.py), the timing harvest, and the proposer against the acyclic
partitioner it falls back to, compared by measured device time.

Tolerances: FP32 kernels against the float64 oracle, forward 1e-4 relative,
gradients 1e-4 of the largest gradient component."""
import numpy as np
import pytest

from hisvsim_b200 import abi, circuits, learned, partition
from hisvsim_b200.gates import part_offsets

pytestmark = pytest.mark.gpu


def _data(n, d, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, d)).astype(np.float32)
    y = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2 % d]).astype(np.float32)
    return x, y


@pytest.mark.parametrize("d,n", [(43, 1), (43, 63), (43, 1000), (5, 200), (64, 130)])
def test_forward_matches_oracle(d, n):
    from oracle import mlp

    m = abi.Mlp(d, seed=11)
    x, _ = _data(n, d, 1)
    got = m.predict(x)
    want, _ = mlp.forward(m.params().astype(np.float64), x)
    assert np.abs(got - want).max() <= 1e-4 * max(1.0, np.abs(want).max())
    m.close()


@pytest.mark.parametrize("d,n", [(43, 1), (43, 64), (43, 777), (43, 20000), (9, 300)])
def test_gradients_match_oracle(d, n):
    from oracle import mlp

    m = abi.Mlp(d, seed=5)
    x, y = _data(n, d, 2)
    loss, g = m.gradients(x, y)
    wl, wg = mlp.loss_and_grad(m.params().astype(np.float64), x, y)
    assert loss == pytest.approx(wl, rel=1e-4)
    assert np.abs(g - wg).max() <= 1e-4 * np.abs(wg).max()
    m.close()


def test_adam_step_matches_oracle():
    from oracle import mlp

    d, n = 43, 200
    m = abi.Mlp(d, seed=9)
    x, y = _data(n, d, 3)
    p0 = m.params().astype(np.float64)
    _, g = mlp.loss_and_grad(p0, x, y)
    m.train(x, y, epochs=1, batch=n, lr=1e-3, seed=1)  # one minibatch = one Adam step
    want = mlp.adam_step(p0.copy(), g, np.zeros_like(p0), np.zeros_like(p0), 1, 1e-3)
    assert np.abs(m.params() - want).max() <= 2e-6
    m.close()


def test_training_fits_a_smooth_target_and_is_deterministic():
    d = 43
    x, y = _data(4000, d, 4)
    a = abi.Mlp(d, seed=1)
    la = a.train(x, y, epochs=40, batch=128, lr=2e-3, seed=7)
    assert la[-1] < 0.1 * la[0]
    b = abi.Mlp(d, seed=1)
    lb = b.train(x, y, epochs=40, batch=128, lr=2e-3, seed=7)
    assert np.array_equal(a.params(), b.params()) and np.array_equal(la, lb)
    a.close()
    b.close()


def test_timed_parts_run_matches_plain_run():
    n = 16
    gates = circuits.random_u3_cz(n, 8, 3)
    parts = partition.partition_acyclic(gates, 7)
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    a = abi.State(n, abi.C64)
    a.set_basis(0)
    ms = a.run_parts_timed(rec, offs)
    b = abi.State(n, abi.C64)
    b.set_basis(0)
    b.run_parts(rec, offs)
    assert len(ms) == len(parts) and (ms > 0).all()
    assert np.array_equal(a.amplitudes(), b.amplitudes())


def test_harvest_features_and_targets():
    X, y, ns, ms = learned.harvest({18: 120, 20: 80}, seed=2, layers=10, chunk=64)
    assert X.shape == (len(y), abi.num_part_features()) and len(y) >= 190
    assert np.isfinite(y).all() and (ms > 0).all()
    assert set(np.unique(ns).tolist()) == {18, 20}


def test_learned_proposal_beats_acyclic_partitioner():
    """The method with the network against the method without it, compared by
    measured device time: a 27-qubit complex64 random circuit (40 layers of
    U3 + CZ), the proposal against the acyclic partitioner at its default
    part size (9, the fallback) and at the best size the network finds."""
    X, y, _, _ = learned.harvest({23: 500, 24: 500, 25: 500, 26: 500, 27: 500}, seed=3,
                                 layers=20)
    model = learned.CostModel(seed=1)
    losses = model.fit(X, y, epochs=150, batch=256, lr=2e-3)
    assert losses[-1] < 0.05 * losses[0]
    n = 27
    gates = circuits.random_u3_cz(n, 40, 2027)
    prop = learned.propose(gates, n, model)
    assert partition.is_valid_partition(gates, prop["parts"])
    st = abi.State(n, abi.C64)
    t_learned = learned.measure(st, gates, prop["parts"], reps=3)
    t_default = learned.measure(st, gates, partition.partition_acyclic(gates, 9), reps=3)
    acyc = {int(k.split("=")[1]): v for k, v in prop["candidates"].items()
            if k.startswith("acyclic")}
    best_k = min(acyc, key=acyc.get)  # the best part size the network predicts
    t_best = learned.measure(st, gates, partition.partition_acyclic(gates, best_k), reps=3)
    st.close()
    # the same state through both partitions: identical results
    a = abi.State(n, abi.C64)
    learned.measure(a, gates, prop["parts"], reps=1, warmup=0)
    b = abi.State(n, abi.C64)
    learned.measure(b, gates, partition.partition_acyclic(gates, 9), reps=1, warmup=0)
    assert abs(a.inner(b)) ** 2 >= 1 - 1e-5
    assert t_learned < 0.97 * t_default, (t_learned, t_default)
    assert t_learned < t_best, (t_learned, t_best, best_k)
    # what the network adds beyond the method without it: the same dynamic
    # program with a trivial cost (fewest parts), and DFS-order and frontier
    # parts at the best part size found by measuring every size
    st = abi.State(n, abi.C64)
    t_fewest = learned.measure(st, gates, learned.propose_fewest(gates, n)["parts"], reps=3)
    t_dfs = {k: learned.measure(st, gates, partition.partition_dfs(gates, k), reps=2)
             for k in (8, 9, 10, 11, 12)}
    t_front = {k: learned.measure(st, gates, partition.partition_frontier(gates, k), reps=2)
               for k in (8, 9, 10, 11, 12)}
    st.close()
    assert t_learned < t_fewest, (t_learned, t_fewest)
    assert t_learned <= 1.02 * min(t_dfs.values()), (t_learned, t_dfs)
    # the frontier partitioner already finds near-fewest parts: the proposal
    # (which prices frontier parts of every size and segments of the
    # frontier order too) stays within the cost model's error (a few
    # percent) of its best size measured
    assert t_learned <= 1.05 * min(t_front.values()), (t_learned, t_front)
