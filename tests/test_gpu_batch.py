"""Batching form (K6, hs_batch_*): many QAOA MaxCut instances of different
qubit counts in one persistent launch under a CUDA graph.

Every instance is checked against a complex128 run of the same circuit
(H on every qubit, then per round RZZ(gamma) on each edge and RX(2 beta) on
each qubit) through the plain form: amplitudes to 1e-5 (complex64 states) and
<H_C> = sum_E (1 - <Z_a Z_b>)/2 to 1e-5 relative to |E|."""
import numpy as np
import pytest

from hisvsim_b200 import abi, circuits, partition
from hisvsim_b200.gates import part_offsets

pytestmark = pytest.mark.gpu
AMP_TOL = 1e-5
HC_TOL = 1e-5


def make_instances(ns, p, seed):
    out = []
    for i, n in enumerate(ns):
        gates, edges, gammas, betas = circuits.qaoa_maxcut(n, p, seed + i)
        out.append((n, edges, gammas, betas, gates))
    return out


def plain_c128(n, gates):
    st = abi.State(n, abi.C128)
    st.set_basis(0)
    parts = partition.partition_acyclic(gates, min(n, 10))
    rec, offs = part_offsets(partition.parts_to_gates(gates, parts))
    st.run_parts(rec, offs)
    return st


def hc_c128(st, edges):
    zz = st.expect_zz(edges)
    return float(np.sum((1.0 - zz) / 2.0))


def check_batch(batch, insts, states=True):
    hc, _ = batch.run()
    for i, (n, edges, _, _, gates) in enumerate(insts):
        ref = plain_c128(n, gates)
        want = hc_c128(ref, edges)
        assert abs(hc[i] - want) <= HC_TOL * len(edges), (i, n, hc[i], want)
        if states:
            got = batch.state(i)
            assert np.abs(got - ref.amplitudes()).max() <= AMP_TOL, (i, n)
    return hc


@pytest.mark.parametrize("cap", [9, 10, 11, 12])
def test_states_and_cost_vs_plain(cap):
    insts = make_instances([6, 7, 9, 12, 14, 16, 17, 21], 3, 500)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 3)
    b.configure(cap, 4)
    check_batch(b, insts)
    b.close()


@pytest.mark.parametrize("ctas", [1, 2, 6, 8])
def test_cta_schedules_agree(ctas):
    insts = make_instances([16, 18, 20, 22], 4, 900)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 4)
    b.configure(12, 4)
    assert b.stats()["threads"] == 256
    base, _ = b.run()
    b.configure(10, ctas)
    b.set_chunk(3)
    b.set_low_keep(2)
    again, _ = b.run()
    assert np.abs(base - again).max() <= 1e-4
    b.close()


def test_replay_is_deterministic_and_params_update():
    insts = make_instances([10, 13, 16, 19], 2, 77)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 2)
    first, _ = b.run()
    second, _ = b.run()
    assert np.array_equal(first, second)
    # a new sweep point through hs_batch_set_params (the captured graph is reused)
    rng = np.random.default_rng(5)
    gam = rng.uniform(0, np.pi, (len(insts), 2))
    bet = rng.uniform(0, np.pi / 2, (len(insts), 2))
    b.set_params(gam, bet)
    hc, _ = b.run()
    for i, (n, edges, _, _, _) in enumerate(insts):
        gates = [g for g in circuits.qaoa_maxcut(n, 2, 77 + i)[0][:n]]
        for r in range(2):
            for a, c in edges:
                gates.append(circuits.Gate("RZZ", (a, c), params=(gam[i, r],)))
            for q in range(n):
                gates.append(circuits.Gate("RX", (q,), params=(2 * bet[i, r],)))
        want = hc_c128(plain_c128(n, gates), edges)
        assert abs(hc[i] - want) <= HC_TOL * len(edges)
    b.close()


def test_tuner_and_mixed_sizes():
    ns = list(range(16, 27)) * 2
    insts = make_instances(ns, 4, 1234)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 4)
    cap, ctas, ms = b.tune()
    assert cap in (9, 10, 11, 12) and 1 <= ctas <= 16 and ms > 0
    caps = b.tile_caps()
    assert set(caps.tolist()) <= {9, 10, 11, 12}
    st = b.stats()
    assert st["items"] > 0 and st["bytes_per_run"] > 0
    check_batch(b, insts, states=False)
    b.close()


def hc_from_amplitudes(n, amps, edges):
    """<H_C> = sum_E (1 - <Z_a Z_b>)/2 from qubit-ordered amplitudes (FP64)."""
    p = np.abs(np.asarray(amps, dtype=np.complex128)) ** 2
    idx = np.arange(1 << n, dtype=np.int64)
    total = 0.0
    for a, b in edges:
        parity = ((idx >> a) ^ (idx >> b)) & 1
        zz = float(np.sum(p * (1 - 2 * parity)))
        total += (1.0 - zz) / 2.0
    return total


def test_batch_against_reference_oracle(ref):
    """K6 pinned to the reference itself: the same QAOA gate list (H on every
    qubit, then per round RZZ(gamma) on each edge and RX(2 beta) on each qubit,
    basic_gates.hpp:341-363,1235-1313) run through the reference's own
    BoundGate::apply (RefOracle), for instances of <= 16 qubits; amplitudes to
    1e-5 and <H_C> to 1e-5 per edge, with no plain-form run in between."""
    from hisvsim_b200.gates import to_records

    insts = make_instances([8, 11, 12, 15, 16, 13], 4, 9100)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 4)
    hc, _ = b.run()
    for i, (n, edges, _, _, gates) in enumerate(insts):
        want = ref.run(n, to_records(gates), mode=0)
        got = b.state(i)
        assert np.abs(got - want).max() <= AMP_TOL, (i, n)
        hw = hc_from_amplitudes(n, want, edges)
        assert abs(hc[i] - hw) <= HC_TOL * len(edges), (i, n, hc[i], hw)
    b.close()


def test_dependency_wait_timeout_is_reported_and_recovers():
    """Failure detection without a GPU fault: one step's dependency wait is
    made unreachable from the host and the poll limit shortened, so the
    persistent launch gives up, ends and reports HS_E_TIMEOUT; with the step
    restored, the next run of the same captured graph returns the same
    <H_C> as before."""
    insts = make_instances([10, 12, 14, 16], 3, 777)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 3)
    b.configure(10, 4)
    good, _ = b.run()
    b.set_wait_limit(2000)  # ~0.2 ms of polls
    b.block_step(2, 1)
    with pytest.raises(abi.HisvError) as e:
        b.run()
    assert e.value.code == abi.HS_E_TIMEOUT
    b.block_step(2, 1, block=False)
    b.set_wait_limit(1 << 24)
    again, _ = b.run()
    assert np.array_equal(good, again)
    for i, (n, edges, _, _, gates) in enumerate(insts):
        want = hc_c128(plain_c128(n, gates), edges)
        assert abs(again[i] - want) <= HC_TOL * len(edges)
    b.close()


def test_wait_hooks_reject_bad_arguments():
    insts = make_instances([8, 9], 2, 5)
    b = abi.QaoaBatch([(n, e, g, bt) for n, e, g, bt, _ in insts], 2)
    with pytest.raises(abi.HisvError):
        b.set_wait_limit(0)
    with pytest.raises(abi.HisvError):
        b.block_step(0, 0)  # the first step waits for nothing
    with pytest.raises(abi.HisvError):
        b.block_step(5, 1)  # no such instance
    b.close()
