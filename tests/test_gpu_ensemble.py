"""Replica ensembles: every replica advanced in one batched ensemble is
bit-identical to the same system advanced alone in its own handle (same
kernels, same row order, same per-replica rebuild schedule); replicas too
small for 3 cells per axis (all-pairs search) follow the CPU oracle."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W
from oracle import lj_oracle as O

pytestmark = pytest.mark.gpu


def replicas():
    return [
        W.fcc_liquid(6, 0.5, 1.0, seed=61, jitter=0.08, rc=2.5, dt=0.005),
        W.fcc_liquid((5, 5, 6), 0.7, 0.8, seed=62, jitter=0.05, rc=2.5, dt=0.005),
        W.fcc_liquid(7, 0.8442, 0.722, seed=63, jitter=0.05, rc=2.5, dt=0.005),
        W.fcc_liquid(4, 0.3, 1.2, seed=64, jitter=0.05, rc=2.5, dt=0.005),
    ]


@pytest.mark.parametrize("precision", [M.FP64, M.FP32_MIXED])
def test_ensemble_bit_identical_to_single(precision):
    reps = replicas()
    ens = M.Ensemble([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005, precision=precision)
    ens.calculate(60)
    got = ens.states_by_id()
    rb, steps = ens.rebuilds()
    for k, r in enumerate(reps):
        s = M.System(r.L, cutoff=2.5, time_step=0.005, capacity=r.n, precision=precision)
        s.set_state(r.q, r.v)
        s.calculate(60)
        q, v = s.state_by_id()
        assert np.array_equal(got[k][0], q), f"replica {k} positions"
        assert np.array_equal(got[k][1], v), f"replica {k} velocities"
        assert rb[k] == s.info()["rebuilds"] and steps[k] == 60
        s.close()
    ke, pe, vir = ens.observe()
    for k, r in enumerate(reps):
        s = M.System(r.L, cutoff=2.5, time_step=0.005, capacity=r.n, precision=precision)
        s.set_state(got[k][0], got[k][1])
        k1, p1, v1 = s.observe()
        assert ke[k] == pytest.approx(k1, rel=1e-12)
        assert pe[k] == pytest.approx(p1, rel=1e-12)
        assert vir[k] == pytest.approx(v1, rel=1e-12)
        s.close()


def test_per_replica_margins_match_single_systems_with_that_margin():
    # each replica's own BufferLength (0 = the common 0.3): its search
    # length, cell grid, skin budget and rebuild schedule are those of a
    # single handle made with that buffer length, bit for bit
    reps = replicas()
    margins = [0.75, 0.2, 0.5, 0.0]  # every replica keeps three or more cells per axis
    ens = M.Ensemble([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005, precision=M.FP32_MIXED,
                     buffer_lengths=margins)
    ens.calculate(80)
    got = ens.states_by_id()
    rb, _ = ens.rebuilds()
    for k, r in enumerate(reps):
        s = M.System(r.L, cutoff=2.5, time_step=0.005, capacity=r.n, precision=M.FP32_MIXED,
                     buffer_length=margins[k] or 0.3)
        s.set_state(r.q, r.v)
        s.calculate(80)
        q, v = s.state_by_id()
        assert np.array_equal(got[k][0], q), f"replica {k} positions"
        assert np.array_equal(got[k][1], v), f"replica {k} velocities"
        assert rb[k] == s.info()["rebuilds"], f"replica {k} rebuilds"
        s.close()
    ens.close()
    # a margin is checked against the replica's own box
    with pytest.raises(M.MdgError) as e:
        M.Ensemble([(reps[3].q, reps[3].v, reps[3].L)], cutoff=2.5, buffer_lengths=[reps[3].L[0] / 2.0])
    assert e.value.status == -7
    with pytest.raises(M.MdgError):
        M.Ensemble([(reps[0].q, reps[0].v, reps[0].L)], cutoff=2.5, buffer_lengths=[-0.1])


def test_margin_tuner_runs_and_keeps_the_fastest_trial():
    reps = replicas()
    margins, report = M.margins.tune_margins([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005,
                                              warm_steps=20, trial_steps=40, costs=(6.0,))
    assert len(margins) == len(reps) and np.all(margins >= 0.1)
    times = [t["ms_per_step"] for t in report["trials"]]
    assert len(times) == 2 and report["chosen_ms_per_step"] == min(times)


def test_small_replica_all_pairs_matches_oracle():
    # 500 atoms at rho 0.9: L = 8.22 < 3 x 2.8, two cells per axis
    small = W.fcc_liquid(5, 0.9, 1.0, seed=65, jitter=0.05, rc=2.5, dt=0.005)
    big = W.fcc_liquid(6, 0.5, 1.0, seed=66, jitter=0.05, rc=2.5, dt=0.005)
    ens = M.Ensemble([(small.q, small.v, small.L), (big.q, big.v, big.L)], cutoff=2.5, time_step=0.005)
    ens.calculate(40)
    q, v = ens.states_by_id()[0]
    o = O.Oracle(small.q, small.v, small.ids, small.L, 2.5, 0.005)
    o.make_pairlist()
    o.step(40)
    oq, ov, oid = o.state()
    qo = np.empty_like(oq)
    vo = np.empty_like(ov)
    qo[oid] = oq
    vo[oid] = ov
    dq = q - qo
    dq -= small.L * np.round(dq / small.L)
    assert np.abs(dq).max() < 1e-9
    assert np.abs(v - vo).max() < 1e-9
    rb, _ = ens.rebuilds()
    assert rb[0] == o.constructions


def test_ensemble_rejects_box_below_two_search_lengths():
    r = W.fcc_liquid(3, 0.9, 1.0, seed=67, rc=2.5)  # L = 4.9 < 5.6
    with pytest.raises(M.MdgError) as e:
        M.Ensemble([(r.q, r.v, r.L)], cutoff=2.5)
    assert e.value.status == -7


def _pairs_within_cutoff(q, L, rc):
    d = q[:, None, :] - q[None, :, :]
    d -= L * np.round(d / L)
    r2 = (d * d).sum(-1)
    iu = np.triu_indices(q.shape[0], 1)
    return int((r2[iu] <= rc * rc).sum())


def test_list_stats_and_kernel_counters():
    # list entries: the sum of the single handles' lists after the same
    # steps (the rebuild schedules are the same); pairs within the cut-off:
    # a brute-force count on the host; the kernel counters agree between
    # graph and eager stepping (the same skin decisions in both)
    reps = replicas()[:3]
    runs = []
    for graphs in (True, False):
        ens = M.Ensemble([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005, precision=M.FP32_MIXED)
        ens.set_graph_mode(graphs)
        ens.set_kernel_timing(True)
        ens.calculate(40)
        fms, fl, kl = ens.kernel_time()
        entries, pairs = ens.list_stats()
        states = ens.states_by_id()
        ens.close()
        runs.append((fms, fl, kl, entries, pairs))
    assert runs[0][1:] == runs[1][1:]
    fms, fl, kl, entries, pairs = runs[0]
    assert fl == 40 and fms > 0.0 and kl >= 40 * 5
    want_entries = 0
    for r in reps:
        s = M.System(r.L, cutoff=2.5, time_step=0.005, capacity=r.n, precision=M.FP32_MIXED)
        s.set_state(r.q, r.v)
        s.calculate(40)
        want_entries += s.info()["list_entries"]
        s.close()
    assert entries == want_entries
    assert pairs == sum(_pairs_within_cutoff(q, np.asarray(r.L), 2.5) for (q, _), r in zip(states, reps))
