"""The tuned launch shapes: lanes per atom of the FP32-mixed force pass
(1, 2, 4), and threads per block (64, 128, 256) and lanes per atom (1, 2,
4) of the list build.  Every
choice must give bit-identical results -- the row sums follow one fixed
summation tree whatever the lane count, and the list rows do not depend on
the block size -- so the autotuner's choice never changes a trajectory."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _system(st, **kw):
    s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=M.FP32_MIXED, **kw)
    s.set_state(st.q, st.v)
    return s


@pytest.mark.parametrize("rho", [0.5, 0.8442])
def test_lanes_and_blocks_bit_identical(rho):
    st = W.fcc_liquid(8, rho, 1.0, seed=71, jitter=0.06, rc=2.5, dt=0.005)
    shapes = [(1, 64, 2), (2, 128, 4), (4, 256, 1), (1, 128, 4), (2, 64, 8)]
    forces, states, pairs = [], [], []
    for tpa, bb, bl in shapes:
        s = _system(st, threads_per_atom=tpa, build_block=bb, build_threads_per_atom=bl)
        forces.append(s.forces_by_id())
        pairs.append(s.neighbor_list())
        s.calculate(60)
        states.append(s.state_by_id())
        info = s.info()
        assert (info["threads_per_atom"], info["build_block"], info["build_threads_per_atom"]) == (tpa, bb, bl)
        s.close()
    for rows, part in pairs[1:]:   # the same rows, entry for entry
        assert np.array_equal(rows, pairs[0][0]) and np.array_equal(part, pairs[0][1])
    for f in forces[1:]:
        assert np.array_equal(f, forces[0])
    for q, v in states[1:]:
        assert np.array_equal(q, states[0][0]) and np.array_equal(v, states[0][1])


@pytest.mark.parametrize("thermostat", ["nose_hoover", "langevin"])
def test_lanes_bit_identical_with_thermostats(thermostat):
    # the Nose-Hoover kinetic energy partials cover the same atoms in the
    # same tree whatever the lane count, and Langevin's noise is per atom
    st = W.fcc_liquid(8, 0.8442, 1.0, seed=73, jitter=0.06, rc=2.5, dt=0.005)
    kw = dict(thermostat=M.NOSE_HOOVER if thermostat == "nose_hoover" else M.LANGEVIN,
              aimed_temperature=0.8, seed=9)
    states = []
    for tpa in (1, 2, 4):
        s = _system(st, threads_per_atom=tpa, build_block=128, build_threads_per_atom=1, **kw)
        s.calculate(60)
        states.append(s.state_by_id())
        s.close()
    for q, v in states[1:]:
        assert np.array_equal(q, states[0][0]) and np.array_equal(v, states[0][1])


def test_autotune_picks_a_shape_and_keeps_the_trajectory():
    st = W.fcc_liquid(10, 0.8442, 0.9, seed=72, jitter=0.05, rc=2.5, dt=0.004)
    a = _system(st)                                    # tuned at the first step
    b = _system(st, threads_per_atom=1, build_block=128, build_threads_per_atom=1)
    a.calculate(40)
    b.calculate(40)
    info = a.info()
    assert info["threads_per_atom"] in (1, 2, 4)
    assert info["build_block"] in (64, 128, 256)
    assert info["build_threads_per_atom"] in (1, 2, 4, 8)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    assert a.info()["rebuilds"] == b.info()["rebuilds"]
    f64 = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=M.FP64)
    f64.set_state(st.q, st.v)
    f64.calculate(1)
    assert f64.info()["threads_per_atom"] == 1


def test_ensemble_lanes_bit_identical():
    reps = [W.fcc_liquid(6, 0.5, 1.0, seed=73, jitter=0.08, rc=2.5, dt=0.005),
            W.fcc_liquid(7, 0.8442, 0.8, seed=74, jitter=0.05, rc=2.5, dt=0.005)]
    out = []
    for tpa in (1, 4, 0):
        e = M.Ensemble([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005, precision=M.FP32_MIXED,
                       threads_per_atom=tpa)
        e.calculate(45)
        out.append(e.states_by_id())
        e.close()
    for got in out[1:]:
        for k in range(len(reps)):
            assert np.array_equal(got[k][0], out[0][k][0]) and np.array_equal(got[k][1], out[0][k][1])


@pytest.mark.parametrize("field,value", [("threads_per_atom", 3), ("build_block", 100),
                                         ("build_threads_per_atom", 16)])
def test_invalid_shapes_rejected(field, value):
    st = W.fcc_liquid(5, 0.5, 1.0, seed=75, rc=2.5)
    with pytest.raises(M.MdgError) as e:
        M.System(st.L, cutoff=2.5, capacity=st.n, **{field: value})
    assert e.value.status == -1


@pytest.mark.parametrize("tpa", [1, 4])
def test_persistent_steps_equal_graph_steps(tpa):
    # the cooperative multi-step pass runs the fused NVE step back to back,
    # takes the displacement checks itself and hands the steps that need a
    # rebuild to the queued rebuild step: the trajectory, the rebuild steps
    # and the check count are the graph path's
    st = W.fcc_liquid(12, 0.5, 1.0, seed=76, jitter=0.05, rc=2.5, dt=0.005)
    a = _system(st, threads_per_atom=tpa, step_mode=M.STEPS_GRAPHS)
    b = _system(st, threads_per_atom=tpa, step_mode=M.STEPS_PERSISTENT)
    a.calculate(200)
    b.calculate(137)
    b.calculate(63)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    ia, ib = a.info(), b.info()
    assert ia["rebuilds"] == ib["rebuilds"] and ia["displacement_checks"] == ib["displacement_checks"]
    assert ia["simulation_time"] == ib["simulation_time"] and ia["buffer_left"] == ib["buffer_left"]
    assert ib["persistent_steps"] > 100 and ia["persistent_steps"] == 0
    assert ib["steps"] == 200
