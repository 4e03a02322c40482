"""The staged FP32-mixed force pass against the pass that gathers partners
from global memory.  The staged pass copies, per block of 128 atoms, the
fixed-point positions of the union of the block's 27-cell stencils into
shared memory and reads partners there through 16-bit stage indices.  Its
pair terms and their order are the global pass's, so trajectories must be
bit-identical: for every thermostat, for force queries, with a stage too
small for some blocks (those gather from global memory), in a box of 3
cells per axis (one block's stencils cover the whole box), in dilute boxes
(blocks spanning many cell rows), and after the neighbour rows grew."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def pair_of(st, stage, **kw):
    out = []
    for atoms in (stage, 0):
        s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=M.FP32_MIXED,
                     stage_atoms=atoms, **kw)
        s.set_state(st.q, st.v)
        out.append(s)
    return out


def assert_same(a, b):
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    assert a.info()["rebuilds"] == b.info()["rebuilds"]


@pytest.mark.parametrize("thermostat", [M.NVE, M.NOSE_HOOVER, M.LANGEVIN])
def test_staged_trajectory_is_bit_identical(thermostat):
    st = W.fcc_liquid(12, 0.8442, 1.0, seed=71, jitter=0.05, rc=2.5, dt=0.005)  # 6912 atoms, 7 cells per axis
    a, b = pair_of(st, -1, thermostat=thermostat, aimed_temperature=0.9, seed=5)
    a.calculate(60)
    b.calculate(60)
    assert a.info()["rebuilds"] >= 2
    assert_same(a, b)


def test_staged_forces_are_bit_identical():
    st = W.fcc_liquid(12, 0.8442, 1.0, seed=72, jitter=0.05, rc=2.5, dt=0.005)
    a, b = pair_of(st, -1)
    assert np.array_equal(a.forces_by_id(), b.forces_by_id())


def test_small_stage_mixes_staged_and_gathering_blocks():
    # a 1700-atom stage holds about a third of the blocks' stencils (8 cells
    # per axis); the others gather from global memory in the same launch
    st = W.fcc_liquid(14, 0.8442, 1.0, seed=73, jitter=0.05, rc=2.5, dt=0.005)
    a, b = pair_of(st, 1700)
    a.calculate(40)
    b.calculate(40)
    assert_same(a, b)


def test_three_cells_per_axis():
    st = W.fcc_liquid(5, 0.80, 1.0, seed=74, jitter=0.05, rc=2.5, dt=0.005)  # L = 8.55: 3 cells per axis
    a, b = pair_of(st, -1)
    a.calculate(50)
    b.calculate(50)
    assert_same(a, b)


@pytest.mark.parametrize("rho", [0.3, 0.5])
def test_dilute_boxes(rho):
    st = W.fcc_liquid((9, 7, 8), rho, 1.2, seed=75, jitter=0.05, rc=2.5, dt=0.005)
    a, b = pair_of(st, -1)
    a.calculate(50)
    b.calculate(50)
    assert_same(a, b)


def test_rows_grow_with_staging():
    st = W.fcc_liquid(8, 0.8442, 0.722, seed=76, jitter=0.05, rc=2.5, dt=0.004)
    a, b = pair_of(st, -1, max_neighbors=16)
    a.calculate(30)
    b.calculate(30)
    assert_same(a, b)
    assert a.info()["max_neighbors"] >= a.info()["max_row"]


def test_staged_after_change_scale_and_restart(tmp_path):
    # a new cell grid (ChangeScale) and a checkpoint restart both rebuild the
    # list, and with it the stage plans
    st = W.fcc_liquid(12, 0.8442, 1.0, seed=78, jitter=0.05, rc=2.5, dt=0.005)
    a, b = pair_of(st, -1)
    for s in (a, b):
        s.calculate(20)
        s.change_scale(1.04)
        s.calculate(25)
    assert_same(a, b)
    a.save_checkpoint(tmp_path / "staged.ckpt")
    c = M.System(a.params.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=M.FP32_MIXED,
                 stage_atoms=-1)
    c.load_checkpoint(tmp_path / "staged.ckpt")
    for s in (a, b, c):
        s.calculate(30)
    assert_same(a, b)
    assert_same(a, c)


def test_stage_size_is_checked():
    st = W.fcc_liquid(5, 0.8442, 1.0, seed=77, rc=2.5)
    for bad in (-2, 12289):
        with pytest.raises(M.MdgError):
            M.System(st.L, cutoff=2.5, capacity=st.n, precision=M.FP32_MIXED, stage_atoms=bad)


def test_stage_wait_that_runs_out_reports_timeout_and_the_device_stays_usable():
    # a one-cycle limit on the first wait for the stage copy makes it give
    # up (the copy takes microseconds): the block sets the timeout flag,
    # waits for its copies with the normal limit before it exits, and the
    # call returns MDG_ERR_TIMEOUT; a handle made afterwards steps normally
    st = W.fcc_liquid(12, 0.8442, 1.0, seed=79, jitter=0.05, rc=2.5, dt=0.005)
    s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=M.FP32_MIXED,
                 stage_atoms=-1, stage_wait_cycles=1)
    s.set_state(st.q, st.v)
    with pytest.raises(M.MdgError) as e:
        s.calculate(5)
    assert e.value.status == -8
    s.close()
    a, b = pair_of(st, -1)
    a.calculate(20)
    b.calculate(20)
    assert_same(a, b)
    with pytest.raises(M.MdgError):
        M.System(st.L, cutoff=2.5, capacity=st.n, precision=M.FP32_MIXED, stage_atoms=-1, stage_wait_cycles=-1)
