"""MDManager::ChangeScale and the cavitation project's density grid on the
device (mdg_change_scale, mdg_density_grid)."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def wrapped(q, L):
    # the wrap a pairlist construction applies (Variables::AdjustPeriodicBoundary)
    q = np.where(q < 0.0, q + L, q)
    return np.where(q > L, q - L, q)


def test_change_scale_equals_a_fresh_system_in_the_scaled_box():
    st = W.fcc_liquid(7, 0.8, 1.0, seed=81, jitter=0.05, rc=2.5, dt=0.005)
    a = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n)
    a.set_state(st.q, st.v)
    a.calculate(30)
    q, v, ids = a.state()
    a.change_scale(1.05)
    b = M.System(st.L * 1.05, cutoff=2.5, time_step=0.005, capacity=st.n)
    b.set_state(wrapped(q, st.L) * 1.05, v)
    qa, va, ia = a.state()
    qb, vb, _ = b.state()
    # same positions (one rounding each) before any step
    assert np.array_equal(np.sort(qa, axis=0), np.sort(qb, axis=0))
    a.calculate(30)
    b.calculate(30)
    qa, va = a.state_by_id()
    qb_slot, vb_slot, ib = b.state()
    # b's upload order is a's slot order at the time of the state read
    qb_by_a = np.empty_like(qb_slot)
    vb_by_a = np.empty_like(vb_slot)
    qb_by_a[ids[ib]] = qb_slot
    vb_by_a[ids[ib]] = vb_slot
    L = st.L * 1.05
    d = qa - qb_by_a
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-10
    assert np.abs(va - vb_by_a).max() < 1e-10


def test_change_scale_rejects_a_box_below_three_cells():
    st = W.fcc_liquid(5, 0.8, 1.0, seed=82, jitter=0.05, rc=2.5, dt=0.005)  # L = 8.55 -> 3 cells
    s = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n)
    s.set_state(st.q, st.v)
    with pytest.raises(M.MdgError):
        s.change_scale(0.9)


def test_density_grid_matches_numpy_histogram():
    st = W.fcc_liquid(8, 0.8, 1.0, seed=83, jitter=0.05, rc=2.5, dt=0.005)
    s = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n)
    s.set_state(st.q, st.v)
    s.calculate(40)
    gs = 3.0
    grid = s.density_grid(gs)
    q, _, _ = s.state()
    g = [int(x / gs + 0.5) for x in st.L]
    step = st.L[0] / g[0]
    w = q - st.L * np.floor(q / st.L)
    idx = np.clip((w / step).astype(int), 0, np.array(g) - 1)
    ref = np.zeros(g[::-1], dtype=np.int64)
    np.add.at(ref, (idx[:, 2], idx[:, 1], idx[:, 0]), 1)
    assert grid.shape == tuple(g[::-1])
    assert np.array_equal(grid.astype(np.int64), ref % 256)
