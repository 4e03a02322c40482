"""Executors of the reference's projects (gravity, piston, shell wall) applied
on the device after every step, against the oracle's restatement of the same
executors run after each of its steps (ljo_apply_external)."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W
from conftest import rankine_start
from oracle import lj_oracle as O

pytestmark = pytest.mark.gpu

STEPS = 100


def state(select=None, ncell=6, seed=61):
    st = W.fcc_liquid(ncell, 0.8442, 1.0, seed, jitter=0.05, rc=2.5, dt=0.005)
    q, v = st.q, st.v
    if select is not None:
        keep = select(q, st.L)
        q, v = q[keep], v[keep]
    return q, v, st.L


def run_both(q, v, L, ext_kw, precision=M.FP64, steps=STEPS):
    o = O.Oracle(q, v, np.arange(q.shape[0], dtype=np.int32), L, 2.5, 0.005)
    ox = O.External()
    ox.kind = ext_kw["kind"]
    ox.axis = ext_kw.get("axis", 0)
    ox.strength = ext_kw.get("strength", 0.0)
    ox.time_step = ext_kw.get("time_step", 0.005)
    ox.position = ext_kw.get("position", 0.0)
    ox.velocity = ext_kw.get("velocity", 0.0)
    ox.center[:] = list(ext_kw.get("center", (0.0, 0.0, 0.0)))
    ox.radius = ext_kw.get("radius", 0.0)
    imp = 0.0
    for _ in range(steps):
        o.step(1)
        imp = o.apply_external(ox)
    s = M.System(L, cutoff=2.5, time_step=0.005, capacity=q.shape[0], precision=precision)
    s.set_state(q, v)
    s.set_external(**ext_kw)
    s.calculate(steps)
    return o, ox, imp, s


def compare(o, s, L, tol=1e-9):
    oq, ov, oid = o.state()
    q, v = s.state_by_id()
    rq, rv = np.empty_like(oq), np.empty_like(ov)
    rq[oid], rv[oid] = oq, ov
    dq = q - rq
    dq -= L * np.round(dq / L)
    assert np.abs(dq).max() < tol
    assert np.abs(v - rv).max() < tol
    assert s.info()["rebuilds"] == o.constructions


def test_gravity_matches_oracle():
    q, v, L = state()
    kw = dict(kind=M.EXTERNAL_GRAVITY, axis=0, strength=0.2, time_step=0.005)
    o, _, _, s = run_both(q, v, L, kw)
    compare(o, s, L)


def test_piston_matches_oracle():
    # atoms kept away from the wall at z = 0 and the piston's start
    def sel(q, L):
        return (q[:, 2] > 1.0) & (q[:, 2] < L[2] - 3.0)
    q, v, L = state(sel)
    kw = dict(kind=M.EXTERNAL_PISTON, position=L[2] - 2.0, velocity=0.004, time_step=0.005)
    o, ox, imp, s = run_both(q, v, L, kw)
    compare(o, s, L)
    pos, gimp = s.external_state()
    assert pos == ox.position  # the same repeated subtraction
    assert gimp == pytest.approx(imp, rel=1e-9, abs=1e-12)


def test_shell_wall_matches_oracle():
    def sel(q, L):
        c = 0.5 * L[0]
        return np.linalg.norm(q - c, axis=1) < 0.32 * L[0]
    q, v, L = state(sel, ncell=8)
    c = 0.5 * L[0]
    kw = dict(kind=M.EXTERNAL_SHELL, center=(c, c, c), radius=0.32 * L[0] + 1.0, time_step=0.005)
    o, _, _, s = run_both(q, v, L, kw)
    compare(o, s, L)


def test_executor_graph_steps_equal_eager_steps():
    q, v, L = state()
    kw = dict(kind=M.EXTERNAL_GRAVITY, axis=2, strength=0.3, time_step=0.005)
    a = M.System(L, cutoff=2.5, time_step=0.005, capacity=q.shape[0])
    b = M.System(L, cutoff=2.5, time_step=0.005, capacity=q.shape[0])
    for s in (a, b):
        s.set_state(q, v)
        s.set_external(**kw)
    a.calculate(40)
    for _ in range(40):
        b.calculate(1)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)


def test_fp32_mixed_with_executor_and_switching_off():
    q, v, L = state()
    kw = dict(kind=M.EXTERNAL_GRAVITY, axis=1, strength=0.2, time_step=0.005)
    ref = M.System(L, cutoff=2.5, time_step=0.005, capacity=q.shape[0])
    s = M.System(L, cutoff=2.5, time_step=0.005, capacity=q.shape[0], precision=M.FP32_MIXED)
    for x in (ref, s):
        x.set_state(q, v)
        x.set_external(**kw)
        x.calculate(30)
        x.set_external()  # off: back to the plain step
        x.calculate(30)
    q64, v64 = ref.state_by_id()
    q32, v32 = s.state_by_id()
    dq = q32 - q64
    dq -= L * np.round(dq / L)
    assert np.abs(dq).max() < 1e-4
    # the executor moved the centre of mass along y, 30 passes of 0.2 * 0.005
    assert v32[:, 1].mean() - v[:, 1].mean() == pytest.approx(30 * 0.2 * 0.005, rel=1e-6)


def test_invalid_executor_rejected():
    q, v, L = state()
    s = M.System(L, cutoff=2.5, time_step=0.005, capacity=q.shape[0])
    with pytest.raises(M.MdgError):
        s.set_external(kind=7)
    with pytest.raises(M.MdgError):
        s.set_external(kind=M.EXTERNAL_GRAVITY, axis=3)


def test_host_kick_through_set_velocities_equals_device_gravity():
    # an executor that changes momenta only, run on the host between steps
    # and uploaded with mdg_set_velocities, keeps the list and the skin
    # budget: the trajectory equals the device executor's bit for bit, with
    # the same rebuild steps
    g = W.fcc_liquid(6, 0.5, 1.0, seed=91, jitter=0.05, rc=2.5, dt=0.005)
    kick = 0.2 * 0.005
    a = M.System(g.L, cutoff=g.rc, time_step=g.dt, capacity=g.n)
    a.set_state(g.q, g.v)
    a.set_external(M.EXTERNAL_GRAVITY, axis=0, strength=kick, time_step=1.0)
    b = M.System(g.L, cutoff=g.rc, time_step=g.dt, capacity=g.n)
    b.set_state(g.q, g.v)
    a.calculate(60)
    for _ in range(60):
        b.calculate(1)
        q4 = np.empty((b.n, 4))
        v4 = np.empty((b.n, 4))
        b.get_state4(q4, v4)
        v4[:, 0] += kick
        b.set_velocities4(v4)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    ia, ib = a.info(), b.info()
    assert ia["rebuilds"] == ib["rebuilds"] and ia["displacement_checks"] == ib["displacement_checks"]



def piston_kick(q, v, position, dt, cl=2.5):
    """MyPiston::Execute (src/rankine.cc:66-97) on host arrays: the wall at
    z = 0 and the piston at `position`; returns the new velocities and the
    impulse (sequential sum)."""
    s2 = 1.0 / (cl * cl)
    s6 = s2 * s2 * s2
    s8 = s6 * s2
    s14 = s6 * s6 * s2
    c2 = 6.0 * s14 - 3.0 * s8
    v = v.copy()
    imp = 0.0
    for i in range(q.shape[0]):
        z = q[i, 2]
        if z < cl:
            r2 = z * z
            r6 = r2 * r2 * r2
            df = ((24.0 * r6 - 48.0) / (r6 * r6 * r2) + c2 * 8.0) * dt
            v[i, 2] -= df * z
        if z > position:
            dz = position - z + cl
            r2 = dz * dz
            r6 = r2 * r2 * r2
            df = ((24.0 * r6 - 48.0) / (r6 * r6 * r2) + c2 * 8.0) * dt
            v[i, 2] += df * dz
            imp -= df * dz
    return v, imp


def test_rankine_piston_observers_match_oracle():
    # the reference's Rankine loop from its start state (the oracle
    # reproduces the project's printed rows): after every step the piston
    # executor changes momenta -- on the device (mdg_set_external) and on the
    # host, uploaded with set_velocities as the drop-in does -- and the
    # observers see the reference's ghost copies, dated by the velocities of
    # the step's drift, not the kicked ones
    q, v, L = rankine_start()
    n = q.shape[0]
    dt, d_pos = 0.005, L[2] * 0.5 / 500
    o = O.Oracle(q, v, np.arange(n, dtype=np.int32), L, 2.5, dt)
    o.make_pairlist()
    ox = O.External()
    ox.kind, ox.position, ox.velocity, ox.time_step = M.EXTERNAL_PISTON, L[2] - 2.0, d_pos, dt
    dev = M.System(L, cutoff=2.5, time_step=dt, capacity=n)
    dev.set_state(q, v)
    dev.set_external(kind=M.EXTERNAL_PISTON, position=L[2] - 2.0, velocity=d_pos, time_step=dt)
    host = M.System(L, cutoff=2.5, time_step=dt, capacity=n)
    host.set_state(q, v)
    position = L[2] - 2.0
    for s in (dev, host):
        s.set_observer_mode(M.OBSERVE_GHOST_LAG)
    q4, v4 = np.empty((n, 4)), np.empty((n, 4))
    for i in range(151):
        o.step(1)
        o.apply_external(ox)
        dev.calculate(1)
        host.calculate(1)
        host.get_state4(q4, v4)
        v4[:, :3], _ = piston_kick(q4[:, :3], v4[:, :3], position, dt)
        host.set_velocities4(v4)
        position -= d_pos
        if i % 50 == 0:
            ref = o.observe()
            for s in (dev, host):
                got = s.observe()
                for k in range(3):
                    assert got[k] == pytest.approx(ref[k], rel=1e-10), (i, k)
    assert dev.external_state()[0] == ox.position
    o.close()
