"""Parity of the CUDA path (through the C ABI) with the reference's outputs
(golden fixtures) and with the CPU oracle on the same seeded inputs.

Bars: pair sets bit-exact; FP64 forces, energy and virial within 1e-12
relative (norm-wise for forces); FP32-mixed forces within 1e-5 relative."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from conftest import force_error, pair_set, rms_force_error
from mdacp_b200 import workloads as W
from oracle import lj_oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def make_system(q, v, L, rc, dt, precision=M.FP64, **kw):
    s = M.System(L, cutoff=rc, time_step=dt, capacity=q.shape[0], precision=precision, **kw)
    s.set_state(q, v)
    return s


def gsys(g, precision=M.FP64, **kw):
    return make_system(g["q"], g["v"], g["L"], float(g["rc"]), float(g["dt"]), precision, **kw)


@pytest.mark.parametrize("precision", [M.FP64, M.FP32_MIXED])
def test_pairs_match_reference(golden, precision):
    s = gsys(golden, precision)
    k, p = s.pairs()
    got = pair_set(k, p)
    assert got.shape[0] == k.shape[0], "duplicate pair in a row"
    assert np.array_equal(got, golden["pairs"].astype(np.int64))


def test_forces_fp64_match_reference(golden):
    s = gsys(golden)
    f = s.forces_by_id()
    assert force_error(f, golden["forces"]) <= FP64_TOL


def test_forces_fp32_mixed_error(golden):
    s = gsys(golden, M.FP32_MIXED)
    f = s.forces_by_id()
    assert force_error(f, golden["forces"]) <= FP32_TOL
    assert rms_force_error(f, golden["forces"]) <= FP32_TOL


def test_observers_fp64_match_reference(golden):
    s = gsys(golden)
    ke, pe, vir = s.observe()
    assert ke == pytest.approx(float(golden["ke"]), rel=FP64_TOL)
    assert pe == pytest.approx(float(golden["pe"]), rel=FP64_TOL)
    assert vir == pytest.approx(float(golden["virial"]), rel=FP64_TOL)


def test_trajectory_fp64_matches_reference(golden):
    nh = str(golden["thermostat"]) == "NoseHoover"
    kw = {}
    if nh:
        kw = dict(thermostat=M.NOSE_HOOVER, aimed_temperature=float(golden["aimed_temperature"]),
                  heatbath_tau=float(golden["heatbath_tau"]))
    s = gsys(golden, **kw)
    steps = int(golden["steps"])
    s.calculate(steps)
    q, v = s.state_by_id()
    L = golden["L"]
    dq = q - golden["traj_q"]
    dq -= L * np.round(dq / L)  # positions may sit in different periodic images
    assert np.abs(dq).max() < 1e-9
    assert np.abs(v - golden["traj_v"]).max() < 1e-9
    info = s.info()
    assert info["steps"] == steps
    # the skin test runs over the reference's ghost copies, so the pairlist
    # is rebuilt at the same steps (MeshList constructions incl. the first)
    assert info["rebuilds"] == int(golden["constructions"])


def test_observers_along_trajectory_match_reference(golden):
    # the reference's KE/N, PE/N and virial every steps/4 steps; its
    # observers see ghost copies half a step old (MDG_OBSERVE_GHOST_LAG)
    nh = str(golden["thermostat"]) == "NoseHoover"
    kw = {}
    if nh:
        kw = dict(thermostat=M.NOSE_HOOVER, aimed_temperature=float(golden["aimed_temperature"]),
                  heatbath_tau=float(golden["heatbath_tau"]))
    s = gsys(golden, **kw)
    s.set_observer_mode(M.OBSERVE_GHOST_LAG)
    n = golden["q"].shape[0]
    every = max(1, int(golden["steps"]) // 4)
    assert golden["traj_obs"].shape[0] == 4
    for row in golden["traj_obs"]:
        s.calculate(every)
        ke, pe, vir = s.observe()
        assert ke / n == pytest.approx(row[0], rel=1e-9)
        assert pe / n == pytest.approx(row[1], rel=1e-9)
        assert vir == pytest.approx(row[2], rel=1e-9)


@pytest.mark.parametrize("rho,temperature", [(0.5, 1.0), (0.8442, 1.0)])
def test_matches_oracle_32k(rho, temperature):
    # 32,000 atoms at the densities of the 32k workloads; the lattice is
    # jittered because forces on a perfect lattice vanish
    st = W.fcc_liquid(20, rho, temperature, seed=31, jitter=0.06, rc=2.5, dt=0.005)
    o = O.Oracle(st.q, st.v, st.ids, st.L, st.rc, st.dt)
    o.make_pairlist()
    ok, op = o.pairs()
    of = o.forces()
    oq, ov, oid = o.state()
    fo = np.empty_like(of)
    fo[oid] = of
    oke, ope, ovir = o.observe()
    s = make_system(st.q, st.v, st.L, st.rc, st.dt)
    k, p = s.pairs()
    assert np.array_equal(pair_set(k, p), pair_set(ok, op))
    assert force_error(s.forces_by_id(), fo) <= FP64_TOL
    ke, pe, vir = s.observe()
    assert ke == pytest.approx(oke, rel=FP64_TOL)
    assert pe == pytest.approx(ope, rel=FP64_TOL)
    assert vir == pytest.approx(ovir, rel=FP64_TOL)
    s32 = make_system(st.q, st.v, st.L, st.rc, st.dt, M.FP32_MIXED)
    f32 = s32.forces_by_id()
    assert force_error(f32, fo) <= FP32_TOL


@pytest.mark.parametrize("precision", [M.FP64, M.FP32_MIXED])
def test_graph_steps_equal_eager_steps(precision):
    g = W.fcc_liquid(6, 0.5, 1.0, seed=21, jitter=0.08, rc=2.5, dt=0.005)
    a = make_system(g.q, g.v, g.L, g.rc, g.dt, precision)
    b = make_system(g.q, g.v, g.L, g.rc, g.dt, precision)
    a.calculate(40)             # two 20-step graph launches
    for _ in range(40):
        b.calculate(1)          # host-driven steps
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    assert a.info()["rebuilds"] == b.info()["rebuilds"]


def test_fused_fp32_step_survives_interleaved_calls():
    # The FP32-mixed NVE step keeps the next step's fixed-point copy between
    # calls; odd step counts, observers, force queries and a state round
    # trip in between must leave the trajectory unchanged.
    g = W.fcc_liquid(6, 0.8442, 1.0, seed=23, jitter=0.05, rc=2.5, dt=0.005)
    a = make_system(g.q, g.v, g.L, g.rc, g.dt, M.FP32_MIXED)
    b = make_system(g.q, g.v, g.L, g.rc, g.dt, M.FP32_MIXED)
    a.calculate(60)
    b.calculate(7)
    b.observe()
    b.calculate(33)
    b.forces()
    q, v = b.state_by_id()
    b.calculate(3)
    b.pairs()
    b.calculate(17)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)


def test_langevin_matches_oracle_noise():
    g = W.fcc_liquid(6, 0.5, 1.0, seed=22, jitter=0.05, rc=2.5, dt=0.005)
    kw = dict(thermostat=M.LANGEVIN, aimed_temperature=1.3, heatbath_gamma=1.0, seed=77)
    s = make_system(g.q, g.v, g.L, g.rc, g.dt, **kw)
    o = O.Oracle(g.q, g.v, g.ids, g.L, g.rc, g.dt, thermostat=O.LANGEVIN, temperature=1.3, gamma=1.0, seed=77)
    o.make_pairlist()
    s.calculate(25)
    o.step(25)
    q, v, ids = o.state()
    vo = np.empty_like(v)
    vo[ids] = v
    _, vg = s.state_by_id()
    assert np.abs(vg - vo).max() < 1e-9


def test_nose_hoover_zeta_matches_oracle():
    g = W.fcc_liquid(6, 0.5, 1.0, seed=23, jitter=0.05, rc=2.5, dt=0.005)
    s = make_system(g.q, g.v, g.L, g.rc, g.dt, thermostat=M.NOSE_HOOVER, aimed_temperature=1.4,
                    heatbath_tau=0.1)
    o = O.Oracle(g.q, g.v, g.ids, g.L, g.rc, g.dt, thermostat=O.NOSE_HOOVER, temperature=1.4, tau=0.1)
    o.make_pairlist()
    s.calculate(60)
    o.step(60)
    assert s.zeta() == pytest.approx(o.zeta, rel=1e-9)


# ---------------------------------------------------------------- errors
def test_too_fast_particle_is_an_error():
    g = W.fcc_liquid(5, 0.5, 1.0, seed=24, rc=2.5, dt=0.005)
    v = g.v.copy()
    v[7] = [100.0, 0.0, 0.0]  # 2 |v| dt = 1.0 > BufferLength 0.3
    s = make_system(g.q, v, g.L, g.rc, g.dt)
    s.calculate(1)  # the first step rebuilds (fresh upload) and spends no budget
    with pytest.raises(M.MdgError) as e:
        s.calculate(1)
    assert e.value.status == -4


def test_nonfinite_state_rejected():
    g = W.fcc_liquid(5, 0.5, 1.0, seed=25, rc=2.5)
    q = g.q.copy()
    q[3, 1] = np.nan
    s = M.System(g.L, cutoff=2.5, time_step=0.005, capacity=g.n)
    with pytest.raises(M.MdgError) as e:
        s.set_state(q, g.v)
    assert e.value.status == -6


def test_box_too_small_rejected():
    with pytest.raises(M.MdgError) as e:
        M.System([8.0, 12.0, 12.0], cutoff=2.5, capacity=10)
    assert e.value.status == -7


def test_capacity_exceeded_rejected():
    g = W.fcc_liquid(5, 0.5, 1.0, seed=26, rc=2.5)
    s = M.System(g.L, cutoff=2.5, time_step=0.005, capacity=g.n - 1)
    with pytest.raises(M.MdgError) as e:
        s.set_state(g.q, g.v)
    assert e.value.status == -3


def test_neighbor_rows_grow_on_overflow():
    g = load = W.fcc_liquid(6, 0.8442, 0.722, seed=27, jitter=0.05, rc=2.5, dt=0.004)
    s = make_system(g.q, g.v, g.L, g.rc, g.dt, max_neighbors=16)
    ref = make_system(g.q, g.v, g.L, g.rc, g.dt)
    s.calculate(30)
    ref.calculate(30)
    qa, va = s.state_by_id()
    qb, vb = ref.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    assert s.info()["max_neighbors"] >= ref.info()["max_row"]
    del load


def test_empty_system():
    s = M.System([12.0, 12.0, 12.0], cutoff=2.5, capacity=4)
    s.set_state(np.zeros((0, 3)), np.zeros((0, 3)))
    s.calculate(5)
    assert s.observe() == (0.0, 0.0, 0.0)
    k, p = s.pairs()
    assert k.size == 0
