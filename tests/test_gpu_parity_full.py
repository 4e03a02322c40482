"""Parity at the benchmark sizes: the CUDA path (through the C ABI) against
the CPU oracle on the exact states the benchmarks time.

* the 2,048,000-atom FCC liquid (rho 0.8442, T 0.722, rc 2.5, search length
  2.8, dt 0.004) that bench.py times, from its start state and after 10 NVE
  steps;
* the 1,000,000-atom liquid-vapour slab at rc 3.0 (search length 3.3) with
  the Langevin thermostat;
* the 32,000-atom FCC start at rho 0.5 with Maxwell-Boltzmann velocities.

Bars, as at the small sizes: directed pair sets bit-exact; FP64 forces,
energy and virial within 1e-12 relative (norm-wise for forces); FP32-mixed
forces within 1e-5 relative of the oracle's FP64 forces (max and RMS,
norm-wise); trajectories within 1e-9 with the same rebuild count.

Forces on a perfect lattice cancel to rounding noise, so the force checks
run on the state the oracle reaches after a few steps (handed to fresh GPU
handles), while pair sets and observer sums are also checked at the start.
Pair sets are compared as sorted int64 keys (key * n + partner), which
keeps the 160-million-entry sets of the 2.05M-atom liquid cheap.  The
oracle's energy and virial are its pair terms added with compensated
summation: the reference's plain running sum over 80 million pair terms of
a lattice (nearly equal terms, correlated roundings) is itself off by
about 4e-10 relative, above the bar."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from conftest import force_error, rms_force_error
from mdacp_b200 import workloads as W
from oracle import lj_oracle as O

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 1e-5
TRAJ_TOL = 1e-9


def pair_keys(k, p, n):
    """Sorted directed-pair keys; asserts no pair appears twice."""
    key = np.asarray(k, dtype=np.int64) * n + np.asarray(p, dtype=np.int64)
    key.sort()
    assert key.size < 2 or bool(np.all(key[1:] != key[:-1])), "duplicate pair"
    return key


def by_id(x, ids):
    out = np.empty_like(x)
    out[ids] = x
    return out


def gpu_system(st, q, v, precision, **kw):
    s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=precision, **kw)
    s.set_state(q, v)
    return s


def check_state(st, q, v, oracle_kw=None, fp32=True, lattice=False):
    """Pair set, FP64 forces and observer sums of the state (q, v) (in id
    order) against the oracle, and the FP32-mixed force error.  lattice: q
    is a perfect lattice, whose forces are rounding residues of cancelling
    pair terms of size about 1, so they are compared absolutely (1e-11)."""
    oracle_kw = oracle_kw or {}
    # a state after some steps has atoms just outside [0, L] (the wrap comes
    # with the next rebuild); both sides get it wrapped as the reference
    # wraps (Variables::AdjustPeriodicBoundary)
    q = np.where(q < 0.0, q + st.L, np.where(q > st.L, q - st.L, q))
    o = O.Oracle(q, v, st.ids, st.L, st.rc, st.dt, **oracle_kw)
    o.make_pairlist()
    ok, op = o.pairs()
    ref_keys = pair_keys(ok, op, st.n)
    del ok, op
    _, _, oid = o.state()
    f_ref = by_id(o.forces(), oid)
    oke, ope, ovir = o.observe(compensated=True)
    o.close()

    s = gpu_system(st, q, v, M.FP64)
    k, p = s.pairs()
    assert np.array_equal(pair_keys(k, p, st.n), ref_keys)
    del k, p
    ke, pe, vir = s.observe()
    assert ke == pytest.approx(oke, rel=FP64_TOL)
    assert pe == pytest.approx(ope, rel=FP64_TOL)
    assert vir == pytest.approx(ovir, rel=FP64_TOL)
    if lattice:
        assert np.abs(s.forces_by_id() - f_ref).max() <= 1e-11
    else:
        assert force_error(s.forces_by_id(), f_ref) <= FP64_TOL
    s.close()
    if not fp32:
        return None
    s = gpu_system(st, q, v, M.FP32_MIXED)
    k, p = s.pairs()
    assert np.array_equal(pair_keys(k, p, st.n), ref_keys)
    del k, p
    f32 = s.forces_by_id()
    s.close()
    err = force_error(f32, f_ref), rms_force_error(f32, f_ref)
    assert err[0] <= FP32_TOL and err[1] <= FP32_TOL, err
    return err


def check_trajectory(st, steps, oracle_kw=None, system_kw=None):
    """steps of the FP64 GPU path against the oracle from the start state;
    returns the oracle's state afterwards (q, v in id order)."""
    o = O.Oracle(st.q, st.v, st.ids, st.L, st.rc, st.dt, **(oracle_kw or {}))
    o.make_pairlist()
    o.step(steps)
    oq, ov, oid = o.state()
    constructions = o.constructions
    o.close()
    oq, ov = by_id(oq, oid), by_id(ov, oid)
    s = gpu_system(st, st.q, st.v, M.FP64, **(system_kw or {}))
    s.calculate(steps)
    q, v = s.state_by_id()
    info = s.info()
    s.close()
    dq = q - oq
    dq -= st.L * np.round(dq / st.L)  # positions may sit in different periodic images
    assert np.abs(dq).max() < TRAJ_TOL
    assert np.abs(v - ov).max() < TRAJ_TOL
    assert info["rebuilds"] == constructions
    return oq, ov


def test_liquid_2048000_start_state():
    # the state bench.py times (rank 0): a perfect FCC lattice, so the
    # check is the pair set and the observer sums
    st = W.config_c2(seed=2026)
    assert st.n == 2_048_000
    check_state(st, st.q, st.v, fp32=False, lattice=True)


def test_liquid_2048000_after_10_steps():
    st = W.config_c2(seed=2026)
    q, v = check_trajectory(st, 10)
    check_state(st, q, v)


def test_slab_1000000_rc3():
    # the Langevin slab: random positions, so the forces are large at the start
    st = W.config_c3(seed=31)
    check_state(st, st.q, st.v)
    kw = dict(thermostat=O.LANGEVIN, temperature=0.9, gamma=1.0, seed=7)
    check_trajectory(st, 10, oracle_kw=kw,
                     system_kw=dict(thermostat=M.LANGEVIN, aimed_temperature=0.9, heatbath_gamma=1.0, seed=7))


def test_fcc_32000_rho05_start_and_trajectory():
    st = W.config_c1(seed=12345)
    check_state(st, st.q, st.v, fp32=False, lattice=True)
    q, v = check_trajectory(st, 200)
    check_state(st, q, v)
