"""Checkpoint and restart (a restored handle continues bit for bit), and the
reference's text snapshots written asynchronously from the device state."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def system(precision=M.FP64, away_from_z0=False, **kw):
    st = W.fcc_liquid(6, 0.8442, 1.0, seed=71, jitter=0.05, rc=2.5, dt=0.005)
    if away_from_z0:  # room for the executor's wall at z = 0 and its piston
        keep = (st.q[:, 2] > 1.0) & (st.q[:, 2] < st.L[2] - 3.0)
        st.q, st.v, st.ids = st.q[keep], st.v[keep], st.ids[: keep.sum()]
    s = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n, precision=precision, **kw)
    s.set_state(st.q, st.v)
    return s, st


CASES = {
    "fp64_nve": dict(precision=M.FP64),
    "fp32_nve": dict(precision=M.FP32_MIXED),
    "fp64_nose_hoover": dict(precision=M.FP64, thermostat=M.NOSE_HOOVER, aimed_temperature=0.8, heatbath_tau=0.2),
    "fp32_langevin": dict(precision=M.FP32_MIXED, thermostat=M.LANGEVIN, aimed_temperature=0.9,
                          heatbath_gamma=1.0, seed=5),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_restart_continues_bit_for_bit(case, tmp_path):
    kw = CASES[case]
    a, st = system(**kw)
    a.calculate(100)
    b, _ = system(**kw)
    b.calculate(43)
    path = tmp_path / "state.ckpt"
    b.save_checkpoint(path)
    c = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n, **kw)
    c.load_checkpoint(path)
    c.calculate(57)
    qa, va = a.state_by_id()
    qc, vc = c.state_by_id()
    assert np.array_equal(qa, qc) and np.array_equal(va, vc)
    ia, ic = a.info(), c.info()
    assert ia["steps"] == ic["steps"] and ia["rebuilds"] == ic["rebuilds"]
    assert a.observe() == c.observe()


def test_restart_with_piston_executor(tmp_path):
    a, st = system(away_from_z0=True)
    b, _ = system(away_from_z0=True)
    kw = dict(kind=M.EXTERNAL_PISTON, position=st.L[2] - 2.0, velocity=0.004, time_step=0.005)
    a.set_external(**kw)
    b.set_external(**kw)
    a.calculate(60)
    b.calculate(25)
    b.save_checkpoint(tmp_path / "p.ckpt")
    c = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n)
    c.load_checkpoint(tmp_path / "p.ckpt")
    c.calculate(35)
    assert np.array_equal(a.state_by_id()[0], c.state_by_id()[0])
    assert a.external_state() == c.external_state()


def test_checkpoint_right_after_upload(tmp_path):
    a, st = system()
    a.save_checkpoint(tmp_path / "fresh.ckpt")
    c = M.System(st.L, cutoff=2.5, time_step=0.005, capacity=st.n)
    c.load_checkpoint(tmp_path / "fresh.ckpt")
    a.calculate(30)
    c.calculate(30)
    assert np.array_equal(a.state_by_id()[0], c.state_by_id()[0])


def test_checkpoint_rejects_other_box_and_garbage(tmp_path):
    a, st = system()
    a.calculate(5)
    a.save_checkpoint(tmp_path / "x.ckpt")
    other = M.System(st.L * 1.1, cutoff=2.5, time_step=0.005, capacity=st.n)
    with pytest.raises(M.MdgError):
        other.load_checkpoint(tmp_path / "x.ckpt")
    (tmp_path / "junk").write_bytes(b"not a checkpoint" * 10)
    with pytest.raises(M.MdgError) as e:
        a.load_checkpoint(tmp_path / "junk")
    assert e.value.status == -11


def test_async_snapshots_match_state(tmp_path):
    a, st = system()
    types = (np.arange(st.n) % 3).astype(np.int32)
    a.set_state(st.q, st.v, types)
    a.calculate(20)
    q, v, _ = a.state()  # slot order, as the snapshot writes it
    a.snapshot_async(tmp_path / "conf0000.cd", M.SNAPSHOT_CDVIEW)
    a.snapshot_async(tmp_path / "conf000.cnf", M.SNAPSHOT_CONFIGURATION)
    a.calculate(20)  # queued behind the copies; the files hold the step-20 state
    a.snapshot_wait()
    cd = np.loadtxt(tmp_path / "conf0000.cd")
    cnf = np.loadtxt(tmp_path / "conf000.cnf")
    assert cd.shape == (st.n, 8) and cnf.shape == (st.n, 6)
    assert np.all(cd[:, 0] == 0)
    np.testing.assert_allclose(cd[:, 2:5], q, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(cd[:, 5:8], v, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(cnf, np.hstack([q, v]), rtol=1e-5, atol=1e-5)
    assert sorted(cd[:, 1].astype(int)) == sorted(types)
