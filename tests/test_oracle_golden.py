"""The CPU oracle against the reference's own outputs (fixtures made by
tests/golden/make_golden.py from the reference compiled from its sources).
The restatement follows the reference's arithmetic operation by operation,
so everything here is bit-exact."""
from __future__ import annotations

import numpy as np

from conftest import pair_set
from oracle import lj_oracle as O


def _oracle_for(g, thermostat=O.NVE, **kw):
    return O.Oracle(g["q"], g["v"], g["ids"], g["L"], float(g["rc"]), float(g["dt"]),
                    thermostat=thermostat, **kw)


def test_pairs_bit_exact(golden):
    o = _oracle_for(golden)
    o.make_pairlist()
    k, p = o.pairs()
    assert np.array_equal(pair_set(k, p), golden["pairs"].astype(np.int64))


def test_forces_bit_exact(golden):
    o = _oracle_for(golden)
    o.make_pairlist()
    f = o.forces()
    _, _, ids = o.state()
    out = np.empty_like(f)
    out[ids] = f
    assert np.array_equal(out, golden["forces"])


def test_observers_bit_exact(golden):
    o = _oracle_for(golden)
    o.make_pairlist()
    ke, pe, vir = o.observe()
    n = golden["q"].shape[0]
    # the fixture holds KE/N and PE/N as MDManager returns them, times N
    assert ke / n == golden["ke"] / n
    assert pe / n == golden["pe"] / n
    assert vir == golden["virial"]


def test_trajectory_bit_exact(golden):
    nh = str(golden["thermostat"]) == "NoseHoover"
    kw = {}
    if nh:
        kw = dict(temperature=float(golden["aimed_temperature"]), tau=float(golden["heatbath_tau"]))
    o = _oracle_for(golden, thermostat=O.NOSE_HOOVER if nh else O.NVE, **kw)
    o.make_pairlist()
    o.step(int(golden["steps"]))
    q, v, ids = o.state()
    qo = np.empty_like(q)
    vo = np.empty_like(v)
    qo[ids] = q
    vo[ids] = v
    assert np.array_equal(qo, golden["traj_q"])
    assert np.array_equal(vo, golden["traj_v"])
    assert o.constructions == int(golden["constructions"])
