"""The CPU oracle against the reference's own outputs (fixtures made by
tests/golden/make_golden.py from the reference compiled from its sources).
The restatement follows the reference's arithmetic operation by operation,
so everything here is bit-exact."""
from __future__ import annotations

import numpy as np

from conftest import GOLDEN, pair_set
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


def rankine_rows(count):
    """The oracle running the reference's Rankine loop (src/rankine.cc:101-128:
    Calculate, the piston executor, the piston's move, observation every 50
    steps) from the project's start state; rows as the project prints them."""
    from conftest import rankine_start
    q, v, L = rankine_start()
    n = q.shape[0]
    o = O.Oracle(q, v, np.arange(n, dtype=np.int32), L, 2.5, 0.005)
    o.make_pairlist()
    ox = O.External()
    ox.kind, ox.position, ox.velocity, ox.time_step = 2, L[2] - 2.0, L[2] * 0.5 / 500, 0.005
    rows = []
    for i in range(50 * (count - 1) + 1):
        o.step(1)
        imp = o.apply_external(ox)
        if i % 50 == 0:
            ke, pe, vir = o.observe()
            t = ke / n / 1.5
            rows.append([(i + 1) * 0.005, t, (t - vir / n) * n / L.prod(), ke / n + pe / n, ox.position, imp])
    o.close()
    return rows


def test_oracle_reproduces_reference_rankine_rows():
    # the reference's own output for its Rankine project (piston executor
    # after every step, observers on ghost copies half a step old), compared
    # at the precision it prints: pins the executor and the ghost-lag
    # observers of the oracle to the reference
    text = (GOLDEN / "dropin_rankine_rc25.ref.txt").read_text().splitlines()
    ref = [l.split("#")[0].split() for l in text if "#observe" in l][:4]
    got = [["%g" % x for x in row] for row in rankine_rows(4)]
    assert got == ref
