"""Known answers for the oracle that do not need the reference: analytic
two-atom forces of the smoothed potential, V and F vanishing at the cut-off,
zero net force on a perfect lattice, and the published Philox4x32-10
known-answer vectors (Random123)."""
from __future__ import annotations

import math

import numpy as np
import pytest

from mdacp_b200 import workloads as W
from oracle import lj_oracle as O


def smoothed(r, rc):
    s2 = 1.0 / (rc * rc)
    s6 = s2 ** 3
    c2 = 6.0 * s6 * s6 * s2 - 3.0 * s6 * s2
    c0 = -s6 * s6 + s6 - c2 / s2
    v = 4.0 * (r ** -12 - r ** -6 + c2 * r * r + c0)
    f = 48.0 * r ** -13 - 24.0 * r ** -7 - 8.0 * c2 * r  # -dV/dr
    return v, f


@pytest.mark.parametrize("r", [0.95, 1.0, 1.12246, 1.5, 2.2, 2.49])
def test_two_atoms(r):
    L = np.array([12.0, 12.0, 12.0])
    q = np.array([[5.0, 6.0, 6.0], [5.0 + r, 6.0, 6.0]])
    v = np.zeros((2, 3))
    o = O.Oracle(q, v, np.arange(2, dtype=np.int32), L, 2.5, 0.005)
    o.make_pairlist()
    f = o.forces()
    _, ids = o.state()[1:]
    fa = f[np.argsort(ids)]
    vr, fr = smoothed(r, 2.5)
    assert fa[1, 0] == pytest.approx(fr, rel=1e-12, abs=1e-12)
    assert fa[0, 0] == pytest.approx(-fr, rel=1e-12, abs=1e-12)
    ke, pe, vir = o.observe()
    assert pe == pytest.approx(vr, rel=1e-12, abs=1e-13)
    assert vir == pytest.approx(-fr * r / 3.0, rel=1e-12, abs=1e-13)


def test_vanishes_at_cutoff():
    for rc in (2.5, 3.0):
        v, f = smoothed(rc, rc)
        assert abs(v) < 1e-14 and abs(f) < 1e-14


def test_pair_across_the_boundary():
    L = np.array([12.0, 12.0, 12.0])
    q = np.array([[0.3, 6.0, 6.0], [11.4, 6.0, 6.0]])  # 0.9 apart through x = 0
    o = O.Oracle(q, np.zeros((2, 3)), np.arange(2, dtype=np.int32), L, 2.5, 0.005)
    o.make_pairlist()
    k, p = o.pairs()
    assert sorted(zip(k.tolist(), p.tolist())) == [(0, 1), (1, 0)]
    f = o.forces()[np.argsort(o.state()[2])]
    _, fr = smoothed(0.9, 2.5)
    assert f[0, 0] == pytest.approx(fr, rel=1e-9)
    assert f[1, 0] == pytest.approx(-fr, rel=1e-9)


def test_lattice_net_force_zero():
    s = W.fcc_liquid(5, 0.8442, 1.0, seed=1, rc=2.5)
    o = O.Oracle(s.q, s.v, s.ids, s.L, 2.5, 0.004)
    o.make_pairlist()
    f = o.forces()
    assert np.abs(f).max() < 1e-10


def test_philox_known_answers():
    assert O.philox4x32([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert O.philox4x32([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert O.philox4x32([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_langevin_normals_distribution():
    z = np.array([O.langevin_normals(7, i, s) for i in range(2000) for s in range(3)]).ravel()
    assert abs(z.mean()) < 0.05
    assert abs(z.std() - 1.0) < 0.05


def test_langevin_thermostat_reaches_temperature():
    s = W.fcc_liquid(5, 0.5, 0.5, seed=3, jitter=0.05, rc=2.5, dt=0.005)
    o = O.Oracle(s.q, s.v, s.ids, s.L, 2.5, 0.005, thermostat=O.LANGEVIN, temperature=1.2, gamma=1.0, seed=9)
    o.make_pairlist()
    o.step(600)
    ke, _, _ = o.observe()
    t = ke / o.n / 1.5
    assert 1.0 < t < 1.4
