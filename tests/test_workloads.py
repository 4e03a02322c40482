"""Seeded workload generators: sizes, densities, temperatures, momentum,
overlap rejection and determinism."""
from __future__ import annotations

import numpy as np
import pytest

from mdacp_b200 import workloads as W


def test_fcc_liquid_density_and_temperature():
    s = W.fcc_liquid(5, 0.8442, 0.722, seed=1)
    assert s.n == 500
    assert s.n / np.prod(s.L) == pytest.approx(0.8442)
    assert np.abs(s.v.sum(axis=0)).max() < 1e-10
    assert (s.v ** 2).sum() / (3 * s.n) == pytest.approx(0.722)
    assert ((s.q >= 0) & (s.q < s.L)).all()


def test_generators_are_deterministic():
    a = W.fcc_liquid(4, 0.5, 1.0, seed=9, jitter=0.05)
    b = W.fcc_liquid(4, 0.5, 1.0, seed=9, jitter=0.05)
    assert np.array_equal(a.q, b.q) and np.array_equal(a.v, b.v)


def test_config_c1_and_c2_shapes():
    c1 = W.config_c1()
    assert c1.n == 32000 and np.array_equal(c1.L, [40.0, 40.0, 40.0])


def test_slab_overlap_rejection_and_layout():
    s = W.slab(3000, 0.75, 0.02, 0.9, seed=5)
    from scipy.spatial import cKDTree

    t = cKDTree(np.minimum(np.mod(s.q, s.L), np.nextafter(s.L, 0)), boxsize=s.L)
    d, _ = t.query(np.minimum(np.mod(s.q, s.L), np.nextafter(s.L, 0)), k=2)
    assert d[:, 1].min() >= 0.9 - 1e-12
    assert s.L[2] == pytest.approx(4 * s.L[0])
    z = s.q[:, 2]
    liquid = ((z >= 0.375 * s.L[2]) & (z < 0.625 * s.L[2])).sum()
    assert liquid == pytest.approx(0.75 * s.L[0] * s.L[1] * 0.25 * s.L[2], rel=0.01)


def test_config_c4_replicas():
    reps = W.config_c4(nrep=16)
    assert len(reps) == 16
    for r in reps:
        assert 400 <= r.n <= 24000
        assert (r.L > 2 * 2.8).all()
        rho = r.n / np.prod(r.L)
        assert 0.29 <= rho <= 0.91
