"""The slab decomposition (mdg_slabs_*) against the single-domain handle:
one periodic system split into 2 or 3 z-slabs of cell layers (here all on
one GPU, exchanging their ghost layers by device-to-device copies) must
reproduce the single domain: the same forces and trajectory bit for bit
(every slab walks the same atoms in the same order), the same rebuild
steps, and observer sums within 1e-12 (summed per slab, then over slabs).
Atoms cross slab boundaries and migrate along the way."""
from __future__ import annotations

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _pair(st, nslabs, precision, steps):
    a = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=precision)
    a.set_state(st.q, st.v)
    b = M.Slabs(st.L, nslabs, cutoff=st.rc, time_step=st.dt, capacity=st.n, precision=precision)
    b.set_state(st.q, st.v)
    fa, fb = a.forces_by_id(), b.forces_by_id()
    a.calculate(steps)
    b.calculate(steps)
    return a, b, fa, fb


@pytest.mark.parametrize("nslabs", [2, 3])
@pytest.mark.parametrize("precision", [M.FP64, M.FP32_MIXED])
def test_slabs_reproduce_single_domain(nslabs, precision):
    # 8 x 8 x 12 FCC cells at rho 0.8442: 4 x 4 x 7 search cells, hot enough
    # for several rebuilds and for atoms to change slab
    st = W.fcc_liquid((8, 8, 12), 0.8442, 1.4, seed=81, jitter=0.05, rc=2.5, dt=0.005)
    a, b, fa, fb = _pair(st, nslabs, precision, 200)
    assert np.array_equal(fa, fb)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    ia, ib = a.info(), b.info()
    assert ib["steps"] == 200 and ib["rebuilds"] == ia["rebuilds"] and ia["rebuilds"] >= 3
    assert sum(ib["owned"]) == st.n and min(ib["ghosts"]) > 0
    ka, pa, wa = a.observe()
    kb, pb, wb = b.observe()
    assert kb == pytest.approx(ka, rel=1e-12)
    assert pb == pytest.approx(pa, rel=1e-12)
    assert wb == pytest.approx(wa, rel=1e-12)


def test_one_layer_slabs_and_migration():
    # as many slabs as there are layers along z (one layer each): every
    # rebuild migrates atoms and every ghost layer is a neighbour's whole slab
    st = W.fcc_liquid((6, 6, 7), 0.7, 1.2, seed=82, jitter=0.06, rc=2.5, dt=0.005)
    nz = int(st.L[2] / 2.8)
    a, b, fa, fb = _pair(st, nz, M.FP64, 120)
    assert np.array_equal(fa, fb)
    qa, va = a.state_by_id()
    qb, vb = b.state_by_id()
    assert np.array_equal(qa, qb) and np.array_equal(va, vb)
    assert b.info()["rebuilds"] == a.info()["rebuilds"]


def test_slabs_reject_bad_layouts():
    st = W.fcc_liquid(6, 0.8442, 1.0, seed=83, rc=2.5)
    with pytest.raises(M.MdgError):
        M.Slabs(st.L, 1, capacity=st.n)                 # at least 2 slabs
    with pytest.raises(M.MdgError):
        M.Slabs(st.L, 50, capacity=st.n)                # more slabs than layers
