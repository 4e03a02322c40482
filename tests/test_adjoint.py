"""Gradients of the trajectory loss (mdg_adjoint_run) against central finite
differences (h = 1e-6) and against the dense PyTorch FP64 autograd
restatement (tests/torch_lj_reference.py).

Bars: 1e-8 relative against autograd of the same discrete model (the exact
derivative, up to summation order); 1e-6 relative against finite
differences at the 32,000-atom size.  The smoothed potential is only C^1 at
the cut-off (U'' jumps by about 0.12 there), so every pair that crosses the
cut-off during the trajectory puts a kink into L(sigma); a central
difference that straddles one is off by the kink's share.  At 500 atoms a
kink lies within 1e-6 of sigma = 1 (the difference shrinks from 1.5e-6 at
h = 1e-6 to 2e-8 at h = 1e-7), so the 500-atom sigma check allows 5e-6; at
32,000 atoms the kinks average out (3e-8)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from mdacp_b200 import workloads as W
import torch_lj_reference as R

H = 1e-6
FD_TOL = 1e-6


def small_state(ncell=5, seed=55, jitter=0.05):
    st = W.fcc_liquid(ncell, 0.8442, 1.0, seed, jitter=jitter, rc=2.5, dt=0.005)
    return st.q, st.v, st.L


def test_torch_reference_matches_finite_differences():
    # the oracle itself, on the CPU: autograd through 10 steps of 108 atoms
    q0, v0, L = small_state(ncell=3, seed=7)
    q = torch.tensor(q0, dtype=torch.float64, requires_grad=True)
    v = torch.tensor(v0, dtype=torch.float64)
    eps = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    Lt = torch.tensor(L, dtype=torch.float64)
    loss = R.trajectory_loss(q, v, Lt, eps, sig, steps=10)
    gq, ge, gs = torch.autograd.grad(loss, (q, eps, sig))
    rng = np.random.default_rng(3)
    d = rng.standard_normal(q0.shape)
    d /= np.linalg.norm(d)

    def f(qq, e, s):
        with torch.no_grad():
            return float(R.trajectory_loss(torch.tensor(qq), v, Lt, torch.tensor(e, dtype=torch.float64),
                                           torch.tensor(s, dtype=torch.float64), steps=10, use_checkpoint=False))

    fd_e = (f(q0, 1 + H, 1.0) - f(q0, 1 - H, 1.0)) / (2 * H)
    fd_s = (f(q0, 1.0, 1 + H) - f(q0, 1.0, 1 - H)) / (2 * H)
    fd_d = (f(q0 + H * d, 1.0, 1.0) - f(q0 - H * d, 1.0, 1.0)) / (2 * H)
    assert float(ge) == pytest.approx(fd_e, rel=FD_TOL)
    assert float(gs) == pytest.approx(fd_s, rel=FD_TOL)
    assert float((gq.numpy() * d).sum()) == pytest.approx(fd_d, rel=FD_TOL)


def _gpu_grads(q0, v0, L, **kw):
    from mdacp_b200 import adjoint as A
    return A.trajectory_gradients(q0, v0, L, **kw)


@pytest.mark.gpu
def test_adjoint_matches_dense_torch_autograd():
    q0, v0, L = small_state()  # 500 atoms, L = 8.40
    loss, de, ds, dq = _gpu_grads(q0, v0, L, steps=200, checkpoint_every=20)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    q = torch.tensor(q0, dtype=torch.float64, device=dev, requires_grad=True)
    v = torch.tensor(v0, dtype=torch.float64, device=dev)
    eps = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, device=dev, requires_grad=True)
    ref = R.trajectory_loss(q, v, torch.tensor(L, dtype=torch.float64, device=dev), eps, sig, steps=200)
    gq, ge, gs = torch.autograd.grad(ref, (q, eps, sig))
    assert loss == pytest.approx(float(ref.detach()), rel=1e-11)
    assert de == pytest.approx(float(ge), rel=1e-8)
    assert ds == pytest.approx(float(gs), rel=1e-8)
    gq = gq.cpu().numpy()
    assert np.linalg.norm(dq - gq) <= 1e-8 * np.linalg.norm(gq)


@pytest.mark.gpu
@pytest.mark.parametrize("size", ["n500", "n32000"])
def test_adjoint_matches_finite_differences(size):
    from mdacp_b200 import adjoint as A
    if size == "n500":
        q0, v0, L = small_state()
    else:
        st = W.config_c5()
        q0, v0, L = st.q, st.v, st.L
    kw = dict(steps=200, checkpoint_every=20)
    loss, de, ds, dq = A.trajectory_gradients(q0, v0, L, **kw)
    f = lambda qq, e=1.0, s=1.0: A.trajectory_loss(qq, v0, L, epsilon=e, sigma=s, **kw)  # noqa: E731
    fd_e = (f(q0, 1 + H) - f(q0, 1 - H)) / (2 * H)
    fd_s = (f(q0, 1.0, 1 + H) - f(q0, 1.0, 1 - H)) / (2 * H)
    assert loss == f(q0)
    assert de == pytest.approx(fd_e, rel=FD_TOL)
    assert ds == pytest.approx(fd_s, rel=FD_TOL if size == "n32000" else 5e-6)
    # initial positions: along the gradient itself (the largest directional
    # derivative, |dL/dq0|), and along a random unit direction, whose
    # derivative is about 40 times smaller at 32,000 atoms, so that rounding
    # noise of the loss (~1e-15 after 200 steps) limits its difference
    # quotient to a few 1e-6
    g = dq / np.linalg.norm(dq)
    fd_g = (f(q0 + H * g) - f(q0 - H * g)) / (2 * H)
    assert float(np.linalg.norm(dq)) == pytest.approx(fd_g, rel=FD_TOL)
    d = np.random.default_rng(11).standard_normal(q0.shape)
    d /= np.linalg.norm(d)
    fd_d = (f(q0 + H * d) - f(q0 - H * d)) / (2 * H)
    assert float((dq * d).sum()) == pytest.approx(fd_d, rel=1e-5)


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_gradients():
    q0, v0, L = small_state()
    a = _gpu_grads(q0, v0, L, steps=60, checkpoint_every=20)
    b = _gpu_grads(q0, v0, L, steps=60, checkpoint_every=7)
    c = _gpu_grads(q0, v0, L, steps=60, checkpoint_every=60)
    for x, y in ((a, b), (a, c)):
        assert x[0] == y[0] and x[1] == y[1] and x[2] == y[2]
        assert np.array_equal(x[3], y[3])


@pytest.mark.gpu
def test_autograd_function_backpropagates():
    from mdacp_b200 import adjoint as A
    q0, v0, L = small_state()
    q = torch.tensor(q0, dtype=torch.float64, requires_grad=True)
    eps = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    opts = {"steps": 40, "checkpoint_every": 10}
    out = 3.0 * A.TrajectoryLoss.apply(q, eps, sig, torch.tensor(v0), tuple(L), opts)
    out.backward()
    loss, de, ds, dq = _gpu_grads(q0, v0, L, **opts)
    assert float(out.detach()) == pytest.approx(3.0 * loss, rel=1e-15)
    assert float(eps.grad) == pytest.approx(3.0 * de, rel=1e-15)
    assert float(sig.grad) == pytest.approx(3.0 * ds, rel=1e-15)
    assert np.allclose(q.grad.numpy(), 3.0 * dq, rtol=1e-15, atol=0.0)


@pytest.mark.gpu
def test_repeated_runs_reuse_the_kept_device_memory():
    # the second run of a shape allocates nothing (device free memory is
    # unchanged) and gives the same numbers; release() frees the workspace
    # and the next run allocates it again
    from mdacp_b200 import adjoint as A
    q0, v0, L = small_state(ncell=8)  # 2,048 atoms
    kw = dict(steps=60, checkpoint_every=10)
    a = _gpu_grads(q0, v0, L, **kw)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    b = _gpu_grads(q0, v0, L, **kw)
    torch.cuda.synchronize()
    free2, _ = torch.cuda.mem_get_info()
    assert free2 == free1
    assert a[0] == b[0] and a[1] == b[1] and a[2] == b[2] and np.array_equal(a[3], b[3])
    A.release()
    c = _gpu_grads(q0, v0, L, **kw)
    assert c[0] == a[0] and np.array_equal(c[3], a[3])


@pytest.mark.gpu
def test_rejects_box_below_three_cells():
    from mdacp_b200 import MdgError
    q0, v0, L = small_state(ncell=3)  # L = 5.04 < 3 cut-offs
    with pytest.raises(MdgError):
        _gpu_grads(q0, v0, L, steps=2)


@pytest.mark.gpu
def test_lanes_per_atom_only_regroup_the_sums():
    # 1, 2, 4 or 8 lanes per atom split each atom's row differently (lane =
    # partner index mod lanes), so only the grouping of the FP64 sums changes
    q0, v0, L = small_state()
    runs = [_gpu_grads(q0, v0, L, steps=40, checkpoint_every=10, threads_per_atom=t) for t in (1, 2, 4, 8)]
    for r in runs[1:]:
        assert r[0] == pytest.approx(runs[0][0], rel=1e-12)
        assert r[1] == pytest.approx(runs[0][1], rel=1e-9)
        assert r[2] == pytest.approx(runs[0][2], rel=1e-9)
        assert np.linalg.norm(r[3] - runs[0][3]) <= 1e-9 * np.linalg.norm(runs[0][3])
    with pytest.raises(Exception):
        _gpu_grads(q0, v0, L, steps=2, threads_per_atom=3)
