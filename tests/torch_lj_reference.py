"""Dense PyTorch FP64 restatement of the differentiable trajectory (test
infrastructure: the oracle of mdg_adjoint_run).

Same model as mdacp_b200/csrc/mdg_adjoint.cu, written with all pairs and the
minimum image, so that torch.autograd gives the gradients:

    U(r) = eps * phi(r / sigma), phi(s) = 4 (s^-12 - s^-6 + C2 s^2 + C0), s <= s_c
    step:  q_h = q + v dt/2;  v' = v + F(q_h) dt;  q' = q_h + v' dt/2
    loss:  1/(T n) sum_t [ PE(q_t) + sum_pairs g((r - lo)/w) g((hi - r)/w) ]

with phi, C0 and C2 as Variables::Variables forms them (src/variables.cc:
16-33) and the steps of MDManager::Calculate (src/mdmanager.cc:153-186).
Forces are the analytic pair forces (so autograd differentiates them once
more for the reverse sweep); every step is checkpointed so that long
trajectories fit in memory.
"""
from __future__ import annotations

import torch
from torch.utils.checkpoint import checkpoint


def constants(sc: float):
    c2 = 6.0 * sc ** -14 - 3.0 * sc ** -8
    c0 = -sc ** -12 + sc ** -6 - c2 * sc * sc
    return c0, c2


def _pairs(q, L, rc):
    d = q[:, None, :] - q[None, :, :]
    d = d - L * torch.round(d / L)
    r2 = (d * d).sum(-1)
    n = q.shape[0]
    mask = (r2 < rc * rc) & ~torch.eye(n, dtype=torch.bool, device=q.device)
    r = torch.sqrt(torch.where(mask, r2, torch.ones_like(r2)))
    return d, r, mask


def _phi(s, c0, c2):
    return 4.0 * (s ** -12 - s ** -6 + c2 * s * s + c0)


def _dphi(s, c2):
    return 4.0 * (-12.0 * s ** -13 + 6.0 * s ** -7 + 2.0 * c2 * s)


def forces(q, L, eps, sigma, sc):
    c0, c2 = constants(sc)
    d, r, mask = _pairs(q, L, sc * sigma)
    u1 = torch.where(mask, eps / sigma * _dphi(r / sigma, c2), torch.zeros_like(r))
    return (-(u1 / r)[..., None] * d).sum(1)


def loss_terms(q, L, eps, sigma, sc, shell):
    c0, c2 = constants(sc)
    lo, hi, w = shell
    d, r, mask = _pairs(q, L, sc * sigma)
    u = torch.where(mask, eps * _phi(r / sigma, c0, c2), torch.zeros_like(r))
    g = torch.sigmoid((r - lo) / w) * torch.sigmoid((hi - r) / w)
    s = torch.where(mask, g, torch.zeros_like(r))
    return 0.5 * (u.sum() + s.sum())


def _step(q, v, L, eps, sigma, sc, dt):
    qh = q + v * (0.5 * dt)
    v2 = v + forces(qh, L, eps, sigma, sc) * dt
    return qh + v2 * (0.5 * dt), v2


def trajectory_loss(q0, v0, L, eps, sigma, steps, dt=0.005, sc=2.5, shell=(1.0, 1.5, 0.05), use_checkpoint=True):
    """Loss of the trajectory from (q0, v0); every argument may be a tensor
    that requires grad (L a float or a length-3 tensor)."""
    q, v = q0, v0
    total = torch.zeros((), dtype=torch.float64, device=q0.device)
    for _ in range(steps):
        if use_checkpoint:
            q, v = checkpoint(_step, q, v, L, eps, sigma, sc, dt, use_reentrant=False)
            total = total + checkpoint(loss_terms, q, L, eps, sigma, sc, shell, use_reentrant=False)
        else:
            q, v = _step(q, v, L, eps, sigma, sc, dt)
            total = total + loss_terms(q, L, eps, sigma, sc, shell)
    return total / (steps * q0.shape[0])
