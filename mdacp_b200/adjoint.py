"""Gradients of an LJ trajectory loss through the C ABI (mdg_adjoint_run).

The loss and its gradients come from mdacp_b200/csrc/mdg_adjoint.cu: a
forward pass of drift-kick-drift steps in FP64 with checkpoints every k
steps, and a hand-written reverse sweep (pair-Hessian-vector products over
the cell grid, segments recomputed from the checkpoints).

    loss, d_eps, d_sigma, d_q0 = trajectory_gradients(q0, v0, L, steps=200)

`TrajectoryLoss` wraps the same call as a torch.autograd.Function, so that a
torch program can backpropagate into epsilon, sigma and the initial positions
(the velocities are held fixed).  The loss is

    L = 1/(T n) sum_{t=1..T} [ PE(q_t) + sum_pairs g((r - lo)/w) g((hi - r)/w) ]

with U(r) = epsilon phi(r/sigma), phi the reference's smoothed 12-6
potential (src/variables.cc:16-33), the cut-off in units of sigma, and g the
logistic function.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import AdjointParams, MdgError, load_library

__all__ = ["params", "trajectory_loss", "trajectory_gradients", "TrajectoryLoss"]

_DP = ctypes.POINTER(ctypes.c_double)


def params(L, steps=200, checkpoint_every=20, time_step=0.005, epsilon=1.0, sigma=1.0, cutoff=2.5,
           shell=(1.0, 1.5, 0.05), threads_per_atom=0, device=0) -> AdjointParams:
    lib = load_library()
    p = AdjointParams()
    lib.mdg_adjoint_default_params(ctypes.byref(p))
    p.L[:] = [float(x) for x in np.broadcast_to(np.asarray(L, dtype=np.float64), (3,))]
    p.steps = int(steps)
    p.checkpoint_every = int(checkpoint_every)
    p.time_step = float(time_step)
    p.epsilon = float(epsilon)
    p.sigma = float(sigma)
    p.cutoff = float(cutoff)
    p.shell_lo, p.shell_hi, p.shell_width = (float(x) for x in shell)
    p.threads_per_atom = int(threads_per_atom)
    p.device = int(device)
    return p


def _run(p: AdjointParams, q0, v0, grad: bool):
    lib = load_library()
    q = np.ascontiguousarray(q0, dtype=np.float64).reshape(-1, 3)
    v = np.ascontiguousarray(v0, dtype=np.float64).reshape(-1, 3)
    n = q.shape[0]
    loss = ctypes.c_double()
    de, ds = ctypes.c_double(), ctypes.c_double()
    dq = np.zeros((n, 3), dtype=np.float64)
    if grad:
        st = lib.mdg_adjoint_run(ctypes.byref(p), q.ctypes.data_as(_DP), v.ctypes.data_as(_DP), n,
                                 ctypes.byref(loss), ctypes.byref(de), ctypes.byref(ds), dq.ctypes.data_as(_DP))
    else:
        st = lib.mdg_adjoint_run(ctypes.byref(p), q.ctypes.data_as(_DP), v.ctypes.data_as(_DP), n,
                                 ctypes.byref(loss), None, None, None)
    if st != 0:
        raise MdgError(st, lib.mdg_status_string(st).decode())
    if not grad:
        return loss.value
    return loss.value, de.value, ds.value, dq


def trajectory_loss(q0, v0, L, **kw) -> float:
    """Forward pass only: the loss of the trajectory from (q0, v0)."""
    return _run(params(L, **kw), q0, v0, grad=False)


def trajectory_gradients(q0, v0, L, **kw):
    """(loss, dL/d epsilon, dL/d sigma, dL/d q0 as an n x 3 array)."""
    return _run(params(L, **kw), q0, v0, grad=True)


def release():
    """Frees the device memory the adjoint keeps between runs (mdg_adjoint_release)."""
    load_library().mdg_adjoint_release()


try:
    import torch

    class TrajectoryLoss(torch.autograd.Function):
        """loss = TrajectoryLoss.apply(q0, epsilon, sigma, v0, L, options):
        q0 (n, 3), epsilon and sigma 0-d float64 tensors, v0 (n, 3) held
        fixed, options a dict of `params` keywords (steps, checkpoint_every,
        time_step, cutoff, shell, device)."""

        @staticmethod
        def forward(ctx, q0, epsilon, sigma, v0, L, options):
            opts = dict(options or {})
            loss, de, ds, dq = trajectory_gradients(
                q0.detach().cpu().double().numpy(), v0.detach().cpu().double().numpy(), L,
                epsilon=float(epsilon), sigma=float(sigma), **opts)
            ctx.save_for_backward(torch.as_tensor(dq, dtype=q0.dtype, device=q0.device),
                                  torch.tensor(de, dtype=torch.float64), torch.tensor(ds, dtype=torch.float64))
            return torch.tensor(loss, dtype=torch.float64, device=q0.device)

        @staticmethod
        def backward(ctx, g):
            dq, de, ds = ctx.saved_tensors
            g = g.detach()
            return (g * dq, (g.cpu() * de).to(g.dtype), (g.cpu() * ds).to(g.dtype), None, None, None)

except ImportError:  # pragma: no cover - torch is optional for the ctypes calls
    TrajectoryLoss = None
