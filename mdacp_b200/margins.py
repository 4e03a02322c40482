"""Per-replica pairlist margins (BufferLength) for replica ensembles.

The reference runs every system with one BufferLength (0.3,
src/simulationinfo.cc:6-7); the ensemble keeps that by default, and parity
runs keep it.  A replica's margin m trades list length against rebuild
frequency: its neighbour rows, and the candidates a rebuild walks, grow as
(cutoff + m)^3, while the steps between rebuilds grow about as m (the skin
budget m is spent at 2 vmax dt per step).  Per step and per atom, relative
to the force pass at the common margin m0,

    cost(m) = ((rc + m) / (rc + m0))^3 * (1 + c * rate * m0 / m)

with ``rate`` the replica's rebuilds per step measured at m0 and ``c`` the
cost of one rebuild of an atom's row in units of one force-pass row.
:func:`choose_margins` minimises this per replica on a grid;
:func:`tune_margins` measures the rates on the device, tries a few values
of ``c`` and keeps the margins whose ensemble ran fastest (the common
margin included), as the force and build autotuners keep the fastest
launch shape.
"""
from __future__ import annotations

import numpy as np


def choose_margins(boxes, cutoff, buffer_length, rates, c, grid=None):
    """Margin per replica minimising the cost model above.

    ``boxes``: (n_atoms, L) per replica; ``rates``: rebuilds per step at
    ``buffer_length``; ``c``: rebuild cost per row in force-pass rows
    (0 keeps ``buffer_length`` everywhere).  Margins keep every box above
    two search lengths and leave a replica with three or more cells per
    axis with three or more (the cell walk), one with fewer with fewer
    (the all-pairs search)."""
    m0 = float(buffer_length)
    rates = np.asarray(rates, dtype=np.float64)
    if len(boxes) != rates.shape[0]:
        raise ValueError("one rate per replica")
    if grid is None:
        grid = np.round(np.arange(0.1, 1.2001, 0.025), 6)
    grid = np.asarray(grid, dtype=np.float64)
    out = np.full(len(boxes), m0)
    if c <= 0.0:
        return out
    for k, ((_, L), rate) in enumerate(zip(boxes, rates)):
        L = np.asarray(L, dtype=np.float64)
        small0 = int(np.min(np.floor(L / (cutoff + m0)))) < 3
        best, best_cost = m0, None
        for m in grid:
            sl = cutoff + m
            if not np.all(L > 2.0 * sl):
                continue
            if (int(np.min(np.floor(L / sl))) < 3) != small0:
                continue
            cost = ((cutoff + m) / (cutoff + m0)) ** 3 * (1.0 + c * max(rate, 0.0) * m0 / m)
            if best_cost is None or cost < best_cost:
                best, best_cost = float(m), cost
        out[k] = best
    return out


def _timed_run(M, states, margins, cutoff, time_step, precision, buffer_length, device, warm, steps):
    import torch

    ens = M.Ensemble(states, cutoff=cutoff, time_step=time_step, precision=precision, device=device,
                     buffer_length=buffer_length, buffer_lengths=margins)
    try:
        ens.calculate(warm)
        r0, _ = ens.rebuilds()
        stream = torch.cuda.ExternalStream(ens.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        ens.calculate(steps)
        e1.record(stream)
        e1.synchronize()
        r1, _ = ens.rebuilds()
        ms = e0.elapsed_time(e1)
    finally:
        ens.close()
    return ms, (r1 - r0).astype(np.float64)


def tune_margins(states, cutoff=2.5, time_step=0.005, precision=None, buffer_length=0.3, device=0,
                 warm_steps=100, trial_steps=200, costs=(3.0, 6.0, 12.0, 24.0)):
    """Per-replica margins for ``states`` ((q, v, L) per replica), chosen by
    timing.  The common margin runs first and gives each replica's rebuild
    rate; each ``c`` in ``costs`` gives one margin set (choose_margins),
    timed over ``trial_steps`` steps after ``warm_steps``; the fastest set
    is returned with a report of every trial."""
    import mdacp_b200 as M

    if precision is None:
        precision = M.FP32_MIXED
    boxes = [(q.shape[0], L) for q, _, L in states]
    atoms = sum(n for n, _ in boxes)
    base = np.zeros(len(states))
    ms, rb = _timed_run(M, states, base, cutoff, time_step, precision, buffer_length, device, warm_steps,
                        trial_steps)
    rates = np.maximum(rb, 0.5) / trial_steps
    trials = [{"c": 0.0, "ms_per_step": ms / trial_steps, "rebuilds": float(rb.sum())}]
    best_ms, best = ms, np.full(len(states), float(buffer_length))
    for c in costs:
        m = choose_margins(boxes, cutoff, buffer_length, rates, c)
        ms_c, rb_c = _timed_run(M, states, m, cutoff, time_step, precision, buffer_length, device,
                                warm_steps, trial_steps)
        trials.append({"c": float(c), "ms_per_step": ms_c / trial_steps, "rebuilds": float(rb_c.sum()),
                       "margin_min": float(m.min()), "margin_median": float(np.median(m)),
                       "margin_max": float(m.max())})
        if ms_c < best_ms:
            best_ms, best = ms_c, m
    report = {"atoms": atoms, "trial_steps": trial_steps, "warm_steps": warm_steps, "trials": trials,
              "chosen_ms_per_step": best_ms / trial_steps}
    return best, report
