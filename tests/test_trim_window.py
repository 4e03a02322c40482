"""The list build's trim windows are conservative: for every pair within
SearchLength (exact FP64 minimum image), the partner's row is walked (its
y-z gap passes the skip test) and the partner's x sub-bin lies inside the
row's window [vlo, vhi).  The window arithmetic is restated here in float32
as build_rows computes it (mdacp_b200/csrc/mdg_device.cuh): the prefilter
coordinates (x global, y and z cell-local), the band's upper edge
SL_hi^2 (prefilter_band), the x reach sqrt(SL_hi^2 - g^2) left by the
row's y-z gap g, and the sub-bins counted from each cell's lower face
(sort_cell_x).  Random states at two densities, boxes of 3 to 6 cells per
axis."""
from __future__ import annotations

import numpy as np
import pytest

KXSUB = 8


def band_hi(sl2, sl, lx):
    u = 1.0 / 16777216.0
    rel = max(1e-4, 4.0 * u * (6.0 * lx / sl + 37.0))
    return np.float32(sl2 * (1.0 + rel))


def f32(x):
    return np.float32(x)


def fmaf(a, b, c):
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def sub_bin(x, cell, cs0):
    """Sub-bin of x inside its cell: the number of bin edges cell*cs0 + k*bin
    (k = 1..KXSUB-1) at or below x."""
    x0, b = cell * cs0, cs0 / KXSUB
    return sum(1 for k in range(1, KXSUB) if not (x < x0 + k * b))


@pytest.mark.parametrize("ms,rho,seed", [(3, 0.8442, 1), (4, 0.5, 2), (6, 0.8442, 3), (5, 0.3, 4)])
def test_every_pair_within_the_search_length_is_in_its_row_window(ms, rho, seed):
    rc, bl = 2.5, 0.3
    sl = rc + bl
    cs = sl * 1.02
    L = ms * cs
    n = int(rho * L ** 3)
    rng = np.random.default_rng(seed)
    q = rng.uniform(0.0, L, (n, 3))
    c = np.minimum((q / cs).astype(int), ms - 1)
    hi = band_hi(sl * sl, sl, L)
    per_bin = KXSUB / cs
    checked = 0
    for i in range(n):
        cx, cy, cz = c[i]
        liy, liz = f32(q[i, 1] - cy * cs), f32(q[i, 2] - cz * cs)
        ubin = f32((q[i, 0] - (cx - 1) * cs) * per_bin)
        d = q - q[i]
        shift = -L * np.round(d / L)
        d += shift
        r2 = (d * d).sum(1)
        for j in np.nonzero(r2 <= sl * sl)[0]:
            if j == i:
                continue
            # the partner's cell offsets (the image the pair is found through)
            off = [int(np.floor((q[j, a] + shift[j, a]) / cs)) - c[i, a] for a in range(3)]
            assert all(-1 <= o <= 1 for o in off)
            dxc, dy, dz = off
            gy = f32(0.0) if dy == 0 else (liy if dy < 0 else f32(f32(cs) - liy))
            gz = f32(0.0) if dz == 0 else (liz if dz < 0 else f32(f32(cs) - liz))
            g2 = fmaf(gy, gy, f32(gz * gz))
            assert not (g2 > hi), "row skipped"
            reach = f32(np.sqrt(f32(hi - g2)) * f32(per_bin))
            vbase = (cx - 1) * KXSUB
            vlo = max(vbase + int(np.floor(f32(ubin - reach - f32(1e-3)))), vbase)
            vhi = min(vbase + int(np.floor(f32(ubin + reach + f32(1e-3)))) + 1, vbase + 3 * KXSUB)
            # the partner's virtual sub-bin in the row of cells cx-1 .. cx+1
            v = (cx + dxc) * KXSUB + sub_bin(q[j, 0], c[j, 0], cs)
            assert vlo <= v < vhi, (i, j, vlo, v, vhi)
            checked += 1
    assert checked > 10 * n
