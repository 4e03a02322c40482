"""Seeded synthetic initial states for the LJ timestep workloads.

The reference builds its starting states inside its Projects
(``ConfigurationMaker`` / ``ExtractConfigurationMaker``, src/confmaker.cc:8-254,
and ``Variables::SetInitialVelocity``, src/variables.cc:86-113).  The
workloads measured here instead use seeded generators with the sizes and
distributions of the benchmark configurations:

* ``fcc_liquid``  FCC lattice (4 atoms per cubic cell, lattice constant
  ``a = (4/rho)^(1/3)``), Maxwell-Boltzmann velocities at temperature ``T``
  with zero total momentum, rescaled to exactly ``T``.
* ``slab``  a liquid slab in the middle quarter of a 1:1:4 box plus vapour
  elsewhere, uniform random positions with overlaps below ``r_min`` rejected.

Every generator is deterministic for a given seed (numpy ``Philox`` bit
generator).  Positions lie in ``[0, L)``.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

__all__ = [
    "State",
    "fcc_positions",
    "maxwell_boltzmann",
    "fcc_liquid",
    "slab",
    "lattice_constant",
    "config_c1",
    "config_c2",
    "config_c3",
    "config_c5",
]


@dataclasses.dataclass
class State:
    """A periodic LJ system: positions ``q`` (n,3), velocities ``v`` (n,3),
    integer ids ``ids`` (n,), box ``L`` (3,) and the run parameters."""

    q: np.ndarray
    v: np.ndarray
    ids: np.ndarray
    L: np.ndarray
    rc: float = 2.5
    dt: float = 0.005
    temperature: float = 1.0
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.q.shape[0])


def lattice_constant(rho: float) -> float:
    """FCC cubic-cell edge for number density ``rho`` (4 atoms per cell)."""
    return (4.0 / rho) ** (1.0 / 3.0)


def fcc_positions(ncells, a: float, offset: float = 0.25) -> np.ndarray:
    """FCC sites of an ``nx x ny x nz`` block of cubic cells of edge ``a``.

    Sites sit at ``(i + b + offset) * a`` with the four basis vectors ``b``;
    the default offset keeps every site a quarter cell away from the faces.
    """
    nx, ny, nz = (ncells, ncells, ncells) if np.isscalar(ncells) else ncells
    basis = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    cells = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
    q = (cells[:, None, :] + basis[None, :, :] + offset) * a
    return q.reshape(-1, 3)


def maxwell_boltzmann(n: int, temperature: float, rng: np.random.Generator) -> np.ndarray:
    """Unit-mass Maxwell-Boltzmann velocities with zero total momentum, rescaled
    so that sum(v^2)/(3n) equals ``temperature`` exactly (the reference's
    Temperature() is KE/N/1.5, src/mdmanager.cc:530-548)."""
    v = rng.standard_normal((n, 3)) * math.sqrt(temperature)
    if n > 1:
        v -= v.mean(axis=0)
    t_now = float((v * v).sum()) / (3.0 * max(n, 1))
    if t_now > 0.0:
        v *= math.sqrt(temperature / t_now)
    return v


def fcc_liquid(ncells, rho: float, temperature: float, seed: int, jitter: float = 0.0,
               rc: float = 2.5, dt: float = 0.005, name: str = "") -> State:
    """FCC start of ``4*nx*ny*nz`` atoms at density ``rho``; ``jitter`` is the
    half-width of a uniform displacement in units of the lattice constant."""
    nx, ny, nz = (ncells, ncells, ncells) if np.isscalar(ncells) else ncells
    a = lattice_constant(rho)
    rng = np.random.Generator(np.random.Philox(seed))
    q = fcc_positions((nx, ny, nz), a)
    L = np.array([nx * a, ny * a, nz * a], dtype=np.float64)
    if jitter > 0.0:
        q = q + rng.uniform(-jitter * a, jitter * a, size=q.shape)
        q = np.mod(q, L)
        q = np.where(q >= L, q - L, q)
    v = maxwell_boltzmann(q.shape[0], temperature, rng)
    ids = np.arange(q.shape[0], dtype=np.int32)
    return State(q=np.ascontiguousarray(q), v=np.ascontiguousarray(v), ids=ids, L=L, rc=rc,
                 dt=dt, temperature=temperature, name=name)


def _rsa_fill(rng, lo, hi, count, r_min, existing=None, batch=None):
    """Random sequential addition of ``count`` points uniformly in the box
    ``[lo, hi)`` with no two points (including ``existing``) closer than
    ``r_min``.  Candidates are tested in batches against a cell grid."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    width = hi - lo
    ncell = np.maximum(1, np.floor(width / r_min).astype(np.int64))
    csize = width / ncell
    slots = 8
    grid = np.full((ncell[0], ncell[1], ncell[2], slots), -1, dtype=np.int64)
    fill = np.zeros((ncell[0], ncell[1], ncell[2]), dtype=np.int64)
    pts = np.empty((count, 3), dtype=np.float64)
    n = 0
    r2 = r_min * r_min
    offs = np.array([[dx, dy, dz] for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1)])

    def cell_of(p):
        c = np.floor((p - lo) / csize).astype(np.int64)
        return np.minimum(np.maximum(c, 0), ncell - 1)

    all_pts = [] if existing is None else [existing]
    base = 0 if existing is None else existing.shape[0]
    store = np.empty((base + count, 3), dtype=np.float64)
    if existing is not None:
        store[:base] = existing
        c = cell_of(existing)
        for k in range(base):  # existing points are few (vapour next to liquid only)
            cx, cy, cz = c[k]
            grid[cx, cy, cz, fill[cx, cy, cz]] = k
            fill[cx, cy, cz] += 1
    total = base
    batch = batch or max(1024, count // 4)
    while n < count:
        m = min(batch, 2 * (count - n) + 256)
        cand = lo + rng.random((m, 3)) * width
        cc = cell_of(cand)
        # conflicts with accepted points
        nb = cc[:, None, :] + offs[None, :, :]
        ok = np.ones(m, dtype=bool)
        for d in range(3):  # periodic only along axes that span the whole box
            nb[..., d] = np.mod(nb[..., d], ncell[d])
        ids = grid[nb[..., 0], nb[..., 1], nb[..., 2]]  # (m, 27, slots)
        valid = ids >= 0
        other = store[np.where(valid, ids, 0)]
        diff = other - cand[:, None, None, :]
        diff -= width * np.round(diff / width)
        close = (np.einsum("mksd,mksd->mks", diff, diff) < r2) & valid
        ok &= ~close.any(axis=(1, 2))
        # conflicts inside the batch: keep a candidate only if no earlier
        # accepted-so-far candidate of this batch is within r_min
        idx = np.nonzero(ok)[0]
        keep = []
        bgrid = {}
        for k in idx:
            cx, cy, cz = cc[k]
            clash = False
            for o in offs:
                key = ((cx + o[0]) % ncell[0], (cy + o[1]) % ncell[1], (cz + o[2]) % ncell[2])
                for j in bgrid.get(key, ()):
                    dd = cand[j] - cand[k]
                    dd -= width * np.round(dd / width)
                    if dd @ dd < r2:
                        clash = True
                        break
                if clash:
                    break
            if clash:
                continue
            if fill[cx, cy, cz] >= slots:
                continue
            bgrid.setdefault((cx, cy, cz), []).append(k)
            keep.append(k)
            if n + len(keep) >= count:
                break
        for k in keep:
            cx, cy, cz = cc[k]
            store[total] = cand[k]
            grid[cx, cy, cz, fill[cx, cy, cz]] = total
            fill[cx, cy, cz] += 1
            total += 1
        pts[n:n + len(keep)] = cand[keep]
        n += len(keep)
    return pts


def slab(n_total: int, rho_liquid: float, rho_vapour: float, temperature: float, seed: int,
         aspect: float = 4.0, r_min: float = 0.9, rc: float = 3.0, dt: float = 0.005,
         name: str = "") -> State:
    """Liquid slab (density ``rho_liquid``) filling the middle ``1/aspect`` of
    the long z axis of an ``1:1:aspect`` box, vapour (``rho_vapour``)
    elsewhere; uniform random positions with overlap rejection at ``r_min``.
    The box volume is chosen so that the expected atom count is ``n_total``."""
    frac = 1.0 / aspect
    mean_rho = frac * rho_liquid + (1.0 - frac) * rho_vapour
    vol = n_total / mean_rho
    lx = (vol / aspect) ** (1.0 / 3.0)
    L = np.array([lx, lx, aspect * lx])
    z0 = 0.5 * L[2] * (1.0 - frac)
    z1 = z0 + frac * L[2]
    n_liq = int(round(rho_liquid * lx * lx * (z1 - z0)))
    n_vap = n_total - n_liq
    rng = np.random.Generator(np.random.Philox(seed))
    liq = _rsa_fill(rng, [0.0, 0.0, z0], [lx, lx, z1], n_liq, r_min)
    # vapour: uniform in the two outer regions, away from the slab by r_min
    vap = []
    need = n_vap
    while need > 0:
        m = 2 * need + 64
        cand = rng.random((m, 3)) * L
        outside = (cand[:, 2] < z0 - r_min) | (cand[:, 2] > z1 + r_min)
        cand = cand[outside]
        vap.append(cand)
        need -= cand.shape[0]
    vap = np.concatenate(vap)[:n_vap]
    vap = _dedupe_vapour(vap, L, r_min)
    q = np.concatenate([liq, vap])
    v = maxwell_boltzmann(q.shape[0], temperature, rng)
    ids = np.arange(q.shape[0], dtype=np.int32)
    return State(q=q, v=v, ids=ids, L=L, rc=rc, dt=dt, temperature=temperature, name=name)


def _dedupe_vapour(p, L, r_min):
    """Drops vapour points that overlap an earlier one (vapour is dilute, so
    this removes a handful at most)."""
    keep = np.ones(p.shape[0], dtype=bool)
    cell = np.floor(p / r_min).astype(np.int64)
    ncell = np.maximum(1, np.floor(L / r_min).astype(np.int64))
    cell = np.minimum(cell, ncell - 1)
    key = (cell[:, 0] * ncell[1] + cell[:, 1]) * ncell[2] + cell[:, 2]
    order = np.argsort(key, kind="stable")
    seen = {}
    for k in order:
        cx, cy, cz = cell[k]
        clash = False
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    kk = ((cx + dx) % ncell[0], (cy + dy) % ncell[1], (cz + dz) % ncell[2])
                    for j in seen.get(kk, ()):
                        d = p[j] - p[k]
                        d -= L * np.round(d / L)
                        if d @ d < r_min * r_min:
                            clash = True
                            break
                    if clash:
                        break
                if clash:
                    break
            if clash:
                break
        if clash:
            keep[k] = False
        else:
            seen.setdefault((cx, cy, cz), []).append(k)
    return p[keep]


def config_c1(seed: int = 12345) -> State:
    """32,000 atoms, FCC 20^3 cells, rho = 0.5 (a = 2.0, L = 40), T = 1.0,
    rc = 2.5, dt = 0.005."""
    s = fcc_liquid(20, 0.5, 1.0, seed, rc=2.5, dt=0.005, name="lj_fcc32000_rho0.5")
    s.L = np.array([40.0, 40.0, 40.0])  # exactly 20 * 2.0
    return s


def config_c2(seed: int = 2026) -> State:
    """2,048,000 atoms, FCC 80^3 cells, rho = 0.8442, T = 0.722, rc = 2.5, dt = 0.004."""
    return fcc_liquid(80, 0.8442, 0.722, seed, rc=2.5, dt=0.004, name="lj_fcc2048000_rho0.8442")


def config_c3(seed: int = 31, n_total: int = 1_000_000) -> State:
    """Liquid-vapour slab, 1:1:4 box, rho_l = 0.75, rho_v = 0.02, T = 0.9,
    rc = 3.0, dt = 0.005 (Langevin, gamma = 1)."""
    return slab(n_total, 0.75, 0.02, 0.9, seed, rc=3.0, dt=0.005, name=f"lj_slab{n_total}")


def config_c5(seed: int = 55) -> State:
    """32,000 atoms, FCC 20^3 cells, rho = 0.8442, T = 1.0, rc = 2.5, dt = 0.005."""
    return fcc_liquid(20, 0.8442, 1.0, seed, rc=2.5, dt=0.005, name="lj_fcc32000_rho0.8442")
