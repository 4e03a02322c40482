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
    "config_c4",
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


_rsa_lib = None


def _rsa():
    """ctypes handle of libmdg_workloads.so (built next to libmdacp_b200.so)."""
    global _rsa_lib
    if _rsa_lib is None:
        import ctypes
        import pathlib

        path = pathlib.Path(__file__).resolve().parent / "libmdg_workloads.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (make -C mdacp_b200/csrc)")
        lib = ctypes.CDLL(str(path))
        dp = ctypes.POINTER(ctypes.c_double)
        lib.mdg_rsa_fill.restype = ctypes.c_long
        lib.mdg_rsa_fill.argtypes = [dp, ctypes.c_double, ctypes.c_int, dp, dp,
                                     ctypes.POINTER(ctypes.c_long), ctypes.c_uint64, ctypes.c_long, dp]
        _rsa_lib = lib
    return _rsa_lib


def rsa_fill(L, r_min, regions, counts, seed, max_tries=None):
    """Random sequential addition: counts[k] points uniform in region k
    (lo, hi corners), all at periodic distance >= r_min in the box L."""
    import ctypes

    lib = _rsa()
    L = np.ascontiguousarray(L, dtype=np.float64)
    lo = np.ascontiguousarray([r[0] for r in regions], dtype=np.float64)
    hi = np.ascontiguousarray([r[1] for r in regions], dtype=np.float64)
    cnt = np.ascontiguousarray(counts, dtype=np.int64)
    total = int(cnt.sum())
    out = np.zeros((max(total, 1), 3), dtype=np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    got = lib.mdg_rsa_fill(L.ctypes.data_as(dp), float(r_min), len(regions), lo.ctypes.data_as(dp),
                           hi.ctypes.data_as(dp), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                           int(seed) & 0xFFFFFFFFFFFFFFFF, int(max_tries or 200 * total + 1000),
                           out.ctypes.data_as(dp))
    if got != total:
        raise RuntimeError(f"random sequential addition placed {got} of {total} points")
    return out[:total]


def slab(n_total: int, rho_liquid: float, rho_vapour: float, temperature: float, seed: int,
         aspect: float = 4.0, r_min: float = 0.9, rc: float = 3.0, dt: float = 0.005,
         name: str = "") -> State:
    """Liquid slab (density ``rho_liquid``) filling the middle ``1/aspect`` of
    the long z axis of an ``1:1:aspect`` box, vapour (``rho_vapour``)
    elsewhere; uniform random positions with overlaps below ``r_min``
    rejected (random sequential addition over the whole periodic box).  The
    box volume is chosen so that the expected atom count is ``n_total``."""
    frac = 1.0 / aspect
    mean_rho = frac * rho_liquid + (1.0 - frac) * rho_vapour
    vol = n_total / mean_rho
    lx = (vol / aspect) ** (1.0 / 3.0)
    L = np.array([lx, lx, aspect * lx])
    z0 = 0.5 * L[2] * (1.0 - frac)
    z1 = z0 + frac * L[2]
    n_liq = int(round(rho_liquid * lx * lx * (z1 - z0)))
    n_vap = n_total - n_liq
    n_low = n_vap // 2
    regions = [([0.0, 0.0, z0], [lx, lx, z1]), ([0.0, 0.0, 0.0], [lx, lx, z0]), ([0.0, 0.0, z1], [lx, lx, L[2]])]
    q = rsa_fill(L, r_min, regions, [n_liq, n_low, n_vap - n_low], seed)
    rng = np.random.Generator(np.random.Philox(seed))
    v = maxwell_boltzmann(q.shape[0], temperature, rng)
    ids = np.arange(q.shape[0], dtype=np.int32)
    return State(q=q, v=v, ids=ids, L=L, rc=rc, dt=dt, temperature=temperature, name=name)


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


def config_c4(seed: int = 404, nrep: int = 256, n_range=(500, 20000), rho_range=(0.3, 0.9),
              t_range=(0.7, 1.5), jitter: float = 0.05):
    """Replica ensemble: ``nrep`` jittered FCC systems, N uniform in
    ``n_range`` (rounded to an FCC block of nx x nx x nz cells), density and
    temperature uniform in their ranges, all drawn from one seed; rc = 2.5,
    dt = 0.005."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for k in range(nrep):
        n_target = rng.uniform(*n_range)
        rho = rng.uniform(*rho_range)
        temp = rng.uniform(*t_range)
        nx = max(1, int(round((n_target / 4.0) ** (1.0 / 3.0))))
        nz = max(1, int(round(n_target / (4.0 * nx * nx))))
        rep_seed = int(rng.integers(0, 2**31))
        st = fcc_liquid((nx, nx, nz), rho, temp, rep_seed, jitter=jitter, rc=2.5, dt=0.005,
                        name=f"replica{k}")
        out.append(st)
    return out
