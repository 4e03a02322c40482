"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built
library; everything else runs on the CPU."""
from __future__ import annotations

import math
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmdacp_b200.so")


def golden_names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(params=golden_names())
def golden(request):
    g = load_golden(request.param)
    g["name"] = request.param
    return g


def pair_set(k, p):
    """Sorted unique (key, partner) rows."""
    return np.unique(np.stack([np.asarray(k), np.asarray(p)], axis=1).astype(np.int64), axis=0)


def force_error(f, f_ref):
    """Norm-wise relative force error: max_i |F_i - F_ref_i| / max(max_i |F_ref_i|, rms |F_ref|)."""
    d = np.linalg.norm(np.asarray(f) - np.asarray(f_ref), axis=1)
    mag = np.linalg.norm(f_ref, axis=1)
    scale = max(mag.max(), np.sqrt((mag ** 2).mean()))
    return d.max() / scale


def rms_force_error(f, f_ref):
    d = np.linalg.norm(np.asarray(f) - np.asarray(f_ref), axis=1)
    mag = np.linalg.norm(f_ref, axis=1)
    return np.sqrt((d ** 2).mean()) / np.sqrt((mag ** 2).mean())


def mt19937_canonical(seed, count):
    """`count` draws of std::uniform_real_distribution<double>(0, 1) from
    std::mt19937(seed) as libstdc++ forms them (generate_canonical<double,
    53>: two 32-bit outputs x0 + x1 2^32, divided by 2^64)."""
    bg = np.random.MT19937()
    bg._legacy_seeding(seed)  # std::mt19937's init_genrand
    raw = bg.random_raw(2 * count).astype(np.float64)
    u = (raw[0::2] + raw[1::2] * 4294967296.0) / 18446744073709551616.0
    return np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)


def rankine_start(density=0.2, L=(16.0, 16.0, 40.0), v0=1.0):
    """The start state of the reference's Rankine project: its configuration
    maker's lattice (src/rankine.cc:8-52: four atoms per cell of side
    (density/4)^(-1/3), layers 1 .. sz-2, every coordinate + 1e-7) and
    Variables::SetInitialVelocity(v0, 0) (src/variables.cc:86-113: speed v0
    in a direction drawn from std::mt19937(0), then the mean removed).
    Returns q, v (n x 3) and L."""
    s = 1.0 / (density * 0.25) ** (1.0 / 3.0)
    hs = s * 0.5
    sx, sy, sz = int(L[0] / s), int(L[1] / s), int(L[2] / s)
    e = 0.0000001
    q = []
    for iz in range(1, sz - 1):
        for iy in range(sy):
            for ix in range(sx):
                q.append((ix * s + e, iy * s + e, iz * s + e))
                q.append((ix * s + e, iy * s + hs + e, iz * s + hs + e))
                q.append((ix * s + hs + e, iy * s + e, iz * s + hs + e))
                q.append((ix * s + hs + e, iy * s + hs + e, iz * s + e))
    q = np.array(q)
    n = q.shape[0]
    u = mt19937_canonical(0, 2 * n)
    v = np.empty((n, 3))
    for i in range(n):  # the C library's sqrt, cos and sin, in the reference's order
        z = u[2 * i] * 2.0 - 1.0
        phi = u[2 * i + 1] * 2.0 * math.pi
        r = math.sqrt(1 - z * z)
        v[i] = (v0 * r * math.cos(phi), v0 * r * math.sin(phi), v0 * z)
    av = [0.0, 0.0, 0.0]
    for i in range(n):  # sequential sums, as the reference's loop
        for d in range(3):
            av[d] += v[i, d]
    for d in range(3):
        v[:, d] -= av[d] / n
    return q, v, np.array(L, dtype=np.float64)
