"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device and the built
library; everything else runs on the CPU."""
from __future__ import annotations

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
