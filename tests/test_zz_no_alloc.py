"""mdg_observe_static: the observer sums for callers that cannot allocate
device memory (they own all of it, or must not trigger the device-wide
synchronisation of cudaMalloc / cudaFree).  The test owns the device buffers
(allocated here with torch); the entry point only reads them and writes the
three sums into the caller's output buffer, using its static scratch.

Two calls in a row, on systems of different size (the second call has
fewer blocks than the first left partial sums for), must each agree with
mdg_observe on the same state within the FP64 tolerance of the parity tests.
The file is named to run last in a full test session."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import mdacp_b200 as M
from mdacp_b200 import workloads as W

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MAX_ATOMS = 8192 * 256


def _device_inputs(sys_, torch):
    """The handle's state and full list, copied into caller-owned device
    buffers in the layout mdg_observe_static takes."""
    q, v, _ = sys_.state()
    rows, partners = sys_.neighbor_list()
    n = q.shape[0]
    q4 = np.zeros((n, 4))
    v4 = np.zeros((n, 4))
    q4[:, :3] = q
    v4[:, :3] = v
    row_start = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(rows, out=row_start[1:])
    dev = torch.device("cuda:0")
    return (torch.from_numpy(q4).to(dev), torch.from_numpy(v4).to(dev),
            torch.from_numpy(row_start).to(dev), torch.from_numpy(partners.astype(np.int32)).to(dev))


def _call(lib, bufs, n, L, cutoff, out, torch):
    q4, v4, rs, part = bufs
    Lh = (ctypes.c_double * 3)(*[float(x) for x in L])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return lib.mdg_observe_static(ctypes.c_void_p(q4.data_ptr()), ctypes.c_void_p(v4.data_ptr()), n,
                                  ctypes.c_void_p(rs.data_ptr()), ctypes.c_void_p(part.data_ptr()), Lh,
                                  float(cutoff), ctypes.c_void_p(out.data_ptr()), stream)


def test_observe_static_matches_observe_twice():
    torch = pytest.importorskip("torch")
    lib = M.load_library()
    big = W.fcc_liquid(20, 0.8442, 1.0, seed=41, jitter=0.06, rc=2.5, dt=0.004)   # 32,000 atoms
    small = W.fcc_liquid(6, 0.5, 1.0, seed=42, jitter=0.08, rc=2.5, dt=0.005)     # 864 atoms
    out = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    for st in (big, small):
        s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n)
        s.set_state(st.q, st.v)
        s.calculate(25)
        ke, pe, vir = s.observe()
        bufs = _device_inputs(s, torch)
        assert _call(lib, bufs, st.n, st.L, st.rc, out, torch) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[0] == pytest.approx(ke, rel=FP64_TOL)
        assert got[1] == pytest.approx(pe, rel=FP64_TOL)
        assert got[2] == pytest.approx(vir, rel=FP64_TOL)
        s.close()


def test_observe_static_refuses_oversize():
    torch = pytest.importorskip("torch")
    lib = M.load_library()
    one = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    idx = torch.zeros(2, dtype=torch.int32, device="cuda:0")
    out = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    st = _call(lib, (one, one, idx, idx), MAX_ATOMS + 1, [20.0, 20.0, 20.0], 2.5, out, torch)
    assert st == -3  # MDG_ERR_CAPACITY, nothing launched
    assert _call(lib, (one, one, idx, idx), 4, [20.0, 20.0, 20.0], -1.0, out, torch) == -1
