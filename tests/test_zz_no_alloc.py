"""mdg_observe_static: the observer sums for callers that cannot allocate
device memory (they own all of it, or must not trigger the device-wide
synchronisation of cudaMalloc / cudaFree).  The test owns the device buffers
(allocated here with torch); the entry point only reads them and writes the
three sums into the caller's output buffer, using its static scratch.

Two calls in a row, on systems of different size (the second call has
fewer blocks than the first left partial sums for), must each agree with
mdg_observe on the same state within the FP64 tolerance of the parity tests;
so must a call on a side stream, and an empty system gives (0, 0, 0).  A
warmed-up call leaves the device's free memory unchanged, and a partner
index outside the atoms is skipped and reported as a NaN energy.  The file
is named to run last in a full test session."""
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


def _call(lib, bufs, n, L, cutoff, out, torch, stream=None):
    q4, v4, rs, part = bufs
    Lh = (ctypes.c_double * 3)(*[float(x) for x in L])
    stream = ctypes.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
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


def test_observe_static_side_stream_empty_and_no_allocation():
    torch = pytest.importorskip("torch")
    lib = M.load_library()
    st = W.fcc_liquid(8, 0.8442, 1.0, seed=43, jitter=0.06, rc=2.5, dt=0.004)   # 2,048 atoms
    s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n)
    s.set_state(st.q, st.v)
    s.calculate(10)
    ke, pe, vir = s.observe()
    bufs = _device_inputs(s, torch)
    s.close()
    out = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    side = torch.cuda.Stream()
    assert _call(lib, bufs, st.n, st.L, st.rc, out, torch) == 0   # warm-up: module and scratch set up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    with torch.cuda.stream(side):
        out.zero_()
        assert _call(lib, bufs, st.n, st.L, st.rc, out, torch, stream=side) == 0
    side.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    got = out.cpu().numpy()
    assert got[0] == pytest.approx(ke, rel=FP64_TOL)
    assert got[1] == pytest.approx(pe, rel=FP64_TOL)
    assert got[2] == pytest.approx(vir, rel=FP64_TOL)
    assert free1 == free0
    # an empty system: the sums are zero
    out.fill_(1.0)
    assert _call(lib, bufs, 0, st.L, st.rc, out, torch) == 0
    torch.cuda.synchronize()
    assert out.cpu().tolist() == [0.0, 0.0, 0.0]


def test_observe_static_bad_partner_gives_nan():
    torch = pytest.importorskip("torch")
    lib = M.load_library()
    st = W.fcc_liquid(6, 0.5, 1.0, seed=44, jitter=0.08, rc=2.5, dt=0.005)      # 864 atoms
    s = M.System(st.L, cutoff=st.rc, time_step=st.dt, capacity=st.n)
    s.set_state(st.q, st.v)
    q4, v4, rs, part = _device_inputs(s, torch)
    s.close()
    part[5] = st.n + 1000   # an index past the atoms: skipped, never read
    out = torch.zeros(3, dtype=torch.float64, device="cuda:0")
    assert _call(lib, (q4, v4, rs, part), st.n, st.L, st.rc, out, torch) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.isnan(got[1])
    assert np.isfinite(got[0])
