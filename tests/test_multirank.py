"""The N > 1 path of bench.py on the CPU: one process per rank over gloo.

With several GPUs every rank advances its own replica (weak scaling, no
data-path collective); the only collectives are the barrier around the timed
region and the max over ranks of its duration.  These tests run those
helpers with world size 2, check that ranks get distinct seeded replicas,
and that the reference arm is run and printed by rank 0 alone."""
from __future__ import annotations

import json
import os
import pathlib
import socket
import subprocess
import sys
import types

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist = bench.init_dist(ws, "gloo")
    bench.barrier(dist)
    m = bench.max_over_ranks(dist, 1.5 + rank)
    bench.barrier(dist)
    out.put((rank, m))
    dist.destroy_process_group()


def test_barrier_and_max_over_ranks_on_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 2.5, 1: 2.5}


def test_ranks_get_their_own_replica():
    args = types.SimpleNamespace(config="c2", cells=4, md_steps_per_step=10, gpus=2)
    s0, c0 = bench.workload(args, 0)
    s1, c1 = bench.workload(args, 1)
    assert s0.n == s1.n and c0["parallelism"] == "replicas"
    assert not np.array_equal(s0.v, s1.v)  # seed + rank


def test_reference_arm_prints_once_under_torchrun():
    binary = ROOT / "oracle" / "_ref" / "mdacp_rc25_avx2"
    if not binary.exists():
        pytest.skip("the reference build (oracle/_ref) is not present")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--config", "c1", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "reference"


def _partition_worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    from mdacp_b200 import workloads as W

    dist = bench.init_dist(ws, "gloo")
    reps = W.config_c4(seed=404)
    mine, loads = bench.replica_share(reps, ws, rank)
    # stand-in per-replica metrics of this rank's share (rebuilds, energy)
    vals = np.array([[k + 1.0, -0.5 * k] for k in mine]).reshape(len(mine), 2)
    full = bench.gather_replica_metrics(dist, len(reps), mine, vals)
    out.put((rank, list(mine), loads.tolist(), full.tolist(), len(reps)))
    dist.destroy_process_group()


def test_replica_partition_and_gather_on_gloo():
    # one 256-replica ensemble split over 2 ranks (balanced by atoms x
    # neighbours); every replica is owned once and the per-replica metrics
    # of both shares reach every rank
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_partition_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        rank, mine, loads, full, nrep = q.get(timeout=300)
        got[rank] = (mine, loads, np.asarray(full), nrep)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    nrep = got[0][3]
    owned = sorted(got[0][0] + got[1][0])
    assert owned == list(range(nrep))
    loads = np.asarray(got[0][1])
    assert loads.max() / loads.mean() - 1.0 < 0.10
    expect = np.array([[k + 1.0, -0.5 * k] for k in range(nrep)])
    assert np.array_equal(got[0][2], expect) and np.array_equal(got[1][2], expect)
