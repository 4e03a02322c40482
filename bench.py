"""Benchmark of the LJ timestep hot path (one JSON line on rank 0).

Workload: 2,048,000 atoms, FCC 80^3 cells at rho = 0.8442 (L = 134.37),
T = 0.722 Maxwell-Boltzmann from a seed, smoothed LJ with rc = 2.5, search
length 2.8, dt = 0.004, NVE.  One bench step is one observation interval of
the reference's Benchmark project (ObserveLoop = 100 MD steps of
MDManager::Calculate, src/benchmark.cc:32-41), rebuilds included as they
fall due.  The headline path is FP32-mixed (FP32 pair forces, FP64
integration and reductions); the plain FP64 drop-in is measured beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mdg|reference]

Under torchrun (N > 1) every rank runs its own replica (weak scaling, no
data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "LJ atom-steps/s at 2.05M atoms, FP32-mixed vs FP64 on 1 B200; force err"
UNIT = "atom-steps/s"
MD_STEPS_PER_STEP = 100
L2_BYTES = 126 * 2 ** 20


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------ distributed
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
    return dist


def max_over_ranks(dist, value, device=None):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device=None):
    if dist is not None:
        if device is not None and str(device).startswith("cuda"):
            dist.barrier(device_ids=[int(str(device).split(":")[1])])
        else:
            dist.barrier()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in pathlib.Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# -------------------------------------------------------------- reference
def ref_threads():
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    return max(1, min(cores, 256))


def local_grid(t, L, sl):
    """Factor t threads into an lx*ly*lz unit grid with every unit at least
    2*SearchLength wide (ParaInfo only factors powers of two by itself,
    src/parainfo.cc:44-58)."""
    best = None
    for lx in range(1, t + 1):
        if t % lx:
            continue
        for ly in range(1, t // lx + 1):
            if (t // lx) % ly:
                continue
            lz = t // lx // ly
            if min(L[0] / lx, L[1] / ly, L[2] / lz) < 2 * sl:
                continue
            score = max(lx, ly, lz)
            if best is None or score < best[0]:
                best = (score, (lx, ly, lz))
    return best[1] if best else None


def run_reference_bench(state, steps, warmup, threads, config):
    """Times the reference's own CPU build (AVX2, oracle/_ref) on the state
    through its OracleBench project; returns (atom_steps_per_s, info)."""
    from oracle import lj_oracle as O

    t = threads
    grid = local_grid(t, state.L, state.rc + 0.3)
    while grid is None or t < 3:  # the reference caps each unit at 1e6 atoms incl. ghosts
        t -= 1 if t > 3 else -1
        grid = local_grid(t, state.L, state.rc + 0.3)
    extra = {"Steps": str(steps), "Warmup": str(warmup), "LocalGridX": str(grid[0]),
             "LocalGridY": str(grid[1]), "LocalGridZ": str(grid[2])}
    if config.get("thermostat") == "Langevin":
        extra.update(ControlTemperature="yes", HeatbathType="Langevin",
                     AimedTemperature=repr(config["temperature"]), HeatbathGamma=repr(config["gamma"]))
    wd, out = O.run_reference("OracleBench", state.q, state.v, state.ids, state.L, state.rc, state.dt,
                              flavour="avx2", threads=t, extra=extra, timeout=1800)
    line = [x for x in out.splitlines() if x.startswith("ORACLE_BENCH")][-1].split()
    kv = {line[i]: float(line[i + 1]) for i in range(1, len(line) - 1, 2)}
    # ConstructionCounter sums over the units, which all rebuild together
    return kv["atom_steps_per_s"], {"cores": t, "grid": grid, "sec": kv["sec"], "steps": int(kv["steps"]),
                                    "rebuilds": int(round(kv["rebuilds"] / kv["units"]))}


def ref_sample_steps(cores, seconds, n):
    # about 5e6 atom-steps/s per core for the AVX2 build at rho 0.84, rc 2.5
    # (8.1e7-8.6e7 measured on 16 host cores of the B200 box)
    est = 5.0e6 * cores
    return int(min(2000, max(10, seconds * est / n)))


# -------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mdg", "reference"], default="mdg")
    ap.add_argument("--md-steps-per-step", type=int, default=MD_STEPS_PER_STEP)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cells", type=int, default=80, help="FCC cells per axis (80 = 2,048,000 atoms)")
    ap.add_argument("--precision", choices=["both", "fp32", "fp64"], default="both",
                    help="restrict the timed runs (profiling); the JSON line needs both")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end run (profiling)")
    ap.add_argument("--no-force-error", action="store_true", help="skip the FP32-vs-FP64 force check")
    ap.add_argument("--drift-steps", type=int, default=10000,
                    help="NVE steps of the energy-drift comparison of the two paths (0: skip); the 2.05M-atom "
                         "configuration's run is 10,000 steps")
    ap.add_argument("--stage-atoms", type=int, default=0,
                    help="FP32-mixed force: partner positions staged per 128-atom block in shared memory, "
                         "at most this many atoms (0: gather from global memory, the default; -1: 2304)")
    ap.add_argument("--eager", action="store_true",
                    help="launch every kernel from the host instead of CUDA graphs (for profilers)")
    ap.add_argument("--threads-per-atom", type=int, default=0,
                    help="FP32-mixed force pass lanes per atom (0: tuned at the first step); with "
                         "--config c5 --adjoint-launches the adjoint pair kernels' lanes (1, 2, 4, 8)")
    ap.add_argument("--build-block", type=int, default=0, help="list build threads per block (0: tuned)")
    ap.add_argument("--build-lanes", type=int, default=0, help="list build lanes per atom (0: tuned)")
    ap.add_argument("--step-mode", choices=["auto", "graphs", "persistent"], default="auto",
                    help="FP32-mixed NVE steps as CUDA graphs or one persistent launch (auto: by size)")
    ap.add_argument("--adjoint-launches", action="store_true",
                    help="c5 profiling: two 40-step gradient runs (checkpoints every 20 steps) and nothing else")
    ap.add_argument("--tune-margins", action="store_true",
                    help="c4: per-replica pairlist margins chosen by timing (mdacp_b200.margins) instead of "
                         "the common BufferLength 0.3")
    ap.add_argument("--config", choices=["c2", "c1", "c3", "c4", "c5"], default="c2",
                    help="c2: 2.05M-atom liquid (headline); c1: 32k atoms rho 0.5; c3: 1M-atom Langevin slab; "
                         "c4: 256-replica ensemble; c5: adjoint gradients of a 32k-atom trajectory")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.config == "c4":
        return main_ensemble(args, ws, rank, local)
    if args.config == "c5":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference computes no gradients "
                                  "(no adjoint or differentiable path)"}), flush=True)
            return 0
        return main_adjoint(args, ws, rank, local)
    state, config = workload(args, rank)
    if args.impl == "reference":
        return main_reference(args, ws, rank, state, config)
    if args.stage_atoms != 0:
        config["force_stage_atoms"] = args.stage_atoms
    for key, val in (("threads_per_atom", args.threads_per_atom), ("build_block", args.build_block),
                     ("build_threads_per_atom", args.build_lanes)):
        if val:
            config.setdefault("pinned_shapes", {})[key] = val
    if args.step_mode != "auto":
        config["step_mode"] = {"graphs": 1, "persistent": 2}[args.step_mode]
    return main_mdg(args, ws, rank, local, state, config)


def workload(args, rank):
    """The synthetic state and the JSON config of the selected workload."""
    from mdacp_b200 import workloads as W

    common = {"md_steps_per_step": args.md_steps_per_step,
              "parallelism": "replicas" if args.gpus > 1 else "single"}
    if args.config == "c1":
        state = W.config_c1(seed=12345 + rank)
        config = dict(common, workload=f"{state.name}: {state.n} atoms, FCC 20^3 cells, rho 0.5, L 40, T 1.0, "
                                      "rc 2.5, search length 2.8, dt 0.005, NVE",
                      n_atoms=state.n, rho=0.5, temperature=1.0, rc=2.5, search_length=2.8, dt=0.005,
                      thermostat="NVE", l2="small system: state (2 MB) and list (6 MB) stay L2-resident")
        return state, config
    if args.config == "c3":
        state = W.config_c3(seed=31 + rank)
        config = dict(common, workload=f"{state.name}: {state.n} atoms, 1:1:4 box {state.L[0]:.2f}^2 x "
                                      f"{state.L[2]:.2f}, liquid slab rho 0.75 in the middle quarter, vapour "
                                      "rho 0.02, overlaps < 0.9 rejected, T 0.9, Langevin gamma 1.0 (Philox "
                                      "noise), rc 3.0, search length 3.3, dt 0.005",
                      n_atoms=state.n, temperature=0.9, rc=3.0, search_length=3.3, dt=0.005,
                      thermostat="Langevin", gamma=1.0,
                      l2="inputs larger than L2 (state 64 MB + pairlist > 400 MB)")
        return state, config
    state = W.fcc_liquid(args.cells, 0.8442, 0.722, seed=2026 + rank, rc=2.5, dt=0.004,
                         name=f"lj_fcc{4 * args.cells ** 3}_rho0.8442")
    config = dict(common, workload=f"{state.name}: {state.n} atoms, FCC {args.cells}^3 cells, rho 0.8442, "
                                  f"L {state.L[0]:.4f}, T 0.722, rc 2.5, search length 2.8, dt 0.004, NVE",
                  n_atoms=state.n, rho=0.8442, temperature=0.722, rc=2.5, search_length=2.8, dt=0.004,
                  thermostat="NVE", l2="inputs larger than L2 (state 131 MB + pairlist > 1 GB per replica)")
    return state, config


def metric_for(config):
    if config["n_atoms"] == 2048000 and config.get("thermostat") == "NVE":
        return METRIC
    return f"LJ atom-steps/s, {config['workload'].split(':')[0]}"


def system_kwargs(state, config, M):
    kw = dict(cutoff=state.rc, time_step=state.dt, capacity=state.n,
              stage_atoms=config.get("force_stage_atoms", 0))
    if config.get("step_mode") is not None:
        kw["step_mode"] = config["step_mode"]
    kw.update(config.get("pinned_shapes", {}))
    if config.get("thermostat") == "Langevin":
        kw.update(thermostat=M.LANGEVIN, aimed_temperature=config["temperature"],
                  heatbath_gamma=config["gamma"], seed=7)
    return kw


def main_reference(args, ws, rank, state, config):
    if rank != 0:
        return 0
    cores = ref_threads()
    md_steps = ref_sample_steps(cores, 60.0, state.n)
    value, info = run_reference_bench(state, md_steps, max(1, min(args.warmup, 5)), cores, config)
    ms_per_md = 1e3 * state.n / value
    line = {
        "metric": metric_for(config), "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": info["steps"],
        "warmup": max(1, min(args.warmup, 5)), "ms_per_step": ms_per_md, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": dict(config, md_steps_per_step=1, precision="fp64 (reference AVX2 CPU build)",
                       unit_grid=list(info["grid"])),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": info["cores"], "kind": "reference",
                         "sample": f"{info['steps']} MD steps of the full {state.n}-atom system "
                                   f"({info['rebuilds']} rebuilds, {info['sec']:.2f} s), OpenMP units "
                                   f"{info['grid']}, 1 MPI rank"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def force_errors(f, f_ref):
    """Norm-wise max and RMS relative force error."""
    d = np.linalg.norm(f - f_ref, axis=1)
    mag = np.linalg.norm(f_ref, axis=1)
    return {"max": float(d.max() / max(mag.max(), np.sqrt((mag ** 2).mean()))),
            "rms": float(np.sqrt((d ** 2).mean()) / np.sqrt((mag ** 2).mean()))}


def force_kernel_bytes(n, list_entries, precision):
    """Algorithmic bytes of one force launch (neighbour gathers count as
    cache-served).  FP64 kick: own position + row length + list + velocity
    read/write.  FP32-mixed NVE pass (both half drifts fused): own
    fixed-point copy + row length + list + velocity and position read/write
    + the next step's fixed-point copy."""
    if precision == "fp32":
        return n * (16 + 4 + 64 + 64 + 16) + 4 * list_entries
    return n * (32 + 4 + 32 + 32) + 4 * list_entries


def timed_run(sys_, args, dist, device, torch):
    """W warm-up + K timed bench steps of md_steps_per_step MD steps."""
    mdn = args.md_steps_per_step
    for _ in range(args.warmup):
        sys_.calculate(mdn)
    sys_.set_kernel_timing(True)
    info0 = sys_.info()
    barrier(dist, device)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(sys_.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        sys_.calculate(mdn)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(dist, device)
    ms = e0.elapsed_time(e1)
    info1 = sys_.info()
    fms, flaunch, klaunch = sys_.kernel_time()
    sys_.set_kernel_timing(False)
    # kernels inside the conditional branches: a rebuild is 10 kernels (11
    # with the staged FP32 force pass's plan), a displacement check 4 (three
    # passes and the rebuild decision)
    staged = sys_.params.precision != 0 and sys_.params.stage_atoms != 0
    launches = klaunch + (11 if staged else 10) * (info1["rebuilds"] - info0["rebuilds"]) + 4 * (
        info1["displacement_checks"] - info0["displacement_checks"])
    return ms, fms, flaunch, launches, info0, info1


def main_mdg(args, ws, rank, local, state, config):
    import torch

    import mdacp_b200 as M

    dist = init_dist(ws, "nccl")
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    n = state.n
    sampler = ClockSampler(local)
    result = {}
    clocks = None
    runs = [("fp32", M.FP32_MIXED), ("fp64", M.FP64)]
    if args.precision != "both":
        runs = [r for r in runs if r[0] == args.precision]
    for prec_name, prec in runs:
        s = M.System(state.L, precision=prec, device=local, **system_kwargs(state, config, M))
        s.set_state(state.q, state.v)
        if args.eager:
            s.set_graph_mode(False)
        if prec_name == "fp32":
            sampler.start()
        ms, fms, flaunch, launches, info0, info1 = timed_run(s, args, dist, device, torch)
        if prec_name == "fp32":
            clocks = sampler.stop()
        ms_max = max_over_ranks(dist, ms, device)
        md_steps = args.steps * args.md_steps_per_step
        within, _ = s.pair_counts()
        result[prec_name] = dict(ms=ms_max, value=ws * n * md_steps / (ms_max * 1e-3), force_ms=fms,
                                 force_launches=flaunch, launches=launches, info0=info0, info1=info1,
                                 pairs=within // 2)
        s.close()

    if args.precision != "both" or args.no_e2e or args.no_force_error:
        for name, r in result.items():
            if rank == 0:
                print(json.dumps({"profiling_run": name, "ms_per_md_step": r["ms"] / (args.steps * args.md_steps_per_step),
                                  "value": r["value"], "force_ms_avg": r["force_ms"] / max(1, r["force_launches"]),
                                  "rebuilds": r["info1"]["rebuilds"] - r["info0"]["rebuilds"]}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return 0

    # end to end through the C ABI from pinned host buffers (FP32-mixed path)
    s = M.System(state.L, precision=M.FP32_MIXED, device=local, **system_kwargs(state, config, M))
    hq = torch.empty((n, 4), dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty((n, 4), dtype=torch.float64, pin_memory=True).numpy()
    hq[:, :3] = state.q
    hq[:, 3] = 0.0
    hv[:, :3] = state.v
    hv[:, 3] = 0.0
    for _ in range(max(1, min(args.warmup, 2))):
        s.set_state4(hq, hv)
        s.calculate(args.md_steps_per_step)
        s.get_state4(hq, hv)
    barrier(dist, device)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.set_state4(hq, hv)
        s.calculate(args.md_steps_per_step)
        s.get_state4(hq, hv)
    t_e2e = time.perf_counter() - t0
    t_e2e = max_over_ranks(dist, t_e2e, device)
    s.close()
    e2e_value = ws * n * args.steps * args.md_steps_per_step / t_e2e

    # FP32-mixed force error against FP64 at full size
    errs = {}
    sa = M.System(state.L, precision=M.FP64, device=local, **system_kwargs(state, config, M))
    sa.set_state(state.q, state.v)
    sa.calculate(50)
    q, v_state = sa.state_by_id()
    f64 = sa.forces_by_id()
    sa.close()
    sb = M.System(state.L, precision=M.FP32_MIXED, device=local, **system_kwargs(state, config, M))
    sb.set_state(q, v_state)
    f32 = sb.forces_by_id()
    sb.close()
    errs = dict(force_errors(f32, f64), state="after 50 FP64 steps from the start state")

    # NVE energy drift of both paths from the same state (total energy per atom
    # observed every 100 MD steps)
    drift = None
    if config.get("thermostat", "NVE") == "NVE" and args.drift_steps > 0:
        drift = {"md_steps": args.drift_steps, "observe_every": 100, "state": "the start state"}
        for prec_name, prec in (("fp32", M.FP32_MIXED), ("fp64", M.FP64)):
            sd = M.System(state.L, precision=prec, device=local, **system_kwargs(state, config, M))
            sd.set_state(state.q, state.v)
            ke, pe, _ = sd.observe()
            e0 = (ke + pe) / n
            es = [e0]
            for _ in range(max(1, args.drift_steps // 100)):
                sd.calculate(100)
                ke, pe, _ = sd.observe()
                es.append((ke + pe) / n)
            sd.close()
            es = np.asarray(es)
            t = np.arange(len(es)) * 100 * state.dt
            slope = float(np.polyfit(t, es, 1)[0]) if len(es) > 2 else 0.0
            drift[prec_name] = {"e0_per_atom": float(e0), "max_abs_dev_per_atom": float(np.abs(es - e0).max()),
                                "max_rel_dev": float(np.abs(es - e0).max() / abs(e0)),
                                "slope_per_atom_per_time": slope}

    r32, r64 = result["fp32"], result["fp64"]
    hbm, peak_kind = peaks()
    rebuilds = r32["info1"]["rebuilds"] - r32["info0"]["rebuilds"]
    entries = r32["info1"]["list_entries"]
    fbytes = force_kernel_bytes(n, entries, "fp32")
    roofline_note = "force kernel timed with CUDA events around every launch of the timed region"
    if r32["force_launches"] == 0:
        # the timed steps ran in the persistent multi-step pass, which has no
        # separate force launches: time the same pass launched per step
        kw = dict(system_kwargs(state, config, M), step_mode=M.STEPS_GRAPHS)
        sg = M.System(state.L, precision=M.FP32_MIXED, device=local, **kw)
        sg.set_state(state.q, state.v)
        gargs = argparse.Namespace(**dict(vars(args), steps=min(args.steps, 3), warmup=min(args.warmup, 3)))
        _, fms_g, fl_g, _, _, _ = timed_run(sg, gargs, None, device, torch)
        sg.close()
        r32 = dict(r32, force_ms=fms_g, force_launches=fl_g)
        roofline_note = ("the timed steps ran in the persistent multi-step pass; its force pass was timed "
                         "launched once per step (CUDA graphs) on the same system")
    f_avg_ms = r32["force_ms"] / max(1, r32["force_launches"])
    achieved = fbytes / (f_avg_ms * 1e-3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "force_fp32_c2.json"
    if prof.exists():
        traffic = json.loads(prof.read_text()).get("dram_bytes_per_launch")
    line = {
        "metric": metric_for(config), "value": r32["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r32["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(config, precision="fp32_mixed: FP32 pair forces on fixed-point minimum-image "
                                         "displacements, FP64 per-atom sums, integration and reductions",
                       rebuilds=rebuilds, mean_row=entries / n,
                       tuned={"threads_per_atom": r32["info1"]["threads_per_atom"],
                              "build_block": r32["info1"]["build_block"],
                              "build_threads_per_atom": r32["info1"]["build_threads_per_atom"],
                              "fp64_build": [r64["info1"]["build_block"], r64["info1"]["build_threads_per_atom"]],
                              "how": "timed once per device and problem shape at the first step"},
                       persistent_steps=r32["info1"]["persistent_steps"] - r32["info0"]["persistent_steps"]),
        "fp64": {"value": r64["value"], "ms_per_md_step": r64["ms"] / (args.steps * args.md_steps_per_step),
                 "speedup_fp32_over_fp64": r32["value"] / r64["value"]},
        "ms_per_md_step": r32["ms"] / (args.steps * args.md_steps_per_step),
        "pair_interactions_per_s": {
            "fp32": ws * r32["pairs"] * args.steps * args.md_steps_per_step / (r32["ms"] * 1e-3),
            "fp64": ws * r64["pairs"] * args.steps * args.md_steps_per_step / (r64["ms"] * 1e-3),
            "pairs_within_cutoff_per_step": r32["pairs"]},
        "force_error_fp32_vs_fp64": errs,
        "nve_energy_drift": drift,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "kernel": "k_force_fp32 (fused NVE step: drift, kick, drift, pack)",
                     "algorithmic_bytes_per_launch": fbytes, "avg_launch_ms": f_avg_ms,
                     "launches": r32["force_launches"], "peak_kind": peak_kind, "timing": roofline_note},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 32 * n,
                "d2h_bytes_per_step": 2 * 32 * n},
        "gpu_launches": r32["launches"],
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        try:
            cores = ref_threads()
            v, info = run_reference_bench(state, ref_sample_steps(cores, 15.0, n), 2, cores, config)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "reference",
                                    "sample": f"{info['steps']} MD steps of the same {n}-atom system, "
                                              f"reference AVX2 build, {info['sec']:.2f} s"}
        except Exception as exc:  # noqa: BLE001
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": None, "kind": "reference",
                                    "sample": f"not run: {exc}"}
        # the checker: both GPU paths' forces at the same state against the
        # CPU oracle's FP64 forces (the reference's arithmetic)
        try:
            from oracle import lj_oracle as O

            # positions drift out of the box between rebuilds; the oracle, as the
            # reference's AddParticle, keeps only atoms inside it: wrap them once
            # as the device's rebuild does
            L = np.asarray(state.L)
            qw = np.where(q < 0.0, q + L, np.where(q > L, q - L, q))
            o = O.Oracle(qw, v_state, state.ids, state.L, state.rc, state.dt)
            o.make_pairlist()
            of = o.forces()
            _, _, oid = o.state()
            o.close()
            f_or = np.empty_like(of)
            f_or[oid] = of
            line["force_error_vs_oracle"] = {"fp32_mixed": force_errors(f32, f_or), "fp64": force_errors(f64, f_or),
                                             "state": errs["state"],
                                             "oracle": "oracle/lj_oracle.c, the reference's FP64 arithmetic"}
        except Exception as exc:  # noqa: BLE001
            line["force_error_vs_oracle"] = {"not_run": str(exc)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main_adjoint(args, ws, rank, local):
    """Gradients of a 200-step trajectory loss (32,000 atoms, rho 0.8442,
    T 1.0, FP64, checkpoints every 20 steps) with respect to epsilon, sigma
    and the initial positions; checked against central finite differences."""
    import torch

    from mdacp_b200 import adjoint as A
    from mdacp_b200 import workloads as W

    dist = init_dist(ws, "nccl")
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    st = W.config_c5(seed=55 + rank)
    if args.adjoint_launches:
        # the sequence of profiles/adjoint_lj32000_launches.md: a warm-up
        # run (with the lanes-per-atom autotuner unless --threads-per-atom
        # pins the lanes), then one 40-step gradient run
        kw = dict(steps=40, checkpoint_every=20, time_step=st.dt, device=local,
                  threads_per_atom=args.threads_per_atom)
        A.trajectory_gradients(st.q, st.v, st.L, **kw)
        t0 = time.perf_counter()
        A.trajectory_gradients(st.q, st.v, st.L, **kw)
        if rank == 0:
            print(json.dumps({"profiling_run": "adjoint, 32000 atoms, 40 steps",
                              "seconds": time.perf_counter() - t0}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return 0
    n, T, k = st.n, 200, 20
    kw = dict(steps=T, checkpoint_every=k, time_step=st.dt, device=local)
    per_tpa = {}
    for t in (1, 2, 4, 8):  # the lane counts the autotuner chooses from
        A.trajectory_gradients(st.q, st.v, st.L, threads_per_atom=t, **kw)
        t0 = time.perf_counter()
        A.trajectory_gradients(st.q, st.v, st.L, threads_per_atom=t, **kw)
        per_tpa[t] = time.perf_counter() - t0
    for _ in range(args.warmup):
        A.trajectory_gradients(st.q, st.v, st.L, **kw)
    barrier(dist, device)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        loss, de, ds, dq = A.trajectory_gradients(st.q, st.v, st.L, **kw)
    t_grad = max_over_ranks(dist, (time.perf_counter() - t0) / args.steps, device)
    t0 = time.perf_counter()
    A.trajectory_loss(st.q, st.v, st.L, **kw)
    t_fwd = time.perf_counter() - t0
    h = 1e-6
    f = lambda qq, e=1.0, s=1.0: A.trajectory_loss(qq, st.v, st.L, epsilon=e, sigma=s, **kw)  # noqa: E731
    d = np.random.default_rng(11).standard_normal(st.q.shape)
    d /= np.linalg.norm(d)
    g = dq / np.linalg.norm(dq)
    fd = {"epsilon": (f(st.q, 1 + h) - f(st.q, 1 - h)) / (2 * h),
          "sigma": (f(st.q, 1.0, 1 + h) - f(st.q, 1.0, 1 - h)) / (2 * h),
          "q0_along_gradient": (f(st.q + h * g) - f(st.q - h * g)) / (2 * h),
          "q0_random_direction": (f(st.q + h * d) - f(st.q - h * d)) / (2 * h)}
    adj = {"epsilon": de, "sigma": ds, "q0_along_gradient": float(np.linalg.norm(dq)),
           "q0_random_direction": float((dq * d).sum())}
    rel = {key: abs(adj[key] - fd[key]) / abs(fd[key]) for key in fd}
    value = ws * n * T / t_grad
    line = {
        "metric": "adjoint atom-steps/s (forward + reverse sweep), 32,000-atom LJ, 200 FP64 steps",
        "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_grad * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "lj_fcc32000_rho0.8442: 32000 atoms, FCC 20^3 cells, T 1.0, rc 2.5 sigma, dt 0.005, "
                               "200 NVE steps, checkpoints every 20 steps, loss = time-averaged PE + smoothed pair "
                               "count in 1.0 < r < 1.5, per atom", "n_atoms": n, "md_steps": T,
                   "checkpoint_every": k},
        "forward_only": {"value": n * T / t_fwd, "unit": UNIT, "seconds": t_fwd},
        "gradient_check": {"h": h, "adjoint": adj, "finite_difference": fd, "relative_error": rel},
        "seconds_per_lanes_per_atom": {str(t): v for t, v in per_tpa.items()},
        "timing": "host wall clock around the C-ABI call (host-driven steps, device sums read once per run)",
        "cpu_baseline": {"value": None, "unit": UNIT, "cores": None, "kind": "port",
                         "sample": "not run: the reference computes no gradients"},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def replica_share(reps, ws, rank, search_length=2.8):
    """The replicas of one 256-replica ensemble this rank advances: the
    balanced partition of mdg_partition_replicas (load = atoms x (41 +
    neighbours within the search length)); returns (indices, loads per rank)."""
    import mdacp_b200 as M

    owner, load = M.partition_replicas([(r.n, r.L) for r in reps], ws, search_length)
    return [k for k in range(len(reps)) if owner[k] == rank], load


def gather_replica_metrics(dist, nrep, mine, values, device=None):
    """Per-replica metrics of every rank's share, summed into full arrays
    (a replica belongs to exactly one rank; the others contribute zeros):
    values is a (len(mine), m) array; returns (nrep, m) on every rank."""
    import torch

    full = np.zeros((nrep, values.shape[1]), dtype=np.float64)
    full[mine] = values
    if dist is None:
        return full
    t = torch.tensor(full, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def main_ensemble(args, ws, rank, local):
    """256 independent replicas (N 500-20000, rho 0.3-0.9, T 0.7-1.5, jittered
    FCC) in one mdg_ensemble, FP32-mixed, against looping the single-system
    handle over the same replicas.  Under torchrun the 256 replicas are
    partitioned over the ranks (replica_share) and every rank advances its
    share; per-replica rebuild counts and energies are gathered to rank 0."""
    import torch

    import mdacp_b200 as M
    from mdacp_b200 import workloads as W

    dist = init_dist(ws, "nccl")
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    all_reps = W.config_c4(seed=404)
    mine, loads = replica_share(all_reps, ws, rank)
    reps = [all_reps[k] for k in mine]
    ntot_all = sum(r.n for r in all_reps)
    ntot = sum(r.n for r in reps)
    mdn = args.md_steps_per_step
    margins, tuning = None, None
    if args.tune_margins:
        # outside the timed region: trial ensembles of this rank's replicas
        margins, tuning = M.margins.tune_margins([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005,
                                                 precision=M.FP32_MIXED, device=local)
    ens = M.Ensemble([(r.q, r.v, r.L) for r in reps], cutoff=2.5, time_step=0.005, precision=M.FP32_MIXED,
                     device=local, buffer_lengths=margins)
    if args.eager:
        ens.set_graph_mode(False)
    for _ in range(args.warmup):
        ens.calculate(mdn)
    ens.set_kernel_timing(True)
    stream = torch.cuda.ExternalStream(ens.stream())
    sampler = ClockSampler(local)
    barrier(dist, device)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    sampler.start()
    e0.record(stream)
    for _ in range(args.steps):
        ens.calculate(mdn)
    e1.record(stream)
    e1.synchronize()
    clocks = sampler.stop()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), device)
    value = ntot_all * args.steps * mdn / (ms * 1e-3)
    fms, flaunch, launches = ens.kernel_time()
    ens.set_kernel_timing(False)
    entries, pairs = ens.list_stats()
    rb, _ = ens.rebuilds()
    ke, pe, _ = ens.observe()
    per_rep = gather_replica_metrics(dist, len(all_reps), mine,
                                     np.stack([np.asarray(rb, dtype=np.float64), ke, pe], axis=1), device)
    rb_all = per_rep[:, 0]
    if dist is not None:
        t = torch.tensor([float(pairs), float(entries)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        pairs, entries_all = int(t[0].item()), int(t[1].item())
    else:
        entries_all = entries
    ens.close()
    # roofline of the ensemble's FP32 force pass (kick + second half drift,
    # all replicas in one launch): own fixed-point copy, row length, list,
    # velocity and position read and write
    force_bytes = ntot * (16 + 4 + 64 + 64) + 4 * entries
    avg_ms = fms / max(1, flaunch)
    achieved = force_bytes / (avg_ms * 1e-3) / 1e9
    hbm, peak_kind = peaks()
    # looping the single-system path: one handle per replica, stepped in turn
    # (replicas narrower than three search lengths on an axis have no
    # single-system cell grid and are left out of the loop)
    loop_steps = max(20, mdn // 5)
    rep_margin = list(margins) if margins is not None else [0.3] * len(reps)
    looped = [(r, m) for r, m in zip(reps, rep_margin) if min(int(x / (2.5 + m)) for x in r.L) >= 3] \
        if ws == 1 else []
    loop_n = sum(r.n for r, _ in looped)
    systems = []
    for r, m in looped:
        sy = M.System(r.L, cutoff=2.5, time_step=0.005, capacity=r.n, precision=M.FP32_MIXED, device=local,
                      buffer_length=m)
        sy.set_state(r.q, r.v)
        sy.calculate(20)  # first build + graph capture outside the timing
        systems.append(sy)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for sy in systems:
        sy.calculate(loop_steps)
    torch.cuda.synchronize()
    loop_s = time.perf_counter() - t0
    loop_value = loop_n * loop_steps / loop_s if looped else None
    for sy in systems:
        sy.close()
    line = {
        "metric": "LJ atom-steps/s, 256-replica ensemble (N 500-20000)", "value": value, "unit": UNIT,
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"256 replicas, {ntot_all} atoms in total, N 500-20000, rho 0.3-0.9, T 0.7-1.5, "
                               f"jittered FCC, rc 2.5, search length "
                               f"{'2.5 + tuned margin' if margins is not None else '2.8'}, dt 0.005, NVE, FP32-mixed",
                   "md_steps_per_step": mdn, "replicas": len(all_reps), "atoms": ntot_all,
                   "buffer_length": ("per replica, chosen by timing (rank 0's share: min %.3f, median %.3f, "
                                     "max %.3f)" % (float(np.min(margins)), float(np.median(margins)),
                                                    float(np.max(margins)))) if margins is not None else 0.3,
                   "margin_tuning": tuning,
                   "rebuilds_per_replica_mean": float(np.mean(rb_all)),
                   "rebuilds_per_replica_max": float(np.max(rb_all)),
                   "energy_per_atom_mean": float(np.mean((per_rep[:, 1] + per_rep[:, 2]) /
                                                         np.array([r.n for r in all_reps]))),
                   "partition": {"ranks": ws, "replicas_rank0": len(reps), "atoms_rank0": ntot,
                                 "load_imbalance": float(loads.max() / loads.mean() - 1.0),
                                 "rule": "largest load first to the least loaded rank; load = atoms x "
                                         "(41 + neighbours within the search length)"},
                   "parallelism": "replica partition" if ws > 1 else "single",
                   "l2": "inputs larger than L2 (state 160 MB + pairlists)"},
        "looped_single_system": {"value": loop_value, "unit": UNIT, "md_steps": loop_steps,
                                 "replicas": len(looped), "atoms": loop_n,
                                 "note": "one handle per replica with >= 3 cells per axis, calculate() in "
                                         "turn, host wall clock"},
        "speedup_vs_looped": value / loop_value if loop_value else None,
        "pair_interactions_per_s": {"fp32": pairs * args.steps * mdn / (ms * 1e-3),
                                    "pairs_within_cutoff_per_step": pairs},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "kernel": "ke_force_fp32 (kick + second half drift, all replicas)",
                     "algorithmic_bytes_per_launch": force_bytes, "avg_launch_ms": avg_ms,
                     "launches": flaunch, "peak_kind": peak_kind},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
