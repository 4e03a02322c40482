"""Generates the golden fixtures in tests/golden/ by running the reference
MDACP itself (kohnakagawa/mdacp, compiled from its own sources by
oracle/ref/build_ref.sh) on seeded synthetic states through the test-only
OracleDump project (oracle/ref/ref_harness.cc).

Every fixture holds the injected state, the reference's pair set (directed,
by atom id), its forces (one kick with TimeStep = 1 on zeroed momenta), its
observer sums, and the end state of a short trajectory.  The reference has
no tests or golden data of its own, so these runs are the pin.

Usage:  python tests/golden/make_golden.py      (needs the reference tree)
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from mdacp_b200 import workloads as W  # noqa: E402
from oracle import lj_oracle as O  # noqa: E402

OUT = pathlib.Path(__file__).resolve().parent


def sorted_pairs(k, p):
    a = np.stack([k, p], axis=1).astype(np.int32)
    a = np.unique(a, axis=0)
    return a


def reference_case(name, state, steps, dt, extra_traj=None, threads=1, check_threads=None):
    L = state.L
    # forces, pairs and observables at the injected state (TimeStep = 1)
    wd, _ = O.run_reference("OracleDump", state.q, state.v, state.ids, L, state.rc, 1.0,
                            threads=threads, extra={"DumpForces": "yes"})
    dumps = [O.read_pair_dump(p) for p in sorted(wd.glob("out_pairs_u*.bin"))]
    k, p = O.reference_pairs_by_id(dumps, L)
    pairs = sorted_pairs(k, p)
    assert pairs.shape[0] == k.shape[0], "duplicate directed pair in the reference list"
    obs0 = O.read_observables(wd / "out_obs.txt")["initial"]
    _, f, fid = O.read_state_dump(wd / "out_forces.bin")
    forces = np.empty_like(f)
    forces[fid] = f
    n = state.n
    if check_threads:
        wd2, _ = O.run_reference("OracleDump", state.q, state.v, state.ids, L, state.rc, 1.0,
                                 threads=check_threads, extra={"DumpForces": "yes"})
        d2 = [O.read_pair_dump(p) for p in sorted(wd2.glob("out_pairs_u*.bin"))]
        k2, p2 = O.reference_pairs_by_id(d2, L)
        assert np.array_equal(sorted_pairs(k2, p2), pairs), f"{name}: unit layout changes the pair set"
        _, f2, fid2 = O.read_state_dump(wd2 / "out_forces.bin")
        ff = np.empty_like(f2)
        ff[fid2] = f2
        rel = np.abs(ff - forces).max() / np.abs(forces).max()
        assert rel < 1e-12, f"{name}: {check_threads}-unit forces differ by {rel}"
    # trajectory
    extra = {"Steps": str(steps), "ObserveLoop": str(max(1, steps // 4))}
    extra.update(extra_traj or {})
    wd3, _ = O.run_reference("OracleDump", state.q, state.v, state.ids, L, state.rc, dt,
                             threads=threads, extra=extra)
    obs = O.read_observables(wd3 / "out_obs.txt")
    tq, tp, tid = O.read_state_dump(wd3 / "out_state.bin")
    traj_q = np.empty_like(tq)
    traj_v = np.empty_like(tp)
    traj_q[tid] = tq
    traj_v[tid] = tp
    traj_obs = np.array([[obs[k]["ke"], obs[k]["pe"], obs[k]["virial"], obs[k]["temperature"],
                          obs[k]["pressure"]] for k in obs if k.startswith("step")])
    np.savez_compressed(
        OUT / f"{name}.npz",
        q=state.q, v=state.v, ids=state.ids, L=L, rc=state.rc, dt=dt, steps=steps,
        pairs=pairs, forces=forces,
        ke=obs0["ke"] * n, pe=obs0["pe"] * n, virial=obs0["virial"],
        temperature=obs0["temperature"], pressure=obs0["pressure"],
        traj_q=traj_q, traj_v=traj_v, traj_obs=traj_obs,
        constructions=obs["constructions"],
        thermostat=np.array(extra_traj.get("HeatbathType", "none") if extra_traj else "none"),
        aimed_temperature=float((extra_traj or {}).get("AimedTemperature", 1.0)),
        heatbath_tau=float((extra_traj or {}).get("HeatbathTau", 0.1)),
    )
    print(f"{name}: n={n} pairs={pairs.shape[0]} constructions={obs['constructions']:.0f}")


def face_gas(seed=5):
    """Dilute gas with atoms crowded against every face, edge and corner of
    the box, so that wrapped pairs and ghost-of-ghost images are frequent."""
    rng = np.random.Generator(np.random.Philox(seed))
    L = np.array([12.0, 12.0, 12.0])
    pts = []
    while len(pts) < 420:
        x = rng.random(3) * L
        # push two thirds of the atoms into the outer 0.6 shell on a random axis set
        if rng.random() < 0.66:
            for d in range(3):
                if rng.random() < 0.6:
                    x[d] = rng.uniform(0.0005, 0.6) if rng.random() < 0.5 else L[d] - rng.uniform(0.0005, 0.6)
        ok = True
        for y in pts:
            dd = x - y
            dd -= L * np.round(dd / L)
            if dd @ dd < 0.81:
                ok = False
                break
        if ok:
            pts.append(x)
    q = np.array(pts)
    v = W.maxwell_boltzmann(q.shape[0], 1.0, rng)
    return W.State(q=q, v=v, ids=np.arange(q.shape[0], dtype=np.int32), L=L, rc=2.5, dt=0.005,
                   temperature=1.0, name="face_gas")


def main():
    if not O.reference_binary(2.5).exists() or not O.reference_binary(3.0).exists():
        raise SystemExit("build the reference first: oracle/ref/build_ref.sh")
    s1 = W.fcc_liquid(6, 0.5, 1.0, seed=11, jitter=0.08, rc=2.5, dt=0.005)
    reference_case("fcc864_rho0.5_rc2.5", s1, steps=200, dt=0.005, check_threads=8)
    s2 = W.fcc_liquid(6, 0.8442, 0.722, seed=12, jitter=0.05, rc=2.5, dt=0.004)
    reference_case("fcc864_rho0.8442_rc2.5", s2, steps=200, dt=0.004)
    s3 = W.slab(2000, 0.75, 0.02, 0.9, seed=13, rc=3.0, dt=0.005)
    reference_case("slab2000_rc3.0", s3, steps=100, dt=0.005)
    s4 = W.fcc_liquid(6, 0.5, 1.0, seed=14, jitter=0.08, rc=2.5, dt=0.005)
    reference_case("nosehoover_fcc864", s4, steps=200, dt=0.005,
                   extra_traj={"ControlTemperature": "yes", "HeatbathType": "NoseHoover",
                               "AimedTemperature": "1.5", "HeatbathTau": "0.1"})
    s5 = face_gas()
    reference_case("face_gas420_rc2.5", s5, steps=200, dt=0.005)


if __name__ == "__main__":
    main()
