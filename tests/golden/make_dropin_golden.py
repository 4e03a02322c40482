"""Runs the reference MDACP (CPU, plain build compiled from its sources into
oracle/_ref/) on the project inputs that tests/test_dropin.py feeds to the
GPU drop-in binary, and stores the reference's stdout as fixtures.  Both
sides start from the same state: the projects build it with the
reference's own seeded generators (one unit, id 0).

Usage:  python tests/golden/make_dropin_golden.py   (needs oracle/_ref built)
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import sys
import tempfile

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
OUT = pathlib.Path(__file__).resolve().parent

# name -> (cut-off, input lines)
CASES = {
    "benchmark_rc25": (2.5, {"Mode": "Benchmark", "Density": "0.5", "SystemSize": "12",
                             "TimeStep": "0.005", "ThermalizeLoop": "50", "TotalLoop": "300",
                             "ObserveLoop": "50", "InitialVelocity": "1.0"}),
    "langevin_nosehoover_rc25": (2.5, {"Mode": "Langevin", "Density": "0.7", "SystemSize": "12",
                                       "TimeStep": "0.005", "TotalLoop": "300", "ObserveLoop": "50",
                                       "InitialVelocity": "1.0", "HeatbathType": "NoseHoover",
                                       "AimedTemperature": "1.5", "HeatbathTau": "0.1"}),
    "collision_rc30": (3.0, {"Mode": "Collision", "SystemSize": "40", "TimeStep": "0.005",
                             "TotalLoop": "300", "ObserveLoop": "50"}),
    # the projects whose executors run after every step: gravity on the
    # atoms of a liquid cylinder (GravityImposer, src/phaseflow.cc:58-73) and
    # a piston compressing a gas against a wall, then cooling it
    # (MyPiston, src/rankine.cc:55-97); Burst thermalises and releases a
    # droplet (its ShellForce executor, src/burst.cc:67-99, is never run)
    "phaseflow_rc25": (2.5, {"Mode": "PhaseFlow", "SystemSize": "16", "TimeStep": "0.005",
                             "TotalLoop": "300", "ObserveLoop": "50", "InitialVelocity": "1.0"}),
    "rankine_rc25": (2.5, {"Mode": "Rankine", "Density": "0.2", "SystemSizeX": "16", "SystemSizeY": "16",
                           "SystemSizeZ": "40", "TimeStep": "0.005", "TotalLoop": "500", "ObserveLoop": "50",
                           "InitialVelocity": "1.0", "AimedTemperature": "0.5"}),
    "burst_rc25": (2.5, {"Mode": "Burst", "Density": "0.8", "SystemSize": "24", "Radius": "6",
                         "TimeStep": "0.005", "ThermalizeLoop": "100", "TotalLoop": "200", "ObserveLoop": "50",
                         "InitialVelocity": "0.9"}),
    # thermalise (Nose-Hoover), ChangeScale 1.05, then bubble histograms
    # (conf%04d.dat, one byte per grid cell) every ObserveLoop steps
    "cavitation_rc25": (2.5, {"Mode": "Cavitation", "Density": "0.7", "SystemSize": "12",
                              "TimeStep": "0.005", "ThermalizeLoop": "100", "TotalLoop": "200",
                              "ObserveLoop": "50", "InitialVelocity": "1.0", "AimedTemperature": "0.9",
                              "ChangeScale": "1.05", "GridSize": "3.0"}),
}


def cfg_text(lines):
    return "".join(f"{k}={v}\n" for k, v in lines.items())


def main():
    for name, (rc, lines) in CASES.items():
        tag = {2.5: "25", 3.0: "30"}[rc]
        binary = ROOT / "oracle" / "_ref" / f"mdacp_rc{tag}_plain"
        with tempfile.TemporaryDirectory() as wd:
            (pathlib.Path(wd) / "input.cfg").write_text(cfg_text(lines))
            out = subprocess.run([str(binary), "-i", "input.cfg"], cwd=wd, capture_output=True, text=True,
                                 env=dict(os.environ, OMP_NUM_THREADS="1"), check=True)
            for dat in sorted(pathlib.Path(wd).glob("conf*.dat")):  # bubble histograms
                (OUT / f"dropin_{name}.{dat.name}").write_bytes(dat.read_bytes())
        (OUT / f"dropin_{name}.cfg").write_text(cfg_text(lines))
        (OUT / f"dropin_{name}.ref.txt").write_text(out.stdout)
        print(name, len(out.stdout.splitlines()), "lines")


if __name__ == "__main__":
    main()
