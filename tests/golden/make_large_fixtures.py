"""Oracle results for the large single systems, written to large_systems.json.

Config "water300": the 300-molecule water cluster (seed 1, 1.0 g/cm^3 cube,
O-O >= 2.6 A), 900 atoms, 2400 AOs.  Config "water96_traj": the first three
frames of the 96-water free-flight trajectory (seed 2, velocities seed 3,
0.5 fs steps, 0.002 A noise), 288 atoms, 768 AOs.  Both are converged tightly
(1e-8 Eh, 1e-7 e) so that a comparison measures arithmetic, not the
convergence threshold.  Run: python tests/golden/make_large_fixtures.py
(CPU only; takes tens of minutes for the 2400-AO system).
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "gfn1-rs_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from gfn1_rs import workloads  # noqa: E402

A2B = 1.8897261246257702
TIGHT = dict(energy_tolerance=1e-8, charge_tolerance=1e-7)


def record(z, x_ang):
    t0 = time.time()
    o = oracle.run(z, x_ang * A2B, options=oracle.make_options(**TIGHT))
    return {"numbers": [int(v) for v in z], "positions_angstrom": np.asarray(x_ang).round(12).tolist(),
            "energy": o.energy, "terms": o.terms, "gradient": o.gradient.tolist(),
            "shell_charges": o.shell_charges.tolist(), "iterations": int(o.iterations),
            "seconds": round(time.time() - t0, 1)}


def main():
    out = {"options": TIGHT}
    z, x = workloads.water_trajectory(96, frames=3)
    out["water96_traj"] = [record(z, x[f]) for f in range(3)]
    print("water96 frames done", [r["seconds"] for r in out["water96_traj"]], flush=True)
    z, x = workloads.water_cluster(300, 1)
    out["water300"] = record(z, x)
    print("water300 done", out["water300"]["seconds"], flush=True)
    with open(os.path.join(HERE, "large_systems.json"), "w") as f:
        json.dump(out, f)


if __name__ == "__main__":
    main()
