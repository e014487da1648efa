"""Throughput of the single-system and trajectory workloads on the GPU.

    python -m gfn1_rs.configs [--frames 256]

* water16: the 16-water cluster (48 atoms, 128 AOs, seed 0), one molecule per
  call through Gfn1NativeCalculator, tight convergence (1e-8 Eh, 1e-7 e);
* water300: the 300-water cluster (900 atoms, 2400 AOs, seed 1), tight
  convergence, through the large-molecule path;
* water96 trajectory: the 96-water free-flight trajectory (seed 2,
  velocities seed 3) in batches of 64 frames, default convergence, every
  starting-guess mode of gfn1_rs.trajectory;
* Hessians: the first 256 molecules of the bench's mixed batch (seeds
  1000 + i), semi-numerical Hessians through gfn1_rs.hessian.hessian_batch
  (6N displaced gradients per molecule, batched).

Each line is JSON: evals/s, SCC iterations, frames per fallback-ladder rung
(trajectories) and, for the guess modes, the largest energy difference to the
zero-guess run.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import trajectory, workloads
from .batch import BatchCalculator
from .native import ANGSTROM_TO_BOHR

TIGHT = dict(energy_tolerance=1e-8, charge_tolerance=1e-7)


def single(z, x_bohr, reps: int, **kw):
    calc = BatchCalculator(**TIGHT, **kw)
    off = [0, len(z)]
    r = calc.calculate_flat(off, z, x_bohr)  # warm-up (allocations)
    t0 = time.perf_counter()
    for _ in range(reps):
        r = calc.calculate_flat(off, z, x_bohr)
    dt = (time.perf_counter() - t0) / reps
    return {"evals_per_s": 1.0 / dt, "seconds": dt, "iterations": int(r.iterations[0]),
            "energy": float(r.energy[0]), "status": int(r.status[0])}


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--frames", type=int, default=256)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--only", choices=("all", "single", "trajectory", "hessian"), default="all")
    ap.add_argument("--modes", default=",".join(trajectory.MODES),
                    help="comma-separated starting-guess modes of the trajectory (the first is the dE reference)")
    a = ap.parse_args()
    if a.only in ("all", "hessian"):
        hessians(256)
    if a.only in ("all", "single"):
        singles()
    if a.only in ("all", "trajectory"):
        trajectories(a.frames, a.batch, tuple(m for m in a.modes.split(",") if m))


def hessians(nmol: int):
    from .hessian import hessian_batch
    off, z, x = workloads.mixed_batch(nmol, 1000)
    xb = np.ascontiguousarray(x * ANGSTROM_TO_BOHR)
    calc = BatchCalculator()
    hessian_batch(calc, off[:9], z[:off[8]], xb[:off[8]])  # warm-up (allocations)
    t0 = time.perf_counter()
    out = hessian_batch(calc, off, z, xb)
    dt = time.perf_counter() - t0
    ndisp = int(6 * (off[-1] - off[0]))
    print(json.dumps({"workload": f"semi-numerical Hessians, {nmol} mixed clusters (seeds 1000+i)",
                      "hessians_per_s": nmol / dt, "seconds": dt, "displaced_gradients": ndisp,
                      "gradients_per_s": (ndisp + nmol) / dt, "engine_calls": out["engine_calls"],
                      "failed": int((out["status"] != 0).sum())}), flush=True)


def singles():
    for name, (z, x), reps in (("water16", workloads.water_cluster(16, 0), 20),
                               ("water300", workloads.water_cluster(300, 1), 2)):
        xb = np.ascontiguousarray(x * ANGSTROM_TO_BOHR)
        plain = single(z, xb, reps)
        learned = single(z, xb, reps, learned_guess=True)
        print(json.dumps({"workload": name, "plain": plain, "learned": learned,
                          "abs_dE": abs(plain["energy"] - learned["energy"])}), flush=True)


def trajectories(frames: int, batch: int, modes=trajectory.MODES):
    z, x = workloads.water_trajectory(96, frames=frames)
    xb = x * ANGSTROM_TO_BOHR
    calc = BatchCalculator()
    ref = None
    for mode in modes:
        trajectory.run_trajectory(z, xb[:batch], batch=batch, mode=mode, calc=calc)  # warm-up
        r = trajectory.run_trajectory(z, xb, batch=batch, mode=mode, calc=calc)
        ref = ref or r
        print(json.dumps({"workload": f"water96 trajectory, {frames} frames in batches of {batch}", "mode": mode,
                          "evals_per_s": frames / r["seconds"], "iterations_mean": float(r["iterations"].mean()),
                          "iterations_p95": float(np.percentile(r["iterations"], 95)),
                          "failed": int((r["status"] != 0).sum()), "rungs": trajectory.rung_usage(r["rung"]),
                          "max_abs_dE_vs_plain": float(np.abs(r["energy"] - ref["energy"]).max())}), flush=True)


if __name__ == "__main__":
    main()
