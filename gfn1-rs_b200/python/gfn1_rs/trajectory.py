"""Energy + gradient along a trajectory, frames evaluated in batches.

Frames of one molecule are independent SCC problems, so a batch of frames is
one batched engine call.  Within a batch, the most recent converged charges
available are those of the previous batch's last frame; the starting guess of
each frame is chosen by `mode`:

* ``plain``: zero shell charges (the reference's default start);
* ``learned``: the learned initial guess of the frame's geometry;
* ``previous``: the converged shell charges of the previous batch's last frame;
* ``learned+previous``: the learned guess of the frame plus the previous
  batch's correction (converged charges minus the learned guess of that
  frame), so the network supplies the geometry dependence and the converged
  result removes its systematic error.

The first batch has no previous frame: ``previous`` starts from zero charges,
``learned+previous`` from the learned guess.  Every mode converges the same
SCC, so energies agree to the SCC tolerance.
"""
from __future__ import annotations

import time

import numpy as np

MODES = ("plain", "learned", "previous", "learned+previous")


def run_trajectory(numbers, frames_bohr, batch: int = 64, mode: str = "learned+previous", calc=None,
                   guess=None, compute_gradient: bool = True) -> dict:
    """frames_bohr: [F, nat, 3].  Returns per-frame energies, iterations,
    statuses, fallback-ladder rungs, gradients (if requested) and the wall time
    of the engine calls."""
    from .batch import BatchCalculator
    if mode not in MODES:
        raise ValueError(f"mode must be one of {MODES}")
    calc = calc or BatchCalculator()
    if mode in ("learned", "learned+previous") and guess is None:
        from .guess import LearnedGuess
        guess = LearnedGuess.from_file(calc.engine)
    z = np.asarray(numbers)
    frames = np.asarray(frames_bohr, dtype=np.float64)
    nf, nat = frames.shape[0], frames.shape[1]
    nsh_atom = calc.shell_offsets([0, nat], z)[-1]
    energy = np.zeros(nf)
    iters = np.zeros(nf, dtype=np.int32)
    status = np.zeros(nf, dtype=np.int32)
    rung = np.zeros(nf, dtype=np.int32)
    grads = np.zeros((nf, nat, 3)) if compute_gradient else None
    last_q = None      # converged shell charges of the last frame of the previous batch
    last_corr = None   # converged minus learned guess of that frame
    seconds = 0.0
    for b0 in range(0, nf, batch):
        b1 = min(nf, b0 + batch)
        k = b1 - b0
        off = (np.arange(k + 1) * nat).astype(np.int32)
        zz = np.tile(z, k)
        xx = frames[b0:b1].reshape(-1, 3)
        t0 = time.perf_counter()
        q0 = None
        learned_q = None
        if mode in ("learned", "learned+previous"):
            learned_q = guess.predict(off, zz, xx).reshape(k, nsh_atom)
        if mode == "learned":
            q0 = learned_q
        elif mode == "previous" and last_q is not None:
            q0 = np.tile(last_q, (k, 1))
        elif mode == "learned+previous":
            q0 = learned_q if last_corr is None else learned_q + last_corr[None, :]
        res = calc.calculate_flat(off, zz, xx, initial_shell_charges=None if q0 is None else q0.reshape(-1),
                                  compute_gradient=compute_gradient)
        seconds += time.perf_counter() - t0
        energy[b0:b1] = res.energy
        iters[b0:b1] = res.iterations
        status[b0:b1] = res.status
        rung[b0:b1] = res.rung
        if compute_gradient:
            grads[b0:b1] = res.gradient.reshape(k, nat, 3)
        qs = res.shell_charges.reshape(k, nsh_atom)
        last_q = qs[-1].copy()
        if learned_q is not None:
            last_corr = qs[-1] - learned_q[-1]
    return {"energy": energy, "iterations": iters, "status": status, "rung": rung, "gradient": grads,
            "seconds": seconds, "mode": mode, "batch": batch}


def rung_usage(rung) -> dict:
    """Frames per fallback-ladder rung ("0".."3"; "none" = not converged)."""
    rung = np.asarray(rung)
    out = {str(k): int(np.sum(rung == k)) for k in range(4)}
    out["none"] = int(np.sum(rung < 0))
    return out


def main():
    import argparse
    import json

    from . import workloads
    from .native import ANGSTROM_TO_BOHR
    ap = argparse.ArgumentParser(description="water-cluster trajectory stream, all guess modes")
    ap.add_argument("--waters", type=int, default=96)
    ap.add_argument("--frames", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=64)
    a = ap.parse_args()
    z, x = workloads.water_trajectory(a.waters, frames=a.frames)
    xb = x * ANGSTROM_TO_BOHR
    ref = None
    out = {}
    for mode in MODES:
        r = run_trajectory(z, xb, batch=a.batch, mode=mode)
        if ref is None:
            ref = r
        out[mode] = {"evals_per_s": a.frames / r["seconds"], "iterations_mean": float(r["iterations"].mean()),
                     "iterations_p95": float(np.percentile(r["iterations"], 95)),
                     "failed": int((r["status"] != 0).sum()), "rungs": rung_usage(r["rung"]),
                     "max_abs_dE_vs_plain": float(np.abs(r["energy"] - ref["energy"]).max())}
        print(mode, json.dumps(out[mode]), flush=True)


if __name__ == "__main__":
    main()
