"""Trajectory stream (frames in batches): every starting-guess mode converges
to the same energies (|dE| <= 1e-6 Eh against the zero guess), and guesses
from the learned network and from the previous batch cut SCC iterations.
Late frames of the 96-water trajectory (768 AOs) land on the oracle's
fallback-ladder rung."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

A2B = 1.8897261246257702


def test_trajectory_modes_agree_and_save_iterations(gpu_calc):
    from gfn1_rs import trajectory, workloads
    z, x = workloads.water_trajectory(16, frames=12, seed=5, vseed=6)
    frames = x * A2B
    res = {m: trajectory.run_trajectory(z, frames, batch=4, mode=m) for m in trajectory.MODES}
    plain = res["plain"]
    assert np.all(plain["status"] == 0)
    for m, r in res.items():
        assert np.all(r["status"] == 0), m
        assert np.abs(r["energy"] - plain["energy"]).max() <= 1e-6, m
        usage = trajectory.rung_usage(r["rung"])
        assert sum(usage.values()) == len(frames) and usage["none"] == 0, m
    it = {m: r["iterations"].mean() for m, r in res.items()}
    print("mean iterations", it)
    assert it["learned"] < it["plain"]
    assert it["learned+previous"] <= it["learned"] + 0.5
    assert it["previous"] < it["plain"]


def test_late_frames_rungs_match_oracle(gpu_calc):
    """Frame 64 of the 96-water trajectory at the default options (the
    trajectory workload's), against tests/golden/trajectory_rungs.json: same
    rung and, since both stop at the default thresholds (1e-6 Eh, 2e-5 e)
    rather than at a tight fixed point, energies within 1e-5 Eh.  The later
    frames of the fixture need 139-170 iterations of a 768-AO SCC on one SM
    (over a minute each); the trajectory workload reports their rungs."""
    from gfn1_rs import BatchCalculator, trajectory
    with open(os.path.join(ROOT, "tests", "golden", "trajectory_rungs.json")) as fh:
        rec = json.load(fh)
    z = np.array(rec["numbers"])
    keys = ["64"]
    frames = [rec["frames"][k] for k in keys]
    x = np.concatenate([np.array(f["positions_angstrom"]) * A2B for f in frames])
    off = (np.arange(len(keys) + 1) * len(z)).astype(np.int32)
    r = BatchCalculator().calculate_flat(off, np.tile(z, len(keys)), x, compute_gradient=False)
    for i, f in enumerate(frames):
        assert r.status[i] == 0, keys[i]
        assert r.rung[i] == f["rung"], keys[i]
        assert abs(r.energy[i] - f["energy"]) <= 1e-5, keys[i]
    print("rungs", trajectory.rung_usage(r.rung), "iterations", r.iterations.tolist(),
          "oracle", [f["iterations"] for f in frames])
