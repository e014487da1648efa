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
    """Frame 64 of the 96-water trajectory (768 AOs, the many-SM path) against
    tests/golden/trajectory_rungs.json.  At the default options (the
    trajectory workload's): the same fallback-ladder rung, and energies within
    1e-5 Eh, since both stop at the default thresholds (1e-6 Eh, 2e-5 e)
    rather than at a fixed point.  Converged tightly (1e-10 Eh, 1e-8 e) on
    both sides: the parity bar, |dE| <= 1e-6 Eh and max|dg| <= 1e-5 Eh/bohr."""
    from gfn1_rs import BatchCalculator, trajectory
    with open(os.path.join(ROOT, "tests", "golden", "trajectory_rungs.json")) as fh:
        rec = json.load(fh)
    z = np.array(rec["numbers"])
    f = rec["frames"]["64"]
    x = np.array(f["positions_angstrom"]) * A2B
    off = np.array([0, len(z)], np.int32)
    r = BatchCalculator().calculate_flat(off, z, x, compute_gradient=False)
    assert r.status[0] == 0
    assert r.rung[0] == f["rung"]
    assert abs(r.energy[0] - f["energy"]) <= 1e-5
    print("rungs", trajectory.rung_usage(r.rung), "iterations", r.iterations.tolist(), "oracle", f["iterations"])
    t = f["tight"]
    rt = BatchCalculator(**t["options"]).calculate_flat(off, z, x)
    assert rt.status[0] == 0 and rt.rung[0] == t["rung"]
    de = abs(rt.energy[0] - t["energy"])
    dg = np.abs(rt.gradient - np.array(t["gradient"])).max()
    print(f"tight: dE {de:.2e} dg {dg:.2e} iterations {rt.iterations[0]} vs {t['iterations']}")
    assert de <= 1e-6 and dg <= 1e-5
