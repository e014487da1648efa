"""The seeded workload generators against the fixtures built from them, and the
trajectory's rung bookkeeping (CPU only)."""
import json
import os

import numpy as np

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def test_trajectory_rung_fixture_frames_match_generator():
    from gfn1_rs import workloads
    with open(os.path.join(GOLDEN, "trajectory_rungs.json")) as fh:
        rec = json.load(fh)
    z, x = workloads.water_trajectory(96, frames=256)
    assert rec["numbers"] == [int(v) for v in z]
    for k, f in rec["frames"].items():
        assert np.max(np.abs(np.array(f["positions_angstrom"]) - x[int(k)])) <= 1e-11, k
        assert f["rung"] in (0, 1, 2, 3)
        assert f["electronic_temperature"] == (300.0 if f["rung"] < 3 else 3000.0)


def test_large_fixture_frames_match_generator():
    from gfn1_rs import workloads
    with open(os.path.join(GOLDEN, "large_systems.json")) as fh:
        rec = json.load(fh)
    z, x = workloads.water_trajectory(96, frames=3)
    for f, r in enumerate(rec["water96_traj"]):
        assert r["numbers"] == [int(v) for v in z]
        assert np.max(np.abs(np.array(r["positions_angstrom"]) - x[f])) <= 1e-11, f


def test_rung_usage_counts():
    from gfn1_rs import trajectory
    assert trajectory.rung_usage([0, 0, 1, 3, -1, 2]) == {"0": 2, "1": 1, "2": 1, "3": 1, "none": 1}
    assert trajectory.rung_usage(np.zeros(0, dtype=np.int32)) == {"0": 0, "1": 0, "2": 0, "3": 0, "none": 0}
