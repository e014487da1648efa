"""Trajectory stream (frames in batches): every starting-guess mode converges
to the same energies (|dE| <= 1e-6 Eh against the zero guess), and guesses
from the learned network and from the previous batch cut SCC iterations."""
import numpy as np
import pytest

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
