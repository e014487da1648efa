"""The large-molecule path (each molecule on a group of SMs: blocked Cholesky,
cooperative Householder reduction, Sturm/Laguerre eigenvalues, inverse
iteration, tensor-core back-transformation; the same SCC stage functions)
against the one-CTA-per-molecule path and the oracle.

Tolerances: between the two device paths |dE| <= 1e-9 Eh, |dg| <= 1e-8 Eh/bohr,
|dq| <= 1e-8 e at tight convergence; against the oracle the parity bar
(1e-6 Eh, 1e-5 Eh/bohr, 1e-5 e)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

A2B = 1.8897261246257702
TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)
LARGE = os.path.join(os.path.dirname(__file__), "golden", "large_systems.json")


def _run(off, z, x, dense_n=None, **opts):
    from gfn1_rs import BatchCalculator
    old = os.environ.get("GFN1_DENSE_N")
    if dense_n is not None:
        os.environ["GFN1_DENSE_N"] = str(dense_n)
    try:
        calc = BatchCalculator(**opts)
        return calc.calculate_flat(off, z, x)
    finally:
        if old is None:
            os.environ.pop("GFN1_DENSE_N", None)
        else:
            os.environ["GFN1_DENSE_N"] = old


def test_dense_path_matches_cta_path(gpu_calc):
    from gfn1_rs import workloads
    zs, xs, off = [], [], [0]
    for seed in (3, 11, 42):
        z, x = workloads.water_cluster(16 + seed % 5, seed)
        zs.append(z), xs.append(x * A2B), off.append(off[-1] + len(z))
    z2, x2 = workloads.mixed_molecule(1007)
    zs.append(z2), xs.append(x2 * A2B), off.append(off[-1] + len(z2))
    off = np.asarray(off, np.int32)
    z = np.concatenate(zs)
    x = np.concatenate(xs)
    ref = _run(off, z, x, **TIGHT)
    got = _run(off, z, x, dense_n=64, **TIGHT)
    assert np.all(ref.status == 0) and np.all(got.status == 0)
    assert np.abs(got.energy - ref.energy).max() <= 1e-9
    assert np.abs(got.gradient - ref.gradient).max() <= 1e-8
    assert np.abs(got.shell_charges - ref.shell_charges).max() <= 1e-8
    assert np.array_equal(got.iterations, ref.iterations)
    for k in (0, 1, 3, 4, 5, 14):
        assert np.abs(got.terms[:, k] - ref.terms[:, k]).max() <= 1e-9


def test_dense_path_zero_and_learned_guess_agree(gpu_calc):
    from gfn1_rs import BatchCalculator, workloads
    z, x = workloads.water_cluster(20, 7)
    off = np.array([0, len(z)], np.int32)
    old = os.environ.get("GFN1_DENSE_N")
    os.environ["GFN1_DENSE_N"] = "64"
    try:
        plain = BatchCalculator(**TIGHT).calculate_flat(off, z, x * A2B)
        learned = BatchCalculator(learned_guess=True, **TIGHT).calculate_flat(off, z, x * A2B)
    finally:
        if old is None:
            os.environ.pop("GFN1_DENSE_N", None)
        else:
            os.environ["GFN1_DENSE_N"] = old
    assert abs(plain.energy[0] - learned.energy[0]) <= 1e-8
    assert learned.iterations[0] <= plain.iterations[0]


@pytest.mark.skipif(not os.path.exists(LARGE), reason="large-system oracle fixtures not generated")
def test_large_systems_match_oracle(gpu_calc):
    from gfn1_rs import BatchCalculator
    fx = json.load(open(LARGE))
    opts = fx["options"]
    calc = BatchCalculator(**opts)
    cases = list(fx.get("water96_traj", []))
    if "water300" in fx:
        cases.append(fx["water300"])
    assert cases
    for rec in cases:
        z = np.array(rec["numbers"])
        x = np.array(rec["positions_angstrom"]) * A2B
        r = calc.calculate_flat([0, len(z)], z, x)
        assert r.status[0] == 0
        de = abs(r.energy[0] - rec["energy"])
        dg = np.abs(r.gradient - np.array(rec["gradient"])).max()
        dq = np.abs(r.shell_charges - np.array(rec["shell_charges"])).max()
        print(f"{len(z)} atoms: dE {de:.2e} dg {dg:.2e} dq {dq:.2e} iterations {r.iterations[0]} vs {rec['iterations']}")
        assert de <= 1e-6 and dg <= 1e-5 and dq <= 1e-5


def test_mixed_sizes_in_one_call_match_the_cta_path(gpu_calc):
    """Large molecules of different sizes in one call run in lockstep on the
    many-SM path (threshold 100 AOs) next to small ones on the one-CTA path;
    every molecule equals its one-CTA result."""
    from gfn1_rs import workloads
    zs, xs, off = [], [], [0]
    for k, seed in ((13, 5), (3, 6), (20, 7), (9, 8), (17, 9)):
        z, x = workloads.water_cluster(k, seed)
        zs.append(z), xs.append(x * A2B), off.append(off[-1] + len(z))
    off = np.asarray(off, np.int32)
    z, x = np.concatenate(zs), np.concatenate(xs)
    ref = _run(off, z, x, **TIGHT)
    got = _run(off, z, x, dense_n=100, **TIGHT)
    assert np.all(ref.status == 0) and np.all(got.status == 0)
    assert np.abs(got.energy - ref.energy).max() <= 1e-9
    assert np.abs(got.gradient - ref.gradient).max() <= 1e-8
    assert np.abs(got.shell_charges - ref.shell_charges).max() <= 1e-8
    assert np.array_equal(got.iterations, ref.iterations)


def test_fallback_ladder_on_the_large_molecule_path(gpu_calc, oracle_mod, fixtures):
    """C-Br...O needs rung 1 of the reference's ladder (linear mixing with a
    level shift, src/electronic.rs:1413-1447); on the many-SM path it takes the
    same rung as the oracle and lands on the oracle's energy."""
    from gfn1_rs import BatchCalculator
    rec = fixtures["halogen_tests"]["CBr...O"]
    z, x = np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * A2B
    off = np.array([0, len(z)], np.int32)
    old = os.environ.get("GFN1_DENSE_N")
    os.environ["GFN1_DENSE_N"] = "8"
    try:
        r = BatchCalculator().calculate_flat(off, z, x)
    finally:
        if old is None:
            os.environ.pop("GFN1_DENSE_N", None)
        else:
            os.environ["GFN1_DENSE_N"] = old
    o = oracle_mod.run(z, x)
    assert r.status[0] == 0 and r.rung[0] == o.rung == 1
    assert abs(r.energy[0] - o.energy) <= 1e-6
    assert np.abs(r.gradient - o.gradient).max() <= 1e-5



def test_last_wide_plan_reports_the_autotuned_reduction(gpu_calc):
    """gfn1_last_wide_plan: the autotuner's choice after a call with a
    large molecule (a panel width and a minimum row count among its
    candidates, at least one CTA per molecule, a measured time), all zeros
    after a call without one."""
    import ctypes

    from gfn1_rs import BatchCalculator, _lib, workloads

    def plan(calc):
        v = [ctypes.c_int32() for _ in range(3)] + [ctypes.c_double(), ctypes.c_int32()]
        _lib.check(_lib.load().gfn1_last_wide_plan(calc.engine.handle, *[ctypes.byref(t) for t in v]),
                   calc.engine.handle)
        return [t.value for t in v]

    old = os.environ.pop("GFN1_WIDE_PANEL", None)
    try:
        calc = BatchCalculator()
        z, x = workloads.water_cluster(40, 7)  # 320 AOs: above the 256-AO threshold
        r = calc.calculate_flat([0, len(z)], z, x * A2B)
        assert r.status[0] == 0
        nb, mr, g, ms, tuned = plan(calc)
        assert nb in (8, 16, 32) and mr in (4, 8, 16, 32, 64, 128) and g >= 1 and ms > 0.0 and tuned == 1
        z, x = workloads.water_cluster(4, 7)  # 32 AOs: one SM
        calc.calculate_flat([0, len(z)], z, x * A2B)
        assert plan(calc) == [0, 0, 0, 0.0, 0]
    finally:
        if old is not None:
            os.environ["GFN1_WIDE_PANEL"] = old
