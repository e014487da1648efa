"""Hessian driver and vibrational analysis on the CPU.

* vibrational_analysis against the reference's own unit tests
  (src/vibrational.rs:86-129): a single harmonic H oscillator and the five
  zero modes of a two-atom Hessian with one bond constant;
* the central-difference assembly is exact for a quadratic energy, the
  five-point stencil for a quartic one;
* the batched driver with the oracle as the gradient source on water:
  symmetric, translation sum rule, diagonal elements equal to the second
  difference of the energy.
"""
import numpy as np
import pytest

from conftest import smoke_molecule
from gfn1_rs import hessian as hs

TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)


def test_single_oscillator_wavenumber():
    h = np.zeros((3, 3))
    h[0, 0] = 1.0
    v = hs.vibrational_analysis(h, [1])
    m = hs.atomic_masses()[1]
    assert abs(m - 1.008) < 1e-12
    assert abs(v["wavenumbers"][-1] - np.sqrt(1.0 / m) * hs.WAVENUMBER_PER_SQRT_AU) < 1e-6
    assert abs(v["wavenumbers"][0]) < 1e-6 and abs(v["wavenumbers"][1]) < 1e-6


def test_translational_modes_are_zero():
    h = np.zeros((6, 6))
    k = 0.5
    h[0, 0] = h[3, 3] = k
    h[0, 3] = h[3, 0] = -k
    v = hs.vibrational_analysis(h, [1, 1])
    assert int(np.sum(np.abs(v["wavenumbers"]) < 1e-6)) == 5
    assert v["wavenumbers"][-1] > 0.0
    # modes are Cartesian: mass-weighted unit vectors divided by sqrt(m)
    assert np.allclose(np.linalg.norm(v["modes"], axis=1), 1.0 / np.sqrt(hs.atomic_masses()[1]))


def test_imaginary_modes_are_negative():
    h = -np.eye(3)
    v = hs.vibrational_analysis(h, [6])
    assert np.all(v["wavenumbers"] < 0.0)


def test_assembly_is_exact_for_a_quadratic_energy():
    rng = np.random.default_rng(3)
    nat = 4
    a = rng.normal(size=(3 * nat, 3 * nat))
    a = a + a.T
    x0 = rng.normal(size=(nat, 3))

    def evaluate(items):
        return [(True, (a @ x.ravel()).reshape(-1, 3)) for _, _, x, _ in items]

    out, calls = hs.hessian(evaluate, [([1] * nat, x0, None)], step=1e-2, chunk=5)
    assert calls == (6 * nat + 4) // 5
    assert np.max(np.abs(out[0] - a)) < 1e-11


def test_five_point_stencil_is_exact_for_a_quartic_energy():
    """g = a x + b x^3 (a quartic energy): central differences miss the
    Hessian a + diag(3 b x^2) by h^2 b, the five-point stencil is exact."""
    rng = np.random.default_rng(5)
    nat = 3
    a = rng.normal(size=(3 * nat, 3 * nat))
    a = a + a.T
    b = rng.uniform(0.5, 1.5, size=3 * nat)
    x0 = rng.normal(size=(nat, 3))
    exact = a + np.diag(3.0 * b * x0.ravel() ** 2)

    def evaluate(items):
        return [(True, (a @ x.ravel() + b * x.ravel() ** 3).reshape(-1, 3)) for _, _, x, _ in items]

    (h2,), _ = hs.hessian(evaluate, [([1] * nat, x0, None)], step=1e-2)
    (h4,), calls = hs.hessian(evaluate, [([1] * nat, x0, None)], step=1e-2, order=4, chunk=7)
    assert calls == (12 * nat + 6) // 7
    assert np.max(np.abs(h4 - exact)) < 1e-10
    assert np.max(np.abs(np.diag(h2 - exact) - b * 1e-4)) < 1e-10
    with pytest.raises(ValueError):
        hs.displacements(nat, 1e-2, order=3)


def test_failed_displacement_marks_the_molecule():
    def evaluate(items):
        return [(k != 3, np.zeros((len(z), 3))) for k, (_, z, _, _) in enumerate(items)]

    out, _ = hs.hessian(evaluate, [([1, 1], np.zeros((2, 3)), None), ([1], np.zeros((1, 3)), None)])
    assert out[0] is None and out[1] is not None


def test_oracle_water_hessian_properties(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "water")
    opt = oracle_mod.make_options(**TIGHT)
    r0 = oracle_mod.run(z, x, options=opt)

    def evaluate(items):
        out = []
        for _, zi, xi, q in items:
            r = oracle_mod.run(zi, xi, options=opt, init_shell_charges=q)
            out.append((r.converged, r.gradient))
        return out

    (h,), calls = hs.hessian(evaluate, [(z, x, r0.shell_charges)])
    assert calls == 1
    # translation sum rule: each row summed over one Cartesian direction of all atoms
    for k in range(3):
        assert np.max(np.abs(h[:, k::3].sum(axis=1))) < 1e-5
    # diagonal against the second difference of the energy
    e = lambda xx: oracle_mod.run(z, xx, options=opt, gradient=False).energy
    step = 5e-3
    for c in (0, 4, 8):
        xp, xm = x.copy(), x.copy()
        xp[c // 3, c % 3] += step
        xm[c // 3, c % 3] -= step
        d2 = (e(xp) - 2.0 * r0.energy + e(xm)) / step ** 2
        assert abs(d2 - h[c, c]) < 1e-4
    v = hs.vibrational_analysis(h, z)
    assert np.sum(v["wavenumbers"] > 1000.0) == 3  # bend and two stretches
