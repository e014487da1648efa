"""Gfn1NativeCalculator.optimize / hessian / vibrational_frequencies (the
reference's pyo3 methods, src/python.rs:490-546, :1747-1850) on the engine."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WATER = [8, 1, 1]
WATER_XYZ = [[0.0, 0.0, 0.12], [0.0, 0.80, -0.45], [0.0, -0.72, -0.50]]  # Angstrom, distorted


def test_optimize_water(gpu_calc, tmp_path):
    from gfn1_rs import Gfn1NativeCalculator

    calc = Gfn1NativeCalculator()
    e0 = calc.calculate(WATER, WATER_XYZ).energy_hartree
    path = tmp_path / "opt.xyz"
    r = calc.optimize(WATER, WATER_XYZ, trajectory_path=str(path))
    assert r.converged and r.max_gradient <= 1e-4
    assert r.energy_hartree < e0
    assert np.array(r.positions_angstrom).shape == (3, 3)
    assert len(r.trajectory_positions_angstrom) == len(r.trajectory_energies_hartree) >= 2
    assert np.allclose(r.trajectory_positions_angstrom[0], WATER_XYZ)
    assert abs(r.trajectory_energies_hartree[-1] - r.energy_hartree) < 1e-12
    # the final geometry's gradient from a fresh single point
    g = np.array(calc.calculate(WATER, r.positions_angstrom, compute_gradient=True).gradient_hartree_per_bohr)
    assert np.max(np.abs(g - np.array(r.gradient_hartree_per_bohr))) < 1e-5
    assert path.read_text().count("energy_hartree=") == len(r.trajectory_energies_hartree)
    with pytest.raises(ValueError):
        calc.optimize(WATER, WATER_XYZ, cell=[[5, 0, 0], [0, 5, 0], [0, 0, 5]])


def test_hessian_and_frequencies(gpu_calc):
    from gfn1_rs import Gfn1NativeCalculator
    from gfn1_rs.hessian import hessian_batch
    from gfn1_rs.native import ANGSTROM_TO_BOHR

    calc = Gfn1NativeCalculator()
    opt = calc.optimize(WATER, WATER_XYZ)
    h = np.array(calc.hessian(WATER, opt.positions_angstrom))
    assert h.shape == (9, 9) and np.allclose(h, h.T)
    ref = hessian_batch(gpu_calc, [0, 3], np.array(WATER), np.array(opt.positions_angstrom) * ANGSTROM_TO_BOHR)
    assert np.max(np.abs(h - ref["hessians"][0])) < 1e-6
    v = calc.vibrational_frequencies(WATER, opt.positions_angstrom)
    w = np.array(v["wavenumbers"])
    assert np.sum(w > 1000.0) == 3  # bend and two stretches
    assert np.all(np.abs(w[:6]) < 100.0)  # translations and rotations at the minimum
    assert np.array(v["modes"]).shape == (9, 9)
