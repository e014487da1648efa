"""ASE calculator on the engine: unit conversions against the atomic-unit
calculator, and the batched path against single calls (1e-10 eV)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class FakeAtoms:
    """The three Atoms methods the calculator reads."""

    def __init__(self, numbers, positions, pbc=False):
        self.numbers = np.asarray(numbers)
        self.positions = np.asarray(positions, dtype=float)
        self.pbc = np.array([pbc] * 3)

    def get_atomic_numbers(self):
        return self.numbers

    def get_positions(self):
        return self.positions

    def get_pbc(self):
        return self.pbc


WATER = FakeAtoms([8, 1, 1], [[0.0, 0.0, 0.1173], [0.0, 0.7572, -0.4692], [0.0, -0.7572, -0.4692]])
AMMONIA = FakeAtoms([7, 1, 1, 1], [[0.0, 0.0, 0.1], [0.94, 0.0, -0.27], [-0.47, 0.81, -0.27], [-0.47, -0.81, -0.27]])


def test_units_match_native_calculator(gpu_calc):
    from gfn1_rs import Gfn1NativeCalculator
    from gfn1_rs.ase import _BOHR, _HARTREE, GFN1RSCalculator
    calc = GFN1RSCalculator()
    calc.calculate(WATER, ["energy", "forces"])
    r = calc.results
    nat = Gfn1NativeCalculator().calculate(WATER.numbers.tolist(), WATER.positions.tolist(), compute_gradient=True)
    assert abs(r["energy"] - nat.energy_hartree * _HARTREE) <= 1e-9
    g = np.asarray(nat.gradient_hartree_per_bohr)
    assert np.abs(r["forces"] + g * _HARTREE / _BOHR).max() <= 1e-8
    assert np.abs(r["charges"] - np.asarray(nat.charges)).max() <= 1e-10
    assert np.abs(r["dipole"] - np.asarray(nat.dipole) * _BOHR).max() <= 1e-10
    assert r["native_converged"] and r["native_iterations"] == nat.iterations
    assert abs(sum(r["charges"])) < 1e-8


def test_batched_many_matches_single(gpu_calc):
    from gfn1_rs.ase import GFN1RSCalculator
    calc = GFN1RSCalculator()
    many = calc.calculate_many([WATER, AMMONIA, WATER])
    for atoms, res in zip([WATER, AMMONIA, WATER], many):
        one = GFN1RSCalculator()
        one.calculate(atoms, ["energy", "forces"])
        assert abs(one.results["energy"] - res["energy"]) <= 1e-10
        assert np.abs(one.results["forces"] - res["forces"]).max() <= 1e-10


def test_learned_guess_same_energy(gpu_calc):
    from gfn1_rs.ase import GFN1RSCalculator
    plain = GFN1RSCalculator()
    learned = GFN1RSCalculator(learned_guess=True)
    a = plain.calculate_many([WATER, AMMONIA])
    b = learned.calculate_many([WATER, AMMONIA])
    for x, y in zip(a, b):
        assert abs(x["energy"] - y["energy"]) <= 1e-6 * 27.2114


def test_periodic_rejected(gpu_calc):
    from gfn1_rs.ase import GFN1RSCalculator
    with pytest.raises(ValueError):
        GFN1RSCalculator().calculate(FakeAtoms([1, 1], [[0, 0, 0], [0.74, 0, 0]], pbc=True), ["energy"])


def test_multiplicity_and_level_shift_parameters(gpu_calc):
    from gfn1_rs import BatchCalculator
    from gfn1_rs.ase import _HARTREE, GFN1RSCalculator
    from gfn1_rs.native import ANGSTROM_TO_BOHR

    o2 = FakeAtoms([8, 8], [[0.0, 0.0, 0.0], [0.0, 0.0, 1.21]])
    calc = GFN1RSCalculator(multiplicity=3, level_shift=0.1)
    calc.calculate(o2, ["energy"])
    ref = BatchCalculator(spin_multiplicity=3).calculate_flat([0, 2], o2.numbers, o2.positions * ANGSTROM_TO_BOHR)
    assert abs(calc.results["energy"] - ref.energy[0] * _HARTREE) <= 1e-5
