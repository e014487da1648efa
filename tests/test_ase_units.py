"""ASE calculator unit contract with the engine replaced by a fake (CPU only),
as the reference's pure-numpy conversion tests do (tests/python/test_ase_units.py
of gfn1-rs): energies, forces, charges, dipoles and the Hessian in ASE units are
the engine's atomic-unit values times the ASE factors, positions go to the
engine in Angstrom, and periodic systems are refused before any engine call."""
import numpy as np
import pytest

A2B = 1.8897261246257702


class Atoms:
    def __init__(self, z, x, pbc=False):
        self.z, self.x, self.pbc = np.asarray(z), np.asarray(x, dtype=float), pbc

    def get_atomic_numbers(self):
        return self.z

    def get_positions(self):
        return self.x

    def get_pbc(self):
        return np.array([self.pbc] * 3)


def _result(off, z, energies, grads, charges, dipoles):
    from gfn1_rs.batch import BatchResult
    nmol, nat = len(off) - 1, len(z)
    terms = np.zeros((nmol, 15))
    terms[:, 0] = energies
    shoff = np.asarray(off) * 2  # two shells per atom in this fake
    return BatchResult(np.asarray(energies, dtype=float), terms, grads, np.zeros(2 * nat), np.asarray(charges),
                       np.asarray(dipoles, dtype=float), np.zeros(nmol), np.full(nmol, 5, dtype=np.int32),
                       np.zeros(nmol, dtype=np.int32), np.asarray(off), shoff, np.zeros(nmol, dtype=np.int32))


class FakeEngine:
    """Stands in for BatchCalculator: a harmonic potential E = 1/2 x.K.x (bohr,
    Eh) per molecule, fixed charges and dipoles."""

    def __init__(self, k):
        self.k = k
        self.opts = {}
        self.seen_units = []

    def _eval(self, off, z, xb, compute_gradient=True):
        xb = np.asarray(xb, dtype=float).reshape(-1, 3)
        e, g = [], []
        for m in range(len(off) - 1):
            xm = xb[off[m]:off[m + 1]].ravel()
            e.append(0.5 * xm @ self.k @ xm)
            g.append((self.k @ xm).reshape(-1, 3))
        grads = np.concatenate(g) if compute_gradient else None
        nat = len(xb)
        return _result(off, z, e, grads, np.linspace(-0.2, 0.2, nat), [[0.1, -0.2, 0.3]] * (len(off) - 1))

    def calculate(self, molecules, unit="angstrom", charges=None, compute_gradient=True, raise_on_error=False):
        self.seen_units.append(unit)
        assert unit == "angstrom"
        off = np.concatenate([[0], np.cumsum([len(z) for z, _ in molecules])])
        z = np.concatenate([z for z, _ in molecules])
        x = np.concatenate([np.asarray(p) for _, p in molecules]) * A2B
        return self._eval(off, z, x, compute_gradient)

    def calculate_flat(self, atom_offsets, numbers, xyz_bohr, charges=None, initial_shell_charges=None,
                       compute_gradient=True, raise_on_error=False):
        return self._eval(np.asarray(atom_offsets), np.asarray(numbers), xyz_bohr, compute_gradient)


@pytest.fixture
def water():
    z = np.array([8, 1, 1])
    x = np.array([[0.0, 0.0, 0.1], [0.0, 0.76, -0.47], [0.0, -0.76, -0.47]])
    rng = np.random.default_rng(3)
    a = rng.normal(size=(9, 9))
    k = a @ a.T / 9.0 + np.eye(9) * 0.2  # symmetric positive definite force constants, Eh/bohr^2
    return z, x, k


def _calc(k):
    from gfn1_rs.ase import GFN1RSCalculator
    calc = GFN1RSCalculator()
    calc._batch = FakeEngine(k)
    return calc


def test_energy_forces_charges_dipole_units(water):
    from gfn1_rs.ase import _BOHR, _HARTREE
    z, x, k = water
    calc = _calc(k)
    atoms = Atoms(z, x)
    xb = (x * A2B).ravel()
    e_h, g = 0.5 * xb @ k @ xb, (k @ xb).reshape(-1, 3)
    assert calc.get_potential_energy(atoms) == pytest.approx(e_h * _HARTREE, rel=1e-14)
    assert np.allclose(calc.get_forces(atoms), -g * _HARTREE / _BOHR, rtol=1e-14, atol=0)
    assert np.allclose(calc.get_charges(atoms), np.linspace(-0.2, 0.2, 3))
    assert np.allclose(calc.get_dipole_moment(atoms), np.array([0.1, -0.2, 0.3]) * _BOHR, rtol=1e-15)
    assert calc.results["native_energy_terms_ev"]["total_free"] == pytest.approx(e_h * _HARTREE, rel=1e-14)
    assert set(calc._batch.seen_units) == {"angstrom"}


def test_calculate_many_matches_single(water):
    z, x, k = water
    calc = _calc(k)
    structures = [Atoms(z, x), Atoms(z, x + 0.05), Atoms(z, x - 0.02)]
    many = calc.calculate_many(structures)
    for s, r in zip(structures, many):
        single = _calc(k)
        assert r["energy"] == pytest.approx(single.get_potential_energy(s), rel=1e-14)
        assert np.allclose(r["forces"], single.get_forces(s), rtol=1e-14, atol=0)


def test_hessian_and_frequency_units(water):
    from gfn1_rs import hessian as hs
    from gfn1_rs.ase import _BOHR, _HARTREE, _INVCM_EV
    z, x, k = water
    calc = _calc(k)
    atoms = Atoms(z, x)
    h_ev = calc.get_hessian(atoms)
    # central differences of a linear gradient are exact: H = K up to rounding
    assert np.allclose(h_ev, k * _HARTREE / _BOHR ** 2, rtol=1e-8, atol=1e-8)
    vib = calc.get_vibrational_frequencies(atoms)
    ref = hs.vibrational_analysis(k, z)["wavenumbers"]
    assert np.allclose(vib["wavenumbers"], ref, rtol=1e-7, atol=1e-6)
    assert np.allclose(vib["energies_ev"], vib["wavenumbers"] * _INVCM_EV)
    assert calc._batch.opts == {}  # the Hessian driver restores the engine options


def test_periodic_atoms_are_refused(water):
    z, x, k = water
    calc = _calc(k)
    with pytest.raises(ValueError, match="non-periodic"):
        calc.get_potential_energy(Atoms(z, x, pbc=True))
