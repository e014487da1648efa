"""Batched Hessians on the GPU against the same central differences of the
oracle's gradient (same step 5e-3 bohr, tight SCC, warm start from the
converged charges): max |dH| <= 1e-5 Eh/bohr^2 and wavenumbers above
100 cm^-1 within 0.05 cm^-1.  Plus the ASE unit conversion (eV/Angstrom^2)."""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, smoke_molecule

pytestmark = pytest.mark.gpu

TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)


def _molecules(fixtures):
    mols = [smoke_molecule(fixtures, n) for n in ("water", "phosphine", "borane")]
    for name in ("ammonia", "methane"):
        rec = fixtures["xyz"][name]
        mols.append((np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR))
    rec = fixtures["halogen_tests"]["CH3Br...OH2 halogen bond"]
    mols.append((np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR))
    return mols


def test_batched_hessians_match_oracle(gpu_calc, oracle_mod, fixtures):
    from gfn1_rs import hessian as hs

    mols = _molecules(fixtures)
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    z = np.concatenate([z for z, _ in mols])
    x = np.concatenate([x for _, x in mols])
    saved = dict(gpu_calc.opts)
    out = hs.hessian_batch(gpu_calc, off, z, x)
    assert gpu_calc.opts == saved  # options restored
    assert out["engine_calls"] == 2
    assert np.all(out["status"] == 0)
    opt = oracle_mod.make_options(**TIGHT)

    def evaluate(items):
        res = []
        for _, zi, xi, q in items:
            r = oracle_mod.run(zi, xi, options=opt, init_shell_charges=q)
            res.append((r.converged, r.gradient))
        return res

    for m, (zm, xm) in enumerate(mols):
        r0 = oracle_mod.run(zm, xm, options=opt)
        (ho,), _ = hs.hessian(evaluate, [(zm, xm, r0.shell_charges)])
        h = out["hessians"][m]
        assert h.shape == (3 * len(zm), 3 * len(zm))
        assert np.max(np.abs(h - ho)) <= 1e-5, m
        wg = hs.vibrational_analysis(h, zm)["wavenumbers"]
        wo = hs.vibrational_analysis(ho, zm)["wavenumbers"]
        big = np.abs(wo) > 100.0
        assert np.max(np.abs(wg[big] - wo[big])) <= 0.05, m


def test_five_point_hessian_matches_oracle(gpu_calc, oracle_mod, fixtures):
    """order=4 (five-point stencil, h = 1e-2 bohr) on water and ammonia against
    the same stencil over the oracle's gradient, and against the central
    differences: the two stencils differ by the O(h^2) truncation only."""
    from gfn1_rs import hessian as hs

    mols = _molecules(fixtures)[:1] + _molecules(fixtures)[3:4]
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    z = np.concatenate([z for z, _ in mols])
    x = np.concatenate([x for _, x in mols])
    out4 = hs.hessian_batch(gpu_calc, off, z, x, order=4)
    out2 = hs.hessian_batch(gpu_calc, off, z, x)
    assert np.all(out4["status"] == 0) and out4["order"] == 4
    opt = oracle_mod.make_options(**TIGHT)

    def evaluate(items):
        return [(r.converged, r.gradient) for r in
                (oracle_mod.run(zi, xi, options=opt, init_shell_charges=q) for _, zi, xi, q in items)]

    for m, (zm, xm) in enumerate(mols):
        r0 = oracle_mod.run(zm, xm, options=opt)
        (ho,), _ = hs.hessian(evaluate, [(zm, xm, r0.shell_charges)], order=4)
        h4, h2 = out4["hessians"][m], out2["hessians"][m]
        assert np.max(np.abs(h4 - ho)) <= 1e-5, m
        assert np.max(np.abs(h4 - h2)) <= 1e-3 * np.max(np.abs(h4)), m


def test_ase_hessian_units(gpu_calc, fixtures):
    from gfn1_rs import hessian as hs
    from gfn1_rs.ase import _BOHR, _HARTREE, _INVCM_EV, GFN1RSCalculator

    class Atoms:
        def __init__(self, z, x):
            self.z, self.x = z, x

        def get_atomic_numbers(self):
            return self.z

        def get_positions(self):
            return self.x

        def get_pbc(self):
            return np.array([False] * 3)

    z, xb = smoke_molecule(fixtures, "water")
    atoms = Atoms(z, xb / ANGSTROM_TO_BOHR)
    calc = GFN1RSCalculator()
    h_ev = calc.get_hessian(atoms)
    ref = hs.hessian_batch(gpu_calc, [0, len(z)], z, xb)["hessians"][0]
    assert np.max(np.abs(h_ev - ref * _HARTREE / _BOHR ** 2)) <= 1e-6
    vib = calc.get_vibrational_frequencies(atoms)
    assert np.allclose(vib["energies_ev"], vib["wavenumbers"] * _INVCM_EV)
    assert np.sum(vib["wavenumbers"] > 1000.0) == 3
