"""The oracle's halogen-bond term against the reference's own halogen tests
(src/halogen.rs unit tests, systems extracted into the golden fixtures):

* no correction for F and Cl donors (no CXB entry for them);
* the correction is active (below -1e-6 Eh) for C-Br...O;
* non-zero for CH3Br...OH2;
* analytic gradient equal to the central finite difference (h = 1e-4 bohr)
  to 1e-8 Eh/bohr;
plus the term's place in the total energy and gradient of a full SCC.
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR


def halogen_system(fixtures, title):
    rec = fixtures["halogen_tests"][title]
    return np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR


@pytest.mark.parametrize("title", ["HF", "CCl...O"])
def test_fluorine_and_chlorine_have_no_correction(oracle_mod, fixtures, title):
    z, x = halogen_system(fixtures, title)
    e, g = oracle_mod.halogen(z, x)
    assert e == 0.0
    assert np.all(g == 0.0)


def test_bromine_correction_is_active(oracle_mod, fixtures):
    z, x = halogen_system(fixtures, "CBr...O")
    e, _ = oracle_mod.halogen(z, x)
    assert e < -1e-6


def test_ch3br_water_is_nonzero(oracle_mod, fixtures):
    z, x = halogen_system(fixtures, "CH3Br...OH2 halogen bond")
    e, g = oracle_mod.halogen(z, x)
    assert e != 0.0
    assert np.max(np.abs(g.sum(axis=0))) < 1e-14  # translation invariance


@pytest.mark.parametrize("title", ["CBr...O", "CH3Br...OH2 halogen bond"])
def test_halogen_gradient_matches_finite_difference(oracle_mod, fixtures, title):
    z, x = halogen_system(fixtures, title)
    _, g = oracle_mod.halogen(z, x)
    h = 1e-4
    for a in range(len(z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (oracle_mod.halogen(z, xp, gradient=False)[0] - oracle_mod.halogen(z, xm, gradient=False)[0]) / (2 * h)
            assert abs(g[a, k] - fd) < 1e-8


def test_halogen_term_in_full_scc(oracle_mod, fixtures):
    """The SCC reports the term under `halogen`, adds it to the totals, and the
    total gradient stays the derivative of the total energy."""
    z, x = halogen_system(fixtures, "CH3Br...OH2 halogen bond")
    opt = oracle_mod.make_options(energy_tolerance=1e-10, charge_tolerance=1e-8)
    r = oracle_mod.run(z, x, options=opt, gradient=True)
    e_hal, _ = oracle_mod.halogen(z, x)
    assert r.terms["halogen"] == e_hal
    parts = ("repulsion", "electronic", "isotropic_scc", "third_order", "dispersion", "halogen")
    assert abs(sum(r.terms[k] for k in parts) - r.terms["total_internal"]) < 1e-10
    h = 1e-4
    for a in (1, 5):  # Br and O
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (oracle_mod.run(z, xp, options=opt, gradient=False).energy
                  - oracle_mod.run(z, xm, options=opt, gradient=False).energy) / (2 * h)
            assert abs(fd - r.gradient[a, k]) < 5e-5
