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


def _direct_form(z, x, tables):
    """The term evaluated in the reference's own arrangement (src/halogen.rs:64-160):
    energy from t^12 and t^6, then separate radial and three angular gradient
    pieces.  An independent restatement to cross-check the oracle's
    squared-distance form."""
    damp, rscale = tables["glob.xbdamp"][0], tables["glob.xbrad"][0]
    rad = np.array(tables["atomic_radius_ang"]) * ANGSTROM_TO_BOHR
    n = len(z)
    g = np.zeros((n, 3))
    e = 0.0
    for X in range(n):
        if z[X] not in (17, 35, 53, 85):
            continue
        nb = [j for j in range(n) if j != X and 1e-24 < ((x[j] - x[X]) ** 2).sum() <= 400.0]
        cc = 0.1 * tables.get(f"elem.{z[X]}.cxb", [0.0])[0]
        if not nb or cc == 0.0:
            continue
        K = min(nb, key=lambda j: ((x[j] - x[X]) ** 2).sum())
        for J in nb:
            if z[J] not in (7, 8, 15, 16):
                continue
            r0 = rscale * (rad[z[X]] + rad[z[J]])
            dxj, dxk, dkj = x[J] - x[X], x[K] - x[X], x[J] - x[K]
            d2jx, d2kx, d2jk = dxj @ dxj, dxk @ dxk, dkj @ dkj
            rjx, rkx = np.sqrt(d2jx) + 1e-18, np.sqrt(d2kx) + 1e-18
            xy = np.sqrt(d2kx * d2jx)
            term = (d2kx + d2jx - d2jk) / xy
            base = 0.5 - 0.25 * term
            t = r0 / rjx
            e += base ** 6 * cc * (t ** 12 - damp * t ** 6) / (1.0 + t ** 12)
            t6 = t ** 6
            num, den = t6 * t6 - damp * t6, 1.0 + t6 * t6
            radial = (12.0 * num * t6 * t6 / (rjx * den * den) + 6.0 * t6 * (damp - 2.0 * t6) / (rjx * den))
            radial *= base ** 6 * cc / rjx
            g[J] += dxj * radial
            g[X] -= dxj * radial
            pre = -1.5 * base ** 5 * cc * num / den
            c_jx = (2.0 / rkx - term / rjx) * pre / rjx
            c_kx = (2.0 / rjx - term / rkx) * pre / rkx
            c_jk = 2.0 * pre / xy
            g[J] += dxj * c_jx - dkj * c_jk
            g[X] -= dxj * c_jx + dxk * c_kx
            g[K] += dxk * c_kx + dkj * c_jk
    return e, g


def test_oracle_equals_direct_form(oracle_mod, fixtures):
    from conftest import ROOT
    import os

    tables = {}
    with open(os.path.join(ROOT, "gfn1-rs_b200", "data", "gfn1_tables.txt")) as fh:
        for line in fh:
            if line.strip() and not line.startswith("#"):
                p = line.split()
                tables[p[0]] = [float(v) for v in p[2:]]
    rng = np.random.default_rng(0)
    for title in fixtures["halogen_tests"]:
        z, x = halogen_system(fixtures, title)
        for trial in range(5):
            xt = x + (rng.normal(scale=0.3, size=x.shape) if trial else 0.0)
            e1, g1 = _direct_form(z, xt, tables)
            e2, g2 = oracle_mod.halogen(z, xt)
            assert abs(e1 - e2) < 1e-15
            assert np.max(np.abs(g1 - g2)) < 1e-15
