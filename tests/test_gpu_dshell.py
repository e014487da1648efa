"""d-shell elements and the halogen-bond term on the GPU against the oracle.

* the reference's own molecules with d shells: phosphine (P 3d) and
  ferrocene (Fe 3d) from tests/nonpbc_smoke.rs;
* the halogen-bond systems of the reference's src/halogen.rs tests (HF,
  C-Cl...O, C-Br...O, CH3Br...OH2): total energy, gradient, shell charges and
  the `halogen` energy term;
* every element Z = 1..86 in one batch: a bent XH2 and a homonuclear X2 per
  element at covalent-radius distances, randomly rotated so that every
  Cartesian component of the d blocks is exercised (seed 7).

Tolerances: |dE| <= 1e-6 Eh, max|dg| <= 1e-5 Eh/bohr, max|dq_shell| <= 1e-5 e,
with the SCC converged tightly (1e-10 Eh / 1e-8 e) on both sides.
"""
import os

import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, ROOT, smoke_molecule

pytestmark = pytest.mark.gpu

E_TOL, G_TOL, Q_TOL = 1e-6, 1e-5, 1e-5
TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)


@pytest.fixture
def calc(gpu_calc):
    saved = dict(gpu_calc.opts)
    gpu_calc.opts.update(TIGHT)
    yield gpu_calc
    gpu_calc.opts.clear()
    gpu_calc.opts.update(saved)


def _check_one(calc, oracle_mod, z, x):
    r = calc.calculate_flat([0, len(z)], z, x, raise_on_error=True)
    o = oracle_mod.run(z, x, options=oracle_mod.make_options(**TIGHT))
    assert r.status[0] == 0
    assert abs(r.energy[0] - o.energy) <= E_TOL
    assert np.max(np.abs(r.gradient - o.gradient)) <= G_TOL
    assert np.max(np.abs(r.shell_charges - o.shell_charges)) <= Q_TOL
    for k, name in ((2, "repulsion"), (3, "electronic"), (7, "dispersion"), (8, "halogen")):
        assert abs(r.terms[0, k] - o.terms[name]) <= E_TOL, name
    return r, o


@pytest.mark.parametrize("name", ["phosphine", "ferrocene"])
def test_reference_d_shell_molecules(calc, oracle_mod, fixtures, name):
    z, x = smoke_molecule(fixtures, name)
    _check_one(calc, oracle_mod, z, x)


@pytest.mark.parametrize("title", ["HF", "CCl...O", "CBr...O", "CH3Br...OH2 halogen bond"])
def test_halogen_systems(calc, oracle_mod, fixtures, title):
    rec = fixtures["halogen_tests"][title]
    z, x = np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR
    r, o = _check_one(calc, oracle_mod, z, x)
    e_hal, _ = oracle_mod.halogen(z, x, gradient=False)
    assert abs(r.terms[0, 8] - e_hal) <= 1e-12
    if "Br" in title:
        assert r.terms[0, 8] < -1e-6  # the correction is active for bromine donors


def _rotation(rng):
    q = rng.normal(size=4)
    a, b, c, d = q / np.linalg.norm(q)
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def periodic_table_set(seed=7):
    """XH2 (bent, 95-120 degrees) and X2 for Z = 1..86 at covalent-radius bond
    lengths from the engine's tables, each randomly rotated and shifted."""
    covrad = None
    with open(os.path.join(ROOT, "gfn1-rs_b200", "data", "gfn1_tables.txt")) as fh:
        for line in fh:
            if line.startswith("covrad_ang "):
                covrad = [float(v) for v in line.split()[2:]]
    rng = np.random.default_rng(seed)
    mols = []
    for zz in range(1, 87):
        r = (covrad[zz] + covrad[1]) * ANGSTROM_TO_BOHR
        ang = np.deg2rad(rng.uniform(95.0, 120.0))
        x = np.array([[0, 0, 0], [r, 0, 0], [r * np.cos(ang), r * np.sin(ang), 0]])
        mols.append(([zz, 1, 1], x @ _rotation(rng).T + rng.normal(size=3)))
        r2 = 2.0 * covrad[zz] * ANGSTROM_TO_BOHR
        mols.append(([zz, zz], np.array([[0, 0, 0], [0, 0, r2]]) @ _rotation(rng).T))
    return mols


def test_every_element_in_one_batch(calc, oracle_mod):
    mols = periodic_table_set()
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    z = np.concatenate([z for z, _ in mols])
    x = np.concatenate([x for _, x in mols])
    r = calc.calculate_flat(off, z, x)
    worst = (0.0, 0.0, 0.0)
    for m, (zm, xm) in enumerate(mols):
        o = oracle_mod.run(zm, xm, options=oracle_mod.make_options(**TIGHT))
        assert r.status[m] == 0, (m, zm)
        a0, a1 = off[m], off[m + 1]
        s0, s1 = r.shell_offsets[m], r.shell_offsets[m + 1]
        de = abs(r.energy[m] - o.energy)
        dg = np.max(np.abs(r.gradient[a0:a1] - o.gradient))
        dq = np.max(np.abs(r.shell_charges[s0:s1] - o.shell_charges))
        assert de <= E_TOL and dg <= G_TOL and dq <= Q_TOL, (zm, de, dg, dq)
        worst = tuple(max(w, v) for w, v in zip(worst, (de, dg, dq)))
    print("worst |dE| %.2e  |dg| %.2e  |dq| %.2e" % worst)


def test_d_elements_on_the_large_molecule_path(oracle_mod, fixtures):
    """The same molecules through the many-SM large-molecule path (size
    threshold lowered to 16 AOs) agree with the one-CTA path and the oracle."""
    from gfn1_rs import BatchCalculator

    names = ["ferrocene", "phosphine"]
    mols = [smoke_molecule(fixtures, n) for n in names]
    rec = fixtures["halogen_tests"]["CH3Br...OH2 halogen bond"]
    mols.append((np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR))
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    z = np.concatenate([z for z, _ in mols])
    x = np.concatenate([x for _, x in mols])
    old = os.environ.get("GFN1_DENSE_N")
    os.environ["GFN1_DENSE_N"] = "16"
    try:
        got = BatchCalculator(**TIGHT).calculate_flat(off, z, x)
    finally:
        if old is None:
            os.environ.pop("GFN1_DENSE_N", None)
        else:
            os.environ["GFN1_DENSE_N"] = old
    ref = BatchCalculator(**TIGHT).calculate_flat(off, z, x)
    assert np.all(got.status == 0) and np.all(ref.status == 0)
    assert np.abs(got.energy - ref.energy).max() <= 1e-9
    assert np.abs(got.gradient - ref.gradient).max() <= 1e-8
    for m, (zm, xm) in enumerate(mols):
        o = oracle_mod.run(zm, xm, options=oracle_mod.make_options(**TIGHT))
        assert abs(got.energy[m] - o.energy) <= E_TOL
        assert abs(got.terms[m, 8] - o.terms["halogen"]) <= 1e-12


def test_learned_guess_with_other_elements():
    """Molecules with elements outside the guess network's H/C/N/O start from
    zero charges; the rest of the batch keeps the learned guess, and every
    molecule converges to the plain run's energy."""
    from gfn1_rs import BatchCalculator

    mols = periodic_table_set(seed=11)
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    z = np.concatenate([z for z, _ in mols])
    x = np.concatenate([x for _, x in mols])
    plain = BatchCalculator(**TIGHT).calculate_flat(off, z, x)
    learned = BatchCalculator(learned_guess=True, **TIGHT).calculate_flat(off, z, x)
    assert np.all(plain.status == 0) and np.all(learned.status == 0)
    assert np.abs(plain.energy - learned.energy).max() <= 1e-6
