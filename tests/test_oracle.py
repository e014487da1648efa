"""The CPU FP64 oracle against the reference's own fixtures and gates.

* examples/h2.engrad (the only stored absolute result): energy to 1e-9 Eh;
  the gradient to 1e-7 Eh/bohr (the file's gradient differs from the exact
  derivative of its own energy by 2.6e-8 Eh/bohr; see test_h2_gradient_is_exact_derivative);
* the finite-difference gradient gate of tests/nonpbc_smoke.rs:108-150
  (h = 1e-4 bohr, 5e-5 Eh/bohr) on its H/B/F/O/P molecules;
* the single-coordinate probe of tests/nonpbc_smoke.rs:152-180 on caffeine;
* mixer independence (tests/scf_accelerators.rs:41-75), translation/rotation
  invariance (tests/physical_consistency.rs:285-302) and the energy bookkeeping
  identity (src/electronic.rs:4057-4125).
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, smoke_molecule


def test_h2_golden(oracle_mod, fixtures):
    g = fixtures["h2_engrad"]
    r = oracle_mod.run(g["numbers"], g["positions_bohr"], gradient=True)
    assert r.converged
    assert abs(r.energy - g["energy"]) < 1e-9
    assert np.max(np.abs(r.gradient - np.array(g["gradient"]))) < 1e-7


# D3(BJ) energy of H2 at 0.74 A with the GFN1 parameters, the reference's
# known answer (src/dispersion.rs:3389-3396, tolerance 5e-10 Eh there)
D3_H2_074 = -0.000035462980


def test_d3_h2_known_answer(oracle_mod):
    x = np.array([[0.0, 0.0, 0.0], [0.74, 0.0, 0.0]]) * ANGSTROM_TO_BOHR
    r = oracle_mod.run([1, 1], x, gradient=False)
    assert abs(r.terms["dispersion"] - D3_H2_074) < 5e-10


def test_h2_gradient_is_exact_derivative(oracle_mod, fixtures):
    g = fixtures["h2_engrad"]
    opt = oracle_mod.make_options(energy_tolerance=1e-12, charge_tolerance=1e-10)
    x0 = np.array(g["positions_bohr"])

    def e(dx):
        x = x0.copy()
        x[1, 0] += dx
        return oracle_mod.run(g["numbers"], x, options=opt, gradient=False).energy

    fd = lambda h: (e(h) - e(-h)) / (2 * h)
    rich = (4 * fd(1e-3) - fd(2e-3)) / 3
    an = oracle_mod.run(g["numbers"], x0, options=opt).gradient[1, 0]
    assert abs(rich - an) < 1e-10


@pytest.mark.parametrize("name", ["hydrogen", "hydrogen fluoride", "water", "phosphine", "borane"])
def test_fd_gradient_gate(oracle_mod, fixtures, name):
    z, x = smoke_molecule(fixtures, name)
    r = oracle_mod.run(z, x, gradient=True)
    h = 1e-4
    for a in range(len(z)):
        for k in range(3):
            xp, xm = x.copy(), x.copy()
            xp[a, k] += h
            xm[a, k] -= h
            fd = (oracle_mod.run(z, xp, gradient=False).energy - oracle_mod.run(z, xm, gradient=False).energy) / (2 * h)
            assert abs(fd - r.gradient[a, k]) < 5e-5


def test_caffeine_single_coordinate_probe(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    r = oracle_mod.run(z, x, gradient=True)
    h = 1e-4
    xp, xm = x.copy(), x.copy()
    xp[0, 0] += h
    xm[0, 0] -= h
    fd = (oracle_mod.run(z, xp, gradient=False).energy - oracle_mod.run(z, xm, gradient=False).energy) / (2 * h)
    assert abs(fd - r.gradient[0, 0]) < 1e-4


def test_mixer_independence(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    tight = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)
    eb = oracle_mod.run(z, x, options=oracle_mod.make_options(scc_broyden=True, **tight), gradient=False).energy
    el = oracle_mod.run(z, x, options=oracle_mod.make_options(scc_broyden=False, max_scc=800, **tight),
                        gradient=False).energy
    assert abs(eb - el) < 1e-7


ACCEL = dict(energy_tolerance=1e-9, charge_tolerance=1e-8, max_scc=1000)


@pytest.mark.parametrize("name", ["water", "bromoethanol"])
def test_accelerator_consistency(oracle_mod, fixtures, name):
    """tests/scf_accelerators.rs:41-75 on its own molecules and options:
    linear mixing lands on Broyden's energy (1e-7 Eh) and a 0.15 Eh level
    shift does not move it (1e-6 Eh)."""
    rec = fixtures["scf_accelerators"][name]
    z, x = rec["numbers"], np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR
    e = {k: oracle_mod.run(z, x, options=oracle_mod.make_options(**kw, **ACCEL), gradient=False)
         for k, kw in (("broyden", {}), ("linear", dict(scc_broyden=False)), ("shift", dict(level_shift=0.15)))}
    assert all(r.rung == 0 for r in e.values())
    assert abs(e["linear"].energy - e["broyden"].energy) < 1e-7
    assert abs(e["shift"].energy - e["broyden"].energy) < 1e-6


def test_translation_rotation_invariance(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "water")
    r0 = oracle_mod.run(z, x)
    rng = np.random.default_rng(5)
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, a, b, c = q
    R = np.array([[1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)],
                  [2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)],
                  [2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)]])
    x2 = x @ R.T + np.array([3.0, -7.0, 11.0])
    r1 = oracle_mod.run(z, x2)
    assert abs(r0.energy - r1.energy) < 1e-9
    assert np.max(np.abs(r0.gradient @ R.T - r1.gradient)) < 1e-7
    assert np.max(np.abs(r0.gradient.sum(axis=0))) < 1e-9


def test_energy_bookkeeping(oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    t = oracle_mod.run(z, x, gradient=False).terms
    comp = sum(t[k] for k in ("repulsion", "electronic", "isotropic_scc", "third_order", "higher_order",
                              "dispersion", "halogen", "multipole", "exchange", "spin_polarization", "plus_u",
                              "external_field"))
    assert abs(comp - t["total_internal"]) < 1e-12
    assert abs(t["total_internal"] + t["electronic_entropy"] - t["total_free"]) < 1e-12


def test_reference_example_geometries(oracle_mod, fixtures):
    for name in ("water", "ammonia", "methane"):
        rec = fixtures["xyz"][name]
        r = oracle_mod.run(rec["numbers"], np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR)
        assert r.converged and np.isfinite(r.energy)
        assert abs(r.atomic_charges.sum()) < 1e-6


def test_robust_ladder_recovers(oracle_mod, fixtures):
    """max_scc = 1 fails rung 0; the linear-mixing + level-shift rungs of the
    fallback ladder (src/electronic.rs:1390-1447) converge to the same energy."""
    z, x = smoke_molecule(fixtures, "water")
    r0 = oracle_mod.run(z, x, gradient=False)
    assert r0.rung == 0 and r0.electronic_temperature == 300.0
    r = oracle_mod.run(z, x, options=oracle_mod.make_options(max_scc=1), gradient=False)
    assert r.converged and r.iterations > 1
    assert r.rung == 1 and r.electronic_temperature == 300.0  # linear mixing 0.2 + level shift 0.2 Eh
    assert abs(r.energy - r0.energy) < 1e-6


def test_ladder_rungs_in_a_batch(oracle_mod, fixtures):
    """Per-molecule rungs from the threaded batch: rung 1 where max_scc = 1
    stops rung 0, -1 (with status SccNotConverged) where no rung converges."""
    z, x = smoke_molecule(fixtures, "water")
    off = np.array([0, len(z), 2 * len(z)], dtype=np.int32)
    zz, xx = np.concatenate([z, z]), np.concatenate([x, x])
    out = oracle_mod.run_batch(off, zz, xx, options=oracle_mod.make_options(max_scc=1), gradient=False,
                               with_rungs=True)
    assert out[-1].tolist() == [1, 1] and out[5].tolist() == [0, 0]
    stuck = oracle_mod.make_options(max_scc=2, energy_tolerance=0.0, charge_tolerance=0.0)
    out = oracle_mod.run_batch(off, zz, xx, options=stuck, gradient=False, with_rungs=True)
    assert out[-1].tolist() == [-1, -1] and out[5].tolist() == [8, 8]


def test_charged_h2_cation_aufbau(oracle_mod):
    """tests/nonpbc_smoke.rs (charged doublet H2+): charge +1, T_el = 0,
    no dispersion; one electron, a singly occupied orbital, atomic charges
    summing to +1."""
    x = np.array([[0.0, 0.0, 0.0], [0.74, 0.0, 0.0]]) * ANGSTROM_TO_BOHR
    opt = oracle_mod.make_options(electronic_temperature=0.0, enable_dispersion=False, charge=1.0)
    r = oracle_mod.run([1, 1], x, options=opt)
    assert r.converged
    assert abs(r.occupations.sum() - 1.0) < 1e-10
    assert np.any(np.abs(r.occupations - 1.0) < 1e-10)
    assert abs(r.atomic_charges.sum() - 1.0) < 1e-6


def test_spin_multiplicity_triplet_o2(oracle_mod):
    """Spin-constrained occupations (src/electronic.rs:3930-4045, tests at
    :4173-4183): O2 as a triplet at T_el = 0 has two singly occupied orbitals;
    the same count with the wrong parity is rejected as incompatible."""
    x = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.21]]) * ANGSTROM_TO_BOHR
    opt = oracle_mod.make_options(electronic_temperature=0.0, spin_multiplicity=3)
    r = oracle_mod.run([8, 8], x, options=opt)
    assert r.converged
    assert int(np.sum(np.abs(r.occupations - 1.0) < 1e-10)) == 2
    assert abs(r.occupations.sum() - 12.0) < 1e-10
    with pytest.raises(oracle_mod.OracleError) as ei:
        oracle_mod.run([8, 8], x, options=oracle_mod.make_options(spin_multiplicity=2))
    assert ei.value.code == 3 and "incompatible" in str(ei.value)
    # multiplicity 1 is the closed-shell filling: the same result as no multiplicity
    a = oracle_mod.run([8, 8], x, options=oracle_mod.make_options(spin_multiplicity=1))
    b = oracle_mod.run([8, 8], x)
    assert abs(a.energy - b.energy) < 1e-10


def test_spin_multiplicity_doublet_h2_cation(oracle_mod):
    """tests/nonpbc_smoke.rs charged doublet with spin_multiplicity = 2."""
    x = np.array([[0.0, 0.0, 0.0], [0.74, 0.0, 0.0]]) * ANGSTROM_TO_BOHR
    opt = oracle_mod.make_options(electronic_temperature=0.0, enable_dispersion=False, charge=1.0,
                                  spin_multiplicity=2)
    r = oracle_mod.run([1, 1], x, options=opt)
    assert r.converged
    assert abs(r.occupations.sum() - 1.0) < 1e-10
    assert np.any(np.abs(r.occupations - 1.0) < 1e-10)
    assert abs(r.atomic_charges.sum() - 1.0) < 1e-6


def test_spin_multiplicity_gradient_is_derivative(oracle_mod):
    """The analytic gradient stays the derivative of the free energy with
    spin-constrained Fermi occupations (triplet CH2, 300 K)."""
    x = np.array([[0.0, 0.0, 0.0], [0.0, 0.95, 0.55], [0.0, -0.95, 0.55]]) * ANGSTROM_TO_BOHR
    opt = oracle_mod.make_options(energy_tolerance=1e-11, charge_tolerance=1e-9, spin_multiplicity=3)
    r = oracle_mod.run([6, 1, 1], x, options=opt)
    h = 1e-4
    for a, k in ((0, 2), (1, 1), (2, 2)):
        xp, xm = x.copy(), x.copy()
        xp[a, k] += h
        xm[a, k] -= h
        fd = (oracle_mod.run([6, 1, 1], xp, options=opt, gradient=False).energy
              - oracle_mod.run([6, 1, 1], xm, options=opt, gradient=False).energy) / (2 * h)
        assert abs(fd - r.gradient[a, k]) < 5e-5


def test_d_shell_rotation_invariance(oracle_mod, fixtures):
    """The five real d functions transform among themselves under rotation only
    with the right combination coefficients (src/basis.rs:406-436): the
    ferrocene energy is invariant under random rotations."""
    z, x = smoke_molecule(fixtures, "ferrocene")
    opt = oracle_mod.make_options(energy_tolerance=1e-10, charge_tolerance=1e-8)
    e0 = oracle_mod.run(z, x, options=opt, gradient=False).energy
    rng = np.random.default_rng(4)
    for _ in range(2):
        q = rng.normal(size=4)
        a, b, c, d = q / np.linalg.norm(q)
        R = np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                      [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                      [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])
        e = oracle_mod.run(z, x @ R.T, options=opt, gradient=False).energy
        assert abs(e - e0) < 1e-8
