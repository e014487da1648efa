"""GPU engine vs the CPU FP64 oracle through the C ABI.

Tolerances (stated per result): |dE| <= 1e-6 Eh, max|dg| <= 1e-5 Eh/bohr,
max|dq_shell| <= 1e-5 e.  Both sides run the same SCC options; the SCC is
converged tightly (1e-10 Eh / 1e-8 e) in the parity cases so the comparison
measures the arithmetic, not the convergence threshold.
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, smoke_molecule

pytestmark = pytest.mark.gpu

E_TOL, G_TOL, Q_TOL = 1e-6, 1e-5, 1e-5
TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)


def _compare(calc, oracle_mod, z, x, opts=None, e_tol=E_TOL, g_tol=G_TOL, q_tol=Q_TOL):
    opts = opts or {}
    calc.opts.update(opts)
    r = calc.calculate_flat([0, len(z)], z, x, raise_on_error=True)
    o = oracle_mod.run(z, x, options=oracle_mod.make_options(**opts))
    assert r.status[0] == 0
    de = abs(r.energy[0] - o.energy)
    dg = np.max(np.abs(r.gradient - o.gradient))
    dq = np.max(np.abs(r.shell_charges - o.shell_charges))
    assert de <= e_tol, f"dE={de:.3e}"
    assert dg <= g_tol, f"dg={dg:.3e}"
    assert dq <= q_tol, f"dq={dq:.3e}"
    for k, name in enumerate(("total_free", "total_internal", "repulsion", "electronic", "isotropic_scc",
                              "third_order")):
        assert abs(r.terms[0, k] - o.terms[name]) <= e_tol, name
    return r, o


@pytest.fixture
def calc(gpu_calc):
    saved = dict(gpu_calc.opts)
    yield gpu_calc
    gpu_calc.opts.clear()
    gpu_calc.opts.update(saved)


def test_h2_golden_on_gpu(calc, fixtures):
    g = fixtures["h2_engrad"]
    r = calc.calculate_flat([0, 2], g["numbers"], g["positions_bohr"], raise_on_error=True)
    assert abs(r.energy[0] - g["energy"]) < 1e-9
    assert np.max(np.abs(r.gradient - np.array(g["gradient"]))) < 1e-7


def test_d3_h2_known_answer_on_gpu(calc):
    """D3(BJ) term of H2 at 0.74 A: the reference's known answer
    -3.5462980e-5 Eh (src/dispersion.rs:3389-3396, tolerance 5e-10 Eh)."""
    x = np.array([[0.0, 0.0, 0.0], [0.74, 0.0, 0.0]]) * ANGSTROM_TO_BOHR
    r = calc.calculate_flat([0, 2], [1, 1], x, raise_on_error=True)
    assert abs(r.terms[0, 7] - -0.000035462980) < 5e-10


@pytest.mark.parametrize("name", ["hydrogen", "hydrogen fluoride", "water", "borane", "caffeine"])
def test_reference_molecules(calc, oracle_mod, fixtures, name):
    z, x = smoke_molecule(fixtures, name)
    _compare(calc, oracle_mod, z, x, TIGHT, e_tol=1e-8, g_tol=1e-7, q_tol=1e-7)


@pytest.mark.parametrize("name", ["water", "ammonia", "methane"])
def test_reference_examples_default_options(calc, oracle_mod, fixtures, name):
    rec = fixtures["xyz"][name]
    z = np.array(rec["numbers"])
    x = np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR
    _compare(calc, oracle_mod, z, x)


def test_water16_cluster(calc, oracle_mod):
    from gfn1_rs import workloads

    z, x = workloads.water_cluster(16, 0)
    _compare(calc, oracle_mod, z, x * ANGSTROM_TO_BOHR, dict(energy_tolerance=1e-8))


def test_mixed_batch_vs_oracle(calc, oracle_mod):
    from gfn1_rs import workloads

    off, z, x = workloads.mixed_batch(48, 1000)
    xb = x * ANGSTROM_TO_BOHR
    r = calc.calculate_flat(off, z, xb, raise_on_error=True)
    e, g, q, shoff, it, st = oracle_mod.run_batch(off, z, xb)
    assert np.all(r.status == 0) and np.all(st == 0)
    assert np.max(np.abs(r.energy - e)) <= E_TOL
    assert np.max(np.abs(r.gradient - g)) <= G_TOL
    assert np.max(np.abs(r.shell_charges - q)) <= Q_TOL


def test_batch_order_independence_and_determinism(calc):
    from gfn1_rs import workloads

    off, z, x = workloads.mixed_batch(24, 2000)
    xb = x * ANGSTROM_TO_BOHR
    r1 = calc.calculate_flat(off, z, xb)
    r2 = calc.calculate_flat(off, z, xb)
    assert np.array_equal(r1.energy, r2.energy)
    assert np.array_equal(r1.gradient, r2.gradient)
    # each molecule alone gives the same numbers as inside the batch
    for m in (0, 7, 23):
        a0, a1 = off[m], off[m + 1]
        rs = calc.calculate_flat([0, a1 - a0], z[a0:a1], xb[a0:a1])
        assert abs(rs.energy[0] - r1.energy[m]) < 1e-12
        assert np.max(np.abs(rs.gradient - r1.gradient[a0:a1])) < 1e-12


def test_translation_invariance_gpu(calc, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    r0 = calc.calculate_flat([0, len(z)], z, x)
    r1 = calc.calculate_flat([0, len(z)], z, x + np.array([5.0, -3.0, 2.0]))
    assert abs(r0.energy[0] - r1.energy[0]) < 1e-9
    assert np.max(np.abs(r0.gradient.sum(axis=0))) < 1e-9


def test_element_without_parameters_is_rejected(calc, fixtures):
    z, x = smoke_molecule(fixtures, "water")
    z = z.copy()
    z[0] = 87  # the GFN1 parametrisation ends at Rn
    r = calc.calculate_flat([0, len(z)], z, x)
    assert r.status[0] == 4  # MissingElement


def test_not_converged_status_matches_oracle(calc, oracle_mod, fixtures):
    """Zero tolerances (|dE| < 0 never holds): every rung of the fallback ladder
    runs to its limit and both report SCC not converged."""
    z, x = smoke_molecule(fixtures, "water")
    opts = dict(max_scc=2, energy_tolerance=0.0, charge_tolerance=0.0)
    calc.opts.update(opts)
    r = calc.calculate_flat([0, len(z)], z, x)
    with pytest.raises(oracle_mod.OracleError) as ei:
        oracle_mod.run(z, x, options=oracle_mod.make_options(**opts), gradient=False)
    assert ei.value.code == 8
    assert r.status[0] == 8 and r.rung[0] == -1
    assert r.iterations[0] == 250  # the last rung's limit, max(max_scc, 250)


@pytest.mark.parametrize("name", ["water", "caffeine"])
def test_fallback_ladder_matches_oracle(calc, oracle_mod, fixtures, name):
    """max_scc = 1 leaves rung 0 unconverged; the device ladder (linear mixing +
    level shift, src/electronic.rs:1390-1447) must land where the oracle's does,
    with the same iteration count."""
    z, x = smoke_molecule(fixtures, name)
    calc.opts.update(max_scc=1)
    r = calc.calculate_flat([0, len(z)], z, x, raise_on_error=True)
    o = oracle_mod.run(z, x, options=oracle_mod.make_options(max_scc=1))
    assert r.status[0] == 0 and o.converged
    assert abs(r.energy[0] - o.energy) <= E_TOL
    assert np.abs(r.gradient - o.gradient).max() <= G_TOL
    assert np.abs(r.shell_charges - o.shell_charges).max() <= Q_TOL
    assert r.iterations[0] == o.iterations
    assert r.rung[0] == o.rung == 1  # linear mixing 0.2 with a 0.2 Eh level shift


def test_fallback_ladder_in_a_batch(calc, oracle_mod, fixtures):
    """Only the molecules rung 0 leaves unconverged are rerun; the others keep
    their rung-0 result."""
    zs, xs, off = [], [], [0]
    mols = [(np.array(fixtures["xyz"][n]["numbers"]), np.array(fixtures["xyz"][n]["positions_angstrom"]) * ANGSTROM_TO_BOHR)
            for n in ("water", "ammonia", "methane")]
    mols.append(smoke_molecule(fixtures, "caffeine"))
    for z, x in mols:
        zs.append(z), xs.append(x), off.append(off[-1] + len(z))
    off = np.array(off, np.int32)
    calc.opts.update(max_scc=7)  # caffeine needs 10 iterations at rung 0, the others 5-6
    r = calc.calculate_flat(off, np.concatenate(zs), np.concatenate(xs), raise_on_error=True)
    for k, (z, x) in enumerate(zip(zs, xs)):
        o = oracle_mod.run(z, x, options=oracle_mod.make_options(max_scc=7), gradient=False)
        assert abs(r.energy[k] - o.energy) <= E_TOL
        assert r.iterations[k] == o.iterations
        assert r.rung[k] == o.rung  # 1 for caffeine, 0 for the others
    assert r.rung.tolist() == [0, 0, 0, 1]


def test_charged_molecule(calc, oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "water")
    r = calc.calculate_flat([0, len(z)], z, x, charges=[1.0], raise_on_error=True)
    o = oracle_mod.run(z, x, options=oracle_mod.make_options(charge=1.0))
    assert abs(r.energy[0] - o.energy) < E_TOL
    assert abs(r.atomic_charges.sum() - 1.0) < 1e-8


def test_initial_guess_converges_to_same_result(calc, oracle_mod, fixtures):
    z, x = smoke_molecule(fixtures, "caffeine")
    o = oracle_mod.run(z, x)
    r = calc.calculate_flat([0, len(z)], z, x, initial_shell_charges=o.shell_charges, raise_on_error=True)
    assert abs(r.energy[0] - o.energy) < E_TOL
    assert r.iterations[0] <= o.iterations


def test_charged_h2_cation_aufbau_on_gpu(calc, oracle_mod):
    """The charged-doublet case of tests/nonpbc_smoke.rs (charge +1, T_el = 0,
    no dispersion) through the batch API: parity with the oracle and the
    reference's assertions on occupations and charges."""
    x = np.array([[0.0, 0.0, 0.0], [0.74, 0.0, 0.0]]) * ANGSTROM_TO_BOHR
    calc.opts.update(electronic_temperature=0.0, enable_dispersion=0)
    r = calc.calculate_flat([0, 2], [1, 1], x, charges=[1.0], raise_on_error=True)
    o = oracle_mod.run([1, 1], x, options=oracle_mod.make_options(electronic_temperature=0.0, enable_dispersion=False,
                                                                  charge=1.0))
    assert r.status[0] == 0
    assert abs(r.energy[0] - o.energy) <= E_TOL
    assert np.max(np.abs(r.gradient - o.gradient)) <= G_TOL
    assert abs(r.atomic_charges.sum() - 1.0) < 1e-6
    occ = calc.molecule_matrices(0)["occupations"]
    assert abs(occ.sum() - 1.0) < 1e-10 and np.any(np.abs(occ - 1.0) < 1e-10)
