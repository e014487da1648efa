"""Repeated calls with the same topology (a trajectory, an optimiser loop, a
benchmark) reuse the one-shot batch's layout and only stage new coordinates:
every result equals that of a fresh calculator, and any change of atom
offsets, atomic numbers, charges, options or learned guess is picked up."""
import numpy as np
import pytest

A2B = 1.8897261246257702
pytestmark = pytest.mark.gpu


def _fresh(off, z, x, **kw):
    from gfn1_rs import BatchCalculator

    calc_kw = {k: kw.pop(k) for k in list(kw) if k in ("learned_guess", "charge_tolerance", "max_scc")}
    return BatchCalculator(**calc_kw).calculate_flat(off, z, x, **kw)


def _same(a, b):
    assert np.array_equal(a.status, b.status)
    assert np.array_equal(a.iterations, b.iterations)
    assert np.array_equal(a.energy, b.energy)
    assert np.array_equal(a.gradient, b.gradient)
    assert np.array_equal(a.shell_charges, b.shell_charges)


def test_repeated_topology_matches_fresh_calculators(gpu_calc):
    from gfn1_rs import BatchCalculator, workloads

    off, z, x = workloads.mixed_batch(64, 7000)
    x = x * A2B
    rng = np.random.default_rng(3)
    calc = BatchCalculator()
    for step in range(3):  # new coordinates, same topology
        xs = x + rng.normal(0.0, 0.02, x.shape)
        _same(calc.calculate_flat(off, z, xs), _fresh(off, z, xs))
    # charges given, then changed, then dropped again
    ch = np.zeros(len(off) - 1)
    ch[::7] = 1.0
    _same(calc.calculate_flat(off, z, x, charges=ch), _fresh(off, z, x, charges=ch))
    ch2 = ch.copy()
    ch2[1] = -1.0
    _same(calc.calculate_flat(off, z, x, charges=ch2), _fresh(off, z, x, charges=ch2))
    _same(calc.calculate_flat(off, z, x), _fresh(off, z, x))
    # initial charges on one call only
    r0 = calc.calculate_flat(off, z, x)
    q0 = r0.shell_charges + rng.normal(0.0, 1e-3, r0.shell_charges.shape)
    _same(calc.calculate_flat(off, z, x, initial_shell_charges=q0), _fresh(off, z, x, initial_shell_charges=q0))
    _same(calc.calculate_flat(off, z, x), r0)
    # a changed atomic number with the same offsets (O -> S: another basis,
    # a d shell, the shell offsets of every later molecule move)
    z2 = np.array(z, copy=True)
    z2[int(np.flatnonzero(z2 == 8)[0])] = 16
    _same(calc.calculate_flat(off, z2, x), _fresh(off, z2, x))
    _same(calc.calculate_flat(off, z, x), r0)
    # a changed option: energies agree with a fresh calculator at that option
    calc.opts["charge_tolerance"] = 1e-7
    _same(calc.calculate_flat(off, z, x), _fresh(off, z, x, charge_tolerance=1e-7))
    calc.opts["charge_tolerance"] = 2e-5
    _same(calc.calculate_flat(off, z, x), r0)


def test_repeated_topology_follows_the_learned_guess(gpu_calc):
    from gfn1_rs import BatchCalculator, workloads

    off, z, x = workloads.mixed_batch(48, 7100)
    x = x * A2B
    calc = BatchCalculator(learned_guess=True)
    learned = calc.calculate_flat(off, z, x)
    _same(learned, _fresh(off, z, x, learned_guess=True))
    calc.guess.detach()  # zero initial charges from here on
    _same(calc.calculate_flat(off, z, x), _fresh(off, z, x))
    calc.guess.attach()
    _same(calc.calculate_flat(off, z, x), learned)
