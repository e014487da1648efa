"""The optional ElectronicResult members (S, H0, P, W, orbital energies,
occupations, Fock matrix, shell potential, coordination numbers) through
gfn1_last_molecule_matrices / gfn1_last_molecule_fock and their resident-batch
twins against the oracle's, on both device paths.

Tolerances: S and H0 to 1e-12 (geometry only), coordination numbers to 1e-10;
P, W, F, orbital energies, occupations and the shell potential to 1e-6 at
tight SCC convergence (1e-10 Eh, 1e-8 e)."""
import os

import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, smoke_molecule

pytestmark = pytest.mark.gpu

TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)


def _molecules(fixtures):
    mols = [smoke_molecule(fixtures, n) for n in ("water", "phosphine", "ferrocene", "caffeine")]
    rec = fixtures["halogen_tests"]["CH3Br...OH2 halogen bond"]
    mols.append((np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR))
    return mols


def _flat(mols):
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    return off, np.concatenate([z for z, _ in mols]), np.concatenate([x for _, x in mols])


def _check(mats, o, full_spectrum):
    assert np.max(np.abs(mats["S"] - o.S)) <= 1e-12
    assert np.max(np.abs(mats["H0"] - o.H0)) <= 1e-12
    assert np.max(np.abs(mats["P"] - o.P)) <= 1e-6
    assert np.max(np.abs(mats["W"] - o.W)) <= 1e-6
    assert np.max(np.abs(mats["occupations"] - o.occupations)) <= 1e-6
    eps = mats["orbital_energies"]
    known = ~np.isnan(eps)
    assert known[-1] and known[:int(np.sum(o.occupations > 1e-12))].all()
    if full_spectrum:
        assert known.all()
    assert np.max(np.abs(eps[known] - o.orbital_energies[known])) <= 1e-6
    # fock, shell_scc_potential, coordination_numbers (src/electronic.rs:600-620)
    assert np.max(np.abs(mats["fock"] - o.F)) <= 1e-6
    assert np.max(np.abs(mats["shell_scc_potential"] - o.shell_potential)) <= 1e-6
    assert np.max(np.abs(mats["coordination_numbers"] - o.coordination_numbers)) <= 1e-10


@pytest.mark.parametrize("dense_n", [None, 16])
def test_matrices_match_oracle(gpu_calc, oracle_mod, fixtures, dense_n):
    from gfn1_rs import BatchCalculator

    mols = _molecules(fixtures)
    off, z, x = _flat(mols)
    calc = BatchCalculator(**TIGHT)
    old = os.environ.get("GFN1_DENSE_N")
    if dense_n is not None:
        os.environ["GFN1_DENSE_N"] = str(dense_n)  # read by each call
    try:
        r = calc.calculate_flat(off, z, x)
    finally:
        if old is None:
            os.environ.pop("GFN1_DENSE_N", None)
        else:
            os.environ["GFN1_DENSE_N"] = old
    assert np.all(r.status == 0)
    for m, (zm, xm) in enumerate(mols):
        o = oracle_mod.run(zm, xm, options=oracle_mod.make_options(**TIGHT), matrices=True)
        mats = calc.molecule_matrices(m)
        _check(mats, o, full_spectrum=False)
    with pytest.raises(IndexError):
        calc.molecule_matrices(len(mols))


def test_resident_batch_matrices(gpu_calc, oracle_mod, fixtures):
    import torch
    from gfn1_rs import BatchCalculator

    mols = _molecules(fixtures)[:3]
    off, z, x = _flat(mols)
    calc = BatchCalculator(**TIGHT)
    rb = calc.resident(off, z)
    rb.set_positions(x)
    s = torch.cuda.Stream()
    rb.launch(s.cuda_stream)
    for m, (zm, xm) in enumerate(mols):
        o = oracle_mod.run(zm, xm, options=oracle_mod.make_options(**TIGHT), matrices=True)
        _check(rb.molecule_matrices(m), o, full_spectrum=False)
    rb.close()
