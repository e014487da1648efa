"""Spin-constrained occupations (a requested spin multiplicity,
src/electronic.rs:545-598 and :3930-4045) on the GPU against the oracle, on
both device paths.  Tolerances: |dE| <= 1e-6 Eh, max|dg| <= 1e-5 Eh/bohr,
max|dq_shell| <= 1e-5 e at tight SCC convergence."""
import os

import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR

pytestmark = pytest.mark.gpu

TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)
A = ANGSTROM_TO_BOHR
CASES = [  # (name, numbers, xyz (Angstrom), charge, multiplicity)
    ("O2 triplet", [8, 8], [[0.0, 0.0, 0.0], [0.0, 0.0, 1.21]], 0.0, 3),
    ("CH2 triplet", [6, 1, 1], [[0.0, 0.0, 0.0], [0.0, 0.95, 0.55], [0.0, -0.95, 0.55]], 0.0, 3),
    ("NH2 doublet", [7, 1, 1], [[0.0, 0.0, 0.0], [0.0, 0.80, 0.60], [0.0, -0.80, 0.60]], 0.0, 2),
    ("H2+ doublet", [1, 1], [[0.0, 0.0, 0.0], [0.74, 0.0, 0.0]], 1.0, 2),
    ("water singlet", [8, 1, 1], [[0.0, 0.0, 0.1173], [0.0, 0.7572, -0.4692], [0.0, -0.7572, -0.4692]], 0.0, 1),
]


def _flat(cases):
    off = np.concatenate([[0], np.cumsum([len(c[1]) for c in cases])]).astype(np.int32)
    z = np.concatenate([c[1] for c in cases])
    x = np.concatenate([np.array(c[2]) * A for c in cases])
    return off, z, x


@pytest.mark.parametrize("etemp", [300.0, 0.0])
@pytest.mark.parametrize("dense_n", [None, 4])
def test_spin_multiplicity_matches_oracle(gpu_calc, oracle_mod, etemp, dense_n):
    from gfn1_rs import BatchCalculator

    for mult in sorted({c[4] for c in CASES}):
        cases = [c for c in CASES if c[4] == mult]
        off, z, x = _flat(cases)
        calc = BatchCalculator(electronic_temperature=etemp, spin_multiplicity=mult, **TIGHT)
        old = os.environ.get("GFN1_DENSE_N")
        if dense_n is not None:
            os.environ["GFN1_DENSE_N"] = str(dense_n)
        try:
            r = calc.calculate_flat(off, z, x, charges=[c[3] for c in cases])
        finally:
            if old is None:
                os.environ.pop("GFN1_DENSE_N", None)
            else:
                os.environ["GFN1_DENSE_N"] = old
        for m, c in enumerate(cases):
            o = oracle_mod.run(c[1], np.array(c[2]) * A,
                               options=oracle_mod.make_options(electronic_temperature=etemp, charge=c[3],
                                                               spin_multiplicity=mult, **TIGHT))
            assert r.status[m] == 0, c[0]
            a0, a1 = off[m], off[m + 1]
            s0, s1 = r.shell_offsets[m], r.shell_offsets[m + 1]
            assert abs(r.energy[m] - o.energy) <= 1e-6, c[0]
            assert np.max(np.abs(r.gradient[a0:a1] - o.gradient)) <= 1e-5, c[0]
            assert np.max(np.abs(r.shell_charges[s0:s1] - o.shell_charges)) <= 1e-5, c[0]
            occ = calc.molecule_matrices(m)["occupations"]
            assert np.max(np.abs(occ - o.occupations)) <= 1e-6, c[0]
            if etemp == 0.0:
                assert int(np.sum(np.abs(occ - 1.0) < 1e-10)) == mult - 1, c[0]


def test_incompatible_multiplicity_is_rejected(gpu_calc):
    from gfn1_rs import BatchCalculator, Gfn1Error

    off, z, x = _flat([CASES[4]])
    calc = BatchCalculator(spin_multiplicity=2)
    r = calc.calculate_flat(off, z, x)
    assert r.status[0] == 3  # InvalidInput: 10 electrons cannot form a doublet
    with pytest.raises(Gfn1Error, match="incompatible"):
        calc.calculate_flat(off, z, x, raise_on_error=True)


def test_native_calculator_multiplicity(gpu_calc, oracle_mod):
    from gfn1_rs import Gfn1NativeCalculator

    name, z, xyz, charge, mult = CASES[0]
    r = Gfn1NativeCalculator(multiplicity=mult).calculate(z, xyz, compute_gradient=True)
    o = oracle_mod.run(z, np.array(xyz) * A, options=oracle_mod.make_options(spin_multiplicity=mult))
    assert r.converged and abs(r.energy_hartree - o.energy) <= 1e-6
    with pytest.raises(ValueError):
        Gfn1NativeCalculator(multiplicity=0)
