"""256 random molecules (2-12 atoms of H, B, C, N, O, F, Si, P, S, Cl, Br, Ti,
Fe, Zn grown atom by atom at covalent-radius distances, charges -1/0/+1, seed
11) in one batch against the oracle at tight convergence: |dE| <= 1e-6 Eh,
max|dg| <= 1e-5 Eh/bohr, max|dq_shell| <= 1e-5 e, and the same status.  A
molecule with two SCC fixed points may land on either (checked against the
oracle's fixed points under 1e-12 bohr perturbations, at most 2% of them)."""
import os

import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, ROOT

pytestmark = pytest.mark.gpu

TIGHT = dict(energy_tolerance=1e-10, charge_tolerance=1e-8)
ELEMENTS = [1, 1, 1, 1, 5, 6, 6, 6, 7, 7, 8, 8, 9, 14, 15, 16, 17, 35, 26, 22, 30]


def random_molecules(n=256, seed=11):
    covrad = None
    with open(os.path.join(ROOT, "gfn1-rs_b200", "data", "gfn1_tables.txt")) as fh:
        for line in fh:
            if line.startswith("covrad_ang "):
                covrad = [float(v) for v in line.split()[2:]]
    rng = np.random.default_rng(seed)
    mols = []
    for _ in range(n):
        nat = int(rng.integers(2, 13))
        z, x = [int(rng.choice(ELEMENTS))], [np.zeros(3)]
        while len(z) < nat:
            zz, k = int(rng.choice(ELEMENTS)), int(rng.integers(len(z)))
            d = rng.normal(size=3)
            p = x[k] + d / np.linalg.norm(d) * (covrad[zz] + covrad[z[k]]) * rng.uniform(0.95, 1.1)
            if all(np.linalg.norm(p - q) > 0.85 * (covrad[zz] + covrad[zi]) for q, zi in zip(x, z)):
                z.append(zz)
                x.append(p)
        mols.append((np.array(z), np.array(x) * ANGSTROM_TO_BOHR))
    charges = rng.choice([-1.0, 0.0, 0.0, 1.0], size=n)
    return mols, charges


def test_random_molecules_match_oracle(oracle_mod):
    from gfn1_rs import BatchCalculator

    mols, ch = random_molecules()
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in mols])]).astype(np.int32)
    z = np.concatenate([m[0] for m in mols])
    x = np.concatenate([m[1] for m in mols])
    r = BatchCalculator(**TIGHT).calculate_flat(off, z, x, charges=ch)
    e, g, q, so, it, st = oracle_mod.run_batch(off, z, x, charges=ch, options=oracle_mod.make_options(**TIGHT),
                                               nthreads=os.cpu_count() or 4)
    assert np.array_equal(r.status, st)
    ok = st == 0
    assert ok.sum() >= 0.95 * len(mols)
    de = np.abs(r.energy - e)[ok]
    assert de.max() <= 1e-6
    multistable = 0
    for m in np.nonzero(ok)[0]:
        a0, a1 = off[m], off[m + 1]
        rg, rq = r.gradient[a0:a1], r.shell_charges[so[m]:so[m + 1]]
        if np.max(np.abs(rg - g[a0:a1])) <= 1e-5 and np.max(np.abs(rq - q[so[m]:so[m + 1]])) <= 1e-5:
            continue
        # Some molecules have two SCC fixed points a few 1e-7 Eh apart (molecule
        # 52: 4.5e-7 Eh, 2.9e-3 Eh/bohr), and which one the iteration reaches
        # changes when the coordinates move by 1e-12 bohr; the device result
        # must then equal one of the fixed points the oracle reaches.
        sols = _oracle_solutions(oracle_mod, mols[m][0], mols[m][1], ch[m])
        assert any(np.max(np.abs(rg - sg)) <= 1e-5 and np.max(np.abs(rq - sq)) <= 1e-5
                   and abs(r.energy[m] - se) <= 1e-6 for se, sg, sq in sols), m
        multistable += 1
    assert multistable <= 0.02 * len(mols)


def _oracle_solutions(oracle_mod, z, x, charge, trials=8):
    off = np.array([0, len(z)], np.int32)
    opts = oracle_mod.make_options(**TIGHT)
    rng = np.random.default_rng(0)
    out = []
    for t in range(trials + 1):
        xt = x if t == 0 else x + 1e-12 * rng.standard_normal(x.shape)
        e, g, q, _, _, st = oracle_mod.run_batch(off, z, xt, charges=np.array([charge]), options=opts, nthreads=1)
        if st[0] == 0:
            out.append((e[0], g, q))
    return out
