"""Batched nuclear Hessians and harmonic vibrational analysis on the engine.

The reference assembles the non-periodic Hessian analytically
(``analytic_hessian``, ``src/hessian/mod.rs:112-296``: fixed-density blocks
plus the CPXTB charge response).  Here each column is the central difference
of the engine's analytic gradient,

    H[:, 3a+k] = (g(R + h e_ak) - g(R - h e_ak)) / 2h,    h = 5e-3 bohr,

symmetrised as (H + H^T) / 2.  The 6N displaced geometries of every molecule
go to the engine together, as one batch per chunk, and each displaced SCC
starts from the converged shell charges at R.  The SCC runs with tight
tolerances (1e-10 Eh, 1e-8 e) so that the gradient noise divided by 2h stays
near 1e-7 Eh/bohr^2; the truncation error is h^2/6 times the third
derivative, about 1e-5 relative.  With order=4 the columns come from the
five-point stencil

    H[:, c] = (8 (g(+h) - g(-h)) - (g(+2h) - g(-2h))) / 12h,

12N displaced gradients per molecule and a truncation error of h^4/30 times
the fifth derivative (below 1e-8 relative at h = 1e-2 bohr, its default
step, where the noise term is about 1e-8 Eh/bohr^2 as well).

``vibrational_analysis`` follows ``src/vibrational.rs:37-84``: mass-weighted,
symmetrised Hessian, ascending eigenvalues lambda, wavenumbers
sign(lambda) sqrt(|lambda|) 5140.4843 cm^-1 and Cartesian modes (mass-weighted
eigenvectors divided by sqrt(m)), with the relative atomic masses of
``src/data_tables.rs``.
"""
from __future__ import annotations

import numpy as np

WAVENUMBER_PER_SQRT_AU = 5140.4843  # cm^-1 per sqrt(Eh / (bohr^2 amu)), src/vibrational.rs:20
DEFAULT_STEP = 5.0e-3  # bohr, central differences
DEFAULT_STEP4 = 1.0e-2  # bohr, the five-point stencil
TIGHT = dict(energy_tolerance=1.0e-10, charge_tolerance=1.0e-8)

_MASSES = None


def atomic_masses() -> np.ndarray:
    """Relative atomic masses (amu) indexed by Z = 0..86, from the engine's tables."""
    global _MASSES
    if _MASSES is None:
        from ._lib import TABLES_PATH

        with open(TABLES_PATH) as fh:
            for line in fh:
                if line.startswith("atomic_mass_amu "):
                    _MASSES = np.array([float(v) for v in line.split()[2:]])
                    break
        if _MASSES is None:
            raise RuntimeError("the tables file has no atomic_mass_amu entry")
    return _MASSES


def _factors(order: int):
    if order == 2:
        return (1.0, -1.0)
    if order == 4:
        return (1.0, -1.0, 2.0, -2.0)
    raise ValueError("order must be 2 or 4")


def displacements(nat: int, step: float, order: int = 2) -> np.ndarray:
    """The displacement vectors [6N, nat, 3] (order 2: +h, -h for each
    coordinate 3a+k in atom-major order) or [12N, nat, 3] (order 4: +h, -h,
    +2h, -2h)."""
    f = _factors(order)
    d = np.zeros((len(f) * 3 * nat, nat, 3))
    for c in range(3 * nat):
        for s, fs in enumerate(f):
            d[len(f) * c + s, c // 3, c % 3] = fs * step
    return d


def assemble(grads_plus_minus: np.ndarray, step: float, order: int = 2) -> np.ndarray:
    """Hessian [3N, 3N] from the displaced gradients in the order of
    ``displacements``, symmetrised."""
    nf = len(_factors(order))
    n3 = grads_plus_minus.shape[0] // nf
    g = grads_plus_minus.reshape(n3, nf, -1)
    if order == 2:
        cols = (g[:, 0] - g[:, 1]) / (2.0 * step)  # row c holds column c
    else:
        cols = (8.0 * (g[:, 0] - g[:, 1]) - (g[:, 2] - g[:, 3])) / (12.0 * step)
    h = cols.T
    return 0.5 * (h + h.T)


def hessian(evaluate, molecules, step: float | None = None, chunk: int = 16384, order: int = 2):
    """Generic batched driver.  ``molecules`` is a list of (numbers, xyz_bohr
    [nat, 3], initial shell charges or None); ``evaluate(items)`` takes a list
    of (molecule index, numbers, xyz [nat, 3], initial shell charges or None)
    and returns a list of (ok, gradient [nat, 3]).  Returns the Hessians (None
    where a displaced evaluation failed) and the number of evaluate calls.
    ``order`` 2 (central differences) or 4 (five-point stencil); ``step``
    defaults to DEFAULT_STEP or DEFAULT_STEP4."""
    if step is None:
        step = DEFAULT_STEP if order == 2 else DEFAULT_STEP4
    pending = []
    for i, (z, x, q) in enumerate(molecules):
        x = np.asarray(x, dtype=np.float64).reshape(-1, 3)
        for d in displacements(len(x), step, order):
            pending.append((i, z, x + d, q))
    grads = [[] for _ in molecules]
    ok = [True] * len(molecules)
    calls = 0
    for c0 in range(0, len(pending), chunk):
        items = pending[c0:c0 + chunk]
        res = evaluate(items)
        calls += 1
        for (i, _, _, _), (good, g) in zip(items, res):
            ok[i] = ok[i] and bool(good)
            grads[i].append(np.asarray(g, dtype=np.float64).reshape(-1, 3))
    out = [assemble(np.stack(g), step, order) if good and g else None for g, good in zip(grads, ok)]
    return out, calls


def hessian_batch(calc, atom_offsets, numbers, xyz_bohr, charges=None, step: float | None = None,
                  warm_start: bool = True, chunk: int = 16384, order: int = 2) -> dict:
    """Hessians (Eh/bohr^2, [3N, 3N] per molecule, atom-major) of every
    molecule of a flat batch.  One engine call at the reference geometries,
    then the displaced geometries in chunks of ``chunk`` molecules per call.
    Returns hessians, energies and gradients at R, per-molecule status (0 when
    every evaluation converged) and the number of engine calls.  ``order`` 4
    takes the five-point stencil (twice the displaced evaluations)."""
    if step is None:
        step = DEFAULT_STEP if order == 2 else DEFAULT_STEP4
    off = np.asarray(atom_offsets, dtype=np.int64)
    z = np.asarray(numbers)
    x = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    nmol = len(off) - 1
    ch = np.zeros(nmol) if charges is None else np.asarray(charges, dtype=np.float64)
    saved = dict(calc.opts)
    calc.opts.update(TIGHT)
    try:
        r0 = calc.calculate_flat(off.astype(np.int32), z, x, charges=ch)
        mols = []
        for m in range(nmol):
            s0, s1 = r0.shell_offsets[m], r0.shell_offsets[m + 1]
            q = None
            if warm_start:  # a molecule that failed at R starts from zero charges, the others stay warm
                q = r0.shell_charges[s0:s1].copy() if r0.status[m] == 0 else np.zeros(s1 - s0)
            mols.append((m, z[off[m]:off[m + 1]], x[off[m]:off[m + 1]], q))

        def evaluate(items):
            sub_off = np.concatenate([[0], np.cumsum([len(zi) for _, zi, _, _ in items])]).astype(np.int32)
            sub_z = np.concatenate([zi for _, zi, _, _ in items])
            sub_x = np.concatenate([xi for _, _, xi, _ in items])
            q0 = None
            if all(q is not None for _, _, _, q in items):
                q0 = np.concatenate([q for _, _, _, q in items])
            r = calc.calculate_flat(sub_off, sub_z, sub_x, charges=ch[[mols[i][0] for i, _, _, _ in items]],
                                    initial_shell_charges=q0)
            return [(r.status[k] == 0, r.gradient[r.atom_offsets[k]:r.atom_offsets[k + 1]])
                    for k in range(len(items))]

        hs, calls = hessian(evaluate, [(zi, xi, q) for _, zi, xi, q in mols], step, chunk, order)
    finally:
        calc.opts.clear()
        calc.opts.update(saved)
    status = np.array([int(r0.status[m]) if r0.status[m] != 0 else (0 if hs[m] is not None else 8)
                       for m in range(nmol)])
    return {"hessians": hs, "energy": r0.energy.copy(), "gradient": r0.gradient.copy(), "status": status,
            "engine_calls": calls + 1, "step": step, "order": order}


def vibrational_analysis(hess, numbers) -> dict:
    """Harmonic analysis of one Cartesian Hessian (Eh/bohr^2, atom-major):
    wavenumbers (cm^-1, ascending, imaginary as negative), mass-weighted
    eigenvalues (Eh/(bohr^2 amu)) and Cartesian modes [3N, 3N] (one per row)."""
    z = np.asarray(numbers, dtype=np.int64)
    h = np.asarray(hess, dtype=np.float64)
    mass = np.maximum(np.repeat(atomic_masses()[z], 3), 1.0e-12)
    mw = h / np.sqrt(np.outer(mass, mass))
    mw = 0.5 * (mw + mw.T)
    lam, vec = np.linalg.eigh(mw)
    w = np.sqrt(np.abs(lam)) * WAVENUMBER_PER_SQRT_AU
    return {"wavenumbers": np.where(lam < 0.0, -w, w), "eigenvalues": lam,
            "modes": (vec / np.sqrt(mass)[:, None]).T}


__all__ = ["hessian", "hessian_batch", "vibrational_analysis", "assemble", "displacements", "atomic_masses",
           "WAVENUMBER_PER_SQRT_AU", "DEFAULT_STEP", "DEFAULT_STEP4"]
