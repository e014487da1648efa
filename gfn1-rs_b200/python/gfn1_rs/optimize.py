"""Batched geometry optimisation with L-BFGS on the engine.

Each molecule follows gfn1-rs ``optimize_geometry`` (``src/optimizer.rs:78-320``)
step for step: the two-loop L-BFGS direction with history 12 and
gamma = y.s / y.y scaling, steepest descent when that direction is not
downhill, the per-atom step cap (0.30 bohr), a backtracking line search
(initial step 1, Armijo c1 = 1e-4, halving, at most 24 trials), the history
update when y.s > 1e-12, and convergence on the largest gradient component
(<= 1e-4 Eh/bohr) or the step norm (<= 1e-7 bohr), at most 250 iterations.

What is batched: every round collects the pending trial geometry of every
molecule that is still optimising and evaluates them in one engine call, so
thousands of molecules advance together.  With ``warm_start`` (default) each
trial's SCC starts from the converged shell charges of the molecule's current
geometry; the reference starts every evaluation from zero charges, which
gives the same energies to the SCC tolerance.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class OptimizeOptions:
    max_iterations: int = 250
    gradient_tolerance: float = 1.0e-4
    step_tolerance: float = 1.0e-7
    history: int = 12
    initial_step: float = 1.0
    max_atom_step: float = 0.30


@dataclass
class _Mol:
    x: np.ndarray
    energy: float = 0.0
    grad: np.ndarray | None = None
    q: np.ndarray | None = None
    s_hist: list = field(default_factory=list)
    y_hist: list = field(default_factory=list)
    rho_hist: list = field(default_factory=list)
    iterations: int = 0
    converged: bool = False
    done: bool = False
    error: str | None = None
    direction: np.ndarray | None = None
    alpha: float = 0.0
    tries: int = 0
    dd: float = 0.0
    trajectory: list = field(default_factory=list)
    frames: list = field(default_factory=list)  # accepted geometries, frame 0 the input


def lbfgs_direction(g, s_hist, y_hist, rho_hist):
    """Two-loop recursion (src/optimizer.rs:259-290)."""
    if not s_hist:
        return -g
    q = g.copy()
    alpha = [0.0] * len(s_hist)
    for i in range(len(s_hist) - 1, -1, -1):
        alpha[i] = rho_hist[i] * float(s_hist[i] @ q)
        q -= alpha[i] * y_hist[i]
    yy = float(y_hist[-1] @ y_hist[-1])
    ys = float(y_hist[-1] @ s_hist[-1])
    q *= ys / yy if yy > 1.0e-18 else 1.0
    for i in range(len(s_hist)):
        beta = rho_hist[i] * float(y_hist[i] @ q)
        q += (alpha[i] - beta) * s_hist[i]
    return -q


def limit_atom_step(direction, max_atom_step):
    """Scale so that no atom moves more than max_atom_step (src/optimizer.rs:292-305)."""
    if max_atom_step <= 0.0:
        return direction
    m = float(np.sqrt((direction.reshape(-1, 3) ** 2).sum(1)).max()) if direction.size else 0.0
    return direction * (max_atom_step / m) if m > max_atom_step else direction


def optimize(evaluate, x0_list, options: OptimizeOptions | None = None):
    """Generic batched driver.  evaluate(items) takes a list of
    (molecule index, flat coordinates, initial shell charges or None) and
    returns a list of (ok, energy, flat gradient, shell charges) in the same
    order.  Returns the per-molecule states."""
    opt = options or OptimizeOptions()
    mols = [_Mol(x=np.asarray(x, dtype=np.float64).ravel().copy()) for x in x0_list]
    res = evaluate([(i, m.x, None) for i, m in enumerate(mols)])
    for m, (ok, e, g, q) in zip(mols, res):
        if not ok:
            m.done, m.error = True, "initial evaluation failed"
            continue
        m.energy, m.grad, m.q = e, np.asarray(g, dtype=np.float64).ravel(), q
        m.converged = float(np.abs(m.grad).max()) <= opt.gradient_tolerance
        m.trajectory.append((0, m.energy, float(np.abs(m.grad).max()), 0.0))
        m.frames.append(m.x.copy())
    hist_len = max(opt.history, 1)
    while True:
        for m in mols:  # start a new step where no line search is pending
            if m.done or m.direction is not None:
                continue
            if m.converged or m.iterations >= opt.max_iterations:
                m.done = True
                continue
            m.iterations += 1
            d = lbfgs_direction(m.grad, m.s_hist, m.y_hist, m.rho_hist)
            if float(d @ m.grad) >= 0.0 or not np.all(np.isfinite(d)):
                d = -m.grad
            d = limit_atom_step(d, opt.max_atom_step)
            m.direction, m.dd = d, float(m.grad @ d)
            m.alpha, m.tries = max(opt.initial_step, 1.0e-8), 0
        active = [i for i, m in enumerate(mols) if not m.done and m.direction is not None]
        if not active:
            break
        trials = [(i, mols[i].x + mols[i].alpha * mols[i].direction, mols[i].q) for i in active]
        res = evaluate(trials)
        for (i, xt, _), (ok, e, g, q) in zip(trials, res):
            m = mols[i]
            if ok and e <= m.energy + 1.0e-4 * m.alpha * m.dd:  # Armijo (src/optimizer.rs:238-244)
                g = np.asarray(g, dtype=np.float64).ravel()
                s, y = xt - m.x, g - m.grad
                ys = float(y @ s)
                if ys > 1.0e-12 and np.all(np.isfinite(s)) and np.all(np.isfinite(y)):
                    if len(m.s_hist) == hist_len:
                        m.s_hist.pop(0), m.y_hist.pop(0), m.rho_hist.pop(0)
                    m.s_hist.append(s), m.y_hist.append(y), m.rho_hist.append(1.0 / ys)
                step_norm = float(np.linalg.norm(s))
                m.x, m.energy, m.grad, m.q = xt, e, g, q
                maxg = float(np.abs(g).max())
                m.trajectory.append((m.iterations, e, maxg, step_norm))
                m.frames.append(xt.copy())
                m.converged = maxg <= opt.gradient_tolerance or step_norm <= opt.step_tolerance
                m.direction = None
            else:
                m.alpha *= 0.5
                m.tries += 1
                if m.tries >= 24:
                    m.done, m.direction = True, None
                    m.error = "L-BFGS line search failed to find a downhill step"
    return mols


def optimize_batch(calc, atom_offsets, numbers, xyz_bohr, charges=None, options: OptimizeOptions | None = None,
                   warm_start: bool = True) -> dict:
    """Optimises every molecule of a flat batch with one engine call per round.
    Returns final coordinates (bohr), energies, max gradients, iterations,
    converged flags, error messages and the number of engine calls."""
    off = np.asarray(atom_offsets, dtype=np.int64)
    z = np.asarray(numbers)
    x = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    nmol = len(off) - 1
    shoff = calc.shell_offsets(off, z)
    ch = np.zeros(nmol) if charges is None else np.asarray(charges, dtype=np.float64)
    calls = [0]

    def evaluate(items):
        idx = [i for i, _, _ in items]
        sub_off = np.concatenate([[0], np.cumsum([off[i + 1] - off[i] for i in idx])]).astype(np.int32)
        sub_z = np.concatenate([z[off[i]:off[i + 1]] for i in idx])
        sub_x = np.concatenate([np.asarray(xi).reshape(-1, 3) for _, xi, _ in items])
        q0 = None
        if warm_start and all(q is not None for _, _, q in items):
            q0 = np.concatenate([q for _, _, q in items])
        r = calc.calculate_flat(sub_off, sub_z, sub_x, charges=ch[idx], initial_shell_charges=q0)
        calls[0] += 1
        out = []
        for k in range(len(idx)):
            a0, a1 = r.atom_offsets[k], r.atom_offsets[k + 1]
            s0, s1 = r.shell_offsets[k], r.shell_offsets[k + 1]
            ok = r.status[k] == 0
            out.append((ok, float(r.energy[k]), r.gradient[a0:a1].ravel().copy(), r.shell_charges[s0:s1].copy()))
        return out

    mols = optimize(evaluate, [x[off[i]:off[i + 1]] for i in range(nmol)], options)
    return {"xyz": np.concatenate([m.x.reshape(-1, 3) for m in mols]) if nmol else x,
            "energy": np.array([m.energy for m in mols]),
            "max_gradient": np.array([float(np.abs(m.grad).max()) if m.grad is not None else np.inf for m in mols]),
            "iterations": np.array([m.iterations for m in mols]),
            "converged": np.array([m.converged for m in mols]),
            "errors": [m.error for m in mols], "engine_calls": calls[0],
            "trajectories": [m.trajectory for m in mols], "frames": [m.frames for m in mols],
            "gradient": [m.grad for m in mols], "shell_offsets": shoff}


def optimize_batch_device(calc, atom_offsets, numbers, xyz_bohr, charges=None,
                          options: OptimizeOptions | None = None) -> dict:
    """The same optimisation with the L-BFGS state on the device
    (gfn1_batch_optimize): the batch's topology and the optimiser's history,
    geometries, gradients and charges stay in device memory, one engine pass
    and one kernel per round, and the host reads only the number of molecules
    still optimising.  Every trial's SCC starts from the converged charges of
    the molecule's current geometry, as optimize_batch(warm_start=True)."""
    opt = options or OptimizeOptions()
    rb = calc.resident(atom_offsets, numbers, charges=charges)
    try:
        rb.set_positions(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3))
        return rb.optimize(max_iterations=opt.max_iterations, gradient_tolerance=opt.gradient_tolerance,
                           step_tolerance=opt.step_tolerance, history=opt.history, initial_step=opt.initial_step,
                           max_atom_step=opt.max_atom_step)
    finally:
        rb.close()

