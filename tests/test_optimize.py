"""Batched L-BFGS driver (the reference's optimize_geometry algorithm per
molecule) on analytic test energies: no GPU needed."""
import numpy as np

from gfn1_rs.optimize import OptimizeOptions, lbfgs_direction, limit_atom_step, optimize


def _quadratic_evaluator(centres, hess):
    def evaluate(items):
        out = []
        for i, x, _ in items:
            d = x - centres[i]
            out.append((True, 0.5 * float(d @ hess[i] @ d), hess[i] @ d, None))
        return out
    return evaluate


def test_converges_on_quadratics_of_different_conditioning():
    rng = np.random.default_rng(0)
    centres, hess, x0 = [], [], []
    for k in range(6):
        n = 3 * (k + 2)
        q, _ = np.linalg.qr(rng.normal(size=(n, n)))
        hess.append(q @ np.diag(np.linspace(0.1, 1.0 + 3 * k, n)) @ q.T)
        centres.append(rng.normal(size=n))
        x0.append(centres[-1] + rng.normal(size=n) * 0.5)
    mols = optimize(_quadratic_evaluator(centres, hess), x0)
    for m, c in zip(mols, centres):
        assert m.converged and m.error is None
        assert np.abs(m.grad).max() <= 1e-4
        assert np.abs(m.x - c).max() < 1e-2
        energies = [t[1] for t in m.trajectory]
        assert all(b <= a + 1e-15 for a, b in zip(energies, energies[1:]))  # Armijo: never uphill


def test_steps_are_capped_per_atom():
    d = np.array([0.0, 0.0, 3.0, 0.1, 0.0, 0.0])
    out = limit_atom_step(d, 0.30)
    assert np.isclose(np.sqrt((out.reshape(-1, 3) ** 2).sum(1)).max(), 0.30)
    assert np.allclose(limit_atom_step(d * 0.01, 0.30), d * 0.01)


def test_two_loop_recursion_matches_dense_bfgs_inverse():
    # with one history pair the two-loop result equals -H g for the BFGS inverse update of gamma I
    rng = np.random.default_rng(1)
    g, s, y = rng.normal(size=6), rng.normal(size=6), rng.normal(size=6)
    y = y + 2 * s  # y.s > 0
    rho = 1.0 / (y @ s)
    gamma = (y @ s) / (y @ y)
    V = np.eye(6) - rho * np.outer(y, s)
    H = V.T @ (gamma * np.eye(6)) @ V + rho * np.outer(s, s)
    assert np.allclose(lbfgs_direction(g, [s], [y], [rho]), -H @ g)


def test_failed_line_search_is_reported():
    # the energy is 0 at the start point and 1 at every trial point: no downhill step exists
    calls = {"n": 0}

    def ev(items):
        calls["n"] += 1
        return [(True, 0.0 if calls["n"] == 1 else 1.0, np.ones_like(x), None) for _, x, _ in items]
    mols = optimize(ev, [np.zeros(3)], OptimizeOptions(max_iterations=5))
    assert not mols[0].converged and "line search" in mols[0].error
