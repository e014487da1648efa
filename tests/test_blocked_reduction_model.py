"""Numpy model of the SCC kernel's blocked Householder tridiagonalisation
(gfn1-rs_b200/csrc/scc.cu, tridiagonalize_blocked), CPU only.

Per panel of `panel` columns: each column k first takes the panel's earlier
rank-2 updates lazily (x = A[k, k:] - sum_l V_l[k] W_l[k:] + W_l[k] V_l[k:]),
builds its reflector v (v0 = x1 - alpha, alpha = -sign(x1) |x[1:]|,
beta = 2 / v.v), forms p = beta (A22 v - V (W^T v) - W (V^T v)) with A22 as of
the panel start, and keeps w = p - (beta p.v / 2) v; at the end of the panel
the trailing matrix takes A22 -= V W^T + W V^T in one pass (the kernel's FP64
tensor-core tiles).  Any panel width gives the same reflectors as the unblocked
reduction (panel = 1), so the tridiagonal (d, e) agrees to rounding and its
eigenvalues are those of A."""
import numpy as np
import pytest


def blocked_tridiagonal(a: np.ndarray, panel: int):
    a = a.copy()
    n = len(a)
    d, e = np.zeros(n), np.zeros(n)
    for k0 in range(0, max(n - 2, 0), panel):
        nbp = min(panel, n - 2 - k0)
        V, W = np.zeros((nbp, n)), np.zeros((nbp, n))
        for j in range(nbp):
            k = k0 + j
            x = a[k, k:].copy()
            for l in range(j):
                x -= V[l, k] * W[l, k:] + W[l, k] * V[l, k:]
            d[k] = x[0]
            xn2 = x[1:] @ x[1:]
            if xn2 - x[1] * x[1] == 0.0:  # already reduced: no reflector
                e[k] = x[1]
                a[k, k + 1:] = x[1:]
                continue
            xn = np.sqrt(xn2)
            alpha = -xn if x[1] >= 0.0 else xn
            v = x[1:].copy()
            v[0] = x[1] - alpha
            beta = 2.0 / (v @ v)
            a[k, k + 1:] = v  # the reflector is stored in row k
            V[j, k + 1:] = v
            a22 = a[k + 1:, k + 1:]
            p = a22 @ v - V[:j, k + 1:].T @ (W[:j, k + 1:] @ v) - W[:j, k + 1:].T @ (V[:j, k + 1:] @ v)
            p *= beta
            W[j, k + 1:] = p - 0.5 * beta * (p @ v) * v
            e[k] = alpha
        s0 = k0 + nbp
        a[s0:, s0:] -= V[:, s0:].T @ W[:, s0:] + W[:, s0:].T @ V[:, s0:]
    if n >= 2:
        d[n - 2], e[n - 2] = a[n - 2, n - 2], a[n - 1, n - 2]
    d[n - 1] = a[n - 1, n - 1]
    return d, e


def _tridiagonal_eigenvalues(d, e):
    t = np.diag(d) + np.diag(e[:-1], 1) + np.diag(e[:-1], -1)
    return np.linalg.eigvalsh(t)


@pytest.mark.parametrize("n", [3, 9, 40, 97])
def test_panels_agree_with_unblocked_and_spectrum(n):
    rng = np.random.default_rng(n)
    b = rng.normal(size=(n, n))
    a = 0.5 * (b + b.T)
    d1, e1 = blocked_tridiagonal(a, 1)
    lam = np.linalg.eigvalsh(a)
    assert np.max(np.abs(_tridiagonal_eigenvalues(d1, e1) - lam)) <= 1e-12 * np.max(np.abs(lam))
    for panel in (4, 8, 16, 32):
        d, e = blocked_tridiagonal(a, panel)
        assert np.max(np.abs(d - d1)) <= 1e-12 * np.max(np.abs(lam)), panel
        assert np.max(np.abs(e - e1)) <= 1e-12 * np.max(np.abs(lam)), panel


def test_already_reduced_columns():
    """A matrix that is tridiagonal from the start takes the no-reflector branch
    in every column and comes back unchanged."""
    n = 12
    rng = np.random.default_rng(1)
    d0, e0 = rng.normal(size=n), rng.normal(size=n - 1)
    a = np.diag(d0) + np.diag(e0, 1) + np.diag(e0, -1)
    for panel in (1, 8):
        d, e = blocked_tridiagonal(a, panel)
        assert np.allclose(d, d0, rtol=0, atol=1e-15)
        assert np.allclose(np.abs(e[:-1]), np.abs(e0), rtol=0, atol=1e-15)
