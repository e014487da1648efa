"""Numpy model of a two-stage Householder tridiagonalisation, CPU only: the
reduction the SCC kernel's per-column pass over the trailing matrix would be
replaced by (stage 1 touches the trailing matrix twice per panel instead of
once per column).

Stage 1, dense to band (bandwidth b): per panel of b columns starting at k,
the b columns below the band, A[k+b:, k:k+b], are factored by Householder QR
(reflectors V, compact-WY factor T with Q = I - V T V^T); the trailing matrix
takes the two-sided update as one symmetric rank-2b correction,
    X = A22 V T,  W = X - 1/2 V (T^T V^T X),  A22 -= V W^T + W V^T,
the two products the kernel would run on the FP64 tensor cores.

Stage 2, band to tridiagonal (bulge chasing): sweep j annihilates column j
below the subdiagonal with a reflector of length <= b on rows j+1..j+b,
applied from both sides; that fills a bulge below the band, whose first column
the next reflector (rows r+b.., length <= b) annihilates, and so on to the end
of the matrix.  The rest of each bulge lies in the rows the next sweep's
reflectors cover.

Back-transformation: with T = Q^T A Q and Q = Q1 Q2 (the panel reflectors,
then the bulge reflectors in the order applied), an eigenvector z of T gives
x = Q1 (Q2 z): the bulge reflectors in reverse order, then the panels'
compact-WY blocks in reverse order."""
import numpy as np
import pytest


def house(x: np.ndarray):
    """Reflector H = I - tau v v^T (v[0] = 1) with H x = (alpha, 0, ...)."""
    v = x.astype(np.float64).copy()
    sigma = v[1:] @ v[1:]
    if sigma == 0.0:
        v[:] = 0.0
        v[0] = 1.0
        return v, 0.0, x[0]
    xn = np.sqrt(x[0] * x[0] + sigma)
    alpha = -xn if x[0] >= 0.0 else xn
    v0 = x[0] - alpha
    v[1:] /= v0
    v[0] = 1.0
    tau = -v0 / alpha
    return v, tau, alpha


def dense_to_band(a: np.ndarray, b: int):
    """Stage 1.  Returns the band matrix and the panels (k, V, T)."""
    a = a.copy()
    n = len(a)
    panels = []
    for k in range(0, max(n - b - 1, 0), b):
        r0 = k + b  # first row below the band of column k
        nb = min(b, n - r0 - 1)  # reflectors of this panel (the last one may be short)
        m = n - r0
        V = np.zeros((m, nb))
        taus = np.zeros(nb)
        P = a[r0:, k:r0].copy()  # the panel's b columns below the band
        for c in range(nb):
            v, tau, alpha = house(P[c:, c])
            V[c:, c] = v
            taus[c] = tau
            P[c:, c:] -= tau * np.outer(v, v @ P[c:, c:])
        T = np.zeros((nb, nb))  # compact WY: H_0 ... H_{nb-1} = I - V T V^T
        for c in range(nb):
            T[c, c] = taus[c]
            if c:
                T[:c, c] = -taus[c] * (T[:c, :c] @ (V[:, :c].T @ V[:, c]))
        a[r0:, k:r0] = P
        a[k:r0, r0:] = P.T
        A22 = a[r0:, r0:]
        X = A22 @ V @ T
        W = X - 0.5 * V @ (T.T @ (V.T @ X))
        a[r0:, r0:] = A22 - V @ W.T - W @ V.T
        panels.append((r0, V, T))
    # entries below the band are zero up to rounding; store them as zeros
    idx = np.arange(n)
    a[np.abs(idx[:, None] - idx[None, :]) > b] = 0.0
    return a, panels


def band_to_tridiagonal(a: np.ndarray, b: int):
    """Stage 2.  Returns the tridiagonal (d, e) and the bulge reflectors in
    the order applied, (row, v, tau)."""
    a = a.copy()
    n = len(a)
    reflectors = []
    for j in range(n - 2):
        c, r = j, j + 1
        while r < n - 1:  # a reflector needs two rows
            ln = min(b, n - r)
            v, tau, _ = house(a[r:r + ln, c])
            if tau != 0.0:
                s = slice(r, r + ln)
                a[s, :] -= tau * np.outer(v, v @ a[s, :])
                a[:, s] -= tau * np.outer(a[:, s] @ v, v)
                reflectors.append((r, v, tau))
            c, r = r, r + b  # the bulge's first column; its entries below the band
    return np.diag(a).copy(), np.diag(a, -1).copy(), a, reflectors


def back_transform(z: np.ndarray, n: int, panels, reflectors) -> np.ndarray:
    """x = Q1 (Q2 z): bulge reflectors in reverse order, then the panels'
    compact-WY blocks (I - V T V^T) in reverse order."""
    x = z.copy()
    for r, v, tau in reversed(reflectors):
        s = slice(r, r + len(v))
        x[s] -= tau * np.outer(v, v @ x[s])
    for r0, V, T in reversed(panels):
        x[r0:] -= V @ (T @ (V.T @ x[r0:]))
    return x


def _random_symmetric(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n))
    return 0.5 * (a + a.T)


@pytest.mark.parametrize("n", [2, 3, 9, 17, 40, 96])
@pytest.mark.parametrize("b", [1, 2, 4, 8, 16])
def test_two_stage_reduction_spectrum_and_vectors(n, b):
    a = _random_symmetric(n, 1000 * n + b)
    band, panels = dense_to_band(a, b)
    idx = np.arange(n)
    assert np.allclose(band, band.T, atol=1e-12)
    d, e, t, reflectors = band_to_tridiagonal(band, b)
    scale = np.abs(a).max()
    off = np.abs(idx[:, None] - idx[None, :]) > 1
    assert np.abs(t[off]).max(initial=0.0) <= 1e-12 * scale  # tridiagonal to rounding
    tri = np.diag(d) + np.diag(e, -1) + np.diag(e, 1)
    lam, z = np.linalg.eigh(tri)
    assert np.allclose(lam, np.linalg.eigvalsh(a), rtol=0, atol=1e-11 * scale)
    x = back_transform(z, n, panels, reflectors)
    assert np.abs(x.T @ x - np.eye(n)).max() <= 1e-12  # orthonormal eigenvectors of A
    assert np.abs(a @ x - x * lam).max() <= 1e-11 * scale


def test_stage_one_reads_the_trailing_matrix_twice_per_panel():
    """Stage 1 forms A22 V T and updates A22 once per panel of b columns, where
    the one-stage reduction multiplies A22 by each column's reflector: for
    n = 180 and b = 8 that is 2 x 22 passes over shrinking trailing matrices
    instead of 178, about 2/b of the elements read (0.24 here); the per-column
    A22 v is where the SCC kernel spends most of its reduction."""
    n, b = 180, 8
    _, panels = dense_to_band(_random_symmetric(n, 7), b)
    one_stage = sum((n - k - 1) ** 2 for k in range(n - 2))
    two_stage = sum(2 * (n - r0) ** 2 for r0, _, _ in panels)
    assert len(panels) == 22
    assert 0.2 * one_stage < two_stage < 2.0 / b * one_stage


def test_already_banded_and_diagonal_inputs():
    for n, b in ((12, 3), (7, 8)):
        a = np.diag(np.arange(n, dtype=np.float64))
        band, panels = dense_to_band(a, b)
        d, e, _, reflectors = band_to_tridiagonal(band, b)
        assert reflectors == [] and np.allclose(d, np.arange(n)) and np.all(e == 0.0)
        assert all(np.all(T == 0.0) for _, _, T in panels)
