"""Numpy model of the large-molecule path (gfn1-rs_b200/csrc/wide.cuh), CPU
only: the same arithmetic in the same order of steps, so that its algebra is
checked before and independently of the GPU.

* Householder reduction (wide_tridiag_kernel): panels of `nb` columns; the
  trailing rows of a panel split among `ga` groups (CTAs), each forming its
  rows of x = A[:, j] - V W[j]^T - W V[j]^T, partial sums |x|^2, V^T x and
  W^T x; dlarfg reflectors (v_{j+1} = 1, tau, beta); p = tau (A v - V (W^T v)
  - W (V^T v)) with A as of the panel start; W keeps p and the scalars
  alpha = -tau (p.v) / 2 until the panel ends; then A22 -= V W^T + W V^T.
  Reflector j is stored in column j below the subdiagonal.
* Back-transformation (wide_bt_*): blocks of 64 reflectors, T by the forward
  columnwise recurrence, applied last block first: Z -= V (T (V^T Z)).
* Orthogonaliser (wide_chol_*, wide_inv_row_kernel): blocked Cholesky with
  the inverse of each diagonal block, L^-1 block row by block row.

The reduction must give the eigenvalues of A for any panel width and group
count, Q^T A Q must be the tridiagonal, and the orthogonaliser must give
L L^T = S and L^-1 L = I."""
import numpy as np
import pytest


def wide_tridiagonal(a, nb, ga_max, min_rows):
    """Returns d, e, tau and the matrix holding the reflectors (columns)."""
    A = a.copy()
    n = len(A)
    d, e, tau = np.zeros(n), np.zeros(n), np.zeros(n)
    for k0 in range(0, n - 2, nb):
        nbc = min(nb, n - 2 - k0)
        nr = n - k0 - 1
        ga = max(1, min(ga_max, nr // min_rows))
        bounds = [k0 + 1 + (nr * c) // ga for c in range(ga + 1)]
        V, Wr = np.zeros((nb, n)), np.zeros((nb, n))
        alpha2 = np.zeros(nb)
        for l in range(nbc):
            j = k0 + l
            Wc = Wr + alpha2[:, None] * V  # W as used: p + alpha v
            vj, wj = V[:l, j], Wc[:l, j]
            x = np.zeros(n)
            parts = []
            for c in range(ga):
                r0, r1 = bounds[c], bounds[c + 1]
                rows = np.arange(max(r0, j + 1), r1)
                x[rows] = A[rows, j] - V[:l, rows].T @ wj - Wc[:l, rows].T @ vj
                tail = np.arange(max(r0, j + 2), r1)
                parts.append(np.concatenate([[x[tail] @ x[tail]], V[:l, tail] @ x[tail], Wc[:l, tail] @ x[tail]]))
            tot = np.sum(parts, axis=0)
            x0, s = x[j + 1], tot[0]
            beta, t, scale = x0, 0.0, 0.0
            if s > 0.0:
                nrm = np.sqrt(x0 * x0 + s)
                beta = -nrm if x0 >= 0.0 else nrm
                t = (beta - x0) / beta
                scale = 1.0 / (x0 - beta)
            d[j] = A[j, j] - 2.0 * vj @ wj
            e[j], tau[j] = beta, t
            vtv = V[:l, j + 1] + scale * tot[1:1 + l]
            wtv = Wc[:l, j + 1] + scale * tot[1 + l:1 + 2 * l]
            v = np.zeros(n)
            v[j + 1] = 1.0
            v[j + 2:] = scale * x[j + 2:]
            pv = 0.0
            for c in range(ga):
                rows = np.arange(max(bounds[c], j + 1), bounds[c + 1])
                q = A[rows][:, j + 1:] @ v[j + 1:]
                p = t * (q - V[:l, rows].T @ wtv - Wc[:l, rows].T @ vtv)
                V[l, rows], Wr[l, rows] = v[rows], p
                below = rows[rows >= j + 2]
                A[below, j] = v[below]
                pv += p @ v[rows]
            alpha2[l] = -0.5 * t * pv
        Wf = Wr + alpha2[:, None] * V
        k1 = k0 + nbc
        A[k1:, k1:] -= V[:nbc, k1:].T @ Wf[:nbc, k1:] + Wf[:nbc, k1:].T @ V[:nbc, k1:]
    d[n - 2], e[n - 2], d[n - 1] = A[n - 2, n - 2], A[n - 1, n - 2], A[n - 1, n - 1]
    return d, e, tau, A


def reflector_block(A, tau, kb, n):
    nref = n - 2
    nbk = min(64, nref - kb)
    V = np.zeros((n, nbk))
    for a in range(nbk):
        r = kb + a + 1
        V[r, a] = 1.0
        V[r + 1:, a] = A[r + 1:, kb + a]
    G = V.T @ V
    T = np.zeros((nbk, nbk))
    for j in range(nbk):
        T[:j, j] = -tau[kb + j] * (T[:j, :j] @ G[:j, j])
        T[j, j] = tau[kb + j]
    return V, T


def back_transform(A, tau, Z):
    n = len(A)
    Z = Z.copy()
    nblk = (n - 2 + 63) // 64
    for b in range(nblk - 1, -1, -1):
        V, T = reflector_block(A, tau, 64 * b, n)
        Z -= V @ (T @ (V.T @ Z))
    return Z


def tridiag_matrix(d, e):
    return np.diag(d) + np.diag(e[:-1], 1) + np.diag(e[:-1], -1)


@pytest.mark.parametrize("n,nb,ga,mr", [(5, 8, 1, 4), (70, 8, 4, 4), (97, 16, 3, 8), (130, 32, 8, 4),
                                        (200, 16, 16, 16), (131, 8, 148, 4)])
def test_reduction_gives_the_spectrum_and_a_similarity(n, nb, ga, mr):
    rng = np.random.default_rng(n + nb)
    m = rng.standard_normal((n, n))
    a = m + m.T
    d, e, tau, A = wide_tridiagonal(a, nb, ga, mr)
    T = tridiag_matrix(d, e)
    assert np.allclose(np.linalg.eigvalsh(T), np.linalg.eigvalsh(a), atol=1e-10 * np.abs(a).max() * n)
    Q = back_transform(A, tau, np.eye(n))
    assert np.allclose(Q.T @ Q, np.eye(n), atol=1e-12 * n)
    assert np.allclose(Q.T @ a @ Q, T, atol=1e-11 * n * np.abs(a).max())


def test_eigenvectors_back_transform():
    n = 150
    rng = np.random.default_rng(3)
    m = rng.standard_normal((n, n))
    a = m + m.T
    d, e, tau, A = wide_tridiagonal(a, 16, 5, 8)
    w, y = np.linalg.eigh(tridiag_matrix(d, e))
    z = back_transform(A, tau, y[:, :60])
    assert np.allclose(a @ z, z * w[:60], atol=1e-9)


def blocked_cholesky_inverse(s):
    n = len(s)
    L = np.tril(s)
    Li = np.zeros_like(s)
    nblk = (n + 63) // 64
    for k in range(nblk):
        kb, nb = 64 * k, min(64, n - 64 * k)
        blk = np.linalg.cholesky(np.tril(L[kb:kb + nb, kb:kb + nb]) + np.tril(L[kb:kb + nb, kb:kb + nb], -1).T)
        inv = np.linalg.inv(blk)
        L[kb:kb + nb, kb:kb + nb] = blk
        Li[kb:kb + nb, kb:kb + nb] = inv
        if kb + 64 < n:
            L[kb + 64:, kb:kb + nb] = L[kb + 64:, kb:kb + nb] @ inv.T
            P = L[kb + 64:, kb:kb + nb]
            L[kb + 64:, kb + 64:] -= np.tril(P @ P.T)
    for i in range(1, nblk):
        ib = 64 * i
        for j in range(i):
            j0 = 64 * j
            t = L[ib:ib + 64, j0:ib] @ Li[j0:ib, j0:j0 + 64]
            Li[ib:ib + 64, j0:j0 + 64] = -Li[ib:ib + 64, ib:ib + 64] @ t
    return np.tril(L), Li


@pytest.mark.parametrize("n", [5, 64, 65, 200])
def test_blocked_cholesky_and_inverse(n):
    rng = np.random.default_rng(n)
    m = rng.standard_normal((n, n))
    s = m @ m.T + n * np.eye(n)
    L, Li = blocked_cholesky_inverse(s)
    assert np.allclose(L @ L.T, s, atol=1e-10 * n)
    assert np.allclose(Li @ L, np.eye(n), atol=1e-12 * n)
