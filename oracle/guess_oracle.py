"""CPU float64 restatement of the learned SCC initial guess (test infrastructure only).

The reference has no learned guess: its SCC always starts from zero shell
charges or a caller-supplied vector (gfn1-rs ``src/electronic.rs:1231-1239``,
``init_shell_q``).  This module defines, in plain numpy, the atom-centred
descriptors, the MLP and its loss, and derives the weight gradients by hand, so
the device kernels (descriptors, forward, backward, projection) have an
independent checker.  Only ``tests/`` use it.

Descriptors, per atom i of H/C/N/O (distances in bohr, cutoff rc = 6):
  fc(r) = (cos(pi r / rc) + 1) / 2
  radial  G[16 c + k] = sum_{j in channel c} exp(-4 (r_ij - mu_k)^2) fc(r_ij),
          mu_k = 0.5 + 5.5 k / 15, k = 0..15, channels c = H, C, N, O
  angular with g_b(r) = exp(-(r - nu_b)^2), nu = (1, 2, 3, 4.5):
          V[c,b] = sum_j g_b fc u_ij,   T[c,b] = sum_j g_b fc (u_ij u_ij^T - I/3)
          A[4 c + b] = |V[c,b]|^2,      A[16 + 4 c + b] = ||T[c,b]||_F^2
Network input: ((G, A) - mean) / std (96) followed by the element one-hot (4);
three SiLU layers of 128, a linear layer to the two shell charges of the atom;
the molecule's shell charges are shifted by a common constant so that they sum
to its total charge.  Loss: mean over shells of (q - q_label)^2.
"""
from __future__ import annotations

import numpy as np

RC = 6.0
N_RAD, N_ANG, N_DESC = 64, 32, 96
N_IN, N_HID, N_OUT = 100, 128, 2
ELEMENTS = (1, 6, 7, 8)
MU_R = 0.5 + 5.5 * np.arange(16) / 15.0
ETA_R = 4.0
NU_A = np.array([1.0, 2.0, 3.0, 4.5])
ETA_A = 1.0


def channel(z):
    z = np.asarray(z)
    out = np.full(z.shape, -1, dtype=np.int64)
    for c, e in enumerate(ELEMENTS):
        out[z == e] = c
    return out


def descriptors(atom_offsets, numbers, xyz_bohr):
    """[natoms, 96] float64 descriptors (rows of unsupported atoms are zero)."""
    off = np.asarray(atom_offsets)
    ch = channel(numbers)
    x = np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((len(ch), N_DESC))
    for m in range(len(off) - 1):
        a0, a1 = off[m], off[m + 1]
        for i in range(a0, a1):
            if ch[i] < 0:
                continue
            V = np.zeros((4, 4, 3))
            T = np.zeros((4, 4, 3, 3))
            for j in range(a0, a1):
                if j == i or ch[j] < 0:
                    continue
                d = x[j] - x[i]
                r = np.sqrt(d @ d)
                if r >= RC or r == 0.0:
                    continue
                c = ch[j]
                fc = 0.5 * (np.cos(np.pi * r / RC) + 1.0)
                out[i, 16 * c:16 * c + 16] += np.exp(-ETA_R * (r - MU_R) ** 2) * fc
                u = d / r
                g = np.exp(-ETA_A * (r - NU_A) ** 2) * fc
                V[c] += g[:, None] * u[None, :]
                T[c] += g[:, None, None] * (np.outer(u, u) - np.eye(3) / 3.0)[None]
            out[i, N_RAD:N_RAD + 16] = (V ** 2).sum(-1).reshape(16)
            out[i, N_RAD + 16:N_RAD + 32] = (T ** 2).sum((-1, -2)).reshape(16)
    return out


def features(desc, numbers, mean, std):
    """[natoms, 100] network input."""
    ch = channel(numbers)
    x = np.zeros((len(ch), N_IN))
    x[:, :N_DESC] = (desc - mean) / std
    ok = ch >= 0
    x[np.nonzero(ok)[0], N_DESC + ch[ok]] = 1.0
    x[~ok] = 0.0
    return x


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    dims = [N_IN, N_HID, N_HID, N_HID, N_OUT]
    p = {}
    for l in range(4):
        p[f"W{l + 1}"] = rng.normal(0.0, 1.0 / np.sqrt(dims[l]), size=(dims[l], dims[l + 1]))
        p[f"b{l + 1}"] = np.zeros(dims[l + 1])
    return p


def forward(p, x):
    zs, hs = [], [x]
    h = x
    for l in range(1, 4):
        z = h @ p[f"W{l}"] + p[f"b{l}"]
        zs.append(z)
        h = silu(z)
        hs.append(h)
    y = h @ p["W4"] + p["b4"]
    return y, zs, hs


def project(y, atom_offsets, numbers, charges):
    """Shift each molecule's shell charges to sum to its charge (2 shells per atom)."""
    off = np.asarray(atom_offsets)
    q = y.copy()
    for m in range(len(off) - 1):
        a0, a1 = off[m], off[m + 1]
        n = 2 * (a1 - a0)
        if n:
            q[a0:a1] += (charges[m] - q[a0:a1].sum()) / n
    return q


def loss_and_grad(p, x, atom_offsets, numbers, charges, labels):
    """Loss and hand-derived gradients with respect to every weight and bias."""
    y, zs, hs = forward(p, x)
    q = project(y, atom_offsets, numbers, charges)
    nsh = q.size
    r = q - labels
    loss = (r ** 2).sum() / nsh
    gq = 2.0 * r / nsh
    off = np.asarray(atom_offsets)
    gy = gq.copy()
    for m in range(len(off) - 1):
        a0, a1 = off[m], off[m + 1]
        if a1 > a0:
            gy[a0:a1] -= gq[a0:a1].mean()
    g = {"W4": hs[3].T @ gy, "b4": gy.sum(0)}
    gh = gy @ p["W4"].T
    for l in range(3, 0, -1):
        gz = gh * dsilu(zs[l - 1])
        g[f"W{l}"] = hs[l - 1].T @ gz
        g[f"b{l}"] = gz.sum(0)
        gh = gz @ p[f"W{l}"].T
    return loss, g
