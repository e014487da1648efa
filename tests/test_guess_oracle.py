"""CPU checks of the learned-guess oracle and of the parameter layout.

The oracle (numpy, float64) derives the MLP weight gradients by hand; here they
are checked against central finite differences of its own loss, so the GPU
training kernels have a trusted reference.  Tolerance: relative 1e-6 on the
largest gradient entry of each block.
"""
import numpy as np
import pytest

import guess_oracle as go


def _batch(seed=0, nmol=4):
    from gfn1_rs import workloads
    off, z, x = workloads.mixed_batch(nmol, seed)
    return off, z, x * 1.8897261246257702


def test_descriptor_invariances():
    off, z, x = _batch()
    d = go.descriptors(off, z, x)
    assert d.shape == (len(z), go.N_DESC)
    assert np.all(d >= 0.0)
    rng = np.random.default_rng(1)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    d2 = go.descriptors(off, z, x @ q.T + np.array([3.0, -1.0, 2.0]))
    assert np.max(np.abs(d2 - d)) <= 1e-10 * max(1.0, np.abs(d).max())
    # permuting atoms inside a molecule permutes the rows
    a0, a1 = off[0], off[1]
    perm = np.arange(len(z))
    perm[a0:a1] = perm[a0:a1][::-1]
    d3 = go.descriptors(off, z[perm], x[perm])
    assert np.max(np.abs(d3 - d[perm])) <= 1e-10 * max(1.0, np.abs(d).max())


def test_hand_gradients_match_finite_differences():
    off, z, x = _batch(nmol=3)
    d = go.descriptors(off, z, x)
    mean, std = d.mean(0), d.std(0) + 1e-3
    feats = go.features(d, z, mean, std)
    p = go.init_params(3)
    rng = np.random.default_rng(4)
    for k in p:
        if k.startswith("b"):
            p[k] = rng.normal(0.0, 0.1, size=p[k].shape)
    charges = np.array([0.0, 1.0, -1.0])
    labels = rng.normal(0.0, 0.3, size=(len(z), 2))
    loss, g = go.loss_and_grad(p, feats, off, z, charges, labels)
    h = 1e-6
    for name in ("W1", "b1", "W2", "b3", "W4", "b4"):
        flat = p[name].reshape(-1)
        idx = rng.choice(flat.size, size=min(6, flat.size), replace=False)
        scale = np.abs(g[name]).max()
        for i in idx:
            old = flat[i]
            flat[i] = old + h
            lp, _ = go.loss_and_grad(p, feats, off, z, charges, labels)
            flat[i] = old - h
            lm, _ = go.loss_and_grad(p, feats, off, z, charges, labels)
            flat[i] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[name].reshape(-1)[i]) <= 1e-6 * scale + 1e-9, (name, i)


def test_projection_conserves_charge():
    off, z, x = _batch(nmol=3)
    y = np.random.default_rng(0).normal(size=(len(z), 2))
    ch = np.array([0.0, 2.0, -1.0])
    q = go.project(y, off, z, ch)
    for m in range(3):
        assert abs(q[off[m]:off[m + 1]].sum() - ch[m]) < 1e-12


def test_parameter_layout_matches_library():
    from gfn1_rs import _lib, guess
    assert _lib.load().gfn1_guess_param_count() == guess.N_PARAMS
    n = go.N_IN * go.N_HID + go.N_HID + 2 * (go.N_HID * go.N_HID + go.N_HID) + go.N_HID * go.N_OUT + go.N_OUT
    assert guess.N_PARAMS == 2 * go.N_DESC + n


def test_parameter_file_round_trip(tmp_path):
    from gfn1_rs import guess
    p = guess.init_params(7)
    path = tmp_path / "g.bin"
    guess.save_params(str(path), p)
    assert np.array_equal(guess.load_params(str(path)), p)
    with pytest.raises(ValueError):
        guess.save_params(str(path), p[:-1])
