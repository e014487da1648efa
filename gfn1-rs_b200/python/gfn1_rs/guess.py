"""Learned SCC initial guess: model files, device inference and GPU training.

The reference has no learned guess; its SCC starts from zero shell charges or
from a caller-supplied vector (gfn1-rs ``src/electronic.rs:1231-1239``).  The
network here predicts that vector from the geometry: per H/C/N/O atom, 64
radial and 32 angular descriptors (cutoff 6 bohr) plus the element one-hot feed
three SiLU layers of 128 and a linear layer to the atom's two shell charges,
which are then shifted so each molecule sums to its charge.  The converged SCC
always decides the result; a worse guess only costs iterations.

Training runs on the GPU through the library's own kernels (descriptors, FP32
GEMMs with fused SiLU epilogues, projection loss, Adam); torch only provides
device memory and the stream.  Inference uses BF16 weights and activations.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from . import _lib
from ._build import PKG_ROOT

MAGIC = b"GFN1MLP1"
DEFAULT_PATH = os.path.join(PKG_ROOT, "data", "guess_mlp.bin")
N_DESC, N_IN, N_HID, N_OUT = 96, 100, 128, 2
LAYOUT = (("mean", N_DESC), ("scale", N_DESC), ("W1", N_IN * N_HID), ("b1", N_HID), ("W2", N_HID * N_HID),
          ("b2", N_HID), ("W3", N_HID * N_HID), ("b3", N_HID), ("W4", N_HID * N_OUT), ("b4", N_OUT))
OFFSETS = {}
_o = 0
for _name, _n in LAYOUT:
    OFFSETS[_name] = (_o, _n)
    _o += _n
N_PARAMS = _o
N_FIXED = 2 * N_DESC  # mean and scale are not trained
SHAPES = {"W1": (N_IN, N_HID), "W2": (N_HID, N_HID), "W3": (N_HID, N_HID), "W4": (N_HID, N_OUT)}
SUPPORTED_Z = (1, 6, 7, 8)


def block(vec: np.ndarray, name: str) -> np.ndarray:
    o, n = OFFSETS[name]
    v = vec[o:o + n]
    return v.reshape(SHAPES[name]) if name in SHAPES else v


def init_params(seed: int = 0) -> np.ndarray:
    """Packed float32 parameters: identity normalisation, scaled normal weights, zero biases."""
    rng = np.random.default_rng(seed)
    vec = np.zeros(N_PARAMS, dtype=np.float32)
    block(vec, "scale")[:] = 1.0
    dims = (N_IN, N_HID, N_HID, N_HID, N_OUT)
    for l in range(4):
        w = rng.normal(0.0, 1.0 / np.sqrt(dims[l]), size=(dims[l], dims[l + 1]))
        block(vec, f"W{l + 1}")[:] = w.astype(np.float32)
    return vec


def save_params(path: str, vec: np.ndarray) -> None:
    vec = np.ascontiguousarray(vec, dtype="<f4")
    if vec.size != N_PARAMS:
        raise ValueError(f"expected {N_PARAMS} parameters, got {vec.size}")
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.int64(vec.size).tobytes())
        f.write(vec.tobytes())


def load_params(path: str = DEFAULT_PATH) -> np.ndarray:
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a GFN1 guess parameter file")
        n = int(np.frombuffer(f.read(8), dtype="<i8")[0])
        vec = np.frombuffer(f.read(4 * n), dtype="<f4").copy()
    if n != N_PARAMS or vec.size != N_PARAMS:
        raise ValueError(f"{path}: expected {N_PARAMS} parameters, found {n}")
    return vec


def _vp(t) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else int(t.data_ptr()))


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class LearnedGuess:
    """A guess model on the engine's device (``gfn1_guess``)."""

    def __init__(self, engine: _lib.Engine, params: np.ndarray):
        L = _lib.load()
        if L.gfn1_guess_param_count() != N_PARAMS:
            raise RuntimeError("library and Python disagree on the guess parameter count")
        self.engine = engine
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        h = ctypes.c_void_p()
        _lib.check(L.gfn1_guess_create(engine.handle, self.params.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                       N_PARAMS, ctypes.byref(h)), engine.handle)
        self.handle = h

    @classmethod
    def from_file(cls, engine: _lib.Engine, path: str = DEFAULT_PATH) -> "LearnedGuess":
        return cls(engine, load_params(path))

    def attach(self) -> None:
        """Make this the engine's default guess (batches prepared afterwards use it)."""
        _lib.check(_lib.load().gfn1_engine_set_guess(self.engine.handle, self.handle), self.engine.handle)

    def detach(self) -> None:
        _lib.check(_lib.load().gfn1_engine_set_guess(self.engine.handle, None), self.engine.handle)

    def close(self) -> None:
        if getattr(self, "handle", None):
            _lib.load().gfn1_guess_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def infer_device(self, x, y) -> None:
        """y[natoms, 2] = network(x[natoms, 100]) on torch CUDA tensors (BF16 inference)."""
        _lib.check(_lib.load().gfn1_guess_infer_device(self.handle, int(x.shape[0]), _vp(x), _vp(y), _stream()),
                   self.engine.handle)

    def predict(self, atom_offsets, numbers, xyz_bohr, charges=None, shell_offsets=None) -> np.ndarray:
        """Initial shell charges [nshells] (engine layout) for flat host inputs."""
        import torch
        dev = torch.device("cuda", self.engine.device)
        off = torch.as_tensor(np.asarray(atom_offsets, dtype=np.int32), device=dev)
        nmol = off.numel() - 1
        if shell_offsets is None:
            from .batch import BatchCalculator
            shell_offsets = BatchCalculator.shell_offsets_for(self.engine, atom_offsets, numbers)
        soff = torch.as_tensor(np.asarray(shell_offsets, dtype=np.int32), device=dev)
        z = torch.as_tensor(np.asarray(numbers, dtype=np.int32), device=dev)
        xyz = torch.as_tensor(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3), device=dev)
        ch = torch.as_tensor(np.zeros(nmol) if charges is None else np.asarray(charges, dtype=np.float64), device=dev)
        natoms = z.numel()
        x = torch.empty((max(natoms, 1), N_IN), dtype=torch.float32, device=dev)
        y = torch.empty((max(natoms, 1), N_OUT), dtype=torch.float32, device=dev)
        q = torch.zeros(max(int(shell_offsets[-1]), 1), dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            _lib.check(_lib.load().gfn1_guess_predict_device(self.handle, nmol, _vp(off), _vp(soff), _vp(z), _vp(xyz),
                                                             _vp(ch), _vp(x), _vp(y), _vp(q), _stream()),
                       self.engine.handle)
            torch.cuda.current_stream().synchronize()
        return q[:int(shell_offsets[-1])].cpu().numpy()


def features_device(atom_off, z, xyz, x, mean=None, scale=None) -> None:
    """x[natoms, 100] (torch CUDA tensors): raw descriptors when mean/scale are None."""
    _lib.check(_lib.load().gfn1_guess_features_device(atom_off.numel() - 1, _vp(atom_off), _vp(z), _vp(xyz),
                                                       _vp(mean), _vp(scale), _vp(x), _stream()))


class GuessTrainer:
    """Trains the guess network on the GPU with the library's kernels.

    Data: molecules (flat atom offsets, numbers, bohr coordinates, charges) and
    their converged shell charges [natoms, 2] (H/C/N/O atoms only)."""

    def __init__(self, params: np.ndarray | None = None, device: int = 0, seed: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.L = _lib.load()
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        self.P = torch.as_tensor(p.copy(), device=self.dev)
        n_train = N_PARAMS - N_FIXED
        self.G = torch.zeros(n_train, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros_like(self.G)
        self.v = torch.zeros_like(self.G)
        self.t = 0
        self.max_rows = 0

    # ---------------------------------------------------------------- data
    def set_data(self, atom_offsets, numbers, xyz_bohr, charges, labels, fit_normalization: bool = True) -> None:
        torch = self.torch
        off = np.asarray(atom_offsets, dtype=np.int32)
        z = np.asarray(numbers, dtype=np.int32)
        if not np.isin(z, SUPPORTED_Z).all():
            raise ValueError("training molecules must contain only H, C, N and O")
        self.off_h = off
        self.nmol = len(off) - 1
        self.natoms = int(off[-1])
        self.off = torch.as_tensor(off, device=self.dev)
        self.z = torch.as_tensor(z, device=self.dev)
        self.xyz = torch.as_tensor(np.asarray(xyz_bohr, dtype=np.float64).reshape(-1, 3), device=self.dev)
        ch = np.zeros(self.nmol) if charges is None else np.asarray(charges, dtype=np.float64)
        self.charge = torch.as_tensor(ch, device=self.dev)
        self.label = torch.as_tensor(np.asarray(labels, dtype=np.float32).reshape(-1, N_OUT), device=self.dev)
        self.x = torch.empty((self.natoms, N_IN), dtype=torch.float32, device=self.dev)
        if fit_normalization:
            features_device(self.off, self.z, self.xyz, self.x)
            raw = self.x[:, :N_DESC].double()
            mean = raw.mean(0)
            scale = raw.std(0).clamp_min(1e-3)
            self.P[OFFSETS["mean"][0]:OFFSETS["mean"][0] + N_DESC] = mean.float()
            self.P[OFFSETS["scale"][0]:OFFSETS["scale"][0] + N_DESC] = scale.float()
        self._refeaturize()
        self.y = torch.zeros((self.natoms, N_OUT), dtype=torch.float32, device=self.dev)
        self.gy = torch.zeros_like(self.y)
        self.loss_mol = torch.zeros(self.nmol, dtype=torch.float64, device=self.dev)

    def _refeaturize(self) -> None:
        mo, so = OFFSETS["mean"][0], OFFSETS["scale"][0]
        features_device(self.off, self.z, self.xyz, self.x, self.P[mo:mo + N_DESC], self.P[so:so + N_DESC])

    def _ensure_rows(self, rows: int) -> None:
        if rows <= self.max_rows:
            return
        torch = self.torch
        self.max_rows = rows
        mk = lambda: torch.empty((rows, N_HID), dtype=torch.float32, device=self.dev)
        self.z1, self.h1, self.z2, self.h2, self.z3, self.h3 = mk(), mk(), mk(), mk(), mk(), mk()
        self.d3, self.d2, self.d1 = mk(), mk(), mk()
        nz = self._ksplit(rows)  # bounds the K-split slices of every smaller row count too
        self.part = torch.empty(nz * N_HID * N_HID + 16, dtype=torch.float32, device=self.dev)
        self.cpart = torch.empty(((rows + 255) // 256) * N_HID + 16, dtype=torch.float32, device=self.dev)

    @staticmethod
    def _ksplit(rows: int) -> int:
        return max(1, min(64, rows // 256))

    # ---------------------------------------------------------------- kernels
    def _p(self, name):
        o, n = OFFSETS[name]
        return self.P[o:o + n]

    def _g(self, name):
        o, n = OFFSETS[name]
        return self.G[o - N_FIXED:o - N_FIXED + n]

    def _gemm(self, ta, tb, epi, M, N, K, A, lda, B, ldb, C, ldc, bias=None, zprev=None, ldz=0, Z=None, ksplit=1):
        _lib.check(self.L.gfn1_mlp_gemm(ta, tb, epi, M, N, K, _vp(A), lda, _vp(B), ldb, _vp(bias), _vp(zprev), ldz,
                                        _vp(C), _vp(Z), ldc, ksplit, _stream()))

    def _weight_grad(self, A, K_in, dY, n_out, rows, gW, gb):
        """gW[K_in, n_out] = A^T dY and gb = column sums of dY over `rows` rows."""
        ks = self._ksplit(rows)
        nz = self.L.gfn1_mlp_gemm_splits(rows, ks)
        self._gemm(1, 0, 0, K_in, n_out, rows, A, K_in, dY, n_out, self.part, n_out, ksplit=ks)
        _lib.check(self.L.gfn1_mlp_reduce(nz, K_in * n_out, _vp(self.part), _vp(gW), K_in * n_out, _stream()))
        mchunk = 256
        nc = max(1, (rows + mchunk - 1) // mchunk)
        _lib.check(self.L.gfn1_mlp_colsum(rows, n_out, _vp(dY), n_out, mchunk, _vp(self.cpart), _stream()))
        _lib.check(self.L.gfn1_mlp_reduce(nc, n_out, _vp(self.cpart), _vp(gb), n_out, _stream()))

    def forward_backward(self, m0: int, m1: int, backward: bool = True) -> None:
        """Loss (per molecule, in loss_mol) and, optionally, gradients in G for molecules [m0, m1)."""
        a0, a1 = int(self.off_h[m0]), int(self.off_h[m1])
        rows = a1 - a0
        self._ensure_rows(max(rows, 1))
        x = self.x[a0:a1]
        y = self.y[a0:a1]
        gy = self.gy[a0:a1]
        H = N_HID
        self._gemm(0, 0, 1, rows, H, N_IN, x, N_IN, self._p("W1"), H, self.h1, H, bias=self._p("b1"), Z=self.z1)
        self._gemm(0, 0, 1, rows, H, H, self.h1, H, self._p("W2"), H, self.h2, H, bias=self._p("b2"), Z=self.z2)
        self._gemm(0, 0, 1, rows, H, H, self.h2, H, self._p("W3"), H, self.h3, H, bias=self._p("b3"), Z=self.z3)
        self._gemm(0, 0, 2, rows, N_OUT, H, self.h3, H, self._p("W4"), N_OUT, y, N_OUT, bias=self._p("b4"))
        inv_nsh = 1.0 / max(N_OUT * rows, 1)
        off = self.off[m0:]
        _lib.check(self.L.gfn1_mlp_project_loss(m1 - m0, _vp(off), _vp(self.y), _vp(self.charge[m0:]),
                                                _vp(self.label), inv_nsh, _vp(self.gy), None,
                                                _vp(self.loss_mol[m0:]), _stream()))
        if not backward:
            return
        self._weight_grad(self.h3, H, gy, N_OUT, rows, self._g("W4"), self._g("b4"))
        self._gemm(0, 1, 3, rows, H, N_OUT, gy, N_OUT, self._p("W4"), N_OUT, self.d3, H, zprev=self.z3, ldz=H)
        self._weight_grad(self.h2, H, self.d3, H, rows, self._g("W3"), self._g("b3"))
        self._gemm(0, 1, 3, rows, H, H, self.d3, H, self._p("W3"), H, self.d2, H, zprev=self.z2, ldz=H)
        self._weight_grad(self.h1, H, self.d2, H, rows, self._g("W2"), self._g("b2"))
        self._gemm(0, 1, 3, rows, H, H, self.d2, H, self._p("W2"), H, self.d1, H, zprev=self.z1, ldz=H)
        self._weight_grad(x, N_IN, self.d1, H, rows, self._g("W1"), self._g("b1"))

    def adam_step(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        self.t += 1
        c1 = 1.0 / (1.0 - beta1 ** self.t)
        c2 = 1.0 / (1.0 - beta2 ** self.t)
        trainable = self.P[N_FIXED:]
        _lib.check(self.L.gfn1_mlp_adam(self.G.numel(), _vp(trainable), _vp(self.G), _vp(self.m), _vp(self.v), lr,
                                        beta1, beta2, eps, c1, c2, _stream()))

    def loss(self, m0: int = 0, m1: int | None = None, chunk: int = 2048) -> float:
        """Mean squared shell-charge error over molecules [m0, m1)."""
        m1 = self.nmol if m1 is None else m1
        tot, nsh = 0.0, 0
        for c0 in range(m0, m1, chunk):
            c1 = min(m1, c0 + chunk)
            self.forward_backward(c0, c1, backward=False)
            rows = int(self.off_h[c1] - self.off_h[c0])
            tot += float(self.loss_mol[c0:c1].sum()) * (N_OUT * rows)
            nsh += N_OUT * rows
        return tot / max(nsh, 1)

    def train(self, epochs: int = 30, batch_mols: int = 128, lr: float = 2e-3, lr_final: float = 5e-5,
              seed: int = 0, log=None) -> list[float]:
        """Adam over shuffled contiguous chunks of batch_mols molecules, cosine learning rate."""
        rng = np.random.default_rng(seed)
        starts = np.arange(0, self.nmol, batch_mols)
        total = epochs * len(starts)
        step = 0
        hist = []
        t0 = time.time()
        for ep in range(epochs):
            for s in rng.permutation(starts):
                frac = step / max(total - 1, 1)
                cur = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * frac))
                self.forward_backward(int(s), int(min(self.nmol, s + batch_mols)))
                self.adam_step(cur)
                step += 1
            l = self.loss()
            hist.append(l)
            if log:
                log(f"epoch {ep + 1}/{epochs}: mse {l:.3e} (rms {np.sqrt(l):.4f} e), {time.time() - t0:.1f} s")
        return hist

    def params(self) -> np.ndarray:
        return self.P.cpu().numpy().copy()

    def gradients(self) -> dict:
        """Current gradient blocks as float64 numpy arrays (after forward_backward)."""
        g = self.G.cpu().numpy().astype(np.float64)
        out = {}
        for name, (o, n) in OFFSETS.items():
            if o < N_FIXED:
                continue
            v = g[o - N_FIXED:o - N_FIXED + n]
            out[name] = v.reshape(SHAPES[name]) if name in SHAPES else v
        return out


def allreduce_weighted(grad, weight: float, total: float, group=None):
    """Data-parallel gradient: grad <- sum over ranks of (weight_r / total) grad_r,
    in place (one all_reduce).  With weight_r the shells of rank r's batch and
    total their sum over ranks, the result is the gradient of the mean loss over
    the union of the ranks' batches, as a single rank computes it."""
    import torch.distributed as dist

    grad.mul_(float(weight) / float(total))
    dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def shard_training_set(nmol: int, rank: int, world: int, seed: int = 0):
    """Molecule indices of rank `rank`: a common shuffle split into `world`
    contiguous parts of equal size (the remainder is dropped so that every rank
    takes the same number of steps)."""
    perm = np.random.default_rng(seed).permutation(nmol)
    per = nmol // world
    return np.sort(perm[rank * per:(rank + 1) * per])


class DataParallelGuessTrainer(GuessTrainer):
    """GuessTrainer over several ranks (one process per GPU, torch.distributed):
    every rank holds its shard of the training set, computes the gradients of
    its batches with the library's kernels, and the ranks average them with one
    all-reduce per step (weighted by shells, allreduce_weighted) before the
    identical Adam step, so all ranks keep the same parameters."""

    def __init__(self, params=None, device: int = 0, seed: int = 0, group=None):
        import torch.distributed as dist

        super().__init__(params, device, seed)
        self.group = group
        self.world = dist.get_world_size(group)
        dist.broadcast(self.P, src=0, group=group)  # one starting point

    def train(self, epochs: int = 30, batch_mols: int = 128, lr: float = 2e-3, lr_final: float = 5e-5,
              seed: int = 0, log=None) -> list[float]:
        import torch.distributed as dist

        rng = np.random.default_rng(seed)  # the same step order on every rank
        starts = np.arange(0, self.nmol, batch_mols)
        total = epochs * len(starts)
        step = 0
        hist = []
        for ep in range(epochs):
            for s in rng.permutation(starts):
                frac = step / max(total - 1, 1)
                cur = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * frac))
                m0, m1 = int(s), int(min(self.nmol, s + batch_mols))
                self.forward_backward(m0, m1)
                rows = float(self.off_h[m1] - self.off_h[m0])
                tot = self.torch.tensor([rows], dtype=self.torch.float64, device=self.dev)
                dist.all_reduce(tot, group=self.group)
                allreduce_weighted(self.G, rows, float(tot.item()), self.group)
                self.adam_step(cur)
                step += 1
            l = self.loss()
            lt = self.torch.tensor([l], dtype=self.torch.float64, device=self.dev)
            dist.all_reduce(lt, group=self.group)
            hist.append(float(lt.item()) / self.world)
            if log:
                log(f"epoch {ep + 1}/{epochs}: mse {hist[-1]:.3e} (mean over ranks)")
        return hist


def label_molecules(calc, atom_offsets, numbers, xyz_bohr, chunk: int = 4096, log=None):
    """Converged shell charges [natoms, 2] and a per-molecule OK mask, from the engine."""
    off = np.asarray(atom_offsets, dtype=np.int32)
    nmol = len(off) - 1
    labels = np.zeros((int(off[-1]), N_OUT))
    ok = np.zeros(nmol, dtype=bool)
    iters = np.zeros(nmol, dtype=np.int32)
    for c0 in range(0, nmol, chunk):
        c1 = min(nmol, c0 + chunk)
        a0, a1 = int(off[c0]), int(off[c1])
        r = calc.calculate_flat(off[c0:c1 + 1] - a0, numbers[a0:a1], xyz_bohr[a0:a1], compute_gradient=False)
        labels[a0:a1] = r.shell_charges.reshape(-1, N_OUT)
        ok[c0:c1] = r.status == 0
        iters[c0:c1] = r.iterations
        if log:
            log(f"labelled {c1}/{nmol} molecules (mean iterations {r.iterations.mean():.2f})")
    return labels, ok, iters


def select_molecules(atom_offsets, numbers, xyz, mask):
    """Flat arrays restricted to molecules where mask is true."""
    off = np.asarray(atom_offsets)
    idx = np.nonzero(mask)[0]
    counts = off[idx + 1] - off[idx]
    new_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    atoms = np.concatenate([np.arange(off[i], off[i + 1]) for i in idx]) if len(idx) else np.zeros(0, np.int64)
    return new_off, np.asarray(numbers)[atoms], np.asarray(xyz).reshape(-1, 3)[atoms], atoms


def train_guess(n_train: int = 50000, seed0: int = 10**6, epochs: int = 30, batch_mols: int = 128,
                lr: float = 2e-3, out: str | None = DEFAULT_PATH, device: int = 0, log=print) -> np.ndarray:
    """Label n_train seed-generated molecules with the engine and train the
    network.  Under torch.distributed (one process per GPU) each rank labels
    and trains on its shard of the training set (DataParallelGuessTrainer);
    rank 0 writes the parameters."""
    import torch.distributed as dist

    from . import workloads
    from .batch import BatchCalculator
    from .native import ANGSTROM_TO_BOHR
    dp = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
    rank, world = (dist.get_rank(), dist.get_world_size()) if dp else (0, 1)
    calc = BatchCalculator(device=device)
    off, z, x = workloads.mixed_batch(n_train, seed0)
    if dp:  # this rank's shard
        from .shard import take
        off, z, x, _, _ = take(off, z, x, shard_training_set(n_train, rank, world, seed=seed0))
    xb = x * ANGSTROM_TO_BOHR
    labels, ok, _ = label_molecules(calc, off, z, xb, log=log)
    off2, z2, x2, atoms = select_molecules(off, z, xb, ok)
    tr = DataParallelGuessTrainer(device=device) if dp else GuessTrainer(device=device)
    tr.set_data(off2, z2, x2, None, labels[atoms])
    if dp:  # the normalisation of the descriptors: rank 0's, so that every rank feeds the same network
        dist.broadcast(tr.P, src=0)
        tr._refeaturize()
    log(f"training on {len(off2) - 1} molecules, {int(off2[-1])} atoms; initial mse {tr.loss():.3e}")
    tr.train(epochs=epochs, batch_mols=batch_mols, lr=lr, log=log)
    p = tr.params()
    if out and rank == 0:
        save_params(out, p)
        log(f"wrote {out}")
    return p


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="train the learned SCC initial guess on the GPU")
    ap.add_argument("--n-train", type=int, default=50000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch-mols", type=int, default=128)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_PATH)
    a = ap.parse_args()
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:  # torchrun: one process per GPU, NCCL
        import datetime

        import torch
        import torch.distributed as dist

        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        try:
            train_guess(a.n_train, epochs=a.epochs, batch_mols=a.batch_mols, lr=a.lr, out=a.out, device=local)
        finally:
            dist.destroy_process_group()
    else:
        train_guess(a.n_train, epochs=a.epochs, batch_mols=a.batch_mols, lr=a.lr, out=a.out)
