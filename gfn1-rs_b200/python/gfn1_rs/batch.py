"""Batched GFN1-xTB energy + gradient of many independent molecules.

``BatchCalculator.calculate`` is the host-buffer path (one C call; the host to
device copies of the inputs and the device to host copies of the results are
inside).  ``ResidentBatch`` keeps the topology and workspace on the device so
coordinates can be replaced and the batch re-run with inputs already in HBM.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .native import build_system, unit_scale


@dataclass
class BatchResult:
    energy: np.ndarray          # [nmol] total_free (Eh)
    terms: np.ndarray           # [nmol, 15]
    gradient: np.ndarray | None  # [natoms, 3] (Eh/bohr)
    shell_charges: np.ndarray   # [nshells]
    atomic_charges: np.ndarray  # [natoms]
    dipole: np.ndarray          # [nmol, 3]
    fermi_level: np.ndarray     # [nmol]
    iterations: np.ndarray      # [nmol]
    status: np.ndarray          # [nmol]
    atom_offsets: np.ndarray
    shell_offsets: np.ndarray
    # [nmol] rung of the reference's fallback ladder (src/electronic.rs:1390-1447)
    # whose SCC converged: 0 = the requested scheme, 1-2 = linear mixing with a
    # level shift, 3 = T_el raised to max(T_el, 3000 K); -1 where none converged
    rung: np.ndarray | None = None


def _flatten(molecules, unit):
    offs = [0]
    zs, xs = [], []
    for numbers, positions in molecules:
        z, x = build_system(numbers, positions, unit)
        zs.append(z)
        xs.append(x)
        offs.append(offs[-1] + len(z))
    return (np.asarray(offs, dtype=np.int32), np.concatenate(zs).astype(np.uint8),
            np.ascontiguousarray(np.concatenate(xs)))


def _options(opts: dict, compute_gradient: bool) -> _lib.Options:
    return _lib.default_options(compute_gradient=int(bool(compute_gradient)), **opts)


def _matrices(engine, off, z, m: int, call, fock_call) -> dict:
    if not 0 <= m < len(off) - 1:
        raise IndexError(f"molecule {m} out of range")
    nao_z, nsh_z = engine.element_sizes()
    zm = np.asarray(z[off[m]:off[m + 1]], dtype=np.int64)
    n, nsh = int(np.sum(nao_z[zm])), int(np.sum(nsh_z[zm]))
    keys = ("S", "H0", "P", "W", "orbital_energies", "occupations")
    out = {k: np.zeros((n, n)) for k in keys[:4]}
    out.update({k: np.zeros(n) for k in keys[4:]})
    _lib.check(call(*[_lib.ptr(out[k]) for k in keys]), engine.handle)
    out["fock"] = np.zeros((n, n))
    out["shell_scc_potential"] = np.zeros(nsh)
    out["coordination_numbers"] = np.zeros(len(zm))
    _lib.check(fock_call(_lib.ptr(out["fock"]), _lib.ptr(out["shell_scc_potential"]),
                         _lib.ptr(out["coordination_numbers"])), engine.handle)
    return out


class BatchCalculator:
    def __init__(self, param_path=None, device=0, max_scc=250, energy_tolerance=1.0e-6, charge_tolerance=2.0e-5,
                 mixing=0.4, scc_broyden=True, scc_broyden_size=250, electronic_temperature=300.0,
                 enable_dispersion=True, learned_guess=None, spin_multiplicity=None, level_shift=0.0):
        """learned_guess: None/False for the reference's zero initial guess, True for
        the packaged trained network, or a path to a parameter file.
        spin_multiplicity: None (the reference's default) or n >= 1 for every
        molecule of a call (spin-constrained occupations).  level_shift: the
        reference's virtual level shift (Eh), molecules of every size."""
        self.engine = _lib.Engine(param_path, device)
        self.guess = None
        if learned_guess:
            from .guess import DEFAULT_PATH, LearnedGuess
            self.guess = LearnedGuess.from_file(self.engine, DEFAULT_PATH if learned_guess is True else learned_guess)
            self.guess.attach()
        self.opts = dict(max_scc=max_scc, energy_tolerance=energy_tolerance, charge_tolerance=charge_tolerance,
                         mixing=mixing, scc_broyden=int(bool(scc_broyden)), scc_broyden_size=scc_broyden_size,
                         electronic_temperature=electronic_temperature,
                         enable_dispersion=int(bool(enable_dispersion)),
                         spin_multiplicity=int(spin_multiplicity or 0), level_shift=float(level_shift))
        self._last = None  # (atom_offsets, numbers) of the last calculate_flat call
        self._last_shoff = None  # its shell offsets (read-only), reused while the topology repeats

    def shell_offsets(self, atom_offsets, numbers) -> np.ndarray:
        """Prefix sums of the shell counts, laid out as the C side does (atoms of
        unsupported elements contribute no shells)."""
        return self.shell_offsets_for(self.engine, atom_offsets, numbers)

    @staticmethod
    def shell_offsets_for(engine, atom_offsets, numbers) -> np.ndarray:
        # one table lookup per atom over the uint8 atomic numbers the C side receives
        table = engine.shell_count_table()
        z = np.asarray(numbers)
        if z.dtype != np.uint8:
            z = z.astype(np.uint8)
        cum = np.zeros(len(z) + 1, dtype=np.int64)
        np.cumsum(table[z], out=cum[1:])
        return cum[np.asarray(atom_offsets)]

    def calculate_flat(self, atom_offsets, numbers, xyz_bohr, charges=None, initial_shell_charges=None,
                       compute_gradient=True, raise_on_error=False) -> BatchResult:
        """Flat inputs: atom_offsets [nmol+1], numbers [natoms], xyz_bohr [natoms,3]."""
        L = _lib.load()
        off = np.ascontiguousarray(atom_offsets, dtype=np.int32)
        z = np.ascontiguousarray(numbers, dtype=np.uint8)
        xyz = np.ascontiguousarray(xyz_bohr, dtype=np.float64).reshape(-1, 3)
        nmol, natoms = len(off) - 1, int(off[-1])
        if (self._last is not None and np.array_equal(self._last[0], off) and np.array_equal(self._last[1], z)):
            off, z = self._last  # the same topology as the last call (trajectories, optimisers, repeated batches)
            shoff = self._last_shoff
        else:
            off, z = off.copy(), z.copy()
            shoff = self.shell_offsets(off, z)
            for a in (off, z, shoff):  # shared by the results and the cache
                a.flags.writeable = False
        nsh = int(shoff[-1])
        ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        q0 = None if initial_shell_charges is None else np.ascontiguousarray(initial_shell_charges, dtype=np.float64)
        energy = np.zeros(nmol)
        terms = np.zeros((nmol, 15))
        grad = np.zeros((natoms, 3)) if compute_gradient else None
        qsh = np.zeros(nsh)
        qat = np.zeros(natoms)
        dip = np.zeros((nmol, 3))
        fermi = np.zeros(nmol)
        iters = np.zeros(nmol, dtype=np.int32)
        status = np.zeros(nmol, dtype=np.int32)
        rung = np.zeros(nmol, dtype=np.int32)
        out = _lib.Outputs(_lib.ptr(energy), _lib.ptr(terms), _lib.ptr(grad), _lib.ptr(qsh), _lib.ptr(qat),
                           _lib.ptr(dip), _lib.ptr(fermi), _lib.ptr(iters, ctypes.c_int32),
                           _lib.ptr(status, ctypes.c_int32), _lib.ptr(rung, ctypes.c_int32))
        opt = _options(self.opts, compute_gradient)
        rc = L.gfn1_batch_energy_gradient(self.engine.handle, nmol, _lib.ptr(off, ctypes.c_int32),
                                          _lib.ptr(z, ctypes.c_uint8), _lib.ptr(xyz), _lib.ptr(ch), _lib.ptr(q0),
                                          ctypes.byref(opt), ctypes.byref(out))
        self._last, self._last_shoff = (off, z), shoff
        if rc != 0 and (raise_on_error or rc not in (3, 4, 8, 12)):
            _lib.check(rc, self.engine.handle)
        return BatchResult(energy, terms, grad, qsh, qat, dip, fermi, iters, status, off, shoff, rung)

    def molecule_matrices(self, m: int) -> dict:
        """S, H0, P, W, fock ([N, N]), orbital energies / occupations ([N]),
        shell_scc_potential ([nshells]) and coordination_numbers ([natoms]) of
        molecule m of the last calculate_flat call: the optional members of the
        reference's ElectronicResult (gfn1-rs src/electronic.rs:600-620).
        Orbital energies the eigensolver did not need are NaN."""
        if self._last is None:
            raise RuntimeError("no calculation on this calculator yet")
        off, z = self._last
        L, h = _lib.load(), self.engine.handle
        return _matrices(self.engine, off, z, m, lambda *p: L.gfn1_last_molecule_matrices(h, int(m), *p),
                         lambda *p: L.gfn1_last_molecule_fock(h, int(m), *p))

    def calculate(self, molecules, unit="angstrom", charges=None, compute_gradient=True, **kw) -> BatchResult:
        """molecules: iterable of (numbers, positions) in `unit`."""
        off, z, xyz = _flatten(molecules, unit)
        return self.calculate_flat(off, z, xyz, charges=charges, compute_gradient=compute_gradient, **kw)

    def resident(self, atom_offsets, numbers, charges=None, compute_gradient=True) -> "ResidentBatch":
        return ResidentBatch(self, atom_offsets, numbers, charges, compute_gradient)


class ResidentBatch:
    """Device-resident batch: topology uploaded once, coordinates replaceable."""

    def __init__(self, calc: BatchCalculator, atom_offsets, numbers, charges=None, compute_gradient=True):
        L = _lib.load()
        self.calc = calc
        self.atom_offsets = np.ascontiguousarray(atom_offsets, dtype=np.int32)
        self.numbers = np.ascontiguousarray(numbers, dtype=np.uint8)
        self.nmol = len(self.atom_offsets) - 1
        ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
        opt = _options(calc.opts, compute_gradient)
        h = ctypes.c_void_p()
        _lib.check(L.gfn1_batch_create(calc.engine.handle, self.nmol, _lib.ptr(self.atom_offsets, ctypes.c_int32),
                                       _lib.ptr(self.numbers, ctypes.c_uint8), _lib.ptr(ch), ctypes.byref(opt),
                                       ctypes.byref(h)), calc.engine.handle)
        self.handle = h
        na, ns, no = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        nl = ctypes.c_int32()
        L.gfn1_batch_info(h, ctypes.byref(na), ctypes.byref(ns), ctypes.byref(no), ctypes.byref(nl))
        self.natoms, self.nshells, self.naos, self.launches = na.value, ns.value, no.value, nl.value
        self.compute_gradient = compute_gradient

    def molecule_matrices(self, m: int) -> dict:
        """As BatchCalculator.molecule_matrices, after this batch's last launch."""
        L = _lib.load()
        return _matrices(self.calc.engine, self.atom_offsets, self.numbers, m,
                         lambda *p: L.gfn1_batch_molecule_matrices(self.handle, int(m), *p),
                         lambda *p: L.gfn1_batch_molecule_fock(self.handle, int(m), *p))

    def optimize(self, max_iterations=250, gradient_tolerance=1.0e-4, step_tolerance=1.0e-7, history=12,
                 initial_step=1.0, max_atom_step=0.30, max_rounds=100000) -> dict:
        """Geometry optimisation of every molecule on the device
        (gfn1_batch_optimize; the reference's optimize_geometry) from the
        positions set with set_positions.  Returns final coordinates (bohr),
        energies, largest gradient components, accepted steps, converged flags,
        statuses and the number of engine passes."""
        L = _lib.load()
        o = _lib.OptOptions()
        L.gfn1_default_opt_options(ctypes.byref(o))
        o.max_iterations, o.gradient_tolerance, o.step_tolerance = int(max_iterations), gradient_tolerance, step_tolerance
        o.history, o.initial_step, o.max_atom_step, o.max_rounds = int(history), initial_step, max_atom_step, int(max_rounds)
        xyz = np.zeros((self.natoms, 3))
        energy = np.zeros(self.nmol)
        maxg = np.zeros(self.nmol)
        iters = np.zeros(self.nmol, dtype=np.int32)
        conv = np.zeros(self.nmol, dtype=np.int32)
        status = np.zeros(self.nmol, dtype=np.int32)
        rounds = ctypes.c_int32()
        rc = L.gfn1_batch_optimize(self.handle, ctypes.byref(o), _lib.ptr(xyz), _lib.ptr(energy), _lib.ptr(maxg),
                                   _lib.ptr(iters, ctypes.c_int32), _lib.ptr(conv, ctypes.c_int32),
                                   _lib.ptr(status, ctypes.c_int32), ctypes.byref(rounds))
        if rc not in (0, 3, 8):
            _lib.check(rc, self.calc.engine.handle)
        return {"xyz": xyz, "energy": energy, "max_gradient": maxg, "iterations": iters,
                "converged": conv.astype(bool), "status": status, "engine_calls": rounds.value + 1}

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().gfn1_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_positions(self, xyz, on_device: bool = False):
        """xyz: numpy array (bohr) or, with on_device=True, an integer device pointer."""
        if on_device:
            p = ctypes.c_void_p(int(xyz))
        else:
            arr = np.ascontiguousarray(xyz, dtype=np.float64)
            self._xyz_keep = arr
            p = arr.ctypes.data_as(ctypes.c_void_p)
        _lib.check(_lib.load().gfn1_batch_set_positions(self.handle, p, int(on_device)), self.calc.engine.handle)

    def set_guess(self, guess):
        """Learned initial guess for launches without initial charges (None: zero guess)."""
        _lib.check(_lib.load().gfn1_batch_set_guess(self.handle, None if guess is None else guess.handle),
                   self.calc.engine.handle)
        self._guess = guess
        na, ns, no = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        nl = ctypes.c_int32()
        _lib.load().gfn1_batch_info(self.handle, ctypes.byref(na), ctypes.byref(ns), ctypes.byref(no), ctypes.byref(nl))
        self.launches = nl.value

    def set_initial_charges(self, q, on_device: bool = False):
        if q is None:
            p = None
        elif on_device:
            p = ctypes.c_void_p(int(q))
        else:
            arr = np.ascontiguousarray(q, dtype=np.float64)
            self._q_keep = arr
            p = arr.ctypes.data_as(ctypes.c_void_p)
        _lib.check(_lib.load().gfn1_batch_set_initial_charges(self.handle, p, int(on_device)), self.calc.engine.handle)

    def launch(self, stream: int | None = None):
        """Enqueue the kernels on a CUDA stream handle (int) or the engine stream."""
        s = None if stream is None else ctypes.c_void_p(int(stream))
        _lib.check(_lib.load().gfn1_batch_launch(self.handle, s), self.calc.engine.handle)

    def launch_stage(self, stage: int, stream: int | None = None):
        """0 = setup, 1 = SCC, 2 = gradient (for per-kernel timing)."""
        s = None if stream is None else ctypes.c_void_p(int(stream))
        _lib.check(_lib.load().gfn1_batch_launch_stage(self.handle, int(stage), s), self.calc.engine.handle)

    STAGES = ("prologue", "fock", "tridiag", "eigval", "fermi", "inviter", "backtr", "pop", "energy", "mix", "final",
              "chol", "linv")

    def stage_cycles(self) -> dict:
        """Per-stage SCC clock totals (batch created with GFN1_PROFILE=1)."""
        buf = (ctypes.c_uint64 * len(self.STAGES))()
        _lib.check(_lib.load().gfn1_batch_stage_cycles(self.handle, buf, len(self.STAGES)), self.calc.engine.handle)
        return dict(zip(self.STAGES, list(buf)))

    def io_bytes(self) -> tuple[int, int]:
        h2d, d2h = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(_lib.load().gfn1_batch_io_bytes(self.handle, ctypes.byref(h2d), ctypes.byref(d2h)),
                   self.calc.engine.handle)
        return h2d.value, d2h.value

    def device_outputs(self) -> dict:
        out = _lib.Outputs()
        _lib.check(_lib.load().gfn1_batch_outputs_device(self.handle, ctypes.byref(out)), self.calc.engine.handle)
        def addr(p):
            return ctypes.cast(p, ctypes.c_void_p).value
        return {k: addr(getattr(out, k)) for k in ("terms", "gradient", "shell_charges", "atomic_charges", "dipole",
                                                   "fermi_level", "iterations", "status", "rung")}

    def download(self) -> BatchResult:
        L = _lib.load()
        energy = np.zeros(self.nmol)
        terms = np.zeros((self.nmol, 15))
        grad = np.zeros((self.natoms, 3)) if self.compute_gradient else None
        qsh = np.zeros(self.nshells)
        qat = np.zeros(self.natoms)
        dip = np.zeros((self.nmol, 3))
        fermi = np.zeros(self.nmol)
        iters = np.zeros(self.nmol, dtype=np.int32)
        status = np.zeros(self.nmol, dtype=np.int32)
        rung = np.zeros(self.nmol, dtype=np.int32)
        out = _lib.Outputs(_lib.ptr(energy), _lib.ptr(terms), _lib.ptr(grad), _lib.ptr(qsh), _lib.ptr(qat),
                           _lib.ptr(dip), _lib.ptr(fermi), _lib.ptr(iters, ctypes.c_int32),
                           _lib.ptr(status, ctypes.c_int32), _lib.ptr(rung, ctypes.c_int32))
        rc = L.gfn1_batch_download(self.handle, ctypes.byref(out))
        if rc not in (0, 3, 4, 8, 12):
            _lib.check(rc, self.calc.engine.handle)
        shoff = self.calc.shell_offsets(self.atom_offsets, self.numbers)
        return BatchResult(energy, terms, grad, qsh, qat, dip, fermi, iters, status, self.atom_offsets, shoff, rung)


__all__ = ["BatchCalculator", "BatchResult", "ResidentBatch", "unit_scale"]
