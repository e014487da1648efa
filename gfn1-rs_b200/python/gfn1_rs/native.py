"""Reference-compatible native calculator on the B200 engine.

``Gfn1NativeCalculator(...).calculate(numbers, positions, unit, compute_gradient)``
mirrors gfn1-rs's pyo3 class (src/python.rs:116-375): same constructor keywords
and defaults, same ``calculate`` signature, a ``CalculationResult`` with the same
fields (src/python.rs:2845-2950), and every error surfaces as ``ValueError``
(src/python.rs:3344-3346).  Options outside the plain GFN1 energy+gradient path
(multipole, exchange, spin polarization, +U, D4, fields, ...) are rejected
with ValueError when set to a non-default value; ``multiplicity`` selects the
reference's spin-constrained occupations in restricted orbitals.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

HARTREE_TO_EV = 27.211386245988                    # src/constants.rs:17
ANGSTROM_TO_BOHR = 1.8897261246257702              # src/constants.rs:27
BOHR_TO_ANGSTROM = 1.0 / ANGSTROM_TO_BOHR
FORCE_HARTREE_PER_BOHR_TO_EV_PER_ANGSTROM = HARTREE_TO_EV / BOHR_TO_ANGSTROM

_SYMBOLS = ("X H He Li Be B C N O F Ne Na Mg Al Si P S Cl Ar K Ca Sc Ti V Cr Mn Fe Co Ni Cu Zn Ga Ge As Se Br Kr "
            "Rb Sr Y Zr Nb Mo Tc Ru Rh Pd Ag Cd In Sn Sb Te I Xe Cs Ba La Ce Pr Nd Pm Sm Eu Gd Tb Dy Ho Er Tm "
            "Yb Lu Hf Ta W Re Os Ir Pt Au Hg Tl Pb Bi Po At Rn").split()

_UNIT_SCALE = {"angstrom": ANGSTROM_TO_BOHR, "Angstrom": ANGSTROM_TO_BOHR, "A": ANGSTROM_TO_BOHR,
               "bohr": 1.0, "Bohr": 1.0, "au": 1.0}

# Keywords of the reference constructor that select paths outside the plain
# non-periodic GFN1 SCC, with the value that keeps them off.
_OFF_PATH_DEFAULTS = {
    "spin_polarization": False, "experimental_d4": False, "d4_cutoff": None,
    "d4_cn_cutoff": None, "d4_atm": True, "d4_atm_cutoff": None, "d4_s9": None, "enable_cn_hamiltonian": True,
    "electric_field": None, "scc_accelerator": None, "multipole": False,
    "multipole_octupole": False, "field_multipole": False, "multipole_third_order": False,
    "multipole_secondary_basis": None, "multipole_order": 0, "multipole_charge_order": (), "lr_exchange": False,
    "onsite_exchange": False, "dynamic_omega": False, "scf_trah": False, "charge_order": 3,
    "multipole_rank_ladder_base": None, "multipole_model": None, "camm_damp": 1.0, "camm_aes_scale": 1.0,
    "camm_onsite_scale": 1.0, "camm_preset": None, "plus_u": False, "hubbard_u": (), "plus_u_v": False,
    "hubbard_v": (), "hubbard_v_cutoff": 10.0, "hubbard_u_linear_response": False, "plus_u_all_d": False,
    "d3_reference_path": None,
}


def _multiplicity(m) -> int:
    """ElectronicOptions::spin_multiplicity: None -> 0 (none), else the integer (>= 1)."""
    if m is None:
        return 0
    m = int(m)
    if m < 1:
        raise ValueError("spin multiplicity must be at least 1")
    return m


def unit_scale(unit: str) -> float:
    try:
        return _UNIT_SCALE[unit]
    except KeyError:
        raise ValueError(f"unsupported coordinate unit `{unit}`") from None


def build_system(numbers, positions, unit: str):
    """Validates and converts to (uint8 Z, bohr xyz); src/python.rs:3216-3252."""
    numbers = list(numbers)
    positions = [list(p) for p in positions]
    if len(numbers) != len(positions):
        raise ValueError(f"numbers has length {len(numbers)}, positions has length {len(positions)}")
    for i, p in enumerate(positions):
        if len(p) != 3:
            raise ValueError(f"positions[{i}] has length {len(p)}, expected 3")
    scale = unit_scale(unit)
    z = np.asarray(numbers, dtype=np.int64)
    if np.any(z < 0) or np.any(z > 255):
        raise ValueError("atomic numbers must fit in u8")
    xyz = np.asarray(positions, dtype=np.float64).reshape(-1, 3) * scale
    return z.astype(np.uint8), np.ascontiguousarray(xyz)


class CalculationResult:
    """Result of ``Gfn1NativeCalculator.calculate`` (src/python.rs:2845-2950)."""

    def __init__(self, energy, terms, gradient, charges, dipole, iterations, converged, shell_charges=None,
                 fermi_level=None):
        self.energy_hartree = float(energy)
        self.energy_ev = float(energy) * HARTREE_TO_EV
        self.gradient_hartree_per_bohr = None if gradient is None else gradient.tolist()
        self.forces_ev_per_angstrom = (None if gradient is None else
                                       (-gradient * FORCE_HARTREE_PER_BOHR_TO_EV_PER_ANGSTROM).tolist())
        self.charges = list(map(float, charges))
        self.dipole = tuple(map(float, dipole))
        self.stress = None
        self.iterations = int(iterations)
        self.converged = bool(converged)
        self.shell_charges = None if shell_charges is None else list(map(float, shell_charges))
        self.fermi_level = fermi_level
        self._terms = [(k, float(v)) for k, v in zip(_lib.TERM_NAMES, terms)]

    def energy_terms_hartree(self) -> dict:
        return dict(self._terms)

    def energy_terms_ev(self) -> dict:
        return {k: v * HARTREE_TO_EV for k, v in self._terms}

    def __repr__(self) -> str:
        return (f"CalculationResult(energy_hartree={self.energy_hartree:.12f}, natoms={len(self.charges)}, "
                f"converged={self.converged}, iterations={self.iterations})")


class Gfn1NativeCalculator:
    """GFN1-xTB single points on a B200 (src/python.rs:116-323 signature)."""

    def __init__(self, param_path=None, charge=0.0, multiplicity=None, spin_polarization=False, max_scc=250,
                 energy_tolerance=1.0e-6, charge_tolerance=2.0e-5, mixing=0.4, scc_broyden=True,
                 scc_broyden_size=250, electronic_temperature=300.0, nprim=0, eigen_tolerance=1.0e-12,
                 enable_dispersion=True, device=0, level_shift=0.0, **kwargs):
        off = dict(spin_polarization=spin_polarization)
        off.update(kwargs)
        for k, v in off.items():
            if k not in _OFF_PATH_DEFAULTS:
                raise TypeError(f"Gfn1NativeCalculator() got an unexpected keyword argument '{k}'")
            dflt = _OFF_PATH_DEFAULTS[k]
            same = (v == dflt) or (v is None and dflt is None) or (isinstance(dflt, tuple) and not v)
            if not same:
                raise ValueError(f"option `{k}` selects a path outside the B200 engine (plain GFN1 SCC only)")
        if nprim not in (0, None):
            raise ValueError("nprim overrides are not supported by the B200 engine (GFN1 primitive-count rule only)")
        if eigen_tolerance != 1.0e-12:
            raise ValueError("eigen_tolerance is fixed at 1e-12 in the B200 engine")
        self.charge = float(charge)
        self._opts = dict(max_scc=max_scc, energy_tolerance=energy_tolerance, charge_tolerance=charge_tolerance,
                          mixing=mixing, scc_broyden=int(bool(scc_broyden)), scc_broyden_size=scc_broyden_size,
                          electronic_temperature=electronic_temperature, enable_dispersion=int(bool(enable_dispersion)),
                          spin_multiplicity=_multiplicity(multiplicity), level_shift=float(level_shift))
        self._param_path = param_path
        self._engine = _lib.Engine(param_path, device)

    def param_source(self) -> str:
        return f"GFN1-xTB (tables: {self._param_path or _lib.TABLES_PATH})"

    def __repr__(self) -> str:
        return f"Gfn1NativeCalculator(parameters: {self.param_source()})"

    def calculate(self, numbers, positions, unit="angstrom", compute_gradient=False,
                  initial_shell_charges=None) -> CalculationResult:
        """Single point (+ gradient) of one molecule (src/python.rs:339-375)."""
        z, xyz = build_system(numbers, positions, unit)
        nat = len(z)
        if nat == 0:
            raise ValueError("cannot run GFN1 SCC for an empty basis")
        L = _lib.load()
        nao, nsh = self._engine.basis_size(z)
        opt = _lib.default_options(compute_gradient=int(bool(compute_gradient)), **self._opts)
        terms = np.zeros(15)
        grad = np.zeros((nat, 3)) if compute_gradient else None
        qat = np.zeros(nat)
        qsh = np.zeros(nsh)
        dip = np.zeros(3)
        fermi = np.zeros(1)
        iters = np.zeros(1, dtype=np.int32)
        status = np.zeros(1, dtype=np.int32)
        out = _lib.Outputs(None, _lib.ptr(terms), _lib.ptr(grad), _lib.ptr(qsh), _lib.ptr(qat), _lib.ptr(dip),
                           _lib.ptr(fermi), _lib.ptr(iters, ctypes.c_int32), _lib.ptr(status, ctypes.c_int32))
        q0 = None
        if initial_shell_charges is not None:
            q0 = np.ascontiguousarray(initial_shell_charges, dtype=np.float64)
            if q0.shape != (nsh,):
                q0 = None  # the reference ignores a guess of the wrong length (src/electronic.rs:1233-1239)
        rc = L.gfn1_run(self._engine.handle, nat, _lib.ptr(z, ctypes.c_uint8), _lib.ptr(xyz), self.charge,
                        _lib.ptr(q0), ctypes.byref(opt), ctypes.byref(out))
        _lib.check(rc, self._engine.handle)
        return CalculationResult(terms[0], terms, grad, qat, dip, iters[0], status[0] == 0, shell_charges=qsh,
                                 fermi_level=float(fermi[0]))

    def calculate_periodic(self, *args, **kwargs):
        """The reference's periodic single point (src/python.rs:386) is outside
        the B200 engine, which runs molecules only; like every engine error it
        raises ValueError."""
        raise ValueError("periodic systems are outside the B200 engine (non-periodic molecules only)")

    # ------------------------------------------------------------------ batch-backed methods
    def _batch(self):
        if getattr(self, "_batch_calc", None) is None:
            from .batch import BatchCalculator
            self._batch_calc = BatchCalculator(param_path=self._param_path, device=self._engine.device, **self._opts)
        return self._batch_calc

    def optimize(self, numbers, positions, unit="angstrom", cell=None, pbc=(True, True, True), max_iterations=250,
                 gradient_tolerance=1.0e-4, step_tolerance=1.0e-7, history=12, max_atom_step=0.30,
                 trajectory_path=None) -> "OptimizationResult":
        """L-BFGS geometry optimisation (src/python.rs:490-546 over
        src/optimizer.rs:78-320); non-periodic only."""
        from .optimize import OptimizeOptions, optimize_batch
        if cell is not None:
            raise ValueError("the B200 engine optimises non-periodic systems only")
        z, xyz = build_system(numbers, positions, unit)
        if len(z) == 0:
            raise ValueError("cannot run GFN1 SCC for an empty basis")
        opts = OptimizeOptions(max_iterations=int(max_iterations), gradient_tolerance=float(gradient_tolerance),
                               step_tolerance=float(step_tolerance), history=int(history),
                               max_atom_step=float(max_atom_step))
        out = optimize_batch(self._batch(), [0, len(z)], z, xyz, charges=[self.charge], options=opts)
        if out["errors"][0] is not None and out["gradient"][0] is None:
            raise ValueError(out["errors"][0])
        res = OptimizationResult(z, out, 0)
        if trajectory_path:
            res.write_trajectory(trajectory_path)
        return res

    def hessian(self, numbers, positions, unit="angstrom"):
        """Nuclear Hessian (Eh/bohr^2) as a 3N x 3N nested list, atom-major
        (src/python.rs:1747-1771); central differences of the analytic
        gradient (gfn1_rs.hessian)."""
        return self._hessian_array(numbers, positions, unit).tolist()

    def vibrational_frequencies(self, numbers, positions, unit="angstrom") -> dict:
        """``wavenumbers`` (cm^-1, imaginary as negative) and ``modes``
        (src/python.rs:1821-1850)."""
        from .hessian import vibrational_analysis
        z, _ = build_system(numbers, positions, unit)
        v = vibrational_analysis(self._hessian_array(numbers, positions, unit), z)
        return {"wavenumbers": v["wavenumbers"].tolist(), "modes": v["modes"].tolist()}

    def _hessian_array(self, numbers, positions, unit):
        from .hessian import hessian_batch
        z, xyz = build_system(numbers, positions, unit)
        if len(z) == 0:
            raise ValueError("cannot run GFN1 SCC for an empty basis")
        out = hessian_batch(self._batch(), [0, len(z)], z, xyz, charges=[self.charge])
        if out["hessians"][0] is None:
            _lib.check(int(out["status"][0]) or 8)
        return out["hessians"][0]


class OptimizationResult:
    """Result of ``Gfn1NativeCalculator.optimize`` (src/python.rs:2954-3010)."""

    def __init__(self, numbers, out: dict, m: int):
        frames = out["frames"][m]
        g = np.asarray(out["gradient"][m]).reshape(-1, 3)
        self.numbers = [int(v) for v in numbers]
        self.energy_hartree = float(out["energy"][m])
        self.energy_ev = self.energy_hartree * HARTREE_TO_EV
        self.positions_angstrom = (np.asarray(frames[-1]).reshape(-1, 3) * BOHR_TO_ANGSTROM).tolist()
        self.gradient_hartree_per_bohr = g.tolist()
        self.forces_ev_per_angstrom = (-g * FORCE_HARTREE_PER_BOHR_TO_EV_PER_ANGSTROM).tolist()
        self.iterations = int(out["iterations"][m])
        self.converged = bool(out["converged"][m])
        self.max_gradient = float(out["max_gradient"][m])
        self.trajectory_positions_angstrom = [(np.asarray(f).reshape(-1, 3) * BOHR_TO_ANGSTROM).tolist()
                                              for f in frames]
        self.trajectory_energies_hartree = [float(t[1]) for t in out["trajectories"][m]]

    def write_trajectory(self, path: str) -> None:
        """XYZ frames of the accepted steps (energy in the comment line)."""
        with open(path, "w") as fh:
            for xyz, e in zip(self.trajectory_positions_angstrom, self.trajectory_energies_hartree):
                fh.write(f"{len(self.numbers)}\nenergy_hartree={e:.12f}\n")
                for zz, p in zip(self.numbers, xyz):
                    fh.write(f"{_SYMBOLS[zz]} {p[0]:.10f} {p[1]:.10f} {p[2]:.10f}\n")

