"""ctypes front end of the CPU FP64 oracle (test infrastructure only).

The oracle is a C++ restatement of gfn1-rs v0.5.1's non-periodic SCC energy +
analytic gradient path (``gfn1_oracle.cpp``).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline use it, always as the
checker and never as the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
TABLES_PATH = os.path.join(os.path.dirname(HERE), "gfn1-rs_b200", "data", "gfn1_tables.txt")

ANGSTROM_TO_BOHR = 1.8897261246257702
TERM_NAMES = (
    "total_free", "total_internal", "repulsion", "electronic", "isotropic_scc", "third_order",
    "higher_order", "dispersion", "halogen", "multipole", "exchange", "spin_polarization",
    "plus_u", "external_field", "electronic_entropy",
)


class OracleOptions(ctypes.Structure):
    _fields_ = [
        ("max_scc", ctypes.c_int),
        ("energy_tolerance", ctypes.c_double),
        ("charge_tolerance", ctypes.c_double),
        ("mixing", ctypes.c_double),
        ("scc_broyden", ctypes.c_int),
        ("scc_broyden_size", ctypes.c_int),
        ("electronic_temperature", ctypes.c_double),
        ("enable_dispersion", ctypes.c_int),
        ("charge", ctypes.c_double),
        ("level_shift", ctypes.c_double),
        ("spin_multiplicity", ctypes.c_int),
    ]


def make_options(max_scc=250, energy_tolerance=1e-6, charge_tolerance=2e-5, mixing=0.4,
                 scc_broyden=True, scc_broyden_size=250, electronic_temperature=300.0,
                 enable_dispersion=True, charge=0.0, level_shift=0.0, spin_multiplicity=None) -> OracleOptions:
    """Defaults of ``ElectronicOptions::default`` (src/electronic.rs:395-452);
    spin_multiplicity None is the reference's None."""
    return OracleOptions(int(max_scc), float(energy_tolerance), float(charge_tolerance), float(mixing),
                         int(bool(scc_broyden)), int(scc_broyden_size), float(electronic_temperature),
                         int(bool(enable_dispersion)), float(charge), float(level_shift),
                         int(spin_multiplicity or 0))


class OracleError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


@dataclass
class OracleResult:
    terms: dict
    energy: float
    gradient: np.ndarray | None
    shell_charges: np.ndarray
    atomic_charges: np.ndarray
    orbital_energies: np.ndarray
    occupations: np.ndarray
    dipole: np.ndarray
    coordination_numbers: np.ndarray
    iterations: int
    converged: bool
    fermi_level: float
    rung: int = 0                        # fallback-ladder attempt that converged (0 = the requested scheme)
    electronic_temperature: float = 0.0  # T_el of that attempt (raised on rung 3)
    S: np.ndarray | None = None
    H0: np.ndarray | None = None
    P: np.ndarray | None = None
    W: np.ndarray | None = None
    F: np.ndarray | None = None                  # Fock matrix of the last diagonalisation (matrices=True)
    shell_potential: np.ndarray | None = None    # shell_scc_potential of the final charges (matrices=True)
    extra: dict = field(default_factory=dict)


_lib = None
_lib_lock = threading.Lock()


def build(force: bool = False) -> str:
    """Compile ``liboracle.so`` with the committed Makefile (seconds)."""
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
            os.path.join(HERE, "gfn1_oracle.cpp")):
        subprocess.run(["make", "-C", HERE, "-s", "liboracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    with _lib_lock:  # first use from several threads: load and initialise once
        return _load()


def _load():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_init.argtypes = [ctypes.c_char_p]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_sizes.argtypes = [ctypes.c_int, ip, ip, ip]
        L.oracle_run.argtypes = [ctypes.c_int, ip, dp, ctypes.POINTER(OracleOptions), dp, ctypes.c_int,
                                 dp, dp, dp, dp, dp, dp, dp, dp, ip, ip, dp, dp, dp, dp, dp, ip, dp, dp, dp]
        L.oracle_halogen.argtypes = [ctypes.c_int, ip, dp, dp, dp]
        L.oracle_classical_term.argtypes = [ctypes.c_int, ctypes.c_int, ip, dp, dp, dp]
        L.oracle_run_batch.argtypes = [ctypes.c_int, ip, ip, dp, dp, ctypes.POINTER(OracleOptions), ctypes.c_int,
                                       ctypes.c_int, dp, dp, ip, dp, ip, ip, ip]
        rc = L.oracle_init(TABLES_PATH.encode())
        if rc != 0:
            raise OracleError(rc, L.oracle_last_error().decode())
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def sizes(numbers) -> tuple[int, int]:
    L = lib()
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    nao, nsh = ctypes.c_int(), ctypes.c_int()
    rc = L.oracle_sizes(len(z), _ip(z), ctypes.byref(nao), ctypes.byref(nsh))
    if rc != 0:
        raise OracleError(rc, L.oracle_last_error().decode())
    return nao.value, nsh.value


def run(numbers, positions_bohr, options: OracleOptions | None = None, gradient: bool = True,
        init_shell_charges=None, matrices: bool = False) -> OracleResult:
    """Single point (+ gradient) of one molecule; positions in bohr."""
    L = lib()
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.ascontiguousarray(positions_bohr, dtype=np.float64).reshape(-1, 3)
    nat = len(z)
    nao, nsh = sizes(z)
    opt = options if options is not None else make_options()
    terms = np.zeros(15)
    grad = np.zeros((nat, 3)) if gradient else None
    qsh = np.zeros(nsh)
    qat = np.zeros(nat)
    eps = np.zeros(nao)
    occ = np.zeros(nao)
    dip = np.zeros(3)
    cn = np.zeros(nat)
    it = ctypes.c_int()
    conv = ctypes.c_int()
    fermi = ctypes.c_double()
    rung = ctypes.c_int()
    etemp = ctypes.c_double()
    mats = [np.zeros((nao, nao)) for _ in range(5)] if matrices else [None] * 5
    spot = np.zeros(nsh) if matrices else None
    q0 = None if init_shell_charges is None else np.ascontiguousarray(init_shell_charges, dtype=np.float64)
    rc = L.oracle_run(nat, _ip(z), _dp(xyz), ctypes.byref(opt), _dp(q0), int(gradient), _dp(terms), _dp(grad),
                      _dp(qsh), _dp(qat), _dp(eps), _dp(occ), _dp(dip), _dp(cn), ctypes.byref(it),
                      ctypes.byref(conv), ctypes.byref(fermi), *[_dp(m) for m in mats[:4]], ctypes.byref(rung),
                      ctypes.byref(etemp), _dp(mats[4]), _dp(spot))
    if rc != 0:
        raise OracleError(rc, L.oracle_last_error().decode())
    return OracleResult(terms=dict(zip(TERM_NAMES, terms.tolist())), energy=float(terms[0]), gradient=grad,
                        shell_charges=qsh, atomic_charges=qat, orbital_energies=eps, occupations=occ,
                        dipole=dip, coordination_numbers=cn, iterations=it.value, converged=bool(conv.value),
                        fermi_level=fermi.value, rung=rung.value, electronic_temperature=etemp.value, S=mats[0], H0=mats[1], P=mats[2], W=mats[3],
                        F=mats[4], shell_potential=spot)


def halogen(numbers, positions_bohr, gradient: bool = True):
    """Halogen-bond energy (Eh) and gradient (Eh/bohr) of one molecule."""
    L = lib()
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    x = np.ascontiguousarray(positions_bohr, dtype=np.float64).reshape(-1, 3)
    e = np.zeros(1)
    g = np.zeros((len(z), 3)) if gradient else None
    rc = L.oracle_halogen(len(z), _ip(z), _dp(x), _dp(e), _dp(g))
    if rc != 0:
        raise OracleError(rc, L.oracle_last_error().decode())
    return float(e[0]), g


CLASSICAL_TERMS = ("repulsion", "dispersion", "halogen")


def classical_term(name: str, numbers, positions_bohr, gradient: bool = True):
    """Energy (Eh) and gradient (Eh/bohr) of one classical term alone:
    "repulsion", "dispersion" (D3(BJ)) or "halogen"."""
    L = lib()
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    x = np.ascontiguousarray(positions_bohr, dtype=np.float64).reshape(-1, 3)
    e = np.zeros(1)
    g = np.zeros((len(z), 3)) if gradient else None
    rc = L.oracle_classical_term(CLASSICAL_TERMS.index(name), len(z), _ip(z), _dp(x), _dp(e), _dp(g))
    if rc != 0:
        raise OracleError(rc, L.oracle_last_error().decode())
    return float(e[0]), g


def run_batch(atom_offsets, numbers, positions_bohr, charges=None, options: OracleOptions | None = None,
              gradient: bool = True, nthreads: int = 0, with_rungs: bool = False):
    """Host-thread batch over molecules (one molecule per thread).  Returns
    (energy[nmol], grad[natoms,3], shell_q (concatenated), shell offsets,
    iterations, status), plus the fallback-ladder rung of each molecule (-1
    where it did not converge) with ``with_rungs``."""
    L = lib()
    off = np.ascontiguousarray(atom_offsets, dtype=np.int32)
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    xyz = np.ascontiguousarray(positions_bohr, dtype=np.float64).reshape(-1, 3)
    nmol = len(off) - 1
    shell_off = np.zeros(nmol + 1, dtype=np.int32)
    for m in range(nmol):
        shell_off[m + 1] = shell_off[m] + sizes(z[off[m]:off[m + 1]])[1]
    ch = None if charges is None else np.ascontiguousarray(charges, dtype=np.float64)
    energy = np.zeros(nmol)
    grad = np.zeros_like(xyz)
    qsh = np.zeros(int(shell_off[-1]))
    iters = np.zeros(nmol, dtype=np.int32)
    status = np.zeros(nmol, dtype=np.int32)
    rungs = np.zeros(nmol, dtype=np.int32)
    opt = options if options is not None else make_options()
    L.oracle_run_batch(nmol, _ip(off), _ip(z), _dp(xyz), _dp(ch), ctypes.byref(opt), int(gradient), int(nthreads),
                       _dp(energy), _dp(grad), _ip(shell_off), _dp(qsh), _ip(iters), _ip(status), _ip(rungs))
    if with_rungs:
        return energy, grad, qsh, shell_off, iters, status, rungs
    return energy, grad, qsh, shell_off, iters, status
