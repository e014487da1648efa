"""ctypes binding of the C ABI in include/gfn1_b200.h.

The engine library must exist: there is no CPU fallback.  A missing or
unloadable ``libgfn1_b200.so`` raises ``ImportError``.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from ._build import LIB_PATH, PKG_ROOT

TABLES_PATH = os.path.join(PKG_ROOT, "data", "gfn1_tables.txt")

GFN1_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "Io", 2: "Parse", 3: "InvalidInput", 4: "MissingElement", 5: "MissingGlobal",
    6: "LinearAlgebra", 7: "SingularCell", 8: "SccNotConverged", 9: "Device", 10: "Timeout",
    11: "NonFinite", 12: "Unsupported",
}
TERM_NAMES = (
    "total_free", "total_internal", "repulsion", "electronic", "isotropic_scc", "third_order",
    "higher_order", "dispersion", "halogen", "multipole", "exchange", "spin_polarization",
    "plus_u", "external_field", "electronic_entropy",
)


class Options(ctypes.Structure):
    _fields_ = [
        ("max_scc", ctypes.c_int32),
        ("energy_tolerance", ctypes.c_double),
        ("charge_tolerance", ctypes.c_double),
        ("mixing", ctypes.c_double),
        ("scc_broyden", ctypes.c_int32),
        ("scc_broyden_size", ctypes.c_int32),
        ("electronic_temperature", ctypes.c_double),
        ("enable_dispersion", ctypes.c_int32),
        ("compute_gradient", ctypes.c_int32),
        ("spin_multiplicity", ctypes.c_int32),
        ("level_shift", ctypes.c_double),
    ]


class OptOptions(ctypes.Structure):
    _fields_ = [
        ("max_iterations", ctypes.c_int32),
        ("gradient_tolerance", ctypes.c_double),
        ("step_tolerance", ctypes.c_double),
        ("history", ctypes.c_int32),
        ("initial_step", ctypes.c_double),
        ("max_atom_step", ctypes.c_double),
        ("max_rounds", ctypes.c_int32),
    ]


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class Outputs(ctypes.Structure):
    _fields_ = [
        ("energy", _dp), ("terms", _dp), ("gradient", _dp), ("shell_charges", _dp),
        ("atomic_charges", _dp), ("dipole", _dp), ("fermi_level", _dp), ("iterations", _ip),
        ("status", _ip), ("rung", _ip),
    ]


class Gfn1Error(ValueError):
    """Engine error; ``code`` is the C status (1..8 mirror gfn1-rs Gfn1Error)."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lib = None
_lock = threading.Lock()


def load():
    """Load the engine library (raises ImportError if it was not built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"GFN1 B200 engine library not built: {LIB_PATH} (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.gfn1_default_options.argtypes = [ctypes.POINTER(Options)]
        L.gfn1_default_options.restype = None
        L.gfn1_last_error.argtypes = [vp]
        L.gfn1_last_error.restype = ctypes.c_char_p
        L.gfn1_engine_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]
        L.gfn1_engine_destroy.argtypes = [vp]
        L.gfn1_engine_destroy.restype = None
        L.gfn1_basis_size.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint8), _ip, _ip]
        L.gfn1_run.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint8), _dp, ctypes.c_double, _dp,
                               ctypes.POINTER(Options), ctypes.POINTER(Outputs)]
        L.gfn1_batch_energy_gradient.argtypes = [vp, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_uint8), _dp, _dp, _dp,
                                                 ctypes.POINTER(Options), ctypes.POINTER(Outputs)]
        L.gfn1_batch_create.argtypes = [vp, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_uint8), _dp,
                                        ctypes.POINTER(Options), ctypes.POINTER(vp)]
        L.gfn1_batch_destroy.argtypes = [vp]
        L.gfn1_batch_destroy.restype = None
        L.gfn1_batch_set_positions.argtypes = [vp, vp, ctypes.c_int]
        L.gfn1_batch_set_initial_charges.argtypes = [vp, vp, ctypes.c_int]
        L.gfn1_batch_launch.argtypes = [vp, vp]
        L.gfn1_batch_download.argtypes = [vp, ctypes.POINTER(Outputs)]
        L.gfn1_batch_outputs_device.argtypes = [vp, ctypes.POINTER(Outputs)]
        L.gfn1_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(ctypes.c_int64), _ip]
        L.gfn1_batch_launch_stage.argtypes = [vp, ctypes.c_int, vp]
        L.gfn1_batch_stage_cycles.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int]
        L.gfn1_batch_io_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        L.gfn1_last_wide_plan.argtypes = [vp, _ip, _ip, _ip, _dp, _ip]
        L.gfn1_last_molecule_matrices.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.gfn1_batch_molecule_matrices.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        L.gfn1_last_molecule_fock.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp]
        L.gfn1_default_opt_options.argtypes = [ctypes.POINTER(OptOptions)]
        L.gfn1_default_opt_options.restype = None
        L.gfn1_batch_optimize.argtypes = [vp, ctypes.POINTER(OptOptions), _dp, _dp, _dp, _ip, _ip, _ip, _ip]
        L.gfn1_batch_molecule_fock.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp]
        L.gfn1_run_noalloc.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint8), _dp, ctypes.c_double, _dp,
                                       ctypes.POINTER(Options), ctypes.POINTER(Outputs), vp]
        fp = ctypes.POINTER(ctypes.c_float)
        i64 = ctypes.c_int64
        L.gfn1_guess_param_count.argtypes = []
        L.gfn1_guess_param_count.restype = i64
        L.gfn1_guess_create.argtypes = [vp, fp, i64, ctypes.POINTER(vp)]
        L.gfn1_guess_destroy.argtypes = [vp]
        L.gfn1_guess_destroy.restype = None
        L.gfn1_engine_set_guess.argtypes = [vp, vp]
        L.gfn1_batch_set_guess.argtypes = [vp, vp]
        L.gfn1_guess_features_device.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, vp]
        L.gfn1_guess_infer_device.argtypes = [vp, i64, vp, vp, vp]
        L.gfn1_guess_predict_device.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.gfn1_mlp_gemm.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    vp, ctypes.c_int, vp, ctypes.c_int, vp, vp, ctypes.c_int, vp, vp, ctypes.c_int,
                                    ctypes.c_int, vp]
        L.gfn1_mlp_gemm_splits.argtypes = [ctypes.c_int, ctypes.c_int]
        L.gfn1_mlp_reduce.argtypes = [ctypes.c_int, i64, vp, vp, i64, vp]
        L.gfn1_mlp_colsum.argtypes = [ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.gfn1_mlp_project_loss.argtypes = [ctypes.c_int, vp, vp, vp, vp, ctypes.c_double, vp, vp, vp, vp]
        L.gfn1_mlp_adam.argtypes = [i64, vp, vp, vp, vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_float, vp]
        for name in ("gfn1_guess_create", "gfn1_engine_set_guess", "gfn1_batch_set_guess", "gfn1_guess_features_device",
                     "gfn1_guess_infer_device", "gfn1_guess_predict_device", "gfn1_mlp_gemm", "gfn1_mlp_gemm_splits",
                     "gfn1_mlp_reduce", "gfn1_mlp_colsum", "gfn1_mlp_project_loss", "gfn1_mlp_adam"):
            getattr(L, name).restype = ctypes.c_int
        for name in ("gfn1_last_molecule_matrices", "gfn1_batch_molecule_matrices", "gfn1_run_noalloc",
                     "gfn1_last_molecule_fock", "gfn1_batch_molecule_fock", "gfn1_batch_optimize",
                     "gfn1_batch_launch_stage", "gfn1_batch_stage_cycles", "gfn1_batch_io_bytes", "gfn1_last_wide_plan",
                     "gfn1_engine_create", "gfn1_basis_size", "gfn1_run", "gfn1_batch_energy_gradient",
                     "gfn1_batch_create", "gfn1_batch_set_positions", "gfn1_batch_set_initial_charges",
                     "gfn1_batch_launch", "gfn1_batch_download", "gfn1_batch_outputs_device", "gfn1_batch_info"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
        return L


def last_error(engine_handle=None) -> str:
    return load().gfn1_last_error(engine_handle).decode()


def check(rc: int, handle=None) -> None:
    if rc != GFN1_OK:
        raise Gfn1Error(rc, last_error(handle))


def default_options(**kw) -> Options:
    o = Options()
    load().gfn1_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, type(getattr(o, k))(v))
    return o


def ptr(a: np.ndarray | None, ctype=ctypes.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Engine:
    """Owns a ``gfn1_engine`` (device tables + stream) for one CUDA device."""

    def __init__(self, param_path: str | None = None, device: int = 0):
        L = load()
        spec = TABLES_PATH if param_path in (None, "", "builtin", "builtin:gfn1") else param_path
        h = ctypes.c_void_p()
        check(L.gfn1_engine_create(spec.encode(), int(device), ctypes.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            load().gfn1_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def element_sizes(self) -> tuple[np.ndarray, np.ndarray]:
        """(nao[Z], nshells[Z]) for Z = 0..86; -1 where the device path lacks the element."""
        if getattr(self, "_elem_sizes", None) is None:
            nao = np.full(87, -1, dtype=np.int64)
            nsh = np.full(87, -1, dtype=np.int64)
            L = load()
            a, s = ctypes.c_int32(), ctypes.c_int32()
            for zz in range(1, 87):
                z = np.array([zz], dtype=np.uint8)
                if L.gfn1_basis_size(self.handle, 1, ptr(z, ctypes.c_uint8), ctypes.byref(a), ctypes.byref(s)) == 0:
                    nao[zz], nsh[zz] = a.value, s.value
            self._elem_sizes = (nao, nsh)
        return self._elem_sizes

    def shell_count_table(self) -> np.ndarray:
        """Shells per atom for each uint8 atomic number (0 where the device path
        lacks the element, as the C side counts them)."""
        if getattr(self, "_nsh_u8", None) is None:
            nsh = self.element_sizes()[1]
            table = np.zeros(256, dtype=np.int64)
            table[1:87] = np.maximum(nsh[1:87], 0)
            self._nsh_u8 = table
        return self._nsh_u8

    def basis_size(self, numbers) -> tuple[int, int]:
        z = np.ascontiguousarray(numbers, dtype=np.uint8)
        nao, nsh = ctypes.c_int32(), ctypes.c_int32()
        check(load().gfn1_basis_size(self.handle, len(z), ptr(z, ctypes.c_uint8), ctypes.byref(nao), ctypes.byref(nsh)),
              self.handle)
        return nao.value, nsh.value
