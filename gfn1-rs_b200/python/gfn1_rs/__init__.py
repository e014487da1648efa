"""B200 GFN1-xTB engine: drop-in for gfn1-rs's non-periodic SCC energy + gradient.

``Gfn1NativeCalculator`` keeps the reference's Python entry point
(``gfn1_rs.Gfn1NativeCalculator``, python/gfn1_rs/native.py:53-64 of gfn1-rs);
``BatchCalculator`` adds batched evaluation of many molecules.
"""
from .native import (  # noqa: F401
    ANGSTROM_TO_BOHR,
    BOHR_TO_ANGSTROM,
    FORCE_HARTREE_PER_BOHR_TO_EV_PER_ANGSTROM,
    HARTREE_TO_EV,
    CalculationResult,
    Gfn1NativeCalculator,
)
from .batch import BatchCalculator, BatchResult, ResidentBatch  # noqa: F401
from ._lib import Gfn1Error, TERM_NAMES  # noqa: F401


def default_param_path() -> str:
    """The bundled tables (the reference returns GFN1_XTB_PARAM or "builtin")."""
    return "builtin"
