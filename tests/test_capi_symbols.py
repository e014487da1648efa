"""The engine library loads and exports every function include/gfn1_b200.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def test_library_exports_header_symbols():
    from gfn1_rs import _build

    lib = _build.build()
    header = open(os.path.join(ROOT, "include", "gfn1_b200.h")).read()
    names = sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(gfn1_\w+)\s*\(", header, flags=re.M)))
    assert len(names) >= 12
    L = ctypes.CDLL(lib)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_default_options_match_reference_defaults():
    from gfn1_rs import _lib

    o = _lib.default_options()
    assert (o.max_scc, o.energy_tolerance, o.charge_tolerance, o.mixing) == (250, 1e-6, 2e-5, 0.4)
    assert (o.scc_broyden, o.scc_broyden_size, o.electronic_temperature) == (1, 250, 300.0)
    assert o.enable_dispersion == 1 and o.compute_gradient == 1


def test_tables_regenerate_identically():
    """gfn1_tables.txt equals what gen_tables.py writes from the reference tree."""
    import subprocess
    import sys

    import pytest

    # a gfn1-rs v0.5.1 checkout: GFN1_REFERENCE_ROOT, else a sibling directory
    # named "reference" next to this repository
    ref = os.environ.get("GFN1_REFERENCE_ROOT") or os.path.join(os.path.dirname(ROOT), "reference")
    if not os.path.isdir(ref):
        pytest.skip("reference tree not present (set GFN1_REFERENCE_ROOT)")
    gen = os.path.join(ROOT, "gfn1-rs_b200", "data", "gen_tables.py")
    out = subprocess.run([sys.executable, gen, ref], check=True, capture_output=True, text=True).stdout
    committed = open(os.path.join(ROOT, "gfn1-rs_b200", "data", "gfn1_tables.txt")).read()
    assert out == committed
