"""gfn1_run_noalloc: the entry point for callers that cannot allocate device or
pinned memory (a memory manager owns all of it, or allocation is forbidden in
the loop).  Its scratch is a fixed library array, so two calls in a row reuse
the same memory; both must match gfn1_run, the allocating entry point.

This file sorts last so a fail-fast run has executed every other test first;
it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, smoke_molecule

pytestmark = pytest.mark.gpu

E_TOL, G_TOL, Q_TOL = 1e-8, 1e-7, 1e-7


def _outputs(nat, nsh):
    from gfn1_rs import _lib

    arrs = dict(energy=np.zeros(1), terms=np.zeros(15), gradient=np.zeros((nat, 3)), shell=np.zeros(nsh),
                atom=np.zeros(nat), dipole=np.zeros(3), fermi=np.zeros(1), iters=np.zeros(1, np.int32),
                status=np.zeros(1, np.int32))
    out = _lib.Outputs(_lib.ptr(arrs["energy"]), _lib.ptr(arrs["terms"]), _lib.ptr(arrs["gradient"]),
                       _lib.ptr(arrs["shell"]), _lib.ptr(arrs["atom"]), _lib.ptr(arrs["dipole"]),
                       _lib.ptr(arrs["fermi"]), _lib.ptr(arrs["iters"], ctypes.c_int32),
                       _lib.ptr(arrs["status"], ctypes.c_int32))
    return out, arrs


def _call(fn_name, engine, z, x, opt, charge=0.0):
    from gfn1_rs import _lib

    L = _lib.load()
    z8 = np.ascontiguousarray(z, dtype=np.uint8)
    xb = np.ascontiguousarray(x, dtype=np.float64)
    nat = len(z8)
    nsh = engine.basis_size(z8)[1]
    out, arrs = _outputs(nat, nsh)
    args = [engine.handle, nat, _lib.ptr(z8, ctypes.c_uint8), _lib.ptr(xb), float(charge), None, ctypes.byref(opt),
            ctypes.byref(out)]
    if fn_name == "gfn1_run_noalloc":
        args.append(None)
    rc = getattr(L, fn_name)(*args)
    return rc, arrs


@pytest.fixture(scope="module")
def engine():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gfn1_rs import _lib

    return _lib.Engine()


def test_noalloc_matches_allocating_entry_point_twice(engine, fixtures):
    from gfn1_rs import _lib, workloads

    opt = _lib.default_options()
    cases = [smoke_molecule(fixtures, "caffeine")]
    z, x = workloads.water_cluster(16, 0)
    cases.append((z, x * ANGSTROM_TO_BOHR))  # 48 atoms, 128 AOs: at the size limit
    for z, x in cases:
        rc, ref = _call("gfn1_run", engine, z, x, opt)
        assert rc == 0, _lib.last_error()
        for _ in range(2):  # the second call reuses the scratch left by the first
            rc, got = _call("gfn1_run_noalloc", engine, z, x, opt)
            assert rc == 0, _lib.last_error()
            assert abs(got["energy"][0] - ref["energy"][0]) <= E_TOL
            assert np.max(np.abs(got["terms"] - ref["terms"])) <= E_TOL
            assert np.max(np.abs(got["gradient"] - ref["gradient"])) <= G_TOL
            assert np.max(np.abs(got["shell"] - ref["shell"])) <= Q_TOL
            assert got["iters"][0] == ref["iters"][0] and got["status"][0] == 0


def _assert_same(got, ref):
    assert abs(got["energy"][0] - ref["energy"][0]) <= E_TOL
    assert np.max(np.abs(got["terms"] - ref["terms"])) <= E_TOL
    assert np.max(np.abs(got["gradient"] - ref["gradient"])) <= G_TOL
    assert np.max(np.abs(got["shell"] - ref["shell"])) <= Q_TOL
    assert got["iters"][0] == ref["iters"][0] and got["status"][0] == ref["status"][0]


@pytest.mark.parametrize("case", ["ferrocene", "CH3Br...OH2 halogen bond", "NH3+ doublet"])
def test_noalloc_d_shells_halogen_and_spin(engine, fixtures, case):
    """d shells (ferrocene), the halogen-bond term (CH3Br...OH2, which converges
    on the requested scheme; C-Br...O needs the fallback ladder, which this
    entry point does not run) and a charged doublet with a requested spin
    multiplicity, each twice in a row, against the allocating entry point."""
    from gfn1_rs import _lib

    charge, kw = 0.0, {}
    if case == "ferrocene":
        z, x = smoke_molecule(fixtures, case)
    elif case == "CH3Br...OH2 halogen bond":
        rec = fixtures["halogen_tests"][case]
        z, x = np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR
    else:  # NH3+ radical cation, spin multiplicity 2
        z = np.array([7, 1, 1, 1])
        x = np.array([[0.0, 0.0, 0.0], [0.0, 0.94, 0.38], [0.81, -0.47, 0.38], [-0.81, -0.47, 0.38]]) * ANGSTROM_TO_BOHR
        charge, kw = 1.0, dict(spin_multiplicity=2)
    opt = _lib.default_options(**kw)
    rc, ref = _call("gfn1_run", engine, z, x, opt, charge)
    assert rc == 0, _lib.last_error()
    for _ in range(2):
        rc, got = _call("gfn1_run_noalloc", engine, z, x, opt, charge)
        assert rc == 0, _lib.last_error()
        _assert_same(got, ref)


def test_noalloc_reports_unconverged_scc(engine, fixtures):
    """max_scc = 1 cannot pass the convergence test (its first energy change is
    infinite): status GFN1_E_SCC_NOT_CONVERGED, as from gfn1_run's rung 0."""
    from gfn1_rs import _lib

    z, x = smoke_molecule(fixtures, "caffeine")
    opt = _lib.default_options(max_scc=1)
    for _ in range(2):
        rc, got = _call("gfn1_run_noalloc", engine, z, x, opt)
        assert rc == 8, _lib.last_error()
        assert got["status"][0] == 8 and got["iters"][0] == 1
        assert "did not converge" in _lib.last_error()


def test_noalloc_uses_the_engines_learned_guess(fixtures):
    """With a learned guess set on the engine, both entry points start from the
    predicted charges: same iteration count and results."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gfn1_rs import _lib
    from gfn1_rs.guess import LearnedGuess

    eng = _lib.Engine()
    guess = LearnedGuess.from_file(eng)
    L = _lib.load()
    _lib.check(L.gfn1_engine_set_guess(eng.handle, guess.handle), eng.handle)
    try:
        from gfn1_rs import workloads

        z, x = workloads.water_cluster(8, 3)  # the kind of molecule the guess was trained on
        x = x * ANGSTROM_TO_BOHR
        opt = _lib.default_options()
        rc, ref = _call("gfn1_run", eng, z, x, opt)
        assert rc == 0, _lib.last_error()
        rc0, plain = _call("gfn1_run_noalloc", _lib.Engine(), z, x, opt)
        assert rc0 == 0
        for _ in range(2):
            rc, got = _call("gfn1_run_noalloc", eng, z, x, opt)
            assert rc == 0, _lib.last_error()
            _assert_same(got, ref)
        assert ref["iters"][0] <= plain["iters"][0]  # the predicted start is no worse than zero charges
    finally:
        L.gfn1_engine_set_guess(eng.handle, None)
        guess.close()


def test_noalloc_keeps_the_callers_device(engine, fixtures):
    import torch

    from gfn1_rs import _lib

    before = torch.cuda.current_device()
    z, x = smoke_molecule(fixtures, "water")
    rc, _ = _call("gfn1_run_noalloc", engine, z, x, _lib.default_options())
    assert rc == 0, _lib.last_error()
    assert torch.cuda.current_device() == before


def test_noalloc_rejects_oversize_molecule(engine):
    from gfn1_rs import _lib, workloads

    z, x = workloads.water_cluster(24, 0)  # 72 atoms > 64
    rc, _ = _call("gfn1_run_noalloc", engine, z, x * ANGSTROM_TO_BOHR, _lib.default_options())
    assert rc == 3
    assert "at most 64 atoms" in _lib.last_error()
