"""Host-side logic of the Python layer that runs before any device call (CPU
only): the reference constructor's option checks, input validation and unit
handling (src/python.rs:116-323, 3216-3252), and the result container's unit
conversions (src/python.rs:2845-2950)."""
import numpy as np
import pytest


@pytest.mark.parametrize("kw", [dict(spin_polarization=True), dict(experimental_d4=True), dict(multipole=True),
                                dict(plus_u=True), dict(hubbard_u=(1.0,)), dict(electric_field=(0.0, 0.0, 0.01)),
                                dict(scc_accelerator="cdiis"), dict(lr_exchange=True)])
def test_off_path_options_are_rejected(kw):
    from gfn1_rs import Gfn1NativeCalculator
    with pytest.raises(ValueError, match="outside the B200 engine"):
        Gfn1NativeCalculator(**kw)


def test_unknown_keyword_and_fixed_options():
    from gfn1_rs import Gfn1NativeCalculator
    with pytest.raises(TypeError, match="unexpected keyword"):
        Gfn1NativeCalculator(no_such_option=1)
    with pytest.raises(ValueError, match="nprim"):
        Gfn1NativeCalculator(nprim=4)
    with pytest.raises(ValueError, match="eigen_tolerance"):
        Gfn1NativeCalculator(eigen_tolerance=1e-10)
    with pytest.raises(ValueError, match="multiplicity"):
        Gfn1NativeCalculator(multiplicity=0)


def test_build_system_validation_and_units():
    from gfn1_rs.native import ANGSTROM_TO_BOHR, build_system, unit_scale
    z, x = build_system([8, 1, 1], [[0, 0, 0], [0.96, 0, 0], [0, 0.96, 0]], "angstrom")
    assert z.dtype == np.uint8 and z.tolist() == [8, 1, 1]
    assert np.allclose(x[1], [0.96 * ANGSTROM_TO_BOHR, 0, 0], rtol=0, atol=1e-15)
    _, xb = build_system([1], [[1.0, 2.0, 3.0]], "bohr")
    assert xb.tolist() == [[1.0, 2.0, 3.0]]
    assert unit_scale("au") == 1.0 and unit_scale("A") == ANGSTROM_TO_BOHR
    with pytest.raises(ValueError, match="unit"):
        unit_scale("nm")
    with pytest.raises(ValueError, match="length"):
        build_system([1, 1], [[0, 0, 0]], "bohr")
    with pytest.raises(ValueError, match="expected 3"):
        build_system([1], [[0, 0]], "bohr")
    with pytest.raises(ValueError, match="u8"):
        build_system([256], [[0, 0, 0]], "bohr")


def test_calculation_result_conversions():
    from gfn1_rs import TERM_NAMES
    from gfn1_rs.native import FORCE_HARTREE_PER_BOHR_TO_EV_PER_ANGSTROM, HARTREE_TO_EV, CalculationResult
    g = np.array([[0.01, -0.02, 0.0], [-0.01, 0.02, 0.0]])
    terms = np.arange(15, dtype=np.float64)
    r = CalculationResult(-1.5, terms, g, [0.1, -0.1], [0.0, 0.0, 0.5], 7, True, fermi_level=-0.3)
    assert r.energy_ev == pytest.approx(-1.5 * HARTREE_TO_EV, rel=1e-15)
    assert np.allclose(r.forces_ev_per_angstrom, -g * FORCE_HARTREE_PER_BOHR_TO_EV_PER_ANGSTROM, rtol=1e-15)
    assert r.stress is None and r.iterations == 7 and r.converged
    assert list(r.energy_terms_hartree()) == list(TERM_NAMES)
    assert r.energy_terms_ev()["repulsion"] == pytest.approx(2.0 * HARTREE_TO_EV)
    r0 = CalculationResult(-1.5, terms, None, [0.0], [0, 0, 0], 1, False)
    assert r0.gradient_hartree_per_bohr is None and r0.forces_ev_per_angstrom is None


def test_periodic_entry_point_raises_value_error():
    from gfn1_rs import Gfn1NativeCalculator
    with pytest.raises(ValueError, match="periodic"):
        Gfn1NativeCalculator.calculate_periodic(None, [1, 1], [[0, 0, 0], [0.74, 0, 0]])
