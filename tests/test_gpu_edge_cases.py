"""Edge cases of the batch path against the oracle: an empty molecule inside a
batch, coincident atoms (overlap not positive definite), a bare proton (no
electrons), dispersion off, T_el = 0 (aufbau), non-finite coordinates."""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR

pytestmark = pytest.mark.gpu

W = np.array([[0.0, 0.0, 0.1173], [0.0, 0.7572, -0.4692], [0.0, -0.7572, -0.4692]]) * ANGSTROM_TO_BOHR


def test_empty_molecule_in_a_batch(gpu_calc):
    off = np.array([0, 3, 3, 6], dtype=np.int32)  # molecule 1 has no atoms
    z = np.array([8, 1, 1, 8, 1, 1])
    x = np.concatenate([W, W + 10.0])
    r = gpu_calc.calculate_flat(off, z, x)
    assert r.status.tolist() == [0, 3, 0]
    single = gpu_calc.calculate_flat([0, 3], z[:3], W)
    assert abs(r.energy[0] - single.energy[0]) < 1e-12 and abs(r.energy[2] - single.energy[0]) < 1e-10


def test_coincident_atoms_are_rejected(gpu_calc, oracle_mod):
    z = [8, 1, 1]
    x = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 1.4, 0.0]])
    with pytest.raises(oracle_mod.OracleError) as ei:
        oracle_mod.run(z, x)
    r = gpu_calc.calculate_flat([0, 3], z, x)
    assert ei.value.code == 3 and r.status[0] == 3


@pytest.mark.parametrize("case", ["proton", "no dispersion", "aufbau"])
def test_option_cases_match_oracle(gpu_calc, oracle_mod, case):
    from gfn1_rs import BatchCalculator

    z, x, ch, kw = {"proton": ([1], np.zeros((1, 3)), 1.0, {}),
                    "no dispersion": ([8, 1, 1], W, 0.0, {"enable_dispersion": False}),
                    "aufbau": ([8, 1, 1], W, 0.0, {"electronic_temperature": 0.0})}[case]
    r = BatchCalculator(**kw).calculate_flat([0, len(z)], z, x, charges=[ch], raise_on_error=True)
    o = oracle_mod.run(z, x, options=oracle_mod.make_options(charge=ch, **kw))
    assert abs(r.energy[0] - o.energy) <= 1e-6
    assert np.max(np.abs(r.gradient - o.gradient)) <= 1e-5
    if case == "no dispersion":
        assert r.terms[0, 7] == 0.0


def test_non_finite_coordinates_raise(gpu_calc):
    from gfn1_rs import Gfn1Error

    x = W.copy()
    x[1, 2] = np.nan
    with pytest.raises(Gfn1Error):
        gpu_calc.calculate_flat([0, 3], [8, 1, 1], x)
