import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gfn1-rs_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

ANGSTROM_TO_BOHR = 1.8897261246257702
GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_fixtures.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def fixtures():
    with open(GOLDEN) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


def smoke_molecule(fixtures, name):
    rec = fixtures["nonpbc_smoke"][name]
    return np.array(rec["numbers"]), np.array(rec["positions_angstrom"]) * ANGSTROM_TO_BOHR


@pytest.fixture(scope="session")
def gpu_calc():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gfn1_rs import BatchCalculator

    return BatchCalculator()
