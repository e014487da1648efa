"""bench.py's roofline inputs on the CPU: the algorithmic FP64 work of the SCC
kernel is the stated per-molecule formula, and the DRAM traffic per launch is
read from the committed profile summary."""
import sys

import numpy as np

from conftest import ROOT

if ROOT not in sys.path:
    sys.path.insert(0, ROOT)  # bench.py sits at the repository root


def test_scc_flops_formula():
    import bench

    nao_z = np.zeros(87, dtype=np.int64)
    nsh_z = np.zeros(87, dtype=np.int64)
    nao_z[1], nsh_z[1] = 2, 2          # H: 1s, 2s
    nao_z[6:9], nsh_z[6:9] = 4, 2      # C, N, O: 2s, 2p
    z = np.array([8, 1, 1, 6, 1, 1, 1, 1])  # H2O (N 8, nsh 6) and CH4 (N 12, nsh 10)
    off = np.array([0, 3, 8])
    iters = np.array([5.0, 7.0])
    want = (5 * (12 * 8 ** 3 + 2 * 8 ** 2 + 2 * 6 ** 2) + 14 * 8 ** 3
            + 7 * (12 * 12 ** 3 + 2 * 12 ** 2 + 2 * 10 ** 2) + 14 * 12 ** 3)
    assert bench.scc_flops(off, z, iters, nao_z, nsh_z) == want


def test_traffic_from_profile_summary():
    import bench

    t = bench.read_traffic()
    assert t is not None and t > 0
