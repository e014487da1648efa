"""Engines on different host threads run concurrently (the C ABI is reentrant
per engine handle; ctypes releases the GIL around each call): results equal
the same calls made one after another."""
import threading

import numpy as np
import pytest

A2B = 1.8897261246257702
pytestmark = pytest.mark.gpu


def test_concurrent_engines_match_sequential(gpu_calc):
    from gfn1_rs import BatchCalculator, workloads

    batches = []
    for t in range(3):
        off, z, x = workloads.mixed_batch(96, 5000 + 100 * t)
        batches.append((off, z, x * A2B))
    calcs = [BatchCalculator() for _ in batches]
    ref = [c.calculate_flat(*b) for c, b in zip(calcs, batches)]
    out = [None] * len(batches)
    errors = []

    def work(i):
        try:
            for _ in range(3):
                out[i] = calcs[i].calculate_flat(*batches[i])
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(batches))]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not errors, errors
    for r, o in zip(ref, out):
        assert np.all(o.status == 0)
        assert np.array_equal(r.energy, o.energy)
        assert np.array_equal(r.gradient, o.gradient)
