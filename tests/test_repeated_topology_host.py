"""Host side of repeated-topology calls (CPU only): BatchCalculator.calculate_flat
reuses the shell offsets while the atom offsets and atomic numbers repeat,
recomputes them as soon as either changes (also when the caller mutates its
own arrays in place between calls), hands the C entry point the current
topology every time, and returns offsets that neither the caller nor a later
call can change.  The engine's batched entry point is replaced by a fake that
records what it receives; the real library's host-only functions (defaults of
the options) are used as they are."""
import ctypes

import numpy as np
import pytest


class _FakeEngine:
    handle = None

    def __init__(self):
        self.table_calls = 0
        self.table = np.zeros(256, dtype=np.int64)
        self.table[1], self.table[6], self.table[8] = 1, 2, 3  # distinct shell counts per element

    def shell_count_table(self):
        self.table_calls += 1
        return self.table


class _FakeLib:
    """Proxies the real library, except the batched entry point."""

    def __init__(self, real):
        self.real = real
        self.seen = []

    def __getattr__(self, name):
        return getattr(self.real, name)

    def gfn1_batch_energy_gradient(self, handle, nmol, off_p, z_p, xyz_p, ch_p, q0_p, opt_ref, out_ref):
        off = np.ctypeslib.as_array(off_p, shape=(nmol + 1,)).copy()
        z = np.ctypeslib.as_array(z_p, shape=(int(off[-1]),)).copy()
        self.seen.append((off, z))
        out = out_ref._obj
        for m in range(nmol):
            out.energy[m] = float(m) + 0.5
            out.status[m] = 0
        return 0


@pytest.fixture()
def calc(monkeypatch):
    from gfn1_rs import _lib
    from gfn1_rs.batch import BatchCalculator

    fake = _FakeLib(_lib.load())
    monkeypatch.setattr(_lib, "load", lambda: fake)
    c = object.__new__(BatchCalculator)  # no device: the engine is the fake above
    c.engine = _FakeEngine()
    c.guess = None
    c.opts = {}
    c._last = None
    c._last_shoff = None
    return c, fake


def test_shell_offsets_reused_while_the_topology_repeats(calc):
    c, fake = calc
    off = np.array([0, 3, 5], dtype=np.int32)
    z = np.array([8, 1, 1, 6, 1], dtype=np.uint8)
    x = np.zeros((5, 3))
    r1 = c.calculate_flat(off, z, x)
    assert r1.shell_offsets.tolist() == [0, 5, 8]
    r2 = c.calculate_flat(off.copy(), z.copy(), x + 0.1)  # equal arrays, other objects
    assert c.engine.table_calls == 1
    assert r2.shell_offsets is r1.shell_offsets
    assert r2.energy.tolist() == [0.5, 1.5]
    for seen_off, seen_z in fake.seen:
        assert seen_off.tolist() == off.tolist() and seen_z.tolist() == z.tolist()


def test_changed_topology_is_picked_up(calc):
    c, fake = calc
    off = np.array([0, 3, 5], dtype=np.int32)
    z = np.array([8, 1, 1, 6, 1], dtype=np.uint8)
    x = np.zeros((5, 3))
    c.calculate_flat(off, z, x)
    z[3] = 8  # the caller mutates its own array in place
    r = c.calculate_flat(off, z, x)
    assert c.engine.table_calls == 2
    assert r.shell_offsets.tolist() == [0, 5, 9]
    assert fake.seen[-1][1].tolist() == [8, 1, 1, 8, 1]
    off2 = np.array([0, 2, 5], dtype=np.int32)  # same atoms, other molecule boundaries
    r = c.calculate_flat(off2, z, x)
    assert c.engine.table_calls == 3
    assert r.shell_offsets.tolist() == [0, 4, 9]
    assert fake.seen[-1][0].tolist() == [0, 2, 5]


def test_returned_offsets_are_read_only_copies(calc):
    c, _ = calc
    off = np.array([0, 3], dtype=np.int32)
    z = np.array([8, 1, 1], dtype=np.uint8)
    r = c.calculate_flat(off, z, np.zeros((3, 3)))
    assert r.atom_offsets is not off
    with pytest.raises(ValueError):
        r.atom_offsets[0] = 1
    with pytest.raises(ValueError):
        r.shell_offsets[0] = 1
    off[1] = 2  # the caller's array stays its own
    assert r.atom_offsets.tolist() == [0, 3]
