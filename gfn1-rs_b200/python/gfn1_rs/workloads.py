"""Seeded synthetic molecular clusters for tests and benchmarks.

All generators use numpy ``default_rng(seed)`` (PCG64) and return coordinates in
Angstrom.  Monomer geometries: rigid H2O (r_OH = 0.9572 A, HOH = 104.52 deg),
NH3 (r_NH = 1.012 A, HNH = 106.7 deg) and CH4 (r_CH = 1.087 A, tetrahedral).
Monomer orientations are uniform random rotations (random unit quaternions);
centres are uniform in a cube, and a placement is rejected when a heavy atom
would come closer than 2.6 A to a heavy atom already placed.

Workloads:
* ``water_cluster(n, seed)``: n waters at 1.0 g/cm^3 (cube side
  (n * 18.015 / N_A / 1.0)^(1/3)); 16 waters with seed 0 give a 48-atom,
  128-AO cluster; 300 waters with seed 1 give 900 atoms, 2400 AOs.
* ``mixed_batch(nmol, seed0)``: molecule i uses seed seed0 + i, k ~ U{1..15}
  monomers drawn uniformly from H2O/NH3/CH4, a cube of 30 A^3 per monomer and
  N(0, 0.05 A) per-atom jitter: 3-75 atoms, 8-180 AOs.
* ``water_trajectory(n, frames, seed, vseed)``: free flight of n waters from
  Maxwell-Boltzmann velocities at 300 K, 0.5 fs per frame plus N(0, 0.002 A)
  noise.
"""
from __future__ import annotations

import math

import numpy as np

N_A = 6.02214076e23
AMU_KG = 1.66053906660e-27
KB_SI = 1.380649e-23
MASS = {1: 1.008, 6: 12.011, 7: 14.007, 8: 15.999}


def _water():
    r, ang = 0.9572, math.radians(104.52)
    h1 = [r * math.sin(ang / 2), r * math.cos(ang / 2), 0.0]
    h2 = [-r * math.sin(ang / 2), r * math.cos(ang / 2), 0.0]
    return [8, 1, 1], np.array([[0.0, 0.0, 0.0], h1, h2])


def _ammonia():
    r, ang = 1.012, math.radians(106.7)
    # H atoms on a cone around z; the H-N-H angle fixes the cone angle
    s = math.sqrt((1.0 - math.cos(ang)) / 1.5)  # sin of the cone half-angle
    c = math.sqrt(max(0.0, 1.0 - s * s))
    hs = [[r * s * math.cos(2 * math.pi * k / 3), r * s * math.sin(2 * math.pi * k / 3), -r * c] for k in range(3)]
    return [7, 1, 1, 1], np.array([[0.0, 0.0, 0.0]] + hs)


def _methane():
    r = 1.087 / math.sqrt(3.0)
    hs = [[r, r, r], [-r, -r, r], [-r, r, -r], [r, -r, -r]]
    return [6, 1, 1, 1, 1], np.array([[0.0, 0.0, 0.0]] + hs)


MONOMERS = {"H2O": _water(), "NH3": _ammonia(), "CH4": _methane()}
MONOMER_ORDER = ("H2O", "NH3", "CH4")


def random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def pack_monomers(kinds, box: float, rng, min_heavy: float = 2.6, max_tries: int = 200000):
    """Random sequential placement with rejection; returns (numbers, xyz_angstrom, rejects)."""
    numbers, coords, heavy = [], [], []
    rejects = 0
    for kind in kinds:
        z, geo = MONOMERS[kind]
        for _ in range(max_tries):
            centre = rng.uniform(0.0, box, size=3)
            if heavy and np.min(np.linalg.norm(np.asarray(heavy) - centre, axis=1)) < min_heavy:
                rejects += 1
                continue
            rot = random_rotation(rng)
            numbers.extend(z)
            coords.extend((geo @ rot.T) + centre)
            heavy.append(centre)
            break
        else:
            raise RuntimeError(f"could not place monomer {kind} after {max_tries} tries")
    return np.asarray(numbers, dtype=np.int64), np.asarray(coords), rejects


def water_box_side(n: int, density_g_cm3: float = 1.0) -> float:
    mass_g = n * 18.015 / N_A
    return (mass_g / density_g_cm3 * 1e24) ** (1.0 / 3.0)


def water_cluster(n: int = 16, seed: int = 0):
    rng = np.random.default_rng(seed)
    numbers, xyz, rejects = pack_monomers(["H2O"] * n, water_box_side(n), rng)
    return numbers, xyz


def mixed_molecule(seed: int, vol_per_monomer: float = 30.0, jitter: float = 0.05):
    rng = np.random.default_rng(seed)
    k = int(rng.integers(1, 16))
    kinds = [MONOMER_ORDER[int(i)] for i in rng.integers(0, 3, size=k)]
    box = (vol_per_monomer * k) ** (1.0 / 3.0)
    numbers, xyz, _ = pack_monomers(kinds, box, rng)
    xyz = xyz + rng.normal(0.0, jitter, size=xyz.shape)
    return numbers, xyz


def mixed_batch(nmol: int = 4096, seed0: int = 1000):
    """Flat arrays (atom_offsets, numbers, xyz_angstrom) of nmol molecules."""
    offs = [0]
    zs, xs = [], []
    for i in range(nmol):
        z, x = mixed_molecule(seed0 + i)
        zs.append(z)
        xs.append(x)
        offs.append(offs[-1] + len(z))
    return np.asarray(offs, dtype=np.int32), np.concatenate(zs), np.concatenate(xs)


def water_trajectory(n: int = 96, frames: int = 2000, seed: int = 2, vseed: int = 3, dt_fs: float = 0.5,
                     noise: float = 0.002, temperature: float = 300.0):
    """Frames of a free-flight water cluster; returns (numbers, xyz[frames, nat, 3])."""
    numbers, xyz0 = water_cluster(n, seed)
    vrng = np.random.default_rng(vseed)
    masses = np.array([MASS[int(z)] for z in numbers]) * AMU_KG
    sigma = np.sqrt(KB_SI * temperature / masses)  # m/s per Cartesian component
    vel = vrng.normal(size=(len(numbers), 3)) * sigma[:, None] * 1e10 * 1e-15  # A per fs
    out = np.empty((frames, len(numbers), 3))
    x = xyz0.copy()
    for f in range(frames):
        out[f] = x
        x = x + vel * dt_fs + vrng.normal(0.0, noise, size=x.shape)
    return numbers, out
