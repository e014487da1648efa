"""Sharding a batch of independent molecules over ranks (one process per GPU).

Molecules are independent, so the data path needs no collective: each rank
evaluates its own shard, and results are gathered once at the end.  Shards are
balanced by greedy longest-processing-time (LPT) assignment on a cost model of
the SCC stage, iterations x 12 N^3, plus the pair work of the integrals.
"""
from __future__ import annotations

import heapq

import numpy as np


def molecule_costs(atom_offsets, numbers, nao_of_z, iterations: float = 8.0) -> np.ndarray:
    """Relative cost per molecule: iterations * 12 N^3 + 160 * nat^2 (pair work)."""
    off = np.asarray(atom_offsets, dtype=np.int64)
    nao = np.asarray(nao_of_z)[np.asarray(numbers, dtype=np.int64)]
    cum = np.concatenate([[0], np.cumsum(nao)])
    n = (cum[off[1:]] - cum[off[:-1]]).astype(np.float64)
    nat = np.diff(off).astype(np.float64)
    return iterations * 12.0 * n ** 3 + 160.0 * nat ** 2


def lpt_partition(costs, world: int) -> list[np.ndarray]:
    """Molecule indices per rank; each list is sorted ascending."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for m in np.argsort(-costs, kind="stable"):
        load, r = heapq.heappop(heap)
        parts[r].append(int(m))
        heapq.heappush(heap, (load + float(costs[m]), r))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def take(atom_offsets, numbers, xyz, index, charges=None):
    """Flat arrays of the molecules in `index` (in that order)."""
    off = np.asarray(atom_offsets, dtype=np.int64)
    xyz = np.asarray(xyz).reshape(-1, 3)
    counts = off[np.asarray(index) + 1] - off[np.asarray(index)]
    new_off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    atoms = (np.concatenate([np.arange(off[i], off[i + 1]) for i in index]) if len(index)
             else np.zeros(0, dtype=np.int64))
    ch = None if charges is None else np.asarray(charges)[np.asarray(index)]
    return new_off, np.asarray(numbers)[atoms], xyz[atoms], ch, atoms


def gather_per_molecule(values: np.ndarray, index: np.ndarray, nmol: int, group=None) -> np.ndarray | None:
    """Collects per-molecule rows from every rank into the original order on
    every rank (all_gather of Python objects; once per batch, not per step)."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    got = [None] * world
    dist.all_gather_object(got, (np.asarray(index), np.asarray(values)), group=group)
    first = np.asarray(got[0][1])
    out = np.zeros((nmol,) + first.shape[1:], dtype=first.dtype)
    seen = np.zeros(nmol, dtype=bool)
    for idx, vals in got:
        out[idx] = vals
        seen[idx] = True
    if not seen.all():
        raise RuntimeError("gathered shards do not cover every molecule")
    return out
