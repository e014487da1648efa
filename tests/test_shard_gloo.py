"""Multi-rank host logic on CPU: LPT sharding of a molecule batch and the final
gather, run as two gloo ranks (the same code path bench.py and users take over
NCCL, one process per GPU; the data path itself has no collective)."""
import os
import socket

import numpy as np
import pytest

NAO = np.zeros(87, dtype=np.int64)
NAO[1], NAO[6], NAO[7], NAO[8] = 2, 4, 4, 4


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _per_molecule_work(off, z, x):
    # stand-in for an evaluation: a deterministic per-molecule reduction
    return np.array([[x[off[m]:off[m + 1]].sum(), float(z[off[m]:off[m + 1]].sum())] for m in range(len(off) - 1)])


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from gfn1_rs import shard, workloads
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, z, x = workloads.mixed_batch(40, 300)
        costs = shard.molecule_costs(off, z, NAO)
        parts = shard.lpt_partition(costs, world)
        mine = parts[rank]
        o2, z2, x2, _, _ = shard.take(off, z, x, mine)
        vals = _per_molecule_work(o2, z2, x2)
        full = shard.gather_per_molecule(vals, mine, len(off) - 1)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), full)
    finally:
        dist.destroy_process_group()


def test_lpt_partition_balances_and_covers():
    from gfn1_rs import shard
    rng = np.random.default_rng(0)
    costs = rng.pareto(1.5, size=500) + 1.0
    for world in (1, 2, 3, 8):
        parts = shard.lpt_partition(costs, world)
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(500))
        loads = np.array([costs[p].sum() for p in parts])
        assert loads.max() <= costs.sum() / world + costs.max() + 1e-9


def test_two_gloo_ranks_shard_and_gather(tmp_path):
    import torch.multiprocessing as mp
    from gfn1_rs import workloads
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    off, z, x = workloads.mixed_batch(40, 300)
    ref = _per_molecule_work(off, z, x)
    for r in range(2):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got, ref)
