"""Multi-rank host logic on CPU, run as two gloo ranks (the same code paths
bench.py, the guess trainer and users take over NCCL, one process per GPU):

* LPT sharding of a molecule batch and the final gather, with each rank
  evaluating its shard with the CPU oracle: the gathered energies, gradients
  and shell charges equal the single-rank evaluation bit for bit;
* the data-parallel gradient of the guess trainer (allreduce_weighted): each
  rank's gradient of its own batch, weighted by its shells and summed over
  the ranks, equals the gradient of the union batch on one rank."""
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


def _oracle_rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import oracle
    from gfn1_rs import shard, workloads
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, z, x = workloads.mixed_batch(12, 500)
        xb = x * 1.8897261246257702
        parts = shard.lpt_partition(shard.molecule_costs(off, z, NAO), world)
        mine = parts[rank]
        o2, z2, x2, _, _ = shard.take(off, z, xb, mine)
        e, g, q, shoff, it, st = oracle.run_batch(o2, z2, x2, nthreads=1)
        nm = len(mine)
        grads = np.empty(nm, dtype=object)
        shells = np.empty(nm, dtype=object)
        for k in range(nm):
            grads[k] = g[o2[k]:o2[k + 1]].copy()
            shells[k] = q[shoff[k]:shoff[k + 1]].copy()
        n = len(off) - 1
        out = {"energy": shard.gather_per_molecule(e, mine, n), "status": shard.gather_per_molecule(st, mine, n),
               "gradient": shard.gather_per_molecule(grads, mine, n),
               "shell_q": shard.gather_per_molecule(shells, mine, n)}
        np.save(os.path.join(out_dir, f"oracle_rank{rank}.npy"), out, allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_evaluate_shards_and_gather(tmp_path):
    import oracle
    import torch.multiprocessing as mp
    from gfn1_rs import workloads
    port = _free_port()
    mp.start_processes(_oracle_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    off, z, x = workloads.mixed_batch(12, 500)
    e, g, q, shoff, it, st = oracle.run_batch(off, z, x * 1.8897261246257702, nthreads=1)
    assert np.all(st == 0)
    for r in range(2):
        got = np.load(tmp_path / f"oracle_rank{r}.npy", allow_pickle=True).item()
        assert np.array_equal(got["energy"], e) and np.all(got["status"] == 0)
        for m in range(len(off) - 1):
            assert np.array_equal(got["gradient"][m], g[off[m]:off[m + 1]])
            assert np.array_equal(got["shell_q"][m], q[shoff[m]:shoff[m + 1]])


def _dp_batch(seed):
    import guess_oracle as go
    from gfn1_rs import workloads
    off, z, x = workloads.mixed_batch(10, seed)
    xb = x * 1.8897261246257702
    d = go.descriptors(off, z, xb)
    mean, std = d.mean(0), d.std(0) + 1e-3
    labels = np.random.default_rng(seed).normal(0.0, 0.3, size=(len(z), 2))
    return off, z, xb, d, mean, std, labels


def _flat_grad(g):
    return np.concatenate([np.ravel(g[k]) for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")])


def _dp_rank_main(rank, world, port, out_dir):
    import guess_oracle as go
    import torch
    import torch.distributed as dist
    from gfn1_rs import shard
    from gfn1_rs.guess import allreduce_weighted, shard_training_set
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        off, z, xb, d, mean, std, labels = _dp_batch(3)
        mine = shard_training_set(len(off) - 1, rank, world, seed=7)
        o2, z2, x2, _, atoms = shard.take(off, z, xb, mine)
        p = go.init_params(1)
        xf = go.features(d[atoms], z2, mean, std)
        _, g = go.loss_and_grad(p, xf, o2, z2, np.zeros(len(mine)), labels[atoms])
        grad = torch.tensor(_flat_grad(g), dtype=torch.float64)
        nsh = torch.tensor([2.0 * len(atoms)], dtype=torch.float64)
        tot = nsh.clone()
        dist.all_reduce(tot)
        allreduce_weighted(grad, float(nsh.item()), float(tot.item()))
        np.save(os.path.join(out_dir, f"dp_rank{rank}.npy"), grad.numpy())
    finally:
        dist.destroy_process_group()


def test_data_parallel_guess_gradients_equal_single_rank(tmp_path):
    import guess_oracle as go
    import torch.multiprocessing as mp
    from gfn1_rs import shard
    from gfn1_rs.guess import shard_training_set
    port = _free_port()
    mp.start_processes(_dp_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    off, z, xb, d, mean, std, labels = _dp_batch(3)
    union = np.sort(np.concatenate([shard_training_set(len(off) - 1, r, 2, seed=7) for r in range(2)]))
    o2, z2, x2, _, atoms = shard.take(off, z, xb, union)
    _, g = go.loss_and_grad(go.init_params(1), go.features(d[atoms], z2, mean, std), o2, z2, np.zeros(len(union)),
                            labels[atoms])
    ref = _flat_grad(g)
    for r in range(2):
        got = np.load(tmp_path / f"dp_rank{r}.npy")
        assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, np.abs(ref).max())

