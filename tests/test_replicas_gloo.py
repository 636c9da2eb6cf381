"""Several-GPU host logic on CPU: molecule partitioning and the step reductions over gloo ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from mlxmolkit_b200 import replicas


def test_partition_keeps_molecules_whole_and_balances_cost():
    rng = np.random.default_rng(3)
    n_atoms = rng.integers(20, 151, size=200)
    counts = rng.integers(1, 11, size=200)
    cost = replicas.molecule_cost(n_atoms, counts)
    for world in (1, 2, 3, 8):
        parts = replicas.partition_molecules(cost, world)
        assert len(parts) == world
        allm = np.concatenate(parts)
        assert sorted(allm.tolist()) == list(range(200))            # each molecule on exactly one rank
        loads = np.array([cost[p].sum() for p in parts])
        assert loads.max() - loads.min() <= cost.max()              # greedy largest-first bound
        assert [p.tolist() for p in parts] == [p.tolist() for p in replicas.partition_molecules(cost, world)]


def test_weak_scaling_seeds_differ_per_rank():
    assert len({replicas.rank_seed(0, r) for r in range(8)}) == 8


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    ms, conv = replicas.reduce_step(dist, 10.0 + rank, rank + 1, "cpu")
    with open(os.path.join(outdir, f"r{rank}.txt"), "w") as f:
        f.write(f"{ms} {conv}")
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_step_reduction_over_two_gloo_ranks(tmp_path):
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        ms, conv = map(float, open(tmp_path / f"r{r}.txt").read().split())
        assert ms == 11.0 and conv == 3.0                           # max over ranks, summed counts


def test_single_process_reduction_is_the_identity():
    assert replicas.reduce_step(None, 7.5, 4) == (7.5, 4.0)
