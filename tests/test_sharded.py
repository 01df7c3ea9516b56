"""The sharded build's protocol (distributed_diskann_b200/sharded.py) on the CPU.

Each rank is the CPU oracle's shard steps (oracle.ShardRankOracle), the
exchanges are gloo all-gathers between two processes, or the lockstep driver
in one process; the graph every rank ends with must be the one-rank build's,
row for row (src/bsp_index.hpp:247-407 splits each round's batch and owns
reverse edges by target % P; both are exact re-partitions of the same work).
"""
import os
import socket

import numpy as np
import pytest

from distributed_diskann_b200 import datasets as D
from distributed_diskann_b200.sharded import run_lockstep, run_rank, slice_of


def test_slices_follow_the_reference_split():
    for floor, ceiling in [(0, 1), (1, 3), (7, 15), (100, 1100), (5, 6)]:
        for world in (1, 2, 3, 4, 7, 8):
            sl = [slice_of(floor, ceiling, r, world) for r in range(world)]
            assert sl[0][0] == floor and sl[-1][1] == ceiling
            assert all(a[1] == b[0] for a, b in zip(sl, sl[1:]))
            sizes = [e - s for s, e in sl]
            assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def _rounds(n):
    from oracle import oracle as O

    return O.schedule(n)


def _points():
    return D.gen_mixture_i8(3_000, 24, 40, 31)


@pytest.mark.parametrize("world", [2, 3])
def test_lockstep_ranks_build_the_one_rank_graph(oracle_mod, world):
    base = _points()
    ref, _ = oracle_mod.build(base, 16, 32, 1.2)
    ranks = [oracle_mod.ShardRankOracle(base, 16, 32, 1.2) for _ in range(world)]
    run_lockstep(ranks, _rounds(base.shape[0]))
    for r in ranks:
        np.testing.assert_array_equal(r.graph, ref)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out_dir):
    import torch.distributed as dist

    from distributed_diskann_b200.sharded import TorchExchange
    from oracle import oracle as O

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    base = _points()
    r = O.ShardRankOracle(base, 16, 32, 1.2)
    run_rank(r, TorchExchange(), rank, world, O.schedule(base.shape[0]))
    np.save(os.path.join(out_dir, f"g{rank}.npy"), r.graph)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_build_the_one_rank_graph(oracle_mod, tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_gloo_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    base = _points()
    ref, _ = oracle_mod.build(base, 16, 32, 1.2)
    for r in range(world):
        np.testing.assert_array_equal(np.load(tmp_path / f"g{r}.npy"), ref)
