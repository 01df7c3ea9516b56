"""Host logic of the multi-GPU bench path on CPU: two ranks over gloo.

Each rank builds an independent, differently seeded partition of the workload;
the job time is the maximum of the ranks' device times and the job rate counts
every rank's points (bench.py, distributed_diskann_b200/multirank.py).
"""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from distributed_diskann_b200 import datasets as D
from distributed_diskann_b200 import multirank as MR


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w = MR.rank_workload(D.WORKLOADS["bigann-u8"], rank)
        base, _ = D.make_workload(w, n=2000, nq=1)
        t_dev = 1.5 + rank  # this rank's device time of its steps
        t_max = MR.max_over_ranks(t_dev, torch.device("cpu"), True)
        digest = torch.tensor([float(base.astype(np.int64).sum())], dtype=torch.float64)
        all_d = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(all_d, digest)
        out.put((rank, t_max, [float(x.item()) for x in all_d], w.seed))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_max_time_and_distinct_partitions():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    # every rank sees the slowest rank's time
    assert [r[1] for r in res] == [2.5, 2.5]
    # the partitions differ (own seeds), and both ranks agree on them
    assert res[0][2] == res[1][2] and res[0][2][0] != res[0][2][1]
    assert res[0][3] != res[1][3]
    assert MR.whole_job_rate(2, 2000, 3, 2.5) == pytest.approx(2 * 2000 * 3 / 2.5)


def test_gpu_index_follows_visible_devices():
    assert MR.gpu_index(1, {"CUDA_VISIBLE_DEVICES": "4,6"}) == "6"
    assert MR.gpu_index(1, {}) == "1"
    assert MR.gpu_index(0, {"CUDA_VISIBLE_DEVICES": ""}) == "0"
