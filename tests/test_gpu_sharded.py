"""The sharded build's GPU steps (dd_shard_* through distributed_diskann_b200.sharded).

This run has one GPU per box, so the ranks are separate index handles on that
GPU driven in lockstep (run_lockstep): each step of one rank finishes before
the next one starts, and no kernel waits on another rank.  The graph every
rank ends with must be dd_build's, which the other tests pin to the
reference's build; the multi-GPU exchange itself (NCCL all-gathers) is the
same protocol the gloo test of tests/test_sharded.py runs between processes.
"""
import numpy as np
import pytest

from distributed_diskann_b200 import datasets as D
from distributed_diskann_b200.index import GpuIndex
from distributed_diskann_b200.sharded import ShardRankGpu, run_lockstep
from tests.golden.make_golden import canon

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("world,mode", [(1, "fast"), (2, "fast"), (3, "plain"), (4, "fast")])
def test_lockstep_gpu_ranks_build_the_single_gpu_graph(world, mode):
    base = D.gen_skewed_u8(60_000, 64, 600, 41)
    ref = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 32)
    ref.upload_points(base)
    ref.build(64, 1.2, mode=mode)
    expect = canon(ref.graph())
    ref.close()
    idx, ranks = [], []
    for _ in range(world):
        gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 32)
        gi.upload_points(base)
        idx.append(gi)
        ranks.append(ShardRankGpu(gi, 64, 1.2, mode=mode, world=world))
    run_lockstep(ranks, ranks[0].rounds)
    for gi in idx:
        np.testing.assert_array_equal(canon(gi.graph()), expect)
        gi.close()
