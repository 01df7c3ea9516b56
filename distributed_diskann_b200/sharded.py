"""The batched build spread over P ranks, one GPU each (the reference's
distributed build, src/bsp_index.hpp:141-434).

Every rank holds the whole points and graph.  Each round [floor, ceiling) of
the schedule is the reference's pair of supersteps:

1. the batch is split into P contiguous slices (src/bsp_index.hpp:247-252) and
   each rank searches and prunes its slice on the round-start graph;
2. the new out-lists are all-gathered, in rank order, which is batch order
   (the reference's first broadcast, include/bsp/broadcast_bsp_framework.cpp:
   166-218), and every rank applies the whole batch (:354-357);
3. each rank runs the reverse edges of the targets it owns, t % P == rank
   (:362-407), append or robustPrune;
4. the changed targets' rows are all-gathered (the second broadcast) and every
   rank applies the other ranks' rows.

Search/prune of a point depends only on the round-start graph, and the reverse
step of a target only on its sources (in batch order) and its row, so every
rank ends each round with the single-GPU build's graph.  The exchanges are
torch.distributed all-gathers (NCCL over NVLink between GPUs; gloo in the CPU
tests); nothing reads another GPU's memory directly.

A rank object provides ``search_prune(lo, hi)``, ``apply_reverse(floor,
ceiling, batch_rows, rank, world) -> (ids, rows)`` and ``set_rows(ids, rows)``;
``ShardRankGpu`` is the GPU one (the C ABI's dd_shard_* entry points).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .index import schedule


def slice_of(floor: int, ceiling: int, rank: int, world: int) -> tuple[int, int]:
    """Batch slice [start, end) of `rank` (src/bsp_index.hpp:247-252)."""
    total = ceiling - floor
    base, rem = divmod(total, world)
    start = floor + rank * base + min(rank, rem)
    return start, start + base + (1 if rank < rem else 0)


class ShardRankGpu:
    """One rank of the sharded build on a GpuIndex whose points are uploaded.
    Rows are torch int32 tensors on the index's GPU, dd_device_row_len wide."""

    def __init__(self, gi, L_, alpha, start_point=0, mode="fast", vcap=0, max_fraction=1.0,
                 max_build=0, world=1):
        import torch

        self.gi = gi
        self.torch = torch
        self.dev = torch.device("cuda", gi.device)
        self.row_len = int(gi.lib.dd_device_row_len(gi.h))
        self.rounds = schedule(gi.n, max_build, max_fraction)
        self.bmax = max(1, max(c - f for f, c in self.rounds))
        self.params = L.BuildParamsC(int(L_), float(alpha), float(max_fraction), int(max_build),
                                     int(start_point), 0, 0, 0, int(vcap), L.MODES[mode])
        # changed rows of one round: at most the targets this rank owns
        self.cap = min(self.bmax * gi.R, -(-gi.n // world))
        self.ids = torch.empty(self.cap, dtype=torch.int32, device=self.dev)
        self.rows = torch.empty((self.cap, self.row_len), dtype=torch.int32, device=self.dev)
        self.begin()

    def begin(self):
        """Sets the launch shapes and empties the graph: the start of a build."""
        self.gi._ck(self.gi.lib.dd_shard_begin(self.gi.h, C.byref(self.params), self.bmax))

    def search_prune(self, lo, hi):
        out = self.torch.empty((hi - lo, self.row_len), dtype=self.torch.int32, device=self.dev)
        self.gi._ck(self.gi.lib.dd_shard_search_prune(self.gi.h, lo, hi, C.c_void_p(out.data_ptr())))
        return out

    def apply_reverse(self, floor, ceiling, batch_rows, rank, world):
        batch_rows = batch_rows.contiguous()
        cnt = C.c_uint64(0)
        self.gi._ck(self.gi.lib.dd_shard_apply_reverse(
            self.gi.h, floor, ceiling, C.c_void_p(batch_rows.data_ptr()), rank, world,
            C.c_void_p(self.ids.data_ptr()), C.c_void_p(self.rows.data_ptr()), self.cap,
            C.byref(cnt)))
        c = int(cnt.value)
        return self.ids[:c].clone(), self.rows[:c].clone()

    def set_rows(self, ids, rows):
        ids, rows = ids.contiguous(), rows.contiguous()
        self.gi._ck(self.gi.lib.dd_shard_set_rows(self.gi.h, C.c_void_p(ids.data_ptr()),
                                                  C.c_void_p(rows.data_ptr()), int(ids.shape[0])))


def _as_torch(x):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)) if isinstance(x, np.ndarray) else x


def _cat(parts):
    import torch

    if isinstance(parts[0], np.ndarray):
        return np.concatenate(parts)
    return torch.cat(parts)


class TorchExchange:
    """All-gather of row blocks of different lengths over a torch.distributed
    group: the lengths are gathered first, every block is padded to the
    longest, gathered, and trimmed back."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group

    def allgather(self, x):
        import torch

        numpy_in = isinstance(x, np.ndarray)
        np_dtype = x.dtype if numpy_in else None
        if numpy_in and x.dtype == np.uint32:  # ids travel as int32 bit patterns
            x = np.ascontiguousarray(x).view(np.int32)
        t = _as_torch(x)
        world = self.dist.get_world_size(self.group)
        n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
        ns = [torch.zeros_like(n) for _ in range(world)]
        self.dist.all_gather(ns, n, group=self.group)
        lens = [int(v.item()) for v in ns]
        m = max(lens)
        pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
        pad[: t.shape[0]] = t
        outs = [torch.empty_like(pad) for _ in range(world)]
        self.dist.all_gather(outs, pad, group=self.group)
        res = [o[:ln] for o, ln in zip(outs, lens)]
        return [r.numpy().view(np_dtype) for r in res] if numpy_in else res


def run_rank(rank_obj, exchange, rank: int, world: int, rounds) -> None:
    """This rank's part of the sharded build; every rank calls it with the same
    rounds, and each round makes the same two all-gathers on every rank."""
    for floor, ceiling in rounds:
        if ceiling <= floor:
            continue
        lo, hi = slice_of(floor, ceiling, rank, world)
        parts = exchange.allgather(rank_obj.search_prune(lo, hi))
        ids, rows = rank_obj.apply_reverse(floor, ceiling, _cat(parts), rank, world)
        all_ids = exchange.allgather(ids)
        all_rows = exchange.allgather(rows)
        for r in range(world):
            if r != rank:
                rank_obj.set_rows(all_ids[r], all_rows[r])


def run_lockstep(rank_objs, rounds) -> None:
    """All ranks of a sharded build driven in one process, one step after the
    other (each rank's own handle; on one GPU the ranks' kernels never wait on
    one another).  Used to check the protocol where fewer GPUs than ranks exist."""
    world = len(rank_objs)
    for floor, ceiling in rounds:
        if ceiling <= floor:
            continue
        parts = [r.search_prune(*slice_of(floor, ceiling, k, world))
                 for k, r in enumerate(rank_objs)]
        batch = _cat(parts)
        changed = [r.apply_reverse(floor, ceiling, batch, k, world)
                   for k, r in enumerate(rank_objs)]
        for k, r in enumerate(rank_objs):
            for j, (ids, rows) in enumerate(changed):
                if j != k:
                    r.set_rows(ids, rows)
