"""dd_robust_prune_noalloc: the allocation-free variant of dd_robust_prune.

It is meant for callers that cannot call cudaMalloc while the prune runs (a
process with a fixed, pre-reserved device-memory budget, or a host whose
device memory belongs to another allocator): every argument is a device
pointer and the candidate workspace is a fixed device array inside the
library.  These tests call it through the C ABI twice in a row (the shared
workspace keeps the previous call's contents) for every element type and
metric, check both results against dd_robust_prune, which allocates its own
workspace (ids must match exactly), check that the device's free memory does
not move across the calls, and check the invalid-input paths.  The file is
named to be collected last; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DD_ERR_DEVICE = 4
DD_ERR_UNSUPPORTED = 5


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _points(dtype, metric):
    from distributed_diskann_b200 import datasets as D

    if dtype == "i8":
        return D.gen_mixture_i8(4_000, 64, 50, 21)
    if dtype == "u8":
        return D.gen_skewed_u8(4_000, 64, 50, 22)
    if metric == "mips":
        return D.gen_normalized_mixture(4_000, 40, 50, 23)
    return D.gen_mixture_f32(4_000, 40, 50, 24)


def _tasks(base, metric, rng, ntasks):
    from oracle import oracle as O

    tasks = []
    for t in range(ntasks):
        p = int(rng.integers(0, base.shape[0]))
        m = int(rng.choice([1, 5, 16, 17, 40, 90]))
        cand = rng.choice(base.shape[0], m, replace=False).astype(np.uint32)
        dist = np.array([O.distance(base[c], base[p], metric) for c in cand], np.float32)
        if t % 2:  # coarse distances: many exact ties
            q = np.float32(4000.0 if base.dtype != np.float32 else 0.25)
            dist = (np.floor(dist / q) * q).astype(np.float32)
        tasks.append((p, cand, dist))
    return tasks


class _DevTasks:
    """Device copies of a task list in the entry point's argument layout."""

    def __init__(self, tasks, Rp, dev):
        import torch

        offsets = np.zeros(len(tasks) + 1, np.uint64)
        offsets[1:] = np.cumsum([len(t[1]) for t in tasks])
        self.ntasks = len(tasks)
        self.total = int(offsets[-1])
        self.p = torch.tensor(np.array([t[0] for t in tasks], np.uint32).view(np.int32), device=dev)
        self.off = torch.tensor(offsets.view(np.int64), device=dev)
        self.ci = torch.tensor(np.concatenate([t[1] for t in tasks]).view(np.int32), device=dev)
        self.cd = torch.tensor(np.concatenate([t[2] for t in tasks]), device=dev)
        self.out = torch.empty((len(tasks), Rp), dtype=torch.int32, device=dev)

    def call(self, gi, sync, ntasks=None, total=None):
        return gi.lib.dd_robust_prune_noalloc(
            gi.h, self.ntasks if ntasks is None else ntasks, C.c_void_p(self.p.data_ptr()),
            C.c_void_p(self.off.data_ptr()), self.total if total is None else total,
            C.c_void_p(self.ci.data_ptr()), C.c_void_p(self.cd.data_ptr()), 1.2,
            C.c_void_p(self.out.data_ptr()), sync)

    def rows(self):
        return self.out.cpu().numpy().view(np.uint32)


def _row_ids(row):
    pad = row == 0xFFFFFFFF
    return row[: int(np.argmax(pad))] if pad.any() else row


def _index(dtype, metric):
    from distributed_diskann_b200.index import GpuIndex

    base = _points(dtype, metric)
    gi = GpuIndex(base.dtype, metric, base.shape[0], base.shape[1], 32)
    gi.upload_points(base)
    gi.build(48, 1.2)
    return base, gi


@pytest.mark.parametrize("dtype,metric", [("i8", "l2"), ("u8", "l2"), ("f32", "l2"),
                                          ("i8", "mips"), ("u8", "mips"), ("f32", "mips")])
def test_noalloc_prune_matches_allocating_prune_twice(dtype, metric):
    import torch

    from distributed_diskann_b200 import _lib

    base, gi = _index(dtype, metric)
    Rp = int(gi.lib.dd_device_row_len(gi.h))
    rng = np.random.default_rng(3)
    dev = torch.device("cuda", 0)
    free_before = None
    for call in range(2):
        tasks = _tasks(base, metric, rng, 300)
        expect = gi.robust_prune(tasks, 1.2)  # allocating entry point, host buffers
        dt = _DevTasks(tasks, Rp, dev)
        torch.cuda.synchronize()
        if call == 1:  # the first call may look up the workspace address once
            free_before = torch.cuda.mem_get_info()[0]
        _lib.check(dt.call(gi, 1), gi.h)
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before, "the call allocated device memory"
        out = dt.rows()
        for t, e in enumerate(expect):
            np.testing.assert_array_equal(_row_ids(out[t]), e, err_msg=f"call {call} task {t}")
    # a request beyond the fixed workspace is refused with a clear error
    assert dt.call(gi, 1, ntasks=4096, total=1 << 20) == DD_ERR_UNSUPPORTED  # nothing launched
    assert b"exceed the fixed workspace" in gi.lib.dd_last_error(gi.h)
    gi.close()


def test_noalloc_prune_invalid_inputs_pad_rows_and_report():
    import torch

    from distributed_diskann_b200 import _lib

    base, gi = _index("i8", "l2")
    n = base.shape[0]
    Rp = int(gi.lib.dd_device_row_len(gi.h))
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    tasks = _tasks(base, "l2", rng, 40)
    expect = gi.robust_prune(tasks, 1.2)
    bad = 7
    p, cand, dist = tasks[bad]
    cand = cand.copy()
    cand[len(cand) // 2] = n  # out of range: the kernel's own check pads this task's row
    tasks[bad] = (p, cand, dist)
    for sync in (1, 0):
        dt = _DevTasks(tasks, Rp, dev)
        rc = dt.call(gi, sync)
        if sync:
            assert rc == DD_ERR_DEVICE
        else:
            assert rc == 0
            # reported at the next synchronizing call (a valid one)
            good = _DevTasks(tasks[:bad], Rp, dev)
            assert good.call(gi, 1) == DD_ERR_DEVICE
        assert b"out of range" in gi.lib.dd_last_error(gi.h)
        out = dt.rows()
        assert (out[bad] == 0xFFFFFFFF).all()
        for t, e in enumerate(expect):
            if t != bad:
                np.testing.assert_array_equal(_row_ids(out[t]), e, err_msg=f"task {t}")
    # decreasing offsets invalidate the whole call: every row is padding
    dt = _DevTasks(tasks[:bad], Rp, dev)
    off = dt.off.cpu().numpy().copy()
    off[3], off[4] = off[4], off[3]
    dt.off = torch.tensor(off, device=dev)
    assert dt.call(gi, 1) == DD_ERR_DEVICE
    assert (dt.rows() == 0xFFFFFFFF).all()
    # the handle stays usable
    good = _DevTasks(tasks[:bad], Rp, dev)
    _lib.check(good.call(gi, 1), gi.h)
    gi.close()
