"""dd_robust_prune_noalloc: the allocation-free variant of dd_robust_prune.

It is meant for callers that cannot call cudaMalloc while the prune runs (a
process with a fixed, pre-reserved device-memory budget, or a host whose
device memory belongs to another allocator): every argument is a device
pointer and the candidate workspace is a fixed device array inside the
library.  This test
calls it through the C ABI twice in a row (the shared workspace keeps the
previous call's contents) and checks both results against dd_robust_prune,
which allocates its own workspace.  Ids must match exactly.  The file is
named to be collected last; it also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tasks(base, rng, ntasks):
    from oracle import oracle as O

    tasks = []
    for t in range(ntasks):
        p = int(rng.integers(0, base.shape[0]))
        m = int(rng.choice([1, 5, 16, 17, 40, 90]))
        cand = rng.choice(base.shape[0], m, replace=False).astype(np.uint32)
        dist = np.array([O.distance(base[c], base[p]) for c in cand], np.float32)
        if t % 2:  # coarse distances: many exact ties
            dist = (np.floor(dist / 4000.0) * 4000.0).astype(np.float32)
        tasks.append((p, cand, dist))
    return tasks


def test_noalloc_prune_matches_allocating_prune_twice():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from distributed_diskann_b200 import _lib
    from distributed_diskann_b200 import datasets as D
    from distributed_diskann_b200.index import GpuIndex

    base = D.gen_mixture_i8(4_000, 64, 50, 21)
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 32)
    gi.upload_points(base)
    gi.build(48, 1.2)
    Rp = int(gi.lib.dd_device_row_len(gi.h))
    rng = np.random.default_rng(3)
    dev = torch.device("cuda", 0)
    for call in range(2):
        tasks = _tasks(base, rng, 300)
        expect = gi.robust_prune(tasks, 1.2)  # allocating entry point, host buffers
        offsets = np.zeros(len(tasks) + 1, np.uint64)
        offsets[1:] = np.cumsum([len(t[1]) for t in tasks])
        total = int(offsets[-1])
        p_d = torch.tensor(np.array([t[0] for t in tasks], np.uint32).view(np.int32), device=dev)
        off_d = torch.tensor(offsets.view(np.int64), device=dev)
        ci_d = torch.tensor(np.concatenate([t[1] for t in tasks]).view(np.int32), device=dev)
        cd_d = torch.tensor(np.concatenate([t[2] for t in tasks]), device=dev)
        out_d = torch.empty((len(tasks), Rp), dtype=torch.int32, device=dev)
        rc = gi.lib.dd_robust_prune_noalloc(gi.h, len(tasks), C.c_void_p(p_d.data_ptr()),
                                            C.c_void_p(off_d.data_ptr()), total,
                                            C.c_void_p(ci_d.data_ptr()),
                                            C.c_void_p(cd_d.data_ptr()), 1.2,
                                            C.c_void_p(out_d.data_ptr()), 1)
        _lib.check(rc, gi.h)
        out = out_d.cpu().numpy().view(np.uint32)
        for t, e in enumerate(expect):
            row = out[t]
            n = int(np.argmax(row == 0xFFFFFFFF)) if (row == 0xFFFFFFFF).any() else Rp
            np.testing.assert_array_equal(row[:n], e, err_msg=f"call {call} task {t}")
    # a request beyond the fixed workspace is refused with a clear error
    big = gi.lib.dd_robust_prune_noalloc(gi.h, 4096, C.c_void_p(p_d.data_ptr()),
                                         C.c_void_p(off_d.data_ptr()), 1 << 20,
                                         C.c_void_p(ci_d.data_ptr()), C.c_void_p(cd_d.data_ptr()),
                                         1.2, C.c_void_p(out_d.data_ptr()), 1)
    assert big == 5  # DD_ERR_UNSUPPORTED, nothing launched
    assert b"exceed the fixed workspace" in gi.lib.dd_last_error(gi.h)
    gi.close()
