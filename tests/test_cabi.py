"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point include/dd_gpu.h declares, the ctypes table agrees with the header,
and the host-only entry points behave."""
import os
import re

import numpy as np
import pytest

from distributed_diskann_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "dd_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dd_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/dd_gpu.h but not exported"
    assert sorted(L.SIGNATURES) == names


def test_schedule_matches_oracle(oracle_mod):
    from distributed_diskann_b200.index import schedule

    for n, mb, x, knn in [(10_000, 0, 1.0, False), (1, 0, 1.0, False), (2, 0, 1.0, False),
                          (5_000, 4_000, 0.02, False), (10_000_000, 0, 1.0, False),
                          (1_000_000, 0, 0.02, False), (3_000, 0, 0.5, True)]:
        assert schedule(n, mb, x, knn) == oracle_mod.schedule(n, mb, x, knn)


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from distributed_diskann_b200.index import GpuIndex

    with pytest.raises(L.DDError):
        GpuIndex(np.uint8, "l2", 100, 16, 8)


def test_invalid_arguments_rejected():
    import ctypes as C

    lib = L.load()
    h = C.c_void_p()
    assert lib.dd_create(7, 0, 10, 4, 4, 0, C.byref(h)) == 1      # bad dtype
    assert lib.dd_create(0, 0, 0, 4, 4, 0, C.byref(h)) == 1       # n = 0
    assert lib.dd_create(2, 0, 10, 4, 200, 0, C.byref(h)) == 5    # R > 128
    assert lib.dd_create(0, 0, 10, 400, 8, 0, C.byref(h)) == 5    # row > 1 KiB
