"""ctypes binding of the CUDA library (include/dd_gpu.h).

The library is built in-tree (distributed_diskann_b200/_lib/libdd_gpu.so).  If
it is missing or fails to load, every entry point raises: there is no CPU
fallback on the product path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libdd_gpu.so")

DD_OK = 0
MODES = {"fast": 0, "plain": 1}
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "device error word", 5: "unsupported parameter", 6: "I/O error"}

vp, u64, u32, i64, i32, dbl = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int64, C.c_int, C.c_double


class DDError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{ERRORS.get(code, code)}] {msg}")
        self.code = code


class BuildParamsC(C.Structure):
    _fields_ = [("L", u32), ("alpha", dbl), ("max_fraction", dbl), ("max_build", u64),
                ("start_point", u32), ("two_pass", C.c_int32), ("knn_mode", C.c_int32),
                ("collect_stats", C.c_int32), ("vcap", u32), ("mode", C.c_int32)]


class StatsC(C.Structure):
    _fields_ = [("rounds", u64), ("visited", u64), ("dist_cmps", u64), ("groups", u64),
                ("reverse_prunes", u64), ("prune_cands", u64), ("big_groups", u64),
                ("build_ms", dbl), ("search_prune_ms", dbl), ("reverse_ms", dbl),
                ("search_ms", dbl), ("search_warps_per_cta", u32), ("prune_warps_per_cta", u32),
                ("search_queue", C.c_int32), ("prune_queue", C.c_int32),
                ("graph_replay", C.c_int32), ("vcap", u32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# exported symbol -> (restype, argtypes); the CPU tests check that this table
# and include/dd_gpu.h agree and that the library exports all of them
SIGNATURES = {
    "dd_create": (i32, [i32, i32, u64, u32, u32, i32, C.POINTER(vp)]),
    "dd_destroy": (i32, [vp]),
    "dd_last_error": (C.c_char_p, [vp]),
    "dd_set_stream": (i32, [vp, vp]),
    "dd_set_search_mode": (i32, [vp, i32]),
    "dd_check_errors": (i32, [vp]),
    "dd_upload_points": (i32, [vp, vp, u64]),
    "dd_upload_points_device": (i32, [vp, vp, u64]),
    "dd_upload_points_async": (i32, [vp, vp, u64]),
    "dd_load_points_file": (i32, [vp, C.c_char_p]),
    "dd_upload_graph": (i32, [vp, vp]),
    "dd_download_graph": (i32, [vp, vp]),
    "dd_load_graph_file": (i32, [vp, C.c_char_p]),
    "dd_save_graph_file": (i32, [vp, C.c_char_p]),
    "dd_build": (i32, [vp, C.POINTER(BuildParamsC), C.POINTER(StatsC)]),
    "dd_schedule": (i32, [u64, u64, dbl, i32, vp, vp, u64, vp]),
    "dd_shard_begin": (i32, [vp, C.POINTER(BuildParamsC), u64]),
    "dd_shard_search_prune": (i32, [vp, u64, u64, vp]),
    "dd_shard_apply_reverse": (i32, [vp, u64, u64, vp, i32, i32, vp, vp, u64, vp]),
    "dd_shard_set_rows": (i32, [vp, vp, vp, u64]),
    "dd_search": (i32, [vp, vp, u64, u64, vp, u32, dbl, u64, u32, u32, i32, vp, vp, vp, vp]),
    "dd_search_device": (i32, [vp, vp, u64, u64, vp, u32, u32, dbl, u64, u32, u32, i32, vp, vp,
                               vp, vp]),
    "dd_beam_search": (i32, [vp, vp, u64, u64, vp, u32, u32, dbl, u64, u32, u32, u32, vp, vp, vp,
                             vp, vp, vp, vp]),
    "dd_robust_prune": (i32, [vp, u32, vp, vp, vp, vp, dbl, vp, vp]),
    "dd_robust_prune_noalloc": (i32, [vp, u32, vp, vp, u64, vp, vp, dbl, vp, i32]),
    "dd_groundtruth": (i32, [vp, vp, u64, u64, u32, vp, vp]),
    "dd_device_points": (vp, [vp]),
    "dd_device_row_stride": (u64, [vp]),
    "dd_device_graph": (vp, [vp]),
    "dd_device_row_len": (u32, [vp]),
    "dd_last_launch_count": (u64, [vp]),
}

_lib = None


def load():
    """Load the CUDA library (building it first if the sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _build

            _build.build()
        except Exception as e:  # no nvcc: the library must have been shipped prebuilt
            raise RuntimeError(f"CUDA library {LIB_PATH} is missing and could not be built: {e}")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc, handle=None):
    if rc != DD_OK:
        msg = load().dd_last_error(handle).decode() if handle else ""
        raise DDError(rc, msg)
