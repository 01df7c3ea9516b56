"""Host-side API of the B200 Vamana hot path.

``GpuIndex`` wraps one device-resident index of the C ABI.  On top of it, the
names and argument meanings of the reference's build/search entry points are
kept so that callers of the reference find the same surface:

=====================================  ==============================================
reference (Mr1BW/distributed_diskann)  here
=====================================  ==============================================
BuildParams (include/utils/types.h:103) ``BuildParams``
QueryParams (include/utils/types.h:145) ``QueryParams``
dataset_para (src/dataset.hpp:30-135)   ``DatasetPara`` (para.json + dataset json)
PointRange (utils/point_range.h:53)     ``PointRange`` (.bin loader, numpy rows)
Graph (include/utils/graph.h:119-210)   ``Graph`` (n x (R+1) rows, save/load)
BSP_index::bsp_build (bsp_index.hpp:551) ``BSPIndex().bsp_build(BP, G, Points, stats, dp)``
knn_index (include/index.h:43-137)      ``KnnIndex(BP).build_index(G, Points, stats)``,
                                        ``KnnIndex.robust_prune``
beam_search (utils/beamSearch.h:41-48)  ``beam_search(p, G, Points, start, QP)``
searchAll (utils/beamSearch.h:314-320)  ``search_all(Q, G, B, stats, start, QP)``
=====================================  ==============================================

Errors: the reference aborts on invalid ids / degree overflow; here a
``DDError`` is raised carrying the C ABI status and message.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .datasets import read_bin, write_bin

DTYPES = {np.dtype(np.float32): 0, np.dtype(np.int8): 1, np.dtype(np.uint8): 2}
DTYPE_NAMES = {"float32": np.float32, "int8": np.int8, "uint8": np.uint8}
METRICS = {"l2": 0, "euclidean": 0, "mips": 1, "ip": 1}


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


class GpuIndex:
    """A device-resident index: points + graph (+ scratch) in HBM of one GPU."""

    def __init__(self, dtype, metric, n, d, R, device=0):
        self.lib = L.load()
        self.device = int(device)
        self.dtype = np.dtype(dtype)
        self.metric = metric
        self.n, self.d, self.R = int(n), int(d), int(R)
        h = C.c_void_p()
        rc = self.lib.dd_create(DTYPES[self.dtype], METRICS[metric], self.n, self.d, self.R,
                                int(device), C.byref(h))
        if rc != 0:
            raise L.DDError(rc, f"dd_create(n={n}, d={d}, R={R}) failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.dd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        L.check(rc, self.h)

    # ---------------------------------------------------------------- data
    def upload_points(self, points):
        """Host numpy rows, or a CUDA tensor / device pointer (with stride)."""
        if isinstance(points, np.ndarray):
            points = np.ascontiguousarray(points, dtype=self.dtype)
            assert points.shape == (self.n, self.d), points.shape
            self._ck(self.lib.dd_upload_points(self.h, _ptr(points), points.strides[0]))
            return
        # torch CUDA tensor
        assert points.is_cuda and points.shape == (self.n, self.d)
        stride = points.stride(0) * points.element_size()
        self._ck(self.lib.dd_upload_points_device(self.h, C.c_void_p(points.data_ptr()), stride))

    def set_stream(self, stream_ptr: int):
        self._ck(self.lib.dd_set_stream(self.h, C.c_void_p(stream_ptr)))

    def set_search_mode(self, mode: str):
        self._ck(self.lib.dd_set_search_mode(self.h, L.MODES[mode]))

    def check_errors(self):
        """Raises if a kernel of an asynchronous call raised the device error word."""
        self._ck(self.lib.dd_check_errors(self.h))

    def graph(self) -> np.ndarray:
        g = np.zeros((self.n, self.R + 1), np.uint32)
        self._ck(self.lib.dd_download_graph(self.h, _ptr(g)))
        return g

    def set_graph(self, g: np.ndarray):
        g = np.ascontiguousarray(g, dtype=np.uint32)
        assert g.shape == (self.n, self.R + 1)
        self._ck(self.lib.dd_upload_graph(self.h, _ptr(g)))

    def save_graph(self, path):
        self._ck(self.lib.dd_save_graph_file(self.h, os.fsencode(path)))

    def load_graph(self, path):
        self._ck(self.lib.dd_load_graph_file(self.h, os.fsencode(path)))

    def load_points(self, path):
        """Reads a reference .bin file ([u32 n][u32 d][rows]) into the index."""
        self._ck(self.lib.dd_load_points_file(self.h, os.fsencode(path)))

    # ---------------------------------------------------------------- build
    def build(self, L_, alpha, max_fraction=1.0, max_build=0, start_point=0, two_pass=False,
              knn_mode=False, collect_stats=True, vcap=0, mode="fast") -> dict:
        """Batched build; mode "fast" (tensor-core tiles, persistent kernels,
        graph-captured rounds) or "plain" (CUDA-core exact form): same graph."""
        p = L.BuildParamsC(int(L_), float(alpha), float(max_fraction), int(max_build),
                           int(start_point), int(two_pass), int(knn_mode), int(collect_stats),
                           int(vcap), L.MODES[mode])
        st = L.StatsC()
        self._ck(self.lib.dd_build(self.h, C.byref(p), C.byref(st)))
        return st.as_dict()

    # ---------------------------------------------------------------- search
    def search(self, queries, k, L_, cut=1.35, limit=0, degree_limit=0, start=0, skip_self=True):
        """searchAll over host queries; L_ may be an int or one beam width per query."""
        q = np.ascontiguousarray(queries, dtype=self.dtype)
        nq = q.shape[0]
        Ls = np.ascontiguousarray(np.broadcast_to(np.asarray(L_, np.uint32), (nq,)))
        ids = np.zeros((nq, k), np.uint32)
        ds = np.zeros((nq, k), np.float32)
        vis = np.zeros(nq, np.uint32)
        cm = np.zeros(nq, np.uint32)
        self._ck(self.lib.dd_search(self.h, _ptr(q), nq, q.strides[0], _ptr(Ls), int(k),
                                    float(cut), int(limit), int(degree_limit), int(start),
                                    int(bool(skip_self)), _ptr(ids), _ptr(ds), _ptr(vis),
                                    _ptr(cm)))
        return ids, ds, vis, cm

    def search_device(self, q_ptr, nq, qstride, Ls_ptr, Lmax, k, ids_ptr, dists_ptr, cut=1.35,
                      limit=0, degree_limit=0, start=0, skip_self=True, vis_ptr=0, cmps_ptr=0):
        self._ck(self.lib.dd_search_device(self.h, C.c_void_p(q_ptr), int(nq), int(qstride),
                                           C.c_void_p(Ls_ptr), int(Lmax), int(k), float(cut),
                                           int(limit), int(degree_limit), int(start),
                                           int(bool(skip_self)), C.c_void_p(ids_ptr),
                                           C.c_void_p(dists_ptr), C.c_void_p(vis_ptr or None),
                                           C.c_void_p(cmps_ptr or None)))

    def beam_search(self, queries, L_, k=0, cut=0.0, self_ids=None, start=0, limit=0,
                    degree_limit=0, vcap=None):
        q = np.ascontiguousarray(np.atleast_2d(queries), dtype=self.dtype)
        nq = q.shape[0]
        vcap = int(vcap or 4 * L_)
        si = np.full(nq, -1, np.int64) if self_ids is None else np.ascontiguousarray(self_ids, np.int64)
        fi = np.zeros((nq, L_), np.uint32)
        fd = np.zeros((nq, L_), np.float32)
        fn = np.zeros(nq, np.uint32)
        vi = np.zeros((nq, vcap), np.uint32)
        vd = np.zeros((nq, vcap), np.float32)
        vn = np.zeros(nq, np.uint32)
        cm = np.zeros(nq, np.uint32)
        self._ck(self.lib.dd_beam_search(self.h, _ptr(q), nq, q.strides[0], _ptr(si), int(L_),
                                         int(k), float(cut), int(limit), int(degree_limit),
                                         int(start), vcap, _ptr(fi), _ptr(fd), _ptr(fn), _ptr(vi),
                                         _ptr(vd), _ptr(vn), _ptr(cm)))
        out = []
        for i in range(nq):
            a, b = int(fn[i]), int(vn[i])
            out.append(((fi[i, :a], fd[i, :a]), (vi[i, :b], vd[i, :b]), int(cm[i])))
        return out

    def robust_prune(self, tasks, alpha):
        """tasks: list of (p, cand_ids, cand_dists); returns one id list per task."""
        nt = len(tasks)
        p = np.array([t[0] for t in tasks], np.uint32)
        off = np.zeros(nt + 1, np.uint64)
        off[1:] = np.cumsum([len(t[1]) for t in tasks])
        ci = np.ascontiguousarray(np.concatenate([np.asarray(t[1], np.uint32) for t in tasks])
                                  if nt else np.zeros(0, np.uint32))
        cd = np.ascontiguousarray(np.concatenate([np.asarray(t[2], np.float32) for t in tasks])
                                  if nt else np.zeros(0, np.float32))
        out = np.zeros((max(nt, 1), self.R), np.uint32)
        ol = np.zeros(max(nt, 1), np.uint32)
        self._ck(self.lib.dd_robust_prune(self.h, nt, _ptr(p), _ptr(off), _ptr(ci), _ptr(cd),
                                          float(alpha), _ptr(out), _ptr(ol)))
        return [out[t, : ol[t]].copy() for t in range(nt)]

    def groundtruth(self, queries, k):
        q = np.ascontiguousarray(queries, dtype=self.dtype)
        ids = np.zeros((q.shape[0], k), np.uint32)
        ds = np.zeros((q.shape[0], k), np.float32)
        self._ck(self.lib.dd_groundtruth(self.h, _ptr(q), q.shape[0], q.strides[0], int(k),
                                         _ptr(ids), _ptr(ds)))
        return ids, ds

    def launches(self) -> int:
        return int(self.lib.dd_last_launch_count(self.h))


def schedule(n, max_build=0, max_fraction=1.0, knn_mode=False):
    lib = L.load()
    cap = 4096
    f = np.zeros(cap, np.uint64)
    c = np.zeros(cap, np.uint64)
    nr = np.zeros(1, np.uint64)
    lib.dd_schedule(int(n), int(max_build), float(max_fraction), int(knn_mode), _ptr(f), _ptr(c),
                    cap, _ptr(nr))
    return [(int(f[i]), int(c[i])) for i in range(min(int(nr[0]), cap))]


# ====================================================================== reference-shaped API
@dataclass
class BuildParams:
    """include/utils/types.h:103-142 (Vamana fields)."""
    R: int
    L: int
    alpha: float
    two_pass: bool = False

    def max_degree(self):
        return self.R


@dataclass
class QueryParams:
    """include/utils/types.h:145-156."""
    k: int
    beamSize: int
    cut: float
    limit: int
    degree_limit: int


class DatasetPara:
    """src/dataset.hpp:30-135: para.json (build parameters) + dataset json."""

    def __init__(self):
        self.build = self.query = self.save = True
        self.two_pass = False
        self.start_point_index = 0
        self.xita = 0.02
        self.alpha = 1.2
        self.L = 128
        self.R = self.L // 2
        self.Ls = 128
        self.num_neighbors_query = 100
        self.max_build = 0
        self.dataset_parafile = ""
        self.output_path = ""

    def set(self, filename):
        with open(filename) as f:
            j = json.load(f)
        self.build, self.query, self.save = j["build"], j["query"], j["save"]
        self.two_pass = j["two_pass"]
        self.start_point_index = j["start_point_index"]
        self.xita, self.alpha = j["xita"], j["alpha"]
        self.L, self.R, self.Ls = j["L"], j["R"], j["Ls"]
        self.max_build = j["max"]
        self.num_neighbors_query = j["num_neighbors_query"]
        self.dataset_parafile = j["data_para"]

    def open(self, filename):
        with open(filename) as f:
            j = json.load(f)
        self.dataset_name = j["dataset"]
        self.nb, self.nq, self.d, self.dtype = j["nb"], j["nq"], j["d"], j["dtype"]
        self.ds_fn, self.qs_fn, self.gt_fn, self.basedir = j["ds_fn"], j["qs_fn"], j["gt_fn"], j["basedir"]
        self.ds_dir = self.basedir + "/" + self.ds_fn
        self.qs_dir = self.basedir + "/" + self.qs_fn
        self.gt_dir = self.basedir + "/" + self.gt_fn
        self.output_path = "results/" + self.dataset_name


class PointRange:
    """include/utils/point_range.h:53-113: rows of a .bin file (or an array)."""

    def __init__(self, src, dtype=None, metric="l2"):
        self.metric = metric
        if isinstance(src, np.ndarray):
            self.values = np.ascontiguousarray(src)
        else:
            self.values = read_bin(src, dtype)
        self.n, self.dims = self.values.shape

    def size(self):
        return self.n

    def dimension(self):
        return self.dims

    def __getitem__(self, i):
        return self.values[i]


class Graph:
    """include/utils/graph.h:119-210: n rows of (R+1) uint32, row[0] = degree."""

    def __init__(self, max_deg=None, n=None, path=None):
        if path is not None:
            raw = np.fromfile(path, dtype=np.uint32)
            n, max_deg = int(raw[0]), int(raw[1])
            deg = raw[2 : 2 + n]
            self.rows = np.zeros((n, max_deg + 1), np.uint32)
            self.rows[:, 0] = deg
            mask = np.arange(max_deg)[None, :] < deg[:, None]
            self.rows[:, 1:][mask] = raw[2 + n :]
        else:
            self.rows = np.zeros((n, max_deg + 1), np.uint32)

    def size(self):
        return self.rows.shape[0]

    def max_degree(self):
        return self.rows.shape[1] - 1

    def __getitem__(self, i):
        return self.rows[i, 1 : 1 + self.rows[i, 0]]

    def save(self, path):
        n, R1 = self.rows.shape
        with open(path, "wb") as f:
            np.array([n, R1 - 1], np.uint32).tofile(f)
            self.rows[:, 0].tofile(f)
            mask = np.arange(R1 - 1)[None, :] < self.rows[:, :1]
            self.rows[:, 1:][mask].tofile(f)


def _gpu_for(Points: PointRange, G: Graph, device=0) -> GpuIndex:
    gi = GpuIndex(Points.values.dtype, Points.metric, Points.n, Points.dims, G.max_degree(), device)
    gi.upload_points(Points.values)
    return gi


class BSPIndex:
    """BSP_index::bsp_build (src/bsp_index.hpp:551-556) on one GPU: the whole
    superstep loop runs device-side; the result is written into ``G`` and, like
    the reference's cleanup (:472-475), saved to ``dp.output_path`` if ``dp.save``."""

    def bsp_build(self, BP: BuildParams, G: Graph, Points: PointRange, BuildStats=None,
                  dp: DatasetPara | None = None, device=0):
        dp = dp or DatasetPara()
        gi = _gpu_for(Points, G, device)
        st = gi.build(BP.L, dp.alpha, max_fraction=dp.xita, max_build=dp.max_build,
                      start_point=dp.start_point_index)
        G.rows[:] = gi.graph()
        if dp.save and dp.output_path:
            os.makedirs(os.path.dirname(dp.output_path) or ".", exist_ok=True)
            G.save(dp.output_path)
        gi.close()
        return st


class KnnIndex:
    """knn_index (include/index.h:43-137): build_index with max_fraction 1.0,
    optional two_pass and the final per-row distance sort."""

    def __init__(self, BP: BuildParams):
        self.BP = BP
        self.start_point = 0

    def build_index(self, G: Graph, Points: PointRange, BuildStats=None, device=0):
        gi = _gpu_for(Points, G, device)
        st = gi.build(self.BP.L, self.BP.alpha, two_pass=self.BP.two_pass, knn_mode=True)
        G.rows[:] = gi.graph()
        gi.close()
        return st

    def robust_prune(self, p, cand, G: Graph, Points: PointRange, alpha, device=0):
        """cand: list of (id, dist) pairs; include/index.h:63-110."""
        gi = _gpu_for(Points, G, device)
        gi.set_graph(G.rows)
        ids = np.array([c[0] for c in cand], np.uint32)
        ds = np.array([c[1] for c in cand], np.float32)
        out = gi.robust_prune([(p, ids, ds)], alpha)[0]
        gi.close()
        return out


def beam_search(p, G: Graph, Points: PointRange, starting_point, QP: QueryParams, p_id=-1,
                device=0):
    """include/utils/beamSearch.h:41-48 -> ((frontier, visited), dist_cmps)."""
    gi = _gpu_for(Points, G, device)
    gi.set_graph(G.rows)
    (fr, vi, cm), = gi.beam_search(np.asarray(p)[None], QP.beamSize, k=QP.k, cut=QP.cut,
                                   self_ids=[p_id], start=starting_point, limit=QP.limit,
                                   degree_limit=QP.degree_limit)
    gi.close()
    return (list(zip(fr[0].tolist(), fr[1].tolist())), list(zip(vi[0].tolist(), vi[1].tolist()))), cm


def search_all(Query_Points: PointRange, G: Graph, Base_Points: PointRange, QueryStats=None,
               starting_point=0, QP: QueryParams | None = None, device=0):
    """include/utils/beamSearch.h:314-346: first k frontier ids per query."""
    if QP.k > QP.beamSize:
        raise ValueError(f"beam search parameter Q = {QP.beamSize} same size or smaller than k = {QP.k}")
    gi = _gpu_for(Base_Points, G, device)
    gi.set_graph(G.rows)
    ids, _, vis, cm = gi.search(Query_Points.values, QP.k, QP.beamSize, cut=QP.cut,
                                limit=QP.limit, degree_limit=QP.degree_limit, start=starting_point)
    gi.close()
    if QueryStats is not None:
        QueryStats["visited"] = vis
        QueryStats["distances"] = cm
    return ids


__all__ = ["GpuIndex", "BuildParams", "QueryParams", "DatasetPara", "PointRange", "Graph",
           "BSPIndex", "KnnIndex", "beam_search", "search_all", "schedule", "write_bin"]
