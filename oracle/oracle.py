"""ctypes wrapper of the CPU oracle (oracle/dd_oracle.cpp) — TEST INFRASTRUCTURE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker.  The product package never does.

Also drives the reference's own sources built as ``oracle/_ref/ref_harness``
(see oracle/Makefile) to pin the oracle and to time the reference CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libdd_oracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
# where the reference tree lies (only the machine that builds the harness has it)
REF_ROOT = os.environ.get("DD_REFERENCE_ROOT", "/root/reference")

DTYPES = {np.dtype(np.float32): 0, np.dtype(np.int8): 1, np.dtype(np.uint8): 2}
DTYPE_NAMES = {0: "f32", 1: "i8", 2: "u8"}
METRICS = {"l2": 0, "mips": 1}

_lib = None


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def build_reference(ref_root: str = REF_ROOT) -> bool:
    """Compile the reference harness if its sources are present (this container)."""
    if os.path.exists(REF_HARNESS):
        return True
    if not os.path.isdir(ref_root):
        return False
    subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_root}"], check=True)
    return os.path.exists(REF_HARNESS)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_oracle()
        L = C.CDLL(LIB_PATH)
        vp, u64, u32, i64, dbl, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int64, C.c_double, C.c_int
        L.ddo_distance.restype = C.c_float
        L.ddo_distance.argtypes = [i32, i32, vp, vp, u32]
        L.ddo_build.restype = i32
        L.ddo_build.argtypes = [i32, i32, vp, u64, u32, u64, u32, u32, dbl, dbl, u64, u32, i32, i32,
                                i32, vp, vp]
        L.ddo_beam_search.restype = i32
        L.ddo_beam_search.argtypes = [i32, i32, vp, u64, u32, u64, vp, u32, vp, i64, u32, i64, i64,
                                      dbl, i64, i64, vp, vp, vp, vp, vp, vp, u32, vp]
        L.ddo_search.restype = i32
        L.ddo_search.argtypes = [i32, i32, vp, u64, u32, u64, vp, u32, vp, u64, u64, vp, i64, dbl,
                                 i64, i64, u32, i32, vp, vp, vp]
        L.ddo_robust_prune.restype = i32
        L.ddo_robust_prune.argtypes = [i32, i32, vp, u64, u32, u64, vp, u32, u32, vp, vp, u32, dbl,
                                       vp, vp]
        L.ddo_groundtruth.restype = i32
        L.ddo_groundtruth.argtypes = [i32, i32, vp, u64, u32, u64, vp, u64, u64, u32, i32, vp, vp]
        L.ddo_schedule.restype = u64
        L.ddo_schedule.argtypes = [u64, u64, dbl, i32, vp, vp, u64]
        L.ddo_shard_search_prune.restype = i32
        L.ddo_shard_search_prune.argtypes = [i32, i32, vp, u64, u32, u64, vp, u32, u32, dbl, u32,
                                             u64, u64, i32, vp]
        L.ddo_shard_apply_reverse.restype = i32
        L.ddo_shard_apply_reverse.argtypes = [i32, i32, vp, u64, u32, u64, vp, u32, dbl, u64, u64,
                                              vp, u32, u32, i32, vp, vp, u64, vp]
        L.ddo_shard_set_rows.restype = i32
        L.ddo_shard_set_rows.argtypes = [vp, u64, u32, vp, vp, u64]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _pts(points: np.ndarray):
    points = np.ascontiguousarray(points)
    return points, DTYPES[points.dtype], points.shape[0], points.shape[1], points.strides[0]


def distance(a: np.ndarray, b: np.ndarray, metric: str = "l2") -> float:
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    return float(lib().ddo_distance(DTYPES[a.dtype], METRICS[metric], _p(a), _p(b), a.shape[-1]))


def build(points, R, L, alpha, metric="l2", xita=1.0, max_build=0, start=0, two_pass=False,
          knn_mode=False, nthreads=0):
    """Batched Vamana build; returns (graph n x (R+1) uint32, stats dict)."""
    points, dt, n, d, stride = _pts(points)
    g = np.zeros((n, R + 1), dtype=np.uint32)
    st = np.zeros(6, dtype=np.uint64)
    rc = lib().ddo_build(dt, METRICS[metric], _p(points), n, d, stride, R, L, float(alpha),
                         float(xita), int(max_build), int(start), int(two_pass), int(knn_mode),
                         int(nthreads), _p(g), _p(st))
    if rc != 0:
        raise ValueError(f"oracle build failed ({rc})")
    keys = ["rounds", "visited", "dist_cmps", "groups", "reverse_prunes", "prune_cands"]
    return g, dict(zip(keys, (int(x) for x in st)))


def beam_search(points, graph, query, L, k=0, cut=0.0, metric="l2", self_id=-1, start=0,
                limit=0, degree_limit=0, vis_cap=1 << 16):
    points, dt, n, d, stride = _pts(points)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    R = graph.shape[1] - 1
    q = np.ascontiguousarray(query, dtype=points.dtype)
    fr_i = np.zeros(L + R + 1, np.uint32)
    fr_d = np.zeros(L + R + 1, np.float32)
    vi_i = np.zeros(vis_cap, np.uint32)
    vi_d = np.zeros(vis_cap, np.float32)
    nf = np.zeros(1, np.uint32)
    nv = np.zeros(1, np.uint32)
    cm = np.zeros(1, np.uint64)
    rc = lib().ddo_beam_search(dt, METRICS[metric], _p(points), n, d, stride, _p(graph), R, _p(q),
                               int(self_id), int(start), int(k), int(L), float(cut), int(limit),
                               int(degree_limit), _p(fr_i), _p(fr_d), _p(nf), _p(vi_i), _p(vi_d),
                               _p(nv), vis_cap, _p(cm))
    if rc != 0:
        raise ValueError("visited list larger than vis_cap")
    a, b = int(nf[0]), int(nv[0])
    return (fr_i[:a].copy(), fr_d[:a].copy()), (vi_i[:b].copy(), vi_d[:b].copy()), int(cm[0])


def search(points, graph, queries, k, L, cut=1.35, metric="l2", start=0, limit=0,
           degree_limit=0, nthreads=0):
    """searchAll; L may be an int or a per-query array. Returns (ids, visited, cmps)."""
    points, dt, n, d, stride = _pts(points)
    queries = np.ascontiguousarray(queries, dtype=points.dtype)
    nq = queries.shape[0]
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    Ls = np.broadcast_to(np.asarray(L, dtype=np.uint32), (nq,)).copy()
    ids = np.zeros((nq, k), np.uint32)
    vis = np.zeros(nq, np.uint32)
    cm = np.zeros(nq, np.uint32)
    lib().ddo_search(dt, METRICS[metric], _p(points), n, d, stride, _p(graph), graph.shape[1] - 1,
                     _p(queries), nq, queries.strides[0], _p(Ls), int(k), float(cut), int(limit),
                     int(degree_limit), int(start), int(nthreads), _p(ids), _p(vis), _p(cm))
    return ids, vis, cm


def robust_prune(points, graph, p, cand_ids, cand_d, alpha, metric="l2"):
    points, dt, n, d, stride = _pts(points)
    graph = np.ascontiguousarray(graph, dtype=np.uint32)
    R = graph.shape[1] - 1
    ci = np.ascontiguousarray(cand_ids, dtype=np.uint32)
    cd = np.ascontiguousarray(cand_d, dtype=np.float32)
    out = np.zeros(R, np.uint32)
    ol = np.zeros(1, np.uint32)
    lib().ddo_robust_prune(dt, METRICS[metric], _p(points), n, d, stride, _p(graph), R, int(p),
                           _p(ci), _p(cd), len(ci), float(alpha), _p(out), _p(ol))
    return out[: int(ol[0])].copy()


def groundtruth(points, queries, k, metric="l2", nthreads=0):
    points, dt, n, d, stride = _pts(points)
    queries = np.ascontiguousarray(queries, dtype=points.dtype)
    nq = queries.shape[0]
    ids = np.zeros((nq, k), np.uint32)
    ds = np.zeros((nq, k), np.float32)
    lib().ddo_groundtruth(dt, METRICS[metric], _p(points), n, d, stride, _p(queries), nq,
                          queries.strides[0], k, int(nthreads), _p(ids), _p(ds))
    return ids, ds


class ShardRankOracle:
    """One rank of the sharded build on the CPU oracle (the per-round steps of
    distributed_diskann_b200.sharded's protocol); rows in the reference layout
    n x (R+1), row[0] = degree.  Test infrastructure, like the rest of this module."""

    def __init__(self, points, R, L, alpha, metric="l2", start=0, nthreads=0):
        self.points, self.dt, self.n, self.d, self.stride = _pts(points)
        self.R, self.L, self.alpha, self.metric, self.start = R, L, alpha, metric, start
        self.nthreads = nthreads
        self.graph = np.zeros((self.n, R + 1), np.uint32)
        self.row_len = R + 1

    def search_prune(self, lo, hi):
        rows = np.zeros((hi - lo, self.R + 1), np.uint32)
        rc = lib().ddo_shard_search_prune(self.dt, METRICS[self.metric], _p(self.points), self.n,
                                          self.d, self.stride, _p(self.graph), self.R, self.L,
                                          float(self.alpha), self.start, lo, hi, self.nthreads,
                                          _p(rows))
        if rc != 0:
            raise ValueError("oracle shard search/prune failed")
        return rows

    def apply_reverse(self, floor, ceiling, batch_rows, rank, world):
        batch_rows = np.ascontiguousarray(batch_rows, np.uint32)
        cap = batch_rows.shape[0] * self.R + 1
        ids = np.zeros(cap, np.uint32)
        rows = np.zeros((cap, self.R + 1), np.uint32)
        cnt = np.zeros(1, np.uint64)
        rc = lib().ddo_shard_apply_reverse(self.dt, METRICS[self.metric], _p(self.points), self.n,
                                           self.d, self.stride, _p(self.graph), self.R,
                                           float(self.alpha), floor, ceiling, _p(batch_rows), rank,
                                           world, self.nthreads, _p(ids), _p(rows), cap, _p(cnt))
        if rc != 0:
            raise ValueError("oracle shard reverse failed")
        c = int(cnt[0])
        return ids[:c].copy(), rows[:c].copy()

    def set_rows(self, ids, rows):
        ids = np.ascontiguousarray(ids, np.uint32)
        rows = np.ascontiguousarray(rows, np.uint32)
        if lib().ddo_shard_set_rows(_p(self.graph), self.n, self.R, _p(ids), _p(rows),
                                    len(ids)) != 0:
            raise ValueError("bad row id")


def schedule(n, max_build=0, xita=1.0, knn_mode=False):
    cap = 4096
    f = np.zeros(cap, np.uint64)
    c = np.zeros(cap, np.uint64)
    r = int(lib().ddo_schedule(n, max_build, float(xita), int(knn_mode), _p(f), _p(c), cap))
    return [(int(f[i]), int(c[i])) for i in range(min(r, cap))]


# ------------------------------------------------------------------ file I/O
def write_bin(path: str, x: np.ndarray) -> None:
    """Reference .bin layout: [u32 n][u32 d][n*d elements] (include/utils/point_range.h:61-97)."""
    x = np.ascontiguousarray(x)
    with open(path, "wb") as f:
        np.array(x.shape, dtype=np.uint32).tofile(f)
        x.tofile(f)


def read_graph(path: str) -> np.ndarray:
    """Reference graph file (include/utils/graph.h:178-200) -> n x (R+1) rows."""
    raw = np.fromfile(path, dtype=np.uint32)
    n, R = int(raw[0]), int(raw[1])
    deg = raw[2 : 2 + n]
    edges = raw[2 + n :]
    g = np.zeros((n, R + 1), dtype=np.uint32)
    g[:, 0] = deg
    off = np.concatenate([[0], np.cumsum(deg.astype(np.int64))])
    for lo in range(0, n, 1 << 20):  # blocks of rows, vectorised inside a block
        hi = min(n, lo + (1 << 20))
        d = deg[lo:hi].astype(np.int64)
        rows = np.repeat(np.arange(lo, hi), d)
        cols = np.arange(off[hi] - off[lo]) - np.repeat(off[lo:hi] - off[lo], d) + 1
        g[rows, cols] = edges[off[lo] : off[hi]]
    return g


def write_graph(path: str, g: np.ndarray) -> None:
    n, R1 = g.shape
    with open(path, "wb") as f:
        np.array([n, R1 - 1], dtype=np.uint32).tofile(f)
        g[:, 0].astype(np.uint32).tofile(f)
        mask = np.arange(R1 - 1)[None, :] < g[:, :1]
        g[:, 1:][mask].astype(np.uint32).tofile(f)


# ------------------------------------------------------------------ reference runs
def _run_ref(args, threads=0):
    env = dict(os.environ)
    if threads:
        env["PARLAY_NUM_THREADS"] = str(threads)
    # knn_index::batch_insert opens ./parlay_graph_log (include/index.h:224): run elsewhere
    with tempfile.TemporaryDirectory() as cwd:
        r = subprocess.run([REF_HARNESS] + [str(a) for a in args], capture_output=True, env=env,
                           check=True, cwd=cwd)
    return r.stdout.decode("utf-8", "replace")


def _parse_seconds(out: str, tag: str) -> float:
    for line in out.splitlines():
        if line.startswith(tag):
            return float(line.split()[1])
    return float("nan")


def ref_build(points, R, L, alpha, metric="l2", xita=1.0, max_build=0, start=0, threads=0,
              knn_mode=False, two_pass=False):
    """Run the reference's own BSP build (or knn_index build); returns (graph, seconds)."""
    points = np.ascontiguousarray(points)
    dt = DTYPE_NAMES[DTYPES[points.dtype]]
    with tempfile.TemporaryDirectory() as td:
        base = os.path.join(td, "base.bin")
        gout = os.path.join(td, "graph.bin")
        write_bin(base, points)
        if knn_mode:
            out = _run_ref(["knnbuild", dt, metric, base, R, L, alpha, int(two_pass), gout], threads)
        else:
            out = _run_ref(["build", dt, metric, base, R, L, alpha, xita, max_build, start, gout],
                           threads)
        return read_graph(gout), _parse_seconds(out, "HARNESS_BUILD_SECONDS")


def ref_search(points, graph, queries, k, L, cut=1.35, metric="l2", start=0, limit=0,
               degree_limit=0, threads=0):
    points = np.ascontiguousarray(points)
    dt = DTYPE_NAMES[DTYPES[points.dtype]]
    nq = queries.shape[0]
    with tempfile.TemporaryDirectory() as td:
        base, qf, gf, of = (os.path.join(td, x) for x in ("b.bin", "q.bin", "g.bin", "o.bin"))
        write_bin(base, points)
        write_bin(qf, np.ascontiguousarray(queries, dtype=points.dtype))
        write_graph(gf, graph)
        out = _run_ref(["search", dt, metric, base, gf, qf, k, L, cut, limit, degree_limit, start,
                        of], threads)
        raw = np.fromfile(of, dtype=np.uint32)
        ids = raw[: nq * k].reshape(nq, k).copy()
        vis = raw[nq * k : nq * k + nq]
        cmps = raw[nq * k + nq : nq * k + 2 * nq]
        fsz = raw[nq * k + 2 * nq : nq * k + 3 * nq]
        # entries past the final frontier are undefined in the reference: mask them
        ids[np.arange(k)[None, :] >= fsz[:, None]] = 0xFFFFFFFF
        return ids, vis, cmps, _parse_seconds(out, "HARNESS_SEARCH_SECONDS")


def ref_qps(points, graph, queries, k, Ls, cut=1.35, metric="l2", start=0, threads=0):
    """The reference's searchAll timed like checkRecall (untimed pass, then a
    timed one) for each beam width in Ls, on one loaded index.  Returns
    {L: (ids nq x k, seconds)}; ids past a short final frontier are undefined
    in the reference and are not masked here."""
    points = np.ascontiguousarray(points)
    dt = DTYPE_NAMES[DTYPES[points.dtype]]
    nq = queries.shape[0]
    with tempfile.TemporaryDirectory() as td:
        base, qf, gf, of = (os.path.join(td, x) for x in ("b.bin", "q.bin", "g.bin", "o.bin"))
        write_bin(base, points)
        write_bin(qf, np.ascontiguousarray(queries, dtype=points.dtype))
        write_graph(gf, graph)
        out = _run_ref(["qps", dt, metric, base, gf, qf, k, cut, start,
                        ",".join(str(int(L)) for L in Ls), of], threads)
        raw = np.fromfile(of, dtype=np.uint32)
    secs = {}
    for line in out.splitlines():
        if line.startswith("HARNESS_QPS"):
            _, L, s = line.split()
            secs[int(L)] = float(s)
    res = {}
    for i, L in enumerate(Ls):
        res[int(L)] = (raw[i * nq * k : (i + 1) * nq * k].reshape(nq, k).copy(), secs[int(L)])
    return res


def ref_beam(points, graph, queries, k, L, cut=0.0, metric="l2", start=0, limit=0,
             degree_limit=0):
    points = np.ascontiguousarray(points)
    dt = DTYPE_NAMES[DTYPES[points.dtype]]
    with tempfile.TemporaryDirectory() as td:
        base, qf, gf, of = (os.path.join(td, x) for x in ("b.bin", "q.bin", "g.bin", "o.bin"))
        write_bin(base, points)
        write_bin(qf, np.ascontiguousarray(queries, dtype=points.dtype))
        write_graph(gf, graph)
        _run_ref(["beam", dt, metric, base, gf, qf, k, L, cut, limit, degree_limit, start, of])
        raw = np.fromfile(of, dtype=np.uint32)
    res, pos = [], 0
    for _ in range(queries.shape[0]):
        nf, nv, cm = (int(x) for x in raw[pos : pos + 3])
        pos += 3
        fr = raw[pos : pos + 2 * nf].reshape(nf, 2)
        pos += 2 * nf
        vi = raw[pos : pos + 2 * nv].reshape(nv, 2)
        pos += 2 * nv
        res.append(((fr[:, 0].copy(), fr[:, 1].view(np.float32).copy()),
                    (vi[:, 0].copy(), vi[:, 1].view(np.float32).copy()), cm))
    return res
