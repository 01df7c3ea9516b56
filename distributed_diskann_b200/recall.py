"""The reference's recall sweep (include/utils/check_nn_recall.h,
include/utils/parse_results.h, include/utils/stats.h) over the GPU searches.

``search_and_parse`` runs searchAll over a sweep of beam widths, then of visit
limits and degree limits, then the reference's "best accuracy" setting, scores
each run with the tie-aware recall of ``checkRecall``, keeps the fastest run per
recall bucket (``parse_result``) and writes the reference's CSV layout
(``write_to_csv``).  The searches are the GPU index's ``dd_search`` calls; the
sweep logic only sees a callable, so any searcher with searchAll's outputs can
drive it.

Limits of this library that the sweep runs into: beam widths above 512 and k
above 32 are rejected by the C ABI (``DD_ERR_UNSUPPORTED``), and a visit limit or
degree limit of 0 means "no limit" there while the reference then visits or
scans nothing.  Settings outside those bounds are left out of the sweep and
listed in ``SweepResult.skipped``.
"""
from __future__ import annotations

import csv
import time
from dataclasses import dataclass, field

import numpy as np

from .datasets import recall_with_ties
from .index import QueryParams

MAX_BEAM = 512
MAX_K = 32

# check_nn_recall.h:171-174, :213-215
BEAMS = (10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 22, 24, 26, 28, 30, 32, 34, 36, 38, 40, 45,
         50, 55, 60, 65, 70, 80, 90, 100, 120, 140, 160, 180, 200, 225, 250, 275, 300, 375, 500,
         750, 1000)
BUCKETS = (.1, .2, .3, .4, .5, .6, .7, .75, .8, .85, .9, .93, .95, .97, .98, .99, .995, .999,
           .9995, .9999, .99995, .99999)


@dataclass
class NNResult:
    """nn_result (include/utils/parse_results.h:124-161)."""
    recall: float
    avg_cmps: int
    tail_cmps: int
    avg_visited: int
    tail_visited: int
    qps: float
    k: int
    beam: int
    cut: float
    limit: int
    degree_limit: int
    num_queries: int


@dataclass
class SweepResult:
    results: list          # every run, in sweep order
    best: list             # parse_result: the fastest run per recall bucket
    buckets: list          # the buckets that had a run
    skipped: list = field(default_factory=list)  # (QueryParams, reason)


def statistics(values) -> tuple[int, int]:
    """stats::statistics (include/utils/stats.h:78-86): the average, truncated
    to an integer, and the entry at 0.99 of the sorted values."""
    s = np.sort(np.asarray(values, dtype=np.int64))
    avg = int(int(s.sum()) / float(s.size))
    tail = int(s[int(0.99 * float(np.float32(s.size)))])  # .99 (double) * (float)size
    return avg, tail


def calculate_limits(upper_bound: int) -> list[int]:
    """check_nn_recall.h:148-155: (long)(i * (float)upper_bound * .1) for
    i = 1..9, without duplicates (ascending)."""
    vals = [int(float(np.float32(i) * np.float32(upper_bound)) * .1) for i in range(1, 10)]
    return sorted(set(vals))


def check_recall(search, gt_ids, gt_dists, k: int, QP: QueryParams) -> NNResult:
    """checkRecall (check_nn_recall.h:33-114): searchAll runs twice and the
    second run is timed; recall counts ground-truth ties at the k-th distance.
    ``search(QP)`` returns (ids nq x k, visited per query, dist_cmps per query)."""
    if k > gt_ids.shape[1]:
        raise ValueError(f"{k}@{k} too large for ground truth data of size {gt_ids.shape[1]}")
    search(QP)
    t0 = time.perf_counter()
    ids, visited, cmps = search(QP)
    secs = time.perf_counter() - t0
    nq = ids.shape[0]
    rec = recall_with_ties(ids, gt_ids, gt_dists, k)
    ac, tc = statistics(cmps)
    av, tv = statistics(visited)
    return NNResult(rec, ac, tc, av, tv, nq / secs if secs > 0 else float("inf"), k,
                    QP.beamSize, QP.cut, QP.limit, QP.degree_limit, nq)


def parse_result(results, buckets=BUCKETS):
    """parse_result (include/utils/parse_results.h:213-238): per bucket b, the
    runs with recall >= b (and <= the next bucket, unless that leaves none or b
    is the last), and of those the first with the highest QPS."""
    best, ret_buckets = [], []
    for i, b in enumerate(buckets):
        cand = [r for r in results if r.recall >= b]
        if i != len(buckets) - 1 and cand:
            c = buckets[i + 1]
            cand = [r for r in cand if r.recall <= c]
        if cand:
            m = cand[0]
            for r in cand[1:]:
                if m.qps < r.qps:
                    m = r
            best.append(m)
            ret_buckets.append(b)
    return best, ret_buckets


def write_to_csv(path, buckets, results, graph_name="", graph_params="", graph_size=0,
                 build_time=0.0, avg_deg=0.0, max_deg=0):
    """write_to_csv (check_nn_recall.h:116-146)."""
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["GRAPH", "Parameters", "Size", "Build time", "Avg degree", "Max degree"])
        w.writerow([graph_name, graph_params, graph_size, build_time, avg_deg, max_deg])
        w.writerow([])
        w.writerow(["Num queries", "Target recall", "Actual recall", "QPS", "Average Cmps",
                    "Tail Cmps", "Average Visited", "Tail Visited", "k", "Q", "cut"])
        for b, r in zip(buckets, results):
            w.writerow([r.num_queries, b, r.recall, r.qps, r.avg_cmps, r.tail_cmps,
                        r.avg_visited, r.tail_visited, r.k, r.beam, r.cut])
        w.writerow([])
        w.writerow([])


def _supported(QP: QueryParams):
    if QP.beamSize > MAX_BEAM:
        return f"beam width {QP.beamSize} > {MAX_BEAM}"
    if QP.k > MAX_K:
        return f"k {QP.k} > {MAX_K}"
    if QP.limit <= 0 or QP.degree_limit <= 0:
        return "a limit of 0 (the reference visits or scans nothing; here 0 means no limit)"
    return None


def search_and_parse(search, n: int, max_degree: int, gt_ids, gt_dists, k: int = 10,
                     res_file: str | None = None, beams=BEAMS, **graph_info) -> SweepResult:
    """search_and_parse (check_nn_recall.h:157-217) for one k (0 means 10)."""
    r = 10 if k == 0 else k
    results, skipped = [], []

    def run(QP):
        why = _supported(QP)
        if why:
            skipped.append((QP, why))
            return
        results.append(check_recall(search, gt_ids, gt_dists, r, QP))

    for Q in beams:  # the beam-width sweep at cut 1.35
        if Q > r:
            run(QueryParams(r, Q, 1.35, n, max_degree))
    if results:  # "limited accuracy": visit and degree limits
        limits = calculate_limits(results[0].avg_visited)
        dlimits = calculate_limits(max_degree) + [max_degree]
        for lim in limits:
            for dl in dlimits:
                run(QueryParams(r, max(lim, r), 1.35, lim, dl))
    run(QueryParams(100, 1000, 10.0, n, max_degree))  # "best accuracy"
    best, buckets = parse_result(results)
    if res_file is not None:
        write_to_csv(res_file, buckets, best, max_deg=max_degree, **graph_info)
    return SweepResult(results, best, buckets, skipped)


def gpu_searcher(gi, queries, start: int = 0):
    """searchAll on a GpuIndex (dd_search) in the sweep's calling form.  Each
    call copies the queries to the device and the results back, as the
    reference's timed searchAll takes host queries; bench.py times the device
    search alone (dd_search_device) for its QPS figures."""
    def search(QP: QueryParams):
        ids, _, vis, cmps = gi.search(queries, QP.k, QP.beamSize, cut=QP.cut, limit=QP.limit,
                                      degree_limit=QP.degree_limit, start=start)
        return ids, vis, cmps
    return search
