"""The recall sweep of the reference (search_and_parse, checkRecall,
parse_result, stats::statistics, calculate_limits: include/utils/
check_nn_recall.h, parse_results.h, stats.h) on the host, driven by a
deterministic stand-in searcher so that no GPU is needed: its beam widths,
limits and degree limits, the tie-aware recall, the bucket selection and the
CSV layout."""
import csv

import numpy as np

from distributed_diskann_b200 import recall as RC


def test_statistics_and_limits_follow_the_reference_arithmetic():
    # avg = (int)sum / (double)n truncated; tail = sorted[(size_t)(.99 * (float)n)]
    assert RC.statistics([5, 1, 3, 2, 100]) == (22, 100)
    assert RC.statistics(list(range(1000))) == (499, 990)
    # (long)(i * (float)ub * .1), i = 1..9, duplicates removed
    assert RC.calculate_limits(64) == [6, 12, 19, 25, 32, 38, 44, 51, 57]
    assert RC.calculate_limits(5) == [0, 1, 2, 3, 4]
    assert RC.calculate_limits(10) == [1, 2, 3, 4, 5, 6, 7, 8, 9]


def _res(recall, qps, beam=10):
    return RC.NNResult(recall, 0, 0, 0, 0, qps, 10, beam, 1.35, 0, 0, 100)


def test_parse_result_keeps_the_fastest_run_per_bucket():
    runs = [_res(0.50, 900.0, 20), _res(0.55, 1000.0, 18), _res(0.94, 50.0, 100),
            _res(0.96, 40.0, 150), _res(0.96, 45.0, 160)]
    best, buckets = RC.parse_result(runs, (0.5, 0.6, 0.95, 0.97))
    # 0.5: recall in [0.5, 0.6] -> the faster of the first two; 0.6: [0.6, 0.95]
    # -> 0.94; 0.95: [0.95, 0.97] -> the faster 0.96 run; 0.97 (last): none
    assert buckets == [0.5, 0.6, 0.95]
    assert [r.beam for r in best] == [18, 100, 160]
    # the upper filter applies whenever runs reach the bucket: a run above the
    # next bucket counts only there (the last bucket has no upper filter)
    best, buckets = RC.parse_result([_res(0.99, 10.0, 300)], (0.5, 0.6))
    assert buckets == [0.6] and [r.beam for r in best] == [300]


def _fake_search(gt_ids, calls):
    """searchAll stand-in: finds more of the true neighbours as the beam grows,
    fewer under a visit limit or a degree limit; visited and cmps grow with them."""
    def search(QP):
        calls.append((QP.k, QP.beamSize, QP.cut, QP.limit, QP.degree_limit))
        nq = gt_ids.shape[0]
        good = min(QP.k, QP.beamSize // 10, QP.limit // 3, QP.degree_limit // 6)
        ids = np.full((nq, QP.k), 10 ** 6, np.uint32)
        ids[:, :good] = gt_ids[:, :good]
        visited = np.minimum(QP.beamSize + np.arange(nq) % 7, QP.limit).astype(np.uint32)
        cmps = (visited * min(QP.degree_limit, 32)).astype(np.uint32)
        return ids, visited, cmps
    return search


def test_search_and_parse_runs_the_reference_sweep(tmp_path):
    nq, n, R, k = 50, 10_000, 64, 10
    rng = np.random.default_rng(0)
    gt_ids = rng.choice(n, (nq, 32)).astype(np.uint32)
    gt_d = np.sort(rng.random((nq, 32)).astype(np.float32), axis=1)
    calls = []
    out = tmp_path / "sweep.csv"
    sw = RC.search_and_parse(_fake_search(gt_ids, calls), n, R, gt_ids, gt_d, k=k,
                             res_file=str(out), graph_name="vamana", graph_size=n)
    # beams > k from the reference's list, each searched twice (the second timed)
    beams = [q for q in RC.BEAMS if q > k and q <= RC.MAX_BEAM]
    assert [c[1] for c in calls[: 2 * len(beams): 2]] == beams
    assert all(calls[2 * i] == calls[2 * i + 1] for i in range(len(calls) // 2))
    assert all(c[3] == n and c[4] == R and c[2] == 1.35 for c in calls[: 2 * len(beams)])
    # then limits from the first run's average visited count x degree limits
    first = sw.results[0]
    assert first.beam == 11 and first.avg_visited == 13  # (int)(11 + mean(arange(50) % 7))
    lim = RC.calculate_limits(first.avg_visited)
    dl = RC.calculate_limits(R) + [R]
    expect = [(k, max(l, k), 1.35, l, d) for l in lim for d in dl if l > 0]
    assert calls[2 * len(beams):: 2] == expect
    # beams above 512 and the k = 100 "best accuracy" run are outside the C ABI
    why = [w for _, w in sw.skipped]
    assert sum("beam width" in w for w in why) == 3  # 750, 1000, best accuracy (1000)
    assert len(sw.results) == len(beams) + len(expect)
    # recall with ties; the fastest run of each bucket in the CSV
    assert sw.results[0].recall == 0.1  # good = 11 // 10 = 1 of 10
    assert max(r.recall for r in sw.results) == 1.0
    rows = list(csv.reader(open(out)))
    assert rows[0][0] == "GRAPH" and rows[1][0] == "vamana" and rows[1][5] == str(R)
    assert rows[3][:4] == ["Num queries", "Target recall", "Actual recall", "QPS"]
    body = [r for r in rows[4:] if r]
    assert len(body) == len(sw.best) == len(sw.buckets)
    assert [float(r[1]) for r in body] == sw.buckets
