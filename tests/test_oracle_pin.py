"""Pin the CPU oracle to the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py from the reference sources).  CPU only."""
import hashlib

import numpy as np
import pytest

from distributed_diskann_b200 import datasets as D
from tests.golden.make_golden import BUILD_CASES, case_inputs, canon, sha


@pytest.mark.parametrize("name", list(BUILD_CASES))
def test_oracle_build_and_search_match_reference(oracle_mod, golden, name):
    O = oracle_mod
    g, arrays = golden
    rec = g["cases"][name]
    R, L, alpha, metric, xita, mx, st, knn, tp, Ls = BUILD_CASES[name]
    base, queries = case_inputs(name)
    assert sha(base) == rec["input_sha256"], "input generator changed"
    graph, stats = O.build(base, R, L, alpha, metric=metric, xita=xita, max_build=mx, start=st,
                           knn_mode=knn, two_pass=tp)
    graph = canon(graph)
    if f"{name}__graph" in arrays:
        np.testing.assert_array_equal(graph, arrays[f"{name}__graph"])
    assert sha(graph) == rec["graph_sha256"]
    for Ls_, s in rec["search"].items():
        ids, vis, cmps = O.search(base, graph, queries, s["k"], int(Ls_), cut=1.35, metric=metric,
                                  start=st)
        assert sha(ids) == s["ids_sha256"], f"search L={Ls_}"
        assert int(vis.sum()) == s["visited_sum"]
        assert int(cmps.sum()) == s["cmps_sum"]


def test_oracle_robust_prune_matches_reference(oracle_mod, golden):
    O = oracle_mod
    g, arrays = golden
    base, _ = case_inputs("i8_small")
    graph, _ = O.build(base, 64, 128, 1.2)
    graph = canon(graph)
    assert sha(graph) == g["cases"]["i8_small"]["graph_sha256"]
    for t in range(g["prune_cases"]):
        p = int(arrays[f"prune{t}__p"][0])
        out = O.robust_prune(base, graph, p, arrays[f"prune{t}__cand"], arrays[f"prune{t}__dist"],
                             1.2)
        np.testing.assert_array_equal(out, arrays[f"prune{t}__out"], err_msg=f"prune case {t}")


def test_oracle_beam_search_matches_reference(oracle_mod, golden):
    O = oracle_mod
    g, arrays = golden
    base, queries = case_inputs("i8_small")
    graph = canon(O.build(base, 64, 128, 1.2)[0])
    for mode, (k, L, cut) in {"build": (0, 128, 0.0), "query": (10, 50, 1.35)}.items():
        for i in range(g["beam_cases"]):
            fr, vi, cm = O.beam_search(base, graph, queries[i], L, k=k, cut=cut, self_id=i)
            np.testing.assert_array_equal(fr[0], arrays[f"beam_{mode}{i}__fr_ids"])
            np.testing.assert_array_equal(fr[1], arrays[f"beam_{mode}{i}__fr_d"])
            np.testing.assert_array_equal(vi[0], arrays[f"beam_{mode}{i}__vi_ids"])
            np.testing.assert_array_equal(vi[1], arrays[f"beam_{mode}{i}__vi_d"])
            assert cm == int(arrays[f"beam_{mode}{i}__cmps"][0])


def test_shipped_random_xs_fixture_regenerates(oracle_mod, golden):
    """The reference's data/random10000 files are regenerated bit-exactly, and the
    oracle reproduces the reference's recall@10 on them (check_nn_recall.h:86-108)."""
    g, _ = golden
    rec = g.get("shipped_random_xs")
    if rec is None:
        pytest.skip("golden made without the reference data")
    base, queries = D.random_xs_like_reference()
    hdr = np.array(base.shape, np.uint32).tobytes()
    assert hashlib.sha256(hdr + base.tobytes()).hexdigest() == rec["data_file_sha256"]
    qh = np.array(queries.shape, np.uint32).tobytes()
    assert hashlib.sha256(qh + queries.tobytes()).hexdigest() == rec["queries_file_sha256"]
    from sklearn.neighbors import NearestNeighbors

    nbrs = NearestNeighbors(n_neighbors=100, metric="euclidean", algorithm="brute").fit(base)
    Dd, I = nbrs.kneighbors(queries)
    gi, gd = I.astype(np.uint32), Dd.astype(np.float32)
    assert sha(gi) == rec["gt_ids_sha256"]
    O = oracle_mod
    graph = canon(O.build(base, 32, 64, 1.2)[0])
    for Ls_, r in rec["recall10"].items():
        ids = O.search(base, graph, queries, 10, int(Ls_), cut=1.35)[0]
        assert D.recall_with_ties(ids, gi, gd, 10) == pytest.approx(r, abs=0)


def test_oracle_schedule(oracle_mod):
    O = oracle_mod
    s = O.schedule(10_000)
    assert s[0] == (0, 1) and s[1] == (1, 3) and s[13] == (8191, 9999) and s[14] == (9999, 10000)
    assert len(s) == 15
    s = O.schedule(10_000_000, xita=1.0)
    assert sum(c - f for f, c in s) == 10_000_000
    assert all(c - f <= 1_000_000 for f, c in s)
    s = O.schedule(5_000, max_build=4_000, xita=0.02)
    assert s[-1][1] == 4_000 and max(c - f for f, c in s) == 80


def test_oracle_matches_full_size_reference_build_with_limits(oracle_mod):
    """The oracle at the full size of the 100,000 x 64 f32 mixture workload
    (R=48, L=96, alpha=1.2) against the reference's own build of the same
    points (tests/golden/golden_full.json, made by make_golden_full.py from the
    unmodified sources): the graph digest, and searchAll's ids and visited /
    dist_cmps sums at several beam widths with and without `limit` (stop after
    that many visits, include/utils/beamSearch.h:108) and `degree_limit`
    (scan only the first neighbours of a row, :123)."""
    import json
    import os

    from tests.golden.make_golden_full import case_data

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_full.json")
    rec = json.load(open(here))["cases"]["mix64-f32"]
    w = D.WORKLOADS["mix64-f32"]
    base, queries = case_data("mix64-f32")
    assert sha(base) == rec["input_sha256"], "input generator changed"
    graph, _ = oracle_mod.build(base, w.R, w.L, w.alpha, metric=w.metric)
    graph = canon(graph)
    assert sha(graph) == rec["graph_sha256"]
    q = queries[: rec["nsearch"]]
    assert any(s["limit"] for s in rec["search"]) and any(s["degree_limit"] for s in rec["search"])
    for s in rec["search"]:
        ids, vis, cmps = oracle_mod.search(base, graph, q, s["k"], s["L"], cut=1.35,
                                           metric=w.metric, limit=s["limit"],
                                           degree_limit=s["degree_limit"])
        tag = f"L={s['L']} limit={s['limit']} degree_limit={s['degree_limit']}"
        assert sha(ids) == s["ids_sha256"], tag
        assert int(vis.sum()) == s["visited_sum"], tag
        assert int(cmps.sum()) == s["cmps_sum"], tag
