"""GPU parity: the CUDA path (through the C ABI) against the reference's own
outputs (tests/golden/, pinned) and against the CPU oracle on the same seeded
inputs.  Integer AND float graphs are compared bit-exactly: the kernels
reproduce the reference's float summation order, its tie orders (std::sort
emulation) and its lossy hash filter, so no tolerance is needed."""
import numpy as np
import pytest

from distributed_diskann_b200 import datasets as D
from distributed_diskann_b200.index import GpuIndex
from tests.golden.make_golden import BUILD_CASES, case_inputs, canon, sha

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def gpu_build(base, R, L, alpha, metric="l2", **kw):
    gi = GpuIndex(base.dtype, metric, base.shape[0], base.shape[1], R)
    gi.upload_points(base)
    st = gi.build(L, alpha, **kw)
    return gi, canon(gi.graph()), st


@pytest.mark.parametrize("mode", ["fast", "plain"])
@pytest.mark.parametrize("name", list(BUILD_CASES))
def test_build_and_search_bit_exact_vs_reference(golden, name, mode):
    """Both computation forms (DD_MODE_FAST, DD_MODE_PLAIN) against the reference."""
    g, arrays = golden
    rec = g["cases"][name]
    R, L, alpha, metric, xita, mx, st, knn, tp, Ls = BUILD_CASES[name]
    base, queries = case_inputs(name)
    gi, graph, stats = gpu_build(base, R, L, alpha, metric=metric, max_fraction=xita, max_build=mx,
                                 start_point=st, knn_mode=knn, two_pass=tp, mode=mode)
    gi.set_search_mode(mode)
    if f"{name}__graph" in arrays:
        np.testing.assert_array_equal(graph, arrays[f"{name}__graph"])
    assert sha(graph) == rec["graph_sha256"], f"{name}: graph differs from the reference build"
    for Ls_, s in rec["search"].items():
        ids, dists, vis, cmps = gi.search(queries, s["k"], int(Ls_), cut=1.35, start=st)
        assert sha(ids) == s["ids_sha256"], f"{name}: search L={Ls_}"
        assert int(vis.sum()) == s["visited_sum"]
        assert int(cmps.sum()) == s["cmps_sum"]
    gi.close()


def test_build_stats_match_oracle(oracle_mod):
    """The plain form replays the reference's lossy seen filter, so even its
    dist_cmps count is the reference's.  The fast form's filter (set-associative
    16-bit tags of a bijective hash) gives the same graph and visited lists;
    only the number of re-evaluated neighbours, dist_cmps, differs: fewer,
    since its buckets keep tags longer than the reference's one-id slots."""
    base, _ = case_inputs("i8_small")
    og, ost = oracle_mod.build(base, 64, 128, 1.2)
    for mode in ("plain", "fast"):
        gi, graph, st = gpu_build(base, 64, 128, 1.2, mode=mode)
        np.testing.assert_array_equal(graph, canon(og))
        assert st["visited"] == ost["visited"]
        if mode == "plain":
            assert st["dist_cmps"] == ost["dist_cmps"]
        else:
            assert 0.5 < st["dist_cmps"] / ost["dist_cmps"] < 1.05
        assert st["groups"] == ost["groups"]
        assert st["reverse_prunes"] == ost["reverse_prunes"]
        assert st["prune_cands"] == ost["prune_cands"]
        gi.close()


def test_beam_search_frontier_and_visited_vs_reference(golden):
    g, arrays = golden
    base, queries = case_inputs("i8_small")
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    gi.upload_points(base)
    gi.build(128, 1.2)
    for mode, (k, L, cut) in {"build": (0, 128, 0.0), "query": (10, 50, 1.35)}.items():
        res = gi.beam_search(queries[: g["beam_cases"]], L, k=k, cut=cut,
                             self_ids=np.arange(g["beam_cases"]))
        for i, (fr, vi, cm) in enumerate(res):
            np.testing.assert_array_equal(fr[0], arrays[f"beam_{mode}{i}__fr_ids"])
            np.testing.assert_array_equal(fr[1], arrays[f"beam_{mode}{i}__fr_d"])
            np.testing.assert_array_equal(vi[0], arrays[f"beam_{mode}{i}__vi_ids"])
            np.testing.assert_array_equal(vi[1], arrays[f"beam_{mode}{i}__vi_d"])
            assert cm == int(arrays[f"beam_{mode}{i}__cmps"][0])
    gi.close()


def test_robust_prune_vs_reference(golden):
    g, arrays = golden
    base, _ = case_inputs("i8_small")
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    gi.upload_points(base)
    gi.build(128, 1.2)
    tasks = [(int(arrays[f"prune{t}__p"][0]), arrays[f"prune{t}__cand"], arrays[f"prune{t}__dist"])
             for t in range(g["prune_cases"])]
    outs = gi.robust_prune(tasks, 1.2)
    for t, o in enumerate(outs):
        np.testing.assert_array_equal(o, arrays[f"prune{t}__out"], err_msg=f"prune case {t}")
    gi.close()


@pytest.mark.parametrize("shape", ["runs", "runs_one_tie", "sorted_ties", "dense_ties"])
def test_robust_prune_run_shaped_lists_vs_oracle(oracle_mod, shape):
    """Candidate lists shaped like a reverse prune's: new sources in batch
    order, then an ascending run (the target's last selection), then a few
    appended sources.  The warp sort ranks these from the run; lists with more
    than 32 elements off the run, or with equal keys, take the other sort
    paths.  Lists with equal keys replay the library's introsort, whose order
    of equal keys the greedy selection depends on; ranges of such a list
    without tied elements are sorted directly: "sorted_ties" is an insert
    prune's list (ascending, a few equal neighbours), "dense_ties" has keys
    from a small range.  Keys below the points' typical distances leave most
    candidates unoccluded, so the first R places of the sorted list are all
    checked.  Every result must equal the oracle's robustPrune."""
    rng = np.random.default_rng({"runs": 17, "runs_one_tie": 23, "sorted_ties": 29,
                                 "dense_ties": 31}[shape])
    n, d, R = 5000, 64, 64
    base = rng.integers(0, 256, (n, d)).astype(np.uint8)
    gi = GpuIndex(base.dtype, "l2", n, d, R)
    gi.upload_points(base)  # rows stay empty: the lists are exactly the candidates
    empty = np.zeros((n, R + 1), np.uint32)
    tasks = []
    for t in range(300):
        p = int(rng.integers(n))
        s, run, app = int(rng.integers(0, 30)), int(rng.integers(1, 220)), int(rng.integers(0, 10))
        m = s + run + app
        ids = rng.choice(np.delete(np.arange(n), p), m, replace=False).astype(np.uint32)
        keys = rng.choice(200_000, m, replace=False).astype(np.float32)
        keys[s:s + run] = np.sort(keys[s:s + run])
        if shape == "runs_one_tie" and m > 1 and t % 2 == 0:
            a, b = rng.choice(m, 2, replace=False)
            keys[a] = keys[b]
        elif shape == "sorted_ties":
            keys = np.sort(rng.integers(0, 4 * m, m)).astype(np.float32)
        elif shape == "dense_ties":
            keys = rng.integers(0, max(2, m // 3), m).astype(np.float32) * 50.0
        tasks.append((p, ids, keys))
    outs = gi.robust_prune(tasks, 1.2)
    for t, (p, ids, keys) in enumerate(tasks):
        exp = oracle_mod.robust_prune(base, empty, p, ids, keys, 1.2)
        np.testing.assert_array_equal(outs[t], exp, err_msg=f"case {t}")
    gi.close()


@pytest.mark.parametrize("dtype,metric,d", [("f32", "l2", 40), ("f32", "mips", 40),
                                            ("i8", "l2", 40), ("u8", "l2", 40), ("i8", "mips", 40),
                                            ("u8", "mips", 40), ("i8", "l2", 100),
                                            ("u8", "l2", 128), ("u8", "l2", 200)])
def test_groundtruth_vs_oracle(oracle_mod, dtype, metric, d):
    """Brute force: FP64 for float data; integer rows of <= 128 bytes on the
    tensor cores (exact int32 Gram tiles), wider ones on the CUDA cores.  Small
    value ranges make many exact distance ties, which order by id."""
    rng = np.random.default_rng(7)
    if dtype == "f32":
        base = rng.standard_normal((20_000, d), dtype=np.float32)
        q = rng.standard_normal((300, d), dtype=np.float32)
    elif dtype == "i8":
        base = rng.integers(-128, 128, (20_000, d)).astype(np.int8)
        q = rng.integers(-128, 128, (300, d)).astype(np.int8)
    else:
        hi = 256 if d != 128 else 3  # d = 128: values 0..2, ties everywhere
        base = rng.integers(0, hi, (20_000, d)).astype(np.uint8)
        q = rng.integers(0, hi, (300, d)).astype(np.uint8)
    gi = GpuIndex(base.dtype, metric, base.shape[0], base.shape[1], 8)
    gi.upload_points(base)
    for k in (32, 10, 1):
        ids, ds = gi.groundtruth(q, k)
        oi, od = oracle_mod.groundtruth(base, q, k, metric=metric)
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(ds, od)
    gi.close()


@pytest.mark.parametrize("mode", ["fast", "plain"])
def test_mixed_beam_widths_in_one_call(golden, mode):
    """Mixed beam widths in one call: one launch sized for the largest width
    (plain form) or one persistent launch per beam-width class (fast form)."""
    g, _ = golden
    base, queries = case_inputs("i8_small")
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    gi.upload_points(base)
    gi.build(128, 1.2)
    gi.set_search_mode(mode)
    Ls = np.array([10, 20, 50, 100, 200], np.uint32)[np.arange(len(queries)) % 5]
    ids_mixed, _, vis_m, cm_m = gi.search(queries, 10, Ls)
    for L in (10, 20, 50, 100, 200):
        ids, _, vis, cm = gi.search(queries, 10, L)
        sel = Ls == L
        np.testing.assert_array_equal(ids_mixed[sel], ids[sel])
        np.testing.assert_array_equal(cm_m[sel], cm[sel])
    gi.close()


def test_graph_file_roundtrip(tmp_path, oracle_mod):
    base, _ = case_inputs("params_u8")
    gi, graph, _ = gpu_build(base, 16, 32, 1.2)
    gi.save_graph(str(tmp_path / "g.bin"))
    np.testing.assert_array_equal(oracle_mod.read_graph(str(tmp_path / "g.bin")), graph)
    gi2 = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 16)
    gi2.upload_points(base)
    gi2.load_graph(str(tmp_path / "g.bin"))
    np.testing.assert_array_equal(canon(gi2.graph()), graph)
    gi.close()
    gi2.close()


@pytest.mark.parametrize("R,L,metric", [(24, 48, "l2"), (64, 96, "l2"), (40, 64, "mips")])
def test_two_pass_graphs_and_their_queries_vs_oracle(oracle_mod, R, L, metric):
    """Two-pass builds append reverse edges to rows that may already hold the
    source, so rows carry duplicate ids and the lossy filter can let one id
    into a step twice: the frontier and visited lists become multisets."""
    both = D.gen_mixture_i8(6_300, 50, 100, 13)
    base, q = both[:6_000], both[6_000:]
    gi, graph, st = gpu_build(base, R, L, 1.2, metric=metric, two_pass=True)
    og, ost = oracle_mod.build(base, R, L, 1.2, metric=metric, two_pass=True)
    np.testing.assert_array_equal(graph, canon(og))
    assert st["visited"] == ost["visited"] and st["dist_cmps"] == ost["dist_cmps"]
    for Lq in (10, 50, 128):
        ids, _, vis, cm = gi.search(q, 10, Lq)
        oi, ov, oc = oracle_mod.search(base, graph, q, 10, Lq, metric=metric)
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(vis, ov)
        np.testing.assert_array_equal(cm, oc)
    gi.close()


def test_mid_size_int8_build_bit_exact_vs_oracle(oracle_mod):
    """100k x 100 int8 (the reference's own measured case) against the oracle.
    The start point collects more than 256 reverse-edge candidates, so the
    hub-target path (one CTA per target) is part of the comparison."""
    base = D.gen_mixture_i8(100_000, 100, 1000, 4)
    gi, graph, st = gpu_build(base, 64, 128, 1.2)
    og, ost = oracle_mod.build(base, 64, 128, 1.2)
    np.testing.assert_array_equal(graph, canon(og))
    assert st["big_groups"] > 0 and st["reverse_prunes"] > 0
    gi.close()


@pytest.mark.parametrize("mode", ["fast", "plain"])
def test_mid_size_uint8_build_bit_exact_vs_oracle(oracle_mod, mode):
    """120k x 128 uint8 with the skewed non-negative values of the BIGANN-shaped
    workload, hub targets included: u8 x u8 tensor-core tiles in the fast form,
    CUDA-core occlusion distances in the plain form."""
    base = D.gen_skewed_u8(120_000, 128, 1200, 6)
    gi, graph, st = gpu_build(base, 64, 128, 1.2, mode=mode)
    og, ost = oracle_mod.build(base, 64, 128, 1.2)
    np.testing.assert_array_equal(graph, canon(og))
    assert st["big_groups"] > 0 and st["reverse_prunes"] > 0
    if mode == "fast":
        # the first fast build of this shape calibrated the CTA shapes; builds
        # without statistics then run as one captured CUDA graph, replayed
        for _ in range(2):
            st2 = gi.build(128, 1.2, collect_stats=False, mode="fast")
            assert st2["graph_replay"] == 1
            np.testing.assert_array_equal(canon(gi.graph()), graph)
    gi.close()


def test_graph_replayed_fast_build_matches_reference(golden):
    """Fast builds without statistics are captured once as a CUDA graph and
    replayed: the replays give the reference's graph, as the stream path does."""
    g, _ = golden
    base, _ = case_inputs("i8_small")
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    gi.upload_points(base)
    for _ in range(3):
        st = gi.build(128, 1.2, collect_stats=False, mode="fast")
        assert st["graph_replay"] == 1
        assert sha(canon(gi.graph())) == g["cases"]["i8_small"]["graph_sha256"]
    st = gi.build(128, 1.2, collect_stats=True, mode="fast")
    assert st["graph_replay"] == 0
    assert sha(canon(gi.graph())) == g["cases"]["i8_small"]["graph_sha256"]
    gi.close()


def test_error_word_reports_bad_graph_ids():
    base = np.zeros((100, 8), np.uint8)
    gi = GpuIndex(base.dtype, "l2", 100, 8, 4)
    gi.upload_points(base)
    bad = np.zeros((100, 5), np.uint32)
    bad[:, 0] = 1
    bad[:, 1] = 1000  # out of range
    from distributed_diskann_b200._lib import DDError

    with pytest.raises(DDError):
        gi.set_graph(bad)
    gi.close()


def test_32bit_hash_table_layout_matches_24bit(monkeypatch):
    """Indexes with n >= 2^24 - 1 keep the lossy filter's ids in 32 bits; here
    DD_HASH32=1 selects that layout on small data.  Graph, search results and
    the reference's visited / dist_cmps counters must equal the 24-bit layout's
    (which the other tests check against the reference)."""
    base = D.gen_mixture_i8(20_000, 48, 200, 7)
    q = D.gen_mixture_i8(500, 48, 200, 8)
    out = []
    for flag in ("0", "1"):
        monkeypatch.setenv("DD_HASH32", flag)
        gi, graph, st = gpu_build(base, 32, 64, 1.2, mode="plain")
        ids, _, vis, cm = gi.search(q, 10, [10, 50, 100, 200, 64] * 100)
        out.append((graph, st["visited"], st["dist_cmps"], ids, vis, cm))
        gi.close()
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


def test_load_points_file_builds_reference_graph(golden, tmp_path, monkeypatch):
    """PointRange(char*): the reference's .bin file read through two pinned
    staging buffers (small chunks here, so that the double buffering turns over
    many times) gives the same points, hence the reference's graph."""
    from distributed_diskann_b200._lib import DDError

    g, _ = golden
    base, _ = case_inputs("i8_small")
    path = tmp_path / "base.bin"
    D.write_bin(str(path), base)
    monkeypatch.setenv("DD_LOAD_CHUNK_BYTES", str(64 * 1024))
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    gi.load_points(str(path))
    gi.build(128, 1.2)
    assert sha(canon(gi.graph())) == g["cases"]["i8_small"]["graph_sha256"]
    gi.close()
    # a header that does not match the index, and a truncated file
    other = GpuIndex(base.dtype, "l2", base.shape[0] - 1, base.shape[1], 64)
    with pytest.raises(DDError):
        other.load_points(str(path))
    other.close()
    raw = path.read_bytes()
    (tmp_path / "short.bin").write_bytes(raw[: len(raw) // 2])
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    with pytest.raises(DDError):
        gi.load_points(str(tmp_path / "short.bin"))
    gi.close()


@pytest.mark.parametrize("mode", ["fast", "plain"])
def test_visited_capacity_overflow_reruns_the_build(golden, mode):
    """The reference's build searches keep every visited node; a visited-list
    slice that overflows makes the build run again with twice the capacity,
    so a tiny starting capacity still gives the reference's graph."""
    g, _ = golden
    base, _ = case_inputs("i8_small")
    gi = GpuIndex(base.dtype, "l2", base.shape[0], base.shape[1], 64)
    gi.upload_points(base)
    st = gi.build(128, 1.2, vcap=8, mode=mode)
    assert st["vcap"] > 128
    assert sha(canon(gi.graph())) == g["cases"]["i8_small"]["graph_sha256"]
    gi.close()


def _screen_stress_points(metric, n=6_000, d=40, seed=31):
    """Float rows that stress the BF16 screen's bound: a mixture at three
    magnitudes (1e-12, 1, 1e15), rows whose values are exact in BF16 (the
    estimate is then exact and only the margins decide), near-duplicates a
    BF16 rounding apart, and exact duplicates (distance 0 at the cutoff)."""
    rng = np.random.default_rng(seed)
    base = D.gen_mixture_f32(n, d, 30, seed)
    third = n // 3
    base[:third] *= np.float32(1e-12)
    base[third:2 * third] *= np.float32(1e15)
    k = n // 10
    base[2 * third:2 * third + k] = np.round(base[2 * third:2 * third + k] * 4) / 4  # exact in BF16
    src = rng.integers(2 * third, n, k)
    nudge = (1 + rng.choice([-1, 1], (k, d)) * np.float32(2 ** -9)).astype(np.float32)
    base[n - 2 * k:n - k] = base[src] * nudge
    base[n - k:] = base[rng.integers(0, n - 2 * k, k)]
    if metric == "mips":
        base /= np.linalg.norm(base.astype(np.float64), axis=1, keepdims=True).astype(np.float32)
    return np.ascontiguousarray(base, np.float32)


@pytest.mark.parametrize("metric", ["l2", "mips"])
def test_bf16_screen_keeps_the_exact_graph_and_searches(oracle_mod, monkeypatch, metric):
    """Fast form, float data, with the opt-in BF16 screen (DD_SCREEN=1): build
    and query searches screen candidates on BF16 copies of the rows and compute
    the exact FP32 distance only for those the bound cannot rule out.  Graph,
    visited counts and query results must be the oracle's, and equal to the
    fast form without the screen (the default, DD_SCREEN=0)."""
    base = _screen_stress_points(metric)
    q = base[::37].copy()
    og, ost = oracle_mod.build(base, 32, 64, 1.2, metric=metric)
    oi, ov, oc = oracle_mod.search(base, og, q, 10, 40, metric=metric)
    runs = []
    for screen in ("1", "0"):
        monkeypatch.setenv("DD_SCREEN", screen)
        gi, graph, st = gpu_build(base, 32, 64, 1.2, metric=metric, mode="fast")
        np.testing.assert_array_equal(graph, canon(og), err_msg=f"screen={screen}")
        assert st["visited"] == ost["visited"]
        gi.set_search_mode("fast")
        ids, _, vis, cmps = gi.search(q, 10, 40)
        np.testing.assert_array_equal(ids, oi)
        np.testing.assert_array_equal(vis, ov)
        np.testing.assert_array_equal(cmps, oc)
        runs.append(st)
        gi.close()
    assert runs[0]["dist_cmps"] == runs[1]["dist_cmps"]
