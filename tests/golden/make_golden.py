"""Generate the golden fixtures from the reference's OWN sources.

Runs ``oracle/_ref/ref_harness`` (the reference's src/bsp_index.hpp,
include/index.h and include/utils/beamSearch.h compiled unmodified with the
single-rank shims, see oracle/Makefile) on seeded inputs and records:

* sha256 digests of the canonical graphs (n x (R+1) uint32, row[0] = degree,
  unused slots zero) and of search results,
* full arrays for the small / edge cases and for robustPrune cases,
* the digest of the reference's shipped random-xs files (data/random10000),
  which ``datasets.random_xs_like_reference`` regenerates bit-exactly.

Run from the repo root in a container that has the reference tree:
    make -C oracle ref && python tests/golden/make_golden.py
Inputs are regenerated by the tests from the same seeds (their digests are
stored too, so a changed generator shows up as an input mismatch).
"""
from __future__ import annotations

import hashlib
import json
import os
import platform
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from distributed_diskann_b200 import datasets as D  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT_DIR = os.path.dirname(os.path.abspath(__file__))
REF_DATA = os.path.join(O.REF_ROOT, "data", "random10000")


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def canon(g):
    g = g.copy()
    R = g.shape[1] - 1
    g[:, 1:][np.arange(R)[None, :] >= g[:, :1]] = 0
    return g


# ------------------------------------------------------------------ case inputs
def case_inputs(name):
    """Seeded inputs of every golden case (shared with the tests)."""
    if name == "xs_ref":
        return D.random_xs_like_reference()
    if name == "xs_seed1":
        return D.gen_iid_normal(10_000, 20, 1), D.gen_iid_normal(1_000, 20, 2)
    if name == "mix64_small":
        b = D.gen_mixture_f32(21_000, 64, 100, 3)
        return b[:20_000], b[20_000:]
    if name == "i8_small":
        b = D.gen_mixture_i8(21_000, 100, 1000, 4)
        return b[:20_000], b[20_000:]
    if name == "mips_small":
        return (D.gen_normalized_mixture(10_000, 200, 400, 5),
                D.gen_normalized_mixture(500, 200, 400, 12, shift=0.3, cent_seed=5))
    if name == "u8_small":
        b = D.gen_skewed_u8(21_000, 128, 500, 6)
        return b[:20_000], b[20_000:]
    if name == "dups_i8":
        rng = np.random.default_rng(11)
        distinct = rng.integers(-3, 4, (300, 12)).astype(np.int8)
        return distinct[rng.integers(0, 300, 2_000)], distinct[rng.integers(0, 300, 100)]
    if name == "params_u8":
        rng = np.random.default_rng(12)
        return rng.integers(0, 256, (5_000, 16)).astype(np.uint8), None
    if name == "knn2_i8":
        b = D.gen_mixture_i8(5_000, 50, 100, 13)
        return b, None
    if name == "mips_i8":
        rng = np.random.default_rng(14)
        return rng.integers(-20, 21, (3_000, 24)).astype(np.int8), rng.integers(-20, 21, (200, 24)).astype(np.int8)
    if name.startswith("tiny_"):
        n = int(name.split("_")[1])
        rng = np.random.default_rng(100 + n)
        return rng.integers(0, 4, (n, 8)).astype(np.uint8), rng.integers(0, 4, (3, 8)).astype(np.uint8)
    raise KeyError(name)


BUILD_CASES = {
    # name: (R, L, alpha, metric, xita, max_build, start, knn_mode, two_pass, search Ls)
    "xs_ref": (32, 64, 1.2, "l2", 1.0, 0, 0, False, False, (10, 20, 50, 100, 200)),
    "xs_seed1": (32, 64, 1.2, "l2", 1.0, 0, 0, False, False, (10, 20, 50, 100, 200)),
    "mix64_small": (48, 96, 1.2, "l2", 1.0, 0, 0, False, False, (10, 50)),
    "i8_small": (64, 128, 1.2, "l2", 1.0, 0, 0, False, False, (10, 20, 50, 100, 200)),
    "mips_small": (64, 128, 1.0, "mips", 1.0, 0, 0, False, False, (10, 100)),
    "u8_small": (64, 128, 1.2, "l2", 1.0, 0, 0, False, False, (10, 50, 200)),
    "dups_i8": (16, 32, 1.2, "l2", 1.0, 0, 0, False, False, (10, 32)),
    "params_u8": (16, 32, 1.2, "l2", 0.02, 4_000, 7, False, False, ()),
    "knn2_i8": (24, 48, 1.2, "l2", 1.0, 0, 0, True, True, ()),
    "mips_i8": (16, 32, 1.1, "mips", 1.0, 0, 0, False, False, (16,)),
    "tiny_1": (4, 8, 1.2, "l2", 1.0, 0, 0, False, False, ()),
    "tiny_2": (4, 8, 1.2, "l2", 1.0, 0, 0, False, False, ()),
    "tiny_3": (4, 8, 1.2, "l2", 1.0, 0, 0, False, False, ()),
    "tiny_5": (4, 8, 1.2, "l2", 1.0, 0, 0, False, False, ()),
    "tiny_17": (4, 8, 1.2, "l2", 1.0, 0, 0, False, False, (4,)),
    "tiny_40": (6, 10, 1.2, "l2", 1.0, 0, 0, False, False, (6,)),
}
SMALL_FULL = {"dups_i8", "params_u8", "tiny_1", "tiny_2", "tiny_3", "tiny_5", "tiny_17", "tiny_40",
              "mips_i8"}


def main():
    if not O.build_reference():
        raise SystemExit("reference harness unavailable (needs the reference tree)")
    golden = {
        "generator": "tests/golden/make_golden.py",
        "toolchain": subprocess.run(["g++", "--version"], capture_output=True,
                                    text=True).stdout.splitlines()[0],
        "numpy": np.__version__,
        "python": platform.python_version(),
        "cases": {},
    }
    full = {}
    for name, (R, L, alpha, metric, xita, mx, st, knn, tp, Ls) in BUILD_CASES.items():
        base, queries = case_inputs(name)
        g, secs = O.ref_build(base, R, L, alpha, metric=metric, xita=xita, max_build=mx,
                              start=st, knn_mode=knn, two_pass=tp)
        g = canon(g)
        rec = {
            "R": R, "L": L, "alpha": alpha, "metric": metric, "xita": xita, "max_build": mx,
            "start": st, "knn_mode": knn, "two_pass": tp,
            "dtype": str(base.dtype), "n": int(base.shape[0]), "d": int(base.shape[1]),
            "input_sha256": sha(base), "graph_sha256": sha(g),
            "edges": int(g[:, 0].sum()), "ref_build_seconds": secs, "search": {},
        }
        if queries is not None:
            rec["queries_sha256"] = sha(queries)
            rec["nq"] = int(queries.shape[0])
        for Ls_ in Ls:
            k = min(10, Ls_)
            ids, vis, cmps, _ = O.ref_search(base, g, queries, k, Ls_, cut=1.35, metric=metric,
                                             start=st)
            rec["search"][str(Ls_)] = {"k": k, "ids_sha256": sha(ids),
                                       "visited_sum": int(vis.sum()), "cmps_sum": int(cmps.sum())}
            if name in SMALL_FULL:
                full[f"{name}__search{Ls_}"] = ids
        if name in SMALL_FULL:
            full[f"{name}__graph"] = g
        golden["cases"][name] = rec
        print(name, rec["graph_sha256"][:16], f"{secs:.3f}s", flush=True)

    # shipped random-xs fixture: digests of the files and the reference GT recall
    if os.path.isdir(REF_DATA):
        raw = np.fromfile(os.path.join(REF_DATA, "data_10000_20"), dtype=np.uint32)
        rq = np.fromfile(os.path.join(REF_DATA, "queries_1000_20"), dtype=np.uint32)
        gi, gd = D.read_groundtruth(os.path.join(REF_DATA, "gt_10000_1000_20"))
        base, queries = case_inputs("xs_ref")
        g = canon(O.ref_build(base, 32, 64, 1.2)[0])
        rec = {"data_file_sha256": hashlib.sha256(raw.tobytes()).hexdigest(),
               "queries_file_sha256": hashlib.sha256(rq.tobytes()).hexdigest(),
               "gt_ids_sha256": sha(gi), "recall10": {}}
        for Ls_ in (10, 20, 50, 100, 200):
            ids = O.ref_search(base, g, queries, 10, Ls_, cut=1.35)[0]
            rec["recall10"][str(Ls_)] = D.recall_with_ties(ids, gi, gd, 10)
        golden["shipped_random_xs"] = rec

    # robustPrune cases on the i8_small reference graph: tie-heavy candidate sets
    base, _ = case_inputs("i8_small")
    g = canon(O.ref_build(base, 64, 128, 1.2)[0])
    rng = np.random.default_rng(21)
    tasks = []
    for t in range(120):
        p = int(rng.integers(0, base.shape[0]))
        m = int(rng.choice([1, 2, 15, 16, 17, 33, 100, 172, 300, 700]))
        cand = rng.choice(base.shape[0], m, replace=False).astype(np.uint32)
        if t % 3 == 0:  # coarse distances: many exact ties
            dists = (np.floor(np.array([O.distance(base[c], base[p]) for c in cand]) / 5000.0)
                     * 5000.0).astype(np.float32)
        else:
            dists = np.array([O.distance(base[c], base[p]) for c in cand], dtype=np.float32)
        tasks.append((p, cand, dists))
    with open("/tmp/dd_prune_tasks.bin", "wb") as f:
        for p, cand, dists in tasks:
            np.array([p, len(cand)], np.uint32).tofile(f)
            inter = np.empty(2 * len(cand), np.uint32)
            inter[0::2] = cand
            inter[1::2] = dists.view(np.uint32)
            inter.tofile(f)
    O.write_graph("/tmp/dd_prune_graph.bin", g)
    O.write_bin("/tmp/dd_prune_base.bin", base)
    O._run_ref(["prune", "i8", "l2", "/tmp/dd_prune_base.bin", "/tmp/dd_prune_graph.bin",
                "/tmp/dd_prune_tasks.bin", 64, 1.2, "/tmp/dd_prune_out.bin"])
    raw = np.fromfile("/tmp/dd_prune_out.bin", dtype=np.uint32)
    pos = 0
    for t, (p, cand, dists) in enumerate(tasks):
        ln = int(raw[pos])
        full[f"prune{t}__p"] = np.array([p], np.uint32)
        full[f"prune{t}__cand"] = cand
        full[f"prune{t}__dist"] = dists
        full[f"prune{t}__out"] = raw[pos + 1 : pos + 1 + ln].copy()
        pos += 1 + ln
    golden["prune_cases"] = len(tasks)

    # beam_search cases (full frontier + visited + dist_cmps), build and query mode
    base, queries = case_inputs("i8_small")
    for mode, (k, L, cut) in {"build": (0, 128, 0.0), "query": (10, 50, 1.35)}.items():
        res = O.ref_beam(base, g, queries[:40], k, L, cut=cut)
        for i, (fr, vi, cm) in enumerate(res):
            full[f"beam_{mode}{i}__fr_ids"] = fr[0]
            full[f"beam_{mode}{i}__fr_d"] = fr[1]
            full[f"beam_{mode}{i}__vi_ids"] = vi[0]
            full[f"beam_{mode}{i}__vi_d"] = vi[1]
            full[f"beam_{mode}{i}__cmps"] = np.array([cm], np.uint64)
    golden["beam_cases"] = 40

    with open(os.path.join(OUT_DIR, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(OUT_DIR, "golden_small.npz"), **full)
    print("wrote", len(golden["cases"]), "build cases,", len(full), "arrays")


if __name__ == "__main__":
    main()
