"""Full-size golden digests of the Vamana workloads, from the reference's OWN build.

Runs ``oracle/_ref/ref_harness`` (the reference's src/bsp_index.hpp and
include/utils/beamSearch.h compiled unmodified with the single-rank shims,
see oracle/Makefile) on the seeded workloads at their stated sizes:

    mix64-f32      100,000 x 64 f32 mixture, L2, R=48, L=96, alpha=1.2
    msspacev-i8    1,000,000 x 100 int8 mixture, L2, R=64, L=128, alpha=1.2
    t2i-mips-f32   1,000,000 x 200 f32 normalised mixture, MIPS, R=64, L=128, alpha=1.0
    bigann-u8      10,000,000 x 128 uint8 skewed mixture, L2, R=64, L=128, alpha=1.2
                   (graph only; hours of host time are not needed for the searches)

and records, per workload, the sha256 of the input points and queries, of the
canonical graph (n x (R+1) uint32, row[0] = degree, unused slots zero) and of
searchAll's ids at several (L, limit, degree_limit) settings with the
reference's visited / dist_cmps sums.  ``limit`` stops a search after that many
visited nodes (include/utils/beamSearch.h:108) and ``degree_limit`` scans only
the first neighbours of each row (:123).

Run from the repo root where the reference tree is (DD_REFERENCE_ROOT):
    make -C oracle ref && python tests/golden/make_golden_full.py [names...]
The result is merged into tests/golden/golden_full.json, one workload at a time.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from distributed_diskann_b200 import datasets as D  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden.make_golden import canon, sha  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_full.json")

# workload -> (queries generated, queries searched, search settings (L, limit, degree_limit))
FULL_CASES = {
    "mix64-f32": (10_000, 10_000, [(10, 0, 0), (50, 0, 0), (100, 0, 0), (50, 20, 0),
                                   (50, 0, 24), (100, 60, 36)]),
    "msspacev-i8": (10_000, 10_000, [(10, 0, 0), (50, 0, 0), (100, 0, 0), (200, 0, 0),
                                     (50, 25, 0), (100, 0, 32), (128, 70, 48)]),
    "t2i-mips-f32": (10_000, 10_000, [(10, 0, 0), (50, 0, 0), (100, 0, 0), (50, 30, 0),
                                      (100, 0, 40)]),
    "bigann-u8": (10_000, 0, []),
}


def case_data(name):
    """Base and query points of a full-size case (shared with the tests)."""
    w = D.WORKLOADS[name]
    nq = FULL_CASES[name][0]
    return D.make_workload(w, n=w.n, nq=nq)


def run_case(name, threads):
    w = D.WORKLOADS[name]
    _, nsearch, settings = FULL_CASES[name]
    t0 = time.time()
    base, queries = case_data(name)
    gen_s = time.time() - t0
    g, secs = O.ref_build(base, w.R, w.L, w.alpha, metric=w.metric, threads=threads)
    g = canon(g)
    rec = {"dtype": w.dtype, "metric": w.metric, "n": int(base.shape[0]), "d": w.d, "R": w.R,
           "L": w.L, "alpha": w.alpha, "input_sha256": sha(base),
           "queries_sha256": sha(queries), "nq": int(queries.shape[0]), "nsearch": nsearch,
           "graph_sha256": sha(g), "edges": int(g[:, 0].sum()), "ref_build_seconds": secs,
           "ref_threads": threads, "datagen_seconds": gen_s, "search": []}
    q = queries[:nsearch]
    for L, limit, dlim in settings:
        ids, vis, cmps, ssec = O.ref_search(base, g, q, 10, L, cut=1.35, metric=w.metric,
                                            limit=limit, degree_limit=dlim, threads=threads)
        rec["search"].append({"L": L, "limit": limit, "degree_limit": dlim, "k": 10,
                              "ids_sha256": sha(ids), "visited_sum": int(vis.sum()),
                              "cmps_sum": int(cmps.sum()), "ref_search_seconds": ssec})
    return rec


def main():
    if not O.build_reference():
        raise SystemExit("reference harness unavailable (needs the reference tree)")
    names = sys.argv[1:] or list(FULL_CASES)
    threads = os.cpu_count() or 1
    for name in names:
        rec = run_case(name, threads)
        data = {}
        if os.path.exists(OUT):
            with open(OUT) as f:
                data = json.load(f)
        data.setdefault("generator", "tests/golden/make_golden_full.py")
        data["toolchain"] = subprocess.run(["g++", "--version"], capture_output=True,
                                           text=True).stdout.splitlines()[0]
        data["numpy"] = np.__version__
        data.setdefault("cases", {})[name] = rec
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        print(name, rec["graph_sha256"][:16], f"build {rec['ref_build_seconds']:.1f}s", flush=True)


if __name__ == "__main__":
    main()
