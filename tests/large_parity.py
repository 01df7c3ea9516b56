"""Parity of the 10M x 128 uint8 build with the reference's own build.

Not a pytest module: the reference needs minutes on the host for this size.
Run on a GPU machine after building (`__graft_entry__.build()`), with the
reference harness in oracle/_ref:

    python tests/large_parity.py [n]      # default: all 10,000,000 points

It builds the leading n points of bench.py's default workload on the GPU and
with the reference's BSP build (its unmodified sources, all host threads),
and compares the two graphs row by row (degree and neighbour order).
The result is printed as one JSON line.
"""
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from distributed_diskann_b200 import datasets as D  # noqa: E402
from distributed_diskann_b200.index import GpuIndex  # noqa: E402
from oracle import oracle as O  # noqa: E402


def canon(x):
    """Rows with the entries past the degree zeroed."""
    x = np.array(x, dtype=np.uint32, copy=True)
    x[:, 1:][np.arange(x.shape[1] - 1)[None, :] >= x[:, :1]] = 0
    return x


def main():
    w = D.WORKLOADS["bigann-u8"]
    n = int(sys.argv[1]) if len(sys.argv) > 1 else w.n
    base, _ = D.make_workload(w, n=w.n, nq=w.nq)  # the bench's points
    base = np.ascontiguousarray(base[:n])
    gi = GpuIndex(base.dtype, w.metric, n, w.d, w.R, device=0)
    gi.upload_points(base)
    st = gi.build(w.L, w.alpha)
    g = canon(gi.graph())
    gi.close()
    t0 = time.time()
    rg, secs = O.ref_build(base, w.R, w.L, w.alpha, threads=os.cpu_count())
    wall = time.time() - t0
    rg = canon(rg)
    differing = int((g != rg).any(axis=1).sum())
    print(json.dumps({"n": n, "identical": differing == 0, "rows_differing": differing,
                      "gpu_build_ms": st["build_ms"], "ref_build_s": secs, "ref_wall_s": wall,
                      "ref_threads": os.cpu_count(), "avg_degree": float(g[:, 0].mean())}))
    return 0 if differing == 0 else 1


if __name__ == "__main__":
    sys.exit(main())
