"""Seeded synthetic point sets with the shapes of the Vamana build/search workloads.

The public datasets the reference's configs name (BIGANN-10M, MSSPACEV-1M,
Text2Image-10M: bigann-10M.json, msspacev-1M.json, text2image-10M.json) are not
available offline, so each workload is a seeded stand-in with the same shape,
element type and value range.  All generators are numpy ``default_rng`` based
and deterministic for a given seed and numpy version.

File I/O follows the reference's ``.bin`` layout ``[u32 n][u32 d][n*d elems]``
(include/utils/point_range.h:61-97; dataset/dataset_io.py) and its ground-truth
layout ``[u32 nq][u32 k][ids nq*k u32][dists nq*k f32]`` (src/dataset.hpp:6-18).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Workload:
    name: str
    dtype: str          # "f32" | "i8" | "u8"
    metric: str         # "l2" | "mips"
    n: int
    nq: int
    d: int
    R: int
    L: int
    alpha: float
    seed: int
    k: int = 10
    sweep_L: tuple = (10, 20, 50, 100, 200)
    extra: dict = field(default_factory=dict)


# The five workload shapes (sizes as named; tests scale n down).
WORKLOADS = {
    "xs-f32": Workload("xs-f32", "f32", "l2", 10_000, 1_000, 20, 32, 64, 1.2, 1),
    "mix64-f32": Workload("mix64-f32", "f32", "l2", 100_000, 10_000, 64, 48, 96, 1.2, 3),
    "msspacev-i8": Workload("msspacev-i8", "i8", "l2", 1_000_000, 30_000, 100, 64, 128, 1.2, 4),
    "t2i-mips-f32": Workload("t2i-mips-f32", "f32", "mips", 1_000_000, 100_000, 200, 64, 128, 1.0, 5),
    "bigann-u8": Workload("bigann-u8", "u8", "l2", 10_000_000, 10_000, 128, 64, 128, 1.2, 6),
}


def _normal(rng, shape, scale=1.0):
    return rng.standard_normal(shape, dtype=np.float32) * np.float32(scale)


def _chunks(total, chunk=1 << 20):
    s = 0
    while s < total:
        e = min(total, s + chunk)
        yield s, e
        s = e


def gen_iid_normal(n, d, seed):
    return _normal(np.random.default_rng(seed), (n, d))


def gen_mixture_f32(n, d, ncent, seed, spread=10.0, sigma=1.0):
    """Centres ~ U[-spread, spread]^d, points = centre + N(0, sigma^2)."""
    rng = np.random.default_rng(seed)
    cent = rng.uniform(-spread, spread, (ncent, d)).astype(np.float32)
    out = np.empty((n, d), np.float32)
    for s, e in _chunks(n):
        lab = rng.integers(0, ncent, e - s)
        out[s:e] = cent[lab] + _normal(rng, (e - s, d), sigma)
    return out


def gen_mixture_i8(n, d, ncent, seed, cscale=40.0, sigma=12.0):
    """Centres ~ N(0, cscale^2)^d; points = round(centre + N(0, sigma^2)) clipped to int8."""
    rng = np.random.default_rng(seed)
    cent = _normal(rng, (ncent, d), cscale)
    out = np.empty((n, d), np.int8)
    for s, e in _chunks(n):
        lab = rng.integers(0, ncent, e - s)
        v = np.rint(cent[lab] + _normal(rng, (e - s, d), sigma))
        out[s:e] = np.clip(v, -128, 127).astype(np.int8)
    return out


def gen_skewed_u8(n, d, ncent, seed, cscale=40.0, sigma=12.0):
    """Centres ~ |N(0, cscale^2)|^d; points = round(|centre + N(0, sigma^2)|) clipped to uint8."""
    rng = np.random.default_rng(seed)
    cent = np.abs(_normal(rng, (ncent, d), cscale))
    out = np.empty((n, d), np.uint8)
    for s, e in _chunks(n):
        lab = rng.integers(0, ncent, e - s)
        v = np.rint(np.abs(cent[lab] + _normal(rng, (e - s, d), sigma)))
        out[s:e] = np.clip(v, 0, 255).astype(np.uint8)
    return out


def gen_normalized_mixture(n, d, ncent, seed, sigma=0.3, shift=0.0, cent_seed=None):
    """L2-normalised rows of centre + N(0, sigma^2); ``shift`` perturbs the centres."""
    crng = np.random.default_rng(seed if cent_seed is None else cent_seed)
    cent = _normal(crng, (ncent, d))
    rng = np.random.default_rng(seed + 1000003)
    if shift:
        cent = cent + _normal(rng, cent.shape, shift)
    out = np.empty((n, d), np.float32)
    for s, e in _chunks(n):
        lab = rng.integers(0, ncent, e - s)
        v = cent[lab] + _normal(rng, (e - s, d), sigma)
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        out[s:e] = v
    return out


def make_workload(w: Workload, n: int | None = None, nq: int | None = None):
    """Base and query sets for workload ``w``; ``n``/``nq`` override the sizes."""
    n = w.n if n is None else n
    nq = w.nq if nq is None else nq
    if w.name.startswith("xs"):
        return gen_iid_normal(n, w.d, w.seed), gen_iid_normal(nq, w.d, w.seed + 1)
    if w.name.startswith("mix64"):
        both = gen_mixture_f32(n + nq, w.d, 100, w.seed)
        return both[:n], both[n:]
    if w.name.startswith("msspacev"):
        both = gen_mixture_i8(n + nq, w.d, 1000, w.seed)
        return both[:n], both[n:]
    if w.name.startswith("t2i"):
        base = gen_normalized_mixture(n, w.d, 2000, w.seed)
        q = gen_normalized_mixture(nq, w.d, 2000, w.seed + 7, shift=0.3, cent_seed=w.seed)
        return base, q
    if w.name.startswith("bigann"):
        both = gen_skewed_u8(n + nq, w.d, 10_000, w.seed)
        return both[:n], both[n:]
    raise KeyError(w.name)


def random_xs_like_reference():
    """The reference's shipped random-xs set (data/random10000), regenerated exactly
    the way dataset/datasets.py:870-899 made it (sklearn make_blobs, random_state=1)."""
    import sklearn.datasets
    import sklearn.model_selection

    X, _ = sklearn.datasets.make_blobs(n_samples=11000, n_features=20, centers=1000,
                                       random_state=1)
    data, queries = sklearn.model_selection.train_test_split(X, test_size=1000, random_state=1)
    return data.astype(np.float32), queries.astype(np.float32)


# ------------------------------------------------------------------ file formats
def write_bin(path, x):
    x = np.ascontiguousarray(x)
    with open(path, "wb") as f:
        np.array(x.shape, dtype=np.uint32).tofile(f)
        x.tofile(f)


def read_bin(path, dtype):
    with open(path, "rb") as f:
        n, d = (int(v) for v in np.fromfile(f, dtype=np.uint32, count=2))
        return np.fromfile(f, dtype=dtype, count=n * d).reshape(n, d)


def write_groundtruth(path, ids, dists):
    with open(path, "wb") as f:
        np.array(ids.shape, dtype=np.uint32).tofile(f)
        ids.astype(np.uint32).tofile(f)
        dists.astype(np.float32).tofile(f)


def read_groundtruth(path):
    raw = np.fromfile(path, dtype=np.uint32)
    nq, k = int(raw[0]), int(raw[1])
    ids = raw[2 : 2 + nq * k].reshape(nq, k)
    dists = raw[2 + nq * k : 2 + 2 * nq * k].view(np.float32).reshape(nq, k)
    return ids, dists


def recall_with_ties(found_ids, gt_ids, gt_dists, k):
    """Recall@k counting ground-truth ties at the k-th distance, as
    include/utils/check_nn_recall.h:86-108 does."""
    nq = found_ids.shape[0]
    correct = 0
    for i in range(nq):
        res = list(gt_ids[i, :k])
        last = gt_dists[i, k - 1]
        for l in range(k, gt_ids.shape[1]):
            if gt_dists[i, l] == last:
                res.append(gt_ids[i, l])
        rep = set(int(x) for x in found_ids[i, :k])
        correct += sum(1 for x in res if int(x) in rep)
    return correct / float(k * nq)
