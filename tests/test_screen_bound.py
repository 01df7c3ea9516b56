"""The bound of the fast form's BF16 screen (search_core.cuh screen_and_rerank),
restated in numpy: the lower bound it computes from a BF16 row must never lie
above the reference's FP32 distance (include/utils/NSGDist.h:113-131 for L2,
include/utils/mips_point.h:60-66 for MIPS), or a candidate that passes the
cutoff could be dropped.  The estimate is summed here in float64 and rounded
once, a tighter sum than the kernel's FP32 one, whose own rounding the bound
covers with its (d + 16) 2^-23 terms."""
import zlib

import numpy as np
import pytest


def bf16(x):
    """Round to nearest even BF16, returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def ref_l2(a, b):
    r = np.float32(0)
    d = a.shape[0]
    i = 0
    while i + 3 < d:
        t = (a[i:i + 4] - b[i:i + 4]).astype(np.float32)
        e = (t * t).astype(np.float32)
        s = np.float32(np.float32(np.float32(e[0] + e[1]) + e[2]) + e[3])
        r = np.float32(r + s)
        i += 4
    while i < d:
        t = np.float32(a[i] - b[i])
        r = np.float32(r + np.float32(t * t))
        i += 1
    return r


def ref_mips(a, b):
    r = np.float32(0)
    for x in (a * b).astype(np.float32):
        r = np.float32(r + x)
    return np.float32(-r)


def screen_lower_bound(a, b, metric):
    d = a.shape[0]
    bt = bf16(b)
    gam3 = np.float32(3 * (d + 16) * 2.0 ** -23 + 2.0 ** -20)
    if metric == "l2":
        t = (a - bt).astype(np.float32)
        acc = np.float32(np.sum(t.astype(np.float64) ** 2))
        bnd = np.float32(np.sum(np.abs(bt.astype(np.float64)) * np.abs(t)))
        nb2 = np.float32(np.sum(bt.astype(np.float64) ** 2))
        return acc - (np.float32(1.01) * (np.float32(2 ** -7) * bnd + np.float32(2 ** -16) * nb2)
                      + acc * gam3 + np.float32(1e-20))
    acc = np.float32(np.sum(a.astype(np.float64) * bt))
    bnd = np.float32(np.sum(np.abs(a.astype(np.float64) * bt)))
    return -acc - (bnd * (np.float32(1.01 * 2 ** -8) + gam3) + np.float32(1e-20))


def _pairs(rng, kind, d):
    if kind == "mixture":
        c = rng.uniform(-10, 10, d)
        a = c + rng.normal(0, 1, d)
        b = c + rng.normal(0, rng.choice([1e-3, 0.1, 1.0]), d)
    elif kind == "normalised":
        a = rng.normal(0, 1, d)
        a /= np.linalg.norm(a)
        b = a + rng.normal(0, 0.3, d)
        b /= np.linalg.norm(b)
    elif kind == "scaled":
        a = rng.normal(0, 1, d) * 10 ** rng.uniform(-12, 15)
        b = a * (1 + rng.normal(0, 1e-3, d))
    else:  # a BF16 rounding apart
        a = rng.normal(0, 1, d)
        b = a * (1 + rng.choice([-1, 1], d) * 2.0 ** -9)
    return a.astype(np.float32), b.astype(np.float32)


@pytest.mark.parametrize("metric", ["l2", "mips"])
@pytest.mark.parametrize("kind", ["mixture", "normalised", "scaled", "bf16_apart"])
def test_screen_lower_bound_never_exceeds_the_reference_distance(metric, kind):
    rng = np.random.default_rng(zlib.crc32(f"{metric}/{kind}".encode()))
    for _ in range(300):
        d = int(rng.choice([7, 13, 20, 64, 100, 200]))
        a, b = _pairs(rng, kind, d)
        ref = ref_l2(a, b) if metric == "l2" else ref_mips(a, b)
        low = screen_lower_bound(a, b, metric)
        assert low <= ref, (metric, kind, d, float(low), float(ref))


def test_screen_is_tight_enough_to_rule_out_far_candidates():
    """The bound is only useful if it rules candidates out: on mixture data a
    candidate from another cluster is proven farther than one from the same
    cluster, so the screen drops it without the exact distance."""
    rng = np.random.default_rng(4)
    d = 64
    c1, c2 = rng.uniform(-10, 10, (2, d))
    q = (c1 + rng.normal(0, 1, d)).astype(np.float32)
    near = (c1 + rng.normal(0, 1, d)).astype(np.float32)
    far = (c2 + rng.normal(0, 1, d)).astype(np.float32)
    assert screen_lower_bound(q, far, "l2") > ref_l2(q, near)
