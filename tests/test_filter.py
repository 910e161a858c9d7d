"""FP32 filter of the free intervals (CPU): its certain answers against the FP64 oracle.

rfd_interval_class is the host build of the function the decision kernels run on the
device.  Every edge it classifies as certainly empty must have the oracle's FP64 interval
(-1, -2), every edge classified as certainly whole must have exactly (+0.0, 1.0), whatever the
scale of the coordinates and however close the radius is to a tangent or to an end point.
"""
import numpy as np
import pytest

import oracle


def edges(rng, n, d, scale, seg, mode):
    """n random edges a -> b around x and one radius r0; in the adversarial modes x is moved
    so that every edge sits at that radius's tangent or end-point case."""
    c = rng.uniform(-scale, scale, size=(n, d))
    a = c + rng.normal(scale=seg, size=(n, d))
    b = a + rng.normal(scale=seg, size=(n, d))
    x = c + rng.normal(scale=seg * rng.choice([0.1, 1.0, 5.0], size=(n, 1)), size=(n, d))
    ab = b - a
    A = np.einsum("ij,ij->i", ab, ab)
    r0 = seg
    jitter = 1 + rng.normal(scale=1e-7, size=(n, 1)) * (mode != "exact_ends")
    if mode == "tangent":      # x at distance r0 from the edge's line: disc ~ 0
        foot = a + (np.einsum("ij,ij->i", x - a, ab) / A)[:, None] * ab
        off = x - foot
        off /= np.sqrt((off ** 2).sum(1))[:, None]
        x = foot + off * r0 * jitter
    elif mode in ("ends", "exact_ends"):   # an end point at distance r0 from x: ta or tb ~ 0, 1
        end = np.where(rng.random((n, 1)) < 0.5, a, b)
        off = x - end
        off /= np.sqrt((off ** 2).sum(1))[:, None]
        x = end + off * r0 * jitter
    return x, a, b, A, r0


@pytest.mark.parametrize("d", [2, 3])
@pytest.mark.parametrize("scale,seg", [(1e-3, 1e-4), (1.0, 0.05), (100.0, 1.7), (1e4, 3.0),
                                       (1e4, 1e-3)])
@pytest.mark.parametrize("mode", ["spread", "tangent", "ends", "exact_ends"])
def test_certain_classes_match_fp64(built, d, scale, seg, mode):
    rng = np.random.default_rng(int(scale * 7) + d * 11 + len(mode))
    n = 20000
    x, a, b, A, r = edges(rng, n, d, scale, seg, mode)
    total = {0: 0, 1: 0, 2: 0}
    for r2 in (r ** 2, (0.5 * r) ** 2, (3 * r) ** 2):
        cls = built.interval_class(x, a, b, A, r2)
        lo, hi = oracle.free_intervals(x, a, b, A, r2)
        empty, whole = cls == 1, cls == 2
        assert np.all(lo[empty] == -1.0) and np.all(hi[empty] == -2.0), (scale, mode)
        assert np.all(lo[whole] == 0.0) and not np.any(np.signbit(lo[whole]))
        assert np.all(hi[whole] == 1.0), (scale, mode)
        for c in (0, 1, 2):
            total[c] += int(np.sum(cls == c))
    if mode == "spread":
        # far from tangents and end points most edges are decided in FP32
        assert total[1] + total[2] > 0.5 * sum(total.values()), total


def test_degenerate_and_nonfinite_go_to_fp64(built):
    x = np.array([[0.0, 0.0], [0.0, 0.0], [np.inf, 0.0], [np.nan, 1.0]])
    a = np.array([[1.0, 1.0], [1e20, 0.0], [1.0, 1.0], [1.0, 1.0]])
    b = np.array([[1.0, 1.0], [1e20 + 1e5, 0.0], [2.0, 1.0], [2.0, 1.0]])
    A = np.array([0.0, 1e10, 1.0, 1.0])
    cls = built.interval_class(x, a, b, A, 4.0)
    assert list(cls) == [0, 0, 0, 0]
