"""FP32 filter on the GPU: searches with RFD_PREC_FP32_FILTER make the same decisions as the
FP64 path (bit-identical distances, bounds and probe counts) and compute fewer cells in FP64.

A search probes radii ever closer to the distance, so it exercises the decisions whose
intervals sit nearest the filter's margins."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def pairs(built):
    out = [built.gen_pair(0, 2, 900, 850, 1.0, 0.05, 31, 0),
           built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 31, 1),
           built.gen_pair(1, 3, 2500, 3100, 1e4, 0.1, 31, 2),      # coordinates ~1e4
           built.gen_pair(0, 3, 700, 4000, 1.0, 0.05, 31, 3)]
    return out


@pytest.mark.parametrize("precise", [True, False])
def test_filter_search_identical(ctx, built, precise):
    for k, (P, Q) in enumerate(pairs(built)):
        a = ctx.distance(P, Q, precise=precise)
        b = ctx.distance(P, Q, precise=precise, precision=built.RFD_PREC_FP32_FILTER)
        # (cells_evaluated is not compared: it includes speculative helper tiles, whose
        # cancellation depends on timing)
        for key in ("distance", "lb", "ub", "dfd", "vefd", "probes"):
            assert a[key] == b[key], (k, key, a[key], b[key])
        assert b["cells_fp64"] < b["cells_evaluated"], (k, b["cells_fp64"], b["cells_evaluated"])
        assert a["cells_fp64"] == a["cells_evaluated"]


def test_filter_batch_identical(ctx, built):
    ps = pairs(built) + [built.gen_pair(k % 2, 2 + k % 2, 200 + 37 * k, 300 + 53 * k,
                                        1e4 if k % 3 == 0 else 1.0, 0.1, 47, k) for k in range(20)]
    Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
    a = ctx.distance_batch(Ps, Qs, precise=True)
    b = ctx.distance_batch(Ps, Qs, precise=True, precision=built.RFD_PREC_FP32_FILTER)
    for k, (x, y) in enumerate(zip(a, b)):
        assert x["distance"] == y["distance"] and x["probes"] == y["probes"], k
    frac = sum(y["cells_fp64"] for y in b) / sum(y["cells_evaluated"] for y in b)
    assert frac < 0.9, frac


def test_precision_option_checked(ctx, built):
    P, Q = pairs(built)[0]
    with pytest.raises(built.RfdError):
        ctx.distance(P, Q, precision=7)
