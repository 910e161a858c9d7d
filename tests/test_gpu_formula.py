"""The reference's two decision paths, each reproduced bit for bit.

The reference decides with the materialised path (interval_calculation + reachability,
src/intersection_algorithm_in_parallel.cu:673-958) whenever its interval arrays fit in free
device memory, and with the fused kernel (reachable, .cu:960-1256) otherwise or when
forceOversize is set (.cu:87-97).  The two compute C of the free-interval quadratic with a
different rounding ((sum mi^2) - r^2 against a sum started at -r^2), so their intervals differ
in the last bits for a few percent of the partial edges (tests/test_oracle.py), and a decision
near the distance can differ.  Here every decision, bound and search of the CUDA path with
RFD_FORMULA_MATERIALISED equals the oracle's materialised restatement, and
RFD_FORMULA_REFERENCE picks the materialised path for pairs that fit in memory.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
MAT = 1


@pytest.mark.parametrize("style,d,n1,n2", [(0, 2, 300, 280), (1, 3, 1000, 900), (0, 3, 97, 1300),
                                           (1, 2, 1500, 40), (1, 3, 65, 33)])
def test_materialised_decisions_bitexact(ctx, built, style, d, n1, n2):
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 51, n1)
    r = oracle.distance(P, Q, stop_mode=1, quirks=False, formula=MAT)
    e_end = float(np.sqrt(((P[-1] - Q[-1]) ** 2).sum()))
    radii = [r["distance"] * (1 + k * 1e-15) for k in range(-3, 4)] + \
            [r["endpoint"], r["dfd"], e_end * 0.9, r["vefd"] * 1.01]
    for e in radii:
        want = oracle.decide(P, Q, e, formula=MAT)
        for dense in (False, True):
            assert ctx.decide(P, Q, e, dense=dense, formula=built.RFD_FORMULA_MATERIALISED) == want


@pytest.mark.parametrize("precise", [False, True])
def test_materialised_searches_bitexact(ctx, built, precise):
    pairs = [built.gen_pair(k % 2, 2 + k % 2, 200 + 97 * k, 150 + 61 * k, 100.0 if k % 2 else 1.0,
                            0.1, 52, k) for k in range(8)]
    res = ctx.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=precise,
                             formula=built.RFD_FORMULA_MATERIALISED)
    ref = ctx.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=precise,
                             formula=built.RFD_FORMULA_REFERENCE)
    for (P, Q), g, h in zip(pairs, res, ref):
        w = oracle.distance(P, Q, stop_mode=1 if precise else 0, quirks=not precise, formula=MAT)
        for k in ("distance", "lb", "ub", "dfd", "vefd", "probes"):
            assert g[k] == w[k], (k, g[k], w[k])
            assert h[k] == w[k], (k, h[k], w[k])


def test_filter_needs_the_fused_formula(ctx, built):
    P, Q = built.gen_pair(0, 2, 100, 90, 1.0, 0.05, 53, 0)
    with pytest.raises(built.RfdError) as e:
        ctx.distance(P, Q, precise=True, precision=built.RFD_PREC_FP32_FILTER,
                     formula=built.RFD_FORMULA_MATERIALISED)
    assert e.value.code == built.RFD_ERR_ARG
