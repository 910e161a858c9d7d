"""Meet in the middle: a lone pair's VE-FD and search decisions as two half-length sweeps.

The forward sweep runs the first half of the team strips; a mirror sweep runs the other half
from the far corner (on the same edge values, intervals negated), and a meet kernel combines
the two rows handed over across the middle boundary: VE-FD as min over the boundary edges of
max(forward, mirror), a decision as "some edge has its forward reachable part meet its
co-reachable part".  Both are exact combinations of the same doubles, so every result must
be bit-identical to the unsplit sweep and to the CPU oracle.  RFD_SPLIT = n splits pairs of
at least n strips (default 64; 0 never): here 2, so small pairs around the strip and chunk
edges, both orientations, 2D and 3D, are split, and the unsplit context is the comparison.
The 200,000-point long pair is split by default and checked against its golden in
test_gpu_config_goldens.py.
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

EXACT = ("distance", "dfd", "vefd", "lb", "ub", "probes", "flags")


def _ctx(built, **env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update({k: str(v) for k, v in env.items()})
    try:
        return built.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


@pytest.fixture(scope="module")
def split_ctx(built):
    c = _ctx(built, RFD_SPLIT=2)
    yield c
    c.close()


@pytest.fixture(scope="module")
def plain_ctx(built):
    c = _ctx(built, RFD_SPLIT=0)
    yield c
    c.close()


PAIRS = [(0, 2, 1000, 700), (0, 2, 700, 1000), (1, 3, 2000, 1900), (1, 3, 32 * 45 + 1, 900),
         (0, 3, 300, 2500), (1, 2, 4100, 130), (0, 2, 66, 70), (1, 3, 97, 3000),
         (0, 2, 3000, 97)]


@pytest.mark.parametrize("style,d,n1,n2", PAIRS)
def test_split_solves_bitexact(split_ctx, built, style, d, n1, n2):
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 51, n1)
    th = oracle.max_threads()
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=th)
    got = split_ctx.distance(P, Q, precise=True)
    for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])
    for dense in (False, True):
        assert split_ctx.bounds(P, Q, quirks=False, dense=dense) == (want["dfd"], want["vefd"]), \
            dense
    want = oracle.distance(P, Q, stop_mode=0, quirks=True, threads=th)
    got = split_ctx.distance(P, Q)
    for k in ("distance", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])


@pytest.mark.parametrize("style,d,n1,n2", PAIRS[:6])
def test_split_forms_equal_unsplit(split_ctx, plain_ctx, built, style, d, n1, n2):
    """Learned bracket, coarse bound, FP32 filter, the materialised formula, dense decisions:
    the split context returns what the unsplit one does, field for field."""
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 53, n1)
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(precise=True, model=model), dict(precise=True, model=model, coarse_ub=6),
                   dict(precise=True, precision=built.RFD_PREC_FP32_FILTER),
                   dict(precise=True, formula=built.RFD_FORMULA_MATERIALISED),
                   dict(precise=True, dense=True), dict(precise=False)):
            a = plain_ctx.distance(P, Q, **kw)
            b = split_ctx.distance(P, Q, **kw)
            for k in EXACT:
                assert a[k] == b[k], (kw, k, a[k], b[k])
    finally:
        model.close()


def test_split_degenerate_and_closed_forms(split_ctx, built):
    """Identical curves, parallel lines, a zero-length segment (the reference's [0, 1]
    interval) and a curve of two points."""
    th = oracle.max_threads()
    t = np.linspace(0.0, 1.0, 700)
    cases = []
    A = np.stack([t, np.sin(7 * t)], 1)
    cases.append((A, A.copy()))
    cases.append((np.stack([t, 0 * t], 1), np.stack([t, 0 * t + 0.5], 1)))
    B = A.copy()
    B[300] = B[299]  # a repeated point: a zero-length segment
    cases.append((B, A[::2].copy()))
    cases.append((np.array([[0.0, 0.0], [1.0, 0.0]]), A))
    for P, Q in cases:
        want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=th)
        got = split_ctx.distance(P, Q, precise=True)
        for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
            assert got[k] == want[k], (len(P), len(Q), k, got[k], want[k])


def test_split_batch_of_one_and_graph(split_ctx, plain_ctx, built):
    """A one-pair batch call splits as a single call does; under CUDA graph capture and
    replay (the mirror kernel runs on a second stream, forked and joined by events) the
    results stay those of the unsplit path."""
    P, Q = built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 57, 0)
    want = plain_ctx.distance(P, Q, precise=True)
    for graph in (False, True, True):
        got = split_ctx.distance_batch([P], [Q], precise=True, graph=graph)[0]
        for k in EXACT:
            assert got[k] == want[k], (graph, k, got[k], want[k])


def test_split_small_batch(split_ctx, plain_ctx, built):
    """A call of a few pairs (at most 8 split): each pair of enough strips gets its own mirror
    and meet, smaller pairs run whole in the same launches; plain, learned and coarse-bound
    forms field for field against the unsplit context, the plain form against the oracle."""
    specs = [(1, 3, 3000, 2800), (0, 2, 900, 2500), (1, 2, 2100, 90), (0, 3, 40, 50),
             (1, 3, 1500, 1700)]
    pairs = [built.gen_pair(st, d, n1, n2, 100.0 if st else 1.0, 0.1, 59, k)
             for k, (st, d, n1, n2) in enumerate(specs)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(precise=True), dict(precise=True, model=model, coarse_ub=6),
                   dict(precise=False)):
            a = plain_ctx.distance_batch(Ps, Qs, **kw)
            b = split_ctx.distance_batch(Ps, Qs, **kw)
            for n, (x, y) in enumerate(zip(a, b)):
                for k in EXACT:
                    assert x[k] == y[k], (kw, n, k, x[k], y[k])
    finally:
        model.close()
    got = split_ctx.distance_batch(Ps, Qs, precise=True)
    th = oracle.max_threads()
    for n in (0, 1, 3):
        want = oracle.distance(Ps[n], Qs[n], stop_mode=1, quirks=False, threads=th)
        for k in ("distance", "dfd", "vefd", "probes"):
            assert got[n][k] == want[k], (n, k, got[n][k], want[k])


@pytest.fixture(scope="module", params=[2, 3, 7])
def win_split_ctx(built, request):
    c = _ctx(built, RFD_SPLIT=2, RFD_TEAM_RING_ROWS=request.param)
    yield c
    c.close()


@pytest.mark.parametrize("style,d,n1,n2", PAIRS[:5])
def test_split_in_launch_windows(win_split_ctx, built, style, d, n1, n2):
    """Both halves in launch windows (rings of 2, 3 and 7 rows each: window g of every half
    at once, the meet after the last): solves, bounds and the reference mode against the
    oracle."""
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 61, n1)
    th = oracle.max_threads()
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=th)
    got = win_split_ctx.distance(P, Q, precise=True)
    for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])
    assert win_split_ctx.bounds(P, Q, quirks=False, dense=True) == (want["dfd"], want["vefd"])
    want = oracle.distance(P, Q, stop_mode=0, quirks=True, threads=th)
    got = win_split_ctx.distance(P, Q)
    for k in ("distance", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])
