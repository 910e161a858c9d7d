"""The boundary ring: rows handed between strips reuse a few rows per pair.

Strip s writes ring row s % ring.  Team strips (VE-FD, decisions) claim a row from a strip
that has ended and clear what it wrote; DFD strips hand a row on column by column.  These
tests force rings of 2 and 3 rows (RFD_RING_ROWS, RFD_DFD_RING_ROWS), so nearly every strip
reuses a row while the strips before it still run, and check the results bit for bit against
the CPU oracle and against the default ring: single pairs in both orientations, every DFD
tile shape, dense and pruned sweeps, the continuous search over an uneven batch, the coarse
upper bound and the learned bracket.  A 1,000,000 x 1,000,000-point pair (about 250 GB of
boundary rows with one row per strip) solves in a ring of 128 rows a pair, checked by the
decisions at its final bracket.  A batch split into workspace-bounded chunks gives the same
results as one call.
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


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


@pytest.fixture(scope="module", params=[2, 3])
def ring_ctx(built, request):
    c = _ctx(built, RFD_RING_ROWS=request.param, RFD_DFD_RING_ROWS=request.param)
    yield c
    c.close()


PAIRS = [(0, 2, 1000, 700), (0, 2, 700, 1000), (1, 3, 2000, 1900), (1, 3, 32 * 45 + 1, 900),
         (0, 3, 300, 2500), (1, 2, 4100, 130)]


@pytest.mark.parametrize("style,d,n1,n2", PAIRS)
def test_small_ring_bitexact(ring_ctx, built, style, d, n1, n2):
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 31, n1)
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
    for dense in (False, True):
        got = ring_ctx.distance(P, Q, precise=True, dense=dense)
        for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
            assert got[k] == want[k], (dense, k, got[k], want[k])
    for e in (want["distance"] * (1 - 1e-9), want["distance"] * (1 + 1e-9), want["dfd"]):
        assert ring_ctx.decide(P, Q, e) == oracle.decide(P, Q, e, threads=oracle.max_threads())


@pytest.mark.parametrize("rows", ["1", "2", "4", "8"])
@pytest.mark.parametrize("skew", ["0", "1"])
def test_small_dfd_ring_every_tile_shape(built, rows, skew):
    c = _ctx(built, RFD_DFD_RING_ROWS=2, RFD_DFD_ROWS=rows, RFD_DFD_SKEW=skew)
    try:
        for n1, n2, d in ((32 * 8 * int(rows) * 3 + 5, 900, 2), (1500, 2100, 3)):
            P, Q = built.gen_pair(1, d, n1, n2, 100.0, 0.1, 32, n1)
            dfd, _ = c.bounds(P, Q, quirks=False)
            assert dfd == np.sqrt(oracle.dfd_sq(P, Q, oracle.max_threads())), (n1, n2, d)
    finally:
        c.close()


def test_small_ring_batch_equals_default(ring_ctx, ctx, built):
    """Uneven pairs in one call: continuous search, learned bracket, coarse bound, FP32
    filter, reference mode; the default ring (rows never reused for these sizes) and the
    small ring agree bit for bit."""
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 120, 13)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 6000),
                            min(int(n2[k]), 6000), float(scales[k]), float(noises[k]), 13, k)
             for k in range(120)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(precise=True), dict(precise=True, model=model),
                   dict(precise=True, model=model, coarse_ub=6),
                   dict(precise=True, precision=built.RFD_PREC_FP32_FILTER),
                   dict(precise=False), dict(precise=True, dense=True, max_probes=4)):
            a = ctx.distance_batch(Ps, Qs, **kw)
            b = ring_ctx.distance_batch(Ps, Qs, **kw)
            for n, (x, y) in enumerate(zip(a, b)):
                for k in ("distance", "lb", "ub", "dfd", "vefd", "probes", "flags"):
                    assert x[k] == y[k], (kw, n, k, x[k], y[k])
    finally:
        model.close()


def test_small_ring_lockstep(built):
    c = _ctx(built, RFD_RING_ROWS=2, RFD_DFD_RING_ROWS=2, RFD_LOCKSTEP=1)
    try:
        dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 24, 14)
        pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 4000),
                                min(int(n2[k]), 4000), float(scales[k]), float(noises[k]), 14, k)
                 for k in range(24)]
        res = c.distance_batch([a for a, _ in pairs], [b for _, b in pairs], precise=True)
        for (P, Q), r in zip(pairs, res):
            w = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
            assert (r["distance"], r["probes"]) == (w["distance"], w["probes"])
    finally:
        c.close()


def test_chunked_batch_equals_whole(ctx, built):
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 40, 15)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 5000),
                            min(int(n2[k]), 5000), float(scales[k]), float(noises[k]), 15, k)
             for k in range(40)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    whole = ctx.distance_batch(Ps, Qs, precise=True)
    brackets = [(r["distance"] * (1 - 1e-6), r["distance"] * (1 + 1e-6)) for r in whole]
    c = _ctx(built, RFD_BATCH_BUDGET=4_000_000)  # a few pairs a chunk
    try:
        for kw in (dict(precise=True), dict(precise=True, brackets=brackets)):
            a = ctx.distance_batch(Ps, Qs, **kw)
            b = c.distance_batch(Ps, Qs, **kw)
            for x, y in zip(a, b):
                for k in ("distance", "lb", "ub", "probes", "flags"):
                    assert x[k] == y[k], (kw, k, x[k], y[k])
    finally:
        c.close()


def test_million_point_pair(ctx, built):
    """One row per strip would need n1 n2 / 4 = 250 GB of boundary rows; the ring needs
    about 1 GB.  The final bracket is checked by its two decisions (lb unreachable, ub
    reachable), and the coarse bound's distance agrees with the exact DFD's within the stop
    rule."""
    P, Q = built.gen_pair(1, 3, 1_000_000, 1_000_000, 100.0, 0.1, 1, 0)
    model = built.Model.pretrained(0)
    try:
        r = ctx.distance(P, Q, precise=True, model=model, coarse_ub=6)
    finally:
        model.close()
    assert r["lb"] < r["ub"] <= r["lb"] * (1 + 2.0 ** -33) * (1 + 1e-15)
    assert ctx.decide(P, Q, r["ub"])[0]
    if r["lb"] > r["vefd"]:
        assert not ctx.decide(P, Q, r["lb"])[0]
    assert r["vefd"] <= r["distance"] <= r["dfd"]
    assert np.isfinite(r["distance"])
