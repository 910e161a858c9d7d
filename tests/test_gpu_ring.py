"""The DFD's boundary ring: rows handed between DFD strips reuse a few rows per pair.

DFD strip s writes ring row s % ring, handing it on column by column: its reader clears each
chunk once read and publishes the cleared count, the row's next writer writes only cleared
columns, and that writer's reader trusts only covered columns.  These tests force rings of 2
and 3 rows (RFD_DFD_RING_ROWS), so nearly every strip reuses a row while the strips before it
still run, and check the DFD bit for bit against the CPU oracle for every tile shape (rows
per lane 1, 2, 4, 8, stacked and skewed), inside full solves and batches (exact and coarse
upper bound), and a batch split into workspace-bounded chunks against one call.
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
    c = _ctx(built, RFD_DFD_RING_ROWS=request.param)
    yield c
    c.close()


PAIRS = [(0, 2, 1000, 700), (0, 2, 700, 1000), (1, 3, 2000, 1900), (1, 3, 32 * 45 + 1, 900),
         (0, 3, 300, 2500), (1, 2, 4100, 130)]


@pytest.mark.parametrize("style,d,n1,n2", PAIRS)
def test_small_dfd_ring_solves_bitexact(ring_ctx, built, style, d, n1, n2):
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 31, n1)
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
    got = ring_ctx.distance(P, Q, precise=True)
    for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])


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


def test_small_dfd_ring_batch_equals_default(ring_ctx, ctx, built):
    """Uneven pairs in one call, exact DFD and the coarse bound's inflated DFD: the default
    ring and the small ring agree bit for bit."""
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 120, 13)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 6000),
                            min(int(n2[k]), 6000), float(scales[k]), float(noises[k]), 13, k)
             for k in range(120)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(precise=True), dict(precise=True, model=model, coarse_ub=6),
                   dict(precise=False)):
            a = ctx.distance_batch(Ps, Qs, **kw)
            b = ring_ctx.distance_batch(Ps, Qs, **kw)
            for n, (x, y) in enumerate(zip(a, b)):
                for k in ("distance", "lb", "ub", "dfd", "vefd", "probes", "flags"):
                    assert x[k] == y[k], (kw, n, k, x[k], y[k])
    finally:
        model.close()


def test_chunked_batch_equals_whole(ctx, built, monkeypatch):
    """RFD_BATCH_BUDGET (read at every call) of a few pairs' workspace splits the call."""
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 40, 15)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 5000),
                            min(int(n2[k]), 5000), float(scales[k]), float(noises[k]), 15, k)
             for k in range(40)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    whole = ctx.distance_batch(Ps, Qs, precise=True)
    brackets = [(r["distance"] * (1 - 1e-6), r["distance"] * (1 + 1e-6)) for r in whole]
    for kw in (dict(precise=True), dict(precise=True, brackets=brackets)):
        a = ctx.distance_batch(Ps, Qs, **kw)
        monkeypatch.setenv("RFD_BATCH_BUDGET", "20000000")
        b = ctx.distance_batch(Ps, Qs, **kw)
        monkeypatch.delenv("RFD_BATCH_BUDGET")
        for x, y in zip(a, b):
            for k in ("distance", "lb", "ub", "probes", "flags"):
                assert x[k] == y[k], (kw, k, x[k], y[k])
