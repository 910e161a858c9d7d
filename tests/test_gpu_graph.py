"""rfd_options.graph: a call's device work captured as one CUDA graph and replayed by later
calls with the same layout.  Results equal the direct launches' bit for bit, a replay reads
the new call's inputs, and a new layout captures a new graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("distance", "lb", "ub", "dfd", "vefd", "endpoint", "probes", "flags")


def batch(built, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(24):
        n1, n2 = 80 + 37 * k, 60 + 53 * ((k * 7) % 11)
        d = 2 + k % 2
        out.append((np.cumsum(rng.normal(size=(n1, d)), 0), np.cumsum(rng.normal(size=(n2, d)), 0)))
    return out


def same(a, b):
    for x, y in zip(a, b):
        for key in KEYS:
            assert x[key] == y[key], (key, x[key], y[key])


def test_graph_replays_with_new_inputs(ctx, built):
    model = built.Model.pretrained(0)
    for kw in ({}, {"model": model}, {"coarse_ub": 4}):
        ps = batch(built, 1)
        Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
        want = ctx.distance_batch(Ps, Qs, precise=True, **kw)
        same(ctx.distance_batch(Ps, Qs, precise=True, graph=True, **kw), want)   # capture
        same(ctx.distance_batch(Ps, Qs, precise=True, graph=True, **kw), want)   # replay
        # same sizes, other coordinates: the replay reads the new staging data
        qs = batch(built, 2)
        Ps2, Qs2 = [p for p, _ in qs], [q for _, q in qs]
        want2 = ctx.distance_batch(Ps2, Qs2, precise=True, **kw)
        assert any(a["distance"] != b["distance"] for a, b in zip(want, want2))
        same(ctx.distance_batch(Ps2, Qs2, precise=True, graph=True, **kw), want2)


def test_graph_new_layout_and_single_pairs(ctx, built):
    ps = batch(built, 3)
    Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
    a = ctx.distance_batch(Ps[:10], Qs[:10], precise=True, graph=True)
    b = ctx.distance_batch(Ps, Qs, precise=True, graph=True)  # another layout: new capture
    same(a, ctx.distance_batch(Ps[:10], Qs[:10], precise=True))
    same(b, ctx.distance_batch(Ps, Qs, precise=True))
    for P, Q in ps[:4]:
        for precise in (False, True):
            same([ctx.distance(P, Q, precise=precise, graph=True)],
                 [ctx.distance(P, Q, precise=precise)])


def test_graph_with_phase_timing(built):
    """Phase events recorded inside the captured graph time the replays as well."""
    c = built.Context(0)
    try:
        ps = batch(built, 4)
        Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
        c.phase_times(1)
        want = c.distance_batch(Ps, Qs, precise=True)
        for rep in range(2):  # capture, then replay
            c.phase_times(1)
            same(c.distance_batch(Ps, Qs, precise=True, graph=True), want)
            pt = c.phase_times(1)
            assert pt["calls"] == 1
            assert pt["dfd_ms"] > 0 and pt["vefd_ms"] > 0 and pt["search_ms"] > 0, pt
    finally:
        c.close()
