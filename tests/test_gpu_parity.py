"""CUDA path (through the C ABI) against the CPU oracle on seeded inputs.

Bar: bit-exact.  DFD and VE-FD are compared as the doubles the reference reports
(sqrt of the DP value), every decision's propagated right UB must be identical, and a
full search must reproduce the oracle's probe count and distance bit for bit (both run
the same bisection on the same decisions).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def walk_pair(seed, n1, n2, d=2, noise=0.05):
    rng = np.random.default_rng(seed)
    P = np.cumsum(rng.normal(size=(n1, d)), 0)
    idx = np.linspace(0, n1 - 1, n2)
    base = np.stack([np.interp(idx, np.arange(n1), P[:, k]) for k in range(d)], 1)
    return P, base + rng.normal(scale=noise, size=(n2, d))


# sizes around the 32-row strip and 32-column chunk boundaries (and multiples), both orientations
SIZES = [(2, 2), (2, 40), (40, 2), (3, 3), (31, 31), (32, 33), (33, 32), (34, 65), (65, 34),
         (64, 64), (63, 40), (66, 70), (97, 130), (129, 50), (130, 129), (200, 150), (257, 31),
         (31, 257)]


@pytest.mark.parametrize("n1,n2", SIZES)
@pytest.mark.parametrize("d", [2, 3])
def test_bounds_bitexact(ctx, n1, n2, d):
    P, Q = walk_pair(n1 * 1000 + n2 + d, n1, n2, d)
    lb = oracle.endpoint(P, Q)
    want_dfd = np.sqrt(oracle.dfd_sq(P, Q))
    want_vefd = np.sqrt(oracle.vefd_sq(P, Q, lb))
    for dense in (False, True):
        dfd, vefd = ctx.bounds(P, Q, quirks=False, dense=dense)
        assert dfd == want_dfd, (dense, dfd, want_dfd)
        assert vefd == want_vefd, (dense, vefd, want_vefd)


@pytest.mark.parametrize("n1,n2", SIZES)
@pytest.mark.parametrize("d", [2, 3])
def test_decisions_bitexact(ctx, n1, n2, d):
    P, Q = walk_pair(n1 * 7 + n2 * 3 + d, n1, n2, d)
    r = oracle.distance(P, Q, stop_mode=1, quirks=False)
    fd = r["distance"]
    radii = [r["endpoint"], fd * 0.5, fd * (1 - 1e-6), fd, fd * (1 + 1e-6), fd * 1.5, r["dfd"],
             r["dfd"] * 3]
    for e in radii:
        want_reach, want_ub = oracle.decide(P, Q, e)
        for dense in (False, True):
            reach, ub = ctx.decide(P, Q, e, dense=dense)
            assert ub == want_ub and reach == want_reach, (e, dense, ub, want_ub)


@pytest.mark.parametrize("n1,n2", [(70, 20), (257, 31), (40, 2), (33, 32), (20, 70)])
@pytest.mark.parametrize("d", [2, 3])
def test_decisions_at_the_last_corner(ctx, n1, n2, d):
    """Pairs with a longer first curve run their decision strips on the transposed grid, whose
    result is the last cell's top edge there.  At radii within a few ulps of the end-point
    distance the last cell's corner sits on the ball's boundary, where the right and top
    edges' intervals are computed from different quadratics; reach and the right edge's UB
    must still be the oracle's, in the given orientation and in the swapped one."""
    for seed in range(3):
        P, Q = walk_pair(seed * 101 + n1 + n2 + d, n1, n2, d)
        Q[0] = P[0]
        Q[-1] = P[-1] + 3.0 / np.sqrt(d)  # the end distance is the endpoint bound
        e = oracle.endpoint(P, Q)
        radii = [e]
        lo = hi = e
        for _ in range(3):
            lo, hi = np.nextafter(lo, 0.0), np.nextafter(hi, np.inf)
            radii += [lo, hi]
        for A, B in ((P, Q), (Q, P)):
            for r in radii:
                want = oracle.decide(A, B, r)
                got = ctx.decide(A, B, r)
                assert got == want, (seed, r, got, want)


@pytest.mark.parametrize("seed,n1,n2,d", [(0, 120, 90, 2), (1, 90, 160, 3), (2, 300, 280, 2),
                                          (3, 64, 400, 3), (4, 700, 650, 3)])
@pytest.mark.parametrize("precise", [False, True])
def test_distance_bitexact(ctx, seed, n1, n2, d, precise):
    P, Q = walk_pair(seed, n1, n2, d)
    want = oracle.distance(P, Q, stop_mode=1 if precise else 0, quirks=not precise, threads=4)
    for dense in (False, True):
        got = ctx.distance(P, Q, precise=precise, dense=dense)
        assert got["probes"] == want["probes"]
        assert got["dfd"] == want["dfd"] and got["vefd"] == want["vefd"]
        assert got["lb"] == want["lb"] and got["ub"] == want["ub"]
        assert got["distance"] == want["distance"]


def test_config0_distance_bitexact(ctx, built):
    P, Q = built.gen_config(0)[0]
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=8)
    got = ctx.distance(P, Q, precise=True)
    assert got["distance"] == want["distance"] and got["probes"] == want["probes"]
    ref = oracle.distance(P, Q, stop_mode=0, quirks=True, threads=8)
    got = ctx.distance(P, Q)
    assert got["distance"] == ref["distance"] and got["probes"] == ref["probes"]
    assert got["cells_evaluated"] < got["cells_nominal"]


def test_spline_pairs_bitexact(ctx, built):
    for style, d, n1, n2 in [(1, 3, 800, 900), (1, 2, 1000, 700), (0, 3, 500, 650)]:
        P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 11, n1)
        want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=8)
        got = ctx.distance(P, Q, precise=True)
        assert got["distance"] == want["distance"] and got["probes"] == want["probes"]


def test_batch_equals_single(ctx, built):
    pairs = [walk_pair(s, 20 + 37 * s, 15 + 53 * s, 2 + s % 2) for s in range(12)]
    singles = [ctx.distance(P, Q, precise=True) for P, Q in pairs]
    batch = ctx.distance_batch([p for p, _ in pairs], [q for _, q in pairs], precise=True)
    for a, b in zip(singles, batch):
        assert a["distance"] == b["distance"] and a["probes"] == b["probes"]


def test_degenerate_single_point(ctx):
    P = np.array([[1.0, 2.0]])
    Q = np.array([[0.0, 0.0], [3.0, 4.0], [1.0, 5.0]])
    want = max(np.linalg.norm(Q - P[0], axis=1))
    r = ctx.distance(P, Q, precise=True)
    assert abs(r["distance"] - want) <= 1e-15 * want
    r = ctx.distance(Q, P, precise=True)
    assert abs(r["distance"] - want) <= 1e-15 * want


def test_compute_distance_parallel_mirror(ctx, built):
    """The reference's entry point: its stop rule and VE-FD rule, and its decision path - the
    materialised intervals where they fit in device memory (always at this size), the fused
    kernel's when forceOversize is set."""
    P, Q = walk_pair(5, 150, 120, 2)
    want = oracle.distance(P, Q, stop_mode=0, quirks=True, formula=1)
    assert built.compute_distance_parallel(P, Q) == want["distance"]
    want = oracle.distance(P, Q, stop_mode=0, quirks=True, formula=0)
    assert built.compute_distance_parallel(P, Q, force_oversize=True) == want["distance"]


@pytest.mark.parametrize("style,d,n", [(1, 3, 20000), (0, 2, 12000), (1, 2, 30000)])
def test_sparse_equals_dense_large(ctx, built, style, d, n):
    """Size-independent property at sizes where consumer strips outrun their producers:
    the pruned / skipping sweeps give the dense results bit for bit, the pruned VE-FD
    needs no dense fallback, and decisions are monotone around the result."""
    P, Q = built.gen_pair(style, d, n, n - 1000, 100.0 if style else 1.0, 0.1, 123, n)
    dfd_d, vefd_d = ctx.bounds(P, Q, quirks=False, dense=True)
    dfd_s, vefd_s = ctx.bounds(P, Q, quirks=False, dense=False)
    assert (dfd_s, vefd_s) == (dfd_d, vefd_d)
    r = ctx.distance(P, Q, precise=True)
    assert not (r["flags"] & built.FLAG_VEFD_DENSE)
    assert r["vefd"] == vefd_d and r["dfd"] == dfd_d
    assert r["vefd"] <= r["distance"] <= r["dfd"]
    fd = r["distance"]
    for e in (r["vefd"], fd * (1 - 1e-7), fd * (1 + 1e-7), (fd + r["dfd"]) / 2):
        sparse = ctx.decide(P, Q, e)
        dense = ctx.decide(P, Q, e, dense=True)
        assert sparse == dense, (e, sparse, dense)
    assert not ctx.decide(P, Q, fd * (1 - 1e-7))[0]
    assert ctx.decide(P, Q, fd * (1 + 1e-7))[0]


@pytest.fixture(scope="module")
def solo_ctx(built):
    """A context whose VE-FD and decisions run on the one-warp strips (RFD_SOLO=1)."""
    import os
    old = os.environ.get("RFD_SOLO")
    os.environ["RFD_SOLO"] = "1"
    try:
        c = built.Context(0)
    finally:
        if old is None:
            del os.environ["RFD_SOLO"]
        else:
            os.environ["RFD_SOLO"] = old
    yield c
    c.close()


@pytest.mark.parametrize("style,d,n1,n2", [(0, 2, 700, 650), (1, 3, 3000, 2800), (0, 3, 97, 1300),
                                           (1, 2, 1500, 40)])
def test_team_equals_solo(ctx, solo_ctx, built, style, d, n1, n2):
    """Helper-warp tiles (team strips) and on-chain geometry (solo strips) agree bit for bit."""
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 77, n1)
    for dense in (False, True):
        a = ctx.distance(P, Q, precise=True, dense=dense)
        b = solo_ctx.distance(P, Q, precise=True, dense=dense)
        for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
            assert a[k] == b[k], (k, dense, a[k], b[k])


@pytest.fixture(scope="module")
def lockstep_ctx(built):
    """A context that runs one launch per probe round (RFD_LOCKSTEP=1)."""
    import os
    old = os.environ.get("RFD_LOCKSTEP")
    os.environ["RFD_LOCKSTEP"] = "1"
    try:
        c = built.Context(0)
    finally:
        if old is None:
            del os.environ["RFD_LOCKSTEP"]
        else:
            os.environ["RFD_LOCKSTEP"] = old
    yield c
    c.close()


@pytest.mark.parametrize("switch", [None, "60"])
def test_continuous_search_equals_lockstep(ctx, lockstep_ctx, built, switch):
    """The continuous search (a pair's next probe queued as its last one ends, one launch)
    and one launch per probe round give the same results bit for bit: every probe's
    boundary words are cleared before the next probe reads them.  Uneven pairs, so pairs end
    their probes at different times; with and without the learned bracket, dense, reference
    mode, and a max_probes cap.  With the default switch (the team count) these 160 pairs
    run continuously from the first probe; with 60, probe rounds run as launches until fewer
    than 60 pairs are left, and the continuous search takes over mid-search."""
    import os
    if switch is not None:
        os.environ["RFD_SEARCH_SWITCH"] = switch
        try:
            ctx = built.Context(0)
        finally:
            del os.environ["RFD_SEARCH_SWITCH"]
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 160, 9)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 3000),
                            min(int(n2[k]), 3000), float(scales[k]), float(noises[k]), 9, k)
             for k in range(160)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    keys = ("distance", "lb", "ub", "dfd", "vefd", "probes", "flags")
    model = built.Model.pretrained(0)
    for kw in (dict(precise=True), dict(precise=True, model=model), dict(precise=False),
               dict(precise=True, dense=True), dict(precise=True, max_probes=5),
               dict(precise=True, graph=True)):
        a = ctx.distance_batch(Ps, Qs, **kw)
        b = lockstep_ctx.distance_batch(Ps, Qs, **kw)
        for n, (x, y) in enumerate(zip(a, b)):
            for k in keys:
                assert x[k] == y[k], (kw, n, k, x[k], y[k])
        assert max(x["probes"] for x in a) > 3
    if switch is not None:
        ctx.close()


def test_reference_driver_golden(ctx, built):
    """The CUDA path in the reference's configuration reproduces the reference's own search
    driver (tests/golden/reference_host.json) bit for bit."""
    import json
    import os
    from tests.golden.cases import build_input
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_host.json")) as f:
        cases = json.load(f)["distance"]
    for c in cases:
        P, Q = build_input(c["input"])
        r = ctx.distance(P, Q)
        assert r["endpoint"] == c["endpoint"], c["name"]
        assert r["distance"] == c["distance"], c["name"]


@pytest.mark.parametrize("skew", ["0", "1"])
@pytest.mark.parametrize("rows", ["1", "2", "4", "8"])
def test_dfd_rows_per_lane_bitexact(built, rows, skew):
    """Dense DFD strips of 32 * rows rows, stacked or skewed rows per lane: sizes around the
    strip and chunk boundaries."""
    import os
    env = {"RFD_DFD_ROWS": rows, "RFD_DFD_SKEW": skew}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        c = built.Context(0)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    h = 32 * int(rows)
    sizes = [(2, 2), (h - 1, 40), (h, 33), (h + 1, 65), (2 * h + 3, 31), (3 * h - 1, 257), (31, 2 * h)]
    try:
        for k, (n1, n2) in enumerate(sizes):
            for d in (2, 3):
                P, Q = walk_pair(k * 31 + n1 + d, n1, n2, d)
                dfd, _ = c.bounds(P, Q, quirks=False)
                assert dfd == np.sqrt(oracle.dfd_sq(P, Q)), (rows, skew, n1, n2, d)
    finally:
        c.close()


@pytest.mark.parametrize("k", [2, 8, 64])
def test_coarse_upper_bound(ctx, built, k):
    """rfd_options.coarse_ub: a certified upper bound in place of the DFD.  VE-FD is pruned by
    it exactly (bit-identical), the FD agrees within the stop rule, and the bound is >= DFD."""
    cases = [built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 61, 0),
             built.gen_pair(0, 2, 900, 850, 1.0, 0.05, 61, 1),
             built.gen_pair(1, 2, 257, 4000, 100.0, 0.1, 61, 2),
             (np.array([[0.5, 0.5]]), built.gen_pair(0, 2, 50, 60, 1.0, 0.05, 61, 3)[1])]
    tol = 2.0 ** -33
    for n, (P, Q) in enumerate(cases):
        a = ctx.distance(P, Q, precise=True)
        b = ctx.distance(P, Q, precise=True, coarse_ub=k)
        assert b["vefd"] == a["vefd"], n
        assert abs(b["distance"] - a["distance"]) <= 2 * tol * a["distance"], n
        if len(P) >= 2 and len(Q) >= 2:
            assert b["flags"] & built.FLAG_DFD_COARSE and b["dfd"] >= a["dfd"], n
        else:  # a one-point curve keeps the exact DFD, its closed-form answer
            assert b["distance"] == a["distance"] and not (b["flags"] & built.FLAG_DFD_COARSE)
    Ps, Qs = [c[0] for c in cases], [c[1] for c in cases]
    got = ctx.distance_batch(Ps, Qs, precise=True, coarse_ub=k, model=built.Model.pretrained(0))
    for n, (P, Q) in enumerate(cases):
        want = ctx.distance(P, Q, precise=True)["distance"]
        assert abs(got[n]["distance"] - want) <= 2 * tol * want, n


def test_coarse_upper_bound_checked(ctx, built):
    P, Q = built.gen_pair(0, 2, 100, 90, 1.0, 0.05, 61, 4)
    for bad in (dict(coarse_ub=1), dict(coarse_ub=-3), dict(coarse_ub=8, precise=False)):
        with pytest.raises(built.RfdError):
            ctx.distance(P, Q, **bad)
