"""Launch windows of the VE-FD and decision strips: O(n+m) boundary memory.

With one boundary row per 32-row strip, the team strips need about n1 n2 / 4 bytes; two
curves of 10^6 points would need 250 GB.  In launch windows of W strips, strip s writes ring
row s % (W + 1), each window's rows are reset right before its launch, and the next window
starts after it ends.  RFD_TEAM_RING_ROWS = R forces windows of R - 1 strips on every call;
a lone pair whose workspace exceeds the budget (RFD_BATCH_BUDGET, else 3/4 of the memory the
context may use) gets them by itself.  Checked here, bit for bit against the CPU oracle:
bounds, decisions at several radii, full solves and batches under rings of 2, 3 and 7 rows
(windows of 1, 2 and 6 strips: nearly every strip reuses a row); the long pair's plain search
under 1025-row rings against its golden; the automatic windows under a small budget; and a
1,000,000 x 1,000,000-point pair, which cannot hold a row per strip on one GPU.
"""
import json
import os

import pytest

import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
REL = 2.0 ** -33


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


@pytest.fixture(scope="module", params=[2, 3, 7])
def win_ctx(built, request):
    c = _ctx(built, RFD_TEAM_RING_ROWS=request.param)
    yield c
    c.close()


# sizes around the 32-row strips and 32-column chunks, both orientations (the team strips
# run on the transposed grid when the first curve is the longer), 2D and 3D
PAIRS = [(0, 2, 1000, 700), (0, 2, 700, 1000), (1, 3, 2000, 1900), (1, 3, 32 * 45 + 1, 900),
         (0, 3, 300, 2500), (1, 2, 4100, 130), (0, 2, 33, 65)]


@pytest.mark.parametrize("style,d,n1,n2", PAIRS)
def test_windowed_solves_bitexact(win_ctx, built, style, d, n1, n2):
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 41, n1)
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
    got = win_ctx.distance(P, Q, precise=True)
    for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])
    # the reference configuration: FLT_EPSILON stop, VE-FD launch quirk
    want = oracle.distance(P, Q, stop_mode=0, quirks=True, threads=oracle.max_threads())
    got = win_ctx.distance(P, Q)
    for k in ("distance", "lb", "ub", "probes"):
        assert got[k] == want[k], (k, got[k], want[k])


@pytest.mark.parametrize("style,d,n1,n2", PAIRS[:5])
def test_windowed_bounds_and_decisions_bitexact(win_ctx, built, style, d, n1, n2):
    P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 43, n1)
    want = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
    for dense in (False, True):
        dfd, vefd = win_ctx.bounds(P, Q, quirks=False, dense=dense)
        assert (dfd, vefd) == (want["dfd"], want["vefd"]), dense
    fd = want["distance"]
    for e in (fd * 0.9, fd * (1 - 1e-9), fd, fd * (1 + 1e-9), fd * 1.1, want["vefd"]):
        want_reach, want_ub = oracle.decide(P, Q, e)
        for dense in (False, True):
            reach, ub = win_ctx.decide(P, Q, e, dense=dense)
            assert (reach, ub) == (want_reach, want_ub), (e, dense)


def test_windowed_batch_bitexact(win_ctx, ctx, built):
    """Uneven pairs in one call: every window is a range of the strip-major item list, so
    pairs of different heights share the windows.  Plain, learned and coarse-bound forms
    equal the one-row-per-strip path, and the plain form equals the oracle."""
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 60, 17)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 3000),
                            min(int(n2[k]), 3000), float(scales[k]), float(noises[k]), 17, k)
             for k in range(60)]
    Ps, Qs = [a for a, _ in pairs], [b for _, b in pairs]
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(precise=True), dict(precise=True, model=model, coarse_ub=6)):
            a = ctx.distance_batch(Ps, Qs, search_arity=1, **kw)
            b = win_ctx.distance_batch(Ps, Qs, **kw)
            for n, (x, y) in enumerate(zip(a, b)):
                for k in ("distance", "lb", "ub", "dfd", "vefd", "probes", "flags"):
                    assert x[k] == y[k], (kw, n, k, x[k], y[k])
    finally:
        model.close()
    got = win_ctx.distance_batch(Ps, Qs, precise=True)
    for n in range(0, 60, 6):
        want = oracle.distance(Ps[n], Qs[n], stop_mode=1, quirks=False,
                               threads=oracle.max_threads())
        for k in ("distance", "dfd", "vefd", "probes"):
            assert got[n][k] == want[k], (n, k, got[n][k], want[k])


def test_long_pair_windowed_golden(built):
    """The 200,000-point long pair's plain search in windows of 1024 strips (7 windows a
    phase) reproduces the oracle's golden bit for bit."""
    gold = json.load(open(os.path.join(HERE, "golden", "config_goldens.json")))["cases"]
    want = gold["config1/0"]
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(1, 1, 1)
    P, Q = built.gen_pair(int(styles[0]), int(dims[0]), int(n1[0]), int(n2[0]),
                          float(scales[0]), float(noises[0]), 1, 0)
    c = _ctx(built, RFD_TEAM_RING_ROWS=1025)
    try:
        got = c.distance(P, Q, precise=True)
        for k in ("endpoint", "dfd", "vefd", "distance", "lb", "ub", "probes"):
            assert got[k] == want[k], (k, got[k], want[k])
        assert c.decide(P, Q, want["threshold"]) == (want["threshold_reach"],
                                                     want["threshold_right_ub"])
    finally:
        c.close()


def test_automatic_windows_under_a_small_budget(built, monkeypatch):
    """A lone pair whose rows exceed RFD_BATCH_BUDGET runs in windows by itself: the same
    results in less than half the device memory."""
    import torch
    P, Q = built.gen_pair(1, 2, 20000, 19000, 100.0, 0.1, 47, 0)
    used = {}
    res = {}
    for budget in (None, "30000000"):
        c = built.Context(0)
        try:
            if budget:
                monkeypatch.setenv("RFD_BATCH_BUDGET", budget)
            free0 = torch.cuda.mem_get_info(0)[0]
            res[budget] = c.distance(P, Q, precise=True)
            used[budget] = free0 - torch.cuda.mem_get_info(0)[0]
            monkeypatch.delenv("RFD_BATCH_BUDGET", raising=False)
        finally:
            c.close()
    for k in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
        assert res[None][k] == res["30000000"][k], k
    # one row per strip: 593 rows of 20,032 doubles (95 MB); windows: under the 30 MB budget
    assert used[None] > 80e6, used
    assert used["30000000"] < 45e6, used


def test_million_point_pair_solves(built):
    """Two 3D spline paths of 1,000,000 points (10^12 cells; a row per strip would take
    250 GB).  The learned form with the coarse upper bound solves it in windows: the
    distance lies within the stop rule between its bounds, and a decision at the final upper
    end (a radius the search found reachable) is reachable again."""
    import torch
    P, Q = built.gen_pair(1, 3, 1_000_000, 1_000_000, 100.0, 0.1, 1, 7)
    assert len(P) == len(Q) == 1_000_000
    c = built.Context(0)
    model = built.Model.pretrained(0)
    try:
        free0 = torch.cuda.mem_get_info(0)[0]
        got = c.distance(P, Q, precise=True, model=model, coarse_ub=6)
        used = free0 - torch.cuda.mem_get_info(0)[0]
        assert used < 60e9, used  # rows of 4097 strips of 10^6 doubles: 33 GB
        assert got["vefd"] <= got["lb"] <= got["distance"] <= got["ub"] <= got["dfd"], got
        assert got["ub"] - got["lb"] <= REL * got["ub"], got
        if got["ub"] < got["dfd"]:
            assert c.decide(P, Q, got["ub"])[0], got
    finally:
        model.close()
        c.close()
