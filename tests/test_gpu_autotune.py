"""The autotuners: rfd_autotune (the DFD sweep's tile shape: rows per lane, stacked or skewed
rows) and rfd_autotune_search (warps per team, the switch point to the continuous search and
its start window), timed on the caller's pairs; the fastest is kept, and results stay
bit-identical whatever they pick."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_keeps_a_candidate_and_results(ctx, built):
    rng = np.random.default_rng(5)
    ps = [(np.cumsum(rng.normal(size=(300 + 97 * k, 2 + k % 2)), 0),
           np.cumsum(rng.normal(size=(250 + 61 * k, 2 + k % 2)), 0)) for k in range(16)]
    Ps, Qs = [p for p, _ in ps], [q for _, q in ps]
    want = ctx.distance_batch(Ps, Qs, precise=True)
    c = built.Context(0)
    try:
        tuned = c.autotune(Ps, Qs, reps=1)
        assert tuned["rows"] in (1, 2, 4, 8) and tuned["skew"] in (0, 1)
        assert len(tuned["ms"]) == 8 and all(v > 0 for v in tuned["ms"].values())
        assert tuned["ms"][(tuned["rows"], tuned["skew"])] == min(tuned["ms"].values())
        got = c.distance_batch(Ps, Qs, precise=True)
        for a, b in zip(want, got):
            for key in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
                assert a[key] == b[key], key
        with pytest.raises(built.RfdError):
            c.autotune(Ps, Qs, reps=0)
    finally:
        c.close()


def test_autotune_search_keeps_a_candidate_and_results(ctx, built):
    """rfd_autotune_search: warps per team (4 or 8), the switch point to the continuous search
    and its start window, timed on whole solves; every candidate gives the same results, and
    the context keeps the fastest."""
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, 96, 21)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), 4000),
                            min(int(n2[k]), 4000), float(scales[k]), float(noises[k]), 21, k)
             for k in range(96)]
    Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
    model = built.Model.pretrained(0)
    c = built.Context(0)
    try:
        for kw in (dict(precise=True), dict(precise=True, model=model)):
            want = ctx.distance_batch(Ps, Qs, **kw)
            tuned = c.autotune_search(Ps, Qs, reps=1, **kw)
            assert tuned["warps"] in (4, 8) and tuned["window"] in (1, 2, 4)
            assert len(tuned["ms"]) == 18 and all(v > 0 for v in tuned["ms"].values())
            got = c.distance_batch(Ps, Qs, **kw)
            for a, b in zip(want, got):
                for key in ("distance", "dfd", "vefd", "lb", "ub", "probes", "flags"):
                    assert a[key] == b[key], key
    finally:
        c.close()
        model.close()


def test_team_of_four_warps_bitexact(built):
    """Teams of 4 warps (3 helpers) against the oracle: the same values as teams of 8."""
    import os

    import oracle
    os.environ["RFD_TEAM_WARPS"] = "4"
    try:
        c = built.Context(0)
    finally:
        del os.environ["RFD_TEAM_WARPS"]
    try:
        for style, d, n1, n2 in ((0, 2, 700, 650), (1, 3, 3000, 2800), (1, 2, 1500, 40)):
            P, Q = built.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, 23, n1)
            w = oracle.distance(P, Q, stop_mode=1, quirks=False, threads=oracle.max_threads())
            for dense in (False, True):
                g = c.distance(P, Q, precise=True, dense=dense)
                for key in ("distance", "dfd", "vefd", "lb", "ub", "probes"):
                    assert g[key] == w[key], (key, dense)
    finally:
        c.close()
