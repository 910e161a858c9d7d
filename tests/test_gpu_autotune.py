"""rfd_autotune: the DFD sweep's tile shape (rows per lane, stacked or skewed rows) timed on
the caller's pairs; the fastest is kept, and results stay bit-identical whatever it picks."""
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
