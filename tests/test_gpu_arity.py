"""k-ary rounds of the batched search (rfd_options.search_arity).

With search_arity = K, the pairs whose probe chains are longest decide K radii per bisection
round once few pairs remain, splitting the bracket into K + 1 parts.  Only the probe sequence
changes, so the bars are those of any search that is not the reference's bisection:
  - DFD and VE-FD bit for bit as without it;
  - every final bracket within the stop rule (ub - lb <= 2^-33 ub), and no probe cap hit;
  - the final bracket's ends decided as the CPU oracle decides them: ub reachable and lb
    unreachable, wherever that end is a probed radius (not the DFD or VE-FD bound);
  - the distance within the stop rule of the plain form's.
RFD_ARITY_GATE forces the rounds from the first continuous probe on, so that small batches
exercise them.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

REL = 2.0 ** -33
SF_MAX_PROBES = 4  # rfd_flag bit of a search stopped by the probe cap


def _batch(built, n, seed, clip):
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(2, n, seed)
    pairs = [built.gen_pair(int(styles[k]), int(dims[k]), min(int(n1[k]), clip),
                            min(int(n2[k]), clip), float(scales[k]), float(noises[k]), seed, k)
             for k in range(n)]
    return [p for p, _ in pairs], [q for _, q in pairs]


@pytest.mark.parametrize("arity", [2, 4, 8])
@pytest.mark.parametrize("learned", [False, True])
def test_kary_rounds_keep_bounds_and_stop_rule(ctx, built, monkeypatch, arity, learned):
    Ps, Qs = _batch(built, 96, 21, 4000)
    model = built.Model.pretrained(0) if learned else None
    try:
        kw = dict(precise=True, model=model) if learned else dict(precise=True)
        plain = ctx.distance_batch(Ps, Qs, **kw)
        monkeypatch.setenv("RFD_ARITY_GATE", "100000")
        kary = ctx.distance_batch(Ps, Qs, search_arity=arity, **kw)
        monkeypatch.delenv("RFD_ARITY_GATE")
    finally:
        if model is not None:
            model.close()
    more = 0
    for a, b in zip(plain, kary):
        assert (b["dfd"], b["vefd"]) == (a["dfd"], a["vefd"])
        assert not b["flags"] & SF_MAX_PROBES
        assert b["lb"] <= b["distance"] <= b["ub"]
        assert b["ub"] - b["lb"] <= REL * b["ub"]
        assert abs(b["distance"] - a["distance"]) <= 2 * REL * a["ub"]
        more += b["probes"] > a["probes"]
    assert more > 0, "no pair ran a k-ary round"
    # the final bracket's probed ends against the oracle, on the pairs with the most probes
    order = sorted(range(len(Ps)), key=lambda k: -kary[k]["probes"])[:6]
    t = oracle.max_threads()
    for k in order:
        r = kary[k]
        if r["ub"] < r["dfd"]:
            assert oracle.decide(Ps[k], Qs[k], r["ub"], threads=t)[0], (k, r)
        if r["lb"] > r["vefd"]:
            assert not oracle.decide(Ps[k], Qs[k], r["lb"], threads=t)[0], (k, r)


def test_kary_default_gate_and_graph_replay(ctx, built):
    """The default gate (rounds once few pairs remain), captured as a CUDA graph and replayed:
    the replay gives the captured call's results."""
    Ps, Qs = _batch(built, 160, 22, 6000)
    model = built.Model.pretrained(0)
    try:
        kw = dict(precise=True, model=model, search_arity=4, graph=True)
        a = ctx.distance_batch(Ps, Qs, **kw)
        b = ctx.distance_batch(Ps, Qs, **kw)
        plain = ctx.distance_batch(Ps, Qs, precise=True, model=model)
    finally:
        model.close()
    for x, y, z in zip(a, b, plain):
        assert x["distance"] == y["distance"] and x["probes"] == y["probes"]
        assert x["ub"] - x["lb"] <= REL * x["ub"]
        assert abs(x["distance"] - z["distance"]) <= 2 * REL * z["ub"]


@pytest.mark.parametrize("precise", [True, False])
def test_single_pair_kary_rounds(ctx, built, precise):
    """A single-pair call runs its probe rounds as launches; with search_arity each launch
    decides K radii of the pair (its members' strips interleaved in the launch's items).
    Reference mode (precise=False) keeps its absolute FLT_EPSILON stop."""
    P, Q = built.gen_pair(1, 3, 3000, 2800, 100.0, 0.1, 23, 0)
    a = ctx.distance(P, Q, precise=precise)
    b = ctx.distance(P, Q, precise=precise, search_arity=4)
    assert (b["dfd"], b["vefd"]) == (a["dfd"], a["vefd"])
    assert not b["flags"] & SF_MAX_PROBES
    tol = REL * b["ub"] if precise else float(np.finfo(np.float32).eps)
    assert b["lb"] <= b["distance"] <= b["ub"] and b["ub"] - b["lb"] <= tol
    assert abs(b["distance"] - a["distance"]) <= 2 * (REL * a["ub"] if precise else tol)
    assert b["probes"] > a["probes"]  # more decisions, in fewer rounds
    t = oracle.max_threads()
    if b["ub"] < b["dfd"]:
        assert oracle.decide(P, Q, b["ub"], threads=t)[0]
    if b["lb"] > b["vefd"]:
        assert not oracle.decide(P, Q, b["lb"], threads=t)[0]
