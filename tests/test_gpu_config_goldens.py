"""The CUDA path against the CPU oracle at the benchmark workloads' own sizes.

tests/golden/config_goldens.json holds the oracle's results (dense FP64) for
  - the long pair (2 x 200,000 points, 3D, 4.0e10 cells a decision);
  - a fixed sample of the 4096-pair uneven batch (every 16th pair and every pair with a
    curve of 30,000 points or more);
  - the first two of the 512 large 3D pairs (up to 383,833 x 378,296 points);
made by tests/golden/make_config_goldens.py.  Checked here:
  - the plain method (bisection of [VE-FD, DFD], the reference's probe sequence): endpoint
    bound, DFD, VE-FD, both bracket ends, the probe count and the distance, bit for bit;
  - the forms that change only the probe sequence (learned bracket, coarse upper bound):
    VE-FD bit for bit, the first probe (the stop threshold over VE-FD) decided as the oracle
    decides it, and the distance within the 2^-33 stop rule of the oracle's;
  - the FP32 filter, whose decisions are the FP64 ones: its plain form bit for bit;
  - for the large pairs: both bounds, and the threshold decision's propagated right UB.
"""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "config_goldens.json")))["cases"]
REL = 2.0 ** -33
EXACT = ("endpoint", "dfd", "vefd", "distance", "lb", "ub", "probes")
SEEDS = {1: 1, 2: 2, 4: 5}


def _pair(built, name):
    cfg, k = (int(v) for v in name.replace("config", "").split("/"))
    dims, n1, n2, styles, scales, noises = built.gen_batch_spec(cfg, k + 1, SEEDS[cfg])
    return built.gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]),
                          float(scales[k]), float(noises[k]), SEEDS[cfg], k)


def _check_plain(got, want, name):
    for key in EXACT:
        assert got[key] == want[key], (name, key, got[key], want[key])


def _check_bracketed(got, want, name):
    """A search on the same decisions with another probe sequence."""
    assert got["vefd"] == want["vefd"], name
    assert got["endpoint"] == want["endpoint"], name
    if got["probes"] == 0:  # the bounds alone closed the gap
        assert got["ub"] - got["lb"] <= REL * got["ub"], name
    elif want["threshold_reach"]:
        # the first probe is the stop threshold over VE-FD; reachable there ends the search
        assert got["probes"] == 1, (name, got["probes"])
        assert got["ub"] == want["threshold"] and got["lb"] == want["vefd"], name
        assert got["distance"] == (want["threshold"] + want["vefd"]) / 2.0, name
    else:
        assert got["lb"] >= want["threshold"], name
    fd = want.get("distance")
    if fd is not None:
        assert got["lb"] <= fd * (1 + 2 * REL) and got["ub"] >= fd * (1 - 2 * REL), name
        assert abs(got["distance"] - fd) <= 2 * REL * fd, (name, got["distance"], fd)


@pytest.mark.gpu
def test_long_pair_plain_and_learned(ctx, built):
    want = GOLD["config1/0"]
    P, Q = _pair(built, "config1/0")
    assert (len(P), len(Q)) == (want["n1"], want["n2"])
    _check_plain(ctx.distance(P, Q, precise=True), want, "config1 plain")
    _check_plain(ctx.distance(P, Q, precise=True, precision=built.RFD_PREC_FP32_FILTER), want,
                 "config1 plain fp32 filter")
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(model=model), dict(model=model, coarse_ub=6),
                   dict(model=model, coarse_ub=6, precision=built.RFD_PREC_FP32_FILTER)):
            _check_bracketed(ctx.distance(P, Q, precise=True, **kw), want, f"config1 {kw}")
    finally:
        model.close()
    reach, ub = ctx.decide(P, Q, want["threshold"])
    assert (reach, ub) == (want["threshold_reach"], want["threshold_right_ub"])


def _batch_names():
    return sorted((k for k in GOLD if k.startswith("config2/")), key=lambda s: int(s[8:]))


@pytest.mark.gpu
def test_uneven_batch_sample(ctx, built):
    names = _batch_names()
    assert len(names) >= 256
    pairs = [_pair(built, n) for n in names]
    Ps, Qs = [p for p, _ in pairs], [q for _, q in pairs]
    for kw in (dict(), dict(precision=built.RFD_PREC_FP32_FILTER)):
        res = ctx.distance_batch(Ps, Qs, precise=True, **kw)
        for n, g in zip(names, res):
            _check_plain(g, GOLD[n], f"{n} {kw}")
    model = built.Model.pretrained(0)
    try:
        for kw in (dict(model=model), dict(model=model, precision=built.RFD_PREC_FP32_FILTER),
                   dict(model=model, coarse_ub=6)):
            res = ctx.distance_batch(Ps, Qs, precise=True, **kw)
            for n, g in zip(names, res):
                _check_bracketed(g, GOLD[n], f"{n} {kw}")
    finally:
        model.close()


@pytest.mark.parametrize("name", ["config4/1", "config4/0"])
@pytest.mark.gpu
def test_large_pair_bounds_and_threshold(ctx, built, name):
    want = GOLD[name]
    P, Q = _pair(built, name)
    assert (len(P), len(Q)) == (want["n1"], want["n2"])
    dfd, vefd = ctx.bounds(P, Q, quirks=False)
    assert dfd == want["dfd"] and vefd == want["vefd"], name
    reach, ub = ctx.decide(P, Q, want["threshold"])
    assert (reach, ub) == (want["threshold_reach"], want["threshold_right_ub"]), name
    model = built.Model.pretrained(0)
    try:
        got = ctx.distance(P, Q, precise=True, model=model, coarse_ub=6,
                           precision=built.RFD_PREC_FP32_FILTER)
    finally:
        model.close()
    _check_bracketed(got, want, name)
    assert np.isfinite(got["distance"])
