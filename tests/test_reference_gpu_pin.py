"""The oracle and the CUDA path against the reference's own GPU kernels.

tests/golden/reference_gpu.json was recorded once on a B200 by
tests/golden/make_reference_gpu_golden.py: the reference's unmodified
src/intersection_algorithm_in_parallel.cu (built for sm_100a from its sources by
oracle/refharness/Makefile) driven by its search driver's steps (src/frechet.cpp:26-63) with
the fused decision kernel (forceOversize), on four seeded pairs (2D and 3D, up to
2000 x 1900 points).  It holds the DFD (Bound_call_gpu's ub), the VE-FD (its lb), every probe
radius with its decision, and the result.

Bars:
  - DFD bit for bit;
  - VE-FD bit for bit in 2D.  In 3D the reference's VE-FD kernel reads an uninitialised
    direction for its top weight (.cu:397), so its 3D VE-FD is not a function of the inputs;
    the engine uses the direction README.md:79 specifies;
  - the decision at every radius the reference probed: the same outcome;
  - the distance bit for bit where the VE-FD agrees, else within the reference's own stop
    width FLT_EPSILON (the bisections start from different lower bounds).
"""
import json
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "reference_gpu.json")
FLT_EPSILON = float(np.finfo(np.float32).eps)


def cases():
    with open(FIXTURE) as f:
        return sorted(json.load(f)["cases"].items())


def _pair(r):
    P, Q = oracle.gen_pair(*r["gen"])
    assert (len(P), len(Q)) == (r["n1"], r["n2"])
    return P, Q


def test_fixture_complete():
    c = dict(cases())
    assert set(c) == {"config0_2000x1900", "spline3d_1500x1400", "walk2d_1200x1100",
                      "spline2d_1800x900"}
    for r in c.values():
        assert r["probes"] == len(r["probe_eps"]) == len(r["probe_dec"]) > 20
        assert r["lb"] <= r["distance"] <= r["ub"] and r["ub"] - r["lb"] <= FLT_EPSILON


@pytest.mark.parametrize("name,r", cases(), ids=[n for n, _ in cases()])
def test_oracle_matches_reference_gpu(built, name, r):
    P, Q = _pair(r)
    t = oracle.max_threads()
    assert oracle.endpoint(P, Q) == r["endpoint"]
    assert np.sqrt(oracle.dfd_sq(P, Q, t)) == r["dfd"]
    got = oracle.distance(P, Q, stop_mode=0, quirks=True, threads=t)
    assert got["dfd"] == r["dfd"]
    if P.shape[1] == 2:
        assert got["vefd"] == r["vefd"]
        assert got["distance"] == r["distance"] and got["probes"] == r["probes"]
    else:
        assert abs(got["distance"] - r["distance"]) <= FLT_EPSILON
    for e, want in zip(r["probe_eps"], r["probe_dec"]):
        assert oracle.decide(P, Q, e, threads=t)[0] == want, e


@pytest.mark.gpu
@pytest.mark.parametrize("name,r", cases(), ids=[n for n, _ in cases()])
def test_engine_matches_reference_gpu(ctx, built, name, r):
    P, Q = _pair(r)
    dfd, vefd = ctx.bounds(P, Q, quirks=True)
    assert dfd == r["dfd"]
    if P.shape[1] == 2:
        assert vefd == r["vefd"]
    for e, want in zip(r["probe_eps"], r["probe_dec"]):
        assert ctx.decide(P, Q, e)[0] == want, e
    got = ctx.distance(P, Q, precise=False)
    assert got["dfd"] == r["dfd"]
    if P.shape[1] == 2:
        assert got["distance"] == r["distance"] and got["probes"] == r["probes"]
    else:
        assert abs(got["distance"] - r["distance"]) <= FLT_EPSILON
    # the stock entry point's mirror, with the fused decision path the reference ran
    fd = built.compute_distance_parallel(P, Q, force_oversize=True)
    if P.shape[1] == 2:
        assert fd == r["distance"]
    else:
        assert abs(fd - r["distance"]) <= FLT_EPSILON
