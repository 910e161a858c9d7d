"""The exact decision verifier (oracle/verify.c), on the CPU.

Its free-interval bounds are checked in exact rational arithmetic (every end point it returns
is tested with Fractions of the same doubles), its decisions against closed-form distances,
and the oracle's FP64 decisions and searches (the reference's formulas) against it: the FP64
decision flips within a few ulps of the exact threshold, and every searched bracket contains
the exact Frechet distance."""
from fractions import Fraction

import numpy as np
import pytest

import oracle

ULP = 2.0 ** -52


def exact_f(x, s, e, t):
    """|s + t (e - s) - x|^2 in rationals."""
    t = Fraction(t)
    return sum((Fraction(a) + t * (Fraction(b) - Fraction(a)) - Fraction(c)) ** 2
               for a, b, c in zip(s, e, x))


def exact_tstar(x, s, e):
    """The exact parameter of the closest point, clamped to [0, 1]."""
    v = [Fraction(b) - Fraction(a) for a, b in zip(s, e)]
    vv = sum(c * c for c in v)
    if vv == 0:
        return Fraction(0)
    t = sum((Fraction(c) - Fraction(a)) * w for a, c, w in zip(s, x, v)) / vv
    return min(max(t, Fraction(0)), Fraction(1))


def check_bounds(x, s, e, r):
    (ilo, ihi), (olo, ohi) = oracle.verify_free_bounds(x, s, e, r)
    r2 = Fraction(r) ** 2
    ts = exact_tstar(x, s, e)
    fmin = exact_f(x, s, e, ts)
    if ilo <= ihi:  # inner: both end points inside (the free set is convex)
        assert 0 <= ilo <= ihi <= 1
        assert exact_f(x, s, e, ilo) <= r2 and exact_f(x, s, e, ihi) <= r2
    if olo > ohi:  # outer empty: the whole segment is outside
        assert fmin > r2
        assert ilo > ihi
        return "empty"
    assert 0 <= olo <= ohi <= 1
    if olo > 0:  # an outside point left of the closest point bounds the free set
        assert exact_f(x, s, e, olo) > r2 and Fraction(olo) < ts
    if ohi < 1:
        assert exact_f(x, s, e, ohi) > r2 and Fraction(ohi) > ts
    if ilo <= ihi:
        assert olo <= ilo and ihi <= ohi
        return "inner"
    return "uncertain"


def test_free_bounds_known_answer():
    # ball of radius sqrt(2) around (0, 1) against y = 0: free t in [0.25, 0.75] of [-2, 2]
    (ilo, ihi), (olo, ohi) = oracle.verify_free_bounds([0, 1], [-2, 0], [2, 0], np.sqrt(2))
    assert olo <= 0.25 <= ilo + 4 * ULP and ihi - 4 * ULP <= 0.75 <= ohi
    assert check_bounds([0, 1], [-2, 0], [2, 0], np.sqrt(2)) == "inner"
    # below the distance to the line: certified empty
    assert check_bounds([0, 1], [-2, 0], [2, 0], 1 - 1e-15) == "empty"
    # exactly tangent: no certainly-inside point, a tight outer interval around 0.5
    (ilo, ihi), (olo, ohi) = oracle.verify_free_bounds([0, 1], [-2, 0], [2, 0], 1.0)
    assert ilo > ihi and olo < 0.5 < ohi and ohi - olo < 1e-6
    # a zero-length segment is a point
    assert check_bounds([0, 0, 0], [1, 1, 1], [1, 1, 1], 2.0) == "inner"
    assert check_bounds([0, 0, 0], [1, 1, 1], [1, 1, 1], 1.7) == "empty"


@pytest.mark.parametrize("d", [2, 3])
def test_free_bounds_exact(d):
    rng = np.random.default_rng(11 + d)
    kinds = set()
    for k in range(400):
        off = 10.0 ** rng.integers(-2, 8) if k % 4 == 0 else 0.0
        x, s, e = (rng.normal(size=d) + off for _ in range(3))
        if k % 5 == 0:
            e = s + rng.normal(size=d) * 1e-9  # short segments
        ts = float(exact_tstar(x, s, e))
        base = float(np.sqrt(float(exact_f(x, s, e, ts))))
        # radii at the closest distance (tangent), just around it, and across the segment
        for r in (base, base * (1 + 4 * ULP), base * (1 - 4 * ULP), base * 1.5,
                  base + float(np.linalg.norm(e - s)) * rng.uniform(0, 1)):
            kinds.add(check_bounds(x, s, e, r))
    assert kinds == {"empty", "inner", "uncertain"}


def test_decision_known_answers():
    # parallel segments one apart: FD 1
    P, Q = np.array([[0.0, 0], [1, 0]]), np.array([[0.0, 1], [1, 1]])
    assert oracle.verify_decision(P, Q, np.nextafter(1.0, 2)) == 1
    assert oracle.verify_decision(P, Q, np.nextafter(1.0, 0)) == -1
    assert oracle.verify_decision(P, Q, 1.0) == 0  # the free space is a single line
    # a backtrack of length 1 along the line: FD 1/2, set by monotonicity, not by an edge
    P = np.array([[0.0, 0], [3, 0]])
    Q = np.array([[0.0, 0], [2, 0], [1, 0], [3, 0]])
    assert oracle.verify_decision(P, Q, 0.5 * (1 + 4 * ULP)) == 1
    assert oracle.verify_decision(P, Q, 0.5 * (1 - 4 * ULP)) == -1
    # a peak of height 1 over a straight curve: FD 1
    P = np.array([[0.0, 0, 0], [2, 0, 0]])
    Q = np.array([[0.0, 0, 0], [1, 1, 0], [2, 0, 0]])
    assert oracle.verify_decision(P, Q, 1 + 4 * ULP) == 1
    assert oracle.verify_decision(P, Q, 1 - 4 * ULP) == -1
    # one-point curves: the largest vertex distance
    P = np.array([[0.0, 0]])
    Q = np.array([[3.0, 4], [1, 0], [0, 2]])
    assert oracle.verify_decision(P, Q, 5 * (1 + 4 * ULP)) == 1
    assert oracle.verify_decision(P, Q, 5 * (1 - 4 * ULP)) == -1
    assert oracle.verify_decision(Q, P, 5 * (1 - 4 * ULP)) == -1
    assert oracle.verify_decision(P, P, 0.0) == 0
    # bad arguments: cannot tell
    assert oracle.verify_decision(P, Q, -1.0) == 0
    assert oracle.verify_decision(P, Q, float("nan")) == 0


def flip(decide, lo, hi):
    """The smallest double in (lo, hi] at which decide() holds (decide(lo) false, hi true)."""
    a, b = lo, hi
    while True:
        m = 0.5 * (a + b)
        if m <= a or m >= b:
            return b
        if decide(m):
            b = m
        else:
            a = m


def random_pairs(seed, count, max_n=60):
    rng = np.random.default_rng(seed)
    for k in range(count):
        n1, n2 = (int(v) for v in rng.integers(2, max_n, 2))
        d = 2 + k % 2
        sc = 10.0 ** rng.integers(-3, 5)
        P = np.cumsum(rng.normal(size=(n1, d)), 0) * sc + 50 * sc
        Q = np.cumsum(rng.normal(size=(n2, d)), 0) * sc + 50 * sc
        yield P, Q


def test_fp64_decision_flips_at_the_exact_threshold():
    """The reference's FP64 decision agrees with the exact one except within a few ulps of
    the Frechet distance."""
    for P, Q in random_pairs(3, 30):
        fd = oracle.distance(P, Q, stop_mode=1)["distance"]
        lo, hi = fd * 0.9, fd * 1.1
        assert oracle.verify_decision(P, Q, lo) == -1 and oracle.verify_decision(P, Q, hi) == 1
        r_hi = flip(lambda r: oracle.verify_decision(P, Q, r) == 1, lo, hi)
        r_lo = flip(lambda r: oracle.verify_decision(P, Q, r) != -1, lo, hi)
        assert r_lo <= r_hi and (r_hi - r_lo) <= 4 * ULP * fd  # the verifier's own band
        f64 = flip(lambda r: oracle.decide(P, Q, r)[0], lo, hi)
        assert r_lo - 4 * ULP * fd <= f64 <= r_hi + 4 * ULP * fd
        for f in (0.99, 1 - 1e-9, 1 + 1e-9, 1.01):
            assert (oracle.verify_decision(P, Q, fd * f) == 1) == oracle.decide(P, Q, fd * f)[0]


@pytest.mark.parametrize("stop_mode", [0, 1])
def test_searched_bracket_contains_the_exact_distance(built, stop_mode):
    pairs = list(random_pairs(5, 12)) + [built.gen_pair(k % 2, 2 + k % 2, 40 + 30 * k,
                                                        70 + 20 * k, 1.0, 0.05, 31, k)
                                         for k in range(6)]
    for P, Q in pairs:
        res = oracle.distance(P, Q, stop_mode=stop_mode)
        lb, ub = res["lb"], res["ub"]
        assert oracle.verify_decision(P, Q, ub * (1 + 8 * ULP)) == 1
        assert oracle.verify_decision(P, Q, lb * (1 - 8 * ULP)) == -1
