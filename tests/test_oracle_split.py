"""Meet in the middle on real geometry, in the CPU oracle.

oracle.split restates the CUDA engine's split pairs (robotfd_b200/csrc: split_meet_kernel and
the mirror instantiation of the team strips) with the oracle's own cell functions: the rows
below a boundary swept from the start, the rows above it swept from the far corner on the
mirrored grid (entry edges' values, free intervals negated), the two rows handed across the
boundary combined by exact min/max (VE-FD) or comparisons (decision).  On seeded pairs of
both generator styles, 2D and 3D, with the first curve the shorter or the longer, at every
kind of boundary row (the first, the last, strip multiples, odd rows) and at radii around the
distance, the split must give the unsplit oracle's squared VE-FD bit for bit and its
decision.  Also: identical curves (distance 0 up to rounding), a repeated point (a
zero-length segment, whose interval the reference clamps to [0, 1]) and parallel lines.
"""
import numpy as np
import pytest

import oracle

K_VEFD, K_DEC = 1, 2


def _check_pair(P, Q, rows):
    R = len(P) - 1
    lb = oracle.endpoint(P, Q)
    ve = oracle.vefd_sq(P, Q, lb)
    r = oracle.distance(P, Q, stop_mode=1, quirks=False)
    fd = r["distance"]
    radii = [fd, fd * (1 - 1e-12), fd * (1 + 1e-12), fd * 0.97, fd * 1.03, np.sqrt(ve), lb,
             r["ub"], r["lb"]]
    for h in rows:
        if not 1 <= h <= R - 1:
            continue
        assert oracle.split(K_VEFD, P, Q, lb, h) == ve, (len(P), len(Q), h)
        for e in radii:
            want = oracle.decide(P, Q, e)[0]
            got = oracle.split(K_DEC, P, Q, e, h) == 1.0
            assert got == want, (len(P), len(Q), h, e)


@pytest.mark.parametrize("style,d,n1,n2,seed", [
    (0, 2, 120, 97, 1), (0, 2, 97, 120, 2), (1, 3, 150, 140, 3), (1, 2, 200, 65, 4),
    (0, 3, 70, 260, 5), (1, 3, 33, 400, 6), (0, 2, 300, 300, 7)])
def test_split_equals_unsplit_on_generated_pairs(style, d, n1, n2, seed):
    P, Q = oracle.gen_pair(style, d, n1, n2, 100.0 if style else 1.0, 0.1, seed, 0)
    R = len(P) - 1
    _check_pair(P, Q, [1, 2, R // 2, R // 2 + 1, 32, 64, R - 32, R - 2, R - 1])


def test_split_on_degenerate_geometry():
    t = np.linspace(0.0, 1.0, 90)
    A = np.stack([t, np.sin(5 * t)], 1)
    B = A.copy()
    B[40] = B[39]  # a repeated point
    cases = [(A, A.copy()), (B, A[::2].copy()), (np.stack([t, 0 * t], 1), np.stack([t, 0 * t + 0.3], 1))]
    for P, Q in cases:
        R = len(P) - 1
        _check_pair(P, Q, [1, R // 3, R // 2, R - 1])
