"""The rule by which a split pair's two halves meet, checked on the CPU.

A lone pair's VE-FD and decisions run as a forward sweep over the lower rows and a mirror sweep
from the far corner over the upper rows (robotfd_b200/csrc/rfd_engine.cu, split_meet_kernel;
rfd_team.cuh, mirror_interval).  The mirror runs the forward propagation unchanged on the
mirrored grid, whose cells carry the entry edges' values - VE-FD weights as they are, free
intervals [lo, hi] as [-hi, -lo] (empty: (-3, -4), dead below -1.5) - and the two rows handed
across the middle boundary combine as
  VE-FD    = min over boundary edges b of max(forward(b), mirror(b)),
  reachable = some b with forward(b) >= 0, mirror(b) >= -1.5 and forward(b) <= -mirror(b).
Here the propagation step of the team kernels is restated cell by cell in Python (the
decision's select form and the VE-FD min-max), and on random grids whose values are drawn from
a few levels (so that ties, empty intervals and whole intervals are common), in both
orientations of the far corner and at every split row, the meet must equal the unsplit sweep.
The GPU tests (test_gpu_split.py) check the kernels themselves against the CPU oracle.
"""
import random

import pytest

FLT_MAX = 3.4028234663852886e38


def sweep_dec(RI, TI, rows, C, left_in, bot0, thr, dv):
    """Rows 0 .. rows-1 of the decision propagation (team_propagator, K_DEC step): returns the
    values handed to row `rows` and the last cell's right- and top-edge results."""
    carry = list(left_in)
    res_r = res_t = None
    for i in range(rows):
        bot = bot0[i]
        out = []
        for j in range(C):
            left = carry[j]
            rLB, rUB = RI[i][j]
            tLB, tUB = TI[i][j]
            bdead, ldead = bot < thr, left < thr
            rinv = left > rUB or ldead
            tinv = bot > tUB or bdead
            ncarry = (dv if rinv else max(rLB, left)) if bdead else rLB
            nbot = (dv if tinv else max(tLB, bot)) if ldead else tLB
            if i == rows - 1 and j == C - 1:
                res_r = (-2.0 if rinv else rUB) if bdead else rUB
                res_t = (-2.0 if tinv else tUB) if ldead else tUB
            out.append(ncarry)
            bot = nbot
        carry = out
    return carry, res_r, res_t


def mirror_interval(iv):
    lo, hi = iv
    return (-3.0, -4.0) if lo < 0.0 else (-hi, -lo)


def interval(levels):
    if random.random() < 0.25:
        return (-1.0, -2.0)  # empty, as free_interval writes it
    a, b = sorted(random.choice(levels) for _ in range(2))
    return (a, b)


def decision_split_equals_whole(R, C, h, tr, levels):
    RI = [[interval(levels) for _ in range(C)] for _ in range(R)]
    TI = [[interval(levels) for _ in range(C)] for _ in range(R)]
    start = [0.0] + [-1.0] * (R - 1)
    _, rr, rt = sweep_dec(RI, TI, R, C, [-1.0] * C, start, 0.0, -1.0)
    whole = (rt if tr else rr) == 1.0
    F, _, _ = sweep_dec(RI, TI, h, C, [-1.0] * C, start[:h], 0.0, -1.0)
    Rm = R - h  # mirror cell (i, j) is cell (R-1-i, C-1-j); its tile: that cell's entry edges
    MR = [[mirror_interval(RI[R - 2 - i][C - 1 - j]) for j in range(C)] for i in range(Rm)]
    MT = [[mirror_interval(TI[R - 1 - i][C - 2 - j]) if C - 1 - j >= 1 else (-3.0, -4.0)
           for j in range(C)] for i in range(Rm)]
    corner = (TI[R - 1][C - 1] if tr else RI[R - 1][C - 1])[1] == 1.0
    left_in = [-1.0 if (j == 0 and not tr and corner) else -3.0 for j in range(C)]
    bot0 = [-1.0 if (i == 0 and tr and corner) else -3.0 for i in range(Rm)]
    M, _, _ = sweep_dec(MR, MT, Rm, C, left_in, bot0, -1.5, -3.0)
    meet = any(F[b] >= 0.0 and M[C - 1 - b] >= -1.5 and F[b] <= -M[C - 1 - b] for b in range(C))
    return whole, meet


def sweep_vefd(WR, WT, rows, C, seed):
    carry = [FLT_MAX] * C
    res = None
    for i in range(rows):
        bot = seed if i == 0 else FLT_MAX
        out = []
        for j in range(C):
            inn = min(carry[j], bot)
            top, right = max(WT[i][j], inn), max(WR[i][j], inn)
            if i == rows - 1 and j == C - 1:
                res = min(top, right)
            out.append(right)
            bot = top
        carry = out
    return carry, res


def vefd_split_equals_whole(R, C, h, levels):
    WR = [[random.choice(levels) for _ in range(C)] for _ in range(R)]
    WT = [[random.choice(levels) for _ in range(C)] for _ in range(R)]
    seed = random.choice(levels)
    _, whole = sweep_vefd(WR, WT, R, C, seed)
    F, _ = sweep_vefd(WR, WT, h, C, seed)
    Rm = R - h
    MWR = [[WR[R - 2 - i][C - 1 - j] for j in range(C)] for i in range(Rm)]
    MWT = [[WT[R - 1 - i][C - 2 - j] if C - 1 - j >= 1 else 0.0 for j in range(C)]
           for i in range(Rm)]
    M, _ = sweep_vefd(MWR, MWT, Rm, C, min(WT[R - 1][C - 1], WR[R - 1][C - 1]))
    return whole, min(max(F[b], M[C - 1 - b]) for b in range(C))


@pytest.mark.parametrize("seed", range(4))
def test_meet_equals_unsplit_sweep(seed):
    random.seed(seed)
    for _ in range(2500):
        R, C = random.randint(2, 7), random.randint(1, 7)
        h = random.randint(1, R - 1)
        levels = random.choice([[0.0, 0.5, 1.0], [0.0, 0.25, 0.5, 0.75, 1.0], [0.0, 1.0],
                                [0.1, 0.3, 0.9, 1.0]])
        whole, meet = decision_split_equals_whole(R, C, h, random.random() < 0.5, levels)
        assert whole == meet, (R, C, h)
        whole, meet = vefd_split_equals_whole(R, C, h, [1.0, 2.0, 3.0, 4.0])
        assert whole == meet, (R, C, h)
