"""Inputs of the golden fixtures (shared by the generator and the tests)."""
import numpy as np


def walk_pair(seed, n1, n2, d, noise=0.05):
    rng = np.random.default_rng(seed)
    P = np.cumsum(rng.normal(size=(n1, d)), 0)
    idx = np.linspace(0, n1 - 1, n2)
    base = np.stack([np.interp(idx, np.arange(n1), P[:, k]) for k in range(d)], 1)
    return P, base + rng.normal(scale=noise, size=(n2, d))


CASES = [
    ("parallel_lines", {"points": [[[0, 0], [1, 0], [2, 0]], [[0, 1], [2, 1]]]}),
    ("walk2d_60x45", {"walk": [0, 60, 45, 2]}),
    ("walk3d_70x90", {"walk": [1, 70, 90, 3]}),
    ("walk2d_101x99", {"walk": [8, 101, 99, 2]}),   # 9999 <= 10000: VE-FD skipped
    ("walk2d_101x100", {"walk": [8, 101, 100, 2]}),  # 10100 > 10000: VE-FD runs
    ("walk2d_150x120", {"walk": [5, 150, 120, 2]}),
    ("walk3d_300x280", {"walk": [2, 300, 280, 3]}),
    ("walk2d_700x650", {"walk": [4, 700, 650, 2]}),
    ("config0_2000x1900", {"gen": [0, 2, 2000, 1900, 1.0, 0.05, 0, 0]}),
    ("spline3d_1000x900", {"gen": [1, 3, 1000, 900, 100.0, 0.1, 11, 1000]}),
    ("spline2d_1500x1200", {"gen": [1, 2, 1500, 1200, 100.0, 0.1, 11, 1500]}),
    ("walk3d_gen_600x650", {"gen": [0, 3, 600, 650, 1.0, 0.1, 11, 600]}),
    ("spline3d_big_scale", {"gen": [1, 3, 800, 700, 1.0e4, 0.1, 5, 1]}),
]

# (file, dims, START, LIMIT) for txtLoader2 / txtLoader3
LOADER_CASES = [
    ("dup2.txt", 2, 0, 10000000), ("dup2.txt", 2, 3, 10000000), ("dup2.txt", 2, 0, 4),
    ("dup2.txt", 2, 1, 2), ("dup3.txt", 3, 0, 10000000), ("badtok.txt", 2, 0, 10000000),
    ("mixed2.txt", 2, 0, 10000000), ("mixed2.txt", 3, 0, 10000000), ("walk3.txt", 3, 0, 10000000),
    ("walk3.txt", 3, 10, 25),
]


def build_input(recipe):
    if "points" in recipe:
        P, Q = recipe["points"]
        return np.array(P, float), np.array(Q, float)
    if "walk" in recipe:
        return walk_pair(*recipe["walk"])
    import robotfd_b200 as rfd
    g = recipe["gen"]
    return rfd.gen_pair(g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7])
