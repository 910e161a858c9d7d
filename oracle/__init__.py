"""CPU oracle for the continuous Frechet distance path (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this package, as the checker or the timed CPU baseline; the product
(``robotfd_b200``) never calls it.  The C source ``rfd_oracle.c`` restates the
reference's DFD, VE-FD and fused-decision cells and its epsilon search (file:line
citations in its header).  Its search driver, endpoint bound and the loaders are pinned by
the reference's own host code run on the same inputs (``tests/golden``); its cells by
mathematical known-answer tests and brute-force definitions (``tests/test_oracle.py``).

``verify.c`` is a separate, formula-independent checker: it decides reachability at a radius
in exact real arithmetic on the given doubles (certified inner and outer free intervals), or
says that it cannot tell (``tests/test_verify.py``).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        i64 = ctypes.c_int64
        L.rfd_oracle_endpoint.restype = ctypes.c_double
        L.rfd_oracle_endpoint.argtypes = [_dp, i64, _dp, i64, ctypes.c_int]
        L.rfd_oracle_dfd_sq.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_int, _dp]
        L.rfd_oracle_vefd_sq.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, _dp]
        L.rfd_oracle_decide.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, _dp]
        L.rfd_oracle_distance.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _dp, _ip, _dp, _ip]
        L.rfd_oracle_decide_formula.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_double,
                                                ctypes.c_int, ctypes.c_int, _dp]
        L.rfd_oracle_distance_formula.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_int, ctypes.c_int, _dp, _ip, _dp, _ip]
        L.rfd_oracle_search.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_int, _dp, _ip]
        L.rfd_oracle_split.argtypes = [ctypes.c_int, _dp, i64, _dp, i64, ctypes.c_int,
                                       ctypes.c_double, i64, _dp]
        L.rfd_oracle_max_threads.restype = ctypes.c_int
        L.rfd_verify_decision.restype = ctypes.c_int
        L.rfd_verify_decision.argtypes = [_dp, i64, _dp, i64, ctypes.c_int, ctypes.c_double]
        L.rfd_verify_free_bounds.argtypes = [_dp, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp]
        L.rfd_oracle_free_intervals.argtypes = [i64, _dp, _dp, _dp, _dp, _dp, ctypes.c_double,
                                                ctypes.c_int, _dp, _dp]
        L.rfd_oracle_free_intervals_formula.argtypes = [i64, _dp, _dp, _dp, _dp, _dp,
                                                        ctypes.c_double, ctypes.c_int,
                                                        ctypes.c_int, _dp, _dp]
        L.rfd_oracle_gen_pair.argtypes = [ctypes.c_int, ctypes.c_int, i64, i64, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_uint64, ctypes.c_uint64, _dp,
                                          ctypes.POINTER(i64), _dp, ctypes.POINTER(i64)]
        L.rfd_oracle_gen_batch_spec.argtypes = [ctypes.c_int, i64, ctypes.c_uint64, _ip,
                                                ctypes.POINTER(i64), ctypes.POINTER(i64), _ip,
                                                _dp, _dp]
        _LIB = L
    return _LIB


def _arr(c):
    a = np.ascontiguousarray(c, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] not in (2, 3):
        raise ValueError("curve must be an (n, 2) or (n, 3) array")
    return a


def _ptr(a):
    return a.ctypes.data_as(_dp)


def max_threads():
    return lib().rfd_oracle_max_threads()


def endpoint(P, Q):
    P, Q = _arr(P), _arr(Q)
    return lib().rfd_oracle_endpoint(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1])


def dfd_sq(P, Q, threads=1):
    P, Q = _arr(P), _arr(Q)
    out = ctypes.c_double()
    rc = lib().rfd_oracle_dfd_sq(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1], threads,
                                 ctypes.byref(out))
    if rc:
        raise RuntimeError(f"oracle dfd failed ({rc})")
    return out.value


def vefd_sq(P, Q, lb, threads=1):
    P, Q = _arr(P), _arr(Q)
    out = ctypes.c_double()
    rc = lib().rfd_oracle_vefd_sq(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1], lb, threads,
                                  ctypes.byref(out))
    if rc:
        raise RuntimeError(f"oracle vefd failed ({rc})")
    return out.value


def decide(P, Q, radius, threads=1, formula=0):
    """Returns (reachable, propagated right UB of the last cell).  formula 0: the reference's
    fused decision kernel's free intervals, 1: its materialised path's (mm - r^2)."""
    P, Q = _arr(P), _arr(Q)
    out = ctypes.c_double()
    rc = lib().rfd_oracle_decide_formula(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1], radius,
                                         formula, threads, ctypes.byref(out))
    if rc:
        raise RuntimeError(f"oracle decide failed ({rc})")
    return out.value == 1.0, out.value


def split(kind, P, Q, x, h):
    """Meet in the middle at row h (see rfd_oracle_split): kind 1 the squared VE-FD seeded
    by x, kind 2 the decision at radius x (1.0 reachable, -2.0 not)."""
    P, Q = _arr(P), _arr(Q)
    out = ctypes.c_double()
    rc = lib().rfd_oracle_split(kind, _ptr(P), len(P), _ptr(Q), len(Q), P.shape[1], x, h,
                                ctypes.byref(out))
    if rc:
        raise RuntimeError(f"oracle split failed ({rc})")
    return out.value


FLT_EPSILON = float(np.finfo(np.float32).eps)
REL_TOL = 2.0 ** -33


def distance(P, Q, stop_mode=0, tol=None, quirks=True, max_probes=200, threads=1, formula=0):
    """Full search.  stop_mode 0 is the reference rule (ub-lb > FLT_EPSILON); formula as in
    decide()."""
    P, Q = _arr(P), _arr(Q)
    if tol is None:
        tol = FLT_EPSILON if stop_mode == 0 else REL_TOL
    out = (ctypes.c_double * 6)()
    probes = ctypes.c_int()
    log_eps = (ctypes.c_double * max(1, max_probes))()
    log_dec = (ctypes.c_int * max(1, max_probes))()
    rc = lib().rfd_oracle_distance_formula(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1],
                                           stop_mode, tol, int(bool(quirks)), max_probes,
                                           threads, formula, out, ctypes.byref(probes), log_eps,
                                           log_dec)
    if rc:
        raise RuntimeError(f"oracle distance failed ({rc})")
    n = probes.value
    return {
        "distance": out[0], "dfd": out[1], "vefd": out[2], "endpoint": out[3],
        "lb": out[4], "ub": out[5], "probes": n,
        "probe_eps": [log_eps[k] for k in range(n)],
        "probe_dec": [bool(log_dec[k]) for k in range(n)],
    }


def search(P, Q, lb, ub, stop_mode=0, tol=None, max_probes=200, threads=1):
    """Bisection from a given bracket; returns (distance, lb, ub, probes)."""
    P, Q = _arr(P), _arr(Q)
    if tol is None:
        tol = FLT_EPSILON if stop_mode == 0 else REL_TOL
    out = (ctypes.c_double * 3)()
    probes = ctypes.c_int()
    rc = lib().rfd_oracle_search(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1], lb, ub, stop_mode,
                                 tol, max_probes, threads, out, ctypes.byref(probes))
    if rc:
        raise RuntimeError(f"oracle search failed ({rc})")
    return out[0], out[1], out[2], probes.value


def free_intervals(x, a, b, A, r2, formula=0):
    """FP64 free intervals of the edges a_e -> b_e around x_e (arrays [n][d]; A [n]); formula
    as in decide()."""
    x, a, b = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, a, b))
    A = np.ascontiguousarray(A, dtype=np.float64)
    inv2A = 0.5 / A
    n, d = x.shape
    lo, hi = np.empty(n), np.empty(n)
    rc = lib().rfd_oracle_free_intervals_formula(n, _ptr(x), _ptr(a), _ptr(b), _ptr(A),
                                                 _ptr(inv2A), float(r2), d, int(formula),
                                                 _ptr(lo), _ptr(hi))
    if rc:
        raise RuntimeError("oracle free_intervals failed")
    return lo, hi


def verify_decision(P, Q, radius):
    """+1 if the free space at `radius` is certainly traversable, -1 if certainly not, 0 if
    the verifier cannot tell (exact real arithmetic on the given doubles)."""
    P, Q = _arr(P), _arr(Q)
    if P.shape[1] != Q.shape[1]:
        raise ValueError("curves differ in dimension")
    return lib().rfd_verify_decision(_ptr(P), len(P), _ptr(Q), len(Q), P.shape[1], float(radius))


def verify_free_bounds(x, s, e, radius):
    """(inner, outer) bounds of the free interval of segment s -> e around x; each a (lo, hi)
    pair, empty when lo > hi."""
    x, s, e = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, s, e))
    out = (ctypes.c_double * 4)()
    lib().rfd_verify_free_bounds(_ptr(x), _ptr(s), _ptr(e), float(radius), len(x), out)
    return (out[0], out[1]), (out[2], out[3])


# ---- seeded workloads (the same generator source as librfd's, compiled into this library,
# so that the CPU baseline makes its inputs without loading the product)
def gen_pair(style, dims, n1, n2, scale, noise, seed, stream=0):
    P = np.empty((n1, dims))
    Q = np.empty((n2, dims))
    m1, m2 = ctypes.c_int64(), ctypes.c_int64()
    rc = lib().rfd_oracle_gen_pair(style, dims, n1, n2, scale, noise, seed, stream, _ptr(P),
                                   ctypes.byref(m1), _ptr(Q), ctypes.byref(m2))
    if rc:
        raise RuntimeError(f"oracle gen_pair failed ({rc})")
    return P[: m1.value].copy(), Q[: m2.value].copy()


def gen_batch_spec(config, npairs, seed):
    dims = np.empty(npairs, np.int32)
    n1 = np.empty(npairs, np.int64)
    n2 = np.empty(npairs, np.int64)
    styles = np.empty(npairs, np.int32)
    scales = np.empty(npairs)
    noises = np.empty(npairs)
    i64p = ctypes.POINTER(ctypes.c_int64)
    rc = lib().rfd_oracle_gen_batch_spec(config, npairs, seed, dims.ctypes.data_as(_ip),
                                         n1.ctypes.data_as(i64p), n2.ctypes.data_as(i64p),
                                         styles.ctypes.data_as(_ip), _ptr(scales), _ptr(noises))
    if rc:
        raise RuntimeError(f"oracle gen_batch_spec failed ({rc})")
    return dims, n1, n2, styles, scales, noises


CONFIG_DEFAULTS = {0: (1, 0), 1: (1, 1), 2: (4096, 2), 3: (200000, 3), 4: (512, 5)}


def gen_config_pair(config, k, seed=None):
    """Pair k of a benchmark workload (see gen_config)."""
    seed = CONFIG_DEFAULTS[config][1] if seed is None else seed
    dims, n1, n2, styles, scales, noises = gen_batch_spec(config, k + 1, seed)
    return gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]), float(scales[k]),
                    float(noises[k]), seed, k)


def gen_config(config, npairs=None, seed=None):
    """Pairs of a benchmark workload: 0 walk 2000x1900 2D (seed 0), 1 spline 200k x 200k 3D
    (seed 1), 2 4096 uneven pairs (seed 2), 3 training pairs (seed 3), 4 512 large 3D pairs
    (seed 5).  Returns a list of (P, Q)."""
    dn, ds = CONFIG_DEFAULTS[config]
    npairs = dn if npairs is None else npairs
    seed = ds if seed is None else seed
    dims, n1, n2, styles, scales, noises = gen_batch_spec(config, npairs, seed)
    return [gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]), float(scales[k]),
                     float(noises[k]), seed, k) for k in range(npairs)]
