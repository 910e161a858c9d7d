"""B200-native continuous Frechet distance engine (Python binding of librfd.so).

The product is the C ABI in ``include/rfd.h`` implemented by ``librfd.so`` (CUDA kernels
for sm_100a plus a C++ drop-in of the reference's ``compute_distance_parallel`` /
``Curve`` / ``txtLoaderX`` API).  This module binds it with ctypes.  There is no CPU
fallback: every distance, bound and decision runs the CUDA kernels, and a missing
library or device raises.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_CSRC = os.path.join(_HERE, "csrc")
LIB_PATH = os.path.join(_HERE, "librfd.so")
FD_PATH = os.path.join(_HERE, "fd")

RFD_OK = 0
RFD_ERR_ARG = 1
RFD_ERR_CUDA = 2
RFD_ERR_NOMEM = 3
RFD_ERR_TIMEOUT = 4
RFD_ERR_NODEV = 5
RFD_ERR_INTERNAL = 6
RFD_ERR_LIMIT = 7

RFD_STOP_ABS = 0
RFD_STOP_REL = 1
RFD_MEM_HOST = 0
RFD_MEM_DEVICE = 1
RFD_PREC_FP64 = 0
RFD_PREC_FP32_FILTER = 1
RFD_FORMULA_FUSED = 0
RFD_FORMULA_MATERIALISED = 1
RFD_FORMULA_REFERENCE = 2

FLAG_VEFD_SKIPPED = 1
FLAG_LB_GT_UB = 2
FLAG_MAX_PROBES = 4
FLAG_STALLED = 8
FLAG_VEFD_DENSE = 16
FLAG_BRACKET_USED = 32
FLAG_BRACKET_WIDENED = 64
FLAG_DEGENERATE = 128
FLAG_DFD_COARSE = 256

FLT_EPSILON = float(np.finfo(np.float32).eps)
REL_TOL = 2.0 ** -33

# Every symbol include/rfd.h declares.
EXPORTS = (
    "rfd_abi_version", "rfd_status_string", "rfd_last_error", "rfd_options_init",
    "rfd_context_create", "rfd_context_destroy", "rfd_context_set_stream",
    "rfd_context_set_wait_budget",
    "rfd_context_phase_times", "rfd_fp64_peak", "rfd_distance",
    "rfd_distance_batch", "rfd_bounds", "rfd_decide", "rfd_decide_formula", "rfd_load_txt",
    "rfd_free",
    "rfd_gen_pair", "rfd_gen_batch_spec", "rfd_search_step", "rfd_decide_noalloc",
    "rfd_model_num_params", "rfd_model_create", "rfd_model_destroy", "rfd_model_set_params",
    "rfd_model_get_params", "rfd_model_forward", "rfd_model_gradients", "rfd_model_train_step",
    "rfd_features", "rfd_gemm_bf16", "rfd_interval_class", "rfd_distance_matrix",
    "rfd_load_txt_fast", "rfd_save_bin", "rfd_load_bin", "rfd_autotune", "rfd_autotune_search",
)


class RfdError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"rfd status {code} ({_status_name(code)}): {msg}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [
        ("stop_mode", ctypes.c_int32),
        ("reference_quirks", ctypes.c_int32),
        ("tol", ctypes.c_double),
        ("max_probes", ctypes.c_int32),
        ("dense", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("memory", ctypes.c_int32),
        ("bracket", ctypes.POINTER(ctypes.c_double)),
        ("model", ctypes.c_void_p),
        ("coarse_ub", ctypes.c_int32),
        ("drop_repeats", ctypes.c_int32),
        ("graph", ctypes.c_int32),
        ("formula", ctypes.c_int32),
        ("search_arity", ctypes.c_int32),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("distance", ctypes.c_double),
        ("dfd", ctypes.c_double),
        ("vefd", ctypes.c_double),
        ("endpoint", ctypes.c_double),
        ("lb", ctypes.c_double),
        ("ub", ctypes.c_double),
        ("cells_nominal", ctypes.c_int64),
        ("cells_evaluated", ctypes.c_int64),
        ("cells_fp64", ctypes.c_int64),
        ("cells_vefd", ctypes.c_int64),
        ("probes", ctypes.c_int32),
        ("flags", ctypes.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_LIB = None
_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)


def build(jobs=8):
    """Compile librfd.so and the fd CLI in-tree for sm_100a (nvcc cross-compiles)."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", _CSRC], check=True)


def lib():
    """Loads librfd.so; raises when it has not been built (no fallback path exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RfdError(RFD_ERR_NODEV, f"{LIB_PATH} is missing: run robotfd_b200.build()")
    L = ctypes.CDLL(LIB_PATH)
    i32, i64, dbl, vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
    L.rfd_abi_version.restype = i32
    L.rfd_status_string.restype = ctypes.c_char_p
    L.rfd_status_string.argtypes = [i32]
    L.rfd_last_error.restype = ctypes.c_char_p
    L.rfd_options_init.argtypes = [ctypes.POINTER(Options), i32]
    L.rfd_options_init.restype = None
    L.rfd_context_create.argtypes = [i32, ctypes.POINTER(vp)]
    L.rfd_context_create.restype = i32
    L.rfd_context_destroy.argtypes = [vp]
    L.rfd_context_destroy.restype = i32
    L.rfd_context_set_stream.argtypes = [vp, vp]
    L.rfd_context_set_stream.restype = i32
    L.rfd_context_set_wait_budget.argtypes = [vp, ctypes.c_int64]
    L.rfd_context_set_wait_budget.restype = i32
    L.rfd_context_phase_times.argtypes = [vp, i32, _dp]
    L.rfd_context_phase_times.restype = i32
    L.rfd_fp64_peak.argtypes = [vp, _dp]
    L.rfd_fp64_peak.restype = i32
    L.rfd_distance.argtypes = [vp, vp, i64, vp, i64, i32, ctypes.POINTER(Options),
                               ctypes.POINTER(Result)]
    L.rfd_distance.restype = i32
    L.rfd_distance_batch.argtypes = [vp, i64, ctypes.POINTER(vp), _i64p, ctypes.POINTER(vp), _i64p,
                                     _i32p, ctypes.POINTER(Options), ctypes.POINTER(Result)]
    L.rfd_distance_batch.restype = i32
    L.rfd_bounds.argtypes = [vp, vp, i64, vp, i64, i32, i32, i32, _dp, _dp]
    L.rfd_bounds.restype = i32
    L.rfd_decide.argtypes = [vp, vp, i64, vp, i64, i32, dbl, i32, _i32p, _dp]
    L.rfd_decide.restype = i32
    L.rfd_decide_formula.argtypes = [vp, vp, i64, vp, i64, i32, dbl, i32, i32, _i32p, _dp]
    L.rfd_decide_formula.restype = i32
    L.rfd_load_txt.argtypes = [ctypes.c_char_p, i32, i32, i32, ctypes.POINTER(_dp), _i64p]
    L.rfd_load_txt.restype = i32
    L.rfd_load_txt_fast.argtypes = [ctypes.c_char_p, i32, i32, i32, i32, ctypes.POINTER(_dp), _i64p]
    L.rfd_load_txt_fast.restype = i32
    L.rfd_save_bin.argtypes = [ctypes.c_char_p, _dp, i64, i32]
    L.rfd_save_bin.restype = i32
    L.rfd_load_bin.argtypes = [ctypes.c_char_p, ctypes.POINTER(_dp), _i64p, _i32p]
    L.rfd_load_bin.restype = i32
    L.rfd_free.argtypes = [vp]
    L.rfd_free.restype = None
    L.rfd_gen_pair.argtypes = [i32, i32, i64, i64, dbl, dbl, ctypes.c_uint64, ctypes.c_uint64,
                               _dp, _i64p, _dp, _i64p]
    L.rfd_gen_pair.restype = i32
    L.rfd_gen_batch_spec.argtypes = [i32, i64, ctypes.c_uint64, _i32p, _i64p, _i64p, _i32p, _dp, _dp]
    L.rfd_gen_batch_spec.restype = i32
    L.rfd_search_step.argtypes = [_dp, _i32p, i32, i32, dbl, i32, _dp]
    L.rfd_search_step.restype = i32
    L.rfd_interval_class.argtypes = [i64, _dp, _dp, _dp, _dp, dbl, i32, _i32p]
    L.rfd_interval_class.restype = i32
    L.rfd_distance_matrix.argtypes = [vp, i64, vp, _i64p, _i32p, vp, dbl, _dp, vp]
    L.rfd_distance_matrix.restype = i32
    L.rfd_autotune.argtypes = [vp, i64, vp, _i64p, vp, _i64p, _i32p, vp, i32, _dp, _i32p]
    L.rfd_autotune.restype = i32
    L.rfd_autotune_search.argtypes = [vp, i64, vp, _i64p, vp, _i64p, _i32p, vp, i32, _dp, _i32p]
    L.rfd_autotune_search.restype = i32
    L.rfd_decide_noalloc.argtypes = [vp, i64, vp, i64, i32, dbl, vp, vp]
    L.rfd_decide_noalloc.restype = i32
    fp = ctypes.POINTER(ctypes.c_float)
    L.rfd_model_num_params.restype = i64
    L.rfd_model_create.argtypes = [i32, ctypes.c_uint64, ctypes.POINTER(vp)]
    L.rfd_model_create.restype = i32
    L.rfd_model_destroy.argtypes = [vp]
    L.rfd_model_destroy.restype = i32
    L.rfd_model_set_params.argtypes = [vp, fp, i64]
    L.rfd_model_set_params.restype = i32
    L.rfd_model_get_params.argtypes = [vp, fp, i64]
    L.rfd_model_get_params.restype = i32
    L.rfd_model_forward.argtypes = [vp, vp, i64, vp]
    L.rfd_model_forward.restype = i32
    L.rfd_model_gradients.argtypes = [vp, vp, vp, i64, fp, fp]
    L.rfd_model_gradients.restype = i32
    L.rfd_model_train_step.argtypes = [vp, vp, vp, i64, ctypes.c_float, fp]
    L.rfd_model_train_step.restype = i32
    L.rfd_features.argtypes = [vp, i64, ctypes.POINTER(vp), _i64p, ctypes.POINTER(vp), _i64p, _i32p,
                               _dp, _dp, fp]
    L.rfd_features.restype = i32
    L.rfd_gemm_bf16.argtypes = [i32, i32, i32, vp, i64, i64, vp, i64, i64, vp]
    L.rfd_gemm_bf16.restype = i32
    _LIB = L
    return L


def _status_name(code):
    try:
        return lib().rfd_status_string(code).decode()
    except Exception:  # library not loadable: plain code
        return str(code)


def _check(code):
    if code != RFD_OK:
        raise RfdError(code, lib().rfd_last_error().decode())


def _curve(c):
    if (type(c) is np.ndarray and c.dtype == np.float64 and c.ndim == 2 and c.flags.c_contiguous
            and c.shape[1] in (2, 3) and c.shape[0] >= 1):
        return c  # already in the C ABI's layout
    a = np.ascontiguousarray(c, dtype=np.float64)
    if a.ndim != 2 or a.shape[1] not in (2, 3) or a.shape[0] < 1:
        raise ValueError("a curve is a non-empty (n, 2) or (n, 3) array")
    return a


def options(precise=False, dense=False, max_probes=64, tol=None, quirks=None, memory=RFD_MEM_HOST,
            precision=RFD_PREC_FP64, model=None, coarse_ub=0, drop_repeats=False, graph=False,
            formula=0, search_arity=0):
    o = Options()
    lib().rfd_options_init(ctypes.byref(o), 1 if precise else 0)
    o.dense = int(bool(dense))
    o.max_probes = int(max_probes)
    o.memory = memory
    o.precision = precision
    if tol is not None:
        o.tol = float(tol)
    if quirks is not None:
        o.reference_quirks = int(bool(quirks))
    if model is not None:
        o.model = model._h.value
    o.coarse_ub = int(coarse_ub)
    o.drop_repeats = int(bool(drop_repeats))
    o.graph = int(bool(graph))
    o.formula = int(formula)
    o.search_arity = int(search_arity)
    return o


class Context:
    """One CUDA device, one stream, a cached device workspace (rfd_context)."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        _check(lib().rfd_context_create(int(device), ctypes.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib().rfd_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        _check(lib().rfd_context_set_stream(self._h, ctypes.c_void_p(stream_handle)))

    def set_wait_budget(self, cycles=0):
        """Budget of every bounded wait in SM clock cycles (<= 0: the default, about 20 s)."""
        _check(lib().rfd_context_set_wait_budget(self._h, int(cycles)))

    def phase_times(self, enable=-1):
        """Per-phase device ms since the last query: dict(dfd, vefd, search, calls, launches)."""
        out = (ctypes.c_double * 7)()
        _check(lib().rfd_context_phase_times(self._h, int(enable), out))
        return dict(zip(("dfd_ms", "vefd_ms", "search_ms", "calls", "launches", "h2d_bytes",
                         "d2h_bytes"), list(out)))

    def features(self, Ps, Qs, endpoint, vefd):
        """Bracket features [npairs][400] (float32) of host curves (rfd_features)."""
        n = len(Ps)
        keep = [_curve(x) for x in Ps] + [_curve(x) for x in Qs]
        A, B = keep[:n], keep[n:]
        p1 = (ctypes.c_void_p * n)(*[a.ctypes.data for a in A])
        p2 = (ctypes.c_void_p * n)(*[b.ctypes.data for b in B])
        n1 = (ctypes.c_int64 * n)(*[len(a) for a in A])
        n2 = (ctypes.c_int64 * n)(*[len(b) for b in B])
        dm = (ctypes.c_int32 * n)(*[a.shape[1] for a in A])
        ep = np.ascontiguousarray(endpoint, dtype=np.float64)
        ve = np.ascontiguousarray(vefd, dtype=np.float64)
        out = np.zeros((n, FEATURE_WIDTH), dtype=np.float32)
        _check(lib().rfd_features(self._h, n, p1, n1, p2, n2, dm, ep.ctypes.data_as(_dp),
                                  ve.ctypes.data_as(_dp),
                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def fp64_peak(self):
        """Measured FP64 FMA throughput in TFLOP/s."""
        out = ctypes.c_double()
        _check(lib().rfd_fp64_peak(self._h, ctypes.byref(out)))
        return out.value

    def distance_device(self, p_ptr, n1, q_ptr, n2, dims, **kw):
        """Single pair whose curves already live in device memory (raw pointers)."""
        o = options(memory=RFD_MEM_DEVICE, **kw)
        r = Result()
        _check(lib().rfd_distance(self._h, ctypes.c_void_p(p_ptr), int(n1), ctypes.c_void_p(q_ptr),
                                  int(n2), int(dims), ctypes.byref(o), ctypes.byref(r)))
        return r.as_dict()

    # ---- single pair
    def distance(self, P, Q, **kw):
        P, Q = _curve(P), _curve(Q)
        if P.shape[1] != Q.shape[1]:
            raise ValueError("curves differ in dimension")
        o = options(**kw)
        r = Result()
        _check(lib().rfd_distance(self._h, P.ctypes.data, len(P), Q.ctypes.data, len(Q), P.shape[1],
                                  ctypes.byref(o), ctypes.byref(r)))
        return r.as_dict()

    def bounds(self, P, Q, quirks=True, dense=False):
        P, Q = _curve(P), _curve(Q)
        dfd = ctypes.c_double()
        vefd = ctypes.c_double(_endpoint_host(P, Q))
        _check(lib().rfd_bounds(self._h, P.ctypes.data, len(P), Q.ctypes.data, len(Q), P.shape[1],
                                int(bool(quirks)), int(bool(dense)), ctypes.byref(dfd),
                                ctypes.byref(vefd)))
        return dfd.value, vefd.value

    def decide(self, P, Q, radius, dense=False, formula=RFD_FORMULA_FUSED):
        P, Q = _curve(P), _curve(Q)
        reach = ctypes.c_int32()
        rub = ctypes.c_double()
        _check(lib().rfd_decide_formula(self._h, P.ctypes.data, len(P), Q.ctypes.data, len(Q),
                                        P.shape[1], float(radius), int(bool(dense)), int(formula),
                                        ctypes.byref(reach), ctypes.byref(rub)))
        return bool(reach.value), rub.value

    # ---- batch
    def autotune(self, Ps, Qs, reps=2, **kw):
        """Times the DFD sweep's tile shapes (rows per lane 1, 2, 4, 8; stacked or skewed rows)
        on these pairs and keeps the fastest in the context (rfd_autotune).  Returns
        {"rows": r, "skew": s, "ms": {(rows, skew): ms per sweep}}."""
        n = len(Ps)
        if n != len(Qs) or n == 0:
            raise ValueError("Ps and Qs: non-empty, same length")
        A = [_curve(p) for p in Ps]
        B = [_curve(q) for q in Qs]
        p1 = (ctypes.c_void_p * n)(*[a.ctypes.data for a in A])
        p2 = (ctypes.c_void_p * n)(*[b.ctypes.data for b in B])
        n1 = np.array([len(a) for a in A], dtype=np.int64)
        n2 = np.array([len(b) for b in B], dtype=np.int64)
        dm = np.array([a.shape[1] for a in A], dtype=np.int32)
        o = options(**kw)
        ms = np.zeros(8)
        best = np.zeros(2, dtype=np.int32)
        _check(lib().rfd_autotune(self._h, n, p1, n1.ctypes.data_as(_i64p), p2,
                                  n2.ctypes.data_as(_i64p), dm.ctypes.data_as(_i32p),
                                  ctypes.byref(o), int(reps), ms.ctypes.data_as(_dp),
                                  best.ctypes.data_as(_i32p)))
        return {"rows": int(best[0]), "skew": int(best[1]),
                "ms": {(r, k): float(ms[i * 2 + k]) for i, r in enumerate((1, 2, 4, 8))
                       for k in (0, 1)}}

    def autotune_search(self, Ps, Qs, reps=1, **kw):
        """Times the team strips' shape (4 or 8 warps) and the search's split (switch point,
        start window) on whole solves of these pairs with these options, and keeps the fastest
        in the context (rfd_autotune_search).  Returns {"warps", "switch", "window", "ms":
        {(warps, switch index, window): ms per solve}}."""
        n = len(Ps)
        if n != len(Qs) or n == 0:
            raise ValueError("Ps and Qs: non-empty, same length")
        A = [_curve(p) for p in Ps]
        B = [_curve(q) for q in Qs]
        p1 = (ctypes.c_void_p * n)(*[a.ctypes.data for a in A])
        p2 = (ctypes.c_void_p * n)(*[b.ctypes.data for b in B])
        n1 = np.array([len(a) for a in A], dtype=np.int64)
        n2 = np.array([len(b) for b in B], dtype=np.int64)
        dm = np.array([a.shape[1] for a in A], dtype=np.int32)
        o = options(**kw)
        ms = np.zeros(18)
        best = np.zeros(3, dtype=np.int32)
        _check(lib().rfd_autotune_search(self._h, n, p1, n1.ctypes.data_as(_i64p), p2,
                                         n2.ctypes.data_as(_i64p), dm.ctypes.data_as(_i32p),
                                         ctypes.byref(o), int(reps), ms.ctypes.data_as(_dp),
                                         best.ctypes.data_as(_i32p)))
        return {"warps": int(best[0]), "switch": int(best[1]), "window": int(best[2]),
                "ms": {(w, si, win): float(ms[(wi * 3 + si) * 3 + ni])
                       for wi, w in enumerate((4, 8)) for si in range(3)
                       for ni, win in enumerate((1, 2, 4))}}

    def distance_matrix(self, curves, budget_bytes=0.0, with_results=False, **kw):
        """All pairwise distances (rfd_distance_matrix): an (n, n) array, symmetric, zero
        diagonal; with with_results also the list of pair results (i < j, row-major)."""
        return _matrix(self, curves, budget_bytes, with_results, **kw)

    def distance_batch(self, Ps, Qs, brackets=None, **kw):
        """Ps, Qs: sequences of host arrays, or (with memory=RFD_MEM_DEVICE) of
        (device_pointer, n, dims) tuples."""
        n = len(Ps)
        if n != len(Qs):
            raise ValueError("Ps and Qs differ in length")
        o = options(**kw)
        keep = []
        p1 = (ctypes.c_void_p * n)()
        p2 = (ctypes.c_void_p * n)()
        n1 = (ctypes.c_int64 * n)()
        n2 = (ctypes.c_int64 * n)()
        dm = (ctypes.c_int32 * n)()
        for k in range(n):
            if o.memory == RFD_MEM_DEVICE:
                (a, la, da), (b, lb_, db) = Ps[k], Qs[k]
                p1[k], p2[k], n1[k], n2[k], dm[k] = a, b, la, lb_, da
            else:
                A, B = _curve(Ps[k]), _curve(Qs[k])
                keep += [A, B]
                p1[k], p2[k], n1[k], n2[k], dm[k] = A.ctypes.data, B.ctypes.data, len(A), len(B), A.shape[1]
        if brackets is not None:
            br = np.ascontiguousarray(brackets, dtype=np.float64).reshape(n, 2)
            keep.append(br)
            o.bracket = br.ctypes.data_as(_dp)
        res = (Result * n)()
        _check(lib().rfd_distance_batch(self._h, n, p1, n1, p2, n2, dm, ctypes.byref(o), res))
        return [r.as_dict() for r in res]


def _matrix(ctx, curves, budget_bytes=0.0, with_results=False, **kw):
    cs = [_curve(c) for c in curves]
    n = len(cs)
    ptrs = (ctypes.c_void_p * n)(*[c.ctypes.data for c in cs])
    ns = (ctypes.c_int64 * n)(*[len(c) for c in cs])
    dm = (ctypes.c_int32 * n)(*[c.shape[1] for c in cs])
    o = options(**kw)
    out = np.empty((n, n))
    res = (Result * (n * (n - 1) // 2))() if with_results else None
    _check(lib().rfd_distance_matrix(ctx._h, n, ptrs, ns, dm, ctypes.byref(o), float(budget_bytes),
                                     out.ctypes.data_as(_dp), res))
    return (out, [r.as_dict() for r in res]) if with_results else out


def _endpoint_host(P, Q):
    a = float(np.sum((P[0] - Q[0]) ** 2))
    b = float(np.sum((P[-1] - Q[-1]) ** 2))
    return float(np.sqrt(max(a, b)))


_DEFAULT_CTX = None


def default_context():
    global _DEFAULT_CTX
    if _DEFAULT_CTX is None:
        _DEFAULT_CTX = Context(0)
    return _DEFAULT_CTX


def compute_distance_parallel(curve1, curve2, force_oversize=False):
    """Mirror of the reference's compute_distance_parallel (include/wrapper.hpp:4): stop rule
    ub - lb <= FLT_EPSILON, VE-FD launch rule of the reference, result (lb + ub) / 2, and the
    reference's choice of decision path: the fused kernel's free intervals when forced, else by
    free device memory (RFD_FORMULA_REFERENCE)."""
    formula = RFD_FORMULA_FUSED if force_oversize else RFD_FORMULA_REFERENCE
    return default_context().distance(curve1, curve2, formula=formula)["distance"]


def _load(path, dims, start, limit, threads=None):
    out = _dp()
    n = ctypes.c_int64()
    if threads is None:
        _check(lib().rfd_load_txt(str(path).encode(), dims, int(start), int(limit),
                                  ctypes.byref(out), ctypes.byref(n)))
    else:
        _check(lib().rfd_load_txt_fast(str(path).encode(), dims, int(start), int(limit),
                                       int(threads), ctypes.byref(out), ctypes.byref(n)))
    try:
        arr = np.ctypeslib.as_array(out, shape=(n.value * dims,)).copy() if n.value else np.zeros(0)
    finally:
        lib().rfd_free(out)
    return arr.reshape(n.value, dims)


def txt_loader2(path, start=0, limit=10000000):
    """txtLoader2 (include/txtReader.hpp:6 of the reference) as an (n, 2) array."""
    return _load(path, 2, start, limit)


def txt_loader3(path, start=0, limit=10000000):
    """txtLoader3 (include/txtReader.hpp:48 of the reference) as an (n, 3) array."""
    return _load(path, 3, start, limit)


def txt_loader_fast(path, dims, start=0, limit=10000000, threads=0):
    """rfd_load_txt_fast: the loaders' rules with the parsing on `threads` host threads
    (0: all cores)."""
    return _load(path, dims, start, limit, threads)


def save_bin(path, pts):
    """Writes a curve as a binary trajectory file (rfd_save_bin)."""
    a = np.ascontiguousarray(pts, dtype=np.float64)
    if a.ndim != 2:
        raise ValueError("a curve is an (n, dims) array")
    _check(lib().rfd_save_bin(str(path).encode(), a.ctypes.data_as(_dp), a.shape[0], a.shape[1]))


def load_bin(path):
    """Reads a binary trajectory file (rfd_load_bin) as an (n, dims) array."""
    out = _dp()
    n = ctypes.c_int64()
    d = ctypes.c_int32()
    _check(lib().rfd_load_bin(str(path).encode(), ctypes.byref(out), ctypes.byref(n), ctypes.byref(d)))
    try:
        arr = np.ctypeslib.as_array(out, shape=(n.value * d.value,)).copy() if n.value else np.zeros(0)
    finally:
        lib().rfd_free(out)
    return arr.reshape(n.value, d.value)


# ---- synthetic workloads
def gen_pair(style, dims, n1, n2, scale, noise, seed, stream=0):
    P = np.empty((n1, dims))
    Q = np.empty((n2, dims))
    m1, m2 = ctypes.c_int64(), ctypes.c_int64()
    _check(lib().rfd_gen_pair(style, dims, n1, n2, scale, noise, seed, stream,
                              P.ctypes.data_as(_dp), ctypes.byref(m1), Q.ctypes.data_as(_dp),
                              ctypes.byref(m2)))
    return P[: m1.value].copy(), Q[: m2.value].copy()


def gen_batch_spec(config, npairs, seed):
    dims = np.empty(npairs, np.int32)
    n1 = np.empty(npairs, np.int64)
    n2 = np.empty(npairs, np.int64)
    styles = np.empty(npairs, np.int32)
    scales = np.empty(npairs)
    noises = np.empty(npairs)
    _check(lib().rfd_gen_batch_spec(config, npairs, seed, dims.ctypes.data_as(_i32p),
                                    n1.ctypes.data_as(_i64p), n2.ctypes.data_as(_i64p),
                                    styles.ctypes.data_as(_i32p), scales.ctypes.data_as(_dp),
                                    noises.ctypes.data_as(_dp)))
    return dims, n1, n2, styles, scales, noises


def gen_config(config, npairs=None, seed=None):
    """Pairs of a benchmark workload: 0 walk 2000x1900 2D (seed 0), 1 spline 200k x 200k 3D
    (seed 1), 2 4096 uneven pairs (seed 2), 3 training pairs (seed 3), 4 512 large 3D pairs
    (seed 5).  Returns a list of (P, Q)."""
    defaults = {0: (1, 0), 1: (1, 1), 2: (4096, 2), 3: (200000, 3), 4: (512, 5)}
    dn, ds = defaults[config]
    npairs = dn if npairs is None else npairs
    seed = ds if seed is None else seed
    dims, n1, n2, styles, scales, noises = gen_batch_spec(config, npairs, seed)
    return [gen_pair(int(styles[k]), int(dims[k]), int(n1[k]), int(n2[k]), float(scales[k]),
                     float(noises[k]), seed, k) for k in range(npairs)]


def search_step(state, istate, stop_mode, have_outcome, eps, reachable):
    """Host copy of the device search state machine (for tests)."""
    st = (ctypes.c_double * 6)(*state)
    ist = (ctypes.c_int32 * 4)(*istate)
    nxt = ctypes.c_double()
    more = lib().rfd_search_step(st, ist, stop_mode, int(bool(have_outcome)), float(eps),
                                 int(bool(reachable)), ctypes.byref(nxt))
    return bool(more), nxt.value, list(st), list(ist)


def interval_class(x, a, b, A, r2):
    """Host copy of the FP32 filter: per edge a_e -> b_e around x_e, 1 = certainly empty,
    2 = certainly (0, 1), 0 = computed in FP64 (rfd_interval_class)."""
    x, a, b = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, a, b))
    A = np.ascontiguousarray(A, dtype=np.float64)
    n, d = x.shape
    cls = np.empty(n, dtype=np.int32)
    _check(lib().rfd_interval_class(n, x.ctypes.data_as(_dp), a.ctypes.data_as(_dp),
                                    b.ctypes.data_as(_dp), A.ctypes.data_as(_dp), float(r2), d,
                                    cls.ctypes.data_as(_i32p)))
    return cls


def decide_noalloc(p_dev, n1, q_dev, n2, dims, radius, stream, out_dev):
    """rfd_decide_noalloc on device pointers: enqueues one decision on `stream` and writes
    the propagated right UB of the last cell to out_dev (one double, device memory)."""
    _check(lib().rfd_decide_noalloc(ctypes.c_void_p(p_dev), int(n1), ctypes.c_void_p(q_dev),
                                    int(n2), int(dims), float(radius), ctypes.c_void_p(stream),
                                    ctypes.c_void_p(out_dev)))


FEATURE_WIDTH = 400
N_FEATURES = 386
_fp = ctypes.POINTER(ctypes.c_float)


class Model:
    """The learned-bracket network (rfd_model): BF16 MLP 400-256-256-256-2 on one GPU."""

    def __init__(self, device=0, seed=0, params=None):
        h = ctypes.c_void_p()
        _check(lib().rfd_model_create(int(device), ctypes.c_uint64(seed), ctypes.byref(h)))
        self._h = h
        self.device = device
        if params is not None:
            self.set_params(params)

    @staticmethod
    def num_params():
        return int(lib().rfd_model_num_params())

    def close(self):
        if self._h:
            lib().rfd_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32)
        _check(lib().rfd_model_set_params(self._h, p.ctypes.data_as(_fp), p.size))

    def get_params(self):
        p = np.empty(self.num_params(), dtype=np.float32)
        _check(lib().rfd_model_get_params(self._h, p.ctypes.data_as(_fp), p.size))
        return p

    def forward(self, x_dev, B, y_dev):
        _check(lib().rfd_model_forward(self._h, ctypes.c_void_p(x_dev), int(B), ctypes.c_void_p(y_dev)))

    def gradients(self, x_dev, t_dev, B):
        g = np.empty(self.num_params(), dtype=np.float32)
        loss = ctypes.c_float()
        _check(lib().rfd_model_gradients(self._h, ctypes.c_void_p(x_dev), ctypes.c_void_p(t_dev),
                                         int(B), g.ctypes.data_as(_fp), ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, x_dev, t_dev, B, lr):
        loss = ctypes.c_float()
        _check(lib().rfd_model_train_step(self._h, ctypes.c_void_p(x_dev), ctypes.c_void_p(t_dev),
                                          int(B), ctypes.c_float(lr), ctypes.byref(loss)))
        return loss.value

    def save(self, path):
        np.save(path, self.get_params())

    @classmethod
    def load(cls, path, device=0):
        return cls(device=device, params=np.load(path))

    @classmethod
    def pretrained(cls, device=0):
        """The network shipped with the package (robotfd_b200/bracket_model.npy), trained by
        robotfd_b200/train_bracket.py on uneven-batch pairs labelled by the plain method."""
        return cls.load(os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                     "bracket_model.npy"), device)


def gemm_bf16(M, N, K, a_ptr, a_sr, a_sc, b_ptr, b_sr, b_sc, c_ptr):
    """The network's GEMM kernel alone (device pointers, FP32 operands rounded to BF16)."""
    _check(lib().rfd_gemm_bf16(M, N, K, ctypes.c_void_p(a_ptr), a_sr, a_sc, ctypes.c_void_p(b_ptr),
                               b_sr, b_sc, ctypes.c_void_p(c_ptr)))
