"""Golden fixtures from the reference's own GPU path, run on a B200 (test infrastructure).

oracle/_ref/libref_gpu.so is built by `make -C oracle/refharness gpu` from the reference's
sources in place (src/intersection_algorithm_in_parallel.cu for sm_100a with its own
optimisation flags and nvcc's default contraction, src/curve.cpp) and gpu_harness.cpp, which
drives the reference's Cuda_intersection with the steps of its search driver
(src/frechet.cpp:26-63) and records the endpoint bound, DFD (Bound_call_gpu's ub), its VE-FD
(lb), every probe radius and decision (intersection_interval_call_gpu) and the result.  The
fused decision kernel is used (forceOversize), as the reference does when memory is short.

Run on a GPU machine with the prebuilt library (the reference checkout is needed only to
build it):

    python tests/golden/make_reference_gpu_golden.py OUT.json

The cases are small seeded pairs (every thread block of the reference's persistent grid owns
rows: at least 4 rows per block of 148).
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

CASES = [
    ("config0_2000x1900", (0, 2, 2000, 1900, 1.0, 0.05, 0, 0)),
    ("spline3d_1500x1400", (1, 3, 1500, 1400, 100.0, 0.1, 11, 1500)),
    ("walk2d_1200x1100", (0, 2, 1200, 1100, 1.0, 0.05, 12, 1200)),
    ("spline2d_1800x900", (1, 2, 1800, 900, 100.0, 0.1, 13, 1800)),
]
FLT_EPSILON = float(np.finfo(np.float32).eps)
MAXP = 200


def main(out_path):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so"))
    dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    lib.ref_gpu_solve.argtypes = [dp, ctypes.c_long, dp, ctypes.c_long, ctypes.c_int,
                                  ctypes.c_double, dp, ip, dp, ip, ctypes.c_int]
    res = {}
    for name, g in CASES:
        P, Q = oracle.gen_pair(*g)
        P, Q = np.ascontiguousarray(P), np.ascontiguousarray(Q)
        out = (ctypes.c_double * 6)()
        n = ctypes.c_int()
        le = (ctypes.c_double * MAXP)()
        ld = (ctypes.c_int * MAXP)()
        rc = lib.ref_gpu_solve(P.ctypes.data_as(dp), len(P), Q.ctypes.data_as(dp), len(Q),
                               P.shape[1], FLT_EPSILON, out, ctypes.byref(n), le, ld, MAXP)
        if rc:
            raise RuntimeError(f"{name}: ref_gpu_solve failed ({rc})")
        res[name] = {"gen": list(g), "n1": len(P), "n2": len(Q), "endpoint": out[0],
                     "dfd": out[1], "vefd": out[2], "distance": out[3], "lb": out[4],
                     "ub": out[5], "probes": n.value,
                     "probe_eps": [le[k] for k in range(n.value)],
                     "probe_dec": [bool(ld[k]) for k in range(n.value)]}
        print(name, res[name]["dfd"], res[name]["vefd"], res[name]["distance"], n.value,
              flush=True)
    with open(out_path, "w") as f:
        json.dump({"note": "the reference's own GPU path (sm_100a build), forceOversize; made by "
                           "tests/golden/make_reference_gpu_golden.py", "cases": res}, f,
                  indent=0, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_gpu.json"))
