"""Golden fixtures from the reference's own host code, run on this CPU.

oracle/_ref/libref_host.so is built by oracle/refharness/Makefile from the reference's
sources in place (src/frechet.cpp, src/compute_distance_wrapper.cpp, src/curve.cpp,
include/geometry_basics.hpp, include/txtReader.hpp) with an oracle-backed GPU class.
This records, for fixed seeded inputs:
  - compute_distance_parallel: the reference's search driver (endpoint bound, bisection,
    FLT_EPSILON stop, midpoint) driving the oracle's DFD, VE-FD and decisions;
  - the endpoint bound as Point::dist_sqr computes it;
  - txtLoader2 / txtLoader3 on the edge-case files in tests/golden/txt/.
The reference's GPU kernels are not run here: this CPU has no GPU, and the harness replaces
its GPU class with the oracle.

    RFD_REFERENCE_DIR=<reference checkout> make -C oracle/refharness
    python tests/golden/make_reference_host_golden.py   # writes tests/golden/reference_host.json
"""
import ctypes
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from tests.golden.cases import CASES, LOADER_CASES, build_input  # noqa: E402

_dp = ctypes.POINTER(ctypes.c_double)


def main():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_host.so"))
    L.refhost_distance.restype = ctypes.c_double
    L.refhost_distance.argtypes = [_dp, ctypes.c_long, _dp, ctypes.c_long, ctypes.c_int]
    L.refhost_endpoint.restype = ctypes.c_double
    L.refhost_endpoint.argtypes = [_dp, ctypes.c_long, _dp, ctypes.c_long, ctypes.c_int]
    L.refhost_load.restype = ctypes.c_long
    L.refhost_load.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                               ctypes.POINTER(ctypes.c_int), ctypes.c_long]
    out = {"source": "reference host code (libref_host.so) with the CPU oracle as its GPU class",
           "distance": [], "loader": []}
    saved = os.dup(1)
    log = open(os.devnull, "w")
    for name, recipe in CASES:
        P, Q = build_input(recipe)
        P, Q = np.ascontiguousarray(P), np.ascontiguousarray(Q)
        args = (P.ctypes.data_as(_dp), len(P), Q.ctypes.data_as(_dp), len(Q), P.shape[1])
        sys.stdout.flush()
        os.dup2(log.fileno(), 1)  # the reference prints its progress
        try:
            dist = L.refhost_distance(*args)
            endpoint = L.refhost_endpoint(*args)
        finally:
            os.dup2(saved, 1)
        out["distance"].append({"name": name, "input": recipe, "n1": len(P), "n2": len(Q),
                                "dims": P.shape[1], "endpoint": endpoint, "distance": dist})
        print(f"{name}: {dist!r}", flush=True)
    for fname, dims, start, limit in LOADER_CASES:
        cap = 1000
        buf = (ctypes.c_double * (cap * dims))()
        nc = (ctypes.c_int * cap)()
        n = L.refhost_load(os.path.join(HERE, "txt", fname).encode(), dims, start, limit, buf, nc, cap)
        pts = [[buf[i * dims + k] for k in range(dims)] for i in range(n)]
        out["loader"].append({"file": fname, "dims": dims, "start": start, "limit": limit,
                              "points": pts, "ncoord": [nc[i] for i in range(n)]})
    with open(os.path.join(HERE, "reference_host.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
