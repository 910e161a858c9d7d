"""The drop-in boundary without a GPU: C ABI exports, loader rules, generators, the search
state machine and the C++ headers (reference interfaces: include/wrapper.hpp,
include/txtReader.hpp, include/curve.hpp, include/geometry_basics.hpp)."""
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "rfd.h")).read()
    return sorted(set(re.findall(r"\b(rfd_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(built):
    lib = built.lib()
    decl = declared_symbols()
    assert len(decl) >= 17
    missing = [s for s in decl if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(built.EXPORTS) == decl
    # exported from the shared object with C linkage
    out = subprocess.run(["nm", "-D", "--defined-only", built.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for s in decl:
        assert re.search(rf"\bT {s}$", out, re.M), s


def test_cpp_dropin_symbols_exported(built):
    out = subprocess.run(["nm", "-DC", "--defined-only", built.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    for sym in ["compute_distance_parallel(Curve const&, Curve const&, bool)",
                "Frechet::Continuous::distance_cuda(Curve const&, Curve const&, double, bool)",
                "Cuda_intersection::Bound_call_gpu(double*, double*)",
                "Cuda_intersection::intersection_interval_call_gpu(double)"]:
        assert sym in out, sym


def test_abi_and_status(built):
    lib = built.lib()
    assert lib.rfd_abi_version() == 1
    assert lib.rfd_status_string(0) == b"ok"
    assert lib.rfd_status_string(4) == b"inter-warp wait timed out"


def test_options_defaults(built):
    o = built.options()
    assert o.stop_mode == built.RFD_STOP_ABS and o.tol == built.FLT_EPSILON
    assert o.reference_quirks == 1
    p = built.options(precise=True)
    assert p.stop_mode == built.RFD_STOP_REL and p.tol == 2.0 ** -33 and p.reference_quirks == 0


def test_no_device_is_reported(built):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(built.RfdError) as e:
        built.Context(0)
    assert e.value.code == built.RFD_ERR_NODEV


def write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_loader_rules(built, tmp_path):
    path = write(tmp_path, "a.txt",
                 "0,0\n0,0\n1,0\n1,0,5\n\n2,abc\n2,1\n  3.5 , 4e0\n3.5,4\n")
    # '1,0,5' has 3 coordinates: the 2D loader keeps it as a point with an extra value,
    # the C ABI (fixed [n][2] layout) rejects such a file
    with pytest.raises(built.RfdError):
        built.txt_loader2(path)
    path = write(tmp_path, "b.txt", "0,0\n0,0\n1,0\n1,0\n\n2,1\n  3.5 , 4e0\n3.5,4\n7,7\n")
    a = built.txt_loader2(path)
    np.testing.assert_array_equal(a, [[0, 0], [1, 0], [2, 1], [3.5, 4], [7, 7]])
    # LIMIT counts every non-empty line read; START skips points counted below START
    np.testing.assert_array_equal(built.txt_loader2(path, limit=3), [[0, 0], [1, 0]])
    np.testing.assert_array_equal(built.txt_loader2(path, start=3), [[1, 0], [2, 1], [3.5, 4], [7, 7]])
    # 3D dedupe compares all three coordinates
    p3 = write(tmp_path, "c.txt", "0,0,0\n0,0,1\n0,0,1\n0,1,1\n")
    np.testing.assert_array_equal(built.txt_loader3(p3), [[0, 0, 0], [0, 0, 1], [0, 1, 1]])
    with pytest.raises(built.RfdError):
        built.txt_loader2(str(tmp_path / "missing.txt"))


def test_generators_deterministic(built):
    a = built.gen_pair(1, 3, 5000, 4000, 100.0, 0.1, 1, 0)
    b = built.gen_pair(1, 3, 5000, 4000, 100.0, 0.1, 1, 0)
    c = built.gen_pair(1, 3, 5000, 4000, 100.0, 0.1, 1, 1)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    (P, Q), = built.gen_config(0)
    assert P.shape == (2000, 2) and Q.shape == (1900, 2)
    steps = np.linalg.norm(np.diff(P, axis=0), axis=1)
    assert 1.0 < steps.mean() < 1.6  # Gaussian walk, sigma 1 per coordinate
    dims, n1, n2, styles, _, _ = built.gen_batch_spec(2, 4096, 2)
    assert set(dims) == {2, 3} and n1.min() >= 100 and n1.max() <= 50000
    assert 1500 < np.median(np.concatenate([n1, n2])) < 2600
    assert 0.4 < styles.mean() < 0.6


def test_generator_workload_sizes(built):
    dims, n1, n2, styles, scales, _ = built.gen_batch_spec(1, 1, 1)
    assert (dims[0], n1[0], n2[0], styles[0], scales[0]) == (3, 200000, 200000, 1, 100.0)
    dims, n1, n2, _, scales, _ = built.gen_batch_spec(4, 512, 5)
    assert (dims == 3).all() and n1.min() >= 100000 and n1.max() <= 400000 and scales[0] == 1e4


def bisect_host(lb, ub, tol, stop_mode, decide, max_probes=64):
    probes = []
    while True:
        gap = ub - lb
        if not (gap > tol if stop_mode == 0 else gap > tol * ub) or len(probes) >= max_probes:
            break
        split = (ub + lb) / 2.0
        if not (lb < split < ub):
            break
        probes.append(split)
        if decide(split):
            ub = split
        else:
            lb = split
    return lb, ub, probes


@pytest.mark.parametrize("stop_mode,tol", [(0, np.finfo(np.float32).eps), (1, 2.0 ** -33)])
def test_search_state_machine_matches_bisection(built, stop_mode, tol):
    fd = 0.7313
    lb, ub, want = bisect_host(0.5, 1.3, tol, stop_mode, lambda e: e >= fd)
    st, ist = [0.5, 1.3, np.nan, np.nan, tol, 0.0], [0, 0, 64, 0]
    got, outcome = [], None
    more, e, st, ist = built.search_step(st, ist, stop_mode, False, 0.0, False)
    while more:
        got.append(e)
        more, e2, st, ist = built.search_step(st, ist, stop_mode, True, e, e >= fd)
        e = e2
    assert got == want and st[0] == lb and st[1] == ub


def test_search_bracket_verification(built):
    fd = 0.7313
    decide = lambda e: e >= fd  # noqa: E731
    def run(lo, hi):
        st, ist = [0.5, 1.3, lo, hi, 2.0 ** -33, 0.0], [1, 0, 64, 0]
        seq = []
        more, e, st, ist = built.search_step(st, ist, 1, False, 0.0, False)
        while more:
            seq.append(e)
            more, e2, st, ist = built.search_step(st, ist, 1, True, e, decide(e))
            e = e2
        return seq, st, ist
    seq, st, ist = run(0.73, 0.732)  # good bracket: hi then lo verified first
    assert seq[:2] == [0.732, 0.73] and not (ist[3] & built.FLAG_BRACKET_WIDENED)
    assert st[0] <= fd <= st[1] and st[1] - st[0] <= 2.0 ** -33 * st[1]
    plain, _, _ = run(np.nan, np.nan)
    assert len(seq) < len(plain)
    seq, st, ist = run(0.70, 0.71)  # too low: hi fails, window moves up geometrically
    assert seq[0] == 0.71 and seq[1] == 0.71 + 2 * 0.01 and ist[3] & built.FLAG_BRACKET_WIDENED
    assert st[0] <= fd <= st[1] and st[1] - st[0] <= 2.0 ** -33 * st[1]
    seq, st, ist = run(0.80, 0.81)  # too high: lo fails, window moves down
    assert st[0] <= fd <= st[1] and st[1] - st[0] <= 2.0 ** -33 * st[1]


def run_search(built, st, ist, stop_mode, decide):
    seq = []
    more, e, st, ist = built.search_step(st, ist, stop_mode, False, 0.0, False)
    while more:
        seq.append(e)
        more, e2, st, ist = built.search_step(st, ist, stop_mode, True, e, decide(e))
        e = e2
    return seq, st, ist


@pytest.mark.parametrize("stop_mode,tol", [(0, np.finfo(np.float32).eps), (1, 2.0 ** -33)])
def test_search_threshold_probe(built, stop_mode, tol):
    """lb is proven: a bracket reaching below lb + tolerance probes that threshold first."""
    lb = 0.7313
    thr = lb + 0.999 * tol if stop_mode == 0 else lb * (1 + 0.999 * tol)
    # distance within the tolerance of lb: one probe ends the search
    fd = lb + 1e-3 * tol
    seq, st, ist = run_search(built, [lb, 1.3, lb - 1e-3, lb + 1e-6 * tol, tol, 0.0], [1, 0, 64, 0],
                              stop_mode, lambda e: e >= fd)
    assert seq == [thr] and st[0] == lb and st[1] == thr and st[5] == thr
    assert not (ist[3] & built.FLAG_BRACKET_WIDENED)
    # distance far above: the threshold fails, the bracket below it is skipped, bisection
    fd = lb + 0.01
    seq, st, ist = run_search(built, [lb, 1.3, lb - 1e-3, lb + 1e-6 * tol, tol, 0.0], [1, 0, 64, 0],
                              stop_mode, lambda e: e >= fd)
    assert seq[0] == thr and seq[1] == (thr + 1.3) / 2
    assert st[0] <= fd <= st[1] and not (ist[3] & built.FLAG_BRACKET_WIDENED)
    # ... or a bracket above the threshold is verified after it
    seq, st, ist = run_search(built, [lb, 1.3, lb - 1e-3, lb + 0.05, tol, 0.0], [1, 0, 64, 0],
                              stop_mode, lambda e: e >= fd)
    assert seq[:2] == [thr, lb + 0.05] and st[0] <= fd <= st[1]
    # a bracket wholly above the threshold skips it
    seq, st, ist = run_search(built, [0.7, 1.3, 0.72, 0.75, tol, 0.0], [1, 0, 64, 0], stop_mode,
                              lambda e: e >= fd)
    assert seq[0] == 0.75


CPP_TEST = r'''
#include <cstdio>
#include "txtReader.hpp"
#include "wrapper.hpp"
int main(int argc, char** argv) {
  Curve c(txtLoader2(argv[1]), 2);
  std::printf("%zu %zu %.1f %.1f\n", c.size(), c.dimensions(), c.back()[0], c[1].dist_sqr(c[0]));
  Curves cs; cs.push_back(c);
  std::printf("%zu\n", cs.get(0).size());
  return 0;
}
'''


def test_cpp_headers_compile_and_load(built, tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text(CPP_TEST)
    exe = tmp_path / "t"
    libdir = os.path.dirname(built.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                    str(exe), "-L", libdir, "-lrfd", f"-Wl,-rpath,{libdir}"], check=True)
    data = write(tmp_path, "d.txt", "0,0\n3,4\n3,4\n6,8\n")
    out = subprocess.run([str(exe), data], capture_output=True, text=True, check=True).stdout
    assert out.split() == ["3", "2", "6.0", "25.0", "3"]


def test_cli_usage(built):
    r = subprocess.run([built.FD_PATH], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr


def test_distance_matrix_checks_arguments_without_a_context(built):
    """The matrix entry point validates its arguments before touching a device."""
    import ctypes
    rc = built.lib().rfd_distance_matrix(None, 2, None, None, None, None, 0.0, None, None)
    assert rc == built.RFD_ERR_ARG


def test_ctypes_structs_match_the_header(built, tmp_path):
    """The Python mirrors of rfd_options and rfd_result have the C layout (size and offsets)."""
    fields = {"rfd_options": (built.Options, [f for f, _ in built.Options._fields_]),
              "rfd_result": (built.Result, [f for f, _ in built.Result._fields_])}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "rfd.h"', "int main(void) {"]
    for name, (_, names) in fields.items():
        lines.append(f'  printf("%zu\\n", sizeof({name}));')
        lines += [f'  printf("%zu\\n", offsetof({name}, {f}));' for f in names]
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    want = []
    for _, (cls, names) in fields.items():
        want.append(ctypes_sizeof(cls))
        want += [getattr(cls, f).offset for f in names]
    assert got == want


def ctypes_sizeof(cls):
    import ctypes
    return ctypes.sizeof(cls)
