"""The oracle and the boundary against outputs of the reference's own code (no GPU).

tests/golden/reference_host.json was recorded by tests/golden/make_reference_host_golden.py
from the reference's host sources (built in place by oracle/refharness/Makefile):
  - compute_distance_parallel -> Frechet::Continuous::distance_cuda (src/frechet.cpp:18-75),
    the reference's own search driver, run with the oracle's DFD / VE-FD / decisions;
  - the endpoint bound of Point::dist_sqr (include/geometry_basics.hpp:72);
  - txtLoader2 / txtLoader3 (include/txtReader.hpp:6-88) on tests/golden/txt/*.
Bars: bit-exact distances and endpoint bounds, identical loaded points.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from tests.golden.cases import CASES, build_input

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIXTURE = os.path.join(HERE, "golden", "reference_host.json")


def golden():
    with open(FIXTURE) as f:
        return json.load(f)


def test_fixture_complete():
    g = golden()
    assert [c["name"] for c in g["distance"]] == [n for n, _ in CASES]
    assert len(g["loader"]) >= 8


@pytest.mark.parametrize("case", golden()["distance"], ids=lambda c: c["name"])
def test_oracle_search_matches_reference_driver(built, case):
    P, Q = build_input(case["input"])
    assert (len(P), len(Q), P.shape[1]) == (case["n1"], case["n2"], case["dims"])
    assert oracle.endpoint(P, Q) == case["endpoint"]
    r = oracle.distance(P, Q, stop_mode=0, quirks=True, threads=8)
    assert r["distance"] == case["distance"]


@pytest.mark.parametrize("lc", golden()["loader"], ids=lambda c: f"{c['file']}-{c['dims']}-{c['start']}-{c['limit']}")
def test_c_abi_loader_matches_reference(built, lc):
    path = os.path.join(HERE, "golden", "txt", lc["file"])
    load = built.txt_loader2 if lc["dims"] == 2 else built.txt_loader3
    if any(n != lc["dims"] for n in lc["ncoord"]):
        # the C ABI returns a fixed [n][dims] array and rejects other coordinate counts
        with pytest.raises(built.RfdError):
            load(path, lc["start"], lc["limit"])
        return
    got = load(path, lc["start"], lc["limit"])
    want = np.array(lc["points"], dtype=float).reshape(-1, lc["dims"])
    assert got.shape == want.shape
    assert np.array_equal(np.signbit(got), np.signbit(want)) and np.array_equal(got, want)


CPP = r'''
#include <cstdio>
#include <cstdlib>
#include "txtReader.hpp"
int main(int argc, char** argv) {
  int dims = std::atoi(argv[2]), start = std::atoi(argv[3]), limit = std::atoi(argv[4]);
  Points p = dims == 2 ? txtLoader2(argv[1], start, limit) : txtLoader3(argv[1], start, limit);
  for (auto& q : p) {
    std::printf("%d", q.size());
    for (double v : q.coordinates) std::printf(" %a", v);
    std::printf("\n");
  }
  return 0;
}
'''


@pytest.fixture(scope="module")
def cpp_loader(tmp_path_factory):
    d = tmp_path_factory.mktemp("ldr")
    (d / "l.cpp").write_text(CPP)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(d / "l.cpp"),
                    "-o", str(d / "l")], check=True)
    return str(d / "l")


@pytest.mark.parametrize("lc", golden()["loader"], ids=lambda c: f"{c['file']}-{c['dims']}-{c['start']}-{c['limit']}")
def test_cpp_loader_matches_reference(cpp_loader, lc):
    path = os.path.join(HERE, "golden", "txt", lc["file"])
    out = subprocess.run([cpp_loader, path, str(lc["dims"]), str(lc["start"]), str(lc["limit"])],
                         capture_output=True, text=True, check=True).stdout.splitlines()
    assert len(out) == len(lc["points"])
    for line, pt, nc in zip(out, lc["points"], lc["ncoord"]):
        f = line.split()
        assert int(f[0]) == nc
        vals = [float.fromhex(x) for x in f[1:]]
        k = min(nc, lc["dims"])
        assert vals[:k] == pt[:k]
