"""Fast parallel loader and binary files (CPU): identical to the loaders' rules."""
import os

import numpy as np
import pytest

GOLDEN_TXT = os.path.join(os.path.dirname(__file__), "golden", "txt")

# lines that exercise the parser: spaces, empty tokens, carriage returns, trailing commas,
# rejected tokens, out-of-range exponents, hexadecimal, inf and nan, duplicates, blank lines
TRICKY = ["1.5,2.5", " 3 , 4 ", "5,,6", "7,8,", "\t9,10\r", "abc,1", "1e-400,2", "1e400,3",
          "0x1p3,4", "inf,5", "nan,6", "", "   ", ",", "11,12", "11,12", "11,12.0", "13",
          "14,15,16", "17,18,19,20", "-0.0,0", "0,-0.0", "1e308,1e-308", "+5,-.5"]


def write(path, lines, trailing_newline=True):
    with open(path, "w") as f:
        f.write("\n".join(lines) + ("\n" if trailing_newline else ""))


@pytest.mark.parametrize("trailing", [True, False])
@pytest.mark.parametrize("dims", [2, 3])
def test_fast_loader_matches_loader(built, tmp_path, trailing, dims):
    rng = np.random.default_rng(dims + 2 * trailing)
    lines = []
    for k in range(30000):
        if rng.random() < 0.05:
            lines.append(TRICKY[rng.integers(len(TRICKY))])
        else:
            v = rng.normal(size=dims) * 10.0 ** rng.integers(-3, 4)
            lines.append(",".join(repr(float(x)) for x in v))
    path = str(tmp_path / "curve.txt")
    write(path, lines, trailing)
    for start, limit in [(0, 10000000), (5, 10000000), (0, 777), (100, 20000)]:
        try:
            want = built.txt_loader2(path, start, limit) if dims == 2 else built.txt_loader3(path, start, limit)
        except built.RfdError:
            with pytest.raises(built.RfdError):
                built.txt_loader_fast(path, dims, start, limit, threads=8)
            continue
        for threads in (1, 3, 8, 0):
            got = built.txt_loader_fast(path, dims, start, limit, threads=threads)
            assert got.shape == want.shape and np.array_equal(got.view(np.int64), want.view(np.int64))


def test_fast_loader_on_golden_files(built):
    for name in sorted(os.listdir(GOLDEN_TXT)):
        path = os.path.join(GOLDEN_TXT, name)
        for dims in (2, 3):
            try:
                want = built.txt_loader2(path) if dims == 2 else built.txt_loader3(path)
            except built.RfdError:
                with pytest.raises(built.RfdError):
                    built.txt_loader_fast(path, dims)
                continue
            got = built.txt_loader_fast(path, dims, threads=4)
            assert np.array_equal(got.view(np.int64), want.view(np.int64)), name


def test_tricky_lines_two_dims(built, tmp_path):
    """Each tricky line on its own, and the lines that keep two coordinates together."""
    for k, line in enumerate(TRICKY + ["1,2,", " 7 , 8 \r"]):
        path = str(tmp_path / f"t{k}.txt")
        write(path, ["0.5,0.25", line, "9,9"])
        try:
            want = built.txt_loader2(path)
        except built.RfdError:
            with pytest.raises(built.RfdError):
                built.txt_loader_fast(path, 2, threads=2)
            continue
        got = built.txt_loader_fast(path, 2, threads=2)
        assert np.array_equal(got.view(np.int64), want.view(np.int64)), line
    ok = ["1.5,2.5", " 3 , 4 ", "7,8,", "\t9,10\r", "0x1p3,4", "inf,5", "", "11,12", "11,12",
          "-0.0,0", "0,-0.0", "+5,-.5"]
    path = str(tmp_path / "ok.txt")
    write(path, ok)
    want = built.txt_loader2(path)
    assert len(want) == 9
    assert np.array_equal(built.txt_loader_fast(path, 2, threads=2).view(np.int64), want.view(np.int64))


def test_binary_round_trip(built, tmp_path):
    rng = np.random.default_rng(3)
    for d in (2, 3):
        P = rng.normal(size=(1234, d)) * 1e3
        P[5] = [np.inf] + [0.0] * (d - 1)
        path = str(tmp_path / f"c{d}.rfdb")
        built.save_bin(path, P)
        Q = built.load_bin(path)
        assert Q.shape == P.shape and np.array_equal(Q.view(np.int64), P.view(np.int64))
    empty = str(tmp_path / "e.rfdb")
    built.save_bin(empty, np.zeros((0, 2)))
    assert built.load_bin(empty).shape == (0, 2)
    bad = str(tmp_path / "bad.rfdb")
    with open(bad, "wb") as f:
        f.write(b"NOPE" + bytes(20))
    with pytest.raises(built.RfdError):
        built.load_bin(bad)
