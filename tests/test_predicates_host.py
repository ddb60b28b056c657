"""Host checks of the staged predicates of galpha_b200/csrc/exact.cuh (the
header the device kernels include), compiled for the CPU with g++:

* the FP32 and FP64 filters never return a sign that differs from the exact
  expansion's, over adversarial families (near-collinear and near-cocircular
  points a few ulps off, lattice points, FP32-subnormal differences,
  differences beyond the FP32 stage's 2^10 span, mixed scales);
* the FP32 stage decides all but a few tests of uniform points in the unit
  square and leaves FP32-subnormal differences to the FP64 stage;
* an independent check in rational arithmetic (Python fractions) of both
  filters' answers on near-degenerate cases.
"""
import os
import shutil
import subprocess
from fractions import Fraction

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "pred_stages_check.cpp")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("pred") / "pred_stages_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "galpha_b200", "csrc"), SRC, "-o", exe],
                   check=True, capture_output=True, text=True)
    return exe


def _run(exe, mode, n):
    r = subprocess.run([exe, mode, str(n)], check=True, capture_output=True, text=True)
    return r.stdout.splitlines()


def test_filters_never_contradict_exact(checker):
    n = 100000
    rows = {}
    for line in _run(checker, "count", n):
        fam, pred, cases, d32, d64, bad32, bad64, ovf = line.split()
        rows[(fam, pred)] = tuple(map(int, (cases, d32, d64, bad32, bad64, ovf)))
    assert len(rows) == 16
    for key, (cases, d32, d64, bad32, bad64, ovf) in rows.items():
        assert cases == n and ovf == 0, key
        assert bad32 == 0 and bad64 == 0, key
    # uniform points in the unit square: the FP32 stage decides all but a few tests
    assert rows[("uniform", "orient")][1] >= 0.999 * n and rows[("uniform", "incircle")][1] >= 0.999 * n
    # exact lattice degeneracies reach neither filter's decision, the rest are decided
    assert 0 < rows[("lattice", "incircle")][1] < n
    # FP32-subnormal differences: the FP32 stage stays undecided, FP64 decides
    assert rows[("subnormal32", "orient")][1] == 0 and rows[("subnormal32", "orient")][2] == n


def _sign(x):
    return (x > 0) - (x < 0)


def _orient(p):
    (ax, ay), (bx, by), (cx, cy) = p[0], p[1], p[2]
    return _sign((ax - cx) * (by - cy) - (ay - cy) * (bx - cx))


def _incircle(p):
    (ax, ay), (bx, by), (cx, cy), (dx, dy) = p
    adx, ady, bdx, bdy, cdx, cdy = ax - dx, ay - dy, bx - dx, by - dy, cx - dx, cy - dy
    al, bl, cl = adx * adx + ady * ady, bdx * bdx + bdy * bdy, cdx * cdx + cdy * cdy
    return _sign(al * (bdx * cdy - cdx * bdy) + bl * (cdx * ady - adx * cdy) + cl * (adx * bdy - bdx * ady))


def test_filters_against_rationals(checker):
    seen = 0
    for line in _run(checker, "dump", 250):
        if not line.startswith("case "):
            continue
        parts = line.split()
        pred = parts[2]
        v = [Fraction(float.fromhex(x)) for x in parts[3:11]]
        pts = [(v[0], v[1]), (v[2], v[3]), (v[4], v[5]), (v[6], v[7])]
        s32, s64 = int(parts[11]), int(parts[12])
        want = _orient(pts) if pred == "orient" else _incircle(pts)
        assert s32 in (2, want), line
        assert s64 in (2, want), line
        seen += 1
    assert seen == 16 * 250
