"""The source-compatible Alpha_Shapes_2D class (include/Alpha_Shapes_2D.h,
replacing gpudt/AlphaShape/Alpha_Shapes_2D.h:43-121).

tests/cpp/alpha_class_main.cpp is the reference caller's call sequence
(main.cu:376-395: gpudtComputeDT, Alpha_Shapes_2D(pInput, pOutput),
computeAlphaShapes(), the master-list iterators, setAlpha/getAlpha) plus a
friend `Visualizer` that writes the members out.  On the CPU it must compile
and link against libgalpha.so, with std::vector and with thrust host vectors;
on a GPU it runs, and every member equals what galphaCompute and
galphaMasterList return for the same triangulation.
"""
import os
import subprocess

import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "cpp", "alpha_class_main.cpp")
LIBDIR = os.path.join(ROOT, "galpha_b200", "lib")


def _compile(out, *extra):
    if not os.path.exists(os.path.join(LIBDIR, "libgalpha.so")):
        from galpha_b200 import build

        build.build()
    cmd = ["g++", "-std=c++17", "-O1", *extra, "-I" + os.path.join(ROOT, "include"), SRC, "-L" + LIBDIR,
           "-lgalpha", "-Wl,-rpath," + LIBDIR, "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def test_reference_call_sequence_compiles(tmp_path):
    _compile(tmp_path / "acm")


def test_reference_call_sequence_compiles_with_thrust_vectors(tmp_path):
    _compile(tmp_path / "acm_thrust", "-DGALPHA_THRUST_HOST_VECTORS", "-I/usr/local/cuda/include")


def _read(path):
    raw = open(path, "rb").read()
    n = np.frombuffer(raw[:32], np.int32)
    off = 32
    out = {"status": int(n[7])}
    for key, dtype, count in (("triangles", G.TRIANGLE_DTYPE, n[0]), ("spectrum", np.float64, n[1]),
                              ("point_list", G.POINT_INTERVAL_DTYPE, n[2]), ("edge_list", G.EDGE_INTERVAL_DTYPE, n[3]),
                              ("tri_list", G.TRIANGLE_INTERVAL_DTYPE, n[4]), ("master_list", G.ALPHA_DTYPE, n[5]),
                              ("spec_pointers", np.int32, n[6])):
        dt = np.dtype(dtype)
        out[key] = np.frombuffer(raw[off:off + dt.itemsize * int(count)], dt)
        off += dt.itemsize * int(count)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(1000, 1), (20000, 31)])
def test_class_members_equal_c_abi(engine, tmp_path, n, seed):
    exe = _compile(tmp_path / "acm")
    pts = D.uniform_points(n, seed)
    with open(tmp_path / "pts.bin", "wb") as f:
        f.write(np.int32(n).tobytes())
        f.write(np.ascontiguousarray(pts, np.float64).tobytes())
    r = subprocess.run([str(exe), str(tmp_path / "pts.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    got = _read(tmp_path / "out.bin")
    assert got["status"] == 0
    # the same triangulation through the C ABI
    p = G.GPUDTParams(pts, fboSize=1024)
    dt = G.DTOutput(got["triangles"].copy())
    a = engine.alpha_of(p, dt)
    ml, sp = engine.master_list()
    for k in ("spectrum", "point_list", "edge_list", "tri_list"):
        assert np.array_equal(got[k], a[k]), k
    assert np.array_equal(got["master_list"], ml)
    assert np.array_equal(got["spec_pointers"], sp)
