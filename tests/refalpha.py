"""Runs the reference's own GPU alpha-shape engine (oracle/_ref/librefalpha.so,
built by oracle/ref.mk from gpudt/AlphaShape of the reference tree) on given
triangulations.  Test infrastructure: the parity tests use it as the checker
of galphaCompute.

    python tests/refalpha.py IN.npz OUT.npz

IN holds pts_<k> (n x 2 float64) and tris_<k> (nTris x 9 int32, gpudtTriangle
records) for every case k; OUT receives spectrum_<k>, point_list_<k> (n x 2),
edge_list_<k> (nEdges x 6: ro, nu_min, nu_max, sc, tIndex, vOpp),
tri_list_<k>, master_list_<k> (nMaster x 3: simplex_index, st, at) and
spec_pointers_<k>.  The engine runs in this separate process so that its
default-stream, synchronous style and its console output stay out of the test
process.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "librefalpha.so")


def load():
    L = ctypes.CDLL(LIB)
    L.refalpha_run.restype = ctypes.c_void_p
    L.refalpha_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    L.refalpha_sizes.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.refalpha_copy.argtypes = [ctypes.c_void_p] * 7
    L.refalpha_free.argtypes = [ctypes.c_void_p]
    return L


def run_one(L, pts, tris):
    pts = np.ascontiguousarray(pts, np.float64)
    tris = np.ascontiguousarray(tris, np.int32).reshape(-1, 9)
    h = L.refalpha_run(pts.ctypes.data, len(pts), tris.ctypes.data, len(tris))
    if not h:
        raise RuntimeError("reference alpha engine failed")
    try:
        sz = np.zeros(6, np.int32)
        L.refalpha_sizes(h, sz.ctypes.data)
        out = {
            "spectrum": np.zeros(sz[0], np.float64),
            "point_list": np.zeros((sz[1], 2), np.int32),
            "edge_list": np.zeros((sz[2], 6), np.int32),
            "tri_list": np.zeros(sz[3], np.int32),
            "master_list": np.zeros((sz[4], 3), np.int32),
            "spec_pointers": np.zeros(sz[5], np.int32),
        }
        L.refalpha_copy(h, *[out[k].ctypes.data for k in ("spectrum", "point_list", "edge_list", "tri_list",
                                                             "master_list", "spec_pointers")])
    finally:
        L.refalpha_free(h)
    return out


def main(src, dst):
    z = np.load(src)
    keys = sorted(k[4:] for k in z.files if k.startswith("pts_"))
    L = load()
    res = {}
    for k in keys:
        out = run_one(L, z["pts_" + k], z["tris_" + k])
        for name, arr in out.items():
            res["%s_%s" % (name, k)] = arr
    np.savez(dst, **res)


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
