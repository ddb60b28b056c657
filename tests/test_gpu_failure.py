"""Failure detection on the GPU without a GPU fault.

Every iterative stage has a round cap and every single-pass look-back wait a
spin bound (galphaSetLimits lowers them per handle).  A test makes one of them
run out -- the cap set to 1 round, or the first tile of the spectrum sort's
look-back withholding its counts so that the next tile's wait ends -- and
checks that the call returns the error status, that the kernel returned (the
context stays usable), and that the next call on the same handle, with the
defaults restored, computes the full result (checked against the CPU oracle).
"""
import ctypes

import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from alphacheck import compare_alpha
from dtcheck import compare_dt

pytestmark = pytest.mark.gpu
NOCONVERGE = -5


def _set(engine, max_rounds, spin, hold):
    L = G.load()
    L.galphaSetLimits.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    assert L.galphaSetLimits(engine._h, max_rounds, spin, hold) == 0


def _check_full(engine, pts, fbo):
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=fbo))
    ok, rep = compare_dt(pts, dt.vtx, dt.tri)
    assert ok and rep["identical"], rep
    a = engine.alpha_resident()
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, 4)
    assert ok, rep


def test_round_cap_reports_noconverge(engine):
    pts = D.uniform_points(30000, 41)
    try:
        _set(engine, 1, 0, 0)
        with pytest.raises(G.GpudtError) as ei:
            engine.triangulate(G.GPUDTParams(pts, fboSize=1024))
        assert ei.value.code == NOCONVERGE
    finally:
        _set(engine, 0, 0, 0)
    _check_full(engine, pts, 1024)


def test_sort_lookback_wait_runs_out(engine):
    pts = D.uniform_points(40000, 42)
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=1024))
    try:
        _set(engine, 0, 2000, 1)
        with pytest.raises(G.GpudtError) as ei:
            engine.alpha_resident()
        assert ei.value.code == NOCONVERGE
        assert "98" in str(ei.value)
    finally:
        _set(engine, 0, 0, 0)
    # the resident mesh is untouched by the failed alpha stage
    a = engine.alpha_resident()
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, 4)
    assert ok, rep
    _check_full(engine, pts, 1024)
