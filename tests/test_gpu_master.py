"""GPU parity of the master list and spec pointers (compute_master_list,
Alpha_Shapes_2D.cu:641-727) against the oracle's restatement, computed from
the engine's own intervals (whose parity the alpha tests establish)."""
import numpy as np
import pytest

import galpha_b200 as G
from galpha_b200 import datasets as D
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _check(engine, pts, fbo):
    dt = engine.triangulate(G.GPUDTParams(pts, fboSize=fbo))
    res = engine.alpha_resident()
    ml, sp = engine.master_list()
    pt, ed, tr = res["point_list"], res["edge_list"], res["tri_list"]
    idx, st, at, wsp = O.master_list(np.stack([pt["nu_min_rank"], pt["nu_max_rank"]], axis=1), ed["ro_rank"],
                                     ed["nu_min_rank"], ed["nu_max_rank"], tr["ro_rank"])
    np.testing.assert_array_equal(ml["simplex_index"], idx)
    np.testing.assert_array_equal(ml["st"], st)
    np.testing.assert_array_equal(ml["at"], at)
    np.testing.assert_array_equal(sp, wsp)
    # a second request reuses the resident list
    ml2, sp2 = engine.master_list()
    np.testing.assert_array_equal(ml2, ml)
    np.testing.assert_array_equal(sp2, sp)
    return res, ml, sp


@pytest.mark.parametrize("n,seed,fbo", [(1000, 1, 512), (30000, 2, 1024), (200000, 3, 2048)])
def test_master_list_uniform(engine, n, seed, fbo):
    res, ml, sp = _check(engine, D.uniform_points(n, seed), fbo)
    # every spectrum rank > 0 starts one run (sp[r] is the first entry of rank r)
    assert len(sp) == len(res["spectrum"])


def test_master_list_duplicates_and_lattice(engine):
    pts = D.uniform_points(4000, 4)
    lat = np.stack(np.meshgrid(np.arange(20) / 20.0, np.arange(20) / 20.0), -1).reshape(-1, 2)
    pts = np.concatenate([pts, pts[:37], lat])
    res, ml, sp = _check(engine, pts, 1024)
    # dropped duplicates keep rank -1 entries at the front, as the reference's sort does
    assert (ml[:74]["st"] == 2).all()


def test_master_list_large_tie_runs(engine):
    """A 256 x 256 lattice of dyadic spacing: every square's two triangles
    share one exact circumradius, so ranks repeat over tens of thousands of
    entries (runs sorted as sub-arrays), next to the short runs of a uniform
    patch."""
    g = np.stack(np.meshgrid(np.arange(256) / 256.0, np.arange(256) / 256.0), -1).reshape(-1, 2)
    pts = np.concatenate([g * 0.5, 0.5 + 0.5 * D.uniform_points(20000, 12)])
    _check(engine, pts, 2048)


def test_master_list_tiny(engine):
    _check(engine, np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]), 256)


def test_alpha_shapes_class_has_master_list(engine):
    pts = D.uniform_points(2000, 9)
    p = G.GPUDTParams(pts, fboSize=512)
    dt = engine.triangulate(p)
    a = G.AlphaShapes2D(p, dt, engine=engine).compute_alpha_shapes()
    assert a.master_list is not None and a.spec_pointers[0] == -1
    assert len(a.master_list) == 2 * len(pts) + 3 * len(a.edge_list) + len(a.tri_list) - \
        int((a.edge_list["ro_rank"] == 0).sum() + (a.edge_list["nu_max_rank"] == 0).sum())
