"""GPU parity tests of the Delaunay triangulation (gpudtComputeDT contract).

Every case runs the CUDA library through its C ABI and compares with the CPU
oracle on the same seeded inputs: identical canonical triangle sets where the
DT is unique, the exact checkResult invariants (main.cu:163-343) plus the same
triangle count, vertex set and hull where it is not (cocircular input).
"""
import os

import numpy as np
import pytest

import galpha_b200 as G
from alphacheck import compare_alpha
from galpha_b200 import datasets as D
from dtcheck import canon_set, compare_dt
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run(engine, pts, fbo, **kw):
    return engine.triangulate(G.GPUDTParams(pts, fboSize=fbo, **kw))


def assert_parity(pts, dt, must_be_identical):
    ok, rep = compare_dt(pts, dt.vtx, dt.tri)
    assert ok, rep
    if must_be_identical:
        assert rep["identical"], rep


def test_config_c1_identical(engine):
    pts, fbo = D.make("c1")
    dt = run(engine, pts, fbo)
    assert_parity(pts, dt, True)
    g = np.load(os.path.join(GOLD, "golden_c1.npz"))
    assert dt.nTris == len(g["triangles"])


@pytest.mark.parametrize("name,fbo", [("bird", 512), ("alpha", 512), ("1000_1", 2048), ("10000_1", 2048)])
def test_reference_fixtures(engine, name, fbo):
    g = np.load(os.path.join(GOLD, "golden_ref_%s.npz" % name))
    pts = g["points"]
    dt = run(engine, pts, fbo)
    # the reference's integer-coordinate fixtures have cocircular quads
    assert_parity(pts, dt, False)
    assert dt.nTris == len(g["triangles"])


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("fbo", [256, 1024])
def test_uniform_random(engine, seed, fbo):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(10, 20000))
    pts = rng.random((n, 2))
    assert_parity(pts, run(engine, pts, fbo), True)


@pytest.mark.parametrize("seed", range(4))
def test_gaussian_and_clusters(engine, seed):
    rng = np.random.default_rng(200 + seed)
    n = 5000
    g = rng.normal(0, 1, (n, 2))
    assert_parity(g, run(engine, g, 512), True)
    c = rng.random((8, 2))
    cl = c[rng.integers(0, 8, n)] + rng.normal(0, 0.002, (n, 2))
    assert_parity(cl, run(engine, cl, 1024), True)


@pytest.mark.parametrize("seed", range(4))
def test_degenerate_mix(engine, seed):
    pts = D.degenerate_mix(20000, 50 + seed)
    dt = run(engine, pts, 2048)
    assert_parity(pts, dt, False)
    assert dt.status.nDuplicates > 0


def test_duplicates_keep_lowest_index(engine):
    rng = np.random.default_rng(5)
    base = rng.random((500, 2))
    pts = np.concatenate([base, base[::-1]])  # index i and 999-i coincide
    dt = run(engine, pts, 512)
    assert_parity(pts, dt, True)
    used = np.unique(dt.vtx)
    assert used.max() < 500


def test_lattice_cocircular(engine):
    g = np.stack(np.meshgrid(np.arange(64), np.arange(64)), -1).reshape(-1, 2) / 64.0
    dt = run(engine, g, 1024)
    assert_parity(g, dt, False)
    assert dt.nTris == 2 * 63 * 63


@pytest.mark.parametrize("pts,ntri", [
    ([[0, 0], [1, 0], [0, 1]], 1),
    ([[0, 0], [1, 0], [0, 1], [1, 1.2]], 2),
    ([[0, 0], [1, 1]], 0),
    ([[0, 0], [1, 1], [2, 2], [3, 3]], 0),
    ([[0.5, 0.5]] * 6, 0),
])
def test_tiny_and_degenerate(engine, pts, ntri):
    pts = np.asarray(pts, dtype=np.float64)
    dt = run(engine, pts, 256)
    assert dt.nTris == ntri
    if ntri:
        assert_parity(pts, dt, True)


def test_precheck_past_first_pass(engine):
    # the input precheck stops once a distinct point (then an off-line point)
    # is found; these sets put the answer, or no answer, beyond the first
    # pass of its grid (148 SMs x 8 blocks x 256 threads = 303,104 points)
    n = 400000
    t = np.arange(n, dtype=np.float64) / (1 << 19)
    line = np.stack([t, 0.25 + 0.5 * t], 1)               # collinear, exactly representable
    assert run(engine, line, 2048).nTris == 0
    dup = np.full((n, 2), 0.375)
    dup[-1] = (0.625, 0.125)                                # two distinct points, the second last
    assert run(engine, dup, 2048).nTris == 0
    rng = np.random.default_rng(21)
    late = np.concatenate([np.full((320000, 2), 0.5), rng.random((2000, 2))])
    dt = run(engine, late, 2048)
    assert_parity(late, dt, True)
    assert dt.status.nDuplicates == 320000 - 1


def test_deterministic_and_reusable(engine):
    rng = np.random.default_rng(9)
    a = rng.random((30000, 2))
    b = rng.random((700, 2))
    d1 = run(engine, a, 2048)
    d2 = run(engine, b, 256)
    d3 = run(engine, a, 2048)
    # the triangle set is deterministic; the slot order, like the reference's,
    # depends on the order of concurrent work-list appends
    assert canon_set(d1.vtx) == canon_set(d3.vtx)
    assert_parity(b, d2, True)


def test_errors(engine):
    pts = np.random.default_rng(1).random((100, 2))
    with pytest.raises(G.GpudtError) as e:
        run(engine, pts, 300)          # not a power of two
    assert e.value.code == -1
    bad = pts.copy()
    bad[3, 0] = np.nan
    with pytest.raises(G.GpudtError) as e:
        run(engine, bad, 512)
    assert e.value.code == -1
    with pytest.raises(G.GpudtError) as e:  # caller bounds that do not hold the points
        run(engine, pts, 512, minX=0.2)
    assert e.value.code == -1
    with pytest.raises(G.GpudtError) as e:
        G.Engine(budget_bytes=1 << 20).triangulate(G.GPUDTParams(pts, fboSize=512))
    assert e.value.code == -3
    # the engine stays usable after errors
    assert_parity(pts, run(engine, pts, 512), True)


def test_reference_entry_point_symbols():
    L = G.load()
    for sym in ["_Z14gpudtComputeDTP11GPUDTPARAMS", "_Z20gpudtReleaseDTOutputP11GPUDTOUTPUT", "gpudtComputeDTEx"]:
        assert hasattr(L, sym)
    out = G.gpudt_compute_dt(G.GPUDTParams(np.random.default_rng(2).random((300, 2)), fboSize=512))
    assert out.nTris > 0


def test_large_uniform_properties(engine):
    """c2 size (4M points, texture 8192): exact validity of the full mesh."""
    pts, fbo = D.make("c2")
    dt = run(engine, pts, fbo)
    chk = O.check_mesh(pts, dt.vtx, dt.tri)
    assert chk["links"] == 0 and chk["ccw"] == 0 and chk["delaunay"] == 0 and chk["bad_index"] == 0, chk
    n = len(np.unique(dt.vtx))
    assert n == len(pts)
    assert dt.nTris == 2 * n - 2 - chk["hull_edges"]


def test_c3_degenerate_properties(engine):
    """c3 size (16.7M points: Gaussian blobs, uniform, lattice-snapped
    duplicates and cocircular quads; texture 8192, about 7.5M sites inserted
    after the Voronoi stage): exact validity of the full mesh, exactly the
    lowest input index of each group of exact duplicates as vertex, the Euler
    count, the predicate stage counts, and a spectrum that increases strictly
    with every rank in range."""
    pts, fbo = D.make("c3")
    dt = run(engine, pts, fbo)
    chk = O.check_mesh(pts, dt.vtx, dt.tri)
    assert chk["links"] == 0 and chk["ccw"] == 0 and chk["delaunay"] == 0 and chk["bad_index"] == 0, chk
    verts = np.unique(dt.vtx)
    _, first = np.unique(pts, axis=0, return_index=True)
    assert np.array_equal(verts, np.sort(first))
    assert dt.nTris == 2 * len(verts) - 2 - chk["hull_edges"]
    # predicate stages: the FP32 filter decides nearly every test; the exact
    # lattice degeneracies (collinear rows, cocircular quads) reach the later stages
    st = dt.status
    for tests, f64, ex in ((st.incircleTests, st.filteredIncircle, st.exactIncircle),
                           (st.orientTests, st.filteredOrient, st.exactOrient)):
        assert tests > 10 ** 7 and 0 < f64 and 0 < ex and f64 + ex < 0.05 * tests
    a = engine.alpha_resident()
    s = a["spectrum"]
    assert s[0] == 0.0 and np.all(np.diff(s[1:]) > 0)
    ro = a["tri_list"]["ro_rank"]
    assert ro.min() >= 1 and ro.max() < len(s)
    assert a["edge_list"]["ro_rank"].max() < len(s)
    # the full alpha result against the CPU oracle on the same triangles
    # (about 100 s on one core): ranks and intervals identical, values within
    # 4 ulp of the exactly rounded FP64 value
    ok, rep = compare_alpha(pts, dt.vtx, dt.tri, a, 4)
    assert ok, rep
    print("c3 alpha vs oracle: %r" % rep)


def test_voronoi_paths(engine):
    """Each discrete-Voronoi path: fused (dense), fused + local island repair,
    escalation to the global island path (sparse Gaussian tails), and the
    envelope path for sparse input (mean spacing above 16 pixels)."""
    rng = np.random.default_rng(5)
    _ = rng.random((20000, 2))
    cases = [
        (rng.random((60000, 2)), 1024),         # dense: island tiles repaired locally
        (rng.normal(0, 1, (1970, 2)), 512),     # large islands in the tails
        (rng.random((300, 2)), 2048),           # sparse: envelope path
        (D.degenerate_mix(200000, 7), 2048),    # duplicates, lattice ties, clusters
    ]
    for pts, fbo in cases:
        dt = run(engine, pts, fbo)
        assert_parity(pts, dt, False)


def test_c1_through_reference_symbol_matches_handle(engine):
    pts, fbo = D.make("c1")
    a = G.gpudt_compute_dt(G.GPUDTParams(pts, fboSize=fbo))
    b = run(engine, pts, fbo)
    assert canon_set(a.vtx) == canon_set(b.vtx)


@pytest.mark.parametrize("flags", [0, 4, 1 | 4, 2 | 4])
def test_run_device_flags(engine, flags):
    """galphaRunDevice on device-resident points: the gpudtTriangle records
    (built inside the call with GALPHA_RUN_TRIANGLES = 4, else on the copy)
    equal the oracle's triangulation."""
    import torch

    pts = D.uniform_points(50000, 77)
    d = torch.from_numpy(pts).cuda()
    engine.run_device_flags(d.data_ptr(), len(pts), (0.0, 0.0, 1.0, 1.0), 1024, flags)
    tri = engine.resident_triangles()
    vtx = tri["vtx"].reshape(-1, 3)
    assert canon_set(vtx) == canon_set(O.dt(pts)[0])
    ok, rep = compare_dt(pts, vtx, tri["tri"].reshape(-1, 3))
    assert ok and rep["identical"], rep


@pytest.mark.parametrize("sched", [(1, 1, 1, 0, 1), (8, 4, 16, 16384, 131072), (2, 8, 64, 1 << 20, 1 << 22)])
def test_schedule_changes_no_result(engine, sched):
    """galphaSetSchedule moves only the counter reads: every schedule gives
    the oracle's triangulation and the same alpha result."""
    pts = D.uniform_points(60000, 91)
    base = engine.triangulate(G.GPUDTParams(pts, fboSize=1024))
    a0 = engine.alpha_resident()
    try:
        engine.set_schedule(*sched)
        dt = engine.triangulate(G.GPUDTParams(pts, fboSize=1024))
        a1 = engine.alpha_resident()
        assert engine.schedule()["flip_sync"] == sched[2]
    finally:
        engine.set_schedule()
    assert canon_set(dt.vtx) == canon_set(base.vtx) == canon_set(O.dt(pts)[0])
    np.testing.assert_array_equal(a1["spectrum"], a0["spectrum"])
    assert dt.status.hostReads != base.status.hostReads or sched[2] == 4


def test_schedule_rejects_out_of_range(engine):
    for bad in [(9, 0, 0, -1, 0), (0, 0, 65, -1, 0), (0, 0, 0, 5000, 4096)]:
        with pytest.raises(G.GpudtError):
            engine.set_schedule(*bad)
    assert engine.schedule() == dict(shift_group=4, missing_group=2, flip_sync=4, flip_tail_enter=4096,
                                     flip_tail_leave=32768)
