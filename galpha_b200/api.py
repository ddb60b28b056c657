"""Python mirror of the reference's DT + alpha-shape interface over libgalpha's C ABI.

Reference interface                               here
------------------------------------------------  --------------------------------------------
``GPUDTPARAMS`` / ``GPUDTOUTPUT`` (gpudt.h:105-128)  :class:`GPUDTParams`, :class:`DTOutput`
``gpudtComputeDT`` (gpudt.h:131)                    :func:`gpudt_compute_dt`
``gpudtReleaseDTOutput`` (gpudt.h:132)              (automatic: arrays are copied out)
``Alpha_Shapes_2D(pInput, pDT)``,                   :class:`AlphaShapes2D` with
``computeAlphaShapes()`` and the public /           ``compute_alpha_shapes()``, ``spectrum``,
friend members (Alpha_Shapes_2D.h:43-121)            ``point_list``, ``edge_list``, ``tri_list``
``ReadDataFromFileBinary`` (main.cu:117-161)        :func:`read_points_file`

Errors raise :class:`GpudtError` with the C status code instead of exiting the
process as the reference does (common.h:55-93).  Every call goes to the CUDA
library; when it is missing or no sm_100 device is present the calls raise --
there is no CPU path.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(_HERE, "lib", "libgalpha.so")

STATUS_TEXT = {
    0: "ok",
    -1: "bad argument",
    -2: "CUDA error",
    -3: "out of memory / budget",
    -4: "mesh topology invariant violated",
    -5: "iteration cap reached",
    -6: "exact arithmetic scratch overflow",
    -7: "no sm_100 device",
}


class GpudtError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        msg = "%s failed: %d (%s)" % (where, code, STATUS_TEXT.get(code, "?"))
        extra = _last_error()
        if extra:
            msg += " -- " + extra
        super().__init__(msg)


class _Vertex(ctypes.Structure):
    _fields_ = [("x", ctypes.c_double), ("y", ctypes.c_double)]


class _Params(ctypes.Structure):
    _fields_ = [
        ("minX", ctypes.c_double), ("minY", ctypes.c_double),
        ("maxX", ctypes.c_double), ("maxY", ctypes.c_double),
        ("nPoints", ctypes.c_int), ("points", ctypes.c_void_p),
        ("nConstraints", ctypes.c_int), ("constraints", ctypes.c_void_p),
        ("fboSize", ctypes.c_int),
    ]


class _Output(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_void_p), ("nTris", ctypes.c_int)]


class Status(ctypes.Structure):
    """gpudtStatus: per-call statistics of the triangulation."""
    _fields_ = [
        ("status", ctypes.c_int), ("nVerts", ctypes.c_int), ("nFake", ctypes.c_int),
        ("nDuplicates", ctypes.c_int), ("nMissing", ctypes.c_int), ("nBadShift", ctypes.c_int),
        ("nIslandPixels", ctypes.c_int), ("nFlips", ctypes.c_int), ("flipRounds", ctypes.c_int),
        ("shiftRounds", ctypes.c_int), ("missingRounds", ctypes.c_int),
        ("nRepairTiles", ctypes.c_int), ("nEscalated", ctypes.c_int), ("nEnvelopeCells", ctypes.c_int),
        ("exactOrient", ctypes.c_longlong), ("exactIncircle", ctypes.c_longlong),
        ("filteredIncircle", ctypes.c_longlong), ("incircleTests", ctypes.c_longlong),
        ("orientTests", ctypes.c_longlong), ("filteredOrient", ctypes.c_longlong),
        ("ms", ctypes.c_float * 12),
        ("kernelMs", ctypes.c_float * 4),
        ("sortKeys", ctypes.c_longlong), ("sortPasses", ctypes.c_int), ("hostReads", ctypes.c_int),
        ("constraintRounds", ctypes.c_int), ("reserved0", ctypes.c_int),
        ("hostReadsStage", ctypes.c_int * 12),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("ms", "kernelMs", "hostReadsStage")}
        d["ms"] = list(self.ms)
        d["kernelMs"] = list(self.kernelMs)
        d["hostReadsStage"] = list(self.hostReadsStage)
        return d


class _AlphaOut(ctypes.Structure):
    _fields_ = [
        ("nSpectrum", ctypes.c_int), ("spectrum", ctypes.c_void_p),
        ("nPoints", ctypes.c_int), ("point_list", ctypes.c_void_p),
        ("nEdges", ctypes.c_int), ("edge_list", ctypes.c_void_p),
        ("nTris", ctypes.c_int), ("tri_list", ctypes.c_void_p),
        ("exactCompares", ctypes.c_longlong), ("exactTies", ctypes.c_longlong),
        ("exactAttached", ctypes.c_longlong),
    ]


# numpy views of the C element layouts (gpudt.h:97-102, headers.h:48-64)
TRIANGLE_DTYPE = np.dtype([("tri", np.int32, 3), ("vtx", np.int32, 3), ("tmp", np.int32, 3)])
POINT_INTERVAL_DTYPE = np.dtype([("nu_min_rank", np.int32), ("nu_max_rank", np.int32)])
EDGE_INTERVAL_DTYPE = np.dtype([
    ("ro_rank", np.int32), ("nu_min_rank", np.int32), ("nu_max_rank", np.int32),
    ("sc", np.int32), ("tIndex", np.int32), ("vOpp", np.int32),
])
TRIANGLE_INTERVAL_DTYPE = np.dtype([("ro_rank", np.int32)])

ALPHA_DTYPE = np.dtype([("simplex_index", np.int32), ("st", np.int32), ("at", np.int32)])


class _MasterOut(ctypes.Structure):
    _fields_ = [("nMaster", ctypes.c_int), ("master_list", ctypes.c_void_p), ("nSpecPointers", ctypes.c_int),
                ("spec_pointers", ctypes.c_void_p)]


class BatchSet(ctypes.Structure):
    """galphaBatchSet: counts and bases of one set of a batch."""
    _fields_ = [("nPoints", ctypes.c_int), ("pointBase", ctypes.c_int), ("nTris", ctypes.c_int),
                ("triBase", ctypes.c_int), ("nEdges", ctypes.c_int), ("edgeBase", ctypes.c_int),
                ("nSpectrum", ctypes.c_int), ("specBase", ctypes.c_int)]


# alpha-complex classes (galpha.h GALPHA_*)
EXTERIOR, SINGULAR, REGULAR, INTERIOR = 0, 1, 2, 3


class QueryResult(ctypes.Structure):
    """galphaQueryResult: counts per class (indexed by EXTERIOR..INTERIOR)."""
    _fields_ = [("alpha", ctypes.c_double), ("rank", ctypes.c_int), ("nPoints", ctypes.c_int * 4),
                ("nEdges", ctypes.c_int * 4), ("nTris", ctypes.c_int * 4)]

    def as_dict(self):
        return {"alpha": self.alpha, "rank": self.rank, "nPoints": list(self.nPoints),
                "nEdges": list(self.nEdges), "nTris": list(self.nTris)}

_lib = None
_lib_path = None


def load(path=None):
    """Load libgalpha (default: the in-tree galpha_b200/lib/libgalpha.so)."""
    global _lib, _lib_path
    path = path or DEFAULT_LIB
    if _lib is not None and _lib_path == path:
        return _lib
    if not os.path.exists(path):
        raise OSError("libgalpha not built: %s (run galpha_b200.build.build())" % path)
    L = ctypes.CDLL(path)
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.galphaCreate.argtypes = [ip, ctypes.c_longlong, ctypes.POINTER(vp)]
    L.galphaDestroy.argtypes = [vp]
    L.galphaSetStream.argtypes = [vp, vp]
    L.galphaTriangulate.argtypes = [vp, ctypes.POINTER(_Params), ctypes.POINTER(_Output), ctypes.POINTER(Status)]
    L.galphaComputeResident.argtypes = [vp, ctypes.POINTER(_AlphaOut)]
    L.galphaCompute.argtypes = [vp, ctypes.POINTER(_Params), ctypes.POINTER(_Output), ctypes.POINTER(_AlphaOut)]
    L.galphaComputeAll.argtypes = [vp, ctypes.POINTER(_Params), ctypes.POINTER(_Output), ctypes.POINTER(_AlphaOut),
                                   ctypes.POINTER(Status)]
    L.galphaRunDevice.argtypes = [vp, vp, ip, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ip, ip, ctypes.POINTER(Status)]
    L.galphaGetCounts.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]
    L.galphaCopyTriangles.argtypes = [vp, vp, ip]
    L.galphaReleaseOutput.argtypes = [ctypes.POINTER(_AlphaOut)]
    L.galphaQuery.argtypes = [vp, ctypes.c_double, ctypes.POINTER(QueryResult)]
    L.galphaQueryQuantile.argtypes = [vp, ctypes.c_double, ctypes.POINTER(QueryResult)]
    L.galphaCopyClasses.argtypes = [vp, vp, vp, vp]
    L.galphaRunBatch.argtypes = [vp, ip, vp, vp, vp, ip, ctypes.POINTER(Status)]
    L.galphaRunBatchHost.argtypes = [vp, ip, vp, vp, vp, ip, ctypes.POINTER(Status)]
    L.galphaBatchSets.argtypes = [vp, vp]
    L.galphaSetBatchDensity.argtypes = [vp, ctypes.c_double]
    L.galphaSetSchedule.argtypes = [vp, ip, ip, ip, ip, ip]
    L.galphaGetSchedule.argtypes = [vp, ctypes.POINTER(ip)]
    L.galphaBatchCopy.argtypes = [vp, vp, vp, vp, vp, vp]
    L.galphaBatchQuery.argtypes = [vp, vp, ip, vp]
    L.galphaMasterList.argtypes = [vp, ctypes.POINTER(_MasterOut)]
    L.galphaReleaseMasterList.argtypes = [ctypes.POINTER(_MasterOut)]
    L.galphaLastError.restype = ctypes.c_char_p
    L.galphaVersion.restype = ctypes.c_char_p
    L.galphaLaunchCount.restype = ctypes.c_ulonglong
    L.gpudtComputeDTEx.argtypes = [ctypes.POINTER(_Params), ctypes.POINTER(_Output), ctypes.POINTER(Status)]
    L.gpudt_release_dt_output.argtypes = [ctypes.POINTER(_Output)]
    _lib, _lib_path = L, path
    return L


def _last_error():
    if _lib is None:
        return ""
    s = _lib.galphaLastError()
    return s.decode() if s else ""


def _check(code, where):
    if code != 0:
        raise GpudtError(code, where)


class GPUDTParams:
    """GPUDTPARAMS (gpudt.h:105-118).  points: (N, 2) float64."""

    def __init__(self, points, fboSize=2048, minX=None, minY=None, maxX=None, maxY=None, constraints=None):
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
        self.points = pts
        self.nPoints = pts.shape[0]
        self.fboSize = int(fboSize)
        lo = pts.min(axis=0) if len(pts) else np.zeros(2)
        hi = pts.max(axis=0) if len(pts) else np.ones(2)
        self.minX = float(lo[0] if minX is None else minX)
        self.minY = float(lo[1] if minY is None else minY)
        self.maxX = float(hi[0] if maxX is None else maxX)
        self.maxY = float(hi[1] if maxY is None else maxY)
        # constrained edges: (M, 2) point indices (gpudt.h: two per constraint)
        self.constraints = None if constraints is None else np.ascontiguousarray(constraints, dtype=np.int32).reshape(-1, 2)
        self.nConstraints = 0 if constraints is None else self.constraints.shape[0]

    def _c(self):
        p = _Params()
        p.minX, p.minY, p.maxX, p.maxY = self.minX, self.minY, self.maxX, self.maxY
        p.nPoints = self.nPoints
        p.points = self.points.ctypes.data if self.nPoints else None
        p.nConstraints = self.nConstraints
        p.constraints = self.constraints.ctypes.data if self.nConstraints else None
        p.fboSize = self.fboSize
        return p


class DTOutput:
    """GPUDTOUTPUT (gpudt.h:124-128): ``triangles`` is a TRIANGLE_DTYPE array."""

    def __init__(self, triangles, status=None):
        self.triangles = triangles
        self.nTris = len(triangles)
        self.status = status

    @property
    def vtx(self):
        return self.triangles["vtx"]

    @property
    def tri(self):
        return self.triangles["tri"]


class _HostPool:
    """Reused host output buffers, pinned when torch is available (one DMA copy
    per result instead of a pageable copy)."""

    def __init__(self):
        self._bufs = {}
        self._keep = {}
        try:
            import torch

            self._torch = torch if torch.cuda.is_available() else None
        except Exception:
            self._torch = None

    def get(self, name, n, dtype):
        dtype = np.dtype(dtype)
        a = self._bufs.get(name)
        if a is None or len(a) < n or a.dtype != dtype:
            if a is not None and a.dtype == dtype:
                n = max(int(n), int(1.5 * len(a)))  # grow geometrically: pinning is slow
            nbytes = max(1, int(n) * dtype.itemsize)
            if self._torch is not None:
                t = self._torch.empty(nbytes, dtype=self._torch.uint8, pin_memory=True)
                self._keep[name] = t
                a = t.numpy().view(dtype)[: max(1, int(n))]
            else:
                a = np.empty(max(1, int(n)), dtype=dtype)
            self._bufs[name] = a
        return a


_stage_pool = None


def _stage(out, arrays, sizes):
    """Concatenates point arrays into `out` (a pinned staging buffer); large
    batches are copied by several threads (NumPy releases the GIL for the
    copies)."""
    global _stage_pool
    n = int(sizes.sum())
    if n < (1 << 20) or len(arrays) < 2:
        np.concatenate(arrays, out=out)
        return
    if _stage_pool is None:
        from concurrent.futures import ThreadPoolExecutor

        _stage_pool = ThreadPoolExecutor(max(2, min(8, os.cpu_count() or 2)))
    offs = np.concatenate([[0], np.cumsum(sizes)])

    def copy(k):
        out[offs[k]:offs[k + 1]] = arrays[k]

    list(_stage_pool.map(copy, range(len(arrays))))


class Engine:
    """A libgalpha handle: one CUDA stream and one device arena, reused across calls."""

    def __init__(self, device=-1, budget_bytes=0, lib=None):
        self._L = load(lib)
        h = ctypes.c_void_p()
        _check(self._L.galphaCreate(device, budget_bytes, ctypes.byref(h)), "galphaCreate")
        self._h = h
        self._pool = _HostPool()
        self._npoints = 0

    def close(self):
        if getattr(self, "_h", None):
            self._L.galphaDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def triangulate(self, params, copy=True):
        """Delaunay triangulation of params (gpudtComputeDT semantics).

        With copy=False the triangle array is a view of a reused pinned buffer,
        valid until the next call on this engine."""
        self._batch_active = False
        cp = params._c()
        cap = 2 * params.nPoints + 64
        buf = self._pool.get("tri", cap, TRIANGLE_DTYPE)
        out = _Output()
        out.triangles = buf.ctypes.data
        out.nTris = len(buf)
        st = Status()
        _check(self._L.galphaTriangulate(self._h, ctypes.byref(cp), ctypes.byref(out), ctypes.byref(st)),
               "galphaTriangulate")
        self._npoints = params.nPoints
        arr = buf[: out.nTris]
        return DTOutput(arr.copy() if copy else arr, st)

    def _alpha_bufs(self, n, nt):
        ne = 3 * max(n, 1) + 8
        out = _AlphaOut()
        sp = self._pool.get("spec", 1 + nt + ne, np.float64)
        pt = self._pool.get("pt", max(n, 1), POINT_INTERVAL_DTYPE)
        ed = self._pool.get("edge", ne, EDGE_INTERVAL_DTYPE)
        tr = self._pool.get("trilist", max(nt, 1), TRIANGLE_INTERVAL_DTYPE)
        out.spectrum, out.nSpectrum = sp.ctypes.data, len(sp)
        out.point_list, out.nPoints = pt.ctypes.data, len(pt)
        out.edge_list, out.nEdges = ed.ctypes.data, len(ed)
        out.tri_list, out.nTris = tr.ctypes.data, len(tr)
        return out, (sp, pt, ed, tr)

    def _alpha_result(self, out, bufs, copy):
        sp, pt, ed, tr = bufs
        res = {
            "spectrum": sp[: out.nSpectrum], "point_list": pt[: out.nPoints],
            "edge_list": ed[: out.nEdges], "tri_list": tr[: out.nTris],
        }
        if copy:
            res = {k: v.copy() for k, v in res.items()}
        res.update(exactCompares=out.exactCompares, exactTies=out.exactTies, exactAttached=out.exactAttached)
        return res

    def alpha_resident(self, copy=True):
        """Alpha spectrum + intervals of the mesh left on the device by triangulate()."""
        nt = self.counts()[0]
        out, bufs = self._alpha_bufs(self._npoints, nt)
        _check(self._L.galphaComputeResident(self._h, ctypes.byref(out)), "galphaComputeResident")
        return self._alpha_result(out, bufs, copy)

    def compute_all(self, params, copy=True):
        """DT + alpha spectrum of params in one call (galphaComputeAll): returns
        (DTOutput, alpha result dict).  The triangles are downloaded while the
        alpha stage runs.  With copy=False the arrays are views of reused pinned
        buffers, valid until the next call on this engine."""
        self._batch_active = False
        cp = params._c()
        n = params.nPoints
        buf = self._pool.get("tri", 2 * n + 64, TRIANGLE_DTYPE)
        o = _Output()
        o.triangles = buf.ctypes.data
        o.nTris = len(buf)
        out, bufs = self._alpha_bufs(n, len(buf))
        st = Status()
        _check(self._L.galphaComputeAll(self._h, ctypes.byref(cp), ctypes.byref(o), ctypes.byref(out),
                                        ctypes.byref(st)), "galphaComputeAll")
        self._npoints = n
        arr = buf[: o.nTris]
        return DTOutput(arr.copy() if copy else arr, st), self._alpha_result(out, bufs, copy)

    def alpha_of(self, params, dt, copy=True):
        """Alpha spectrum + intervals of a given triangulation (Alpha_Shapes_2D(pInput, pDT))."""
        self._batch_active = False
        cp = params._c()
        tri = np.ascontiguousarray(dt.triangles)
        o = _Output()
        o.triangles = tri.ctypes.data if len(tri) else None
        o.nTris = len(tri)
        out, bufs = self._alpha_bufs(params.nPoints, len(tri))
        self._npoints = params.nPoints
        _check(self._L.galphaCompute(self._h, ctypes.byref(cp), ctypes.byref(o), ctypes.byref(out)),
               "galphaCompute")
        return self._alpha_result(out, bufs, copy)

    def run_device(self, d_xy_ptr, n, bounds, fbo_size, with_alpha=True, triangles=False):
        """Hot path on device-resident points (d_xy_ptr: device address of 2n doubles).
        ``triangles``: also build the gpudtTriangle records on the device."""
        return self.run_device_flags(d_xy_ptr, n, bounds, fbo_size, (1 if with_alpha else 0) | (4 if triangles else 0))

    def resident_triangles(self):
        """The resident triangles as a TRIANGLE_DTYPE array (galphaCopyTriangles)."""
        nt, _, _ = self.counts()
        out = np.empty(nt, TRIANGLE_DTYPE)
        _check(self._L.galphaCopyTriangles(self._h, out.ctypes.data if nt else None, nt), "galphaCopyTriangles")
        return out

    def run_device_flags(self, d_xy_ptr, n, bounds, fbo_size, flags):
        """galphaRunDevice with its flag word: flags & 3 = 0 (DT only), 1 (+ alpha),
        2 (+ alpha + master list); flags & 4: build the gpudtTriangle records."""
        self._batch_active = False
        st = Status()
        _check(self._L.galphaRunDevice(self._h, ctypes.c_void_p(d_xy_ptr), n, bounds[0], bounds[1], bounds[2],
                                       bounds[3], fbo_size, flags, ctypes.byref(st)),
               "galphaRunDevice")
        self._npoints = n
        return st

    def query(self, alpha=None, quantile=None):
        """Alpha-complex query on the resident result: classify every simplex at
        ``alpha`` (a squared radius) or at the spectrum quantile ``quantile``."""
        res = QueryResult()
        if quantile is not None:
            _check(self._L.galphaQueryQuantile(self._h, float(quantile), ctypes.byref(res)), "galphaQueryQuantile")
        else:
            _check(self._L.galphaQuery(self._h, float(alpha), ctypes.byref(res)), "galphaQuery")
        return res

    # ---------------------------------------------------------------- batches
    @staticmethod
    def batch_bounds(sets):
        """Per-set (minX, minY, maxX, maxY) from the data, as GPUDTPARAMS would hold."""
        b = np.zeros((len(sets), 4))
        for k, p in enumerate(sets):
            p = np.asarray(p, dtype=np.float64).reshape(-1, 2)
            if len(p):
                x, y = p[:, 0], p[:, 1]  # column reductions: several times faster than axis=0
                b[k] = (x.min(), y.min(), x.max(), y.max())
            else:
                b[k] = (0.0, 0.0, 1.0, 1.0)
        return b

    def run_batch(self, sets, bounds=None, with_alpha=True):
        """DT (+ alpha) of many independent point sets in one pipeline run
        (galphaRunBatchHost).  sets: list of (n_k, 2) arrays."""
        sizes = np.array([len(p) for p in sets], dtype=np.int32)
        n = int(sizes.sum())
        # staged in a reused pinned buffer: one DMA copy to the device
        xy = self._pool.get("batch_xy", 2 * n, np.float64)[: 2 * n].reshape(-1, 2)
        if n:
            _stage(xy, [np.asarray(p, dtype=np.float64).reshape(-1, 2) for p in sets], sizes)
        b = np.ascontiguousarray(self.batch_bounds(sets) if bounds is None else bounds, dtype=np.float64)
        st = Status()
        _check(self._L.galphaRunBatchHost(self._h, len(sets), sizes.ctypes.data, xy.ctypes.data if len(xy) else None,
                                          b.ctypes.data, 1 if with_alpha else 0, ctypes.byref(st)),
               "galphaRunBatchHost")
        self._batch = (len(sets), bool(with_alpha))
        self._batch_active = True
        return st

    def run_batch_device(self, d_xy_ptr, sizes, bounds, with_alpha=True):
        """The same on points already in device memory (galphaRunBatch)."""
        sizes = np.ascontiguousarray(sizes, dtype=np.int32)
        b = np.ascontiguousarray(bounds, dtype=np.float64)
        st = Status()
        _check(self._L.galphaRunBatch(self._h, len(sizes), sizes.ctypes.data, ctypes.c_void_p(d_xy_ptr),
                                      b.ctypes.data, 1 if with_alpha else 0, ctypes.byref(st)), "galphaRunBatch")
        self._batch = (len(sizes), bool(with_alpha))
        self._batch_active = True
        return st

    def set_batch_density(self, pixels_per_point):
        """Texture pixels per point of every set in later batches
        (galphaSetBatchDensity; default 10, tuned by galpha_b200.autotune)."""
        _check(self._L.galphaSetBatchDensity(self._h, float(pixels_per_point)), "galphaSetBatchDensity")
        self._density = float(pixels_per_point)

    SCHEDULE_KEYS = ("shift_group", "missing_group", "flip_sync", "flip_tail_enter", "flip_tail_leave")

    def set_schedule(self, shift_group=0, missing_group=0, flip_sync=0, flip_tail_enter=-1, flip_tail_leave=0):
        """Loop schedule of later calls (galphaSetSchedule): rounds per counter
        read of the shifting, missing-site and flip loops, and the flip-tail
        hand-over lengths.  No value changes a result; 0 (-1 for
        flip_tail_enter) keeps the default.  Tuned by galpha_b200.autotune."""
        _check(self._L.galphaSetSchedule(self._h, int(shift_group), int(missing_group), int(flip_sync),
                                         int(flip_tail_enter), int(flip_tail_leave)), "galphaSetSchedule")

    def schedule(self):
        """The schedule in force, as a dict (galphaGetSchedule)."""
        out = (ctypes.c_int * 5)()
        _check(self._L.galphaGetSchedule(self._h, out), "galphaGetSchedule")
        return dict(zip(self.SCHEDULE_KEYS, list(out)))

    def batch_sets(self):
        k = self._batch[0]
        arr = (BatchSet * k)()
        _check(self._L.galphaBatchSets(self._h, arr), "galphaBatchSets")
        return arr

    def batch_results(self, copy=True):
        """Per-set results of the last batch: list of dicts with ``triangles``
        (TRIANGLE_DTYPE, set-local indices) and, with alpha, ``spectrum``,
        ``point_list``, ``edge_list``, ``tri_list``.  With copy=False the arrays
        are views of reused pinned buffers (one DMA copy each), valid until the
        next batch_results call on this engine."""
        k, alpha = self._batch
        sets = self.batch_sets()
        nt = sum(s.nTris for s in sets)
        npt = sum(s.nPoints for s in sets)
        ne = sum(s.nEdges for s in sets)
        nsp = sum(s.nSpectrum for s in sets)
        if copy:
            new = lambda name, m, dt: np.empty(m, dt)
        else:
            new = lambda name, m, dt: self._pool.get(name, m, dt)[:m]
        tri = new("b_tri", nt, TRIANGLE_DTYPE)
        pt = new("b_pt", npt, POINT_INTERVAL_DTYPE) if alpha else None
        ed = new("b_edge", ne, EDGE_INTERVAL_DTYPE) if alpha else None
        tr = new("b_trilist", nt, TRIANGLE_INTERVAL_DTYPE) if alpha else None
        sp = new("b_spec", nsp, np.float64) if alpha else None
        ptr = lambda a: a.ctypes.data if a is not None and len(a) else None
        _check(self._L.galphaBatchCopy(self._h, ptr(tri), ptr(pt), ptr(ed), ptr(tr), ptr(sp)), "galphaBatchCopy")
        out = []
        for s in sets:
            d = {"triangles": tri[s.triBase:s.triBase + s.nTris]}
            if alpha:
                d.update(spectrum=sp[s.specBase:s.specBase + s.nSpectrum],
                         point_list=pt[s.pointBase:s.pointBase + s.nPoints],
                         edge_list=ed[s.edgeBase:s.edgeBase + s.nEdges],
                         tri_list=tr[s.triBase:s.triBase + s.nTris])
            out.append(d)
        return out

    def batch_query(self, values, by_quantile=False):
        """Alpha-complex query on every set of the last batch (galphaBatchQuery):
        values[s] is set s's alpha (or spectrum quantile).  Returns QueryResults."""
        k = self._batch[0]
        vals = np.ascontiguousarray(np.broadcast_to(np.asarray(values, dtype=np.float64), (k,)))
        res = (QueryResult * k)()
        _check(self._L.galphaBatchQuery(self._h, vals.ctypes.data, 1 if by_quantile else 0, res), "galphaBatchQuery")
        return res

    def master_list(self):
        """master_list (ALPHA_DTYPE array) and spec_pointers of the resident alpha
        result (Alpha_Shapes_2D::compute_master_list)."""
        out = _MasterOut()
        _check(self._L.galphaMasterList(self._h, ctypes.byref(out)), "galphaMasterList")
        try:
            ml = np.empty(out.nMaster, ALPHA_DTYPE)
            sp = np.empty(out.nSpecPointers, np.int32)
            if out.nMaster:
                ctypes.memmove(ml.ctypes.data, out.master_list, ml.nbytes)
            if out.nSpecPointers:
                ctypes.memmove(sp.ctypes.data, out.spec_pointers, sp.nbytes)
        finally:
            self._L.galphaReleaseMasterList(ctypes.byref(out))
        return ml, sp

    def classes(self):
        """Classes of the last query: (points, edges, triangles) uint8 arrays."""
        nt, ne, _ = self.counts()
        npts = self._npoints
        if getattr(self, "_batch_active", False):
            npts = sum(s.nPoints for s in self.batch_sets())
        pt = np.empty(npts, np.uint8)
        ed = np.empty(ne, np.uint8)
        tr = np.empty(nt, np.uint8)
        _check(self._L.galphaCopyClasses(self._h, pt.ctypes.data if len(pt) else None,
                                         ed.ctypes.data if len(ed) else None,
                                         tr.ctypes.data if len(tr) else None), "galphaCopyClasses")
        return pt, ed, tr

    def counts(self):
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._L.galphaGetCounts(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return a.value, b.value, c.value

    def set_stream(self, stream_ptr):
        _check(self._L.galphaSetStream(self._h, ctypes.c_void_p(stream_ptr)), "galphaSetStream")


_default_engine = None


def _engine():
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine()
    return _default_engine


def gpudt_compute_dt(params):
    """gpudtComputeDT(pParam) (gpudt.h:131): returns a DTOutput."""
    return _engine().triangulate(params)


class AlphaShapes2D:
    """Alpha_Shapes_2D(pInput, pDT) + computeAlphaShapes() (Alpha_Shapes_2D.h:43-121).

    After compute_alpha_shapes(): ``spectrum`` (float64, [0] = 0 sentinel),
    ``point_list`` / ``edge_list`` / ``tri_list`` (structured arrays with the
    reference's field names), ``master_list`` (ALPHA_DTYPE) and
    ``spec_pointers``, ``alpha`` and ``alpha_index`` as in the reference.
    """

    def __init__(self, params, dt, engine=None):
        self.pInput = params
        self.pDT = dt
        self._engine = engine
        self.spectrum = None
        self.point_list = None
        self.edge_list = None
        self.tri_list = None
        self.master_list = None
        self.spec_pointers = None
        self.alpha = 0.0
        self.alpha_index = 0

    def compute_alpha_shapes(self):
        eng = self._engine or _engine()
        r = eng.alpha_of(self.pInput, self.pDT)
        self.spectrum = r["spectrum"]
        self.point_list = r["point_list"]
        self.edge_list = r["edge_list"]
        self.tri_list = r["tri_list"]
        self.stats = {k: r[k] for k in ("exactCompares", "exactTies", "exactAttached")}
        self.master_list, self.spec_pointers = eng.master_list()
        return self

    computeAlphaShapes = compute_alpha_shapes

    def set_alpha(self, index):
        """setAlpha (Alpha_Shapes_2D.cu): select the alpha value spectrum[index]."""
        self.alpha_index = int(index)
        self.alpha = float(self.spectrum[self.alpha_index]) if self.spectrum is not None else 0.0

    setAlpha = set_alpha


def read_points_file(path):
    """The reference's input format (main.cu:117-161): first line N, then 'index x y' lines."""
    with open(path) as f:
        n = int(f.readline().split()[0])
        pts = np.zeros((n, 2), dtype=np.float64)
        for _ in range(n):
            parts = f.readline().split()
            pts[int(parts[0])] = (float(parts[1]), float(parts[2]))
    return pts
