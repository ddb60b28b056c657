"""galpha-b200: B200-native 2D Delaunay triangulation and alpha shapes.

A drop-in for the GPU-DT + GAlpha path of the reference (gpudtComputeDT over
GPUDTPARAMS / GPUDTOUTPUT, and the Alpha_Shapes_2D interval output).  The
engine is libgalpha.so (CUDA, sm_100a, C ABI in include/gpudt.h and
include/galpha.h); this package is its Python host mirror.
"""
from .api import (  # noqa: F401
    ALPHA_DTYPE,
    AlphaShapes2D,
    DTOutput,
    Engine,
    GPUDTParams,
    GpudtError,
    Status,
    EDGE_INTERVAL_DTYPE,
    POINT_INTERVAL_DTYPE,
    TRIANGLE_DTYPE,
    TRIANGLE_INTERVAL_DTYPE,
    gpudt_compute_dt,
    load,
    read_points_file,
)

__version__ = "0.1.0"
