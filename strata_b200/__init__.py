"""strata_b200: the B200 (sm_100a) device backend of strata's raster-stencil
path - Horn gradient/slope/aspect/hillshade, Zevenbergen-Thorne curvature,
ruggedness, focal correlate/separable/mean/min/max at radius 1-8, and
Lookup/Reclass - behind strata's plain / Tiled / Chunked entry points.

The compute path is libstrata_cuda.so (hand-written CUDA, C ABI in
include/strata_cuda.h); these modules mirror the reference's Go packages
(terrain, focal, transfer, engine, raster, graph) and call it through
ctypes.
"""
from . import engine, focal, raster, terrain, transfer  # noqa: F401

__all__ = ["engine", "focal", "raster", "terrain", "transfer"]
