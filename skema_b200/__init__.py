"""B200 SketchySVD sketch update: a CUDA library for sm_100a behind a C ABI
(include/skema_c.h), with a Python mirror of Skema's SketchySVD interface."""
from ._lib import SkemaError, load
from .sketchy import (
    AlgParams,
    GaussDimRedux,
    SketchySPD,
    SketchySVD,
    SparseSignDimRedux,
    rbf_sketch_fwd,
    rbf_sketch_vjp,
    read_crs_rows,
    read_matrix,
    read_reference_map_dump,
    sketchysvd,
    write_matrix,
    write_reference_map_dump,
)

__all__ = [
    "AlgParams",
    "GaussDimRedux",
    "SparseSignDimRedux",
    "SketchySVD",
    "SketchySPD",
    "sketchysvd",
    "read_matrix",
    "read_crs_rows",
    "read_reference_map_dump",
    "write_matrix",
    "write_reference_map_dump",
    "rbf_sketch_fwd",
    "rbf_sketch_vjp",
    "SkemaError",
    "load",
]
