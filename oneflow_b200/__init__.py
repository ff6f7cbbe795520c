"""B200 (sm_100a) implementation of OneFLOW's unstructured finite-volume
residual + LU-SGS update path, behind a C ABI (include/oneflow_b200.h)."""
from . import params
from .meshio import Mesh, read_ofl, write_ofl
from .solver import LUSGS_SEQUENCE, NS_SOLVER, TURB_SOLVER, Batch, Incompressible, OfgError, Solver, colour_order, \
    load_library, rcm_order

__all__ = ["params", "Mesh", "read_ofl", "write_ofl", "Solver", "Batch", "Incompressible", "OfgError", "load_library",
           "colour_order",
           "rcm_order",
           "LUSGS_SEQUENCE", "NS_SOLVER", "TURB_SOLVER"]
