"""edgeb200 — host side of the sm_100a EDGE flow-map solver.

The compute lives in libedgeb200.so (CUDA kernels for sm_100a behind a C ABI,
include/edge_b200.h); this package holds the ctypes binding, torch tensor
plumbing, the projection handle and the device-resident substep driver.  The
reference-named drop-in modules are edge-flow-maps_b200/sim and
edge-flow-maps_b200/util.
"""
from ._native import (EDGE_EALIGN, EDGE_EINVAL, EDGE_ENAN, EDGE_ENOCONV, EDGE_OK, HERMITE_FD, HERMITE_FULL,
                      HERMITE_GARM, EdgeError, load)

__all__ = ["load", "EdgeError", "EDGE_OK", "EDGE_EINVAL", "EDGE_EALIGN", "EDGE_ENOCONV", "EDGE_ENAN",
           "HERMITE_FD", "HERMITE_GARM", "HERMITE_FULL"]
