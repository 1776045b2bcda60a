"""phem_graph_b200 -- B200-native (sm_100a) rebuild of PHEM's two graph hot paths.

* Connected components + spanning forest by union-find
  (reference: CC/ExternalSpanningTree.cu, CC/GPUSpanningTree.cu).
* Boruvka minimum spanning forest under the (weight, edge id) order
  (reference: MST/src/kernels.cu, MST/src/new_boruvka.cu).

The compute path is libphem.so (hand-written CUDA for sm_100a behind the C ABI
of include/phem.h).  This package is a thin Python view of that ABI plus the
seeded input generators; there is no CPU implementation of either path here.
"""
from ._lib import (  # noqa: F401
    PHEM_CC_CANONICAL, PHEM_CC_DEFAULT, PHEM_FOREST_EMPTY, PHEM_MAX_ROUNDS, PhemError, lib,
)
from .api import Context, EDGE_DTYPE  # noqa: F401
from . import gen  # noqa: F401

__all__ = ["Context", "EDGE_DTYPE", "PhemError", "gen", "lib", "PHEM_CC_CANONICAL", "PHEM_CC_DEFAULT",
           "PHEM_FOREST_EMPTY", "PHEM_MAX_ROUNDS"]
