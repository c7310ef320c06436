"""B200-native (sm_100a) tree gravity with the call surface of GIZMO's shared-memory tree.

The compute path is libgt.so (CUDA, built from csrc/ for sm_100a), reached through the C ABI of
include/gt.h.  This package holds its ctypes binding (``_gt``), the seeded synthetic workloads
(``ics``), the C++ shim of the reference's shmem/tree.h surface (``shim/``) and the multi-GPU
target sharding helpers (``sharding``).
"""
from . import ics  # noqa: F401
from ._gt import (  # noqa: F401
    GT_DIRECT_FP32, GT_DIRECT_FP64, GT_GROUP_BATCH, GT_GROUP_LEAF, GT_GROUP_NODE, GT_GROUP_SINGLE,
    GT_KEY_MORTON, GT_KEY_PEANO, GT_MAC_LEARNED, GT_MAC_NODE, GT_MAC_NODE_FEATURES, GT_MAC_PLAIN,
    GT_NGB_GATHER, GT_NGB_PAIRS, GT_NGB_REVERSE, GT_OUT_ORIGINAL, GT_OUT_TARGETS,
    Context, GTError, Tree, load_library,
)

__all__ = ["Context", "Tree", "GTError", "load_library", "ics"]
