"""NumPy dtypes byte-identical to the reference structs (include/types.h).

DualQuat       include/types.h:86-94    32 B (two float4, 16-B aligned)
DeformNode     include/types.h:185-192  96 B
Correspondence include/types.h:198-206  76 B (C++ bool + 3 pad bytes)
"""
import numpy as np

K_NEIGHBORS = 4  # include/types.h:182
K_GRAPH = 8  # include/types.h:183
BLOCK_DIM = 6
BLOCK_SIZE = 36

DQ_DTYPE = np.dtype([("real", "<f4", (4,)), ("dual", "<f4", (4,))], align=True)
NODE_DTYPE = np.dtype(
    [
        ("pos", "<f4", (3,)),
        ("normal", "<f4", (3,)),
        ("radius", "<f4"),
        ("neighbors", "<i4", (K_GRAPH,)),
        ("neighbor_w", "<f4", (K_GRAPH,)),
        ("num_neighbors", "<i4"),
    ]
)
CORR_DTYPE = np.dtype(
    [
        ("src", "<f4", (3,)),
        ("dst", "<f4", (3,)),
        ("normal", "<f4", (3,)),
        ("node_ids", "<i4", (K_NEIGHBORS,)),
        ("node_ws", "<f4", (K_NEIGHBORS,)),
        ("weight", "<f4"),
        ("valid", "u1"),
        ("pad", "u1", (3,)),
    ]
)

assert DQ_DTYPE.itemsize == 32
assert NODE_DTYPE.itemsize == 96
assert CORR_DTYPE.itemsize == 76


def identity_transforms(n):
    """DualQuat::identity() for n nodes (include/types.h:90-93)."""
    t = np.zeros(n, DQ_DTYPE)
    t["real"][:, 3] = 1.0
    return t


def dq_as_array(t):
    """(n, 8) float32 view of a DualQuat array: real xyzw, dual xyzw."""
    return np.ascontiguousarray(t).view(np.float32).reshape(-1, 8)
