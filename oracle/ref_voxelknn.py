"""ctypes front end of the reference's own voxel kNN field
(oracle/_ref/libcfref_voxelknn.so: WarpField::compute_voxel_knn of
src/warp_field.cu with the TSDFVolume of src/tsdf_volume.cu, unmodified,
built for sm_100a with the reference's flags, driven by
oracle/ref_voxelknn_harness.cu).

TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU parity tests, by
tests/golden/make_voxelknn_golden.py and by `bench.py --impl reference
--workload voxelknn`.  Needs a GPU.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcfref_voxelknn.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.refk_create.restype = vp
        L.refk_create.argtypes = [vp, f, vp, i]
        L.refk_destroy.argtypes = [vp]
        L.refk_set_voxels.restype = i
        L.refk_set_voxels.argtypes = [vp, vp]
        L.refk_set_nodes.restype = i
        L.refk_set_nodes.argtypes = [vp, vp, i]
        L.refk_compute.restype = i
        L.refk_compute.argtypes = [vp, vp, vp, ctypes.POINTER(f)]
        L.refk_kernel.restype = i
        L.refk_kernel.argtypes = [vp, ctypes.POINTER(f)]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class RefVoxelKnn:
    """A reference TSDFVolume holding `vox` (float32 (V, 3) voxel records) and
    a WarpField holding `nodes`; params = dict(dims, origin, voxel_size)."""

    def __init__(self, params, vox, nodes):
        L = lib()
        self._dims = np.ascontiguousarray(params["dims"], np.int32)
        self._org = np.ascontiguousarray(params["origin"], np.float32)
        self.V = int(np.prod(self._dims.astype(np.int64)))
        self.h = L.refk_create(_p(self._dims), float(params["voxel_size"]), _p(self._org),
                               max(8192, int(len(nodes))))
        v = np.ascontiguousarray(vox, np.float32)
        assert v.shape == (self.V, 3)
        if L.refk_set_voxels(self.h, _p(v)) != 0:
            raise RuntimeError("reference voxel upload failed")
        nd = np.ascontiguousarray(nodes)
        if L.refk_set_nodes(self.h, _p(nd), int(len(nd))) != 0:
            raise RuntimeError("reference node upload failed")

    def compute(self, read=True):
        """One WarpField::compute_voxel_knn: (ids int32 (V, 4), ws float32
        (V, 4), ms) with read=True, else (None, None, ms)."""
        ids = np.zeros((self.V, 4), np.int32) if read else None
        ws = np.zeros((self.V, 4), np.float32) if read else None
        ms = ctypes.c_float()
        rc = lib().refk_compute(self.h, _p(ids), _p(ws), ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference compute_voxel_knn failed: {rc}")
        return ids, ws, ms.value

    def kernel_ms(self):
        """compute_voxel_knn_kernel alone (the reference's launch shape) into
        the outputs of the last compute(); its CUDA-event time in ms."""
        ms = ctypes.c_float()
        rc = lib().refk_kernel(self.h, ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference compute_voxel_knn_kernel failed: {rc}")
        return ms.value

    def close(self):
        if self.h:
            lib().refk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
