"""ctypes front end of the reference's own live-surface prediction
(oracle/_ref/libcfref_raster.so: src/mesh_raster_kernels.cu and
src/skinning_kernels.cu unmodified, built for sm_100a with the reference's
flags, driven by oracle/ref_raster_harness.cu).

TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU parity tests, by
tests/golden/make_raster_golden.py and by `bench.py --impl reference
--workload raster`.  Needs a GPU.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcfref_raster.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.refr_create.restype = vp
        L.refr_create.argtypes = [i, i, vp, vp, i, vp, i, vp, vp, i, vp, vp, ctypes.c_longlong]
        L.refr_destroy.argtypes = [vp]
        L.refr_run.restype = i
        L.refr_run.argtypes = [vp, vp, vp, vp, vp, i, ctypes.POINTER(ctypes.c_float)]
        L.refr_download.restype = i
        L.refr_download.argtypes = [vp] * 6
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class RefRaster:
    """One mesh frame (synth.MeshFrame) uploaded to the reference's buffers."""

    def __init__(self, frame, warped=None, with_graph=True):
        L = lib()
        self.W, self.H = frame.width, frame.height
        self._keep = dict(
            canon=np.ascontiguousarray(frame.canonical, np.float32),
            warped=np.ascontiguousarray(frame.warped if warped is None else warped, np.float32),
            tris=np.ascontiguousarray(frame.triangles, np.int32),
            nodes=np.ascontiguousarray(frame.nodes), T=np.ascontiguousarray(frame.transforms),
            vk=np.ascontiguousarray(frame.voxel_knn, np.int32), vw=np.ascontiguousarray(frame.voxel_knn_w, np.float32),
            cam=np.ascontiguousarray(frame.cam, np.float32), cw=np.ascontiguousarray(frame.T_cam_world, np.float32),
            grid=np.array(list(frame.grid_origin) + [frame.voxel_size], np.float32),
            dims=np.ascontiguousarray(frame.dims, np.int32))
        k = self._keep
        self.V = k["canon"].shape[0]
        g = with_graph
        self.h = L.refr_create(self.W, self.H, _p(k["canon"]), _p(k["warped"]), self.V, _p(k["tris"]),
                               k["tris"].shape[0], _p(k["nodes"]) if g else None, _p(k["T"]) if g else None,
                               k["nodes"].shape[0] if g else 0, _p(k["vk"]) if g else None,
                               _p(k["vw"]) if g else None, k["vk"].shape[0] if g else 0)
        if not self.h:
            raise RuntimeError("reference raster harness: allocation or upload failed")

    def run(self, skin=False):
        """One prediction; returns the device ms of the sequence."""
        k = self._keep
        ms = ctypes.c_float(0.0)
        if lib().refr_run(self.h, _p(k["cam"]), _p(k["cw"]), _p(k["grid"]), _p(k["dims"]), int(bool(skin)),
                          ctypes.byref(ms)) != 0:
            raise RuntimeError("reference raster harness: CUDA error")
        return float(ms.value)

    def download(self):
        """(live vertices f32[P,3], live normals f32[P,3], hit int32[P], warped f32[V,3], keys uint64[P])."""
        P = self.W * self.H
        lv = np.zeros((P, 3), np.float32)
        ln = np.zeros((P, 3), np.float32)
        hit = np.zeros(P, np.int32)
        wv = np.zeros((self.V, 3), np.float32)
        z = np.zeros(P, np.uint64)
        if lib().refr_download(self.h, _p(lv), _p(ln), _p(hit), _p(wv), _p(z)) != 0:
            raise RuntimeError("reference raster harness: download failed")
        return lv, ln, hit, wv, z

    def close(self):
        if self.h:
            lib().refr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
