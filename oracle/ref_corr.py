"""ctypes front end of the reference's own correspondence search
(oracle/_ref/libcfref_corr.so: kernels/tsdf_kernels.cu unmodified, built for
sm_100a with the reference's flags, driven by oracle/ref_corr_harness.cu).

TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU parity tests, by
tests/golden/make_corr_golden.py and by `bench.py --impl reference
--workload corr`.  Needs a GPU.
"""
import ctypes
import os

import numpy as np

from cudafusion_b200.types import CORR_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcfref_corr.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.refc_create.restype = vp
        L.refc_create.argtypes = [i, i] + [vp] * 7 + [ctypes.c_longlong]
        L.refc_destroy.argtypes = [vp]
        L.refc_run.restype = i
        L.refc_run.argtypes = [vp, vp, vp, vp, f, f, f, i, i, ctypes.POINTER(f)]
        L.refc_upload.restype = i
        L.refc_upload.argtypes = [vp] * 6
        L.refc_download.restype = i
        L.refc_download.argtypes = [vp] * 5
        L.refc_sizeof_correspondence.restype = i
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefCorrSearch:
    """One frame uploaded to the reference's buffers (synth.CorrFrame)."""

    def __init__(self, frame):
        L = lib()
        assert L.refc_sizeof_correspondence() == CORR_DTYPE.itemsize
        self._keep = [np.ascontiguousarray(a, dt) for a, dt in (
            (frame.live_vertices, np.float32), (frame.live_normals, np.float32), (frame.depth, np.float32),
            (frame.depth_normals, np.float32), (frame.hit_voxel_idx, np.int32), (frame.voxel_knn, np.int32),
            (frame.voxel_knn_w, np.float32))]
        lv, ln, d, dn, hit, vk, vw = self._keep
        self.P = frame.width * frame.height
        self.cam = np.ascontiguousarray(frame.cam, np.float32)
        self.cw = np.ascontiguousarray(frame.T_cam_world, np.float32)
        self.wc = np.ascontiguousarray(frame.T_world_cam, np.float32)
        self.h = L.refc_create(frame.width, frame.height, _p(lv), _p(ln), _p(d), _p(dn), _p(hit), _p(vk), _p(vw),
                               vk.shape[0])
        if not self.h:
            raise RuntimeError("reference correspondence harness: allocation or upload failed")

    def run(self, dist_threshold, angle_threshold, view_threshold, search_radius_px, debug=True):
        """One find_correspondences call; returns (valid count, device ms)."""
        ms = ctypes.c_float(0.0)
        n = lib().refc_run(self.h, _p(self.cam), _p(self.cw), _p(self.wc), dist_threshold, angle_threshold,
                           view_threshold, int(search_radius_px), int(bool(debug)), ctypes.byref(ms))
        if n < 0:
            raise RuntimeError("reference correspondence harness: CUDA error")
        return n, float(ms.value)

    def upload(self):
        """Copies the frame's per-pixel inputs to the device again (host -> device)."""
        lv, ln, d, dn, hit = self._keep[:5]
        if lib().refc_upload(self.h, _p(lv), _p(ln), _p(d), _p(dn), _p(hit)) != 0:
            raise RuntimeError("reference correspondence harness: upload failed")

    def download_records(self, out):
        """Copies the last run's records into `out` (CORR_DTYPE[P], host)."""
        if lib().refc_download(self.h, _p(out), None, None, None) != 0:
            raise RuntimeError("reference correspondence harness: download failed")

    def download(self):
        """(records CORR_DTYPE[P], pixel_knn int32[P,4], pixel_knn_w f32[P,4], stats int32[6])."""
        out = np.zeros(self.P, CORR_DTYPE)
        pk = np.zeros((self.P, 4), np.int32)
        pw = np.zeros((self.P, 4), np.float32)
        st = np.zeros(6, np.int32)
        if lib().refc_download(self.h, _p(out), _p(pk), _p(pw), _p(st)) != 0:
            raise RuntimeError("reference correspondence harness: download failed")
        return out, pk, pw, st

    def close(self):
        if self.h:
            lib().refc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
