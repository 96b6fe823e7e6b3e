"""ctypes front end of the reference's own TSDF integration
(oracle/_ref/libcfref_tsdf.so: src/tsdf_volume.cu and kernels/tsdf_kernels.cu
unmodified, built for sm_100a with the reference's flags, driven by
oracle/ref_tsdf_harness.cu).

TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU parity tests, by
tests/golden/make_tsdf_golden.py and by `bench.py --impl reference
--workload tsdf`.  Needs a GPU.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcfref_tsdf.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.reft_create.restype = vp
        L.reft_create.argtypes = [vp, f, f, vp, f, f]
        L.reft_destroy.argtypes = [vp]
        L.reft_set_voxels.restype = i
        L.reft_set_voxels.argtypes = [vp, vp]
        L.reft_get_voxels.restype = i
        L.reft_get_voxels.argtypes = [vp, vp]
        L.reft_upload.restype = i
        L.reft_upload.argtypes = [vp, vp, i, i, vp, vp, i, vp, vp, vp]
        L.reft_integrate.restype = i
        L.reft_integrate.argtypes = [vp, vp, vp, i, ctypes.POINTER(f)]
        L.reft_mark.restype = i
        L.reft_mark.argtypes = [vp, vp, i, vp, i, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class RefTsdf:
    """A reference TSDFVolume with one synth.TsdfFrame's inputs uploaded;
    warp=False integrates rigidly, gate=False passes no counts."""

    def __init__(self, frame, warp=True, gate=True):
        L = lib()
        pr = frame.params
        self._keep = [np.ascontiguousarray(pr["dims"], np.int32), np.ascontiguousarray(pr["origin"], np.float32)]
        self.h = L.reft_create(_p(self._keep[0]), pr["voxel_size"], pr["truncation"], _p(self._keep[1]),
                               pr["decay_alpha"], pr["max_weight"])
        if not self.h:
            raise RuntimeError("reft_create failed")
        self.n = frame.voxels.shape[0]
        self.frame = frame
        self.set_voxels(frame.voxels)
        N = frame.nodes.shape[0] if warp else 0
        arrs = [np.ascontiguousarray(frame.depth, np.float32), np.ascontiguousarray(frame.nodes),
                np.ascontiguousarray(frame.transforms), np.ascontiguousarray(frame.voxel_knn, np.int32),
                np.ascontiguousarray(frame.voxel_knn_w, np.float32),
                np.ascontiguousarray(frame.counts, np.int32) if gate else None]
        if L.reft_upload(self.h, _p(arrs[0]), frame.width, frame.height, _p(arrs[1]), _p(arrs[2]), N, _p(arrs[3]),
                         _p(arrs[4]), _p(arrs[5])) != 0:
            raise RuntimeError("reft_upload failed")

    def set_voxels(self, vox):
        v = np.ascontiguousarray(vox, np.float32)
        assert v.shape == (self.n, 3)
        if lib().reft_set_voxels(self.h, _p(v)) != 0:
            raise RuntimeError("reft_set_voxels failed")

    def voxels(self):
        out = np.zeros((self.n, 3), np.float32)
        if lib().reft_get_voxels(self.h, _p(out)) != 0:
            raise RuntimeError("reft_get_voxels failed")
        return out

    def integrate(self, min_opt=3):
        cam = np.ascontiguousarray(self.frame.cam, np.float32)
        pose = np.ascontiguousarray(self.frame.camera_pose, np.float32)
        ms = ctypes.c_float(0.0)
        if lib().reft_integrate(self.h, _p(cam), _p(pose), int(min_opt), ctypes.byref(ms)) != 0:
            raise RuntimeError("reft_integrate failed")
        return ms.value

    def close(self):
        if self.h:
            lib().reft_destroy(self.h)
            self.h = None


def mark(recs, vidx, dims, frame, counts, frames):
    """mark_optimized_voxels_kernel on host arrays; returns new counts, frames."""
    r = np.ascontiguousarray(recs)
    vm = np.ascontiguousarray(vidx, np.int32)
    d = np.ascontiguousarray(dims, np.int32)
    c = np.array(counts, np.int32)
    f = np.array(frames, np.int32)
    if lib().reft_mark(_p(r), _p(vm), vm.size, _p(d), int(frame), _p(c), _p(f)) != 0:
        raise RuntimeError("reft_mark failed")
    return c, f
