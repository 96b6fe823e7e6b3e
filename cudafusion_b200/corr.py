"""Python mirror of CUDAFusion's correspondence search.

DynamicFusionPipeline::find_correspondences (include/fusion_app.h:1791-1845)
with the pipeline's search parameters (dist_threshold, angle_threshold,
view_threshold, search_radius_px; config/params.yaml:60-63), on the sm_100a
library through its C ABI.  Like the reference method, `find_correspondences`
synchronises and returns the valid count; the records stay on the device
(`corrs`, the counterpart of the pipeline's d_corrs_), ready for
GaussNewtonSolver.solve with num_corrs = width * height.
"""
import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check
from .types import CORR_DTYPE

CORR_BYTES = CORR_DTYPE.itemsize


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


@dataclass
class CorrParams:
    """The search parameters; the defaults are the stock configuration's
    (config/params.yaml:60-63)."""

    dist_threshold: float = 0.2
    angle_threshold: float = 0.0
    view_threshold: float = 0.0
    search_radius_px: int = 50

    def c(self):
        return _lib.CorrParams(self.dist_threshold, self.angle_threshold, self.view_threshold,
                               int(self.search_radius_px))


def _mat4(m):
    a = np.ascontiguousarray(m, np.float32).reshape(16)
    return _lib.Mat4((ctypes.c_float * 16)(*a.tolist()))


def frame_args(frame, use_voxels=False, pixel_knn_out=None):
    """cf_corr_frame for a DeviceCorrFrame: the per-pixel node lists, or the
    hit voxels with the voxel tables (use_voxels); pixel_knn_out = (ids,
    weights) tensors for the gathered lists (voxel path)."""
    f = _lib.CorrFrameArgs()
    f.live_vertices = frame.live_vertices.data_ptr()
    f.live_normals = frame.live_normals.data_ptr()
    f.depth = frame.depth.data_ptr()
    f.depth_normals = frame.depth_normals.data_ptr()
    if use_voxels:
        f.hit_voxel_idx = frame.hit_voxel_idx.data_ptr()
        f.voxel_knn = frame.voxel_knn.data_ptr()
        f.voxel_knn_w = frame.voxel_knn_w.data_ptr()
        f.num_voxels = frame.num_voxels
        if pixel_knn_out is not None:
            f.pixel_knn_out = pixel_knn_out[0].data_ptr()
            f.pixel_knn_w_out = pixel_knn_out[1].data_ptr()
    else:
        f.pixel_knn = frame.pixel_knn.data_ptr()
        f.pixel_knn_w = frame.pixel_knn_w.data_ptr()
    return f


class DeviceCorrFrame:
    """The device-resident inputs of one search: a synth.CorrFrame's arrays as
    torch tensors (row-major over height x width)."""

    def __init__(self, frame, device="cuda"):
        def up(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a, dt).reshape(-1).copy()).to(device)

        self.width, self.height = int(frame.width), int(frame.height)
        self.cam = np.asarray(frame.cam, np.float32)
        self.T_cam_world = np.asarray(frame.T_cam_world, np.float32)
        self.T_world_cam = np.asarray(frame.T_world_cam, np.float32)
        self.live_vertices = up(frame.live_vertices, np.float32)
        self.live_normals = up(frame.live_normals, np.float32)
        self.depth = up(frame.depth, np.float32)
        self.depth_normals = up(frame.depth_normals, np.float32)
        self.hit_voxel_idx = up(frame.hit_voxel_idx, np.int32)
        self.voxel_knn = up(frame.voxel_knn, np.int32)
        self.voxel_knn_w = up(frame.voxel_knn_w, np.float32)
        self.num_voxels = int(np.asarray(frame.voxel_knn).shape[0])
        self.pixel_knn = up(frame.pixel_knn, np.int32)
        self.pixel_knn_w = up(frame.pixel_knn_w, np.float32)

    @property
    def num_pixels(self):
        return self.width * self.height

    def camera(self):
        fx, fy, cx, cy = (float(v) for v in self.cam)
        return _lib.Camera(fx, fy, cx, cy, self.width, self.height)


class CorrespondenceSearch:
    """Owns the search handle (per-pixel candidate records for frames up to
    max_width x max_height) and the output records of the last search."""

    def __init__(self, max_width, max_height, device="cuda"):
        self._h = ctypes.c_void_p()
        check(_lib.lib().cf_corr_search_create(int(max_width), int(max_height), ctypes.byref(self._h)),
              "cf_corr_search_create")
        self.device = device
        P = int(max_width) * int(max_height)
        self.corrs = torch.zeros(P * CORR_BYTES, dtype=torch.uint8, device=device)
        self.num_valid = torch.zeros(1, dtype=torch.int32, device=device)
        self.stats = torch.zeros(6, dtype=torch.int32, device=device)
        self.pixel_knn = torch.zeros(P * 4, dtype=torch.int32, device=device)
        self.pixel_knn_w = torch.zeros(P * 4, dtype=torch.float32, device=device)

    def close(self):
        if self._h:
            _lib.lib().cf_corr_search_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch(self, frame, params=None, debug=False, use_voxels=False, pixel_knn_out=False, stream=None):
        """Enqueues one search on `stream` (no synchronisation).  use_voxels:
        gather each pixel's node lists from its canonical voxel in the same
        kernel (compute_pixel_knn fused); otherwise read frame.pixel_knn.
        pixel_knn_out (voxel path): also write the gathered lists to
        self.pixel_knn / self.pixel_knn_w."""
        params = params or CorrParams()
        f = frame_args(frame, use_voxels, (self.pixel_knn, self.pixel_knn_w) if pixel_knn_out else None)
        cam = frame.camera()
        check(_lib.lib().cf_find_correspondences(self._h, ctypes.byref(f), ctypes.byref(cam),
                                                 ctypes.byref(_mat4(frame.T_cam_world)),
                                                 ctypes.byref(_mat4(frame.T_world_cam)),
                                                 ctypes.byref(params.c()), _ptr(self.corrs), _ptr(self.num_valid),
                                                 _ptr(self.stats) if debug else None, _stream_ptr(stream)),
              "cf_find_correspondences")

    def find_correspondences(self, frame, params=None, debug=False, use_voxels=False, stream=None):
        """DynamicFusionPipeline::find_correspondences: runs the search and
        returns the valid count (synchronises).  With debug, self.stats holds
        the reference's counters (invalid_live, out_proj, no_depth, far,
        angle, valid)."""
        self.launch(frame, params, debug=debug, use_voxels=use_voxels, stream=stream)
        (stream or torch.cuda.current_stream()).synchronize()
        return int(self.num_valid.item())

    def records(self, num_pixels):
        """The first num_pixels output records as a CORR_DTYPE array (host)."""
        raw = self.corrs[: num_pixels * CORR_BYTES].cpu().numpy()
        return raw.view(CORR_DTYPE).copy()

    def set_chunks(self, chunks):
        """Row chunks per tile of the search (0 = chosen per frame); results
        do not depend on it."""
        check(_lib.lib().cf_corr_search_set_chunks(self._h, int(chunks)), "cf_corr_search_set_chunks")

    def launch_count(self):
        n = ctypes.c_longlong()
        check(_lib.lib().cf_corr_search_launch_count(self._h, ctypes.byref(n)), "cf_corr_search_launch_count")
        return int(n.value)


def compute_pixel_knn(frame, stream=None):
    """compute_pixel_knn_kernel on its own: (pixel_knn int32[P*4],
    pixel_knn_w float32[P*4]) device tensors gathered from frame's voxels."""
    P = frame.num_pixels
    pk = torch.empty(P * 4, dtype=torch.int32, device=frame.depth.device)
    pw = torch.empty(P * 4, dtype=torch.float32, device=frame.depth.device)
    check(_lib.lib().cf_compute_pixel_knn(_ptr(frame.hit_voxel_idx), frame.width, frame.height,
                                          _ptr(frame.voxel_knn), _ptr(frame.voxel_knn_w),
                                          ctypes.c_longlong(frame.num_voxels), _ptr(pk), _ptr(pw),
                                          _stream_ptr(stream)), "cf_compute_pixel_knn")
    return pk, pw
