"""Python mirror of CUDAFusion's TSDF volume integration.

TSDFVolume (include/tsdf_volume.h:10-84, src/tsdf_volume.cu:11-60): the
canonical volume of 12-byte voxels (tsdf, weight, colour) and its warped,
decaying projective integration (tsdf_integrate_kernel,
kernels/tsdf_kernels.cu:85-174), plus the optimisation counts that gate it
(mark_optimized_voxels_kernel, kernels/tsdf_kernels.cu:606-650), on the
sm_100a library through its C ABI.
"""
import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check
from .raster import _ptr, _stream_ptr

VOXEL_BYTES = 12


@dataclass
class TsdfParams:
    """TSDFVolume::Params (include/tsdf_volume.h:10-19) with the reference's defaults."""

    dims: tuple = (256, 256, 256)
    voxel_size: float = 0.006
    truncation: float = 0.03
    origin: tuple = (-0.768, -0.768, 0.5)
    decay_alpha: float = 0.90
    max_weight: float = 50.0

    def c(self):
        return _lib.TsdfParams((ctypes.c_int * 3)(*[int(v) for v in self.dims]), float(self.voxel_size),
                               float(self.truncation), (ctypes.c_float * 3)(*[float(v) for v in self.origin]),
                               float(self.decay_alpha), float(self.max_weight))


def _mat4(m):
    a = np.ascontiguousarray(m, np.float32).reshape(16)
    return _lib.Mat4((ctypes.c_float * 16)(*a.tolist()))


def world_to_camera(camera_pose):
    """T_cam_world as TSDFVolume::integrate forms it from camera_pose
    (src/tsdf_volume.cu:34-50)."""
    out = _lib.Mat4()
    check(_lib.lib().cf_tsdf_world_to_camera(ctypes.byref(_mat4(camera_pose)), ctypes.byref(out)),
          "cf_tsdf_world_to_camera")
    return np.array(list(out.m), np.float32).reshape(4, 4)


class TSDFVolume:
    """The volume on the device: `voxels` is a uint8 tensor of 12 bytes per
    voxel in the reference's TSDFVoxel layout, x fastest; `tsdf()` and
    `weight()` view its fields."""

    def __init__(self, params=None, device="cuda"):
        self.params = params or TsdfParams()
        self._c = self.params.c()
        self.n = int(np.prod(np.asarray(self.params.dims, np.int64)))
        self.voxels = torch.empty(self.n * VOXEL_BYTES, dtype=torch.uint8, device=device)
        self._plain = None
        self.reset()

    def reset(self, stream=None):
        """The constructor's state: tsdf 1, weight 0, colour 128 (src/tsdf_volume.cu:11-19)."""
        check(_lib.lib().cf_tsdf_reset(_ptr(self.voxels), self.n, _stream_ptr(stream)), "cf_tsdf_reset")

    def fields(self):
        return self.voxels.view(torch.float32).view(self.n, 3)

    def tsdf(self):
        return self.fields()[:, 0]

    def weight(self):
        return self.fields()[:, 1]

    def total_voxels(self):
        return self.n

    def idx_to_xyz(self, idx):
        dx, dy, _ = self.params.dims
        return idx % dx, (idx // dx) % dy, idx // (dx * dy)

    def voxel_to_world(self, xyz):
        o, vs = self.params.origin, self.params.voxel_size
        return tuple(o[a] + xyz[a] * vs for a in range(3))

    def _scratch(self, n):
        if self._plain is None or self._plain.numel() < 8 * max(n, 1):
            self._plain = torch.empty(8 * max(n, 1), dtype=torch.float32, device=self.voxels.device)
        return self._plain

    def integrate(self, depth, cam, camera_pose, nodes=None, transforms=None, num_nodes=0, voxel_knn=None,
                  voxel_knn_w=None, voxel_opt_counts=None, min_opt_count=0, stream=None):
        """TSDFVolume::integrate (src/tsdf_volume.cu:23-60): depth is a device
        float32 map of cam.width x cam.height; with nodes (num_nodes > 0) the
        voxel centres are warped through voxel_knn / voxel_knn_w and gated by
        voxel_opt_counts >= min_opt_count when given."""
        warp = nodes is not None and num_nodes > 0
        plain = self._scratch(num_nodes) if warp else None
        check(_lib.lib().cf_tsdf_integrate(_ptr(self.voxels), ctypes.byref(self._c), _ptr(depth), ctypes.byref(cam),
                                           ctypes.byref(_mat4(camera_pose)), _ptr(nodes), _ptr(transforms),
                                           int(num_nodes), _ptr(voxel_knn), _ptr(voxel_knn_w),
                                           _ptr(voxel_opt_counts), int(min_opt_count), _ptr(plain),
                                           _stream_ptr(stream)), "cf_tsdf_integrate")

    def warp_voxel_centres(self, nodes=None, transforms=None, num_nodes=0, voxel_knn=None, voxel_knn_w=None,
                           out=None, stream=None):
        """The (warped) voxel centres the integration projects: device float32 [n*3]."""
        out = out if out is not None else torch.empty(3 * self.n, dtype=torch.float32, device=self.voxels.device)
        warp = nodes is not None and num_nodes > 0
        plain = self._scratch(num_nodes) if warp else None
        check(_lib.lib().cf_tsdf_warp_voxel_centres(_ptr(out), ctypes.byref(self._c), _ptr(nodes), _ptr(transforms),
                                                    int(num_nodes), _ptr(voxel_knn), _ptr(voxel_knn_w), _ptr(plain),
                                                    _stream_ptr(stream)), "cf_tsdf_warp_voxel_centres")
        return out


    def compute_voxel_knn(self, nodes, num_nodes, voxel_knn=None, voxel_knn_w=None, stream=None):
        """WarpField::compute_voxel_knn (src/warp_field.cu:957-981) over this
        volume: nodes is the device DeformNode array (uint8, 96 bytes each).
        Returns (voxel_knn int32 [n*4], voxel_knn_w float32 [n*4]) on the
        device, allocated here unless given; with no nodes they are returned
        untouched, as the reference leaves them."""
        dev = self.voxels.device
        if voxel_knn is None:
            voxel_knn = torch.empty(4 * self.n, dtype=torch.int32, device=dev)
        if voxel_knn_w is None:
            voxel_knn_w = torch.empty(4 * self.n, dtype=torch.float32, device=dev)
        check(_lib.lib().cf_compute_voxel_knn(_ptr(self.voxels), ctypes.byref(self._c), _ptr(nodes), int(num_nodes),
                                              _ptr(voxel_knn), _ptr(voxel_knn_w), _stream_ptr(stream)),
              "cf_compute_voxel_knn")
        return voxel_knn, voxel_knn_w


def mark_optimized_voxels(corrs, canonical_vidx, num_pixels, dims, frame_id, counts, frames, stream=None):
    """mark_optimized_voxels_kernel: corrs is the device correspondence
    records (uint8, 76 bytes each), canonical_vidx / counts / frames device
    int32; counts and frames are updated in place."""
    d = (ctypes.c_int * 3)(*[int(v) for v in dims])
    check(_lib.lib().cf_mark_optimized_voxels(_ptr(corrs), _ptr(canonical_vidx), int(num_pixels), ctypes.byref(d),
                                              int(frame_id), _ptr(counts), _ptr(frames), _stream_ptr(stream)),
          "cf_mark_optimized_voxels")
