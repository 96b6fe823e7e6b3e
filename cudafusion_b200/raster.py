"""Python mirror of CUDAFusion's live-surface prediction.

DynamicFusionPipeline::rasterize_deformed_mesh_live_surface
(include/fusion_app.h:1216-1318): the canonical mesh skinned by the
deformation graph through the canonical voxels' node lists
(skin_vertices_from_voxel_knn_kernel, src/skinning_kernels.cu:29-63), then
rasterised into the live vertex / normal / canonical-voxel maps that the
correspondence search reads (src/mesh_raster_kernels.cu:76-200), on the
sm_100a library through its C ABI.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def voxel_grid(origin, voxel_size, dims):
    return _lib.VoxelGrid((ctypes.c_float * 3)(*[float(v) for v in origin]), float(voxel_size),
                          (ctypes.c_int * 3)(*[int(v) for v in dims]))


class DeviceMesh:
    """A synth.MeshFrame on the device: canonical and warped vertices,
    triangles, the deformation graph and the voxel grid's node lists."""

    def __init__(self, frame, device="cuda"):
        from .solver import to_device

        def up(a, dt):
            return torch.from_numpy(np.ascontiguousarray(a, dt).reshape(-1).copy()).to(device)

        self.width, self.height = int(frame.width), int(frame.height)
        self.cam = np.asarray(frame.cam, np.float32)
        self.T_cam_world = np.asarray(frame.T_cam_world, np.float32)
        self.canonical = up(frame.canonical, np.float32)
        self.warped = up(frame.warped, np.float32)
        self.triangles = up(frame.triangles, np.int32)
        self.num_vertices = int(np.asarray(frame.canonical).shape[0])
        self.num_triangles = int(np.asarray(frame.triangles).shape[0])
        self.grid = voxel_grid(frame.grid_origin, frame.voxel_size, frame.dims)
        self.voxel_knn = up(frame.voxel_knn, np.int32)
        self.voxel_knn_w = up(frame.voxel_knn_w, np.float32)
        self.nodes = to_device(frame.nodes)
        self.transforms = to_device(frame.transforms)
        self.num_nodes = int(frame.nodes.shape[0])

    def camera(self):
        fx, fy, cx, cy = (float(v) for v in self.cam)
        return _lib.Camera(fx, fy, cx, cy, self.width, self.height)


def skin_mesh(mesh, out=None, stream=None):
    """skin_vertices_from_voxel_knn_kernel: the canonical vertices warped by
    the nodes of their voxels; device float32 [V*3]."""
    out = out if out is not None else torch.empty_like(mesh.canonical)
    check(_lib.lib().cf_skin_mesh_vertices(_ptr(mesh.canonical), _ptr(out), mesh.num_vertices,
                                           ctypes.byref(mesh.grid), _ptr(mesh.nodes), _ptr(mesh.transforms),
                                           mesh.num_nodes, _ptr(mesh.voxel_knn), _ptr(mesh.voxel_knn_w),
                                           _stream_ptr(stream)), "cf_skin_mesh_vertices")
    return out


class LiveSurfaceRaster:
    """Owns the raster handle (the depth buffer of frames up to
    max_width x max_height) and the live maps of the last frame."""

    def __init__(self, max_width, max_height, device="cuda"):
        self._h = ctypes.c_void_p()
        check(_lib.lib().cf_raster_create(int(max_width), int(max_height), ctypes.byref(self._h)),
              "cf_raster_create")
        P = int(max_width) * int(max_height)
        self.live_vertices = torch.zeros(P * 3, dtype=torch.float32, device=device)
        self.live_normals = torch.zeros(P * 3, dtype=torch.float32, device=device)
        self.hit_voxel_idx = torch.zeros(P, dtype=torch.int32, device=device)

    def close(self):
        if self._h:
            _lib.lib().cf_raster_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def rasterize(self, mesh, warped=None, stream=None):
        """The rasterisation and resolve (no synchronisation)."""
        from .corr import _mat4

        cam = mesh.camera()
        check(_lib.lib().cf_rasterize_live_surface(
            self._h, _ptr(mesh.canonical), _ptr(mesh.warped if warped is None else warped), _ptr(mesh.triangles),
            mesh.num_vertices, mesh.num_triangles, ctypes.byref(cam), ctypes.byref(_mat4(mesh.T_cam_world)),
            ctypes.byref(mesh.grid), _ptr(self.live_vertices), _ptr(self.live_normals), _ptr(self.hit_voxel_idx),
            _stream_ptr(stream)), "cf_rasterize_live_surface")

    def predict(self, mesh, warped_out=None, stream=None):
        """rasterize_deformed_mesh_live_surface: skin the mesh by the graph,
        then rasterise it, in one call (no synchronisation).  Returns the
        warped vertices."""
        from .corr import _mat4

        warped = warped_out if warped_out is not None else torch.empty_like(mesh.canonical)
        cam = mesh.camera()
        check(_lib.lib().cf_predict_live_surface(
            self._h, _ptr(mesh.canonical), _ptr(warped), _ptr(mesh.triangles), mesh.num_vertices,
            mesh.num_triangles, _ptr(mesh.nodes), _ptr(mesh.transforms), mesh.num_nodes, _ptr(mesh.voxel_knn),
            _ptr(mesh.voxel_knn_w), ctypes.byref(cam), ctypes.byref(_mat4(mesh.T_cam_world)),
            ctypes.byref(mesh.grid), _ptr(self.live_vertices), _ptr(self.live_normals), _ptr(self.hit_voxel_idx),
            _stream_ptr(stream)), "cf_predict_live_surface")
        return warped

    def maps(self, num_pixels):
        """(live vertices f32[P,3], live normals f32[P,3], hit voxel int32[P]) on the host."""
        return (self.live_vertices[: 3 * num_pixels].cpu().numpy().reshape(-1, 3),
                self.live_normals[: 3 * num_pixels].cpu().numpy().reshape(-1, 3),
                self.hit_voxel_idx[:num_pixels].cpu().numpy())

    def launch_count(self):
        n = ctypes.c_longlong()
        check(_lib.lib().cf_raster_launch_count(self._h, ctypes.byref(n)), "cf_raster_launch_count")
        return int(n.value)
