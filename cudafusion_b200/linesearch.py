"""Python mirror of CUDAFusion's GN-step acceptance.

The validation of the solve's increment and the ten-trial line search of
DynamicFusionPipeline's GN loop (include/fusion_app.h:409-641), with
correspondence_rmse (:1331-1350) and upload_scaled_delta_x (:1352-1375), on
the sm_100a library through its C ABI: the trials run on the device without a
host round trip (the reference downloads every correspondence record per
trial).
"""
import ctypes
from dataclasses import dataclass

import torch

from . import _lib
from ._lib import check
from .corr import _mat4, frame_args


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


@dataclass
class LineSearchParams:
    """The pipeline's update parameters (update_scale, max_update_rot,
    max_update_trans, max_dx_mean, min_valid_corrs)."""

    update_scale: float = 1.0
    max_update_rot: float = 0.12
    max_update_trans: float = 0.04
    max_dx_mean: float = 0.0
    min_valid_corrs: int = 100

    def c(self):
        return _lib.LineSearchParams(self.update_scale, self.max_update_rot, self.max_update_trans,
                                     self.max_dx_mean, int(self.min_valid_corrs), 0)


def validate_update(delta_x, num_nodes, params=None, stream=None):
    """The increment statistics and the acceptance (fusion_app.h:409-490); synchronises."""
    params = params or LineSearchParams()
    st = _lib.UpdateStats()
    check(_lib.lib().cf_validate_update(_ptr(delta_x), int(num_nodes), ctypes.byref(params.c()), ctypes.byref(st),
                                        _stream_ptr(stream)), "cf_validate_update")
    return {f: getattr(st, f) for f, _ in _lib.UpdateStats._fields_ if f != "pad_"}


def scale_delta(delta_x, num_nodes, max_rot, max_trans, scale, out=None, stream=None):
    """upload_scaled_delta_x on the device (no synchronisation)."""
    out = out if out is not None else torch.empty_like(delta_x)
    check(_lib.lib().cf_scale_delta(_ptr(delta_x), int(num_nodes), float(max_rot), float(max_trans), float(scale),
                                    _ptr(out), _stream_ptr(stream)), "cf_scale_delta")
    return out


def correspondence_rmse(corrs, num_corrs, stream=None):
    """correspondence_rmse on the device: (sum w r^2, sum w, rmse); synchronises."""
    dev = corrs.device
    part = torch.empty(2 * _lib.CF_RMSE_BLOCKS, dtype=torch.float64, device=dev)
    out = torch.empty(2, dtype=torch.float64, device=dev)
    check(_lib.lib().cf_correspondence_rmse(_ptr(corrs), int(num_corrs), _ptr(part), _ptr(out), _stream_ptr(stream)),
          "cf_correspondence_rmse")
    s, w = (float(v) for v in out.cpu())
    return s, w, (s / w) ** 0.5 if w > 0 else float("inf")


class LineSearch:
    """The device scratch of cf_line_search for warps of up to max_nodes nodes."""

    def __init__(self, max_nodes, device="cuda"):
        self.transforms = torch.empty(max_nodes * 32, dtype=torch.uint8, device=device)
        self.delta = torch.empty(max_nodes * 6, dtype=torch.float32, device=device)
        self.rmse = torch.empty(_lib.CF_LINE_SEARCH_SCRATCH, dtype=torch.float64, device=device)

    def run(self, raster, search, mesh, frame, transforms, delta_x, base_rmse, base_valid, params=None,
            corr_params=None, warped=None, pixel_knn_out=None, stream=None):
        """One GN iteration's line search (fusion_app.h:493-641): `transforms`
        (device DQs of mesh's graph) is updated in place; frame's live maps and
        hit voxels, search.corrs and search.num_valid hold the accepted warp's,
        and so do the (ids, weights) device tensors pixel_knn_out (4 per
        pixel) when given.  Returns dict(best_scale, best_rmse, trial_rmse,
        trial_valid)."""
        from .corr import CorrParams

        params = params or LineSearchParams()
        corr_params = corr_params or CorrParams()
        warped = warped if warped is not None else torch.empty_like(mesh.canonical)
        f = frame_args(frame, use_voxels=True, pixel_knn_out=pixel_knn_out)
        cam = frame.camera()
        bs = ctypes.c_float()
        br = ctypes.c_double()
        tr = (ctypes.c_double * _lib.CF_LINE_SEARCH_TRIALS)()
        tv = (ctypes.c_int * _lib.CF_LINE_SEARCH_TRIALS)()
        check(_lib.lib().cf_line_search(
            raster._h, search._h, _ptr(mesh.canonical), _ptr(warped), _ptr(mesh.triangles), mesh.num_vertices,
            mesh.num_triangles, ctypes.byref(mesh.grid), _ptr(mesh.nodes), _ptr(transforms), mesh.num_nodes,
            _ptr(mesh.voxel_knn), _ptr(mesh.voxel_knn_w), _ptr(delta_x), ctypes.byref(params.c()), ctypes.byref(f),
            ctypes.byref(cam), ctypes.byref(_mat4(frame.T_cam_world)), ctypes.byref(_mat4(frame.T_world_cam)),
            ctypes.byref(corr_params.c()), _ptr(search.corrs), _ptr(search.num_valid), float(base_rmse),
            int(base_valid), _ptr(self.transforms), _ptr(self.delta), _ptr(self.rmse), ctypes.byref(bs),
            ctypes.byref(br), tr, tv, _stream_ptr(stream)), "cf_line_search")
        return {"best_scale": bs.value, "best_rmse": br.value, "trial_rmse": list(tr), "trial_valid": list(tv)}
