"""ctypes binding of the C ABI (include/cudafusion_b200.h).

Loading fails loudly when libcfb200.so is missing: there is no fallback path.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcfb200.so")

CF_OK = 0
CF_ERR_INVALID_ARG = 1
CF_ERR_OOM = 2
CF_ERR_NON_FINITE = 3
CF_ERR_TIMEOUT = 4
CF_ERR_CUDA = 5
CF_ERR_CAPACITY = 6
CF_ERR_NOT_IMPLEMENTED = 7
CF_ERR_NO_DEVICE = 8

CF_OPT_ARAP_CONSISTENT = 1
CF_OPT_PCG_CTAS = 2
CF_OPT_PCG_MODE = 3
CF_OPT_PCG_PIPELINED = 4
CF_OPT_GRAPH = 5
CF_OPT_GRAPH_ACTIVE = 6
CF_OPT_SPIN_LIMIT = 7
CF_OPT_TEST_BARRIER_EXTRA = 8
CF_OPT_STREAM_TILE = 9
CF_OPT_PCG_ACTIVE = 10
CF_MAX_GN_ITERS = 32
CF_PROF_SLOTS = 12
CF_MPNN_IN = 20
CF_MPNN_HIDDEN = 64
CF_MPNN_OUT = 6
CF_MPNN_PARAMS = 19526
CF_MPNN_ROT_SCALE = 10.0
CF_MPNN_TRANS_SCALE = 100.0
CF_MPNN_RES_SCALE = 1000.0
CF_NOALLOC_MAX_NODES = 8192

# Every symbol the public header declares (the ABI test checks the list
# against include/cudafusion_b200.h).
EXPORTS = [
    "cf_status_string",
    "cf_gn_params_default",
    "cf_gn_create",
    "cf_gn_destroy",
    "cf_gn_set_params",
    "cf_gn_get_params",
    "cf_gn_set_option",
    "cf_gn_get_option",
    "cf_gn_check",
    "cf_gn_linearize_solve",
    "cf_gn_invalidate_pattern",
    "cf_gn_get_system",
    "cf_gn_solve",
    "cf_gn_solve_batched",
    "cf_gn_last_stats",
    "cf_gn_autotune",
    "cf_mpnn_create",
    "cf_mpnn_destroy",
    "cf_mpnn_set_weights",
    "cf_mpnn_get_weights",
    "cf_mpnn_set_graph",
    "cf_mpnn_forward",
    "cf_mpnn_gradients",
    "cf_mpnn_train_step",
    "cf_dq_increments",
    "cf_gn_features",
    "cf_gn_solve_learned",
    "cf_energy_noalloc",
    "cf_warp_apply_twist",
    "cf_warp_skin_points",
    "cf_gn_profile_enable",
    "cf_gn_profile_read",
    "cf_gn_profile_name",
    "cf_gn_launch_count",
    "cf_corr_search_create",
    "cf_corr_search_destroy",
    "cf_find_correspondences",
    "cf_compute_pixel_knn",
    "cf_corr_search_launch_count",
    "cf_corr_search_set_chunks",
    "cf_skin_mesh_vertices",
    "cf_raster_create",
    "cf_raster_destroy",
    "cf_rasterize_live_surface",
    "cf_raster_launch_count",
    "cf_predict_live_surface",
    "cf_validate_update",
    "cf_scale_delta",
    "cf_correspondence_rmse",
    "cf_line_search",
    "cf_tsdf_reset",
    "cf_tsdf_world_to_camera",
    "cf_tsdf_integrate",
    "cf_tsdf_warp_voxel_centres",
    "cf_mark_optimized_voxels",
    "cf_compute_voxel_knn",
    "cf_get_version",
    "cf_last_cuda_error",
]


class GNParams(ctypes.Structure):
    """cf_gn_params = GaussNewtonSolver::Params (include/solver.h:13-22)."""

    _fields_ = [
        ("gn_iterations", ctypes.c_int),
        ("pcg_iterations", ctypes.c_int),
        ("pcg_tolerance", ctypes.c_float),
        ("lambda_smooth", ctypes.c_float),
        ("lambda_rot", ctypes.c_float),
        ("lambda_damping", ctypes.c_float),
        ("debug", ctypes.c_int),
    ]


class Problem(ctypes.Structure):
    _fields_ = [
        ("nodes", ctypes.c_void_p),
        ("num_nodes", ctypes.c_int),
        ("canon_points", ctypes.c_void_p),
        ("corrs", ctypes.c_void_p),
        ("num_corrs", ctypes.c_int),
        ("max_rot", ctypes.c_float),
        ("max_trans", ctypes.c_float),
        ("update_scale", ctypes.c_float),
    ]


class Camera(ctypes.Structure):
    """cf_camera = CameraIntrinsics (include/types.h:148-162)."""

    _fields_ = [("fx", ctypes.c_float), ("fy", ctypes.c_float), ("cx", ctypes.c_float), ("cy", ctypes.c_float),
                ("width", ctypes.c_int), ("height", ctypes.c_int)]


class Mat4(ctypes.Structure):
    """cf_mat4 = Mat4 (include/types.h:26-27), row-major."""

    _fields_ = [("m", ctypes.c_float * 16)]


class CorrParams(ctypes.Structure):
    _fields_ = [("dist_threshold", ctypes.c_float), ("angle_threshold", ctypes.c_float),
                ("view_threshold", ctypes.c_float), ("search_radius_px", ctypes.c_int)]


class CorrFrameArgs(ctypes.Structure):
    """cf_corr_frame: device pointers of one frame's inputs."""

    _fields_ = [
        ("live_vertices", ctypes.c_void_p),
        ("live_normals", ctypes.c_void_p),
        ("depth", ctypes.c_void_p),
        ("depth_normals", ctypes.c_void_p),
        ("pixel_knn", ctypes.c_void_p),
        ("pixel_knn_w", ctypes.c_void_p),
        ("hit_voxel_idx", ctypes.c_void_p),
        ("voxel_knn", ctypes.c_void_p),
        ("voxel_knn_w", ctypes.c_void_p),
        ("num_voxels", ctypes.c_longlong),
        ("pixel_knn_out", ctypes.c_void_p),
        ("pixel_knn_w_out", ctypes.c_void_p),
    ]


class VoxelGrid(ctypes.Structure):
    """cf_voxel_grid: the canonical grid's origin, voxel size and dims."""

    _fields_ = [("origin", ctypes.c_float * 3), ("voxel_size", ctypes.c_float), ("dims", ctypes.c_int * 3)]


class UpdateStats(ctypes.Structure):
    """cf_update_stats: the increment's validation statistics and decision."""

    _fields_ = [("rot_sum", ctypes.c_double), ("trans_sum", ctypes.c_double), ("eff_rot_sum", ctypes.c_double),
                ("eff_trans_sum", ctypes.c_double), ("rot_max", ctypes.c_float), ("trans_max", ctypes.c_float),
                ("eff_rot_max", ctypes.c_float), ("eff_trans_max", ctypes.c_float), ("finite", ctypes.c_int),
                ("num_nodes", ctypes.c_int), ("iter_ok", ctypes.c_int), ("pad_", ctypes.c_int)]


class LineSearchParams(ctypes.Structure):
    _fields_ = [("update_scale", ctypes.c_float), ("max_update_rot", ctypes.c_float),
                ("max_update_trans", ctypes.c_float), ("max_dx_mean", ctypes.c_float),
                ("min_valid_corrs", ctypes.c_int), ("pad_", ctypes.c_int)]


class TsdfParams(ctypes.Structure):
    """cf_tsdf_params: TSDFVolume::Params (include/tsdf_volume.h:10-19)."""

    _fields_ = [("dims", ctypes.c_int * 3), ("voxel_size", ctypes.c_float), ("truncation", ctypes.c_float),
                ("origin", ctypes.c_float * 3), ("decay_alpha", ctypes.c_float), ("max_weight", ctypes.c_float)]


CF_RMSE_BLOCKS = 296
CF_LINE_SEARCH_TRIALS = 10
CF_LINE_SEARCH_SCRATCH = 2 * CF_RMSE_BLOCKS + 3 * CF_LINE_SEARCH_TRIALS


class SolveStats(ctypes.Structure):
    _fields_ = [
        ("energy_initial", ctypes.c_double),
        ("energy_final", ctypes.c_double),
        ("energy_per_iter", ctypes.c_double * CF_MAX_GN_ITERS),
        ("pcg_iterations", ctypes.c_int * CF_MAX_GN_ITERS),
        ("pcg_residual", ctypes.c_double * CF_MAX_GN_ITERS),
        ("gn_iterations_run", ctypes.c_int),
        ("num_blocks", ctypes.c_int),
        ("precond_fallbacks", ctypes.c_int),
        ("error_flags", ctypes.c_int),
        ("init_rejected", ctypes.c_int),
        ("energy_warm_start", ctypes.c_double),
        ("energy_predicted", ctypes.c_double),
    ]


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("pcg_mode", ctypes.c_int),
        ("pcg_ctas", ctypes.c_int),
        ("stream_tile", ctypes.c_int),
        ("candidates", ctypes.c_int),
        ("ms_best", ctypes.c_double),
        ("ms_default", ctypes.c_double),
        ("from_cache", ctypes.c_int),
    ]


class CFError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        msg = lib().cf_status_string(status).decode()
        buf = ctypes.create_string_buffer(256)
        lib().cf_last_cuda_error(buf, 256)
        detail = buf.value.decode()
        super().__init__(f"{where}: {msg} ({status})" + (f" [{detail}]" if detail else ""))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cudafusion_b200.build` "
                "(there is no CPU fallback)"
            )
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.cf_status_string.restype = ctypes.c_char_p
        L.cf_status_string.argtypes = [i]
        L.cf_gn_profile_name.restype = ctypes.c_char_p
        L.cf_gn_params_default.argtypes = [ctypes.POINTER(GNParams)]
        L.cf_gn_create.argtypes = [ctypes.POINTER(GNParams), i, i, ctypes.POINTER(vp)]
        L.cf_gn_destroy.argtypes = [vp]
        L.cf_gn_set_params.argtypes = [vp, ctypes.POINTER(GNParams)]
        L.cf_gn_get_params.argtypes = [vp, ctypes.POINTER(GNParams)]
        L.cf_gn_set_option.argtypes = [vp, i, i]
        L.cf_gn_get_option.argtypes = [vp, i, ctypes.POINTER(i)]
        L.cf_gn_check.argtypes = [vp, vp]
        L.cf_gn_linearize_solve.argtypes = [vp, vp, i, vp, vp, i, vp, vp]
        L.cf_gn_invalidate_pattern.argtypes = [vp]
        L.cf_gn_get_system.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i), vp, vp, vp, vp, vp]
        L.cf_gn_solve.argtypes = [vp, ctypes.POINTER(Problem), vp, ctypes.POINTER(SolveStats), vp]
        L.cf_gn_solve_batched.argtypes = [vp, ctypes.POINTER(Problem), i, ctypes.POINTER(vp),
                                          ctypes.POINTER(SolveStats), vp]
        L.cf_gn_last_stats.argtypes = [vp, ctypes.POINTER(SolveStats), i, vp]
        L.cf_gn_autotune.argtypes = [vp, ctypes.POINTER(Problem), i, ctypes.POINTER(vp), ctypes.POINTER(TuneResult), vp]
        pf = ctypes.POINTER(ctypes.c_float)
        L.cf_mpnn_create.argtypes = [i, ctypes.POINTER(vp)]
        L.cf_mpnn_destroy.argtypes = [vp]
        L.cf_mpnn_set_weights.argtypes = [vp, vp, i]
        L.cf_mpnn_get_weights.argtypes = [vp, vp, i]
        L.cf_mpnn_set_graph.argtypes = [vp, vp, i, vp]
        L.cf_mpnn_forward.argtypes = [vp, vp, vp, vp]
        L.cf_mpnn_gradients.argtypes = [vp, vp, vp, vp, ctypes.POINTER(ctypes.c_double), vp]
        L.cf_mpnn_train_step.argtypes = [vp, vp, vp, f, ctypes.POINTER(ctypes.c_double), vp]
        L.cf_dq_increments.argtypes = [vp, vp, i, vp, vp]
        L.cf_gn_features.argtypes = [vp, ctypes.POINTER(Problem), vp, vp, vp, vp]
        L.cf_gn_solve_learned.argtypes = [vp, vp, ctypes.POINTER(Problem), vp, vp, ctypes.POINTER(SolveStats), vp]
        L.cf_energy_noalloc.argtypes = [ctypes.POINTER(Problem), vp, f, vp, vp]
        L.cf_warp_apply_twist.argtypes = [vp, vp, i, f, f, f, vp]
        L.cf_warp_skin_points.argtypes = [vp, vp, vp, i, vp, vp, i, vp, vp]
        L.cf_gn_profile_enable.argtypes = [vp, i]
        L.cf_gn_profile_read.argtypes = [vp, vp, vp, i]
        L.cf_gn_profile_name.argtypes = [i]
        L.cf_gn_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.cf_corr_search_create.argtypes = [i, i, ctypes.POINTER(vp)]
        L.cf_corr_search_destroy.argtypes = [vp]
        L.cf_find_correspondences.argtypes = [vp, ctypes.POINTER(CorrFrameArgs), ctypes.POINTER(Camera),
                                              ctypes.POINTER(Mat4), ctypes.POINTER(Mat4), ctypes.POINTER(CorrParams),
                                              vp, vp, vp, vp]
        L.cf_compute_pixel_knn.argtypes = [vp, i, i, vp, vp, ctypes.c_longlong, vp, vp, vp]
        L.cf_corr_search_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.cf_corr_search_set_chunks.argtypes = [vp, i]
        L.cf_skin_mesh_vertices.argtypes = [vp, vp, i, ctypes.POINTER(VoxelGrid), vp, vp, i, vp, vp, vp]
        L.cf_raster_create.argtypes = [i, i, ctypes.POINTER(vp)]
        L.cf_raster_destroy.argtypes = [vp]
        L.cf_rasterize_live_surface.argtypes = [vp, vp, vp, vp, i, i, ctypes.POINTER(Camera), ctypes.POINTER(Mat4),
                                                ctypes.POINTER(VoxelGrid), vp, vp, vp, vp]
        L.cf_raster_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
        L.cf_validate_update.argtypes = [vp, i, ctypes.POINTER(LineSearchParams), ctypes.POINTER(UpdateStats), vp]
        L.cf_scale_delta.argtypes = [vp, i, f, f, f, vp, vp]
        L.cf_correspondence_rmse.argtypes = [vp, i, vp, vp, vp]
        L.cf_line_search.argtypes = [vp, vp, vp, vp, vp, i, i, ctypes.POINTER(VoxelGrid), vp, vp, i, vp, vp, vp,
                                     ctypes.POINTER(LineSearchParams), ctypes.POINTER(CorrFrameArgs),
                                     ctypes.POINTER(Camera), ctypes.POINTER(Mat4), ctypes.POINTER(Mat4),
                                     ctypes.POINTER(CorrParams), vp, vp, ctypes.c_double, i, vp, vp, vp,
                                     ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), vp]
        L.cf_predict_live_surface.argtypes = [vp, vp, vp, vp, i, i, vp, vp, i, vp, vp, ctypes.POINTER(Camera),
                                              ctypes.POINTER(Mat4), ctypes.POINTER(VoxelGrid), vp, vp, vp, vp]
        L.cf_tsdf_reset.argtypes = [vp, ctypes.c_longlong, vp]
        L.cf_tsdf_world_to_camera.argtypes = [ctypes.POINTER(Mat4), ctypes.POINTER(Mat4)]
        L.cf_tsdf_integrate.argtypes = [vp, ctypes.POINTER(TsdfParams), vp, ctypes.POINTER(Camera),
                                        ctypes.POINTER(Mat4), vp, vp, i, vp, vp, vp, i, vp, vp]
        L.cf_tsdf_warp_voxel_centres.argtypes = [vp, ctypes.POINTER(TsdfParams), vp, vp, i, vp, vp, vp, vp]
        L.cf_mark_optimized_voxels.argtypes = [vp, vp, i, ctypes.POINTER(ctypes.c_int * 3), i, vp, vp, vp]
        L.cf_compute_voxel_knn.argtypes = [vp, ctypes.POINTER(TsdfParams), vp, i, vp, vp, vp]
        L.cf_get_version.argtypes = [ctypes.POINTER(i)] * 3
        L.cf_last_cuda_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        for name in EXPORTS:
            if name not in ("cf_status_string", "cf_gn_profile_name"):
                getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def check(status, where=""):
    if status != CF_OK:
        raise CFError(status, where)
    return status
