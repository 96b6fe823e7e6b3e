"""ctypes front end of the CPU oracle (oracle/cf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product library never loads
it.  `precision` is "f32" (reference operand order, FP32) or "f64".
"""
import ctypes
import os
import subprocess

import numpy as np

from cudafusion_b200.types import CORR_DTYPE, DQ_DTYPE, NODE_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcforacle.so")

_lib = None


class GNParams(ctypes.Structure):
    """cf_gn_params (include/cudafusion_b200.h) = GaussNewtonSolver::Params."""

    _fields_ = [
        ("gn_iterations", ctypes.c_int),
        ("pcg_iterations", ctypes.c_int),
        ("pcg_tolerance", ctypes.c_float),
        ("lambda_smooth", ctypes.c_float),
        ("lambda_rot", ctypes.c_float),
        ("lambda_damping", ctypes.c_float),
        ("debug", ctypes.c_int),
    ]


def params(gn_iterations=3, pcg_iterations=10, pcg_tolerance=1e-4, lambda_smooth=1.0, lambda_rot=1.0,
           lambda_damping=1e-2, debug=0):
    return GNParams(gn_iterations, pcg_iterations, pcg_tolerance, lambda_smooth, lambda_rot, lambda_damping, debug)


def build():
    """Compiles the oracle with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _fn(name, precision):
    f = getattr(lib(), f"{name}_{precision}")
    return f


def build_pattern(nodes):
    """kernels/solver_kernels.cu:498-541 -> (row_ptr, col_idx)."""
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    n = nodes.shape[0]
    row_ptr = np.zeros(n + 1, np.int32)
    f = lib().cfo_build_pattern
    f.restype = ctypes.c_int
    nnzb = f(_p(nodes), n, _p(row_ptr), None, 0)
    col_idx = np.zeros(max(nnzb, 1), np.int32)
    f(_p(nodes), n, _p(row_ptr), _p(col_idx), nnzb)
    return row_ptr, col_idx[:nnzb]


def exp_se3(twist, precision="f32"):
    tw = np.ascontiguousarray(twist, np.float32)
    out = np.zeros(16, np.float32)
    _fn("cfo_exp_se3", precision)(_p(tw), _p(out))
    return out.reshape(4, 4)


def mat4_to_dq(T, precision="f32"):
    T = np.ascontiguousarray(T, np.float32).reshape(16)
    out = np.zeros(1, DQ_DTYPE)
    _fn("cfo_mat4_to_dq", precision)(_p(T), _p(out))
    return out[0]


def dq_mul(a, b, precision="f32"):
    a = np.ascontiguousarray(np.atleast_1d(a), DQ_DTYPE)
    b = np.ascontiguousarray(np.atleast_1d(b), DQ_DTYPE)
    out = np.zeros(1, DQ_DTYPE)
    _fn("cfo_dq_mul", precision)(_p(a), _p(b), _p(out))
    return out[0]


def dq_centered(a, c, precision="f32"):
    a = np.ascontiguousarray(np.atleast_1d(a), DQ_DTYPE)
    c = np.ascontiguousarray(c, np.float32)
    out = np.zeros(1, DQ_DTYPE)
    _fn("cfo_dq_centered", precision)(_p(a), _p(c), _p(out))
    return out[0]


def dq_transform_point(a, p, precision="f32"):
    a = np.ascontiguousarray(np.atleast_1d(a), DQ_DTYPE)
    p = np.ascontiguousarray(p, np.float32)
    out = np.zeros(3, np.float32)
    _fn("cfo_dq_transform_point", precision)(_p(a), _p(p), _p(out))
    return out


def dq_transform_point_centered(a, p, c, precision="f32"):
    a = np.ascontiguousarray(np.atleast_1d(a), DQ_DTYPE)
    p = np.ascontiguousarray(p, np.float32)
    c = np.ascontiguousarray(c, np.float32)
    out = np.zeros(3, np.float32)
    _fn("cfo_dq_transform_point_centered", precision)(_p(a), _p(p), _p(c), _p(out))
    return out


def skin(canon, ids, ws, nodes, transforms, precision="f32"):
    canon = np.ascontiguousarray(canon, np.float32)
    ids = np.ascontiguousarray(ids, np.int32)
    ws = np.ascontiguousarray(ws, np.float32)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    transforms = np.ascontiguousarray(transforms, DQ_DTYPE)
    out = np.zeros_like(canon)
    _fn("cfo_skin", precision)(_p(canon), _p(ids), _p(ws), canon.shape[0], _p(nodes), _p(transforms),
                               nodes.shape[0], _p(out))
    return out


def apply_twist(transforms, dx, max_rot=0.0, max_trans=0.0, scale=1.0, precision="f32"):
    T = np.array(transforms, DQ_DTYPE, copy=True)
    dx = np.ascontiguousarray(dx, np.float32)
    _fn("cfo_apply_twist", precision)(_p(T), _p(dx), T.shape[0], ctypes.c_float(max_rot), ctypes.c_float(max_trans),
                                      ctypes.c_float(scale))
    return T


def assemble(corrs, nodes, transforms, row_ptr, col_idx, lambda_smooth=1.0, lambda_damping=1e-2,
             precision="f64", nthreads=1):
    corrs = np.ascontiguousarray(corrs, CORR_DTYPE)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    transforms = np.ascontiguousarray(transforms, DQ_DTYPE)
    n = nodes.shape[0]
    A = np.zeros((len(col_idx), 6, 6), np.float64)
    b = np.zeros(n * 6, np.float64)
    f = _fn("cfo_assemble", precision)
    f.restype = ctypes.c_double
    e = f(_p(corrs), corrs.shape[0], _p(nodes), _p(transforms), n, _p(row_ptr), _p(col_idx),
          ctypes.c_float(lambda_smooth), ctypes.c_float(lambda_damping), _p(A), _p(b), nthreads)
    return A, b, e


def linearize_solve(corrs, nodes, transforms, prm, row_ptr=None, col_idx=None, precision="f64", nthreads=1):
    """GaussNewtonSolver::solve restated: returns (dx[N*6], iterations,
    energy, final_r, fallbacks)."""
    corrs = np.ascontiguousarray(corrs, CORR_DTYPE)
    nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
    transforms = np.ascontiguousarray(transforms, DQ_DTYPE)
    if row_ptr is None:
        row_ptr, col_idx = build_pattern(nodes)
    n = nodes.shape[0]
    dx = np.zeros(n * 6, np.float32)
    st = np.zeros(3, np.float64)
    f = _fn("cfo_linearize_solve", precision)
    f.restype = ctypes.c_int
    it = f(_p(corrs), corrs.shape[0], _p(nodes), _p(transforms), n, _p(row_ptr), _p(col_idx), ctypes.byref(prm),
           _p(dx), _p(st), nthreads)
    return dx, it, st[0], st[1], int(st[2])


def gn_solve(problem, prm, max_rot=0.0, max_trans=0.0, scale=1.0, transforms=None, precision="f64", nthreads=1):
    """G GN iterations with re-skinning (the cf_gn_solve schedule).
    Returns (transforms, energies[G+1], pcg_iters[G])."""
    nodes = np.ascontiguousarray(problem.nodes, NODE_DTYPE)
    corrs = np.ascontiguousarray(problem.corrs, CORR_DTYPE)
    canon = np.ascontiguousarray(problem.canon, np.float32)
    T = np.array(problem.init_transforms if transforms is None else transforms, DQ_DTYPE, copy=True)
    row_ptr, col_idx = build_pattern(nodes)
    G = prm.gn_iterations
    energies = np.zeros(G + 1, np.float64)
    iters = np.zeros(max(G, 1), np.int32)
    _fn("cfo_gn_solve", precision)(_p(canon), _p(corrs), corrs.shape[0], _p(nodes), nodes.shape[0], _p(row_ptr),
                                   _p(col_idx), ctypes.byref(prm), ctypes.c_float(max_rot),
                                   ctypes.c_float(max_trans), ctypes.c_float(scale), _p(T), _p(energies), _p(iters),
                                   nthreads)
    return T, energies, iters[:G]


def energy(problem, transforms, lambda_smooth, precision="f64", nthreads=1):
    nodes = np.ascontiguousarray(problem.nodes, NODE_DTYPE)
    corrs = np.ascontiguousarray(problem.corrs, CORR_DTYPE)
    canon = np.ascontiguousarray(problem.canon, np.float32)
    T = np.ascontiguousarray(transforms, DQ_DTYPE)
    f = _fn("cfo_energy", precision)
    f.restype = ctypes.c_double
    return f(_p(canon), _p(corrs), corrs.shape[0], _p(nodes), _p(T), nodes.shape[0], ctypes.c_float(lambda_smooth),
             nthreads)


# ---- projective correspondence search (oracle/cf_oracle_corr.c) ----


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def find_correspondences(frame, dist_threshold, angle_threshold, view_threshold, search_radius_px, pixels=None,
                         pixel_knn=None, pixel_knn_w=None):
    """find_correspondences_kernel (kernels/tsdf_kernels.cu:386-563) over all
    pixels of `frame` (a synth.CorrFrame) or over `pixels` (int array).
    Returns (records CORR_DTYPE[n], valid count, debug counters int[6])."""
    L = lib()
    f = L.cfo_find_correspondences
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5 + \
        [ctypes.c_float] * 3 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    lv, ln = _f32(frame.live_vertices), _f32(frame.live_normals)
    d, dn = _f32(frame.depth), _f32(frame.depth_normals)
    cam, cw, wc = _f32(frame.cam), _f32(frame.T_cam_world), _f32(frame.T_world_cam)
    pk = np.ascontiguousarray(frame.pixel_knn if pixel_knn is None else pixel_knn, np.int32)
    pw = _f32(frame.pixel_knn_w if pixel_knn_w is None else pixel_knn_w)
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.int32)
    n = frame.width * frame.height if pix is None else pix.shape[0]
    out = np.zeros(n, CORR_DTYPE)
    stats = np.zeros(6, np.int32)
    nv = f(_p(lv), _p(ln), _p(d), _p(dn), frame.width, frame.height, _p(cam), _p(cw), _p(wc), _p(pk), _p(pw),
           dist_threshold, angle_threshold, view_threshold, int(search_radius_px), _p(pix), int(n), _p(out),
           _p(stats))
    return out, int(nv), stats


def compute_pixel_knn(hit_voxel_idx, voxel_knn, voxel_knn_w):
    """compute_pixel_knn_kernel (kernels/tsdf_kernels.cu:573-604)."""
    L = lib()
    f = L.cfo_compute_pixel_knn
    f.restype = None
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                  ctypes.c_void_p, ctypes.c_void_p]
    hit = np.ascontiguousarray(hit_voxel_idx, np.int32)
    vk = np.ascontiguousarray(voxel_knn, np.int32)
    vw = _f32(voxel_knn_w)
    P = hit.shape[0]
    pk = np.zeros((P, 4), np.int32)
    pw = np.zeros((P, 4), np.float32)
    f(_p(hit), P, _p(vk), _p(vw), vk.shape[0], _p(pk), _p(pw))
    return pk, pw


# ---- live-surface rasterisation (oracle/cf_oracle_raster.c) ----


def rasterize(frame, warped=None, width=None, height=None):
    """rasterize_triangles_z_kernel + resolve_rasterized_triangles_kernel
    (src/mesh_raster_kernels.cu:76-200) of `frame` (a synth.MeshFrame) with
    its warped vertices (or `warped`).  Returns (live vertices f32[P,3],
    live normals f32[P,3], hit voxel int32[P], depth keys uint64[P])."""
    L = lib()
    f = L.cfo_rasterize
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 8
    W = frame.width if width is None else width
    H = frame.height if height is None else height
    canon = _f32(frame.canonical)
    wv = _f32(frame.warped if warped is None else warped)
    tris = np.ascontiguousarray(frame.triangles, np.int32)
    cam, cw = _f32(frame.cam), _f32(frame.T_cam_world)
    grid = np.array(list(frame.grid_origin) + [frame.voxel_size], np.float32)
    dims = np.ascontiguousarray(frame.dims, np.int32)
    P = W * H
    lv = np.zeros((P, 3), np.float32)
    ln = np.zeros((P, 3), np.float32)
    hit = np.zeros(P, np.int32)
    z = np.zeros(P, np.uint64)
    f(_p(canon), _p(wv), _p(tris), canon.shape[0], tris.shape[0], W, H, _p(cam), _p(cw), _p(grid), _p(dims),
      _p(lv), _p(ln), _p(hit), _p(z))
    return lv, ln, hit, z


def voxel_of_points(points, grid_origin, voxel_size, dims):
    """The canonical voxel of each point (src/skinning_kernels.cu:13-24), -1 outside."""
    L = lib()
    f = L.cfo_voxel_of_points
    f.restype = None
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    pts = _f32(points)
    grid = np.array(list(grid_origin) + [voxel_size], np.float32)
    dims = np.ascontiguousarray(dims, np.int32)
    out = np.zeros(pts.shape[0], np.int32)
    f(_p(pts), pts.shape[0], _p(grid), _p(dims), _p(out))
    return out


# ---- the GN step's acceptance (oracle/cf_oracle_ls.c) ----


def scale_delta(dx, max_rot, max_trans, scale):
    """upload_scaled_delta_x (include/fusion_app.h:1352-1375)."""
    L = lib()
    f = L.cfo_scale_delta
    f.restype = None
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_void_p]
    d = _f32(dx).reshape(-1)
    out = np.zeros_like(d)
    f(_p(d), d.size // 6, max_rot, max_trans, scale, _p(out))
    return out


def update_stats(dx, update_scale, max_rot, max_trans):
    """The increment statistics (include/fusion_app.h:427-458): (sums f64[4], maxima f32[4], finite)."""
    L = lib()
    f = L.cfo_update_stats
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_void_p,
                  ctypes.c_void_p]
    d = _f32(dx).reshape(-1)
    sums = np.zeros(4, np.float64)
    maxima = np.zeros(4, np.float32)
    fin = f(_p(d), d.size // 6, update_scale, max_rot, max_trans, _p(sums), _p(maxima))
    return sums, maxima, bool(fin)


def corr_rmse(recs):
    """correspondence_rmse (include/fusion_app.h:1331-1350): (sum w r^2, sum w, rmse)."""
    L = lib()
    f = L.cfo_corr_rmse
    f.restype = None
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    r = np.ascontiguousarray(recs)
    out = np.zeros(2, np.float64)
    f(_p(r), r.shape[0], _p(out))
    rmse = float(np.sqrt(out[0] / out[1])) if out[1] > 0 else float("inf")
    return float(out[0]), float(out[1]), rmse


# ---- warped TSDF integration (oracle/cf_oracle_tsdf.c) ----


def _tsdf_fn(name, restype, argtypes):
    f = getattr(lib(), name)
    f.restype = restype
    f.argtypes = argtypes
    return f


def tsdf_reset(num_voxels):
    """The TSDFVolume constructor's voxels (src/tsdf_volume.cu:11-19): float32 (n, 3), the third
    column the colour bytes 128 128 128 0."""
    vox = np.zeros((num_voxels, 3), np.float32)
    _tsdf_fn("cfo_tsdf_reset", None, [ctypes.c_void_p, ctypes.c_longlong])(_p(vox), num_voxels)
    return vox


def tsdf_world_to_camera(camera_pose):
    """T_cam_world as src/tsdf_volume.cu:34-50 forms it: a 4x4 float32 matrix."""
    pose = np.ascontiguousarray(camera_pose, np.float32)
    rows = np.zeros(12, np.float32)
    _tsdf_fn("cfo_tsdf_world_to_camera", None, [ctypes.c_void_p, ctypes.c_void_p])(_p(pose), _p(rows))
    out = np.eye(4, dtype=np.float32)
    out[:3] = rows.reshape(3, 4)
    return out


def tsdf_centres(dims, origin, voxel_size, lo=0, hi=None):
    """The centres of voxels [lo, hi) (kernels/tsdf_kernels.cu:117-121), float32 (n, 3)."""
    dims = np.ascontiguousarray(dims, np.int32)
    hi = int(np.prod(dims.astype(np.int64))) if hi is None else hi
    org = np.ascontiguousarray(origin, np.float32)
    out = np.zeros((hi - lo, 3), np.float32)
    _tsdf_fn("cfo_tsdf_centres", None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_longlong,
                                        ctypes.c_longlong, ctypes.c_void_p])(_p(dims), _p(org), voxel_size, lo, hi,
                                                                              _p(out))
    return out


def tsdf_integrate(vox, params, depth, cam, camera_pose, live=None, counts=None, gate=False, min_opt=0, lo=0,
                   hi=None):
    """tsdf_integrate_kernel (kernels/tsdf_kernels.cu:85-174) over voxels [lo, hi) of `vox`
    (float32 (n, 3), updated in place).  params = dict(dims, origin, voxel_size, truncation,
    decay_alpha, max_weight); cam = (fx, fy, cx, cy, width, height); live = the warped centres of
    the range (None: rigid).  Returns the number of voxels updated."""
    dims = np.ascontiguousarray(params["dims"], np.int32)
    hi = vox.shape[0] if hi is None else hi
    org = np.ascontiguousarray(params["origin"], np.float32)
    rows = np.ascontiguousarray(tsdf_world_to_camera(camera_pose)[:3].reshape(-1))
    c = np.array(cam[:4], np.float32)
    d = np.ascontiguousarray(depth, np.float32).reshape(-1)
    lv = None if live is None else np.ascontiguousarray(live, np.float32)
    cn = None if counts is None else np.ascontiguousarray(counts, np.int32)
    assert vox.dtype == np.float32 and vox.flags.c_contiguous
    f = _tsdf_fn("cfo_tsdf_integrate", ctypes.c_longlong,
                 [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_longlong, ctypes.c_longlong])
    return f(_p(vox), _p(dims), _p(org), params["voxel_size"], params["truncation"], _p(d), int(cam[4]), int(cam[5]),
             _p(c), _p(rows), _p(lv), _p(cn), int(bool(gate)), min_opt, params["decay_alpha"], params["max_weight"],
             lo, hi)


def mark_optimized_voxels(recs, vidx_map, dims, frame, counts, frames):
    """mark_optimized_voxels_kernel (kernels/tsdf_kernels.cu:606-650) on the correspondence records;
    counts and frames (int32) are updated in place."""
    valid = np.ascontiguousarray(recs["valid"], np.uint8)
    weight = np.ascontiguousarray(recs["weight"], np.float32)
    vm = np.ascontiguousarray(vidx_map, np.int32)
    dims = np.ascontiguousarray(dims, np.int32)
    assert counts.dtype == np.int32 and frames.dtype == np.int32
    _tsdf_fn("cfo_mark_optimized_voxels", None,
             [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
              ctypes.c_void_p, ctypes.c_void_p])(_p(valid), _p(weight), _p(vm), vm.size, _p(dims), frame, _p(counts),
                                                 _p(frames))


# ---- voxel kNN field (oracle/cf_oracle_voxelknn.c) ----


def voxel_knn(vox, params, nodes, lo=0, hi=None, nthreads=1):
    """compute_voxel_knn_kernel (src/warp_field.cu:299-405) over voxels [lo, hi) of `vox`
    (float32 (V, 3) voxel records); params = dict(dims, origin, voxel_size).  Returns
    (ids int32 (n, 4), ws float32 (n, 4)); with no nodes the arrays stay -2 / NaN (untouched)."""
    dims = np.ascontiguousarray(params["dims"], np.int32)
    hi = vox.shape[0] if hi is None else hi
    org = np.ascontiguousarray(params["origin"], np.float32)
    nd = np.ascontiguousarray(nodes, NODE_DTYPE)
    v = np.ascontiguousarray(vox, np.float32)
    ids = np.full((hi - lo, 4), -2, np.int32)
    ws = np.full((hi - lo, 4), np.nan, np.float32)
    _tsdf_fn("cfo_voxel_knn", None,
             [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
              ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int])(
        _p(v), _p(dims), _p(org), params["voxel_size"], _p(nd), nd.shape[0], lo, hi, _p(ids), _p(ws), nthreads)
    return ids, ws


def voxel_knn_list(vox, params, nodes, vidx, nthreads=1):
    """The same for the voxels listed in `vidx` (int64): (ids (n, 4), ws (n, 4))."""
    dims = np.ascontiguousarray(params["dims"], np.int32)
    org = np.ascontiguousarray(params["origin"], np.float32)
    nd = np.ascontiguousarray(nodes, NODE_DTYPE)
    v = np.ascontiguousarray(vox, np.float32)
    vi = np.ascontiguousarray(vidx, np.int64)
    ids = np.full((vi.size, 4), -2, np.int32)
    ws = np.full((vi.size, 4), np.nan, np.float32)
    _tsdf_fn("cfo_voxel_knn_list", None,
             [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
              ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int])(
        _p(v), _p(dims), _p(org), params["voxel_size"], _p(nd), nd.shape[0], _p(vi), vi.size, _p(ids), _p(ws),
        nthreads)
    return ids, ws
