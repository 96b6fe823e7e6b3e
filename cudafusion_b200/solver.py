"""Python mirror of CUDAFusion's solve-path call surface.

GaussNewtonSolver  include/solver.h:10-89
WarpField          include/warp_field.h:12-126 (the subset on the solve path)

Both call the sm_100a library through its C ABI.  Device memory is held in
torch tensors (torch is the allocator and stream provider here, nothing
else).  Like the reference, methods synchronise before they return unless
their docstring says otherwise.
"""
import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import check
from .types import CORR_DTYPE, DQ_DTYPE, NODE_DTYPE, identity_transforms


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def to_device(arr, device="cuda"):
    """Uploads a numpy array (structured or plain) as a flat uint8/float tensor
    whose bytes are the array's bytes."""
    a = np.ascontiguousarray(arr)
    if a.dtype.fields is not None:
        return torch.from_numpy(a.view(np.uint8).reshape(-1).copy()).to(device)
    return torch.from_numpy(a.copy()).to(device)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


@dataclass
class Params:
    """GaussNewtonSolver::Params (include/solver.h:13-22), same defaults."""

    gn_iterations: int = 3
    pcg_iterations: int = 10
    pcg_tolerance: float = 1e-4
    lambda_smooth: float = 1.0
    lambda_rot: float = 1.0
    lambda_damping: float = 1e-2
    debug: bool = False

    def c(self):
        return _lib.GNParams(
            self.gn_iterations,
            self.pcg_iterations,
            self.pcg_tolerance,
            self.lambda_smooth,
            self.lambda_rot,
            self.lambda_damping,
            int(bool(self.debug)),
        )


class DeviceProblem:
    """A solve problem resident on the device (nodes, canonical points,
    correspondences), uploaded once."""

    def __init__(self, problem, device="cuda"):
        self.num_nodes = problem.num_nodes
        self.num_corrs = problem.num_corrs
        self.nodes = to_device(problem.nodes, device)
        self.canon = to_device(np.ascontiguousarray(problem.canon, np.float32), device)
        self.corrs = to_device(problem.corrs, device)
        self.init_transforms = to_device(problem.init_transforms, device)

    def c(self, max_rot=0.0, max_trans=0.0, update_scale=1.0):
        return _lib.Problem(
            self.nodes.data_ptr(),
            self.num_nodes,
            self.canon.data_ptr() if self.num_corrs else None,
            self.corrs.data_ptr() if self.num_corrs else None,
            self.num_corrs,
            max_rot,
            max_trans,
            update_scale,
        )


class GaussNewtonSolver:
    """include/solver.h:10-89 on the B200 kernels.

    solve()      one linearisation -> delta_x (GaussNewtonSolver::solve)
    gn_solve()   G full GN iterations with re-skinning and node updates
    """

    Params = Params

    def __init__(self, params=None, max_nodes=8192, max_corrs=1 << 20):
        self.params = params if params is not None else Params()
        self.max_nodes = max_nodes
        self.max_corrs = max_corrs
        h = ctypes.c_void_p()
        cp = self.params.c()
        check(_lib.lib().cf_gn_create(ctypes.byref(cp), max_nodes, max_corrs, ctypes.byref(h)), "cf_gn_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib.lib().cf_gn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params):
        self.params = params
        cp = params.c()
        check(_lib.lib().cf_gn_set_params(self._h, ctypes.byref(cp)), "cf_gn_set_params")

    def set_option(self, option, value):
        check(_lib.lib().cf_gn_set_option(self._h, option, int(value)), "cf_gn_set_option")

    def get_option(self, option):
        v = ctypes.c_int()
        check(_lib.lib().cf_gn_get_option(self._h, option, ctypes.byref(v)))
        return v.value

    def set_arap_consistent(self, on=True):
        self.set_option(_lib.CF_OPT_ARAP_CONSISTENT, 1 if on else 0)

    def invalidate_pattern(self):
        check(_lib.lib().cf_gn_invalidate_pattern(self._h))

    def solve(self, corrs, num_corrs, d_nodes, d_transforms, num_nodes, delta_x=None, stream=None, sync=True):
        """GaussNewtonSolver::solve (kernels/solver_kernels.cu:543-570).
        corrs, d_nodes, d_transforms: device byte tensors of the reference
        structs.  Returns delta_x (float32 [6*num_nodes] on the device); a
        passed tensor is reused when large enough (the reference always
        reallocates it, solver_kernels.cu:551)."""
        if delta_x is None or delta_x.numel() < 6 * num_nodes:
            delta_x = torch.zeros(max(6 * num_nodes, 1), dtype=torch.float32, device=d_nodes.device)
        st = _stream_ptr(stream)
        check(
            _lib.lib().cf_gn_linearize_solve(
                self._h, _ptr(corrs), num_corrs, _ptr(d_nodes), _ptr(d_transforms), num_nodes, _ptr(delta_x), st
            ),
            "cf_gn_linearize_solve",
        )
        if sync:
            check(_lib.lib().cf_gn_check(self._h, st), "cf_gn_linearize_solve")
        return delta_x

    def gn_solve(self, dproblem, d_transforms, max_rot=0.0, max_trans=0.0, update_scale=1.0, stats=True,
                 stream=None):
        """G Gauss-Newton iterations (params.gn_iterations) updating
        d_transforms in place.  With stats=True returns a dict and
        synchronises; otherwise asynchronous and returns None."""
        p = dproblem.c(max_rot, max_trans, update_scale)
        st = _stream_ptr(stream)
        if stats:
            s = _lib.SolveStats()
            check(_lib.lib().cf_gn_solve(self._h, ctypes.byref(p), _ptr(d_transforms), ctypes.byref(s), st),
                  "cf_gn_solve")
            G = s.gn_iterations_run
            return dict(
                energy_initial=s.energy_initial,
                energy_final=s.energy_final,
                energy=[s.energy_per_iter[g] for g in range(G + 1)],
                pcg_iterations=[s.pcg_iterations[g] for g in range(G)],
                pcg_residual=[s.pcg_residual[g] for g in range(G)],
                num_blocks=s.num_blocks,
                precond_fallbacks=s.precond_fallbacks,
                error_flags=s.error_flags,
            )
        check(_lib.lib().cf_gn_solve(self._h, ctypes.byref(p), _ptr(d_transforms), None, st), "cf_gn_solve")
        return None

    def gn_solve_batched(self, dproblems, d_transforms, max_rot=0.0, max_trans=0.0, update_scale=1.0, stats=True,
                         stream=None):
        """cf_gn_solve_batched: every problem of `dproblems` (DeviceProblem)
        through G GN iterations in one pass, d_transforms[i] updated in place.
        With stats=True returns one dict per problem and synchronises."""
        n = len(dproblems)
        probs = (_lib.Problem * max(n, 1))(*[d.c(max_rot, max_trans, update_scale) for d in dproblems])
        ptrs = (ctypes.c_void_p * max(n, 1))(*[t.data_ptr() for t in d_transforms])
        st = _stream_ptr(stream)
        if not stats:
            check(_lib.lib().cf_gn_solve_batched(self._h, probs, n, ptrs, None, st), "cf_gn_solve_batched")
            return None
        out = (_lib.SolveStats * max(n, 1))()
        check(_lib.lib().cf_gn_solve_batched(self._h, probs, n, ptrs, out, st), "cf_gn_solve_batched")
        res = []
        for k in range(n):
            s = out[k]
            G = s.gn_iterations_run
            res.append(dict(
                energy_initial=s.energy_initial,
                energy_final=s.energy_final,
                energy=[s.energy_per_iter[g] for g in range(G + 1)],
                pcg_iterations=[s.pcg_iterations[g] for g in range(G)],
                pcg_residual=[s.pcg_residual[g] for g in range(G)],
                num_blocks=s.num_blocks,
                precond_fallbacks=s.precond_fallbacks,
                error_flags=s.error_flags,
            ))
        return res

    def autotune(self, dproblems, d_transforms, max_rot=0.0, max_trans=0.0, update_scale=1.0, stream=None):
        """cf_gn_autotune over `dproblems` (one: the single solve; several:
        the batched solve); returns the choice as a dict."""
        n = len(dproblems)
        probs = (_lib.Problem * n)(*[d.c(max_rot, max_trans, update_scale) for d in dproblems])
        ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in d_transforms])
        r = _lib.TuneResult()
        check(_lib.lib().cf_gn_autotune(self._h, probs, n, ptrs, ctypes.byref(r), _stream_ptr(stream)),
              "cf_gn_autotune")
        return {k: getattr(r, k) for k, _ in _lib.TuneResult._fields_}

    def last_stats(self, stream=None):
        """Statistics of the handle's last solve (cf_gn_last_stats)."""
        s = _lib.SolveStats()
        check(_lib.lib().cf_gn_last_stats(self._h, ctypes.byref(s), 1, _stream_ptr(stream)), "cf_gn_last_stats")
        G = s.gn_iterations_run
        return dict(energy_initial=s.energy_initial, energy_final=s.energy_final,
                    energy=[s.energy_per_iter[g] for g in range(G + 1)], init_rejected=s.init_rejected,
                    energy_warm_start=s.energy_warm_start, energy_predicted=s.energy_predicted,
                    pcg_iterations=[s.pcg_iterations[g] for g in range(G)], error_flags=s.error_flags)

    def profile_enable(self, on=True):
        """Per-phase CUDA-event timing of every launch (resets totals)."""
        check(_lib.lib().cf_gn_profile_enable(self._h, 1 if on else 0))

    def profile_read(self):
        """{phase: (device ms summed, kernel launches)} since profile_enable."""
        n = _lib.CF_PROF_SLOTS
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int * n)()
        check(_lib.lib().cf_gn_profile_read(self._h, ms, cnt, n))
        return {_lib.lib().cf_gn_profile_name(i).decode(): (ms[i], cnt[i]) for i in range(n) if cnt[i]}

    def launch_count(self):
        v = ctypes.c_longlong()
        check(_lib.lib().cf_gn_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def system(self, stream=None):
        """system_matrix() and rhs() (include/solver.h:38-39) as host arrays:
        (row_ptr, col_idx, values[nnzb,6,6], rhs[6N])."""
        n = ctypes.c_int()
        nb = ctypes.c_int()
        st = _stream_ptr(stream)
        check(_lib.lib().cf_gn_get_system(self._h, ctypes.byref(n), ctypes.byref(nb), None, None, None, None, st))
        row_ptr = np.zeros(n.value + 1, np.int32)
        col_idx = np.zeros(max(nb.value, 1), np.int32)
        values = np.zeros((max(nb.value, 1), 6, 6), np.float32)
        rhs = np.zeros(6 * max(n.value, 1), np.float32)
        check(
            _lib.lib().cf_gn_get_system(
                self._h,
                ctypes.byref(n),
                ctypes.byref(nb),
                row_ptr.ctypes.data_as(ctypes.c_void_p),
                col_idx.ctypes.data_as(ctypes.c_void_p),
                values.ctypes.data_as(ctypes.c_void_p),
                rhs.ctypes.data_as(ctypes.c_void_p),
                st,
            )
        )
        return row_ptr, col_idx[: nb.value], values[: nb.value], rhs[: 6 * n.value]

    def system_matrix(self):
        row_ptr, col_idx, values, _ = self.system()
        return row_ptr, col_idx, values

    def rhs(self):
        return self.system()[3]


class WarpField:
    """include/warp_field.h:12-126, solve-path subset: node storage, the
    transforms and their save/restore, and the twist update.  Graph
    construction (add_nodes_*, prune_nodes, compute_voxel_knn) is not part of
    this library."""

    MAX_NODES = 8192

    def __init__(self, node_radius, max_nodes=MAX_NODES, device="cuda"):
        self.node_radius = node_radius
        self.max_nodes = max_nodes
        self._n = 0
        self._d_nodes = torch.zeros(max_nodes * NODE_DTYPE.itemsize, dtype=torch.uint8, device=device)
        self._d_T = torch.zeros(max_nodes * DQ_DTYPE.itemsize, dtype=torch.uint8, device=device)
        self._d_Tprev = torch.zeros_like(self._d_T)

    def num_nodes(self):
        return self._n

    def device_nodes(self):
        return self._d_nodes

    def device_transforms(self):
        return self._d_T

    def device_transforms_prev(self):
        return self._d_Tprev

    def upload_nodes(self, nodes):
        """WarpField::upload_nodes (src/warp_field.cu:1160-1177): resets the
        transforms to identity when the node count changes."""
        nodes = np.ascontiguousarray(nodes, NODE_DTYPE)
        n = min(nodes.shape[0], self.max_nodes)
        self._d_nodes[: n * NODE_DTYPE.itemsize].copy_(torch.from_numpy(nodes[:n].view(np.uint8).reshape(-1)))
        if n != self._n:
            ident = torch.from_numpy(identity_transforms(n).view(np.uint8).reshape(-1))
            self._d_T[: n * DQ_DTYPE.itemsize].copy_(ident)
            self._d_Tprev[: n * DQ_DTYPE.itemsize].copy_(ident)
        self._n = n

    def upload_transforms(self, transforms):
        """WarpField::upload_transforms (src/warp_field.cu:1179-1192)."""
        t = np.ascontiguousarray(transforms, DQ_DTYPE)
        n = min(t.shape[0], self.max_nodes)
        if self._n == 0:
            self._n = n
        n = min(n, self._n)
        b = torch.from_numpy(t[:n].view(np.uint8).reshape(-1))
        self._d_T[: n * DQ_DTYPE.itemsize].copy_(b)
        self._d_Tprev[: n * DQ_DTYPE.itemsize].copy_(b)

    def download_nodes(self):
        return self._d_nodes[: self._n * NODE_DTYPE.itemsize].cpu().numpy().view(NODE_DTYPE).copy()

    def download_transforms(self):
        return self._d_T[: self._n * DQ_DTYPE.itemsize].cpu().numpy().view(DQ_DTYPE).copy()

    def save_transforms(self):
        """WarpField::save_transforms (src/warp_field.cu:1106-1110)."""
        nb = self._n * DQ_DTYPE.itemsize
        self._d_Tprev[:nb].copy_(self._d_T[:nb])

    def restore_transforms(self):
        """WarpField::restore_transforms (src/warp_field.cu:1112-1119)."""
        nb = self._n * DQ_DTYPE.itemsize
        self._d_T[:nb].copy_(self._d_Tprev[:nb])
        torch.cuda.current_stream().synchronize()

    def reset_transforms(self):
        """WarpField::reset_transforms (src/warp_field.cu:1143-1148)."""
        ident = torch.from_numpy(identity_transforms(self._n).view(np.uint8).reshape(-1))
        self._d_T[: self._n * DQ_DTYPE.itemsize].copy_(ident)

    def apply_twist_increment(self, delta_x, max_rot, max_trans, update_scale=1.0, stream=None):
        """WarpField::apply_twist_increment (src/warp_field.cu:1121-1141):
        T_i <- exp(clamp(update_scale * dx_i)) * T_i, synchronised."""
        if self._n == 0:
            return
        st = _stream_ptr(stream)
        check(
            _lib.lib().cf_warp_apply_twist(
                _ptr(self._d_T), _ptr(delta_x), self._n, max_rot, max_trans, update_scale, st
            ),
            "cf_warp_apply_twist",
        )
        (stream or torch.cuda.current_stream()).synchronize()


def skin_points(points, node_ids, node_ws, d_nodes, d_transforms, num_nodes, out=None, stream=None):
    """warp_point over many points (include/se3_math.cuh:450-510); device
    tensors in, device float32 [M,3] out."""
    M = points.shape[0] if points.dim() == 2 else points.numel() // 3
    if out is None:
        out = torch.empty((M, 3), dtype=torch.float32, device=points.device)
    check(
        _lib.lib().cf_warp_skin_points(
            _ptr(points), _ptr(node_ids), _ptr(node_ws), M, _ptr(d_nodes), _ptr(d_transforms), num_nodes, _ptr(out),
            _stream_ptr(stream),
        ),
        "cf_warp_skin_points",
    )
    return out
