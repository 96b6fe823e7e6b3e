"""ctypes front end of the reference's own CUDA warp-field solve
(oracle/_ref/libcfref_cuda.so: kernels/solver_kernels.cu and
src/warp_field.cu unmodified, built for sm_100a with the reference's
--use_fast_math, driven by oracle/ref_cuda_harness.cu).

TEST AND REFERENCE-ARM INFRASTRUCTURE ONLY: used by the GPU parity tests and
by `bench.py --impl reference`.  Needs a GPU.

What each call runs in the reference:
  linearize_solve  GaussNewtonSolver::solve (kernels/solver_kernels.cu:543-570)
                   at the uploaded correspondences' own src
  system           system_matrix() / rhs() (include/solver.h:38-39) of the
                   last solve
  gn_solve         G x (warp_point skinning of the canonical points,
                   include/se3_math.cuh:450-510 -> GaussNewtonSolver::solve ->
                   WarpField::apply_twist_increment, src/warp_field.cu:1121-1141)
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libcfref_cuda.so")

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        L.ref_create.restype = vp
        L.ref_create.argtypes = [vp, vp, i]
        L.ref_destroy.argtypes = [vp]
        L.ref_upload.restype = i
        L.ref_upload.argtypes = [vp, vp, i, vp, vp, i, vp]
        L.ref_set_transforms.restype = i
        L.ref_set_transforms.argtypes = [vp, vp, i]
        L.ref_get_transforms.restype = i
        L.ref_get_transforms.argtypes = [vp, vp, i]
        L.ref_linearize_solve.restype = i
        L.ref_linearize_solve.argtypes = [vp, vp]
        L.ref_get_system.restype = i
        L.ref_get_system.argtypes = [vp, vp, vp, vp, vp]
        L.ref_gn_solve.restype = i
        L.ref_gn_solve.argtypes = [vp, i, f, f, f]
        L.ref_gn_solve_timed.restype = i
        L.ref_gn_solve_timed.argtypes = [vp, i, f, f, f, ctypes.POINTER(f)]
        L.ref_get_corrs.restype = i
        L.ref_get_corrs.argtypes = [vp, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class RefSolver:
    """The reference GaussNewtonSolver + WarpField with one synth.Problem
    uploaded.  Parameters mirror GaussNewtonSolver::Params
    (include/solver.h:13-22)."""

    def __init__(self, problem, gn_iterations=3, pcg_iterations=10, pcg_tolerance=1e-4, lambda_smooth=1.0,
                 lambda_rot=1.0, lambda_damping=1e-2, max_nodes=8192):
        L = lib()
        self.problem = problem
        self.N, self.M = problem.num_nodes, problem.num_corrs
        ip = (ctypes.c_int * 3)(gn_iterations, pcg_iterations, 0)
        fp = (ctypes.c_float * 4)(pcg_tolerance, lambda_smooth, lambda_rot, lambda_damping)
        self.h = ctypes.c_void_p(L.ref_create(ip, fp, max(max_nodes, self.N)))
        self._nodes = np.ascontiguousarray(problem.nodes)
        self._canon = np.ascontiguousarray(problem.canon, np.float32)
        self._corrs = np.ascontiguousarray(problem.corrs)
        self.upload(problem.init_transforms)

    def upload(self, transforms):
        """Nodes, canonical points, correspondences (with their src) and
        transforms, as the reference's DeviceArray / WarpField uploads."""
        T = np.ascontiguousarray(transforms)
        rc = lib().ref_upload(self.h, _p(self._nodes), self.N, _p(self._canon), _p(self._corrs), self.M, _p(T))
        if rc != 0:
            raise RuntimeError(f"reference upload failed: cudaError {rc}")

    def set_transforms(self, transforms):
        T = np.ascontiguousarray(transforms)
        rc = lib().ref_set_transforms(self.h, _p(T), self.N)
        if rc != 0:
            raise RuntimeError(f"reference set_transforms failed: cudaError {rc}")

    def transforms(self):
        out = np.zeros(self.N, self.problem.init_transforms.dtype)
        rc = lib().ref_get_transforms(self.h, _p(out), self.N)
        if rc != 0:
            raise RuntimeError(f"reference get_transforms failed: cudaError {rc}")
        return out

    def linearize_solve(self):
        """One GaussNewtonSolver::solve; delta_x [6N] (omega, v per node)."""
        dx = np.zeros(6 * self.N, np.float32)
        rc = lib().ref_linearize_solve(self.h, _p(dx))
        if rc != 0:
            raise RuntimeError(f"reference solve failed: cudaError {rc}")
        return dx

    def system(self):
        """(row_ptr, col_idx, values [nnzb, 36], rhs [6N]) of the last solve."""
        cap = 17 * self.N + 1
        row_ptr = np.zeros(self.N + 1, np.int32)
        col_idx = np.zeros(cap, np.int32)
        vals = np.zeros((cap, 36), np.float32)
        rhs = np.zeros(6 * self.N, np.float32)
        nnzb = lib().ref_get_system(self.h, _p(row_ptr), _p(col_idx), _p(vals), _p(rhs))
        if nnzb > cap:
            raise RuntimeError(f"reference pattern has {nnzb} blocks, more than the {cap} read back")
        return row_ptr, col_idx[:nnzb].copy(), vals[:nnzb].copy(), rhs

    def gn_solve(self, gn_iterations, max_rot=0.0, max_trans=0.0, update_scale=1.0, transforms=None):
        """G reference GN iterations from `transforms` (default: the
        problem's initial transforms); returns the final transforms."""
        self.set_transforms(self.problem.init_transforms if transforms is None else transforms)
        rc = lib().ref_gn_solve(self.h, gn_iterations, max_rot, max_trans, update_scale)
        if rc != 0:
            raise RuntimeError(f"reference GN solve failed: cudaError {rc}")
        return self.transforms()

    def gn_solve_timed(self, gn_iterations, max_rot=0.0, max_trans=0.0, update_scale=1.0):
        ms = ctypes.c_float()
        rc = lib().ref_gn_solve_timed(self.h, gn_iterations, max_rot, max_trans, update_scale, ctypes.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference GN solve failed: cudaError {rc}")
        return ms.value

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
