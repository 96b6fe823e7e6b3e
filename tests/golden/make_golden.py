"""Generates tests/golden/se3_kat.npz: known-answer vectors of the reference's
own se3 functions (CUDAFusion include/se3_math.cuh, include/fusion_math.h),
compiled for the host from the reference sources by oracle/Makefile (target
`ref`) and run here.  Needs the reference checkout (REF, by default a
`reference` directory beside this repository); the committed .npz is what the
tests read.

    python tests/golden/make_golden.py
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from cudafusion_b200 import synth  # noqa: E402
from cudafusion_b200.types import DQ_DTYPE  # noqa: E402

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libcfref_host.so")


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), REF_SO], check=True)
    ref = ctypes.CDLL(REF_SO)
    rng = np.random.default_rng(20261203)
    n = 600
    scales = np.array([1e-8, 1e-7, 5e-7, 1e-5, 1e-3, 0.05, 0.3, 1.0, 2.5, 3.1])
    tw = (rng.normal(size=(n, 6)) * scales[rng.integers(0, len(scales), n)][:, None]).astype(np.float32)
    tw[:20, :3] = 0.0  # pure translations
    exp_out = np.zeros((n, 16), np.float32)
    m2dq_out = np.zeros(n, DQ_DTYPE)
    twist_dq = np.zeros(n, DQ_DTYPE)
    for i in range(n):
        ref.ref_exp_se3(P(tw[i]), P(exp_out[i]))
        ref.ref_mat4_to_dq(P(exp_out[i]), P(m2dq_out[i:i + 1]))
        ref.ref_dq_from_twist(P(tw[i]), P(twist_dq[i:i + 1]))
    # rotation matrices with negative trace exercise the other three branches
    mats = np.zeros((n, 16), np.float32)
    for i in range(n):
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        ang = rng.uniform(2.0, np.pi) if i % 2 == 0 else rng.uniform(0, np.pi)
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        R = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
        T = np.eye(4)
        T[:3, :3] = R
        T[:3, 3] = rng.normal(size=3) * 0.1
        mats[i] = T.astype(np.float32).ravel()
    mats_dq = np.zeros(n, DQ_DTYPE)
    for i in range(n):
        ref.ref_mat4_to_dq(P(mats[i]), P(mats_dq[i:i + 1]))
    a = twist_dq.copy()
    b = np.roll(twist_dq, 7)
    mul_out = np.zeros(n, DQ_DTYPE)
    pts = (rng.normal(size=(n, 3)) * 0.5).astype(np.float32)
    ctr = (rng.normal(size=(n, 3)) * 0.5).astype(np.float32)
    cent_out = np.zeros(n, DQ_DTYPE)
    tp_out = np.zeros((n, 3), np.float32)
    tpc_out = np.zeros((n, 3), np.float32)
    for i in range(n):
        ref.ref_dq_mul(P(a[i:i + 1]), P(b[i:i + 1]), P(mul_out[i:i + 1]))
        ref.ref_dq_centered(P(a[i:i + 1]), P(ctr[i]), P(cent_out[i:i + 1]))
        ref.ref_dq_transform_point(P(a[i:i + 1]), P(pts[i]), P(tp_out[i]))
        ref.ref_dq_transform_point_centered(P(a[i:i + 1]), P(pts[i]), P(ctr[i]), P(tpc_out[i]))
    # skinning: a small sphere problem with a random warp
    prob = synth.sphere_problem(num_nodes=64, num_corrs=500, radius=0.3, node_radius=0.06, seed=7)
    T = prob.gt_transforms.copy()
    ids = np.ascontiguousarray(prob.corrs["node_ids"], np.int32)
    ws = np.ascontiguousarray(prob.corrs["node_ws"], np.float32)
    ids[::37, 3] = -1  # missing slots
    ws[::41, 2] = 0.0  # zero weights
    skin_out = np.zeros((prob.num_corrs, 3), np.float32)
    ref.ref_skin(P(prob.canon), P(ids), P(ws), prob.num_corrs, P(prob.nodes), P(T), prob.num_nodes, P(skin_out))
    out = os.path.join(ROOT, "tests", "golden", "se3_kat.npz")
    np.savez_compressed(
        out,
        tw=tw, exp_out=exp_out, m2dq_out=m2dq_out.view(np.uint8), twist_dq=twist_dq.view(np.uint8),
        mats=mats, mats_dq=mats_dq.view(np.uint8), a=a.view(np.uint8), b=b.view(np.uint8),
        mul_out=mul_out.view(np.uint8), pts=pts, ctr=ctr, cent_out=cent_out.view(np.uint8), tp_out=tp_out,
        tpc_out=tpc_out, skin_nodes=prob.nodes.view(np.uint8), skin_T=T.view(np.uint8), skin_canon=prob.canon,
        skin_ids=ids, skin_ws=ws, skin_out=skin_out,
    )
    print("wrote", out)


if __name__ == "__main__":
    main()
