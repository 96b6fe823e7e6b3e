"""The TSDF integration oracle (oracle/cf_oracle_tsdf.c) on the CPU: against
an independent FP64 NumPy restatement of tsdf_integrate_kernel
(kernels/tsdf_kernels.cu:85-174) and of mark_optimized_voxels_kernel
(:606-650), against the reference's own outputs in tests/golden/tsdf_ref.npz
(made on a B200 by tests/golden/make_tsdf_golden.py), and the library's
host-side T_cam_world (src/tsdf_volume.cu:34-50) against the oracle's, bit
for bit."""
import os

import numpy as np
import pytest

from cudafusion_b200 import synth
from cudafusion_b200.types import CORR_DTYPE, DQ_DTYPE, NODE_DTYPE

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tsdf_ref.npz")


def _numpy_integrate(f, live=None, gate=False, min_opt=3):
    """FP64 restatement: the set of voxels updated and their new values."""
    p = f.params
    dims = np.asarray(p["dims"], np.int64)
    V = int(np.prod(dims))
    i = np.arange(V)
    x, y, z = i % dims[0], (i // dims[0]) % dims[1], i // (dims[0] * dims[1])
    org = np.asarray(p["origin"], np.float64)
    vs = float(p["voxel_size"])
    c = np.stack([org[0] + (x + 0.5) * vs, org[1] + (y + 0.5) * vs, org[2] + (z + 0.5) * vs], -1)
    if live is not None:
        c = live.astype(np.float64)
    pose = f.camera_pose.astype(np.float64)
    R = pose[:3, :3].T
    pc = c @ R.T - R @ pose[:3, 3]
    fx, fy, cx, cy = (float(v) for v in f.cam)
    with np.errstate(divide="ignore", invalid="ignore"):
        u = np.rint(fx * pc[:, 0] / pc[:, 2] + cx)
        v = np.rint(fy * pc[:, 1] / pc[:, 2] + cy)
    ok = (pc[:, 2] > 0) & (u >= 0) & (u < f.width) & (v >= 0) & (v < f.height)
    if gate:
        ok &= f.counts >= min_opt
    d = np.zeros(V)
    d[ok] = f.depth.astype(np.float64)[(v[ok] * f.width + u[ok]).astype(np.int64)]
    with np.errstate(invalid="ignore"):
        ok &= ~(d <= 0)
        sdf = d - pc[:, 2]
        ok &= ~(sdf < -float(p["truncation"]))
        obs = np.fmin(1.0, sdf / float(p["truncation"]))
    out = f.voxels.astype(np.float64)[:, :2].copy()
    dec = out[ok, 1] * float(np.float32(p["decay_alpha"]))
    nw = dec + 1.0
    out[ok, 0] = (out[ok, 0] * dec + obs[ok]) / nw
    out[ok, 1] = np.minimum(nw, float(p["max_weight"]))
    return ok, out


def _cam(f):
    return tuple(float(c) for c in f.cam) + (f.width, f.height)


@pytest.mark.parametrize("seed", [61, 62])
def test_rigid_against_numpy(oracle, seed):
    f = synth.tsdf_frame(96, 72, dims=(40, 32, 28), nodes_xy=(6, 5), invalid_frac=0.02, seed=seed)
    vox = f.voxels.copy()
    n = oracle.tsdf_integrate(vox, f.params, f.depth, _cam(f), f.camera_pose)
    ok, want = _numpy_integrate(f)
    changed = np.any(vox[:, :2] != f.voxels[:, :2], axis=1)
    assert n > 1000 and abs(n - ok.sum()) <= 2e-3 * n
    both = ok & changed
    assert both.sum() >= 0.998 * ok.sum()
    assert np.abs(vox[both, :2] - want[both]).max() < 1e-5
    # the colour bytes are never written
    assert np.array_equal(vox.view(np.uint32)[:, 2], f.voxels.view(np.uint32)[:, 2])


def test_invalid_depth_semantics(oracle):
    """A NaN depth passes d <= 0 and gives sdf NaN, which is not below
    -truncation, and fminf(1, NaN) = 1: the voxel takes an observation of 1.
    A negative depth is skipped."""
    f = synth.tsdf_frame(96, 72, dims=(40, 32, 28), nodes_xy=(6, 5), holes=False, seed=63)
    clean = f.voxels.copy()
    oracle.tsdf_integrate(clean, f.params, f.depth, _cam(f), f.camera_pose)
    for val, expect_obs in ((np.nan, 1.0), (-0.5, None)):
        f2 = synth.tsdf_frame(96, 72, dims=(40, 32, 28), nodes_xy=(6, 5), holes=False, seed=63)
        f2.depth[:] = val
        vox = f2.voxels.copy()
        n = oracle.tsdf_integrate(vox, f2.params, f2.depth, _cam(f2), f2.camera_pose)
        if expect_obs is None:
            assert n == 0 and np.array_equal(vox, f2.voxels)
        else:
            ch = np.any(vox[:, :2] != f2.voxels[:, :2], axis=1)
            assert n > 0 and ch.sum() > 0
            dec = f2.voxels[ch, 1] * np.float32(0.9)
            want = (f2.voxels[ch, 0] * dec + np.float32(1.0)) / (dec + np.float32(1.0))
            assert np.allclose(vox[ch, 0], want, rtol=1e-6, atol=1e-6)


def test_gate(oracle):
    f = synth.tsdf_frame(96, 72, dims=(40, 32, 28), nodes_xy=(6, 5), seed=64)
    vox = f.voxels.copy()
    oracle.tsdf_integrate(vox, f.params, f.depth, _cam(f), f.camera_pose, counts=f.counts, gate=True, min_opt=3)
    low = f.counts < 3
    assert np.array_equal(vox[low], f.voxels[low])
    ok, want = _numpy_integrate(f, gate=True)
    assert ok.sum() > 100 and not np.any(ok & low)


def _numpy_mark(recs, vidx, dims, frame, counts, frames):
    counts, frames = counts.copy(), frames.copy()
    keep = (recs["valid"] != 0) & ~(recs["weight"] <= 0) & (vidx >= 0)
    touched = set()
    for vi in vidx[keep]:
        x, y, z = vi % dims[0], (vi // dims[0]) % dims[1], vi // (dims[0] * dims[1])
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    X, Y, Z = x + ox, y + oy, z + oz
                    if 0 <= X < dims[0] and 0 <= Y < dims[1] and 0 <= Z < dims[2]:
                        touched.add((Z * dims[1] + Y) * dims[0] + X)
    for n in touched:
        if frames[n] != frame:
            counts[n] += 1
        frames[n] = frame
    return counts, frames


def test_mark_against_numpy(oracle):
    rng = np.random.default_rng(65)
    dims = (13, 11, 7)
    V = int(np.prod(dims))
    P = 800
    recs = np.zeros(P, CORR_DTYPE)
    recs["valid"] = rng.random(P) < 0.7
    recs["weight"] = rng.uniform(-0.5, 1.0, P)
    recs["weight"][::37] = np.nan
    vidx = rng.integers(-1, V, P).astype(np.int32)
    counts = rng.integers(0, 5, V).astype(np.int32)
    frames = rng.integers(0, 4, V).astype(np.int32)
    c, fr = counts.copy(), frames.copy()
    oracle.mark_optimized_voxels(recs, vidx, dims, 3, c, fr)
    wc, wf = _numpy_mark(recs, vidx, dims, 3, counts, frames)
    assert np.array_equal(c, wc) and np.array_equal(fr, wf)


def test_world_to_camera_library_matches_oracle(oracle, cflib):
    from cudafusion_b200.tsdf import world_to_camera

    rng = np.random.default_rng(66)
    for _ in range(20):
        f = synth.tsdf_frame(32, 24, dims=(4, 4, 4), nodes_xy=(3, 3), cam_rot_deg=float(rng.uniform(0, 90)),
                             cam_trans=tuple(rng.normal(size=3)), seed=int(rng.integers(1 << 30)))
        m = world_to_camera(f.camera_pose)
        want = oracle.tsdf_world_to_camera(f.camera_pose)
        assert np.array_equal(m.view(np.uint32), want.view(np.uint32))


def _golden_case(g, k):
    pre = f"c{k}_"
    s = g[pre + "scalars"]
    params = dict(dims=g[pre + "dims"], origin=g[pre + "origin"], voxel_size=float(s[0]), truncation=float(s[1]),
                  decay_alpha=float(s[2]), max_weight=float(s[3]))
    w, h = (int(v) for v in g[pre + "size"])
    f = synth.TsdfFrame(params=params, width=w, height=h, cam=g[pre + "cam"], camera_pose=g[pre + "camera_pose"],
                        depth=g[pre + "depth"], voxels=g[pre + "voxels"], nodes=g[pre + "nodes"].view(NODE_DTYPE),
                        transforms=g[pre + "transforms"].view(DQ_DTYPE), voxel_knn=g[pre + "voxel_knn"],
                        voxel_knn_w=g[pre + "voxel_knn_w"], counts=g[pre + "counts"])
    return f, int(s[4])


def test_oracle_against_reference_golden(oracle):
    if not os.path.exists(GOLDEN):
        pytest.skip("tests/golden/tsdf_ref.npz not made yet")
    g = np.load(GOLDEN)
    k = 0
    while f"c{k}_size" in g:
        f, min_opt = _golden_case(g, k)
        cen = oracle.tsdf_centres(f.params["dims"], f.params["origin"], f.params["voxel_size"])
        live = oracle.skin(cen, f.voxel_knn, f.voxel_knn_w, f.nodes, f.transforms, precision="f32")
        for mode, lv, gate in (("rigid", None, False), ("warped", live, False), ("gated", live, True)):
            vox = f.voxels.copy()
            oracle.tsdf_integrate(vox, f.params, f.depth, _cam(f), f.camera_pose, live=lv, counts=f.counts,
                                  gate=gate, min_opt=min_opt)
            ref = g[f"c{k}_{mode}"]
            up_o = np.any(vox.view(np.uint32) != f.voxels.view(np.uint32), axis=1)
            up_r = np.any(ref.view(np.uint32) != f.voxels.view(np.uint32), axis=1)
            both = up_o & up_r
            tol = 1e-5 if mode == "rigid" else 2e-5
            close = np.abs(vox[both, :2] - ref[both, :2]).max(axis=1) <= tol
            assert up_r.sum() > 100, (k, mode)
            assert np.mean(up_o == up_r) >= 0.999, (k, mode)
            assert close.mean() >= 0.999, (k, mode)
        recs = g[f"c{k}_mark_recs"].view(CORR_DTYPE)
        vidx = g[f"c{k}_mark_vidx"]
        c, fr = g[f"c{k}_mark_counts0"].copy(), g[f"c{k}_mark_frames0"].copy()
        for j, frame in enumerate((2, 2, 3)):
            oracle.mark_optimized_voxels(recs, vidx, f.params["dims"], frame, c, fr)
            assert np.array_equal(c, g[f"c{k}_mark_counts{j + 1}"]) and np.array_equal(fr, g[f"c{k}_mark_frames{j + 1}"])
        k += 1
    assert k >= 2


def test_voxel_range_matches_full_volume(oracle):
    """Integrating voxels [lo, hi) with that range's centres (the form the
    full-volume GPU test and the CPU baseline use) gives the full run's
    values there and leaves the rest alone."""
    f = synth.tsdf_frame(96, 72, dims=(40, 32, 28), nodes_xy=(6, 5), invalid_frac=0.01, seed=67)
    cen = oracle.tsdf_centres(f.params["dims"], f.params["origin"], f.params["voxel_size"])
    live = oracle.skin(cen, f.voxel_knn, f.voxel_knn_w, f.nodes, f.transforms, precision="f32")
    full = f.voxels.copy()
    oracle.tsdf_integrate(full, f.params, f.depth, _cam(f), f.camera_pose, live=live, counts=f.counts, gate=True,
                          min_opt=3)
    plane = 40 * 32
    lo, hi = 13 * plane, 17 * plane + 5
    part = f.voxels.copy()
    n = oracle.tsdf_integrate(part, f.params, f.depth, _cam(f), f.camera_pose, live=live[lo:hi], counts=f.counts,
                              gate=True, min_opt=3, lo=lo, hi=hi)
    assert n > 0
    assert np.array_equal(part[lo:hi].view(np.uint32), full[lo:hi].view(np.uint32))
    assert np.array_equal(part[:lo], f.voxels[:lo]) and np.array_equal(part[hi:], f.voxels[hi:])
    assert np.array_equal(oracle.tsdf_centres(f.params["dims"], f.params["origin"], f.params["voxel_size"], lo, hi),
                          cen[lo:hi])


def test_camera_facing_away_updates_nothing(oracle):
    """Every voxel behind the camera (z <= 0) is skipped: a pose turned 180
    degrees about y leaves the volume as it was; an empty range does nothing."""
    f = synth.tsdf_frame(96, 72, dims=(40, 32, 28), nodes_xy=(6, 5), seed=68)
    pose = f.camera_pose.copy()
    pose[:3, :3] = pose[:3, :3] @ np.diag([-1.0, 1.0, -1.0]).astype(np.float32)
    vox = f.voxels.copy()
    assert oracle.tsdf_integrate(vox, f.params, f.depth, _cam(f), pose) == 0
    assert np.array_equal(vox, f.voxels)
    assert oracle.tsdf_integrate(vox, f.params, f.depth, _cam(f), f.camera_pose, lo=5, hi=5) == 0
