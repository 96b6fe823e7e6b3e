"""Projective correspondence search on the B200 (cf_find_correspondences)
against the CPU oracle (oracle/cf_oracle_corr.c, which follows
kernels/tsdf_kernels.cu:386-604 candidate by candidate) and against the
reference's own kernel (oracle/_ref/libcfref_corr.so).

Against the oracle the bar is bit-for-bit: every record byte, the valid count
and the six debug counters.  Against the reference's build (--use_fast_math:
approximate divide and square root) the bar is agreement to rounding on the
pixels whose choice does not hinge on a last-bit tie: the same valid flag on
>= 99.5 % of pixels, the same candidate on >= 99 % of the pixels both call
valid, and there dst within 1e-5 m, the normal within 1e-5 and the weight
within 1e-4."""
import dataclasses

import numpy as np
import pytest
import torch

from cudafusion_b200 import synth
from cudafusion_b200.corr import CorrespondenceSearch, CorrParams, DeviceCorrFrame, compute_pixel_knn

pytestmark = pytest.mark.gpu

STOCK = CorrParams()  # config/params.yaml:60-63
CLASSIC = CorrParams(0.015, 0.75, 0.15, 3)  # config/params.yaml:53-56
UPPER = CorrParams(0.08, 0.5, 0.2, 20)  # config/upperbody.yaml:62-65


def _bytes(recs):
    return np.ascontiguousarray(recs).view(np.uint8)


def _differ(a, b):
    """Pixels whose records differ in any bit, where any two NaNs count as
    equal (the GPU writes the canonical NaN, the host keeps the input's)."""
    wa = np.ascontiguousarray(a).view(np.uint32).reshape(len(a), -1)
    wb = np.ascontiguousarray(b).view(np.uint32).reshape(len(b), -1)
    fa, fb = wa.view(np.float32), wb.view(np.float32)
    return np.nonzero(((wa != wb) & ~(np.isnan(fa) & np.isnan(fb))).any(1))[0]


def run_gpu(frame, params, use_voxels=False, search=None):
    dev = DeviceCorrFrame(frame)
    s = search or CorrespondenceSearch(max(frame.width, 1), max(frame.height, 1))
    n = s.find_correspondences(dev, params, debug=True, use_voxels=use_voxels)
    recs = s.records(frame.width * frame.height)
    return recs, n, s.stats.cpu().numpy().copy(), s


def check_exact(oracle, frame, params, use_voxels=False):
    recs, n, st, _ = run_gpu(frame, params, use_voxels)
    ref, nv, rst = oracle.find_correspondences(frame, params.dist_threshold, params.angle_threshold,
                                               params.view_threshold, params.search_radius_px)
    assert n == nv == int(recs["valid"].sum())
    assert np.array_equal(st, rst), (st, rst)
    bad = _differ(recs, ref)
    assert bad.size == 0, f"{bad.size} records differ, first pixel {bad[:5]}"
    return n, st


@pytest.mark.parametrize("params", [STOCK, CLASSIC, UPPER, CorrParams(0.05, 0.3, 0.1, 0),
                                    CorrParams(0.1, 0.0, 0.0, 9)], ids=["stock", "classic", "upper", "r0", "r9"])
def test_small_frame_bit_exact(oracle, params):
    f = synth.corr_frame(96, 72, cam_rot_deg=1.0, seed=31)
    n, st = check_exact(oracle, f, dataclasses.replace(params, search_radius_px=min(params.search_radius_px, 12)))
    assert n > 0.5 * f.num_pixels


@pytest.mark.parametrize("chunks", [1, 2, 3, 8])
def test_row_chunks_give_one_result(oracle, chunks):
    """The search's row chunks merge to the sequential scan's result whatever
    their count."""
    f = synth.corr_frame(128, 96, cam_rot_deg=1.2, seed=41)
    s = CorrespondenceSearch(128, 96)
    s.set_chunks(chunks)
    for prm in (dataclasses.replace(STOCK, search_radius_px=15), CLASSIC):
        recs, n, st, _ = run_gpu(f, prm, search=s)
        ref, nv, rst = oracle.find_correspondences(f, prm.dist_threshold, prm.angle_threshold,
                                                   prm.view_threshold, prm.search_radius_px)
        assert n == nv and np.array_equal(st, rst)
        assert np.array_equal(_bytes(recs), _bytes(ref))


def test_non_finite_inputs_follow_the_sequential_rule(oracle):
    """A NaN depth makes the frame take the sequential scan (the reference
    accepts a NaN distance and every later candidate within the bound); a
    NaN live vertex does the same for its pixel."""
    f = synth.corr_frame(64, 48, seed=42)
    d = f.depth.copy()
    d[[100, 1500, 2000]] = np.nan
    check_exact(oracle, dataclasses.replace(f, depth=d), CorrParams(0.05, 0.3, 0.1, 4))
    lv = f.live_vertices.copy()
    lv[[7, 900]] = [np.nan, 0.0, 0.1]
    check_exact(oracle, dataclasses.replace(f, live_vertices=lv), CorrParams(0.05, 0.3, 0.1, 4))
    check_exact(oracle, f, CorrParams(float("nan"), 0.3, 0.1, 2))


def test_voxel_path_matches_pixel_path(oracle):
    f = synth.corr_frame(80, 60, seed=32)
    recs_p, n_p, st_p, _ = run_gpu(f, CLASSIC, use_voxels=False)
    recs_v, n_v, st_v, s = run_gpu(f, CLASSIC, use_voxels=True)
    assert n_p == n_v and np.array_equal(st_p, st_v)
    assert np.array_equal(_bytes(recs_p), _bytes(recs_v))
    # the fused gather's per-pixel lists equal compute_pixel_knn's
    dev = DeviceCorrFrame(f)
    s.launch(dev, CLASSIC, use_voxels=True, pixel_knn_out=True)
    torch.cuda.synchronize()
    pk, pw = compute_pixel_knn(dev)
    ok, ow = oracle.compute_pixel_knn(f.hit_voxel_idx, f.voxel_knn, f.voxel_knn_w)
    assert np.array_equal(pk.cpu().numpy().reshape(-1, 4), ok)
    assert np.array_equal(pw.cpu().numpy().reshape(-1, 4), ow)
    P = f.num_pixels
    assert np.array_equal(s.pixel_knn[: 4 * P].cpu().numpy().reshape(-1, 4), ok)
    assert np.array_equal(s.pixel_knn_w[: 4 * P].cpu().numpy().reshape(-1, 4), ow)


@pytest.mark.parametrize("wh", [(37, 23), (1, 1), (1, 40), (50, 1), (33, 9)])
def test_ragged_sizes(oracle, wh):
    w, h = wh
    f = synth.corr_frame(64, 48, seed=33)
    # crop the 64 x 48 frame to w x h (intrinsics kept: the crop's corner is the frame's)
    def crop(a):
        a = np.asarray(a)
        return a.reshape(48, 64, *a.shape[1:])[:h, :w].reshape(w * h, *a.shape[1:])
    g = dataclasses.replace(f, width=w, height=h, live_vertices=crop(f.live_vertices),
                            live_normals=crop(f.live_normals), depth=crop(f.depth),
                            depth_normals=crop(f.depth_normals), hit_voxel_idx=crop(f.hit_voxel_idx),
                            pixel_knn=crop(f.pixel_knn), pixel_knn_w=crop(f.pixel_knn_w))
    check_exact(oracle, g, CorrParams(0.1, 0.2, 0.05, 4))


def test_empty_and_invalid_frames(oracle):
    f = synth.corr_frame(64, 48, seed=34)
    s = CorrespondenceSearch(64, 48)
    # 0 x 0: nothing launched, count and counters zeroed
    dev = DeviceCorrFrame(f)
    dev.width, dev.height = 0, 0
    s.num_valid.fill_(7)
    s.stats.fill_(7)
    assert s.find_correspondences(dev, STOCK, debug=True) == 0
    assert s.stats.cpu().numpy().tolist() == [0] * 6
    # no live surface at all: every pixel is invalid_live
    g = dataclasses.replace(f, live_vertices=np.zeros_like(f.live_vertices))
    n, st = check_exact(oracle, g, dataclasses.replace(STOCK, search_radius_px=5))
    assert n == 0 and st[0] == g.num_pixels
    # no depth: every searching pixel is no_depth
    g = dataclasses.replace(f, depth=np.zeros_like(f.depth))
    n, st = check_exact(oracle, g, dataclasses.replace(STOCK, search_radius_px=5))
    assert n == 0 and st[2] > 0.5 * g.num_pixels
    # depth normals all missing: depth seen, nothing close
    g = dataclasses.replace(f, depth_normals=np.zeros_like(f.depth_normals))
    n, st = check_exact(oracle, g, dataclasses.replace(STOCK, search_radius_px=5))
    assert n == 0 and st[3] > 0.5 * g.num_pixels
    # negative radius acts as 0; a radius past the image reads the whole image
    check_exact(oracle, f, dataclasses.replace(CLASSIC, search_radius_px=-4))
    check_exact(oracle, f, dataclasses.replace(STOCK, search_radius_px=200))


def _scattered(width, height, seed):
    """A frame whose live vertices are a random cloud in front of the camera:
    neighbouring pixels project far apart, so a CTA's window union spans the
    image (the banded shared-memory path with narrow bands, or the direct
    path when the union is wider than a band buffer holds)."""
    f = synth.corr_frame(64, 48, seed=seed)
    rng = np.random.default_rng(seed)
    P = width * height
    fx = fy = 570.342 * width / 640.0
    cx, cy = width / 2.0, height / 2.0
    u = rng.uniform(-2.0, width + 1.0, P)  # a few project off the image
    v = rng.uniform(-2.0, height + 1.0, P)
    z = rng.uniform(0.1, 0.2, P)
    lv = np.stack([(u - cx) / fx * z, (v - cy) / fy * z, z], -1).astype(np.float32)
    ln = np.tile(np.array([0.0, 0.0, -1.0], np.float32), (P, 1))
    d = rng.uniform(0.1, 0.2, P).astype(np.float32)
    d[rng.random(P) < 0.05] = 0
    dn = np.tile(np.array([0.0, 0.0, -1.0], np.float32), (P, 1))
    dn[rng.random(P) < 0.05] = 0
    pk = rng.integers(0, 100, (P, 4)).astype(np.int32)
    pw = rng.random((P, 4)).astype(np.float32)
    eye = np.eye(4, dtype=np.float32)
    return dataclasses.replace(f, width=width, height=height, cam=np.array([fx, fy, cx, cy], np.float32),
                               live_vertices=lv, live_normals=ln, depth=d, depth_normals=dn, T_cam_world=eye,
                               T_world_cam=eye, hit_voxel_idx=np.full(P, -1, np.int32), pixel_knn=pk,
                               pixel_knn_w=pw)


def test_scattered_projections_banded(oracle):
    check_exact(oracle, _scattered(640, 40, 35), CorrParams(0.002, 0.5, 0.1, 3))


def test_scattered_projections_direct(oracle):
    # a union 2400 columns wide: one row of it is more than the band buffer holds
    check_exact(oracle, _scattered(2400, 12, 36), CorrParams(0.002, 0.5, 0.1, 2))


def test_full_frame_stock_sampled(oracle):
    """640 x 480, the stock configuration (radius 50): counters and count
    consistent, 3000 random pixels bit for bit against the oracle."""
    f = synth.corr_frame(seed=37)
    recs, n, st, _ = run_gpu(f, STOCK)
    assert int(st.sum()) == f.num_pixels and st[5] == n == int(recs["valid"].sum())
    assert n > 0.9 * f.num_pixels
    pix = np.sort(np.random.default_rng(0).choice(f.num_pixels, 3000, replace=False)).astype(np.int32)
    ref, _, _ = oracle.find_correspondences(f, STOCK.dist_threshold, STOCK.angle_threshold, STOCK.view_threshold,
                                            STOCK.search_radius_px, pixels=pix)
    assert np.array_equal(_bytes(recs[pix]), _bytes(ref))
    v = recs["valid"] == 1
    # the pairs are close on the surface: point-to-plane distance well inside the bound
    d = recs["dst"][v] - recs["src"][v]
    pd = np.abs(np.sum(d * recs["normal"][v], -1))
    assert np.median(pd) < 0.005


def test_repeat_is_deterministic():
    f = synth.corr_frame(160, 120, seed=38)
    dev = DeviceCorrFrame(f)
    s = CorrespondenceSearch(160, 120)
    s.find_correspondences(dev, UPPER, debug=True)
    a = s.corrs.clone()
    s.find_correspondences(dev, UPPER, debug=True)
    assert torch.equal(a, s.corrs)


def test_capacity_and_arguments():
    from cudafusion_b200 import _lib

    f = synth.corr_frame(64, 48, seed=39)
    dev = DeviceCorrFrame(f)
    s = CorrespondenceSearch(32, 48)
    with pytest.raises(_lib.CFError) as e:
        s.find_correspondences(dev, STOCK)
    assert e.value.status == _lib.CF_ERR_CAPACITY


def _ref_agreement(recs, ref):
    vg, vr = recs["valid"] == 1, ref["valid"] == 1
    flag = float(np.mean(vg == vr))
    both = vg & vr
    same = both & (np.linalg.norm(recs["dst"] - ref["dst"], axis=-1) < 1e-5)
    return flag, float(same.sum()) / max(int(both.sum()), 1), both, same


@pytest.mark.parametrize("params", [STOCK, CLASSIC, UPPER], ids=["stock", "classic", "upper"])
def test_against_reference_kernel(params):
    import ref_corr

    if not ref_corr.available():
        pytest.skip("oracle/_ref/libcfref_corr.so not built (needs the CUDAFusion sources)")
    f = synth.corr_frame(seed=40)
    recs, n, st, _ = run_gpu(f, params)
    ref = ref_corr.RefCorrSearch(f)
    rn, _ = ref.run(params.dist_threshold, params.angle_threshold, params.view_threshold, params.search_radius_px)
    rrecs, rpk, rpw, rst = ref.download()
    ref.close()
    assert np.array_equal(rpk, f.pixel_knn) and np.array_equal(rpw, f.pixel_knn_w)
    flag, same_frac, both, same = _ref_agreement(recs, rrecs)
    assert flag >= 0.995, flag
    assert same_frac >= 0.99, same_frac
    assert abs(n - rn) <= 0.005 * f.num_pixels
    assert np.abs(recs["normal"][same] - rrecs["normal"][same]).max() < 1e-5
    assert np.abs(recs["weight"][same] - rrecs["weight"][same]).max() < 1e-4
    assert np.array_equal(recs["node_ids"][same], rrecs["node_ids"][same])
    assert np.array_equal(recs["src"][same], rrecs["src"][same])
    print(f"{params}: valid {n} vs {rn}; flags agree {flag:.5f}; same candidate {same_frac:.5f}")
