"""The correspondence-search oracle (oracle/cf_oracle_corr.c) pinned to the
reference: tests/golden/corr_ref.npz holds the reference's own
find_correspondences_kernel (kernels/tsdf_kernels.cu:386-563, built for
sm_100a with --use_fast_math) run on a B200 over four 64 x 48 frames with four
threshold sets (tests/golden/make_corr_golden.py).  The reference's build
divides and takes square roots approximately, so the bar is agreement to
rounding: the same valid flag on >= 99.5 % of pixels, the same candidate
(dst within 1e-5 m) on >= 99 % of the pixels both call valid, there normals
within 1e-5 and weights within 1e-4, and every debug counter within 0.5 % of
the pixels.  Plus the oracle's own consistency (pixel subsets, counters,
compute_pixel_knn)."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from cudafusion_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "corr_ref.npz")


def _cases():
    z = np.load(GOLDEN)
    out = []
    k = 0
    while f"c{k}_case" in z:
        g = {n[len(f"c{k}_"):]: z[n] for n in z.files if n.startswith(f"c{k}_")}
        seed, rot, d, a, v, r = g["case"]
        frame = SimpleNamespace(width=64, height=48, **{n: g[n] for n in (
            "cam", "live_vertices", "live_normals", "depth", "depth_normals", "T_cam_world", "T_world_cam",
            "pixel_knn", "pixel_knn_w")})
        out.append((k, frame, (float(d), float(a), float(v), int(r)), g))
        k += 1
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: f"case{c[0]}")
def test_oracle_against_reference_golden(oracle, case):
    k, frame, (d, a, v, r), g = case
    recs, n, st = oracle.find_correspondences(frame, d, a, v, r)
    P = frame.width * frame.height
    vo, vr = recs["valid"] == 1, g["ref_valid"] == 1
    flag = float(np.mean(vo == vr))
    both = vo & vr
    same = both & (np.linalg.norm(recs["dst"] - g["ref_dst"], axis=-1) < 1e-5)
    same_frac = float(same.sum()) / max(int(both.sum()), 1)
    print(f"case {k}: valid {n} vs {int(g['ref_num_valid'][0])}, flags agree {flag:.5f}, "
          f"same candidate {same_frac:.5f}")
    assert flag >= 0.995 and same_frac >= 0.99
    assert np.abs(recs["normal"][same] - g["ref_normal"][same]).max() < 1e-5
    assert np.abs(recs["weight"][same] - g["ref_weight"][same]).max() < 1e-4
    assert np.all(np.abs(st - g["ref_stats"]) <= max(1, 0.005 * P)), (st, g["ref_stats"])


def test_oracle_pixel_subsets_and_counters(oracle):
    f = synth.corr_frame(80, 60, seed=51)
    recs, n, st = oracle.find_correspondences(f, 0.08, 0.5, 0.2, 6)
    assert int(st.sum()) == f.num_pixels and st[5] == n == int(recs["valid"].sum())
    pix = np.array([0, 5, 799, 2400, 4799, 17], np.int32)
    sub, _, _ = oracle.find_correspondences(f, 0.08, 0.5, 0.2, 6, pixels=pix)
    assert np.array_equal(sub.view(np.uint8), recs[pix].view(np.uint8))
    # invalid records are zero but for ids = -1
    inv = recs[recs["valid"] == 0]
    assert np.all(inv["node_ids"] == -1) and np.all(inv["weight"] == 0) and np.all(inv["dst"] == 0)
    # valid pairs sit within the distance bound along the target normal
    val = recs[recs["valid"] == 1]
    pd = np.abs(np.sum((val["dst"] - val["src"]) * val["normal"], -1))
    assert np.median(pd) < 0.01


def test_oracle_pixel_knn(oracle):
    f = synth.corr_frame(64, 48, seed=52)
    pk, pw = oracle.compute_pixel_knn(f.hit_voxel_idx, f.voxel_knn, f.voxel_knn_w)
    assert np.array_equal(pk, f.pixel_knn) and np.array_equal(pw, f.pixel_knn_w)
    # out-of-range voxel indices count as none
    hit = f.hit_voxel_idx.copy()
    hit[:10] = f.voxel_knn.shape[0] + 5
    pk2, pw2 = oracle.compute_pixel_knn(hit, f.voxel_knn, f.voxel_knn_w)
    assert np.all(pk2[:10] == -1) and np.all(pw2[:10] == 0)
