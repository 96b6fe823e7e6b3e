"""The rasterisation oracle (oracle/cf_oracle_raster.c) pinned to the
reference: tests/golden/raster_ref.npz holds the reference's own
rasterize_triangles_z_kernel + resolve_rasterized_triangles_kernel
(src/mesh_raster_kernels.cu:76-200, built for sm_100a with --use_fast_math) run
on a B200 over three small two-cylinder meshes (coarse, very coarse with a
larger camera turn, sub-pixel triangles; tests/golden/make_raster_golden.py).
The reference's build divides and takes square roots approximately, so the
bar is agreement to rounding: the same pixels hit on >= 99.5 %, the same
triangle (the low 32 bits of the depth key) on >= 99 % of the pixels both
hit, there live vertices within 1e-5 m, normals within 1e-4 and hit voxels
equal on >= 99 %.  Plus the oracle's own consistency."""
import os
from types import SimpleNamespace

import numpy as np
import pytest

from cudafusion_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "raster_ref.npz")
EMPTY = np.uint64(0xFFFFFFFFFFFFFFFF)


def _cases():
    z = np.load(GOLDEN)
    out = []
    k = 0
    while f"c{k}_case" in z:
        g = {n[len(f"c{k}_"):]: z[n] for n in z.files if n.startswith(f"c{k}_")}
        seed, w, h = (int(v) for v in g["case"][:3])
        frame = SimpleNamespace(width=w, height=h, voxel_size=float(g["voxel_size"][0]), **{n: g[n] for n in (
            "cam", "canonical", "warped", "triangles", "T_cam_world", "grid_origin", "dims")})
        out.append((k, frame, g))
        k += 1
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: f"case{c[0]}")
def test_oracle_against_reference_golden(oracle, case):
    k, frame, g = case
    lv, ln, hit, keys = oracle.rasterize(frame)
    on, ron = keys != EMPTY, g["ref_keys"] != EMPTY
    flag = float(np.mean(on == ron))
    both = on & ron
    tri_same = both & ((keys & np.uint64(0xFFFFFFFF)) == (g["ref_keys"] & np.uint64(0xFFFFFFFF)))
    frac = float(tri_same.sum()) / max(int(both.sum()), 1)
    print(f"case {k}: hit {int(on.sum())} vs {int(ron.sum())}, flags agree {flag:.5f}, same triangle {frac:.5f}")
    assert flag >= 0.995 and frac >= 0.99
    assert np.abs(lv[tri_same] - g["ref_live_vertices"][tri_same]).max() < 1e-5
    assert np.abs(ln[tri_same] - g["ref_live_normals"][tri_same]).max() < 1e-4
    assert np.mean(hit[tri_same] == g["ref_hit"][tri_same]) >= 0.99


def test_oracle_consistency(oracle):
    f = synth.mesh_frame(80, 60, n_theta=48, n_axial=24, seed=81)
    lv, ln, hit, keys = oracle.rasterize(f)
    on = keys != EMPTY
    # every hit pixel has a live point on a unit normal; misses are zero / -1
    assert np.all(np.linalg.norm(lv[on], axis=1) > 0)
    assert np.allclose(np.linalg.norm(ln[on], axis=1), 1.0, atol=1e-5)
    assert not lv[~on].any() and np.all(hit[~on] == -1)
    # the depth key's triangle covers the pixel, and its depth is the point's camera z
    T = f.T_cam_world.astype(np.float64)
    zc = (lv[on].astype(np.float64) @ T[:3, :3].T + T[:3, 3])[:, 2]
    zk = (keys[on] >> np.uint64(32)).astype(np.uint32).view(np.float32)
    assert np.abs(zc - zk).max() < 1e-5
    # voxels of the canonical points
    vox = oracle.voxel_of_points(f.canonical, f.grid_origin, f.voxel_size, f.dims)
    assert np.all(vox >= 0) and np.all(vox < int(np.prod(f.dims)))
