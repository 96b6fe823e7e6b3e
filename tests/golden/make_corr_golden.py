"""Makes tests/golden/corr_ref.npz: the reference's own correspondence search
(kernels/tsdf_kernels.cu:386-604, built for sm_100a with its own flags in
oracle/_ref/libcfref_corr.so) run on a B200 over seeded 64 x 48 two-cylinder
frames, with the frames' inputs, so that the CPU oracle can be checked
against the reference without a GPU.

    python tests/golden/make_corr_golden.py [out.npz]

Needs a GPU and the built oracle/_ref/libcfref_corr.so.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from cudafusion_b200 import synth  # noqa: E402
import ref_corr  # noqa: E402

# (frame seed, camera rotation deg, dist, angle, view, radius): the stock
# thresholds, the tighter ones kept commented in config/params.yaml:53-56, the
# upper-body configuration (config/upperbody.yaml:62-65) and a window of one pixel
CASES = [
    (21, 0.6, 0.2, 0.0, 0.0, 8),
    (22, 1.5, 0.015, 0.75, 0.15, 3),
    (23, 0.6, 0.08, 0.5, 0.2, 5),
    (24, 3.0, 0.05, 0.3, 0.1, 0),
]


def main(out_path):
    arrays = {}
    for k, (seed, rot, d, a, v, r) in enumerate(CASES):
        f = synth.corr_frame(64, 48, cam_rot_deg=rot, seed=seed)
        ref = ref_corr.RefCorrSearch(f)
        n, _ = ref.run(d, a, v, r, debug=True)
        recs, pk, pw, st = ref.download()
        ref.close()
        arrays[f"c{k}_case"] = np.array([seed, rot, d, a, v, r], np.float64)
        for name in ("cam", "live_vertices", "live_normals", "depth", "depth_normals", "T_cam_world", "T_world_cam",
                     "pixel_knn", "pixel_knn_w"):
            arrays[f"c{k}_{name}"] = np.asarray(getattr(f, name))
        arrays[f"c{k}_ref_valid"] = recs["valid"].astype(np.uint8)
        arrays[f"c{k}_ref_dst"] = recs["dst"].astype(np.float32)
        arrays[f"c{k}_ref_normal"] = recs["normal"].astype(np.float32)
        arrays[f"c{k}_ref_weight"] = recs["weight"].astype(np.float32)
        # the reference's per-pixel gather equals the frame's, and valid
        # records carry it: neither is stored
        assert np.array_equal(pk, f.pixel_knn) and np.array_equal(pw, f.pixel_knn_w)
        v = recs["valid"] == 1
        assert np.array_equal(recs["node_ids"][v], f.pixel_knn[v])
        arrays[f"c{k}_ref_stats"] = st
        arrays[f"c{k}_ref_num_valid"] = np.array([n], np.int32)
        print(f"case {k}: seed {seed} radius {r} valid {n} stats {st.tolist()}")
    np.savez_compressed(out_path, **arrays)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                              "corr_ref.npz"))
