"""Makes tests/golden/raster_ref.npz: the reference's own rasteriser
(src/mesh_raster_kernels.cu:76-200, built for sm_100a with its own flags in
oracle/_ref/libcfref_raster.so) run on a B200 over seeded small two-cylinder
meshes, with their inputs, so that the CPU oracle can be checked against the
reference without a GPU.

    python tests/golden/make_raster_golden.py [out.npz]

Needs a GPU and the built oracle/_ref/libcfref_raster.so.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from cudafusion_b200 import synth  # noqa: E402
import ref_raster  # noqa: E402

# (seed, width, height, n_theta, n_axial, bend deg, camera rotation deg)
CASES = [(61, 64, 48, 40, 20, 30.0, 0.6), (62, 80, 60, 24, 12, 10.0, 2.0), (63, 64, 48, 96, 48, 45.0, 1.0)]


def main(out_path):
    arrays = {}
    for k, (seed, w, h, nt, na, bend, rot) in enumerate(CASES):
        f = synth.mesh_frame(w, h, n_theta=nt, n_axial=na, bend_deg=bend, cam_rot_deg=rot, seed=seed)
        ref = ref_raster.RefRaster(f, with_graph=False)
        ref.run(skin=False)
        lv, ln, hit, _, z = ref.download()
        ref.close()
        arrays[f"c{k}_case"] = np.array([seed, w, h, nt, na, bend, rot], np.float64)
        for name in ("cam", "canonical", "warped", "triangles", "T_cam_world", "grid_origin", "dims"):
            arrays[f"c{k}_{name}"] = np.asarray(getattr(f, name))
        arrays[f"c{k}_voxel_size"] = np.array([f.voxel_size], np.float64)
        arrays[f"c{k}_ref_live_vertices"] = lv
        arrays[f"c{k}_ref_live_normals"] = ln
        arrays[f"c{k}_ref_hit"] = hit
        arrays[f"c{k}_ref_keys"] = z
        print(f"case {k}: {f.meta['triangles']} triangles, {int((z != np.uint64(2**64 - 1)).sum())} pixels hit")
    np.savez_compressed(out_path, **arrays)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                              "raster_ref.npz"))
