"""Makes tests/golden/tsdf_ref.npz: the reference's own TSDF integration
(TSDFVolume::integrate, src/tsdf_volume.cu:23-60, with
tsdf_integrate_kernel, kernels/tsdf_kernels.cu:85-174) and its
mark_optimized_voxels_kernel (:606-650), built for sm_100a with the
reference's flags in oracle/_ref/libcfref_tsdf.so, run on a B200 over seeded
small volumes, with their inputs, so that the CPU oracle can be checked
against the reference without a GPU.

    python tests/golden/make_tsdf_golden.py [out.npz]

Needs a GPU and the built oracle/_ref/libcfref_tsdf.so.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from cudafusion_b200 import synth  # noqa: E402
from cudafusion_b200.types import CORR_DTYPE  # noqa: E402
import ref_tsdf  # noqa: E402

# (seed, width, height, dims, nodes_xy, invalid fraction)
CASES = [(31, 96, 72, (40, 32, 28), (8, 6), 0.02), (32, 120, 90, (36, 36, 30), (10, 8), 0.0)]
MIN_OPT = 3


def mark_case(seed, dims):
    rng = np.random.default_rng(seed)
    P = 3000
    V = int(np.prod(dims))
    recs = np.zeros(P, CORR_DTYPE)
    recs["valid"] = rng.random(P) < 0.8
    recs["weight"] = rng.uniform(-0.3, 1.0, P)
    vidx = rng.integers(0, V, P).astype(np.int32)
    vidx[::17] = -1
    vidx[1::29] = 0  # a corner
    vidx[2::31] = V - 1
    counts = rng.integers(0, 4, V).astype(np.int32)
    frames = rng.integers(0, 3, V).astype(np.int32)
    return recs, vidx, counts, frames


def main(out_path):
    arrays = {}
    for k, (seed, w, h, dims, nxy, bad) in enumerate(CASES):
        f = synth.tsdf_frame(w, h, dims=dims, nodes_xy=nxy, invalid_frac=bad, seed=seed)
        pre = f"c{k}_"
        for name in ("cam", "camera_pose", "depth", "voxels", "voxel_knn", "voxel_knn_w", "counts"):
            arrays[pre + name] = getattr(f, name)
        arrays[pre + "nodes"] = f.nodes.view(np.uint8)
        arrays[pre + "transforms"] = f.transforms.view(np.uint8)
        arrays[pre + "size"] = np.array([w, h], np.int32)
        for key in ("dims", "origin"):
            arrays[pre + key] = np.asarray(f.params[key])
        arrays[pre + "scalars"] = np.array([f.params["voxel_size"], f.params["truncation"], f.params["decay_alpha"],
                                            f.params["max_weight"], MIN_OPT], np.float32)
        for mode, warp, gate in (("rigid", False, False), ("warped", True, False), ("gated", True, True)):
            r = ref_tsdf.RefTsdf(f, warp=warp, gate=gate)
            r.integrate(MIN_OPT)
            arrays[pre + mode] = r.voxels()
            r.close()
        recs, vidx, counts, frames = mark_case(seed, dims)
        c1, f1 = ref_tsdf.mark(recs, vidx, dims, 2, counts, frames)
        c2, f2 = ref_tsdf.mark(recs, vidx, dims, 2, c1, f1)  # the same frame again: no change
        c3, f3 = ref_tsdf.mark(recs, vidx, dims, 3, c2, f2)
        arrays[pre + "mark_recs"] = recs.view(np.uint8)
        arrays[pre + "mark_vidx"] = vidx
        arrays[pre + "mark_counts0"] = counts
        arrays[pre + "mark_frames0"] = frames
        for j, (c, fr) in enumerate(((c1, f1), (c2, f2), (c3, f3))):
            arrays[pre + f"mark_counts{j + 1}"] = c
            arrays[pre + f"mark_frames{j + 1}"] = fr
    np.savez_compressed(out_path, **arrays)
    print("wrote", out_path, sum(a.nbytes for a in arrays.values()), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                            "tsdf_ref.npz"))
