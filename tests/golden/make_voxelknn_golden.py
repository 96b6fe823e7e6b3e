"""Makes tests/golden/voxelknn_ref.npz: the reference's own voxel kNN field
(WarpField::compute_voxel_knn, src/warp_field.cu:957-981, with
compute_voxel_knn_kernel, :299-405), built for sm_100a with the reference's
flags in oracle/_ref/libcfref_voxelknn.so, run on a B200 over three small
volumes, with their inputs, so that the CPU oracle can be checked against the
reference without a GPU:

  scene   the integrated bumpy-surface volume of synth.voxelknn_frame at
          48x40x40 voxels, 432 surface nodes and 24 nodes repeating others'
          positions (exact distance ties);
  lattice an 8x8x8 volume of 0.25 m voxels at the origin, all active, with
          nodes on the voxel corners: every centre is equidistant from
          several nodes, exactly (all coordinates are dyadic);
  edge    a 12x10x9 volume whose weights are positive, zero, negative or NaN
          (the reference computes a NaN-weight voxel), over three nodes, one
          of them at a NaN position and one far away (squared distances
          beyond 1e30 are never taken).

    python tests/golden/make_voxelknn_golden.py [out.npz]

Needs a GPU and the built oracle/_ref/libcfref_voxelknn.so.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from cudafusion_b200 import synth  # noqa: E402
from cudafusion_b200.types import NODE_DTYPE  # noqa: E402
import ref_voxelknn  # noqa: E402


def records(weights):
    """12-byte voxel records (tsdf 1, the weights, colour 128) as float32 (V, 3)."""
    vox = np.zeros((weights.size, 3), np.float32)
    vox[:, 0] = 1.0
    vox[:, 1] = weights
    vox.view(np.uint32)[:, 2] = 0x00808080
    return vox


def nodes_at(pos, radius):
    nodes = np.zeros(len(pos), NODE_DTYPE)
    nodes["pos"] = pos
    nodes["radius"] = radius
    nodes["neighbors"] = -1
    return nodes


def cases():
    f = synth.voxelknn_frame(dims=(48, 40, 40), nodes_xy=(24, 18), duplicate_nodes=24, seed=41)
    yield "scene", f.params, f.voxels[:, 1].copy(), f.nodes
    dims = np.array([8, 8, 8], np.int32)
    g = np.arange(0, 9, 2, dtype=np.float32) * 0.25
    corners = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    yield ("lattice", dict(dims=dims, origin=np.zeros(3, np.float32), voxel_size=0.25),
           np.full(512, 2.0, np.float32), nodes_at(corners, 0.3))
    rng = np.random.default_rng(43)
    dims = np.array([12, 10, 9], np.int32)
    w = rng.choice(np.array([1.0, 0.0, -1.0, 7.5, np.nan], np.float32), size=int(np.prod(dims)))
    pos = np.array([[0.1, 0.2, 0.3], [np.nan, 0.0, 0.0], [0.4, -0.1, 0.5], [3e15, 0.0, 0.0]], np.float32)
    yield ("edge", dict(dims=dims, origin=np.array([-0.2, -0.1, 0.0], np.float32), voxel_size=0.05), w,
           nodes_at(pos, np.array([0.05, 0.05, 0.0, 0.05], np.float32)))


def main(out_path):
    arrays = {}
    for name, params, weights, nodes in cases():
        ref = ref_voxelknn.RefVoxelKnn(params, records(weights), nodes)
        ids, ws, _ = ref.compute()
        ref.close()
        arrays[name + "_dims"] = np.asarray(params["dims"], np.int32)
        arrays[name + "_origin"] = np.asarray(params["origin"], np.float32)
        arrays[name + "_voxel_size"] = np.float32(params["voxel_size"])
        arrays[name + "_weights"] = weights
        arrays[name + "_nodes"] = nodes.view(np.uint8)
        arrays[name + "_ids"] = ids
        arrays[name + "_ws"] = ws
        print(name, "voxels", weights.size, "active", int(np.sum(~(weights <= 0))), "nodes", len(nodes))
    np.savez_compressed(out_path, **arrays)
    print("wrote", out_path)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden", "voxelknn_ref.npz"))
