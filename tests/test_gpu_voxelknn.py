"""The voxel kNN field on sm_100a (cf_compute_voxel_knn) against the oracle,
the golden fixture made by the reference's kernel, and the reference's own
kernel run live (WarpField::compute_voxel_knn, src/warp_field.cu:957-981,
oracle/_ref/libcfref_voxelknn.so), through the C ABI.

Bars: ids bit for bit; weights within 1e-6 of the oracle (both IEEE) and 2e-6
of the reference (its --use_fast_math exp and divisions)."""
import ctypes
import os

import numpy as np
import pytest
import torch

import oracle as O
import ref_voxelknn as RK
from cudafusion_b200 import _lib, synth
from cudafusion_b200.tsdf import TsdfParams, TSDFVolume
from cudafusion_b200.types import NODE_DTYPE
from test_voxelknn_oracle import GOLDEN, W_TOL, W_TOL_REF, golden_case

pytestmark = pytest.mark.gpu
THREADS = os.cpu_count() or 1


def device_field(params, vox, nodes):
    """cf_compute_voxel_knn on the volume `vox` (float32 (V, 3)) and `nodes`:
    host (ids (V, 4), ws (V, 4))."""
    vol = TSDFVolume(TsdfParams(dims=tuple(int(v) for v in params["dims"]), voxel_size=float(params["voxel_size"]),
                                origin=tuple(float(v) for v in params["origin"])))
    vol.voxels.copy_(torch.from_numpy(np.ascontiguousarray(vox, np.float32).view(np.uint8).reshape(-1)))
    dn = torch.from_numpy(np.ascontiguousarray(nodes, NODE_DTYPE).view(np.uint8).reshape(-1).copy()).cuda()
    ids, ws = vol.compute_voxel_knn(dn, len(nodes))
    torch.cuda.synchronize()
    return ids.cpu().numpy().reshape(-1, 4), ws.cpu().numpy().reshape(-1, 4)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("name", ["scene", "lattice", "edge"])
def test_matches_reference_golden(golden, name):
    params, vox, nodes, ids_ref, ws_ref = golden_case(golden, name)
    ids, ws = device_field(params, vox, nodes)
    assert np.array_equal(ids, ids_ref)
    assert np.abs(ws - ws_ref).max() <= W_TOL_REF
    oi, ow = O.voxel_knn(vox, params, nodes, nthreads=THREADS)
    assert np.abs(ws - ow).max() <= W_TOL


@pytest.fixture(scope="module")
def frame256():
    return synth.voxelknn_frame()


@pytest.fixture(scope="module")
def field256(frame256):
    return device_field(frame256.params, frame256.voxels, frame256.nodes)


def test_full_volume_matches_reference_kernel(frame256, field256):
    """The reference's 256^3 x 6 mm volume after a frame was integrated
    (2.1 M voxels hold data, 1728 nodes): every voxel's ids equal the
    reference kernel's, weights within the bar."""
    if not RK.available():
        pytest.skip("oracle/_ref/libcfref_voxelknn.so was not built")
    ref = RK.RefVoxelKnn(frame256.params, frame256.voxels, frame256.nodes)
    rid, rws, _ = ref.compute()
    ref.close()
    ids, ws = field256
    assert np.array_equal(ids, rid)
    assert np.abs(ws - rws).max() <= W_TOL_REF


def test_full_volume_matches_oracle_sample(frame256, field256):
    """A seeded sample of 20,000 voxels with data and 20,000 without, against
    the oracle; every empty voxel carries -1 / 0."""
    ids, ws = field256
    w = frame256.voxels[:, 1]
    active = np.where(~(w <= 0))[0]
    empty = np.where(w <= 0)[0]
    assert np.all(ids[empty] == -1) and np.all(ws[empty] == 0)
    rng = np.random.default_rng(9)
    vidx = np.concatenate([rng.choice(active, 20000, replace=False), rng.choice(empty, 20000, replace=False)])
    oi, ow = O.voxel_knn_list(frame256.voxels, frame256.params, frame256.nodes, vidx.astype(np.int64),
                              nthreads=THREADS)
    assert np.array_equal(ids[vidx], oi)
    assert np.abs(ws[vidx] - ow).max() <= W_TOL
    assert np.all(ids[active] >= 0)
    # normalised, or all zero where the exponentials underflow (far from
    # every node, src/warp_field.cu:398)
    s = ws[active].sum(1)
    assert np.all((np.abs(s - 1) < 1e-5) | (s == 0)) and (np.abs(s - 1) < 1e-5).mean() > 0.5


def test_deterministic(frame256, field256):
    ids, ws = device_field(frame256.params, frame256.voxels, frame256.nodes)
    assert np.array_equal(ids, field256[0]) and np.array_equal(ws.view(np.uint32), field256[1].view(np.uint32))


def test_ragged_volume_and_many_nodes():
    """A volume whose sides are not multiples of the 8-voxel tile, and a graph
    of 12,000 nodes, past what the kernel stages in shared memory (nodes read
    from global memory): the whole field against the oracle."""
    f = synth.voxelknn_frame(dims=(50, 37, 21), nodes_xy=(120, 100), seed=29)
    assert len(f.nodes) == 12000
    ids, ws = device_field(f.params, f.voxels, f.nodes)
    oi, ow = O.voxel_knn(f.voxels, f.params, f.nodes, nthreads=THREADS)
    assert np.array_equal(ids, oi)
    assert np.abs(ws - ow).max() <= W_TOL


@pytest.mark.parametrize("n", [1, 3, 4, 5])
def test_few_nodes(n):
    f = synth.voxelknn_frame(dims=(24, 24, 24), nodes_xy=(6, 4), seed=30)
    nodes = f.nodes[:n]
    ids, ws = device_field(f.params, f.voxels, nodes)
    oi, ow = O.voxel_knn(f.voxels, f.params, nodes, nthreads=THREADS)
    assert np.array_equal(ids, oi)
    assert np.abs(ws - ow).max() <= W_TOL


def test_no_nodes_and_no_data():
    """No nodes: nothing is written (the reference returns before its
    launch).  No voxel with data: every list is -1 / 0."""
    f = synth.voxelknn_frame(dims=(16, 16, 16), nodes_xy=(4, 3))
    vol = TSDFVolume(TsdfParams(dims=(16, 16, 16), voxel_size=float(f.params["voxel_size"]),
                                origin=tuple(float(v) for v in f.params["origin"])))
    ids = torch.full((4 * 4096,), -7, dtype=torch.int32, device="cuda")
    ws = torch.full((4 * 4096,), 3.0, dtype=torch.float32, device="cuda")
    dn = torch.from_numpy(f.nodes.view(np.uint8).reshape(-1).copy()).cuda()
    vol.compute_voxel_knn(dn, 0, ids, ws)
    torch.cuda.synchronize()
    assert bool((ids == -7).all()) and bool((ws == 3.0).all())
    vol.compute_voxel_knn(dn, len(f.nodes), ids, ws)  # the reset volume: weight 0 everywhere
    torch.cuda.synchronize()
    assert bool((ids == -1).all()) and bool((ws == 0).all())


def test_rejects_bad_arguments():
    f = synth.voxelknn_frame(dims=(8, 8, 8), nodes_xy=(4, 3))
    vol = TSDFVolume(TsdfParams(dims=(8, 8, 8)))
    ids = torch.empty(4 * 512 + 4, dtype=torch.int32, device="cuda")
    ws = torch.empty(4 * 512 + 4, dtype=torch.float32, device="cuda")
    dn = torch.from_numpy(f.nodes.view(np.uint8).reshape(-1).copy()).cuda()
    L = _lib.lib()
    c = vol.params.c()
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    assert L.cf_compute_voxel_knn(P(vol.voxels), ctypes.byref(c), P(dn), 49153, P(ids), P(ws), None) == \
        _lib.CF_ERR_CAPACITY
    assert L.cf_compute_voxel_knn(P(vol.voxels), ctypes.byref(c), P(dn), len(f.nodes), ctypes.c_void_p(
        ids.data_ptr() + 4), P(ws), None) == _lib.CF_ERR_INVALID_ARG
    assert L.cf_compute_voxel_knn(P(vol.voxels), ctypes.byref(c), P(dn), -1, P(ids), P(ws), None) == \
        _lib.CF_ERR_INVALID_ARG
