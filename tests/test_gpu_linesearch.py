"""The GN step's acceptance on the B200 (cf_scale_delta, cf_validate_update,
cf_correspondence_rmse, cf_line_search) against the host flow of
include/fusion_app.h:409-641 restated with the oracle (oracle/cf_oracle_ls.c).

The scaled increment is bit-for-bit the oracle's.  The statistics' FP64
sums agree to 1e-12 relative (another summation order), the maxima and the
decision exactly.  The device RMSE agrees with the oracle's sequential sum to
1e-12 relative.  The line search's ten trials agree with the reference's
host loop driven step by step (restore, scale, twist, predict, search,
download the records, RMSE on the host): the same valid counts, RMSEs to
1e-12, the same chosen scale and bit-identical transforms afterwards, and
the accepted trial's warped mesh, live maps, hit voxels, records, valid
count and pixel node lists bit for bit (the last trial's maps and records
when none is accepted)."""
import ctypes
import dataclasses

import numpy as np
import pytest
import torch

from cudafusion_b200 import _lib, synth
from cudafusion_b200.corr import CORR_BYTES, CorrespondenceSearch, CorrParams, DeviceCorrFrame
from cudafusion_b200.linesearch import (LineSearch, LineSearchParams, correspondence_rmse, scale_delta,
                                        validate_update)
from cudafusion_b200.raster import DeviceMesh, LiveSurfaceRaster

pytestmark = pytest.mark.gpu


def _dx(n, seed, scale_rot=0.05, scale_trans=0.02):
    rng = np.random.default_rng(seed)
    d = np.concatenate([rng.normal(scale=scale_rot, size=(n, 3)), rng.normal(scale=scale_trans, size=(n, 3))], 1)
    d[::17] *= 20.0  # some beyond the clamps
    d[5::23] = 0.0
    return d.astype(np.float32)


@pytest.mark.parametrize("args", [(0.12, 0.04, 1.0), (0.12, 0.04, -0.25), (0.0, 0.04, 0.5), (0.05, -1.0, 0.0625)])
def test_scale_delta_bit_exact(oracle, args):
    mr, mt, sc = args
    dx = _dx(777, 1)
    out = scale_delta(torch.from_numpy(dx.reshape(-1)).cuda(), 777, mr, mt, sc).cpu().numpy()
    assert np.array_equal(out.view(np.uint32), oracle.scale_delta(dx, mr, mt, sc).view(np.uint32))


def _decision(sums, maxima, fin, n, p):
    """fusion_app.h:460-489 on the oracle's statistics."""
    n1 = np.float32(max(1, n))
    er_mean, et_mean = np.float32(sums[2]) / n1, np.float32(sums[3]) / n1
    rr = 5.0 * p.max_update_rot if p.max_update_rot > 0 else np.inf
    rt = 5.0 * p.max_update_trans if p.max_update_trans > 0 else np.inf
    spike = p.update_scale * maxima[0] > rr or p.update_scale * maxima[1] > rt
    mean_ok = p.max_dx_mean <= 0 or (er_mean <= p.max_dx_mean and et_mean <= p.max_dx_mean)
    return bool(fin and np.isfinite(er_mean) and np.isfinite(et_mean) and np.isfinite(maxima[2]) and
                np.isfinite(maxima[3]) and maxima[2] < rr and maxima[3] < rt and mean_ok and not spike)


@pytest.mark.parametrize("case", ["nominal", "spike", "mean", "nan", "empty"])
def test_validate_update(oracle, case):
    p = LineSearchParams(update_scale=1.0, max_update_rot=0.12, max_update_trans=0.04)
    dx = _dx(2048, 2, 0.01, 0.004)
    dx[::17] /= 20.0
    if case == "spike":
        dx[100, 0] = 2.0
    if case == "mean":
        p = dataclasses.replace(p, max_dx_mean=0.005)
    if case == "nan":
        dx[7, 4] = np.nan
    if case == "empty":
        dx = dx[:0]
    n = dx.shape[0]
    st = validate_update(torch.from_numpy(dx.reshape(-1).copy()).cuda() if n else torch.zeros(1).cuda(), n, p)
    sums, maxima, fin = oracle.update_stats(dx, p.update_scale, p.max_update_rot, p.max_update_trans)
    assert st["finite"] == int(fin)
    if fin:
        got = np.array([st["rot_sum"], st["trans_sum"], st["eff_rot_sum"], st["eff_trans_sum"]])
        assert np.allclose(got, sums, rtol=1e-12, atol=0)
        assert np.array_equal(np.array([st["rot_max"], st["trans_max"], st["eff_rot_max"], st["eff_trans_max"]],
                                       np.float32), maxima)
    want = _decision(sums, maxima, fin, n, p)
    assert st["iter_ok"] == int(want)
    assert want == (case in ("nominal", "empty"))


def test_correspondence_rmse(oracle):
    f = synth.corr_frame(160, 120, seed=95)
    s = CorrespondenceSearch(160, 120)
    s.find_correspondences(DeviceCorrFrame(f), CorrParams(0.08, 0.5, 0.2, 6))
    recs = s.records(160 * 120)
    recs["weight"][::13] = -0.5  # negative weights are skipped
    recs["weight"][5::17] = 0.0
    d = torch.from_numpy(recs.view(np.uint8).reshape(-1).copy()).cuda()
    gs, gw, grm = correspondence_rmse(d, recs.shape[0])
    os_, ow, orm = oracle.corr_rmse(recs)
    assert abs(gs - os_) <= 1e-12 * abs(os_) and abs(gw - ow) <= 1e-12 * abs(ow)
    assert abs(grm - orm) <= 1e-12 * orm
    assert correspondence_rmse(d, 0)[2] == float("inf")


def _scene(seed=96):
    """A 96x72 frame: the depth rendered from the mesh bent 30 deg, the warp
    at 24 deg, the graph's increment random and small."""
    true = synth.mesh_frame(96, 72, n_theta=64, n_axial=32, bend_deg=30.0, seed=seed)
    est = synth.mesh_frame(96, 72, n_theta=64, n_axial=32, bend_deg=24.0, seed=seed)
    assert np.array_equal(true.nodes.view(np.uint8), est.nodes.view(np.uint8))
    r = LiveSurfaceRaster(96, 72)
    r.rasterize(DeviceMesh(true))
    torch.cuda.synchronize()
    lv, ln, _ = r.maps(96 * 72)
    T = true.T_cam_world.astype(np.float64)
    vc = lv.astype(np.float64) @ T[:3, :3].T + T[:3, 3]
    on = np.linalg.norm(lv, axis=1) > 0
    nc = ln.astype(np.float64) @ T[:3, :3].T
    nc = np.where((np.sum(nc * vc, -1) > 0)[:, None], -nc, nc) * on[:, None]
    P = 96 * 72
    cf = synth.corr_frame(64, 48, seed=1)
    frame = dataclasses.replace(
        cf, width=96, height=72, cam=est.cam, live_vertices=np.zeros((P, 3), np.float32),
        live_normals=np.zeros((P, 3), np.float32), depth=np.where(on, vc[:, 2], 0.0).astype(np.float32),
        depth_normals=nc.astype(np.float32), T_cam_world=est.T_cam_world,
        T_world_cam=np.linalg.inv(T).astype(np.float32), hit_voxel_idx=np.full(P, -1, np.int32),
        voxel_knn=est.voxel_knn, voxel_knn_w=est.voxel_knn_w, pixel_knn=np.zeros((P, 4), np.int32),
        pixel_knn_w=np.zeros((P, 4), np.float32))
    dx = (np.random.default_rng(seed).normal(size=(est.nodes.shape[0], 6)) * [0.01, 0.01, 0.01, 0.003, 0.003, 0.003])
    return est, frame, dx.astype(np.float32)


@pytest.mark.parametrize("knn_out", [True, False])
def test_line_search_matches_host_flow(oracle, knn_out):
    est, frame, dx = _scene()
    N = est.nodes.shape[0]
    P = 96 * 72
    mesh = DeviceMesh(est)
    dframe = DeviceCorrFrame(frame)
    raster = LiveSurfaceRaster(96, 72)
    search = CorrespondenceSearch(96, 72)
    cprm = CorrParams(0.02, 0.3, 0.05, 4)
    lp = LineSearchParams(update_scale=1.0, max_update_rot=0.12, max_update_trans=0.04, min_valid_corrs=50)
    d_dx = torch.from_numpy(dx.reshape(-1).copy()).cuda()
    T0 = mesh.transforms.clone()

    def predict_and_search(T):
        w = torch.empty_like(mesh.canonical)
        mesh.transforms = T
        raster.predict(mesh, w)
        dframe.live_vertices.copy_(raster.live_vertices[: 3 * P])
        dframe.live_normals.copy_(raster.live_normals[: 3 * P])
        dframe.hit_voxel_idx.copy_(raster.hit_voxel_idx[: P])
        search.launch(dframe, cprm, use_voxels=True, pixel_knn_out=True)
        torch.cuda.synchronize()
        n = int(search.num_valid.item())
        outs = dict(warped=w, lv=dframe.live_vertices.clone(), ln=dframe.live_normals.clone(),
                    hit=dframe.hit_voxel_idx.clone(), corrs=search.corrs[: P * CORR_BYTES].clone(),
                    pk=search.pixel_knn.clone(), pkw=search.pixel_knn_w.clone())
        return n, search.records(P), outs

    # the base: the warp as it stands
    base_valid, base_recs, _ = predict_and_search(T0.clone())
    base_rmse = oracle.corr_rmse(base_recs)[2]
    # the reference's host loop, step by step
    u = lp.update_scale
    scales = [u, 0.5 * u, 0.25 * u, 0.125 * u, 0.0625 * u, -0.0625 * u, -0.125 * u, -0.25 * u, -0.5 * u, -u]
    host = []
    for sc in scales:
        T = T0.clone()
        sd = scale_delta(d_dx, N, lp.max_update_rot, lp.max_update_trans, np.float32(sc))
        _lib.check(_lib.lib().cf_warp_apply_twist(ctypes.c_void_p(T.data_ptr()), ctypes.c_void_p(sd.data_ptr()), N,
                                                  lp.max_update_rot, lp.max_update_trans, 1.0, None), "twist")
        torch.cuda.synchronize()
        n, recs, outs = predict_and_search(T)
        host.append((n, oracle.corr_rmse(recs)[2], T.clone(), outs))
    best, best_rmse = 0.0, base_rmse
    need = int(np.float32(0.75) * np.float32(base_valid))
    for sc, (n, rm, _, _) in zip(scales, host):
        if n >= lp.min_valid_corrs and n >= need and np.isfinite(rm) and rm < best_rmse:
            best, best_rmse = sc, rm
    # the device line search from the same start, its outputs poisoned first
    mesh.transforms = T0.clone()
    Tls = mesh.transforms
    warped = torch.full_like(mesh.canonical, float("nan"))
    pk = torch.full((P * 4,), -7, dtype=torch.int32, device="cuda")
    pkw = torch.full((P * 4,), float("nan"), dtype=torch.float32, device="cuda")
    search.corrs.fill_(0xA5)
    ls = LineSearch(N)
    res = ls.run(raster, search, mesh, dframe, Tls, d_dx, base_rmse, base_valid, lp, cprm, warped=warped,
                 pixel_knn_out=(pk, pkw) if knn_out else None)
    torch.cuda.synchronize()
    for t, (n, rm, _, _) in enumerate(host):
        assert res["trial_valid"][t] == n
        assert abs(res["trial_rmse"][t] - rm) <= 1e-12 * rm, (t, res["trial_rmse"][t], rm)
    assert res["best_scale"] == np.float32(best)
    if best != 0.0:
        n_want, _, T_want, outs = host[scales.index(best)]
        assert torch.equal(Tls, T_want)
        assert abs(res["best_rmse"] - best_rmse) <= 1e-12 * best_rmse
        # the accepted warp's skinned mesh (the host flow's skins the same warp)
        assert torch.equal(warped.view(torch.int32), outs["warped"].view(torch.int32))
    else:
        n_want, _, _, outs = host[-1]
        assert torch.equal(Tls, T0)
    # maps, hit voxels, records, valid count and node lists: the accepted
    # trial's (the last trial's when none was accepted)
    assert int(search.num_valid.item()) == n_want
    assert torch.equal(dframe.live_vertices.view(torch.int32), outs["lv"].view(torch.int32))
    assert torch.equal(dframe.live_normals.view(torch.int32), outs["ln"].view(torch.int32))
    assert torch.equal(dframe.hit_voxel_idx, outs["hit"])
    assert torch.equal(search.corrs[: P * CORR_BYTES], outs["corrs"])
    if knn_out:
        assert torch.equal(pk, outs["pk"])
        assert torch.equal(pkw.view(torch.int32), outs["pkw"].view(torch.int32))
    print(f"base RMSE {base_rmse:.6e} ({base_valid} valid); trials {np.array(res['trial_rmse'])}; "
          f"best scale {res['best_scale']}")


def test_line_search_no_step():
    est, frame, dx = _scene(97)
    mesh = DeviceMesh(est)
    T0 = mesh.transforms.clone()
    ls = LineSearch(est.nodes.shape[0])
    res = ls.run(LiveSurfaceRaster(96, 72), CorrespondenceSearch(96, 72), mesh, DeviceCorrFrame(frame),
                 mesh.transforms, torch.from_numpy(dx.reshape(-1).copy()).cuda(), float("inf"), 1000)
    assert res["best_scale"] == 0.0 and all(v == -1 for v in res["trial_valid"])
    assert torch.equal(mesh.transforms, T0)
