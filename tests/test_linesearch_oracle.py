"""The GN-step acceptance oracle (oracle/cf_oracle_ls.c) against independent
FP64 NumPy restatements of include/fusion_app.h:427-458 (the increment
statistics), :1331-1350 (correspondence_rmse) and :1352-1375
(upload_scaled_delta_x): the scaled increment to one float rounding, the sums
and the RMSE to 1e-12 relative, the maxima and clamps exactly."""
import numpy as np

from cudafusion_b200.types import CORR_DTYPE


def _dx(n, seed):
    rng = np.random.default_rng(seed)
    d = np.concatenate([rng.normal(scale=0.05, size=(n, 3)), rng.normal(scale=0.02, size=(n, 3))], 1)
    d[::11] *= 30.0
    d[3::13] = 0.0
    return d.astype(np.float32)


def test_scale_delta(oracle):
    dx = _dx(500, 1)
    for mr, mt, sc in [(0.12, 0.04, 1.0), (0.12, 0.04, -0.5), (0.0, 0.04, 0.25), (0.05, 0.0, 0.0625)]:
        got = oracle.scale_delta(dx, mr, mt, sc).reshape(-1, 6).astype(np.float64)
        d = dx.astype(np.float64)
        rn, tn = np.linalg.norm(d[:, :3], axis=1), np.linalg.norm(d[:, 3:], axis=1)
        rs = np.where((mr > 0) & (rn > mr), mr / np.maximum(rn, 1e-300), 1.0)
        ts = np.where((mt > 0) & (tn > mt), mt / np.maximum(tn, 1e-300), 1.0)
        want = np.concatenate([d[:, :3] * (rs * sc)[:, None], d[:, 3:] * (ts * sc)[:, None]], 1)
        assert np.allclose(got, want, rtol=3e-7, atol=1e-30)
        # the clamps hold: no node rotates or translates beyond |scale| x the bound
        if mr > 0:
            assert np.all(np.linalg.norm(got[:, :3], axis=1) <= mr * abs(sc) * (1 + 1e-6))
        if mt > 0:
            assert np.all(np.linalg.norm(got[:, 3:], axis=1) <= mt * abs(sc) * (1 + 1e-6))


def test_update_stats(oracle):
    dx = _dx(2000, 2)
    sums, maxima, fin = oracle.update_stats(dx, 0.5, 0.12, 0.04)
    d = dx.astype(np.float64)
    rn, tn = np.linalg.norm(d[:, :3], axis=1), np.linalg.norm(d[:, 3:], axis=1)
    er, et = np.minimum(0.5 * rn, 0.12), np.minimum(0.5 * tn, 0.04)
    assert fin
    assert np.allclose(sums, [rn.sum(), tn.sum(), er.sum(), et.sum()], rtol=1e-6)
    assert np.allclose(maxima, [rn.max(), tn.max(), er.max(), et.max()], rtol=1e-6)
    assert maxima[2] <= np.float32(0.12) and maxima[3] <= np.float32(0.04)
    dx[5, 1] = np.nan
    assert not oracle.update_stats(dx, 0.5, 0.12, 0.04)[2]


def test_corr_rmse(oracle):
    rng = np.random.default_rng(3)
    M = 5000
    r = np.zeros(M, CORR_DTYPE)
    r["src"] = rng.normal(size=(M, 3))
    r["dst"] = r["src"] + rng.normal(scale=0.01, size=(M, 3))
    n = rng.normal(size=(M, 3))
    r["normal"] = n / np.linalg.norm(n, axis=1, keepdims=True)
    r["weight"] = rng.uniform(-0.2, 1.0, M)
    r["valid"] = rng.random(M) < 0.9
    s, w, rmse = oracle.corr_rmse(r)
    keep = (r["valid"] == 1) & (r["weight"] > 0)
    diff = (r["src"].astype(np.float32) - r["dst"].astype(np.float32)).astype(np.float64)
    res = np.sum(r["normal"].astype(np.float64) * diff, axis=1)
    ww = r["weight"].astype(np.float64)
    assert abs(s - np.sum((ww * res * res)[keep])) <= 1e-12 * s
    assert abs(w - ww[keep].sum()) <= 1e-12 * w
    assert abs(rmse - np.sqrt(s / w)) <= 1e-15 * rmse
    r["valid"] = 0
    assert oracle.corr_rmse(r)[2] == float("inf")
