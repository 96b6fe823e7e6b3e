"""GPU parity of the sm_100a solve against the FP64 CPU oracle (and the FP32
reference-order oracle), through the C ABI.

Tolerances (written here): node transforms
within 1e-5 per component and energies within 1e-4 relative of the FP64
oracle after the full 5 x 10 GN/PCG solve; the assembled system within 1e-6
(values, relative to the largest entry) and 1e-5 (rhs); one linearisation's
delta_x within 2e-4 relative (the spread between the FP32 and FP64 oracles on
the same problem is 4e-5: PCG amplifies FP32 rounding)."""
import ctypes

import numpy as np
import pytest
import torch

from cudafusion_b200 import _lib, synth
from cudafusion_b200.solver import DeviceProblem, GaussNewtonSolver, Params, skin_points, to_device
from cudafusion_b200.types import CORR_DTYPE, DQ_DTYPE, NODE_DTYPE, dq_as_array, identity_transforms

pytestmark = pytest.mark.gpu

# (PCG mode, pipelined): grid-wide standard, grid-wide pipelined, single
# cluster, streaming
MODES = [(1, 0), (1, 1), (2, 0), (3, 0)]


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.fixture(scope="module")
def p1():
    return synth.config1()


def make_solver(params, max_nodes=8192, max_corrs=1 << 18, mode=(0, 0), consistent=False):
    s = GaussNewtonSolver(params, max_nodes=max_nodes, max_corrs=max_corrs)
    s.set_option(_lib.CF_OPT_PCG_MODE, mode[0])
    s.set_option(_lib.CF_OPT_PCG_PIPELINED, mode[1])
    if consistent:
        s.set_arap_consistent(True)
    return s


def linearize(s, corrs, nodes, T):
    dn, dT, dc = to_device(nodes), to_device(T), to_device(corrs)
    dx = s.solve(dc, corrs.shape[0], dn, dT, nodes.shape[0])
    torch.cuda.synchronize()
    return dx.cpu().numpy()[: 6 * nodes.shape[0]]


@pytest.mark.parametrize("mode", MODES)
def test_linearize_system_and_dx(p1, oracle, mode):
    prm = Params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    s = make_solver(prm, mode=mode)
    dx = linearize(s, p1.corrs, p1.nodes, p1.init_transforms)
    row_ptr, col_idx, vals, rhs = s.system()
    orp, oci = oracle.build_pattern(p1.nodes)
    assert np.array_equal(row_ptr, orp) and np.array_equal(col_idx, oci)
    A, b, _ = oracle.assemble(p1.corrs, p1.nodes, p1.init_transforms, orp, oci, 10.0, 1e-2, precision="f64")
    assert rel(vals, A) < 1e-6
    assert rel(rhs, b) < 1e-5
    dxo, it, *_ = oracle.linearize_solve(p1.corrs, p1.nodes, p1.init_transforms,
                                         oracle.params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0))
    assert it == 10
    # the pipelined recurrences amplify FP32 rounding at this barely positive
    # definite system (damping 1e-2): a different FMA contraction anywhere
    # upstream moves this gap between 4e-3 and 6e-3 (standard: ~1e-5)
    assert rel(dx, dxo) < (1e-2 if mode[1] else 2e-4)


def fp32_spread(oracle, p, prm_kw, clamps=(0.12, 0.04)):
    """How far the FP32 reference-order oracle lands from the FP64 oracle on
    the same solve: the rounding floor any FP32 implementation shares."""
    prm = oracle.params(**prm_kw)
    T64, E64, I64 = oracle.gn_solve(p, prm, *clamps, precision="f64")
    T32, _, _ = oracle.gn_solve(p, prm, *clamps, precision="f32")
    return T64, E64, I64, float(np.abs(dq_as_array(T64) - dq_as_array(T32)).max())


# (lambda_smooth, lambda_damping): the reference's own damping 1.0
# (config/params.yaml) gives a well-conditioned system; 1e-2 (solver.h
# default) leaves config 1 barely positive definite (lambda_min ~ 7e-5)
CASES = [(10.0, 1.0), (10.0, 1e-2)]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", CASES)
def test_gn_solve_matches_fp64_oracle(p1, oracle, mode, case):
    lam, damp = case
    kw = dict(gn_iterations=5, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=lam, lambda_damping=damp)
    s = make_solver(Params(**kw), mode=mode)
    dp = DeviceProblem(p1)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
    Tg = T.cpu().numpy().view(DQ_DTYPE)
    To, Eo, Io, spread = fp32_spread(oracle, p1, kw)
    assert st["error_flags"] == 0
    assert st["pcg_iterations"] == list(Io)
    # 1e-5 per component or the FP32 floor of this
    # problem, whichever is larger; the pipelined schedule amplifies rounding
    # (pipelined CG residual gap) and gets 20x that floor
    tol = max(1e-5, 1.5 * spread) * (20.0 if mode[1] else 1.0)
    err = np.abs(dq_as_array(Tg) - dq_as_array(To)).max()
    assert err < tol, (err, tol, spread)
    for g, e in enumerate(st["energy"]):
        assert abs(e - Eo[g]) / abs(Eo[g]) < 1e-4, (g, e, Eo[g])


def test_pcg_modes_agree(p1):
    prm = Params(gn_iterations=3, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    dp = DeviceProblem(p1)
    out = []
    for mode in MODES:
        s = make_solver(prm, mode=mode)
        T = dp.init_transforms.clone()
        s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
        out.append(dq_as_array(T.cpu().numpy().view(DQ_DTYPE)))
    assert np.abs(out[0] - out[2]).max() < 1e-5  # grid-wide vs single cluster (same schedule)
    # standard vs pipelined: the pipelined recurrences amplify FP32 rounding
    # (its oracle bar above is 20x the FP32 floor); any change of summation
    # order upstream moves this gap by ~1e-5
    assert np.abs(out[0] - out[1]).max() < 5e-4
    assert np.abs(out[0] - out[3]).max() < 1e-5  # shared-memory vs streaming (FP32-stored inverses)


def test_large_graph_fallback_paths(oracle):
    """17,000 nodes: past the sizes of the shared-memory fast paths of the
    sort (per-warp scatter cursors, the node-to-column map of expand), so the
    global-cursor scatter and the binary-search column lookup run; the solve
    still matches the FP64 oracle within the bar of the other solves."""
    p = synth.sphere_problem(num_nodes=17000, num_corrs=250000, seed=7)
    kw = dict(gn_iterations=2, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0, lambda_damping=1.0)
    s = make_solver(Params(**kw), max_nodes=17000, max_corrs=p.num_corrs)
    dp = DeviceProblem(p)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
    assert st["error_flags"] == 0
    prm = oracle.params(**kw)
    T64, E64, _ = oracle.gn_solve(p, prm, 0.12, 0.04, precision="f64")
    T32, _, _ = oracle.gn_solve(p, prm, 0.12, 0.04, precision="f32")
    spread = float(np.abs(dq_as_array(T64) - dq_as_array(T32)).max())
    err = np.abs(dq_as_array(T.cpu().numpy().view(DQ_DTYPE)) - dq_as_array(T64)).max()
    assert err < max(1e-5, 1.5 * spread), (err, spread)
    assert abs(st["energy_final"] - E64[-1]) / E64[-1] < 1e-4


def test_pcg_kernel_choice_and_full_frame_cluster():
    """Mode 0 runs the single-cluster PCG on a small problem and the grid-wide
    one on the full frame; forced onto one 16-CTA cluster, the full frame
    (2048 nodes, upper blocks in distributed shared memory, transposed
    products pushed between CTAs) lands on the grid-wide result (well
    conditioned: consistent ARAP Jacobian, damping 1)."""
    prm = Params(gn_iterations=2, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0, lambda_damping=1.0)
    p2 = synth.config2()
    dp = DeviceProblem(p2)
    out, active = [], []
    for mode in (0, 1, 2):
        s = make_solver(prm, max_corrs=p2.num_corrs, mode=(mode, 0), consistent=True)
        T = dp.init_transforms.clone()
        st = s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
        assert st["error_flags"] == 0
        active.append(s.get_option(_lib.CF_OPT_PCG_ACTIVE))
        out.append(dq_as_array(T.cpu().numpy().view(DQ_DTYPE)))
    assert active == [1, 1, 2]
    assert np.abs(out[1] - out[2]).max() < 1e-5
    s = make_solver(prm, mode=(0, 0))
    s.gn_solve(DeviceProblem(synth.config1()), DeviceProblem(synth.config1()).init_transforms.clone(), 0.12, 0.04)
    assert s.get_option(_lib.CF_OPT_PCG_ACTIVE) == 2


@pytest.mark.parametrize("mode", MODES)
def test_deterministic(p1, mode):
    prm = Params(gn_iterations=5, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    s = make_solver(prm, mode=mode)
    dp = DeviceProblem(p1)
    runs = []
    for _ in range(3):
        T = dp.init_transforms.clone()
        s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
        runs.append(T.cpu().numpy().tobytes())
    assert runs[0] == runs[1] == runs[2]


def test_tolerance_stop_matches_oracle(p1, oracle):
    """The absolute ||r|| < tol stop (solver_kernels.cu:669) with a tolerance
    that trips mid-solve."""
    prm = Params(gn_iterations=1, pcg_iterations=50, pcg_tolerance=2e-3, lambda_smooth=1.0)
    s = make_solver(prm)
    dp = DeviceProblem(p1)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T)
    _, _, Io = oracle.gn_solve(p1, oracle.params(gn_iterations=1, pcg_iterations=50, pcg_tolerance=2e-3,
                                                 lambda_smooth=1.0))
    assert 0 < st["pcg_iterations"][0] < 50
    assert abs(st["pcg_iterations"][0] - int(Io[0])) <= 1


def test_consistent_arap_decreases_energy(p1, oracle):
    prm = Params(gn_iterations=5, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    s = make_solver(prm, consistent=True)
    dp = DeviceProblem(p1)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
    e = st["energy"]
    assert all(e[k + 1] <= e[k] * (1 + 1e-6) for k in range(len(e) - 1)), e
    oracle.lib().cfo_set_arap_consistent(1)
    try:
        To, Eo, _ = oracle.gn_solve(p1, oracle.params(gn_iterations=5, pcg_iterations=10, pcg_tolerance=0.0,
                                                      lambda_smooth=10.0), max_rot=0.12, max_trans=0.04)
    finally:
        oracle.lib().cfo_set_arap_consistent(0)
    assert abs(e[-1] - Eo[-1]) / Eo[-1] < 1e-4
    assert np.abs(dq_as_array(T.cpu().numpy().view(DQ_DTYPE)) - dq_as_array(To)).max() < 1e-5


def test_apply_twist_matches_oracle(oracle):
    rng = np.random.default_rng(3)
    n = 1000
    T = synth.centred_dq(synth.quat_from_rotvec(rng.normal(size=(n, 3)) * 0.5), rng.normal(size=(n, 3)) * 0.05)
    dx = (rng.normal(size=(n, 6)) * rng.choice([1e-8, 1e-3, 0.05, 0.5], size=(n, 1))).astype(np.float32)
    for max_rot, max_trans, scale in [(0.0, 0.0, 1.0), (0.12, 0.04, 1.0), (0.05, 0.01, -0.5)]:
        dT = to_device(T)
        ddx = torch.from_numpy(dx.ravel().copy()).cuda()
        st = _lib.lib().cf_warp_apply_twist(ctypes.c_void_p(dT.data_ptr()), ctypes.c_void_p(ddx.data_ptr()), n,
                                            max_rot, max_trans, scale, None)
        assert st == 0
        torch.cuda.synchronize()
        got = dT.cpu().numpy().view(DQ_DTYPE)
        want = oracle.apply_twist(T, dx, max_rot, max_trans, scale, precision="f32")
        assert np.abs(dq_as_array(got) - dq_as_array(want)).max() < 2e-6


def test_skin_points_matches_oracle(p1, oracle):
    ids = np.ascontiguousarray(p1.corrs["node_ids"], np.int32)
    ws = np.ascontiguousarray(p1.corrs["node_ws"], np.float32)
    ids[::17, 2] = -1
    ws[::19, 1] = 0.0
    ids[::23, 0] = p1.num_nodes + 5  # out of range: skipped
    out = skin_points(torch.from_numpy(p1.canon.copy()).cuda(), torch.from_numpy(ids).cuda(),
                      torch.from_numpy(ws).cuda(), to_device(p1.nodes), to_device(p1.gt_transforms), p1.num_nodes)
    want = oracle.skin(p1.canon, ids, ws, p1.nodes, p1.gt_transforms, precision="f32")
    assert np.abs(out.cpu().numpy() - want).max() < 2e-6


def degenerate_corrs(p):
    c = p.corrs.copy()
    rng = np.random.default_rng(5)
    M = c.shape[0]
    c["valid"][rng.choice(M, M // 20, replace=False)] = 0
    c["weight"][rng.choice(M, M // 50, replace=False)] = -1.0
    c["weight"][rng.choice(M, M // 50, replace=False)] = 0.0
    c["weight"][rng.choice(M, 7, replace=False)] = np.nan
    sel = rng.choice(M, M // 30, replace=False)
    c["node_ids"][sel, 3] = -1
    sel = rng.choice(M, M // 30, replace=False)
    c["node_ids"][sel, 2] = p.num_nodes + 3  # out of range
    sel = rng.choice(M, M // 40, replace=False)
    c["node_ws"][sel, 1] = 1e-9  # below the 1e-8 weight cut
    sel = rng.choice(M, M // 40, replace=False)
    c["node_ids"][sel, 1] = c["node_ids"][sel, 0]  # duplicated node
    far = rng.choice(M, M // 50, replace=False)
    c["dst"][far] += 1.0  # Huber-damped outliers
    return c


@pytest.mark.parametrize("mode", MODES)
def test_degenerate_correspondences(p1, oracle, mode):
    c = degenerate_corrs(p1)
    prm = Params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=3.0)
    s = make_solver(prm, mode=mode)
    T = p1.gt_transforms
    dx = linearize(s, c, p1.nodes, T)
    row_ptr, col_idx, vals, rhs = s.system()
    A, b, _ = oracle.assemble(c, p1.nodes, T, row_ptr, col_idx, 3.0, 1e-2, precision="f64")
    assert rel(vals, A) < 1e-6
    assert rel(rhs, b) < 1e-5
    dxo, *_ = oracle.linearize_solve(c, p1.nodes, T, oracle.params(pcg_iterations=10, pcg_tolerance=0.0,
                                                                   lambda_smooth=3.0))
    # the pipelined recurrences amplify FP32 rounding at this barely positive
    # definite system (damping 1e-2): a different FMA contraction anywhere
    # upstream moves this gap between 4e-3 and 6e-3 (standard: ~1e-5)
    assert rel(dx, dxo) < (1e-2 if mode[1] else 2e-4)


def test_no_correspondences(p1, oracle):
    prm = Params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=1.0)
    s = make_solver(prm)
    empty = np.zeros(0, CORR_DTYPE)
    T = p1.gt_transforms
    dx = linearize(s, empty, p1.nodes, T)
    dxo, *_ = oracle.linearize_solve(empty, p1.nodes, T, oracle.params(pcg_iterations=10, pcg_tolerance=0.0))
    assert rel(dx, dxo) < 2e-4
    _, _, vals, rhs = s.system()
    assert np.isfinite(vals).all() and np.isfinite(rhs).all()


def test_isolated_nodes_and_single_node(oracle):
    p = synth.sphere_problem(num_nodes=40, num_corrs=2000, seed=11)
    nodes = p.nodes.copy()
    nodes["num_neighbors"][:5] = 0  # no outgoing edges
    nodes["neighbors"][5:8, 3:] = -1  # shortened lists
    prm = Params(pcg_iterations=8, pcg_tolerance=0.0)
    s = make_solver(prm)
    dx = linearize(s, p.corrs, nodes, p.gt_transforms)
    dxo, *_ = oracle.linearize_solve(p.corrs, nodes, p.gt_transforms, oracle.params(pcg_iterations=8,
                                                                                   pcg_tolerance=0.0))
    assert rel(dx, dxo) < 2e-4
    one = nodes[:1].copy()
    one["num_neighbors"] = 0
    c = p.corrs.copy()
    c["node_ids"][:] = np.array([0, -1, -1, -1])
    c["node_ws"][:] = np.array([1.0, 0, 0, 0])
    s1 = make_solver(prm)
    dx1 = linearize(s1, c, one, identity_transforms(1))
    dxo1, *_ = oracle.linearize_solve(c, one, identity_transforms(1), oracle.params(pcg_iterations=8,
                                                                                     pcg_tolerance=0.0))
    assert rel(dx1, dxo1) < 2e-4


def test_pattern_invalidation(p1, oracle):
    """Topology change at constant N: the reference keeps its cached pattern
    (solver_kernels.cu:554); cf_gn_invalidate_pattern rebuilds it."""
    prm = Params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=2.0)
    s = make_solver(prm)
    linearize(s, p1.corrs, p1.nodes, p1.init_transforms)
    nodes2 = p1.nodes.copy()
    nodes2["neighbors"] = np.roll(nodes2["neighbors"], 1, axis=0)
    s.invalidate_pattern()
    dx = linearize(s, p1.corrs, nodes2, p1.gt_transforms)
    dxo, *_ = oracle.linearize_solve(p1.corrs, nodes2, p1.gt_transforms,
                                     oracle.params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=2.0))
    assert rel(dx, dxo) < 2e-4


def test_capacity_and_argument_errors(p1):
    prm = Params()
    s = make_solver(prm, max_nodes=64, max_corrs=100)
    dn, dT, dc = to_device(p1.nodes), to_device(p1.init_transforms), to_device(p1.corrs)
    dx = torch.zeros(6 * p1.num_nodes, device="cuda")
    L = _lib.lib()
    vp = ctypes.c_void_p
    st = L.cf_gn_linearize_solve(s._h, vp(dc.data_ptr()), 1000, vp(dn.data_ptr()), vp(dT.data_ptr()), 50,
                                 vp(dx.data_ptr()), None)
    assert st == _lib.CF_ERR_CAPACITY
    st = L.cf_gn_linearize_solve(s._h, vp(dc.data_ptr()), 10, None, vp(dT.data_ptr()), 50, vp(dx.data_ptr()), None)
    assert st == _lib.CF_ERR_INVALID_ARG
    st = L.cf_gn_linearize_solve(s._h, vp(dc.data_ptr() + 2), 10, vp(dn.data_ptr()), vp(dT.data_ptr()), 50,
                                 vp(dx.data_ptr()), None)
    assert st == _lib.CF_ERR_INVALID_ARG


def test_unaligned_correspondence_array(p1, oracle):
    """Correspondences at a 4-byte (not 16-byte) aligned address take the
    word-wise staging path."""
    prm = Params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    s = make_solver(prm)
    raw = np.ascontiguousarray(p1.corrs).view(np.uint8)
    buf = torch.zeros(raw.size + 16, dtype=torch.uint8, device="cuda")
    buf[4:4 + raw.size].copy_(torch.from_numpy(raw.copy()))
    dn, dT = to_device(p1.nodes), to_device(p1.init_transforms)
    dx = torch.zeros(6 * p1.num_nodes, device="cuda")
    vp = ctypes.c_void_p
    st = _lib.lib().cf_gn_linearize_solve(s._h, vp(buf.data_ptr() + 4), p1.num_corrs, vp(dn.data_ptr()),
                                          vp(dT.data_ptr()), p1.num_nodes, vp(dx.data_ptr()), None)
    assert st == 0
    torch.cuda.synchronize()
    dxo, *_ = oracle.linearize_solve(p1.corrs, p1.nodes, p1.init_transforms,
                                     oracle.params(pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0))
    assert rel(dx.cpu().numpy(), dxo) < 2e-4


def test_graph_replay_matches_direct_launches(p1):
    """The captured GN loop (CF_OPT_GRAPH, on a non-default stream) gives the
    bits of direct launches, on the capturing call, on replay, and with new
    correspondence buffers of the same sizes (replayed, not re-captured)."""
    prm = Params(gn_iterations=3, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    side = torch.cuda.Stream()
    dp = DeviceProblem(p1)
    out = {}
    for graph in (0, 1):
        s = make_solver(prm)
        s.set_option(_lib.CF_OPT_GRAPH, graph)
        runs = []
        with torch.cuda.stream(side):
            for k in range(3):
                if k == 2:  # new buffers holding the same correspondences
                    dp.corrs = dp.corrs.clone()
                    dp.canon = dp.canon.clone()
                T = dp.init_transforms.clone()
                n0 = s.launch_count()
                st = s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04, stream=side)
                runs.append((T.cpu().numpy().tobytes(), st["energy_final"], s.launch_count() - n0))
                assert s.get_option(_lib.CF_OPT_GRAPH_ACTIVE) == graph
        side.synchronize()
        out[graph] = runs
    for k in range(3):
        assert out[1][k][0] == out[0][k][0]
        assert out[1][k][1] == out[0][k][1]
        assert out[1][k][2] == out[0][k][2]  # the launches a replay stands for


@pytest.mark.parametrize("mode", [1, 3])
def test_barrier_timeout_is_reported_and_the_context_survives(p1, oracle, mode):
    """Failure detection without a GPU fault: a PCG barrier that waits for an
    arrival nobody makes gives up after its (short) poll limit; the solve
    reports CF_ERR_TIMEOUT, and the next solve on the same handle is exact."""
    prm = Params(gn_iterations=2, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0)
    s = make_solver(prm, mode=(mode, 0))
    dp = DeviceProblem(p1)
    s.set_option(_lib.CF_OPT_SPIN_LIMIT, 20000)
    s.set_option(_lib.CF_OPT_TEST_BARRIER_EXTRA, 1)
    T = dp.init_transforms.clone()
    with pytest.raises(_lib.CFError) as e:
        s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
    assert e.value.status == _lib.CF_ERR_TIMEOUT
    s.set_option(_lib.CF_OPT_TEST_BARRIER_EXTRA, 0)
    s.set_option(_lib.CF_OPT_SPIN_LIMIT, 0)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T, max_rot=0.12, max_trans=0.04)
    assert st["error_flags"] == 0
    ref = make_solver(prm, mode=(mode, 0))
    T2 = dp.init_transforms.clone()
    ref.gn_solve(dp, T2, max_rot=0.12, max_trans=0.04)
    assert torch.equal(T, T2)
