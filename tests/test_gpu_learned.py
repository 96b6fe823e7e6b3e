"""The learned initial increment (cf_mpnn.cu, cf_gn_solve_learned).

Gradients and forward outputs of the BF16 kernels are checked against the
FP64 oracle of the network (oracle/mpnn_oracle.py, which rounds the same
quantities to BF16): loss within 1e-4 relative, forward outputs and every
parameter group's gradient within 1e-2 of the group's largest entry (FP32
against FP64 sums over BF16-rounded activations).  Increments and features are
checked against numpy restatements; the solve's fallback against the plain
solve (bitwise); and the trained network's gain on a held-out sequence."""
import numpy as np
import pytest
import torch

from cudafusion_b200 import _lib, learned as L, synth
from cudafusion_b200.solver import DeviceProblem
from cudafusion_b200.synth import _qconj, _qmul, _qrotate, centred_dq, quat_from_rotvec
from cudafusion_b200.types import DQ_DTYPE

pytestmark = pytest.mark.gpu


def _random_graph(rng, N):
    nbr = rng.integers(0, N, size=(N, 8))
    nbr[rng.random((N, 8)) < 0.2] = -1
    return nbr


@pytest.fixture(scope="module")
def net_case():
    import mpnn_oracle as O

    rng = np.random.default_rng(3)
    N = 96
    nbr = _random_graph(rng, N)
    x = rng.normal(size=(N, L.IN)).astype(np.float32)
    y = rng.normal(size=(N, L.OUT)).astype(np.float32)
    w = L.init_weights(7)
    w[-(6 * 64 + 6):] = rng.normal(scale=0.1, size=6 * 64 + 6)  # a live output layer
    net = L.MPNN(N, w)
    net.set_graph(torch.from_numpy(nbr.astype(np.int32)).cuda())
    return O, net, nbr, x, y, w


def test_forward_matches_oracle(net_case):
    O, net, nbr, x, y, w = net_case
    out = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, _ = O.forward(w.astype(np.float64), x, nbr)
    assert np.abs(out - ref).max() <= 1e-2 * np.abs(ref).max()


def test_gradients_match_oracle(net_case):
    O, net, nbr, x, y, w = net_case
    loss, g = net.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda())
    loss_o, g_o = O.loss_and_grad(w.astype(np.float64), x, y, nbr)
    assert abs(loss - loss_o) / loss_o < 1e-4
    o = 0
    for name, shp in O.SHAPES:
        n = int(np.prod(shp))
        a, b = g[o:o + n], g_o[o:o + n]
        assert np.abs(a - b).max() <= 1e-2 * max(np.abs(b).max(), 1e-12), name
        o += n


def test_training_step_lowers_loss(net_case):
    O, net, nbr, x, y, w = net_case
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    l0 = net.gradients(xd, yd)[0]
    for _ in range(20):
        net.train_step(xd, yd, 1e-2)
    l1 = net.gradients(xd, yd)[0]
    net.set_weights(w)
    assert l1 < 0.8 * l0


def _np_increment(Ta, Tb):
    qa, qb = Ta["real"].astype(np.float64), Tb["real"].astype(np.float64)
    ta = 2.0 * _qmul(Ta["dual"].astype(np.float64), _qconj(qa))[:, :3]
    tb = 2.0 * _qmul(Tb["dual"].astype(np.float64), _qconj(qb))[:, :3]
    qd = _qmul(qa, _qconj(qb))
    qd = qd * np.where(qd[:, 3:4] < 0, -1.0, 1.0)
    vn = np.linalg.norm(qd[:, :3], axis=-1, keepdims=True)
    ang = 2 * np.arctan2(vn, qd[:, 3:4])
    w = np.where(vn > 1e-12, qd[:, :3] / np.maximum(vn, 1e-300) * ang, 2 * qd[:, :3])
    return np.concatenate([w, ta - _qrotate(qd, tb)], -1)


def _random_T(rng, n, rot=0.3, trans=0.05):
    return centred_dq(quat_from_rotvec(rng.normal(scale=rot, size=(n, 3))), rng.normal(scale=trans, size=(n, 3)))


def test_increments_match_numpy():
    rng = np.random.default_rng(5)
    Ta, Tb = _random_T(rng, 500), _random_T(rng, 500)
    d = L.increments(torch.from_numpy(Ta.view(np.uint8)).cuda(), torch.from_numpy(Tb.view(np.uint8)).cuda())
    assert np.abs(d.cpu().numpy() - _np_increment(Ta, Tb)).max() < 2e-5


def test_features_match_numpy():
    rng = np.random.default_rng(6)
    p = synth.sphere_problem(num_nodes=128, num_corrs=6000, seed=21)
    N = p.num_nodes
    T = p.init_transforms
    hist = [_random_T(rng, N, 0.05, 0.01) for _ in range(3)]
    s = L.seq_solver(1, N, p.num_corrs)
    dp = DeviceProblem(p)
    dh = torch.from_numpy(np.concatenate(hist).view(np.uint8)).cuda()
    f = L.features(s, dp, dp.init_transforms, dh).cpu().numpy()
    # increments
    chain = [T] + hist
    for k in range(3):
        inc = _np_increment(chain[k], chain[k + 1])
        assert np.abs(f[:, 6 * k:6 * k + 3] - inc[:, :3] * _lib.CF_MPNN_ROT_SCALE).max() < 1e-3
        assert np.abs(f[:, 6 * k + 3:6 * k + 6] - inc[:, 3:] * _lib.CF_MPNN_TRANS_SCALE).max() < 1e-3
    # residual statistics at T (mm)
    src, _ = synth.skin_points_f64(p.canon, p.corrs["node_ids"], p.corrs["node_ws"],
                                   p.nodes["pos"].astype(np.float64), T)
    r = np.abs(np.sum(p.corrs["normal"] * (src - p.corrs["dst"]), -1))
    ok = (p.corrs["valid"] > 0) & (p.corrs["weight"] > 0)
    mean = np.zeros(N)
    mx = np.zeros(N)
    cnt = np.zeros(N)
    for k in range(4):
        ids, ws = p.corrs["node_ids"][:, k], p.corrs["node_ws"][:, k]
        sel = ok & (ids >= 0) & (ws > 1e-8)
        np.add.at(mean, ids[sel], r[sel])
        np.add.at(cnt, ids[sel], 1)
        np.maximum.at(mx, ids[sel], r[sel])
    mean = np.where(cnt > 0, mean / np.maximum(cnt, 1), 0.0)
    assert np.abs(f[:, 18] - mean * 1000).max() < 2e-3
    assert np.abs(f[:, 19] - mx * 1000).max() < 2e-3


def test_rejected_prediction_falls_back_to_plain_bitwise():
    """A history that makes the prediction absurd: the gate rejects it and the
    solve continues from the warm start, bit for bit the plain solve."""
    sf = L.SequenceFrames(synth.cylinder_sequence(seed=5))
    N, M = sf.dp.num_nodes, sf.dp.num_corrs
    dp = sf.frame(10)
    warm = sf.dp.init_transforms.clone()
    rng = np.random.default_rng(1)
    far = torch.from_numpy(np.concatenate([_random_T(rng, N, 0.8, 0.2) for _ in range(3)]).view(np.uint8)).cuda()
    net = L.MPNN(N, np.zeros(L.PARAMS, np.float32))  # prediction = the last increment (absurd here)
    s_l, s_p = L.seq_solver(2, N, M), L.seq_solver(2, N, M)
    Tl, Tp = warm.clone(), warm.clone()
    st = L.solve_learned(s_l, net, dp, Tl, far, *L.CLAMPS)
    s_p.gn_solve(dp, Tp, *L.CLAMPS)
    assert st["init_rejected"] == 1
    assert st["energy_predicted"] > st["energy_warm_start"]
    assert torch.equal(Tl, Tp)


def test_training_beats_constant_velocity():
    data = L.generate([200, 201], 40, gn_target=6)
    net = L.train(data, epochs=6, batch_frames=4)
    val = L.generate([202], 24, gn_target=6)
    net.set_graph(L.graph_of(val[0][0], 1))
    err = np.mean([float(((net.forward(x) - y) ** 2).mean()) for x, y in zip(val[0][1], val[0][2])])
    assert err < 0.8 * L.constant_velocity_loss(val)


def test_trained_network_gain_on_held_out_sequence():
    """The committed network (trained on 2010 frames of other seeds): one GN
    iteration from its start reaches the plain 5-iteration energy within 1 %
    on nearly every frame of the held-out sequence; one iteration from the
    plain warm start does not."""
    net = L.MPNN(4096, np.load(L.WEIGHTS))
    r = L.evaluate(net, frames=40, learned_gn=1, time_it=False)
    ratio = r["learned_energy"] / r["plain_energy"]
    assert np.mean(ratio <= 1.01) >= 0.95
    # the plain solve with one iteration from the same warm starts
    sf = L.SequenceFrames(synth.cylinder_sequence(seed=5))
    N, M = sf.dp.num_nodes, sf.dp.num_corrs
    p5, p1 = L.seq_solver(5, N, M), L.seq_solver(1, N, M)
    tr = L.Track(sf.dp.init_transforms)
    plain1 = []
    for t in range(1, 41):
        dp = sf.frame(t)
        T = tr.warm.clone()
        e5 = p5.gn_solve(dp, T, *L.CLAMPS)["energy_final"]
        if t >= 4:
            e1 = p1.gn_solve(dp, tr.warm.clone(), *L.CLAMPS)["energy_final"]
            plain1.append(e1 / e5)
        tr.push(T)
    assert np.median(ratio) < np.median(plain1)
    assert np.mean(np.array(plain1) <= 1.01) < np.mean(ratio <= 1.01)
