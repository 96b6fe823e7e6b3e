"""Seeded synthetic warp-field problems.

CUDAFusion tracks real RGB-D sequences (VolumeDeform recordings referenced by
config/params.yaml:2-3); none ship with it, so these generators build problems
of the same shapes and statistics.  Nothing here is on the solve path: it
creates inputs for the tests and the benchmark.

Conventions follow the reference:
  * node transforms are DualQuats centred at their node, T(p) = R(p-c)+c+t
    (include/se3_math.cuh:379-415);
  * a point is skinned by its 4 nearest nodes with weights
    exp(-d^2 / (2 r^2)) normalised (src/warp_field.cu:379-404);
  * graph edges go to the K_GRAPH=8 nearest nodes with weights
    exp(-d^2 / (2 r^2)) (src/warp_field.cu:889, Euclidean instead of geodesic);
  * depth normals use forward differences flipped toward the camera
    (kernels/tsdf_kernels.cu:180-230).
"""
from dataclasses import dataclass, field

import numpy as np
from scipy.spatial import cKDTree

from .types import CORR_DTYPE, DQ_DTYPE, K_GRAPH, K_NEIGHBORS, NODE_DTYPE, identity_transforms


@dataclass
class Problem:
    """One warp-field solve: graph, correspondences with canonical points,
    initial transforms, and (when known) the ground-truth transforms."""

    nodes: np.ndarray  # NODE_DTYPE[N]
    canon: np.ndarray  # float32[M, 3]
    corrs: np.ndarray  # CORR_DTYPE[M] (src = canonical point)
    init_transforms: np.ndarray  # DQ_DTYPE[N]
    gt_transforms: np.ndarray = None  # DQ_DTYPE[N]
    meta: dict = field(default_factory=dict)

    @property
    def num_nodes(self):
        return int(self.nodes.shape[0])

    @property
    def num_corrs(self):
        return int(self.corrs.shape[0])

    def save(self, path):
        np.savez_compressed(
            path,
            nodes=self.nodes.view(np.uint8),
            canon=self.canon,
            corrs=self.corrs.view(np.uint8),
            init_transforms=self.init_transforms.view(np.uint8),
            gt_transforms=(self.gt_transforms if self.gt_transforms is not None else identity_transforms(0)).view(
                np.uint8
            ),
        )

    @staticmethod
    def load(path):
        z = np.load(path)
        gt = z["gt_transforms"].view(DQ_DTYPE)
        return Problem(
            nodes=z["nodes"].view(NODE_DTYPE).copy(),
            canon=z["canon"].copy(),
            corrs=z["corrs"].view(CORR_DTYPE).copy(),
            init_transforms=z["init_transforms"].view(DQ_DTYPE).copy(),
            gt_transforms=gt.copy() if gt.shape[0] else None,
        )


# --------------------------------------------------------------------------
# small FP64 quaternion helpers (x, y, z, w storage)
# --------------------------------------------------------------------------


def _qmul(a, b):
    ax, ay, az, aw = np.moveaxis(a, -1, 0)
    bx, by, bz, bw = np.moveaxis(b, -1, 0)
    return np.stack(
        [
            aw * bx + ax * bw + ay * bz - az * by,
            aw * by - ax * bz + ay * bw + az * bx,
            aw * bz + ax * by - ay * bx + az * bw,
            aw * bw - ax * bx - ay * by - az * bz,
        ],
        -1,
    )


def _qconj(q):
    return q * np.array([-1.0, -1.0, -1.0, 1.0])


def quat_from_rotvec(w):
    w = np.asarray(w, np.float64)
    th = np.linalg.norm(w, axis=-1, keepdims=True)
    s = np.where(th > 1e-12, np.sin(0.5 * th) / np.maximum(th, 1e-300), 0.5)
    return np.concatenate([w * s, np.cos(0.5 * th)], -1)


def _qrotate(q, v):
    vq = np.concatenate([v, np.zeros(v.shape[:-1] + (1,))], -1)
    return _qmul(_qmul(q, vq), _qconj(q))[..., :3]


def centred_dq(q, t):
    """Centred DualQuat from rotation quaternion q and centred translation t."""
    out = np.zeros(q.shape[0], DQ_DTYPE)
    tq = np.concatenate([t, np.zeros((t.shape[0], 1))], -1)
    out["real"] = q
    out["dual"] = 0.5 * _qmul(tq, q)
    return out


def skin_points_f64(points, ids, ws, node_pos, transforms):
    """FP64 DQ-blend skinning (the math of se3_math.cuh:450-510) for data
    generation.  Returns warped points and the blended rotation quaternions."""
    real = transforms["real"].astype(np.float64)
    dual = transforms["dual"].astype(np.float64)
    t = 2.0 * _qmul(dual, _qconj(real))[:, :3]
    rc = _qrotate(real, node_pos.astype(np.float64))
    t_plain = t + node_pos - rc  # dq_centered: plain translation
    dual_plain = 0.5 * _qmul(np.concatenate([t_plain, np.zeros((len(t_plain), 1))], -1), real)
    br = np.zeros((points.shape[0], 4))
    bd = np.zeros((points.shape[0], 4))
    wsum = np.zeros(points.shape[0])
    for k in range(K_NEIGHBORS):
        nid = ids[:, k]
        w = ws[:, k].astype(np.float64)
        ok = (nid >= 0) & (w >= 1e-8)
        nidc = np.where(ok, nid, 0)
        qr = real[nidc]
        qd = dual_plain[nidc]
        flip = np.sum(qr * br, -1) < 0
        sgn = np.where(flip, -1.0, 1.0)[:, None]
        wk = np.where(ok, w, 0.0)[:, None]
        br += wk * sgn * qr
        bd += wk * sgn * qd
        wsum += wk[:, 0]
    n = np.linalg.norm(br, axis=-1, keepdims=True)
    br = br / np.maximum(n, 1e-300)
    bd = bd / np.maximum(n, 1e-300)
    tb = 2.0 * _qmul(bd, _qconj(br))[:, :3]
    out = _qrotate(br, points.astype(np.float64)) + tb
    keep = wsum < 1e-8
    out[keep] = points[keep]
    br[keep] = np.array([0.0, 0.0, 0.0, 1.0])
    return out, br


def _graph(node_pos, node_radius):
    n = node_pos.shape[0]
    tree = cKDTree(node_pos)
    kq = min(K_GRAPH + 1, n)
    d, idx = tree.query(node_pos, k=kq)
    d = d.reshape(n, kq)[:, 1:]
    idx = idx.reshape(n, kq)[:, 1:]
    nb = np.full((n, K_GRAPH), -1, np.int32)
    nw = np.zeros((n, K_GRAPH), np.float32)
    nb[:, : kq - 1] = idx
    r = np.maximum(node_radius, 1e-6)
    nw[:, : kq - 1] = np.exp(-(d**2) / (2.0 * r * r))
    return nb, nw, kq - 1


def _skin_weights(points, node_pos, node_radius, tree=None):
    tree = tree if tree is not None else cKDTree(node_pos)
    d, idx = tree.query(points, k=K_NEIGHBORS, workers=-1)
    d2 = (d.astype(np.float64)) ** 2
    r = np.maximum(node_radius, 1e-6)
    w = np.exp(-d2 / (2.0 * r * r))
    s = w.sum(-1, keepdims=True)
    w = np.where(s > 1e-8, w / np.maximum(s, 1e-300), 0.0)
    return idx.astype(np.int32), w.astype(np.float32)


def _make_nodes(pos, normals, radius, nb, nw, kcount):
    nodes = np.zeros(pos.shape[0], NODE_DTYPE)
    nodes["pos"] = pos
    nodes["normal"] = normals
    nodes["radius"] = radius
    nodes["neighbors"] = nb
    nodes["neighbor_w"] = nw
    nodes["num_neighbors"] = kcount
    return nodes


def _smooth_field(rng, x, amplitude, scale, terms=3):
    """Low-frequency random vector field with max norm `amplitude` over x."""
    f = np.zeros((x.shape[0], 3))
    for _ in range(terms):
        k = rng.normal(size=3) / scale
        a = rng.normal(size=3)
        ph = rng.uniform(0, 2 * np.pi)
        f += np.sin(x @ k + ph)[:, None] * a[None, :]
    m = np.linalg.norm(f, axis=-1).max()
    return f * (amplitude / max(m, 1e-12))


def _fibonacci_sphere(n, rng):
    i = np.arange(n) + 0.5
    phi = np.arccos(1 - 2 * i / n)
    th = np.pi * (1 + 5**0.5) * i
    p = np.stack([np.cos(th) * np.sin(phi), np.sin(th) * np.sin(phi), np.cos(phi)], -1)
    # random global rotation + small jitter: a blue-noise (Poisson-disk-like) set
    q = quat_from_rotvec(rng.normal(size=3))
    p = _qrotate(np.broadcast_to(q, (n, 4)), p)
    p += rng.normal(scale=0.15 * np.sqrt(4 * np.pi / n), size=p.shape)
    return p / np.linalg.norm(p, axis=-1, keepdims=True)


def sphere_problem(
    num_nodes=256,
    num_corrs=20000,
    radius=0.3,
    node_radius=0.025,
    max_rot_deg=15.0,
    max_trans=0.02,
    noise=0.001,
    outlier_frac=0.05,
    outlier_radius=0.05,
    seed=1,
    center=(0.0, 0.0, 1.0),
):
    """Sphere of `radius` with Poisson-disk-like nodes, uniform surface
    correspondences, a low-frequency ground-truth warp (<= max_rot_deg,
    <= max_trans), point-to-plane targets with sigma=`noise` along the normal
    and `outlier_frac` uniform outliers within `outlier_radius`.  The initial
    transforms are identity."""
    rng = np.random.default_rng(seed)
    c = np.asarray(center, np.float64)
    nrm_nodes = _fibonacci_sphere(num_nodes, rng)
    node_pos = c + radius * nrm_nodes
    nb, nw, kc = _graph(node_pos, node_radius)
    nodes = _make_nodes(node_pos, nrm_nodes, node_radius, nb, nw, kc)

    v = rng.normal(size=(num_corrs, 3))
    nrm = v / np.linalg.norm(v, axis=-1, keepdims=True)
    canon = c + radius * nrm
    tree = cKDTree(node_pos)
    ids, ws = _skin_weights(canon, node_pos, node_radius, tree)

    rotv = _smooth_field(rng, node_pos - c, np.deg2rad(max_rot_deg), radius)
    trans = _smooth_field(rng, node_pos - c, max_trans, radius)
    gt = centred_dq(quat_from_rotvec(rotv), trans)

    live, q = skin_points_f64(canon, ids, ws, node_pos, gt)
    n_live = _qrotate(q, nrm)
    dst = live + rng.normal(scale=noise, size=(num_corrs, 1)) * n_live
    n_out = int(round(outlier_frac * num_corrs))
    out_idx = rng.choice(num_corrs, size=n_out, replace=False)
    u = rng.normal(size=(n_out, 3))
    u /= np.linalg.norm(u, axis=-1, keepdims=True)
    dst[out_idx] += u * (outlier_radius * rng.uniform(0, 1, size=(n_out, 1)) ** (1 / 3))

    corrs = np.zeros(num_corrs, CORR_DTYPE)
    corrs["src"] = canon
    corrs["dst"] = dst
    corrs["normal"] = n_live
    corrs["node_ids"] = ids
    corrs["node_ws"] = ws
    corrs["weight"] = 1.0
    corrs["valid"] = 1
    return Problem(
        nodes=nodes,
        canon=canon.astype(np.float32),
        corrs=corrs,
        init_transforms=identity_transforms(num_nodes),
        gt_transforms=gt,
        meta=dict(kind="sphere", seed=seed, num_nodes=num_nodes, num_corrs=num_corrs, outliers=n_out),
    )


# --------------------------------------------------------------------------
# articulated two-cylinder surface seen by a pinhole camera
# --------------------------------------------------------------------------


def _rot_y(angle):
    return quat_from_rotvec(np.array([0.0, angle, 0.0]))


def _blue_noise_subsample(points, n, rng):
    """Indices of exactly n points of a dense cloud, one per occupied cell of
    a grid whose cell size is tuned to give about n cells (Poisson-disk-like),
    and that cell size."""
    lo = points.min(0)
    ext = float((points.max(0) - lo).max())
    perm = rng.permutation(points.shape[0])
    pts = points[perm]
    a, b = ext / (4 * n) ** 0.5 * 1e-2, ext
    for _ in range(40):
        h = 0.5 * (a + b)
        keys = np.floor((pts - lo) / h).astype(np.int64)
        k = (keys[:, 0] * 73856093) ^ (keys[:, 1] * 19349663) ^ (keys[:, 2] * 83492791)
        cnt = np.unique(k).shape[0]
        if cnt >= n:
            a = h
        else:
            b = h
    h = a
    keys = np.floor((pts - lo) / h).astype(np.int64)
    k = (keys[:, 0] * 73856093) ^ (keys[:, 1] * 19349663) ^ (keys[:, 2] * 83492791)
    _, first = np.unique(k, return_index=True)
    if first.shape[0] > n:
        first = rng.choice(first, size=n, replace=False)
    return np.sort(perm[first]), h


def _ray_tube(dirs, axis_pt, axis_dir, radius, smin, smax):
    """Nearest intersection of rays from the origin with a capless tube."""
    o = -axis_pt
    w = axis_dir
    dw = dirs @ w
    ow = o @ w
    dperp = dirs - dw[:, None] * w
    operp = o - ow * w
    a = np.sum(dperp * dperp, -1)
    b = 2.0 * (dperp @ operp)
    c = operp @ operp - radius * radius
    disc = b * b - 4 * a * c
    ok = disc > 0
    sq = np.sqrt(np.where(ok, disc, 0.0))
    t = (-b - sq) / np.maximum(2 * a, 1e-300)
    s = ow + t * dw
    ok &= (t > 0) & (s >= smin) & (s <= smax)
    return np.where(ok, t, np.inf), s


def cylinder_problem(
    width=640,
    height=480,
    fx=570.342,
    fy=570.342,
    cx=320.0,
    cy=240.0,
    num_nodes=2048,
    radii=(0.06, 0.05),
    lengths=(0.08, 0.09),
    distance=0.14,
    bend_deg=30.0,
    init_bend_deg=24.0,
    twist_deg=0.0,
    init_twist_deg=0.0,
    noise=0.001,
    seed=2,
    nodes_cache=None,
):
    """Articulated two-cylinder surface (radii 6 and 5 cm) bent by `bend_deg`
    at the joint, rendered as a width x height depth image.  Canonical pose is
    straight; the live depth is at (bend_deg, twist_deg); the initial
    transforms are the exact warp at (init_bend_deg, init_twist_deg), i.e. a
    warm start from the previous frame.  Correspondences are the valid depth
    pixels with forward-difference depth normals; targets carry sigma=`noise`
    depth noise."""
    rng = np.random.default_rng(seed)
    joint = np.array([0.0, 0.0, distance])

    def seg2_quat(bend, twist):
        qb = _rot_y(np.deg2rad(bend))
        qt = quat_from_rotvec(np.array([np.deg2rad(twist), 0.0, 0.0]))
        return _qmul(qb, qt)

    q_live = seg2_quat(bend_deg, twist_deg)
    w2 = _qrotate(q_live, np.array([1.0, 0.0, 0.0]))

    u, v = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    dirs = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u)], -1).reshape(-1, 3)
    t1, _ = _ray_tube(dirs, joint, np.array([1.0, 0.0, 0.0]), radii[0], -lengths[0], 0.0)
    t2, _ = _ray_tube(dirs, joint, w2, radii[1], 0.0, lengths[1])
    seg = np.where(t2 < t1, 1, 0)
    t = np.minimum(t1, t2)
    hit = np.isfinite(t)
    depth = np.where(hit, t, 0.0).reshape(height, width)  # z of dir is 1 -> t is depth
    segimg = np.where(hit, seg, -1).reshape(height, width)

    # forward-difference normals from the clean depth (tsdf_kernels.cu:180-230)
    P = dirs.reshape(height, width, 3) * depth[..., None]
    dx = P[:-1, 1:] - P[:-1, :-1]
    dy = P[1:, :-1] - P[:-1, :-1]
    n = np.cross(dx, dy)
    nn = np.linalg.norm(n, axis=-1, keepdims=True)
    n = -n / np.maximum(nn, 1e-12)
    d00, d01, d10 = depth[:-1, :-1], depth[:-1, 1:], depth[1:, :-1]
    s00, s01, s10 = segimg[:-1, :-1], segimg[:-1, 1:], segimg[1:, :-1]
    good = (d00 > 0) & (d01 > 0) & (d10 > 0) & (s00 == s01) & (s00 == s10) & (nn[..., 0] > 1e-12)
    good &= (np.abs(d01 - d00) < 0.01) & (np.abs(d10 - d00) < 0.01)
    vv, uu = np.nonzero(good)
    pix = vv * width + uu
    live = P[vv, uu]
    nrm = n[vv, uu]
    sg = s00[vv, uu]

    # canonical point: undo the live articulation of segment 2
    canon = live.copy()
    m2 = sg == 1
    qi = np.broadcast_to(_qconj(q_live), (int(m2.sum()), 4))
    if np.any(m2):
        canon[m2] = joint + _qrotate(qi, live[m2] - joint)
    if nodes_cache is None:
        # the canonical model holds the surface seen so far: sample the nodes
        # from the visible canonical surface (blue-noise subsampling)
        cnrm = nrm.copy()
        if np.any(m2):
            cnrm[m2] = _qrotate(qi, nrm[m2])
        sel, h = _blue_noise_subsample(canon, num_nodes, rng)
        node_pos = canon[sel]
        node_radius = h
        nb, nw, kc = _graph(node_pos, node_radius)
        nodes = _make_nodes(node_pos, cnrm[sel], node_radius, nb, nw, kc)
        tree = cKDTree(node_pos)
    else:
        nodes, tree = nodes_cache
        node_pos = nodes["pos"].astype(np.float64)
        node_radius = float(nodes["radius"][0])
    # noisy target: depth noise along the viewing ray
    z = depth[vv, uu] + rng.normal(scale=noise, size=vv.shape[0])
    dst = dirs[pix] * z[:, None]

    ids, ws = _skin_weights(canon, node_pos, node_radius, tree)
    M = canon.shape[0]
    corrs = np.zeros(M, CORR_DTYPE)
    corrs["src"] = canon
    corrs["dst"] = dst
    corrs["normal"] = nrm
    corrs["node_ids"] = ids
    corrs["node_ws"] = ws
    corrs["weight"] = 1.0
    corrs["valid"] = 1

    def warp_at(bend, twist):
        q2 = seg2_quat(bend, twist)
        on2 = node_pos[:, 0] > joint[0]
        q = np.where(on2[:, None], np.broadcast_to(q2, (len(node_pos), 4)), np.array([0.0, 0.0, 0.0, 1.0]))
        # centred translation: t = R (x - J) + J - x
        t = _qrotate(q, node_pos - joint) + joint - node_pos
        return centred_dq(q, t)

    return Problem(
        nodes=nodes,
        canon=canon.astype(np.float32),
        corrs=corrs,
        init_transforms=warp_at(init_bend_deg, init_twist_deg),
        gt_transforms=warp_at(bend_deg, twist_deg),
        meta=dict(
            kind="cylinders",
            seed=seed,
            width=width,
            height=height,
            num_nodes=int(nodes.shape[0]),
            num_corrs=int(M),
            coverage=float(hit.mean()),
            bend_deg=bend_deg,
            twist_deg=twist_deg,
        ),
    )


# --------------------------------------------------------------------------
# named workloads
# --------------------------------------------------------------------------


def config1(seed=1):
    """Small plain solve: sphere r=0.3 m, N=256, M=20k, <=15 deg / 2 cm warp."""
    return sphere_problem(num_nodes=256, num_corrs=20000, seed=seed)


def config2(seed=2):
    """Full frame: 640x480 two-cylinder depth, N=2048, M~300k."""
    return cylinder_problem(seed=seed)


def config3(seed=3):
    """Precision study: 1280x960, N=8192, M~1.2M."""
    return cylinder_problem(
        width=1280, height=960, fx=2 * 570.342, fy=2 * 570.342, cx=640.0, cy=480.0, num_nodes=8192, seed=seed
    )


def config4(num_problems=64, seed=4, n_range=(500, 8000), corr_per_node=150):
    """Batched uneven solves: N ~ U[500, 8000], M = 150 N +- 20 %, warps
    <= 20 deg / 3 cm, sigma 1 mm, 5 % outliers (sphere generator)."""
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(num_problems):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        m = int(round(corr_per_node * n * rng.uniform(0.8, 1.2)))
        radius = float(rng.uniform(0.2, 0.4))
        spacing = np.sqrt(4 * np.pi * radius**2 / n)
        probs.append(
            sphere_problem(
                num_nodes=n,
                num_corrs=m,
                radius=radius,
                node_radius=spacing,
                max_rot_deg=20.0,
                max_trans=0.03,
                seed=int(rng.integers(1 << 30)),
            )
        )
    return probs


# --------------------------------------------------------------------------
# sequences (the learned-initialisation workload)
# --------------------------------------------------------------------------


@dataclass
class Sequence:
    """A two-cylinder surface articulating over time.  The canonical model
    (nodes, surface points, their skin weights) is fixed; frame t places the
    second segment at bend(t), twist(t) about the joint and observes every
    model point with depth noise along its viewing ray.  Motion:
    bend(t) = A/2 (1 - cos(2 pi (t + t0) / period)), twist(t) = W sin(2 pi (t + t1) / twist_period)."""

    nodes: np.ndarray
    canon: np.ndarray  # float32 [M, 3]
    canon_normals: np.ndarray  # float64 [M, 3]
    on_seg2: np.ndarray  # bool [M]
    node_ids: np.ndarray  # int32 [M, 4]
    node_ws: np.ndarray  # float32 [M, 4]
    joint: np.ndarray
    bend_amp_deg: float = 45.0
    period: float = 60.0
    phase: float = 0.0
    twist_amp_deg: float = 10.0
    twist_period: float = 150.0
    twist_phase: float = 0.0
    noise: float = 0.001
    seed: int = 5

    @property
    def num_nodes(self):
        return int(self.nodes.shape[0])

    @property
    def num_corrs(self):
        return int(self.canon.shape[0])

    def pose(self, t):
        bend = 0.5 * self.bend_amp_deg * (1.0 - np.cos(2.0 * np.pi * (t + self.phase) / self.period))
        twist = self.twist_amp_deg * np.sin(2.0 * np.pi * (t + self.twist_phase) / self.twist_period)
        return bend, twist

    def _seg2_quat(self, t):
        bend, twist = self.pose(t)
        return _qmul(_rot_y(np.deg2rad(bend)), quat_from_rotvec(np.array([np.deg2rad(twist), 0.0, 0.0])))

    def gt_transforms(self, t):
        """Exact articulation of the nodes at frame t (centred DualQuats)."""
        q2 = self._seg2_quat(t)
        pos = self.nodes["pos"].astype(np.float64)
        on2 = pos[:, 0] > self.joint[0]
        q = np.where(on2[:, None], np.broadcast_to(q2, (len(pos), 4)), np.array([0.0, 0.0, 0.0, 1.0]))
        tr = _qrotate(q, pos - self.joint) + self.joint - pos
        return centred_dq(q, tr)

    def frame(self, t):
        """Correspondences of frame t (src = canonical point)."""
        rng = np.random.default_rng((self.seed, int(t)))
        q2 = self._seg2_quat(t)
        live = self.canon.astype(np.float64).copy()
        nrm = self.canon_normals.copy()
        m = self.on_seg2
        qb = np.broadcast_to(q2, (int(m.sum()), 4))
        live[m] = self.joint + _qrotate(qb, live[m] - self.joint)
        nrm[m] = _qrotate(qb, nrm[m])
        z = live[:, 2]
        dst = live * ((z + rng.normal(scale=self.noise, size=z.shape)) / z)[:, None]
        corrs = np.zeros(self.num_corrs, CORR_DTYPE)
        corrs["src"] = self.canon
        corrs["dst"] = dst
        corrs["normal"] = nrm
        corrs["node_ids"] = self.node_ids
        corrs["node_ws"] = self.node_ws
        corrs["weight"] = 1.0
        corrs["valid"] = 1
        return corrs

    def problem(self, t, init_transforms):
        return Problem(nodes=self.nodes, canon=self.canon, corrs=self.frame(t), init_transforms=init_transforms,
                       gt_transforms=self.gt_transforms(t), meta=dict(kind="sequence", seed=self.seed, frame=t))


def cylinder_sequence(seed=5, num_nodes=2048, randomize=False, **kw):
    """The learned-initialisation workload: 640x480 two-cylinder model
    (radii 6 and 5 cm, N=2048, M~300k), bending 0-45 deg with period 60
    frames and twisting +-10 deg.  randomize=True draws the motion's phases,
    periods and amplitudes from the seed (training sequences)."""
    base = cylinder_problem(num_nodes=num_nodes, bend_deg=0.0, init_bend_deg=0.0, noise=0.0, seed=seed)
    rng = np.random.default_rng(seed + 7919)
    canon = base.canon
    joint = np.array([0.0, 0.0, 0.14])
    params = dict(bend_amp_deg=45.0, period=60.0, phase=0.0, twist_amp_deg=10.0, twist_period=150.0,
                  twist_phase=0.0)
    if randomize:
        params = dict(bend_amp_deg=float(rng.uniform(30.0, 50.0)), period=float(rng.uniform(45.0, 80.0)),
                      phase=float(rng.uniform(0.0, 80.0)), twist_amp_deg=float(rng.uniform(5.0, 12.0)),
                      twist_period=float(rng.uniform(100.0, 200.0)), twist_phase=float(rng.uniform(0.0, 200.0)))
    params.update(kw)
    return Sequence(
        nodes=base.nodes,
        canon=canon,
        canon_normals=base.corrs["normal"].astype(np.float64),
        on_seg2=canon[:, 0].astype(np.float64) > joint[0],
        node_ids=base.corrs["node_ids"].copy(),
        node_ws=base.corrs["node_ws"].copy(),
        joint=joint,
        seed=seed,
        **params,
    )


# --------------------------------------------------------------------------
# projective correspondence search frames
# --------------------------------------------------------------------------


@dataclass
class CorrFrame:
    """The inputs of one projective correspondence search
    (DynamicFusionPipeline::find_correspondences, include/fusion_app.h:1791-1845):
    the raycast live surface, the observed depth with its normals, the camera
    motion and the canonical voxel hit per pixel with the voxels' node lists.
    Per-pixel arrays are row-major over height x width."""

    width: int
    height: int
    cam: np.ndarray  # float32[4]: fx, fy, cx, cy
    live_vertices: np.ndarray  # float32[H*W, 3], (0,0,0) where the ray missed
    live_normals: np.ndarray  # float32[H*W, 3]
    depth: np.ndarray  # float32[H*W], 0 = no depth
    depth_normals: np.ndarray  # float32[H*W, 3], (0,0,0) = none
    T_cam_world: np.ndarray  # float32[4, 4]
    T_world_cam: np.ndarray  # float32[4, 4]
    hit_voxel_idx: np.ndarray  # int32[H*W], -1 = none
    voxel_knn: np.ndarray  # int32[V, 4]
    voxel_knn_w: np.ndarray  # float32[V, 4]
    pixel_knn: np.ndarray  # int32[H*W, 4]: the voxel lists gathered per pixel
    pixel_knn_w: np.ndarray  # float32[H*W, 4]
    meta: dict = field(default_factory=dict)

    @property
    def num_pixels(self):
        return self.width * self.height


def _rotmat(q):
    x, y, z, w = q
    return np.array(
        [
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
        ]
    )


def _tube_normals(P, axis_pt, axis_dir):
    q = P - axis_pt
    radial = q - (q @ axis_dir)[:, None] * axis_dir
    n = radial / np.maximum(np.linalg.norm(radial, axis=-1, keepdims=True), 1e-300)
    # face the camera at the origin
    return np.where((np.sum(n * P, -1) > 0)[:, None], -n, n)


def corr_frame(
    width=640,
    height=480,
    bend_deg=30.0,
    est_bend_deg=27.0,
    cam_rot_deg=0.6,
    cam_trans=(0.003, -0.002, 0.002),
    noise=0.001,
    hole_frac=0.01,
    voxel_size=0.004,
    num_nodes=None,
    seed=11,
):
    """Two-cylinder frame (radii 6 and 5 cm, the full-frame workload's
    surface) for the correspondence search.  The live maps are the model
    warped by the current estimate (joint bent by `est_bend_deg`) raycast from
    the previous camera, which is the world frame; the depth is the surface at
    `bend_deg` seen from the camera moved by `cam_rot_deg` about a random axis
    and `cam_trans` metres (T_cam_world), with sigma=`noise` depth noise and a
    `hole_frac` share of pixels without depth.  Depth normals are the
    reference's forward differences flipped toward the camera
    (kernels/tsdf_kernels.cu:180-230).  Each live pixel's canonical point (the
    estimate's articulation undone) falls in a voxel of a `voxel_size` grid;
    the voxels hit carry their 4 nearest nodes with weights
    exp(-d^2 / (2 r^2)) normalised (src/warp_field.cu:379-404).  Intrinsics
    scale with width from fx = fy = 570.342 at 640 x 480."""
    rng = np.random.default_rng(seed)
    s = width / 640.0
    fx = fy = 570.342 * s
    cx, cy = width / 2.0, height / 2.0
    radii, lengths = (0.06, 0.05), (0.08, 0.09)
    joint = np.array([0.0, 0.0, 0.14])
    ex = np.array([1.0, 0.0, 0.0])
    q_est = _rot_y(np.deg2rad(est_bend_deg))
    q_true = _rot_y(np.deg2rad(bend_deg))

    u, v = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    dirs = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u)], -1).reshape(-1, 3)

    # live maps: the estimate raycast from the previous camera (= world)
    w2 = _qrotate(q_est, ex)
    t1, _ = _ray_tube(dirs, joint, ex, radii[0], -lengths[0], 0.0)
    t2, _ = _ray_tube(dirs, joint, w2, radii[1], 0.0, lengths[1])
    seg2 = t2 < t1
    t = np.minimum(t1, t2)
    hit = np.isfinite(t)
    P = dirs * np.where(hit, t, 0.0)[:, None]
    n1 = _tube_normals(P, joint, ex)
    n2 = _tube_normals(P, joint, w2)
    live_n = np.where(seg2[:, None], n2, n1) * hit[:, None]

    # the observed frame: the true surface from the moved camera
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    R = _rotmat(quat_from_rotvec(axis * np.deg2rad(cam_rot_deg)))
    tc = np.asarray(cam_trans, np.float64)
    T_cw = np.eye(4)
    T_cw[:3, :3] = R
    T_cw[:3, 3] = tc
    T_wc = np.eye(4)
    T_wc[:3, :3] = R.T
    T_wc[:3, 3] = -R.T @ tc
    jc = R @ joint + tc
    t1c, _ = _ray_tube(dirs, jc, R @ ex, radii[0], -lengths[0], 0.0)
    t2c, _ = _ray_tube(dirs, jc, R @ _qrotate(q_true, ex), radii[1], 0.0, lengths[1])
    tcam = np.minimum(t1c, t2c)
    dhit = np.isfinite(tcam)
    depth = np.where(dhit, tcam + rng.normal(scale=noise, size=tcam.shape), 0.0)
    depth[rng.random(depth.shape) < hole_frac] = 0.0
    depth = depth.astype(np.float32)

    # forward-difference depth normals (kernels/tsdf_kernels.cu:180-230)
    D = depth.reshape(height, width).astype(np.float64)
    Pc = dirs.reshape(height, width, 3) * D[..., None]
    dn = np.zeros((height, width, 3))
    dxv = Pc[:-1, 1:] - Pc[:-1, :-1]
    dyv = Pc[1:, :-1] - Pc[:-1, :-1]
    nn = np.cross(dxv, dyv)
    nrm = np.linalg.norm(nn, axis=-1, keepdims=True)
    nn = -np.where(nrm > 1e-9, nn / np.maximum(nrm, 1e-300), nn)
    ok = (D[:-1, :-1] > 0) & (D[:-1, 1:] > 0) & (D[1:, :-1] > 0)
    dn[:-1, :-1] = np.where(ok[..., None], nn, 0.0)

    # canonical voxel per live pixel and the voxels' node lists
    canon = P.copy()
    if np.any(seg2 & hit):
        m = seg2 & hit
        canon[m] = joint + _qrotate(np.broadcast_to(_qconj(q_est), (int(m.sum()), 4)), P[m] - joint)
    ch = canon[hit]
    lo = ch.min(0) - 2 * voxel_size
    dims = np.ceil((ch.max(0) - lo) / voxel_size).astype(np.int64) + 3
    ijk = np.floor((canon - lo) / voxel_size).astype(np.int64)
    vidx = (ijk[:, 2] * dims[1] + ijk[:, 1]) * dims[0] + ijk[:, 0]
    hit_voxel = np.where(hit, vidx, -1).astype(np.int32)
    V = int(np.prod(dims))
    if num_nodes is None:
        num_nodes = max(16, int(round(2048 * s * s)))
    num_nodes = min(num_nodes, max(4, ch.shape[0] // 4))
    sel, h = _blue_noise_subsample(ch, num_nodes, rng)
    node_pos = ch[sel]
    used = np.unique(hit_voxel[hit])
    centers = lo + (np.stack([used % dims[0], (used // dims[0]) % dims[1], used // (dims[0] * dims[1])], -1) + 0.5) * voxel_size
    ids, ws = _skin_weights(centers, node_pos, h)
    voxel_knn = np.full((V, K_NEIGHBORS), -1, np.int32)
    voxel_knn_w = np.zeros((V, K_NEIGHBORS), np.float32)
    voxel_knn[used] = ids
    voxel_knn_w[used] = ws
    pk = np.where(hit[:, None], voxel_knn[np.maximum(hit_voxel, 0)], -1).astype(np.int32)
    pw = np.where(hit[:, None], voxel_knn_w[np.maximum(hit_voxel, 0)], 0.0).astype(np.float32)

    return CorrFrame(
        width=width,
        height=height,
        cam=np.array([fx, fy, cx, cy], np.float32),
        live_vertices=P.astype(np.float32),
        live_normals=live_n.astype(np.float32),
        depth=depth.reshape(-1),
        depth_normals=dn.reshape(-1, 3).astype(np.float32),
        T_cam_world=T_cw.astype(np.float32),
        T_world_cam=T_wc.astype(np.float32),
        hit_voxel_idx=hit_voxel,
        voxel_knn=voxel_knn,
        voxel_knn_w=voxel_knn_w,
        pixel_knn=pk,
        pixel_knn_w=pw,
        meta=dict(kind="cylinders-corr", seed=seed, width=width, height=height, live_coverage=float(hit.mean()),
                  depth_coverage=float((depth > 0).mean()), num_voxels=V, num_nodes=int(node_pos.shape[0]),
                  bend_deg=bend_deg, est_bend_deg=est_bend_deg),
    )


@dataclass
class MeshFrame:
    """The inputs of one live-surface prediction
    (DynamicFusionPipeline::rasterize_deformed_mesh_live_surface,
    include/fusion_app.h:1216-1318): the canonical mesh, its warp (analytic
    and by the deformation graph), the camera and the canonical voxel grid
    with the voxels' node lists."""

    width: int
    height: int
    cam: np.ndarray  # float32[4]: fx, fy, cx, cy
    canonical: np.ndarray  # float32[V, 3]
    warped: np.ndarray  # float32[V, 3]: the articulated mesh (exact warp)
    triangles: np.ndarray  # int32[T, 3]
    T_cam_world: np.ndarray  # float32[4, 4]
    grid_origin: np.ndarray  # float32[3]
    voxel_size: float
    dims: np.ndarray  # int32[3]
    voxel_knn: np.ndarray  # int32[V_grid, 4]
    voxel_knn_w: np.ndarray  # float32[V_grid, 4]
    nodes: np.ndarray  # NODE_DTYPE[N]
    transforms: np.ndarray  # DQ_DTYPE[N]: the articulation as centred node DQs
    meta: dict = field(default_factory=dict)


def _tube_mesh(joint, radius, s0, s1, n_theta, n_axial):
    th = np.linspace(0.0, 2 * np.pi, n_theta, endpoint=False)
    s = np.linspace(s0, s1, n_axial + 1)
    S, TH = np.meshgrid(s, th, indexing="ij")
    v = np.stack([joint[0] + S, joint[1] + radius * np.cos(TH), joint[2] + radius * np.sin(TH)], -1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(n_axial), np.arange(n_theta), indexing="ij")
    a = i * n_theta + j
    b = i * n_theta + (j + 1) % n_theta
    c = (i + 1) * n_theta + j
    d = (i + 1) * n_theta + (j + 1) % n_theta
    tri = np.concatenate([np.stack([a, c, b], -1).reshape(-1, 3), np.stack([b, c, d], -1).reshape(-1, 3)])
    return v, tri


def mesh_frame(width=640, height=480, n_theta=256, n_axial=160, bend_deg=30.0, cam_rot_deg=0.6,
               cam_trans=(0.003, -0.002, 0.002), voxel_size=0.004, num_nodes=None, seed=13):
    """The two-cylinder surface (radii 6 and 5 cm, lengths 8 and 9 cm, joint
    at z = 0.14 m) as a triangle mesh: two tubes of n_theta x n_axial quads
    each, 4 * n_theta * n_axial triangles in all.  `warped` bends the second
    tube by `bend_deg` about the joint; the deformation graph (nodes sampled
    from the canonical vertices, 4-NN voxel lists as in
    src/warp_field.cu:379-404) carries the same articulation as centred node
    DQs.  Intrinsics scale with width from fx = fy = 570.342 at 640 x 480."""
    rng = np.random.default_rng(seed)
    s = width / 640.0
    fx = fy = 570.342 * s
    cx, cy = width / 2.0, height / 2.0
    joint = np.array([0.0, 0.0, 0.14])
    v1, t1 = _tube_mesh(joint, 0.06, -0.08, 0.0, n_theta, n_axial)
    v2, t2 = _tube_mesh(joint, 0.05, 0.0, 0.09, n_theta, n_axial)
    canon = np.concatenate([v1, v2])
    tris = np.concatenate([t1, t2 + v1.shape[0]]).astype(np.int32)
    on2 = np.zeros(canon.shape[0], bool)
    on2[v1.shape[0]:] = True
    q = _rot_y(np.deg2rad(bend_deg))
    warped = canon.copy()
    warped[on2] = joint + _qrotate(np.broadcast_to(q, (int(on2.sum()), 4)), canon[on2] - joint)

    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    R = _rotmat(quat_from_rotvec(axis * np.deg2rad(cam_rot_deg)))
    T_cw = np.eye(4)
    T_cw[:3, :3] = R
    T_cw[:3, 3] = np.asarray(cam_trans, np.float64)

    lo = (canon.min(0) - 2 * voxel_size).astype(np.float32)
    dims = (np.ceil((canon.max(0) - lo) / voxel_size).astype(np.int64) + 3).astype(np.int32)
    # the vertices' voxels in FP32, as the skinning kernel finds them
    ijk = np.floor((canon.astype(np.float32) - lo) / np.float32(voxel_size)).astype(np.int64)
    vidx = (ijk[:, 2] * dims[1] + ijk[:, 1]) * dims[0] + ijk[:, 0]
    if num_nodes is None:
        num_nodes = 2048
    num_nodes = min(num_nodes, max(4, canon.shape[0] // 4))
    sel, h = _blue_noise_subsample(canon, num_nodes, rng)
    node_pos = canon[sel]
    nb, nw, kc = _graph(node_pos, h)
    nrm = np.zeros_like(node_pos)
    nodes = _make_nodes(node_pos, nrm, h, nb, nw, kc)
    used = np.unique(vidx)
    centers = lo + (np.stack([used % dims[0], (used // dims[0]) % dims[1], used // (dims[0] * dims[1])], -1)
                    + 0.5) * voxel_size
    ids, ws = _skin_weights(centers, node_pos, h)
    G = int(np.prod(dims.astype(np.int64)))
    voxel_knn = np.full((G, K_NEIGHBORS), -1, np.int32)
    voxel_knn_w = np.zeros((G, K_NEIGHBORS), np.float32)
    voxel_knn[used] = ids
    voxel_knn_w[used] = ws
    node_on2 = node_pos[:, 0] > joint[0]
    qn = np.where(node_on2[:, None], np.broadcast_to(q, (len(node_pos), 4)), np.array([0.0, 0.0, 0.0, 1.0]))
    tn = _qrotate(qn, node_pos - joint) + joint - node_pos
    return MeshFrame(
        width=width, height=height, cam=np.array([fx, fy, cx, cy], np.float32),
        canonical=canon.astype(np.float32), warped=warped.astype(np.float32), triangles=tris,
        T_cam_world=T_cw.astype(np.float32), grid_origin=lo.astype(np.float32), voxel_size=float(voxel_size),
        dims=dims, voxel_knn=voxel_knn, voxel_knn_w=voxel_knn_w, nodes=nodes, transforms=centred_dq(qn, tn),
        meta=dict(kind="cylinders-mesh", seed=seed, width=width, height=height, vertices=int(canon.shape[0]),
                  triangles=int(tris.shape[0]), grid_voxels=G, num_nodes=int(node_pos.shape[0]),
                  bend_deg=bend_deg))


@dataclass
class TsdfFrame:
    """The inputs of one warped TSDF integration (TSDFVolume::integrate,
    src/tsdf_volume.cu:23-60, as DynamicFusionPipeline calls it,
    include/fusion_app.h:655-666): the volume's parameters and prior state,
    the depth frame and camera pose, the deformation graph with every voxel's
    node list, and the voxels' optimisation counts."""

    params: dict  # dims, origin, voxel_size, truncation, decay_alpha, max_weight
    width: int
    height: int
    cam: np.ndarray  # float32[4]: fx, fy, cx, cy
    camera_pose: np.ndarray  # float32[4, 4]: camera -> world
    depth: np.ndarray  # float32[H * W], metres; 0 = none
    voxels: np.ndarray  # float32[V, 3]: tsdf, weight, colour bytes
    nodes: np.ndarray  # NODE_DTYPE[N]
    transforms: np.ndarray  # DQ_DTYPE[N]: node-centred
    voxel_knn: np.ndarray  # int32[V, 4]
    voxel_knn_w: np.ndarray  # float32[V, 4]
    counts: np.ndarray  # int32[V]
    meta: dict = field(default_factory=dict)


def tsdf_frame(width=640, height=480, dims=(256, 256, 256), extent=1.536, origin=(-0.768, -0.768, 0.5),
               truncation_voxels=5.0, nodes_xy=(48, 36), knn_band_voxels=None, cam_rot_deg=0.8,
               cam_trans=(0.004, -0.003, 0.002), warp_rot_deg=3.0, warp_trans=0.01, holes=True, invalid_frac=0.0,
               seed=21):
    """A depth frame of a smooth bumpy surface about 1.1 m in front of the
    camera, inside a volume of `dims` voxels spanning `extent` metres along x
    from `origin` (the reference's 256^3 x 6 mm at the defaults).  The camera
    pose is a small rigid motion.  Nodes sit on the surface on a
    nodes_xy lattice of pixels, warped by a smooth field of rotations up to
    warp_rot_deg and translations up to warp_trans; every voxel within
    knn_band_voxels of the surface (all voxels when None) holds its 4 nearest
    nodes weighted as src/warp_field.cu:379-404.  The prior volume holds the
    truncated surface distance with random weights in the band; counts are
    random 0..6 in the band and 0 elsewhere.  invalid_frac of the depth
    pixels are NaN or negative; `holes` zeroes two rectangles."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, np.int32)
    vs = float(np.float32(extent / float(dims[0])))
    trunc = float(np.float32(truncation_voxels * vs))
    s = width / 640.0
    fx = fy = 570.342 * s
    cx, cy = width / 2.0, height / 2.0
    u, v = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    z = 1.1 + 0.12 * np.sin(2 * np.pi * 1.5 * u / width) * np.cos(2 * np.pi * v / height) + 0.06 * (u / width)
    depth = z.copy()
    if holes:
        depth[height // 5: height // 5 + height // 8, width // 6: width // 6 + width // 7] = 0.0
        depth[3 * height // 5: 3 * height // 5 + height // 10, 3 * width // 5: 3 * width // 5 + width // 9] = 0.0
    depth = depth.reshape(-1)
    if invalid_frac > 0:
        bad = rng.random(depth.size) < invalid_frac
        depth[bad] = np.where(rng.random(int(bad.sum())) < 0.5, np.nan, -0.5)
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    pose = np.eye(4)
    pose[:3, :3] = _rotmat(quat_from_rotvec(axis * np.deg2rad(cam_rot_deg)))
    pose[:3, 3] = cam_trans
    # surface points (world) and the nodes on a pixel lattice
    pc = np.stack([z * (u - cx) / fx, z * (v - cy) / fy, z], -1)
    nu, nv = nodes_xy
    iu = np.linspace(0.04 * width, 0.96 * width, nu).astype(int)
    iv = np.linspace(0.04 * height, 0.96 * height, nv).astype(int)
    npc = pc[iv[:, None], iu[None, :]].reshape(-1, 3)
    node_pos = npc @ pose[:3, :3].T + pose[:3, 3]
    spacing = np.median(np.linalg.norm(np.diff(pc[iv[nv // 2], iu], axis=0), axis=-1))
    h = 1.5 * spacing
    nb, nw, kc = _graph(node_pos, h)
    nodes = _make_nodes(node_pos, np.zeros_like(node_pos), h, nb, nw, kc)
    rv = _smooth_field(rng, node_pos, np.deg2rad(warp_rot_deg), 0.5)
    tn = _smooth_field(rng, node_pos, warp_trans, 0.5)
    transforms = centred_dq(quat_from_rotvec(rv), tn)
    # voxel centres (float64; the generator's own), their camera depth and
    # the surface distance along the ray through their pixel
    V = int(np.prod(dims.astype(np.int64)))
    org = np.asarray(origin, np.float64)
    knn = np.full((V, K_NEIGHBORS), -1, np.int32)
    knn_w = np.zeros((V, K_NEIGHBORS), np.float32)
    vox = np.zeros((V, 3), np.float32)
    vox[:, 0] = 1.0
    vox.view(np.uint32)[:, 2] = 0x00808080
    counts = np.zeros(V, np.int32)
    Rcw = pose[:3, :3].T
    tcw = -Rcw @ pose[:3, 3]
    tree = cKDTree(node_pos)
    plane = int(dims[0]) * int(dims[1])
    gx, gy = np.meshgrid(np.arange(dims[0]), np.arange(dims[1]))
    gx, gy = gx.reshape(-1), gy.reshape(-1)
    band = None if knn_band_voxels is None else knn_band_voxels * vs
    for zi in range(int(dims[2])):
        c = np.stack([org[0] + (gx + 0.5) * vs, org[1] + (gy + 0.5) * vs,
                      np.full(gx.shape, org[2] + (zi + 0.5) * vs)], -1)
        p = c @ Rcw.T + tcw
        with np.errstate(divide="ignore", invalid="ignore"):
            pu = np.rint(fx * p[:, 0] / p[:, 2] + cx)
            pv = np.rint(fy * p[:, 1] / p[:, 2] + cy)
        ok = (p[:, 2] > 0) & (pu >= 0) & (pu < width) & (pv >= 0) & (pv < height)
        sdf = np.full(gx.shape, np.inf)
        idx = (np.where(ok, pv, 0) * width + np.where(ok, pu, 0)).astype(np.int64)
        sdf[ok] = z.reshape(-1)[idx[ok]] - p[ok, 2]
        near = np.abs(sdf) < band if band is not None else np.ones(gx.shape, bool)
        sl = slice(zi * plane, (zi + 1) * plane)
        if near.any():
            ids, ws = _skin_weights(c[near], node_pos, h, tree)
            knn[sl][near] = ids
            knn_w[sl][near] = ws
        inb = np.abs(sdf) < 3 * trunc
        if inb.any():
            vt = vox[sl]
            vt[inb, 0] = np.clip(sdf[inb] / trunc, -1.0, 1.0)
            vt[inb, 1] = rng.uniform(0.0, 50.0, int(inb.sum()))
            vox[sl] = vt
            ct = counts[sl]
            ct[inb] = rng.integers(0, 7, int(inb.sum()))
            counts[sl] = ct
    params = dict(dims=dims, origin=np.asarray(origin, np.float32), voxel_size=vs, truncation=trunc,
                  decay_alpha=0.9, max_weight=50.0)
    return TsdfFrame(params=params, width=width, height=height, cam=np.array([fx, fy, cx, cy], np.float32),
                     camera_pose=pose.astype(np.float32), depth=depth.astype(np.float32), voxels=vox, nodes=nodes,
                     transforms=transforms, voxel_knn=knn, voxel_knn_w=knn_w, counts=counts,
                     meta=dict(node_radius=h, band_voxels=int((counts > 0).sum())))


@dataclass
class VoxelKnnFrame:
    """The inputs of WarpField::compute_voxel_knn: a canonical volume (12-byte
    voxel records as float32 (V, 3)), its TSDFVolume::Params fields, and the
    deformation nodes."""

    params: dict
    voxels: np.ndarray
    nodes: np.ndarray
    meta: dict = field(default_factory=dict)


def voxelknn_frame(width=640, height=480, dims=(256, 256, 256), extent=1.536, origin=(-0.768, -0.768, 0.5),
                   truncation_voxels=5.0, nodes_xy=(48, 36), cam_rot_deg=0.8, cam_trans=(0.004, -0.003, 0.002),
                   duplicate_nodes=0, seed=23):
    """The canonical volume as compute_voxel_knn sees it once a frame of the
    smooth bumpy surface of tsdf_frame (about 1.1 m in front of the camera)
    has been integrated: a voxel holds weight > 0 where the integration
    updates it (kernels/tsdf_kernels.cu:85-174: its centre projects to a
    pixel with depth d > 0 and d - z >= -truncation), so the free space in
    front of the surface holds data as well as the band around it; weights
    are random in (0, 50], elsewhere 0.  Nodes sit on the surface on a
    nodes_xy lattice of pixels (radius 1.5 x the lattice spacing);
    `duplicate_nodes` more nodes repeat the positions of random ones (exact
    distance ties, which the reference resolves to the lower index)."""
    rng = np.random.default_rng(seed)
    dims = np.asarray(dims, np.int32)
    vs = float(np.float32(extent / float(dims[0])))
    trunc = float(np.float32(truncation_voxels * vs))
    s = width / 640.0
    fx = fy = 570.342 * s
    cx, cy = width / 2.0, height / 2.0
    u, v = np.meshgrid(np.arange(width, dtype=np.float64), np.arange(height, dtype=np.float64))
    z = 1.1 + 0.12 * np.sin(2 * np.pi * 1.5 * u / width) * np.cos(2 * np.pi * v / height) + 0.06 * (u / width)
    axis = rng.normal(size=3)
    axis /= np.linalg.norm(axis)
    pose = np.eye(4)
    pose[:3, :3] = _rotmat(quat_from_rotvec(axis * np.deg2rad(cam_rot_deg)))
    pose[:3, 3] = cam_trans
    pc = np.stack([z * (u - cx) / fx, z * (v - cy) / fy, z], -1)
    nu, nv = nodes_xy
    iu = np.linspace(0.04 * width, 0.96 * width, nu).astype(int)
    iv = np.linspace(0.04 * height, 0.96 * height, nv).astype(int)
    node_pos = pc[iv[:, None], iu[None, :]].reshape(-1, 3) @ pose[:3, :3].T + pose[:3, 3]
    spacing = np.median(np.linalg.norm(np.diff(pc[iv[nv // 2], iu], axis=0), axis=-1))
    h = 1.5 * spacing
    if duplicate_nodes:
        node_pos = np.concatenate([node_pos, node_pos[rng.integers(0, len(node_pos), duplicate_nodes)]])
    nb, nw, kc = _graph(node_pos, h)
    nodes = _make_nodes(node_pos, np.zeros_like(node_pos), h, nb, nw, kc)
    V = int(np.prod(dims.astype(np.int64)))
    vox = np.zeros((V, 3), np.float32)
    vox[:, 0] = 1.0
    vox.view(np.uint32)[:, 2] = 0x00808080
    org = np.asarray(origin, np.float64)
    Rcw = pose[:3, :3].T
    tcw = -Rcw @ pose[:3, 3]
    plane = int(dims[0]) * int(dims[1])
    gx, gy = np.meshgrid(np.arange(dims[0]), np.arange(dims[1]))
    gx, gy = gx.reshape(-1), gy.reshape(-1)
    zf = z.reshape(-1)
    for zi in range(int(dims[2])):
        c = np.stack([org[0] + (gx + 0.5) * vs, org[1] + (gy + 0.5) * vs,
                      np.full(gx.shape, org[2] + (zi + 0.5) * vs)], -1)
        p = c @ Rcw.T + tcw
        with np.errstate(divide="ignore", invalid="ignore"):
            pu = np.rint(fx * p[:, 0] / p[:, 2] + cx)
            pv = np.rint(fy * p[:, 1] / p[:, 2] + cy)
        ok = (p[:, 2] > 0) & (pu >= 0) & (pu < width) & (pv >= 0) & (pv < height)
        idx = (np.where(ok, pv, 0) * width + np.where(ok, pu, 0)).astype(np.int64)
        sdf = np.where(ok, zf[idx] - p[:, 2], -np.inf)
        upd = ok & (sdf >= -trunc)
        if upd.any():
            sl = vox[zi * plane:(zi + 1) * plane]
            sl[upd, 0] = np.minimum(1.0, sdf[upd] / trunc)
            sl[upd, 1] = rng.uniform(0.0, 50.0, int(upd.sum())) + np.float32(1e-3)
    params = dict(dims=dims, origin=np.asarray(origin, np.float32), voxel_size=vs)
    return VoxelKnnFrame(params=params, voxels=vox, nodes=nodes,
                         meta=dict(active=int((vox[:, 1] > 0).sum()), node_radius=h, nodes=len(nodes)))
