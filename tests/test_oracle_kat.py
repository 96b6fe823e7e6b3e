"""Pins the CPU oracle to the reference: its FP32 se3 functions must
reproduce, bit for bit, the known-answer vectors produced by the reference's
own host-compiled functions (tests/golden/make_golden.py), and its FP64
instantiation must agree with them to FP32 rounding."""
import os

import numpy as np
import pytest

from cudafusion_b200.types import DQ_DTYPE, NODE_DTYPE

GOLD = os.path.join(os.path.dirname(__file__), "golden", "se3_kat.npz")


@pytest.fixture(scope="module")
def kat():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def dq(a):
    return np.ascontiguousarray(a).view(DQ_DTYPE)


def bits(x):
    return np.ascontiguousarray(x).view(np.uint32)


def test_exp_se3_bitwise(oracle, kat):
    out = np.stack([oracle.exp_se3(t).ravel() for t in kat["tw"]])
    assert np.array_equal(bits(out), bits(kat["exp_out"]))


def test_mat4_to_dq_bitwise(oracle, kat):
    got = np.array([oracle.mat4_to_dq(m) for m in kat["exp_out"]], DQ_DTYPE)
    assert np.array_equal(bits(got), bits(dq(kat["m2dq_out"])))
    got2 = np.array([oracle.mat4_to_dq(m) for m in kat["mats"]], DQ_DTYPE)
    assert np.array_equal(bits(got2), bits(dq(kat["mats_dq"])))


def test_dq_mul_centered_transform_bitwise(oracle, kat):
    a, b = dq(kat["a"]), dq(kat["b"])
    mul = np.array([oracle.dq_mul(a[i], b[i]) for i in range(len(a))], DQ_DTYPE)
    assert np.array_equal(bits(mul), bits(dq(kat["mul_out"])))
    cen = np.array([oracle.dq_centered(a[i], kat["ctr"][i]) for i in range(len(a))], DQ_DTYPE)
    assert np.array_equal(bits(cen), bits(dq(kat["cent_out"])))
    tp = np.stack([oracle.dq_transform_point(a[i], kat["pts"][i]) for i in range(len(a))])
    assert np.array_equal(bits(tp), bits(kat["tp_out"]))
    tpc = np.stack([oracle.dq_transform_point_centered(a[i], kat["pts"][i], kat["ctr"][i]) for i in range(len(a))])
    assert np.array_equal(bits(tpc), bits(kat["tpc_out"]))


def test_skinning_bitwise(oracle, kat):
    nodes = np.ascontiguousarray(kat["skin_nodes"]).view(NODE_DTYPE)
    T = dq(kat["skin_T"])
    out = oracle.skin(kat["skin_canon"], kat["skin_ids"], kat["skin_ws"], nodes, T, precision="f32")
    assert np.array_equal(bits(out), bits(kat["skin_out"]))


def test_f64_agrees_with_reference(oracle, kat):
    out = np.stack([oracle.exp_se3(t, precision="f64").ravel() for t in kat["tw"]])
    assert np.allclose(out, kat["exp_out"], rtol=2e-6, atol=2e-6)
    nodes = np.ascontiguousarray(kat["skin_nodes"]).view(NODE_DTYPE)
    out = oracle.skin(kat["skin_canon"], kat["skin_ids"], kat["skin_ws"], nodes, dq(kat["skin_T"]), precision="f64")
    assert np.allclose(out, kat["skin_out"], atol=2e-6)


@pytest.mark.skipif(
    not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libcfref_host.so")),
    reason="reference host build (oracle/_ref) not present",
)
def test_live_reference_random(oracle):
    """Fresh random cases against the live reference build, when present."""
    import ctypes

    ref = ctypes.CDLL(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "libcfref_host.so"))
    rng = np.random.default_rng(99)
    for _ in range(300):
        tw = (rng.normal(size=6) * rng.choice([1e-7, 1e-3, 0.2, 2.0])).astype(np.float32)
        r = np.zeros(1, DQ_DTYPE)
        ref.ref_dq_from_twist(tw.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p))
        T = oracle.exp_se3(tw)
        o = oracle.mat4_to_dq(T)
        assert np.array_equal(bits(np.array([o], DQ_DTYPE)), bits(r))


def test_mpnn_oracle_gradient_matches_finite_differences():
    """The FP64 network oracle's analytic gradient (the checker of the BF16
    kernels) against central differences of its own loss."""
    import mpnn_oracle as O

    rng = np.random.default_rng(0)
    N = 40
    nbr = rng.integers(-1, N, size=(N, 8))
    x = rng.normal(size=(N, O.IN))
    tgt = rng.normal(size=(N, O.OUT))
    th = rng.normal(size=O.PARAMS) * 0.2
    _, g = O.loss_and_grad(th, x, tgt, nbr, rounding=False)
    idx = rng.choice(O.PARAMS, 40, replace=False)
    fd = O.finite_differences(th, x, tgt, nbr, idx)
    assert np.abs(fd - g[idx]).max() < 1e-6 * max(1.0, np.abs(g[idx]).max())


def test_mpnn_oracle_bf16_rounding():
    import mpnn_oracle as O

    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-3])
    r = O.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even
    assert r[2] == 1.0078125
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8)
