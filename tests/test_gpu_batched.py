"""Batched solves (cf_gn_solve_batched): uneven problems solved together must
give each problem the result of its own solve — checked against the FP64
oracle per problem (tolerance: max(1e-5, 1.5x the FP32 oracle's own
deviation) per transform component, 1e-4 relative energy) and against the
single-problem entry point."""
import numpy as np
import pytest
import torch

from cudafusion_b200 import _lib, synth
from cudafusion_b200.solver import DeviceProblem, GaussNewtonSolver, Params
from cudafusion_b200.types import DQ_DTYPE, dq_as_array

pytestmark = pytest.mark.gpu

KW = dict(gn_iterations=4, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=10.0, lambda_damping=1.0)
CLAMPS = (0.12, 0.04)


@pytest.fixture(scope="module")
def batch():
    sizes = [(96, 8000), (256, 20000), (150, 12000), (200, 15000)]
    return [synth.sphere_problem(num_nodes=n, num_corrs=m, node_radius=np.sqrt(4 * np.pi * 0.09 / n), seed=10 + k)
            for k, (n, m) in enumerate(sizes)]


def _solver(batch, mode=0, **kw):
    prm = Params(**{**KW, **kw})
    s = GaussNewtonSolver(prm, max_nodes=sum(p.num_nodes for p in batch), max_corrs=sum(p.num_corrs for p in batch))
    s.set_option(_lib.CF_OPT_PCG_MODE, mode)
    return s


def _run_batched(s, batch):
    dps = [DeviceProblem(p) for p in batch]
    Ts = [d.init_transforms.clone() for d in dps]
    st = s.gn_solve_batched(dps, Ts, *CLAMPS)
    return [dq_as_array(T.cpu().numpy().view(DQ_DTYPE)) for T in Ts], st


# PCG with the system in shared memory (automatic at this size) and streamed
PCG_MODES = [0, 3]


@pytest.mark.parametrize("mode", PCG_MODES)
def test_batched_matches_fp64_oracle(batch, oracle, mode):
    s = _solver(batch, mode)
    Tb, st = _run_batched(s, batch)
    prm = oracle.params(**KW)
    for k, p in enumerate(batch):
        To, Eo, Io = oracle.gn_solve(p, prm, *CLAMPS, precision="f64")
        T32, _, _ = oracle.gn_solve(p, prm, *CLAMPS, precision="f32")
        spread = float(np.abs(dq_as_array(To) - dq_as_array(T32)).max())
        tol = max(1e-5, 1.5 * spread)
        err = float(np.abs(Tb[k] - dq_as_array(To)).max())
        assert err < tol, (k, err, tol)
        assert st[k]["error_flags"] == 0
        assert st[k]["pcg_iterations"] == list(Io)
        for g, e in enumerate(st[k]["energy"]):
            assert abs(e - Eo[g]) / abs(Eo[g]) < 1e-4, (k, g, e, Eo[g])


@pytest.mark.parametrize("mode", PCG_MODES)
def test_batched_matches_single_solves(batch, mode):
    s = _solver(batch, mode)
    Tb, st = _run_batched(s, batch)
    for k, p in enumerate(batch):
        s1 = GaussNewtonSolver(Params(**KW), max_nodes=p.num_nodes, max_corrs=p.num_corrs)
        s1.set_option(_lib.CF_OPT_PCG_MODE, 1)
        d = DeviceProblem(p)
        T = d.init_transforms.clone()
        st1 = s1.gn_solve(d, T, *CLAMPS)
        Ts = dq_as_array(T.cpu().numpy().view(DQ_DTYPE))
        # same algorithm, different CTA split of the PCG dot products
        assert np.abs(Tb[k] - Ts).max() < 2e-5
        assert abs(st[k]["energy_final"] - st1["energy_final"]) / abs(st1["energy_final"]) < 1e-5


@pytest.mark.parametrize("mode", PCG_MODES)
def test_batched_deterministic(batch, mode):
    s = _solver(batch, mode)
    a, _ = _run_batched(s, batch)
    b, _ = _run_batched(s, batch)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("mode", PCG_MODES)
def test_batched_per_problem_tolerance_stop(batch, mode):
    """Each problem's PCG stops on its own ||r|| < tol test."""
    kw = dict(gn_iterations=1, pcg_iterations=60, pcg_tolerance=2e-3, lambda_damping=1e-2, lambda_smooth=1.0)
    s = _solver(batch, mode, **kw)
    _, st = _run_batched(s, batch)
    for k, p in enumerate(batch):
        s1 = GaussNewtonSolver(Params(**{**KW, **kw}), max_nodes=p.num_nodes, max_corrs=p.num_corrs)
        s1.set_option(_lib.CF_OPT_PCG_MODE, 1)
        d = DeviceProblem(p)
        st1 = s1.gn_solve(d, d.init_transforms.clone(), *CLAMPS)
        assert abs(st[k]["pcg_iterations"][0] - st1["pcg_iterations"][0]) <= 1


def test_batched_skips_empty_problem_and_checks_capacity(batch):
    s = _solver(batch)
    empty = synth.Problem(nodes=batch[0].nodes[:0], canon=batch[0].canon[:0], corrs=batch[0].corrs[:0],
                          init_transforms=batch[0].init_transforms[:0])
    dps = [DeviceProblem(batch[0]), DeviceProblem(empty), DeviceProblem(batch[1])]
    Ts = [d.init_transforms.clone() for d in dps[:1]] + [torch.zeros(32, dtype=torch.uint8, device="cuda")] + \
         [dps[2].init_transforms.clone()]
    st = s.gn_solve_batched(dps, Ts, *CLAMPS)
    assert st[1]["energy_final"] == 0.0 and st[0]["energy_final"] > 0 and st[2]["energy_final"] > 0
    small = GaussNewtonSolver(Params(**KW), max_nodes=100, max_corrs=100000)
    with pytest.raises(_lib.CFError):
        small.gn_solve_batched([DeviceProblem(batch[1])], [DeviceProblem(batch[1]).init_transforms.clone()])


def test_autotune_chooses_times_and_remembers(batch):
    """The autotuner times several PCG configurations on the batch, leaves
    the fastest on the handle (results still exact), never writes the
    caller's transforms, and answers the same shape from its cache."""
    s = _solver(batch)
    dps = [DeviceProblem(p) for p in batch]
    Ts = [d.init_transforms.clone() for d in dps]
    r = s.autotune(dps, Ts, *CLAMPS)
    assert r["candidates"] >= 2 and r["from_cache"] == 0
    assert r["ms_best"] <= r["ms_default"]
    assert all(torch.equal(T, d.init_transforms) for T, d in zip(Ts, dps))
    assert s.get_option(_lib.CF_OPT_PCG_MODE) == r["pcg_mode"]
    assert s.get_option(_lib.CF_OPT_PCG_CTAS) == r["pcg_ctas"]
    st = s.gn_solve_batched(dps, Ts, *CLAMPS)
    assert all(x["error_flags"] == 0 for x in st)
    s2 = _solver(batch)
    r2 = s2.autotune(dps, [d.init_transforms.clone() for d in dps], *CLAMPS)
    assert r2["from_cache"] == 1 and r2["pcg_mode"] == r["pcg_mode"] and r2["stream_tile"] == r["stream_tile"]


def test_batched_large_sort_grid(batch):
    """A batch past 2 sort CTAs per SM (one per 4096 correspondences: 1.8M
    correspondences, ~440 sort CTAs), after a small batch on the same handle
    (the sort table grows): each problem still gets its own solve's result."""
    big = [synth.sphere_problem(num_nodes=3000, num_corrs=600000, node_radius=np.sqrt(4 * np.pi * 0.09 / 3000),
                                seed=40 + k) for k in range(3)]
    s = GaussNewtonSolver(Params(**KW), max_nodes=sum(p.num_nodes for p in big),
                          max_corrs=sum(p.num_corrs for p in big))
    _run_batched(s, batch)
    Tb, st = _run_batched(s, big)
    for k, p in enumerate(big):
        s1 = GaussNewtonSolver(Params(**KW), max_nodes=p.num_nodes, max_corrs=p.num_corrs)
        s1.set_option(_lib.CF_OPT_PCG_MODE, 1)
        d = DeviceProblem(p)
        T = d.init_transforms.clone()
        st1 = s1.gn_solve(d, T, *CLAMPS)
        assert st[k]["error_flags"] == 0
        assert np.abs(Tb[k] - dq_as_array(T.cpu().numpy().view(DQ_DTYPE))).max() < 2e-5
        assert abs(st[k]["energy_final"] - st1["energy_final"]) / abs(st1["energy_final"]) < 1e-5
