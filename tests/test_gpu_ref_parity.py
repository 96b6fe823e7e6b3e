"""Parity against the reference's own CUDA solver: CUDAFusion's
GaussNewtonSolver::solve (kernels/solver_kernels.cu:543-614, PCG :616-687)
and WarpField::apply_twist_increment (src/warp_field.cu:1121-1141), built
unmodified for sm_100a with the reference's --use_fast_math
(oracle/_ref/libcfref_cuda.so) and run on the same GPU, on the same inputs.

The reference is not deterministic: its assembly adds with float atomics
(solver_kernels.cu:52-138, 202-352), so two of its runs differ.  Each case
therefore runs it REF_RUNS times and measures:
  spread   how far its runs land from each other (max over runs of the
           distance from its first run),
  dev      how far its runs land from the FP64 oracle's answer.

Bars (the contract: node transforms within 1e-5 per component, energies within
1e-4 relative; increments within 1e-4 relative to their largest entry):
  * the block pattern is the reference's bit for bit; A and b agree with
    every reference run to 1e-5 relative to their largest entry;
  * ours is at least as accurate as the reference: its distance from the
    FP64 answer is within max(contract, the reference's dev);
  * ours agrees with every reference run within max(contract, 1.5 x (spread
    + dev)): two FP32 solvers that each land within their rounding floor of
    the answer differ by at most the sum of those floors;
  * where the reference reproduces itself within the contract (damping 1.0),
    ours agrees with every reference run within the contract itself.

The full-frame solve at solver.h defaults (lambda_smooth 1, damping 1e-2, the
reference's ARAP Jacobian sign) is indefinite after skin pairs are dropped by
find_block (solver_kernels.cu:25-44), so its later GN iterations are chaotic
in both implementations; there the test holds the first linearisation to the
bars above and the full solve to the reference's own run-to-run cloud.
"""
import numpy as np
import pytest
import torch

import oracle as O
import ref_solver as R
from cudafusion_b200 import synth
from cudafusion_b200.solver import DeviceProblem, GaussNewtonSolver, Params, to_device
from cudafusion_b200.types import DQ_DTYPE, dq_as_array

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref/libcfref_cuda.so was not built "
                                 "(make -C oracle ref needs the CUDAFusion sources)")]

REF_RUNS = 10
T_TOL = 1e-5        # per node-transform component
E_TOL = 1e-4        # relative energy
DX_TOL = 1e-4       # increment, relative to its largest entry
SYS_TOL = 1e-5      # A and b, relative to their largest entry
MAX_ROT, MAX_TRANS = 0.12, 0.04
THREADS = 16


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def tdist(a, b):
    return float(np.abs(dq_as_array(a) - dq_as_array(b)).max())


@pytest.fixture(scope="module")
def p1():
    return synth.config1()


@pytest.fixture(scope="module")
def p2():
    return synth.config2()


def ours_linearize(p, kw):
    s = GaussNewtonSolver(Params(**kw), max_nodes=max(p.num_nodes, 256), max_corrs=p.num_corrs)
    dx = s.solve(to_device(p.corrs), p.num_corrs, to_device(p.nodes), to_device(p.init_transforms), p.num_nodes)
    torch.cuda.synchronize()
    row_ptr, col_idx, vals, rhs = s.system()
    s.close()
    return dx.cpu().numpy()[: 6 * p.num_nodes], row_ptr, col_idx, vals.reshape(-1, 36), rhs


def ours_gn(p, kw):
    s = GaussNewtonSolver(Params(**kw), max_nodes=max(p.num_nodes, 256), max_corrs=p.num_corrs)
    dp = DeviceProblem(p)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T, max_rot=MAX_ROT, max_trans=MAX_TRANS)
    s.close()
    assert st["error_flags"] == 0
    return T.cpu().numpy().view(DQ_DTYPE).copy(), st


def ref_linearizations(p, kw, runs=REF_RUNS):
    ref = R.RefSolver(p, **kw)
    out = []
    for _ in range(runs):
        ref.upload(p.init_transforms)
        dx = ref.linearize_solve()
        row_ptr, col_idx, vals, rhs = ref.system()
        out.append((dx, row_ptr, col_idx, vals, rhs))
    ref.close()
    return out


def ref_gn_runs(p, kw, runs=REF_RUNS):
    ref = R.RefSolver(p, **kw)
    Ts = [ref.gn_solve(kw["gn_iterations"], MAX_ROT, MAX_TRANS, 1.0) for _ in range(runs)]
    ref.close()
    return Ts


def check_floor(name, ours_vs_ref, ours_vs_f64, spread, dev, contract, reproducible=False):
    """The three bars of the module docstring for one quantity."""
    msg = (f"{name}: ours-ref {max(ours_vs_ref):.3g}, ours-f64 {ours_vs_f64:.3g}, "
           f"reference spread {spread:.3g}, reference-f64 {dev:.3g}")
    print(msg)
    assert ours_vs_f64 <= max(contract, dev), msg
    assert max(ours_vs_ref) <= max(contract, 1.5 * (spread + dev)), msg
    if reproducible:
        assert spread <= contract, msg
        assert max(ours_vs_ref) <= contract, msg


# (lambda_smooth, lambda_damping, reproducible): the reference's own damping
# 1.0 (config/params.yaml:29) gives a well-conditioned system; the solver.h
# default 1e-2 leaves config 1 barely positive definite (lambda_min ~7e-5),
# where the reference's runs differ from each other by more than 1e-5
CASES = [(10.0, 1.0, True), (10.0, 1e-2, False), (1.0, 1e-2, False)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"lambda{c[0]:g}-damping{c[1]:g}")
def test_linearization_matches_reference_solver(p1, case):
    """One GaussNewtonSolver::solve on the sphere (N=256, M=20k, 10 PCG):
    pattern, A, b and delta_x against the reference's system_matrix(),
    rhs() and delta_x."""
    lam, damp, reproducible = case
    kw = dict(gn_iterations=1, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=lam, lambda_damping=damp)
    dx, row_ptr, col_idx, vals, rhs = ours_linearize(p1, kw)
    refs = ref_linearizations(p1, kw)
    for _, rrp, rci, rvals, rrhs in refs:
        assert np.array_equal(row_ptr, rrp) and np.array_equal(col_idx, rci)
        assert rel(vals, rvals) < SYS_TOL
        assert rel(rhs, rrhs) < SYS_TOL
    dx64, it, *_ = O.linearize_solve(p1.corrs, p1.nodes, p1.init_transforms, O.params(**kw), nthreads=THREADS)
    assert it == 10
    spread = max(rel(r[0], refs[0][0]) for r in refs)
    dev = max(rel(r[0], dx64) for r in refs)
    check_floor("delta_x", [rel(dx, r[0]) for r in refs], rel(dx, dx64), spread, dev, DX_TOL,
                reproducible=reproducible)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"lambda{c[0]:g}-damping{c[1]:g}")
def test_gn_solve_matches_reference_solver(p1, case):
    """Five full GN iterations (re-skin, solve, apply_twist_increment with
    the 0.12 / 0.04 clamps) on the sphere: node transforms and the FP64
    energy at the final transforms against the reference's."""
    lam, damp, reproducible = case
    kw = dict(gn_iterations=5, pcg_iterations=10, pcg_tolerance=0.0, lambda_smooth=lam, lambda_damping=damp)
    T, st = ours_gn(p1, kw)
    Trefs = ref_gn_runs(p1, kw)
    T64, E64, _ = O.gn_solve(p1, O.params(**kw), MAX_ROT, MAX_TRANS, precision="f64", nthreads=THREADS)
    spread = max(tdist(t, Trefs[0]) for t in Trefs)
    dev = max(tdist(t, T64) for t in Trefs)
    check_floor("transforms", [tdist(T, t) for t in Trefs], tdist(T, T64), spread, dev, T_TOL,
                reproducible=reproducible)
    e_ours = O.energy(p1, T, lam, nthreads=THREADS)
    for t in Trefs:
        e_ref = O.energy(p1, t, lam, nthreads=THREADS)
        assert abs(e_ours - e_ref) / abs(e_ref) < E_TOL, (e_ours, e_ref)
    # the solver's own FP64 energy at its final transforms is the oracle's
    assert abs(st["energy_final"] - e_ours) / abs(e_ours) < 1e-6


def test_pcg_tolerance_stop_matches_reference(p1):
    """The reference's default absolute tolerance (1e-4, include/solver.h:17)
    with the early stop of solver_kernels.cu:669: the same solve as the
    reference's within the bars."""
    kw = dict(gn_iterations=5, pcg_iterations=10, pcg_tolerance=1e-4, lambda_smooth=10.0, lambda_damping=1.0)
    T, _ = ours_gn(p1, kw)
    Trefs = ref_gn_runs(p1, kw)
    assert max(tdist(T, t) for t in Trefs) < T_TOL


@pytest.mark.parametrize("lam,damp", [(1.0, 1e-2), (10.0, 1.0)], ids=["solver_h_defaults", "lambda10-damping1"])
def test_full_frame_linearization_matches_reference(p2, lam, damp):
    """The 640x480 two-cylinder frame (N=2048, M=304k, 20 PCG): the first
    linearisation's pattern, A, b and delta_x against the reference's and the
    FP64 oracle's, at the solver.h defaults and at lambda 10 / damping 1."""
    kw = dict(gn_iterations=1, pcg_iterations=20, pcg_tolerance=0.0, lambda_smooth=lam, lambda_damping=damp)
    dx, row_ptr, col_idx, vals, rhs = ours_linearize(p2, kw)
    refs = ref_linearizations(p2, kw, runs=4)
    orp, oci = O.build_pattern(p2.nodes)
    A64, b64, _ = O.assemble(p2.corrs, p2.nodes, p2.init_transforms, orp, oci, lam, damp, precision="f64",
                             nthreads=THREADS)
    for _, rrp, rci, rvals, rrhs in refs:
        assert np.array_equal(row_ptr, rrp) and np.array_equal(col_idx, rci)
        assert rel(vals, rvals) < SYS_TOL and rel(rhs, rrhs) < SYS_TOL
        # the reference's own rounding is the larger part of the gap
        assert rel(vals, A64.reshape(-1, 36)) <= rel(rvals, A64.reshape(-1, 36))
    assert rel(vals, A64.reshape(-1, 36)) < 1e-6 and rel(rhs, b64) < 1e-6
    dx64, *_ = O.linearize_solve(p2.corrs, p2.nodes, p2.init_transforms, O.params(**kw), nthreads=THREADS)
    spread = max(rel(r[0], refs[0][0]) for r in refs)
    dev = max(rel(r[0], dx64) for r in refs)
    check_floor("delta_x (full frame)", [rel(dx, r[0]) for r in refs], rel(dx, dx64), spread, dev, DX_TOL)


def test_full_frame_solve_matches_reference_well_posed(p2):
    """The full frame at lambda_smooth 10 and the reference's production
    damping 1.0, 5 GN x 20 PCG: the solve converges (energy 4.36 -> 0.23) and
    lands on the reference's transforms and energy within the contract."""
    kw = dict(gn_iterations=5, pcg_iterations=20, pcg_tolerance=0.0, lambda_smooth=10.0, lambda_damping=1.0)
    T, st = ours_gn(p2, kw)
    Trefs = ref_gn_runs(p2, kw, runs=4)
    assert st["energy_final"] < 0.1 * st["energy_initial"]
    d = [tdist(T, t) for t in Trefs]
    print("full frame, lambda 10 / damping 1: ours-ref", max(d))
    assert max(d) < T_TOL
    e_ours = O.energy(p2, T, 10.0, nthreads=THREADS)
    for t in Trefs:
        e_ref = O.energy(p2, t, 10.0, nthreads=THREADS)
        assert abs(e_ours - e_ref) / abs(e_ref) < E_TOL


def test_full_frame_solve_at_solver_h_defaults_within_reference_cloud(p2):
    """The headline frame at the solver.h defaults (lambda_smooth 1, damping
    1e-2), 5 GN x 20 PCG.  The system is indefinite (dropped skin pairs), so
    both solvers' energies rise over the GN iterations and the reference's
    own runs land far apart (its float atomics change the rounding of every
    run).  Ours must look like one more reference run: its median distance
    to the reference's runs within 1.5x their median distance to each other,
    its energy within the reference's range widened by half that range, and
    the energy rising in both."""
    kw = dict(gn_iterations=5, pcg_iterations=20, pcg_tolerance=1e-4, lambda_smooth=1.0, lambda_damping=1e-2)
    T, st = ours_gn(p2, kw)
    Trefs = ref_gn_runs(p2, kw, runs=10)
    e0 = O.energy(p2, p2.init_transforms, 1.0, nthreads=THREADS)
    e_ours = O.energy(p2, T, 1.0, nthreads=THREADS)
    e_refs = [O.energy(p2, t, 1.0, nthreads=THREADS) for t in Trefs]
    d_ours = float(np.median([tdist(T, t) for t in Trefs]))
    d_ref = float(np.median([tdist(a, b) for i, a in enumerate(Trefs) for b in Trefs[i + 1:]]))
    lo, hi = min(e_refs), max(e_refs)
    print(f"solver.h defaults: energy {e0:.4g} -> ours {e_ours:.4g}, reference {[round(e, 4) for e in e_refs]}; "
          f"transforms: median distance ours-reference {d_ours:.3g}, reference-reference {d_ref:.3g}")
    assert e_ours > e0 and lo > e0
    assert d_ours <= 1.5 * d_ref
    assert lo - 0.5 * (hi - lo) <= e_ours <= hi + 0.5 * (hi - lo)
