"""The C++ drop-in classes (include/cudafusion_b200.hpp) compiled with g++
against reference-layout types and driven the way the reference's pipeline
drives its solver (include/fusion_app.h:386-390, :525-550).

CPU: the header compiles and links against the library, and without a GPU
the constructor throws CF_ERR_NO_DEVICE (no silent fallback).
GPU: the C++ loop gives bit-identical results to the same calls made through
the Python mirror, and the GPU-side loop (solve_frame) matches cf_gn_solve."""
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import ROOT, has_gpu, reference_dir

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_loop.cpp")
LIBDIR = os.path.join(ROOT, "cudafusion_b200")

G, P, LAM, MAX_ROT, MAX_TRANS = 3, 10, 10.0, 0.12, 0.04


@pytest.fixture(scope="module")
def exe(cflib, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("cpp") / "dropin_loop")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), SRC, "-o", out, "-L", LIBDIR, "-lcfb200",
           f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_dropin_compiles_and_fails_loudly_without_gpu(exe):
    r = subprocess.run([exe, "nodev"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "no CUDA device" in r.stdout or "status" in r.stdout


@pytest.mark.gpu
def test_dropin_loop_matches_python_mirror(exe, tmp_path):
    from cudafusion_b200 import synth
    from cudafusion_b200.solver import DeviceProblem, GaussNewtonSolver, Params, WarpField, to_device

    p = synth.config1()
    p.nodes.tofile(tmp_path / "nodes.bin")
    p.corrs.tofile(tmp_path / "corrs.bin")
    np.ascontiguousarray(p.canon, np.float32).tofile(tmp_path / "canon.bin")
    p.init_transforms.tofile(tmp_path / "init.bin")
    r = subprocess.run([exe, str(tmp_path), str(G), str(P), str(LAM), str(MAX_ROT), str(MAX_TRANS)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr

    # the same calls through the Python mirror
    prm = Params(gn_iterations=G, pcg_iterations=P, lambda_smooth=LAM)
    s = GaussNewtonSolver(prm, max_nodes=p.num_nodes, max_corrs=p.num_corrs)
    wf = WarpField(0.025, max_nodes=p.num_nodes)
    wf.upload_nodes(p.nodes)
    wf.upload_transforms(p.init_transforms)
    dc = to_device(p.corrs)
    dx = None
    for g in range(G):
        dx = s.solve(dc, p.num_corrs, wf.device_nodes(), wf.device_transforms(), wf.num_nodes(), dx)
        if g == 0:
            dx0 = dx.cpu().numpy()[: 6 * p.num_nodes].copy()
            _, _, vals, rhs = s.system()
        wf.apply_twist_increment(dx, MAX_ROT, MAX_TRANS)
    loop = wf.download_transforms()

    assert np.array_equal(np.fromfile(tmp_path / "dx0.bin", np.float32), dx0)
    sysv = np.fromfile(tmp_path / "sys.bin", np.float32)
    assert np.array_equal(sysv, np.concatenate([vals.reshape(-1), rhs]))
    assert np.array_equal(np.fromfile(tmp_path / "loop.bin", np.uint8), loop.view(np.uint8))

    dp = DeviceProblem(p)
    T = dp.init_transforms.clone()
    st = s.gn_solve(dp, T, max_rot=MAX_ROT, max_trans=MAX_TRANS)
    torch.cuda.synchronize()
    assert np.array_equal(np.fromfile(tmp_path / "frame.bin", np.uint8), T.cpu().numpy())
    e0, e1 = (float(v) for v in r.stdout.split()[1:3])
    assert e0 == pytest.approx(st["energy_initial"], rel=1e-12)
    assert e1 == pytest.approx(st["energy_final"], rel=1e-12)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_frontend_classes_compile_and_fail_loudly_without_gpu(cflib, tmp_path):
    """CorrespondenceSearch, LiveSurfaceRaster and TSDFIntegrator compile
    against the reference's type layouts (-Wall -Werror) and, with no GPU,
    throw CF_ERR_NO_DEVICE from their constructors."""
    out = str(tmp_path / "dropin_frontend")
    src = os.path.join(ROOT, "tests", "cpp", "dropin_frontend.cpp")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), src, "-o", out, "-L", LIBDIR, "-lcfb200",
           f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([out, "nodev"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr



def _compile_only(src, extra_includes=()):
    cmd = ["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include")]
    for d in extra_includes:
        cmd += ["-I", d]
    return subprocess.run(cmd + [src], capture_output=True, text=True)


@pytest.mark.skipif(reference_dir() is None, reason="the CUDAFusion sources are not on this machine "
                    "(set CF_REFERENCE_DIR)")
def test_layouts_checked_against_reference_headers():
    """Every templated method of the drop-in classes instantiated with the
    reference's own types from its include/types.h and include/tsdf_volume.h:
    the size and per-field offset checks hold for the real definitions."""
    src = os.path.join(ROOT, "tests", "cpp", "dropin_reftypes.cpp")
    r = _compile_only(src, [os.path.join(reference_dir(), "include")])
    assert r.returncode == 0, r.stderr


def test_layout_check_catches_field_order_drift(tmp_path):
    """A Correspondence of the right size with dst and normal swapped must not
    compile: the checks compare field offsets, not only sizes."""
    src = tmp_path / "drift.cpp"
    src.write_text("""
#include "cudafusion_b200.hpp"
struct DualQuat { float4 real; float4 dual; };
struct DeformNode { float3 pos; float3 normal; float radius; int neighbors[8]; float neighbor_w[8];
                    int num_neighbors; };
struct Correspondence { float3 src, normal, dst; int node_ids[4]; float node_ws[4]; float weight; bool valid; };
static_assert(sizeof(Correspondence) == sizeof(cf_correspondence), "same size");
static_assert(cudafusion_b200::layouts_match<DeformNode, DualQuat, Correspondence>(), "drift detected");
""")
    r = _compile_only(str(src))
    assert r.returncode != 0
    assert "drift detected" in r.stderr
    assert "same size" not in r.stderr
