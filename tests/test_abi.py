"""The C-ABI library builds, loads and exports exactly what
include/cudafusion_b200.h declares; struct layouts match the reference's
(include/types.h).  No compute calls: these run without a GPU."""
import ctypes
import os
import re

import numpy as np

from cudafusion_b200.types import CORR_DTYPE, DQ_DTYPE, NODE_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cudafusion_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^CF_API\s+[^;(]*?\b(cf_[a-z0-9_]+)\s*\(", src, flags=re.M)))


def test_header_lists_match(cflib):
    from cudafusion_b200 import _lib

    decl = declared_functions()
    assert decl, "no declarations parsed"
    assert sorted(_lib.EXPORTS) == decl


def test_library_exports_every_symbol(cflib):
    out = os.popen(f"nm -D --defined-only {cflib._name}").read()
    exported = set(re.findall(r" T (cf_[a-z0-9_]+)", out))
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(cflib, name)


def test_struct_sizes_match_reference(oracle):
    sizes = (ctypes.c_int * 4)()
    oracle.lib().cfo_struct_sizes(sizes)
    assert list(sizes)[:3] == [32, 96, 76]
    assert DQ_DTYPE.itemsize == 32 and NODE_DTYPE.itemsize == 96 and CORR_DTYPE.itemsize == 76
    assert CORR_DTYPE.fields["valid"][1] == 72
    assert NODE_DTYPE.fields["num_neighbors"][1] == 92


def test_params_defaults(cflib):
    from cudafusion_b200 import _lib

    p = _lib.GNParams()
    assert cflib.cf_gn_params_default(ctypes.byref(p)) == 0
    assert (p.gn_iterations, p.pcg_iterations) == (3, 10)
    assert np.isclose(p.pcg_tolerance, 1e-4) and np.isclose(p.lambda_damping, 1e-2)
    assert p.lambda_smooth == 1.0 and p.lambda_rot == 1.0 and p.debug == 0


def test_argument_errors_without_device(cflib):
    """Invalid arguments return status codes (never exit like CUDA_CHECK)."""
    from cudafusion_b200 import _lib

    assert cflib.cf_gn_params_default(None) == _lib.CF_ERR_INVALID_ARG
    assert cflib.cf_gn_create(None, 10, 10, None) == _lib.CF_ERR_INVALID_ARG
    p = _lib.GNParams()
    cflib.cf_gn_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    assert cflib.cf_gn_create(ctypes.byref(p), -1, 10, ctypes.byref(h)) == _lib.CF_ERR_INVALID_ARG
    assert cflib.cf_gn_destroy(None) == _lib.CF_ERR_INVALID_ARG
    assert cflib.cf_warp_apply_twist(None, None, -1, 0.0, 0.0, 1.0, None) == _lib.CF_ERR_INVALID_ARG
    assert cflib.cf_warp_apply_twist(None, None, 0, 0.0, 0.0, 1.0, None) == 0
    assert cflib.cf_status_string(_lib.CF_ERR_TIMEOUT).decode().startswith("in-kernel barrier")


def test_create_reports_missing_device(cflib):
    import torch

    from cudafusion_b200 import _lib

    if torch.cuda.is_available():
        return
    p = _lib.GNParams()
    cflib.cf_gn_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    assert cflib.cf_gn_create(ctypes.byref(p), 16, 16, ctypes.byref(h)) == _lib.CF_ERR_NO_DEVICE
    assert not h.value


def test_library_is_sm100a(cflib):
    """The library carries sm_100a device code (cuobjdump lists only the
    ELF targets; nothing is disassembled)."""
    out = os.popen(f"cuobjdump --list-elf {cflib._name} 2>/dev/null").read()
    assert "sm_100a" in out


def test_pipeline_argument_errors_without_device(cflib):
    """The pipeline entry points check their arguments before any CUDA call:
    null handles and outputs, negative sizes and sizes past the handles'
    index range return status codes; empty work succeeds."""
    from cudafusion_b200 import _lib

    bad, cap = _lib.CF_ERR_INVALID_ARG, _lib.CF_ERR_CAPACITY
    h = ctypes.c_void_p()
    # handles
    assert cflib.cf_raster_create(64, 48, None) == bad
    assert cflib.cf_raster_create(0, 48, ctypes.byref(h)) == bad and not h.value
    assert cflib.cf_raster_create(1 << 16, 1 << 16, ctypes.byref(h)) == cap and not h.value
    assert cflib.cf_corr_search_create(64, 48, None) == bad
    assert cflib.cf_corr_search_create(64, -1, ctypes.byref(h)) == bad and not h.value
    assert cflib.cf_corr_search_create(1 << 15, 1 << 15, ctypes.byref(h)) == cap and not h.value
    # calls on a null handle
    assert cflib.cf_find_correspondences(*([None] * 10)) == bad
    assert cflib.cf_predict_live_surface(None, None, None, None, 0, 0, None, None, 0, None, None, None, None, None,
                                         None, None, None, None) == bad
    ls = [None] * 32
    for k in (5, 6, 10, 23):
        ls[k] = 0
    ls[22] = 0.0
    assert cflib.cf_line_search(*ls) == bad
    # the update's statistics, scaled increment and RMSE
    lp = _lib.LineSearchParams()
    stats = _lib.UpdateStats()
    assert cflib.cf_validate_update(None, -1, ctypes.byref(lp), ctypes.byref(stats), None) == bad
    assert cflib.cf_validate_update(None, 4, ctypes.byref(lp), ctypes.byref(stats), None) == bad
    assert cflib.cf_scale_delta(None, -1, 0.1, 0.1, 1.0, None, None) == bad
    assert cflib.cf_scale_delta(None, 0, 0.1, 0.1, 1.0, None, None) == 0
    assert cflib.cf_scale_delta(None, 8, 0.1, 0.1, 1.0, None, None) == bad
    assert cflib.cf_correspondence_rmse(None, -1, None, None, None) == bad
    assert cflib.cf_correspondence_rmse(None, 10, None, None, None) == bad
    # the volume's integration and kNN field without a volume description
    assert cflib.cf_tsdf_integrate(None, None, None, None, None, None, None, 0, None, None, None, 0, None,
                                   None) == bad
    assert cflib.cf_compute_voxel_knn(None, None, None, 0, None, None, None) == bad
