"""The C-ABI library on a CPU-only host: it loads, exports every entry point
that include/gs_capi.h declares, its struct layouts match the Python mirror,
and calls that need a device fail with a status instead of crashing."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu

HEADER = os.path.join(ROOT, "include", "gs_capi.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gs_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["gs_sim_create", "gs_sim_step", "gs_sim_stats", "gs_sim_set_field", "gs_sim_get_field",
                 "gs_sim_destroy", "gs_last_error", "gs_params_default"]:
        assert must in names


def test_library_exports_every_declared_symbol(gb):
    L = gb.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match(gb):
    L = gb.lib()
    assert L.gs_sizeof_params() == C.sizeof(gb.GsParams)
    assert L.gs_sizeof_stats() == C.sizeof(gb.GsStats)
    assert L.gs_version() == 1


def test_defaults_reference_values(gb):
    p = gb.default_params(gb.GS_MODEL_MART, gb.GS_MODE_REFCOMPAT)
    # src/dynamics_mart.cu:20-27,40,80
    assert (p.dt, p.transition_temperature, p.weight_gradient, p.weight_elastic) == (0.01, 450.0, 2.5, 1e5)
    assert (p.lpc[2], p.lpc[3]) == (32.05, 37.5)
    C4 = p.get_cijkl()
    assert (C4[0, 0, 0, 0], C4[0, 0, 1, 1], C4[0, 1, 0, 1]) == (3.5, 1.5, 1.0)
    q = gb.default_params(gb.GS_MODEL_PRECIPITATE, gb.GS_MODE_REFCOMPAT)
    # src/dynamics_precipitate.cu:21-28
    assert [q.coef[i] for i in range(1, 8)] == [54.0, -17.0, 7.0, 2.5, 0.2, 0.2, 0.2]
    assert (q.kappa_eta, q.kappa_c, q.mobility_c, q.mobility_eta, q.xi, q.c1, q.c2) == (
        300.0, 300.0, 0.4, 0.4, 400.0, 0.1, 0.44)
    s = gb.default_params(gb.GS_MODEL_STRESS, gb.GS_MODE_REFCOMPAT)
    assert s.xi == 4000.0 and s.get_cijkl()[2, 2, 2, 2] == 5.22


def test_host_only_defaults_equal_the_library_defaults(gb):
    """The benchmark's CPU arm fills the headline parameters in Python so that
    it never maps libgsb200.so; the bytes must equal the library's."""
    for n, noise, dt in ((256, 1e-3, gb.GS_DTYPE_F32), (32, 0.0, gb.GS_DTYPE_F64)):
        a = gb.mart3d_params(n, dtype=dt, noise=noise)
        b = gb.mart3d_params(n, dtype=dt, noise=noise, host_only=True)
        assert bytes(a) == bytes(b)
    assert bytes(gb._mart_baseline_defaults_host()) == bytes(gb.default_params(gb.GS_MODEL_MART))


def test_bad_model_is_einval(gb):
    p = gb.GsParams()
    assert gb.lib().gs_params_default(C.byref(p), 99, 0) == -10
    assert "unknown model" in gb.last_error()


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_enodev(gb):
    p = gb.mart3d_params(16)
    h = C.c_void_p()
    rc = gb.lib().gs_sim_create(C.byref(p), C.byref(h))
    assert rc == -15 and not h.value
    assert "device" in gb.last_error()


def test_unsupported_grid_rejected_before_device(gb):
    # odd last axis is rejected by geometry checks (ENOTSUP) or by the device probe (ENODEV)
    p = gb.mart3d_params(16)
    p.nz = 15
    h = C.c_void_p()
    rc = gb.lib().gs_sim_create(C.byref(p), C.byref(h))
    assert rc in (-14, -15)


def test_bounds_check_build_exports_every_declared_symbol(gb):
    """libgsb200_bc.so (kernels with index asserts) is a drop-in for the
    normal library: the same entry points, and it says which build it is."""
    import build

    L = C.CDLL(build.LIB_BC)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    L.gs_bounds_check_build.restype = C.c_int
    assert L.gs_bounds_check_build() == 1


def test_normal_build_has_no_index_asserts(gb):
    L = gb.lib()
    if gb.BOUNDS_CHECK_BUILD:
        pytest.skip("this process loaded the bounds-check build")
    assert L.gs_bounds_check_build() == 0
    rec = (C.c_longlong * 6)()
    assert L.gs_bounds_check_read(rec, 0) == gb.GS_ENOTSUP
    assert list(rec) == [0] * 6
    # the unchecked self-test kernel would write beyond cap: refused before any launch
    dummy = (C.c_int * 4)()
    assert L.gs_bounds_selftest(C.cast(dummy, C.c_void_p), 2, 4, None) == gb.GS_ENOTSUP
    assert "not the bounds-check build" in gb.last_error()
    assert L.gs_bounds_site_name(1) == b"selftest"
    assert L.gs_bounds_site_name(999) == b"unknown"


def test_launch_range_check_switch(gb):
    L = gb.lib()
    was = L.gs_bounds_check_enabled()
    try:
        gb.set_bounds_check(True)
        assert L.gs_bounds_check_enabled() == 1
        gb.set_bounds_check(False)
        assert L.gs_bounds_check_enabled() == 0
    finally:
        gb.set_bounds_check(bool(was))
