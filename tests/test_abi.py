"""Host-side checks of the C-ABI library that need no GPU: symbols, parser
rules, field-file round trip, error statuses."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available


def test_library_exports_every_declared_symbol():
    from wildfires_b200 import _abi
    L = _abi.lib()
    header = open(os.path.join(ROOT, "include", "wildfires_b200.h")).read()
    header = re.sub(r"/\*.*?\*/", "", header, flags=re.S)
    declared = set(re.findall(r"\b(wf_[a-z_]+)\s*\([^()]*\)\s*;", header))
    assert declared == set(_abi.EXPORTS), declared ^ set(_abi.EXPORTS)
    for name in declared:
        assert hasattr(L, name), name


def test_dropin_archive_defines_every_declared_entry_point():
    """include/wf_dropin.h: the reference's C++ entry points, with the
    reference's parameter types, defined by libwildfires_b200_dropin.a."""
    import subprocess
    header = open(os.path.join(ROOT, "include", "wf_dropin.h")).read()
    header = re.sub(r"/\*.*?\*/", "", header, flags=re.S)
    declared = set(re.findall(r"^void\s+(\w+)\s*\(", header, flags=re.M))
    assert declared == {"create_y_0", "solve_PDE", "Phi", "euler", "RK2", "RK4", "solve_pressure",
                        "solve_pressure_iterative"}
    archive = os.path.join(ROOT, "wildfires_b200", "libwildfires_b200_dropin.a")
    out = subprocess.run(["nm", "-C", "--defined-only", archive], capture_output=True, text=True, check=True).stdout
    defined = {m.group(1): m.group(2) for m in re.finditer(r" T (\w+)\(([^)]*)\)", out)}
    for name in declared:
        assert name in defined, name
        assert "_parameters" in defined[name], (name, defined[name])   # takes the record by value
    assert defined["solve_PDE"] == "double*, double*, _parameters"


def test_parser_defaults_and_override(params_from_text):
    P = params_from_text("Nx = 8\nNy = 9\nNz = 10\nNt = 4\nx_max = 7\ny_max = 8\nz_max = 9\nt_max = 1\n"
                         "C_s = 0.1\nC_s = 0.3\nunknown_key = 5\nT_min = 290\nmethod = RK2\n")
    r = P.rec
    assert (r.Nx, r.Ny, r.Nz, r.Nt) == (8, 9, 10, 4)
    assert r.C_s == 0.3                   # later lines override earlier ones
    assert r.T_min == 290.0
    assert r.mu == 1.802e-5 and r.T_act == 18040.8533 and r.variable_density == 1   # defaults
    assert r.method == b"RK2"
    assert r.dx == 1.0 and r.dt == 0.25
    assert r.NT == 4                      # missing save interval -> Nt
    assert r.field_indexes.T == 3 * 8 * 9 * 10


def test_parser_missing_file_is_an_error(tmp_path):
    from wildfires_b200 import WfError, read_parameters
    with pytest.raises(WfError) as e:
        read_parameters(tmp_path / "nope.txt")
    assert e.value.status == 3


def test_wavenumbers_and_hill_tables(params_from_text):
    P = params_from_text("Nx = 12\nNy = 10\nNz = 8\nNt = 1\nx_max = 22\ny_max = 18\nz_max = 7\nt_max = 1\n"
                         "topo_shape = hill\nhill_center_x = 11\nhill_center_y = 9\nhill_length = 4\n"
                         "hill_width = 4\nhill_height = 3\nY_h = 0.5\n")
    r = P.rec
    kx = np.ctypeslib.as_array(r.kx, shape=(11,))
    expect = 2 * np.pi * np.fft.fftfreq(11, 1.0 / 11) / 22.0
    np.testing.assert_allclose(kx, expect, rtol=0, atol=1e-15)
    cut = P.cut_nodes()
    assert cut.max() == 2 and cut.min() == 0      # peak 3 exp(-1/8) = 2.65 m
    assert r.Nz_Y_max == 4


def test_field_files_round_trip(tmp_path, params_from_text):
    from wildfires_b200 import _abi, load_fields
    P = params_from_text("Nx = 5\nNy = 6\nNz = 7\nNt = 1\nx_max = 4\ny_max = 5\nz_max = 6\nt_max = 1\nY_h = 1.5\n")
    S, N = P.state_size, 5 * 6 * 7
    y = np.arange(S, dtype=np.float64)
    p = -np.arange(N, dtype=np.float64)
    d = str(tmp_path) + "/"
    dp = C.POINTER(C.c_double)
    _abi.check(_abi.lib().wf_save_fields(C.byref(P.rec), d.encode(), 3, y.ctypes.data_as(dp), p.ctypes.data_as(dp)), "save")
    for nm in "uvwTYp":
        os.rename(os.path.join(d, nm + ".bin.3"), os.path.join(d, nm + ".bin"))
    y2, p2 = load_fields(P, d)
    assert np.array_equal(y, y2) and np.array_equal(p, p2)
    os.truncate(os.path.join(d, "T.bin"), 8 * 10)
    with pytest.raises(Exception):
        load_fields(P, d)


@pytest.mark.skipif(gpu_available(), reason="checks the error path without a device")
def test_create_without_device_reports_no_device(params_from_text):
    from wildfires_b200 import Solver, WfError
    P = params_from_text("Nx = 8\nNy = 8\nNz = 8\nNt = 1\nx_max = 7\ny_max = 7\nz_max = 7\nt_max = 1\n")
    with pytest.raises(WfError) as e:
        Solver(P)
    assert e.value.status in (2, 7)


@pytest.mark.parametrize("text,expect", [
    ("Nx = 8\nNy = 8\nNz = 513\n", "Nz-1 must be <= 511"),        # longest tridiagonal system
    ("Nx = 2050\nNy = 5\nNz = 8\n", "Nx-1 and Ny-1 must be <= 2048"),  # longest transform
    ("Nx = 5\nNy = 2050\nNz = 8\n", "Nx-1 and Ny-1 must be <= 2048"),
    ("Nx = 8\nNy = 8\nNz = 4\n", "too small"),   # the parser takes Nz = 4, the solver needs 5
])
def test_create_rejects_grids_beyond_the_engine_limits(text, expect, params_from_text):
    """Argument checks come before any device call, so they hold on any host."""
    from wildfires_b200 import Solver, WfError
    P = params_from_text(text + "Nt = 1\nx_max = 7\ny_max = 7\nz_max = 7\nt_max = 1\n")
    with pytest.raises(WfError) as e:
        Solver(P)
    assert e.value.status == 1 and expect in str(e.value), str(e.value)


def test_parser_rejects_grids_below_four_nodes(params_from_text):
    from wildfires_b200 import WfError
    with pytest.raises(WfError) as e:
        params_from_text("Nx = 3\nNy = 8\nNz = 8\nNt = 1\nx_max = 7\ny_max = 7\nz_max = 7\nt_max = 1\n")
    assert e.value.status == 4 and "Nx, Ny, Nz >= 4" in str(e.value), str(e.value)


def test_create_rejects_unknown_precision_and_high_terrain(params_from_text):
    from wildfires_b200 import Solver, WfError, _abi
    P = params_from_text("Nx = 8\nNy = 8\nNz = 8\nNt = 1\nx_max = 7\ny_max = 7\nz_max = 7\nt_max = 1\n")
    h = C.c_void_p()
    assert _abi.lib().wf_create(C.byref(P.rec), 7, C.byref(h)) == 1 and not h.value
    assert b"unknown precision" in _abi.lib().wf_last_error()
    # a column whose terrain reaches the top planes leaves no room for the boundary rules
    topo = np.zeros((8, 8))
    topo[3, 4] = 6.5
    P.set_topography(topo)
    with pytest.raises(WfError) as e:
        Solver(P)
    assert e.value.status == 1 and "above Nz-4" in str(e.value), str(e.value)


def test_every_entry_point_rejects_null_arguments():
    """Null handles and buffers give WF_ERR_ARG (or the documented neutral
    value) before any device call: no entry point dereferences them."""
    from wildfires_b200 import _abi
    L = _abi.lib()
    ARG = _abi.WF_ERR_ARG
    calls = {
        "wf_read_parameters": ((None, None), ARG),
        "wf_set_topography": ((None, None), ARG),
        "wf_state_size": ((None,), 0),
        "wf_load_fields": ((None, None, None, None), ARG),
        "wf_save_fields": ((None, None, 0, None, None), ARG),
        "wf_create": ((None, 0, None), ARG),
        "wf_destroy": ((None,), 0),
        "wf_upload_state": ((None, None, None), ARG),
        "wf_upload_state_async": ((None, None, None), ARG),
        "wf_download_state": ((None, None, None), ARG),
        "wf_step": ((None, 1), ARG),
        "wf_synchronize": ((None,), ARG),
        "wf_time": ((None, None, None), ARG),
        "wf_diagnostics": ((None, None), ARG),
        "wf_device_state": ((None, None, None), ARG),
        "wf_stream": ((None,), None),
        "wf_phi": ((None, None, None), ARG),
        "wf_pressure": ((None, None, None, None, None), ARG),
        "wf_launches_per_step": ((None,), 0),
        "wf_profile_phases": ((None, 1, None, None), ARG),
        "wf_pressure_noalloc": ((None, None, None, None), ARG),
        "wf_rk": ((None, None, None), ARG),
        "wf_ensemble_create": ((None, 0, 0, None), ARG),
        "wf_ensemble_destroy": ((None,), 0),
        "wf_ensemble_size": ((None,), 0),
        "wf_ensemble_member": ((None, 0), None),
        "wf_ensemble_step": ((None, 1), ARG),
        "wf_ensemble_synchronize": ((None,), ARG),
        "wf_set_closure": ((None, 0, None), ARG),
        "wf_closure_coefficients": ((None, None, None), ARG),
        "wf_mlp_loss_grad": ((None, None, None, 0, None, None), ARG),
        "wf_mlp_train": ((None, None, None, 0, 0, 0, 0.0, 0, None), ARG),
        "wf_pressure_report": ((None, None, None), ARG),
        "wf_timestep_reports": ((None, None), ARG),
        "wf_dump_async": ((None, None, 0), ARG),
        "wf_dump_wait": ((None,), ARG),
        "wf_save_domain": ((None, None), ARG),
        "wf_save_topography": ((None, None), ARG),
        "wf_initial_conditions": ((None,), ARG),
        "wf_stage_tile": ((None, None, None, None), ARG),
        "wf_set_stage_tile": ((None, 8, 16, 0), ARG),
        "wf_set_stream": ((None, None), ARG),
        "wf_phi_device": ((None, None, None), ARG),
        "wf_rk_device": ((None, None, None), ARG),
        "wf_pressure_device": ((None, None, None, None), ARG),
        "wf_closure_predict": ((None, None, 0, None), ARG),
        "wf_set_closure_wait_limit": ((None, 0), ARG),
        "wf_ibm_parameters_device": ((None,), ARG),
        "wf_set_topography_hills": ((None, 0, None), ARG),
        "wf_ensemble_stream": ((None,), None),
    }
    for name, (args, expect) in calls.items():
        assert getattr(L, name)(*args) == expect, name
    L.wf_free_parameters(None)
    assert L.wf_phase_name(-1) is None and L.wf_phase_name(_abi.WF_NPHASES) is None
    assert L.wf_phase_name(0) is not None and L.wf_status_string(ARG)
    # every declared entry point that takes a pointer is in the table above
    takes_pointer = {n for n in _abi.EXPORTS if n not in ("wf_status_string", "wf_last_error", "wf_phase_name",
                                                          "wf_closure_param_count", "wf_free_parameters",
                                                          "wf_inject_allocation_failure")}
    assert takes_pointer == set(calls), takes_pointer ^ set(calls)


@pytest.mark.parametrize("extra, grid, message", [
    ("variable_density = 1\n", (16, 16, 16), "variable_density"),
    ("variable_density = 0\n", (2050, 8, 16), "Nx-1, Ny-1 must be <="),
    ("variable_density = 0\n", (8, 2050, 16), "Nx-1, Ny-1 must be <="),
    ("variable_density = 0\n", (8, 8, 600), "Nz-1 <="),
    ("variable_density = 0\n", (512, 512, 64), "MiB of scratch"),
])
def test_noalloc_pressure_rejects_before_any_cuda_call(params_from_text, extra, grid, message):
    """wf_pressure_noalloc checks the density mode, the transform and tridiagonal
    limits and the size of its fixed array on the host, before it touches a
    device: the buffers passed here are not device memory and are never read."""
    from wildfires_b200 import _abi
    L = _abi.lib()
    Nx, Ny, Nz = grid
    P = params_from_text("Nx = %d\nNy = %d\nNz = %d\nNt = 1\nx_max = 10\ny_max = 10\nz_max = 5\nt_max = 1\n%s"
                         % (Nx, Ny, Nz, extra))
    st = L.wf_pressure_noalloc(C.byref(P.rec), C.c_void_p(16), C.c_void_p(16), None)
    assert st == _abi.WF_ERR_ARG
    assert message in L.wf_last_error().decode()
