"""Checkpoint path on the GPU: the reference's timestep_reports
(functions.cu:82-185) reduced on the device against its numpy restatement
(exact: maxima, minima and the CFL expression are the same operations), the
first-NaN node in the reference's scan order, and asynchronous double-buffered
dumps against the synchronous writer (byte-identical files)."""
import filecmp
import os

import numpy as np
import pytest

import oracle_py as O
from conftest import load_golden

pytestmark = pytest.mark.gpu


def _solver(P, prec):
    from wildfires_b200 import Solver
    return Solver(P, prec)


def _check(rep, ref):
    cfl, Y_min, Y_max, T_min, T_max, first = ref
    assert rep["cfl"] == cfl and rep["T_min"] == T_min and rep["T_max"] == T_max
    assert rep["Y_min"] == Y_min and rep["Y_max"] == Y_max
    got = None if rep["nan_field"] < 0 else (rep["nan_field"], rep["nan_i"], rep["nan_j"], rep["nan_k"])
    assert got == first


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("narrow", [False, True])
def test_timestep_reports_match_restatement(prec, narrow, params_from_text):
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    r = P.rec
    if narrow:   # a fuel rectangle inside the domain: T and Y ranges only there
        x = np.ctypeslib.as_array(r.x, shape=(r.Nx,))
        y = np.ctypeslib.as_array(r.y, shape=(r.Ny,))
        r.Y0_x_start, r.Y0_x_end = x[3], x[r.Nx // 2]
        r.Y0_y_start, r.Y0_y_end = y[r.Ny // 3], y[r.Ny - 4]
    with _solver(P, prec) as s:
        s.upload(g["y0"], g["p0"])
        for _ in range(3):
            s.step(1)
            yd, _ = s.download()
            _check(s.timestep_reports(), O.timestep_reports(P, yd))


def test_first_nan_in_scan_order(params_from_text):
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    y = np.array(g["y0"], copy=True)

    def at(i, j, k):
        return (i * r.Ny + j) * r.Nz + k
    y[3 * N + at(5, 2, 7)] = np.nan                      # T
    y[1 * N + at(5, 2, 9)] = np.nan                      # v, later in the scan
    y[4 * N + (4 * r.Ny + 12) * r.Nz_Y_max + 0] = np.nan  # Y at (4, 12, 0): first in the scan
    with _solver(P, "fp64") as s:
        s.upload(y, g["p0"])
        rep = s.timestep_reports()
    ref = O.timestep_reports(P, y)
    assert ref[5] == (4, 4, 12, 0)
    _check(rep, ref)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_async_dumps_equal_synchronous_writes(prec, tmp_path, params_from_text):
    from wildfires_b200 import save_fields
    g = load_golden("flat_33x33x16_10")
    P = params_from_text(g["params"])
    a, b = tmp_path / "async", tmp_path / "sync"
    a.mkdir()
    b.mkdir()
    with _solver(P, prec) as s:
        s.upload(g["y0"], g["p0"])
        for n, steps in enumerate([1, 2, 1, 1], start=1):   # four dumps: two wait for a free buffer
            s.step(steps)
            s.dump_async(a, n)
            y, p = s.download()
            save_fields(P, b, n, y, p)
        s.dump_wait()
    names = sorted(os.listdir(b))
    assert len(names) == 24 and sorted(os.listdir(a)) == names
    for nm in names:
        assert filecmp.cmp(a / nm, b / nm, shallow=False), nm


def test_dump_write_error_is_reported(tmp_path, params_from_text):
    from wildfires_b200 import WfError
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    with _solver(P, "fp64") as s:
        s.upload(g["y0"], g["p0"])
        s.dump_async(tmp_path / "missing" / "dir", 1)
        with pytest.raises(WfError):
            s.dump_wait()
        s.dump_async(tmp_path, 2)       # the error was consumed; the next dump works
        s.dump_wait()
    assert (tmp_path / "u.bin.2").exists()
