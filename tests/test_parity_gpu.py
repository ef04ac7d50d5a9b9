"""GPU path against the reference outputs (golden fixtures from the
reference's own solver sources) and against the CPU oracle.

Tolerances: the FP64 path must match within 1e-10 per-field relative L2 and
L-infinity (relative to the field's largest magnitude) after the stated step
count; single operators are held to 1e-11.  The FP32 stencil path is held to
1e-5 relative L2 per field against the FP64 reference.
"""
import numpy as np
import pytest

import oracle_py as O
from conftest import field_errors, golden_names, load_golden

pytestmark = pytest.mark.gpu
NAMES = golden_names()


def _solver(P, prec="fp64"):
    from wildfires_b200 import Solver
    return Solver(P, prec)


def _assert_fields(P, a, b, tol, what):
    errs = field_errors(P, a, b)
    bad = {f: e for f, e in errs.items() if e[0] > tol or e[1] > tol}
    assert not bad, "%s: %s" % (what, bad)


@pytest.mark.parametrize("name", NAMES)
def test_phi_fp64_matches_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    with _solver(P) as s:
        R = s.phi(g["y0"])
    _assert_fields(P, R, g["phi"], 1e-11, "phi")


@pytest.mark.parametrize("name", NAMES)
def test_pressure_fp64_matches_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    with _solver(P) as s:
        p, _ = s.pressure(g["y0"], g["y0"], g["p0"])
    scale = np.max(np.abs(g["pressure"]))
    assert np.max(np.abs(p - g["pressure"])) <= 1e-11 * scale
    assert np.linalg.norm(p - g["pressure"]) <= 1e-11 * np.linalg.norm(g["pressure"])


@pytest.mark.parametrize("name", NAMES)
def test_steps_fp64_match_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    with _solver(P) as s:
        s.upload(g["y0"], g["p0"])
        s.step(int(g["nsteps"]))
        y, p = s.download()
    _assert_fields(P, y, g["steps_y"], 1e-10, "state after %d steps" % int(g["nsteps"]))
    assert np.max(np.abs(p - g["steps_p"])) <= 1e-10 * np.max(np.abs(g["steps_p"]))


@pytest.mark.parametrize("name", NAMES)
def test_steps_fp32_close_to_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    with _solver(P, "fp32") as s:
        s.upload(g["y0"], g["p0"])
        s.step(int(g["nsteps"]))
        y, p = s.download()
    errs = field_errors(P, y, g["steps_y"])
    for f, (linf, l2) in errs.items():
        assert l2 <= 1e-5, (f, linf, l2)


def test_graph_replay_is_deterministic(params_from_text):
    g = load_golden("flat_33x33x16_10")
    P = params_from_text(g["params"])
    outs = []
    for _ in range(2):
        with _solver(P) as s:
            s.upload(g["y0"], g["p0"])
            s.step(4)
            outs.append(s.download())
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_steps_one_at_a_time_equal_batched(params_from_text):
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    with _solver(P) as s:
        s.upload(g["y0"], g["p0"])
        for _ in range(3):
            s.step(1)
        a = s.download()
    with _solver(P) as s:
        s.upload(g["y0"], g["p0"])
        s.step(3)
        b = s.download()
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def _numpy_integrals(P, y):
    """Mass, energy and fuel of a packed state: sums over the periodic cell set
    (duplicate planes i = Nx-1, j = Ny-1 left out) with the node volume
    dx dy (z_{k+1} - z_{k-1}) / 2 (one-sided at the walls); mass and energy
    over the cells at or above the cut node, fuel over the stored fuel cells
    k < Nz_Y(i, j)."""
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    z = P.z()
    zl = np.concatenate([[z[0]], z[:-1]])
    zh = np.concatenate([z[1:], [z[-1]]])
    dV = r.dx * r.dy * 0.5 * (zh - zl)
    T3 = y[3 * N:4 * N].reshape(r.Nx, r.Ny, r.Nz)[:-1, :-1, :]
    cut = P.cut_nodes()[:-1, :-1, None]
    above = np.arange(r.Nz)[None, None, :] >= cut
    rho = r.T_inf * r.rho_inf / T3
    mass = np.sum(np.where(above, rho * dV[None, None, :], 0.0))
    energy = np.sum(np.where(above, rho * r.c_p * T3 * dV[None, None, :], 0.0))
    NzY = r.Nz_Y_max
    Y3 = y[4 * N:].reshape(r.Nx, r.Ny, NzY)[:-1, :-1, :]
    stored = np.arange(NzY)[None, None, :] < P.nz_y()[:-1, :-1, None]
    fuel = np.sum(np.where(stored, Y3 * dV[None, None, :NzY], 0.0))
    return mass, energy, fuel


def test_diagnostics_match_numpy(params_from_text):
    """Every FP64 diagnostic against a numpy restatement: extrema and NaN count
    exactly, mass, energy and fuel to 1e-12 of their size (the summation
    order differs), and the fuel consumed over three steps to 1e-12 of the
    initial fuel."""
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    y0 = g["y0"]
    with _solver(P) as s:
        s.upload(y0, g["p0"])
        d0 = s.diagnostics()
        s.step(3)
        d3 = s.diagnostics()
        y3, _ = s.download()
    u, v, w, T = (y0[q * N:(q + 1) * N] for q in range(4))
    assert d0["max_abs_u"] == np.max(np.abs(u)) and d0["max_abs_v"] == np.max(np.abs(v))
    assert d0["max_abs_w"] == np.max(np.abs(w))
    assert d0["T_min"] == np.min(T) and d0["T_max"] == np.max(T)
    stored = (np.arange(r.Nz_Y_max)[None, None, :] < P.nz_y()[:, :, None]).reshape(-1)
    assert d0["Y_min"] == np.min(y0[4 * N:][stored]) and d0["Y_max"] == np.max(y0[4 * N:][stored])
    z = P.z()
    cfl = r.dt * (np.max(np.abs(u)) / r.dx + np.max(np.abs(v)) / r.dy + np.max(np.abs(w)) / r.dz)
    assert abs(d0["cfl"] - cfl) <= 1e-14 * cfl
    for d, y in ((d0, y0), (d3, y3)):
        mass, energy, fuel = _numpy_integrals(P, y)
        assert abs(d["mass"] - mass) <= 1e-12 * mass
        assert abs(d["energy"] - energy) <= 1e-12 * energy
        assert abs(d["fuel"] - fuel) <= 1e-12 * fuel
        assert d["nan_count"] == 0
    fuel0 = _numpy_integrals(P, y0)[2]
    fuel3 = _numpy_integrals(P, y3)[2]
    assert fuel0 - fuel3 > 0, "the ignition consumes fuel within three steps"
    assert abs(d0["fuel_consumed"]) <= 1e-13 * fuel0
    assert abs(d3["fuel_consumed"] - (fuel0 - fuel3)) <= 1e-12 * fuel0
    assert z.size == r.Nz


def test_full_size_flat_one_step_matches_oracle():
    """The 128 x 128 x 64 flat workload, one FP64 step against the oracle."""
    from wildfires_b200 import configs
    case = configs.flat()
    import tempfile
    import os
    from wildfires_b200 import read_parameters
    with tempfile.TemporaryDirectory() as d:
        ppath = os.path.join(d, "parameters.txt")
        with open(ppath, "w") as f:
            f.write(configs.param_text(case.params))
        P = read_parameters(ppath)
        y0, p0 = case.fields(P)
        yo, po = O.steps(P, y0, p0, 1)
        with _solver(P) as s:
            s.upload(y0, p0)
            s.step(1)
            y, p = s.download()
        _assert_fields(P, y, yo, 1e-11, "full-size flat step")
        assert np.max(np.abs(p - po)) <= 1e-10 * max(np.max(np.abs(po)), 1e-30)


@pytest.mark.parametrize("nx,ny", [(512, 9), (9, 512), (96, 160), (192, 256), (128, 65), (33, 17),
                                   (1025, 5), (5, 1001), (1701, 5), (5, 2049), (4, 7)])
def test_pressure_fft_lengths_match_oracle(nx, ny, params_from_text):
    """Transform lengths Nx-1, Ny-1 of every workload (511, 95, 159, 191, 255,
    127, 64, 32, 16) and the extremes of the FFT engine (1024 direct, 1000 and
    1700 by Bluestein with inner lengths 2048 and 4096, 2048 direct, 3 and 6)
    through the pressure solve, against the oracle."""
    from wildfires_b200 import configs
    case = configs.flat(Nx=nx, Ny=ny, Nz=8, Nt=1, jitter=0.3, seed=nx + ny)
    P = params_from_text(configs.param_text(case.params))
    y0, p0 = case.fields(P)
    po, _ = O.pressure(P, y0, y0, p0)
    with _solver(P) as s:
        p, _ = s.pressure(y0, y0, p0)
    scale = np.max(np.abs(po))
    assert np.max(np.abs(p - po)) <= 1e-11 * scale


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_async_upload_steps_like_the_blocking_one(prec, params_from_text):
    """wf_upload_state_async (p's copy overlapping the RK stages) followed by
    steps and a download gives the same bits as wf_upload_state, also when the
    host buffer of p is overwritten right after the download and uploaded
    again (the step must have waited for the first copy)."""
    import ctypes as C
    from wildfires_b200 import configs
    from wildfires_b200._abi import check, lib
    case = configs.hill(Nx=65, Ny=65, Nz=32, Nt=4, L=120.0, H=20.0, jitter=0.1, seed=3)
    P = params_from_text(configs.param_text(case.params))
    y0, p0 = case.fields(P)
    import torch
    dp = C.POINTER(C.c_double)
    out = {}
    for name in ("wf_upload_state", "wf_upload_state_async"):
        with _solver(P, prec) as s:
            # pinned host buffers: the copies are truly asynchronous
            y = torch.empty(len(y0), dtype=torch.float64, pin_memory=True).numpy()
            p = torch.empty(len(p0), dtype=torch.float64, pin_memory=True).numpy()
            y[:] = y0
            p[:] = p0
            for _ in range(2):
                check(getattr(lib(), name)(s._h, y.ctypes.data_as(dp), p.ctypes.data_as(dp)), name)
                s.step(2)
                check(lib().wf_download_state(s._h, y.ctypes.data_as(dp), p.ctypes.data_as(dp)), "download")
            out[name] = (y.copy(), p.copy())
    assert np.array_equal(out["wf_upload_state"][0], out["wf_upload_state_async"][0])
    assert np.array_equal(out["wf_upload_state"][1], out["wf_upload_state_async"][1])


@pytest.mark.parametrize("nx,ny", [(512, 128), (192, 96), (256, 160)])
def test_rader_and_bluestein_engines_agree(nx, ny, params_from_text, monkeypatch):
    """The prime-factor + Rader transforms (511 = 7 x 73, 127 and 191 with a
    three-factor inner transform, 255, 159, 95) against the same lengths by
    Bluestein (WF_FFT_RADER=0) through the pressure solve: the two engines
    round differently, so they agree to rounding, not bit for bit."""
    from wildfires_b200 import configs
    case = configs.flat(Nx=nx, Ny=ny, Nz=8, Nt=1, jitter=0.3, seed=nx * ny)
    P = params_from_text(configs.param_text(case.params))
    y0, p0 = case.fields(P)
    with _solver(P) as s:
        p_pr, _ = s.pressure(y0, y0, p0)
    monkeypatch.setenv("WF_FFT_RADER", "0")
    with _solver(P) as s:
        p_bl, _ = s.pressure(y0, y0, p0)
    scale = np.max(np.abs(p_bl))
    assert np.max(np.abs(p_pr - p_bl)) <= 1e-12 * scale


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", 1e-5)])
def test_tallest_column_one_step_matches_oracle(prec, tol, params_from_text):
    """The longest tridiagonal system wf_create accepts (Nz - 1 = 511) and the
    widest projection block (512 threads): one step of a 9 x 9 x 512 flat case
    against the oracle."""
    from wildfires_b200 import configs
    case = configs.flat(Nx=9, Ny=9, Nz=512, Nt=1, jitter=0.2, seed=5)
    P = params_from_text(configs.param_text(case.params))
    y0, p0 = case.fields(P)
    yo, po = O.steps(P, y0, p0, 1)
    with _solver(P, prec) as s:
        s.upload(y0, p0)
        s.step(1)
        y, p = s.download()
    _assert_fields(P, y, yo, tol, "9x9x512 step (%s)" % prec)
