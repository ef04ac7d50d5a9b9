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


def test_diagnostics_match_numpy(params_from_text):
    g = load_golden("hill_rk4")
    P = params_from_text(g["params"])
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    y0 = g["y0"]
    with _solver(P) as s:
        s.upload(y0, g["p0"])
        d = s.diagnostics()
    u, v, w, T = (y0[q * N:(q + 1) * N] for q in range(4))
    assert d["max_abs_u"] == np.max(np.abs(u)) and d["max_abs_w"] == np.max(np.abs(w))
    assert d["T_min"] == np.min(T) and d["T_max"] == np.max(T)
    z = P.z()
    zl = np.concatenate([[z[0]], z[:-1]])
    zh = np.concatenate([z[1:], [z[-1]]])
    dV = r.dx * r.dy * 0.5 * (zh - zl)
    T3 = T.reshape(r.Nx, r.Ny, r.Nz)[:-1, :-1, :]
    cut = P.cut_nodes()[:-1, :-1, None]
    above = np.arange(r.Nz)[None, None, :] >= cut
    rho = r.T_inf * r.rho_inf / T3
    mass = np.sum(np.where(above, rho * dV[None, None, :], 0.0))
    assert abs(d["mass"] - mass) <= 1e-12 * mass
    assert d["nan_count"] == 0 and d["cfl"] > 0


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
