"""The variable-density pressure fixed point (reference pressure.cu:551-606),
which runs on the device as a CUDA graph WHILE node, against the oracle's
loop: the same number of solves, the same pressure (1e-11 of its largest
magnitude) and the same reported change and iteration index.  The tolerance
of each case is placed between two consecutive changes of the oracle's own
iteration, a factor of at least 4 apart, so the stopping iteration does not
hinge on rounding."""
import re

import numpy as np
import pytest

import oracle_py as O
from conftest import field_errors, load_golden

pytestmark = pytest.mark.gpu


def _text(tol, maxit):
    t = str(load_golden("vardens_rk4")["params"])
    t = re.sub(r"(?m)^pressure_solver_tol = .*$", "pressure_solver_tol = %r" % float(tol), t)
    return re.sub(r"(?m)^pressure_solver_iter = .*$", "pressure_solver_iter = %d" % int(maxit), t)


def _solver(P):
    from wildfires_b200 import Solver
    return Solver(P, "fp64")


def _changes(params_from_text, y, p0, n):
    """Max-norm change of oracle iterations 1..n (tolerance off)."""
    out = []
    for m in range(1, n + 1):
        _, it, e = O.pressure_full(params_from_text(_text(-1.0, m)), y, y, p0)
        assert it == m
        out.append(e)
    return out


def _stop_tolerance(ch, first=2):
    for k in range(first, len(ch)):
        if ch[k] > 0 and ch[k - 1] >= 4 * ch[k]:
            return np.sqrt(ch[k - 1] * ch[k]), k + 1   # the loop ends after k+1 solves
    pytest.skip("no clear drop in the oracle's changes")


def test_tolerance_stops_at_the_oracle_iteration(params_from_text):
    g = load_golden("vardens_rk4")
    y, p0 = g["y0"], g["p0"]
    ch = _changes(params_from_text, y, p0, 8)
    tol, solves = _stop_tolerance(ch)
    P = params_from_text(_text(tol, 50))
    po, ito, eo = O.pressure_full(P, y, y, p0)
    assert ito == solves
    with _solver(P) as s:
        for _ in range(2):   # the second call replays the cached loop graph
            p, it = s.pressure(y, y, p0)
            err, ref_iter = s.pressure_report()
            assert it == ito and ref_iter == ito - 1
            scale = np.max(np.abs(po))
            assert np.max(np.abs(p - po)) <= 1e-11 * scale
            assert abs(err - eo) <= 1e-11 * scale and err <= tol


def test_iteration_cap_without_convergence(params_from_text):
    g = load_golden("vardens_rk4")
    y, p0 = g["y0"], g["p0"]
    ch = _changes(params_from_text, y, p0, 3)
    P = params_from_text(_text(ch[2] / 100.0, 3))     # not met within 3 solves
    po, ito, eo = O.pressure_full(P, y, y, p0)
    assert ito == 3
    with _solver(P) as s:
        p, it = s.pressure(y, y, p0)
        err, ref_iter = s.pressure_report()
    assert it == 3 and ref_iter == 3
    scale = np.max(np.abs(po))
    assert np.max(np.abs(p - po)) <= 1e-11 * scale and abs(err - eo) <= 1e-11 * scale


def test_steps_with_tolerance_match_oracle(params_from_text):
    """Full steps: the loop runs inside the replayed step graph."""
    g = load_golden("vardens_rk4")
    y0, p0 = g["y0"], g["p0"]
    ch = _changes(params_from_text, y0, p0, 8)
    tol, _ = _stop_tolerance(ch)
    P = params_from_text(_text(tol, 50))
    n = int(g["nsteps"])
    yo, po = O.steps(P, y0, p0, n)
    with _solver(P) as s:
        s.upload(y0, p0)
        s.step(n)
        y, p = s.download()
        err, ref_iter = s.pressure_report()
    bad = {f: e for f, e in field_errors(P, y, yo).items() if e[0] > 1e-10 or e[1] > 1e-10}
    assert not bad, bad
    assert np.max(np.abs(p - po)) <= 1e-10 * np.max(np.abs(po))
    assert 0 <= ref_iter < 50 and err <= tol
