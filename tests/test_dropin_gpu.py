"""The literal drop-in: the reference's own main.o, parameters.o, ibm.o,
functions.o, input.o, output.o, logs.o and utils.o linked against the B200
solver's C++ entry points (include/wf_dropin.h) instead of the reference's
solver, pde, turbulence and pressure objects (oracle/Makefile target
`dropin`), run on a parameter file and input fields the way the reference's
program is run.

Gates: (1) the fields it saves match the reference's own solver built for the
host (oracle/_ref/ref_host, deterministic) to 1e-12 per field; (2) they are as
close to the reference's GPU program on the same inputs as that host build is
(within 1.5x).  The reference's GPU build is not reproducible run to run on
these grids (two runs of the same binary on the same inputs differ by up to
1e-2 in w after 10 steps), so it cannot be the 1e-12 anchor.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

import ref_runner
from conftest import field_errors

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")
DROPIN = os.path.join(REF, "wildfires_dropin")
REFMAIN = os.path.join(REF, "wildfires_cu_ref")


def _run(binary, case, work):
    from wildfires_b200.configs import write_case
    write_case(case, str(work))
    os.makedirs(os.path.join(str(work), "data", "output"), exist_ok=True)
    r = subprocess.run([binary, "parameters.txt"], cwd=str(work), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    (save,) = glob.glob(os.path.join(str(work), "data", "output", "*", ""))
    return save, r.stdout


def _fields(save, P, n):
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    y = np.empty(P.state_size)
    for q, nm in enumerate("uvwT"):
        y[q * N:(q + 1) * N] = np.fromfile(os.path.join(save, "%s.bin.%d" % (nm, n)))
    y[4 * N:] = np.fromfile(os.path.join(save, "Y.bin.%d" % n))
    return y, np.fromfile(os.path.join(save, "p.bin.%d" % n))


@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFMAIN) and ref_runner.available("host")),
                    reason="reference objects were not available when oracle/Makefile ran")
def test_reference_main_links_and_matches(tmp_path, params_from_text):
    from wildfires_b200 import configs
    case = configs.hill(Nx=33, Ny=33, Nz=16, Nt=10, NT=10, L=100.0, H=20.0, jitter=0.2, seed=3)
    P = params_from_text(configs.param_text(case.params))
    ours, out_ours = _run(DROPIN, case, tmp_path / "dropin")
    ref1, out_ref1 = _run(REFMAIN, case, tmp_path / "reference1")
    ref2, _ = _run(REFMAIN, case, tmp_path / "reference2")
    y_o, p_o = _fields(ours, P, 1)
    host = ref_runner.run(case, "step", flavour="host")
    for f, (linf, l2) in field_errors(P, y_o, host["y"]).items():
        assert linf <= 1e-12 and l2 <= 1e-12, (f, linf, l2)
    assert np.max(np.abs(p_o - host["p"])) <= 1e-12 * np.max(np.abs(host["p"]))
    y1, _ = _fields(ref1, P, 1)
    y2, _ = _fields(ref2, P, 1)
    spread = field_errors(P, y1, y2)
    host_gap = field_errors(P, host["y"], y1)
    for f, (linf, l2) in field_errors(P, y_o, y1).items():
        assert l2 <= 1.5 * host_gap[f][1] + 1e-12, (f, l2, host_gap[f], spread[f])
    # the drop-in reported through the reference's own logging
    log = open(os.path.join(ours, "log.txt")).read()
    assert "Solver time" in log
    # checkpoint report: the restatement reproduces what the reference program
    # printed for its own saved state, and the drop-in (device reduction)
    # prints what the restatement gives for the drop-in's saved state
    assert _report_lines(out_ref1) == _expected_lines(P, y1)
    assert _report_lines(out_ours) == _expected_lines(P, y_o)


def _report_lines(stdout):
    keys = ("CFL:", "Temperature:", "Fuel:")
    return [ln.strip() for ln in stdout.splitlines() if ln.startswith(keys)]


def _expected_lines(P, y):
    import oracle_py as O
    cfl, Y_min, Y_max, T_min, T_max, first = O.timestep_reports(P, y)
    assert first is None
    return ["CFL: %f" % cfl, "Temperature: Min = %.2f, Max = %.2f" % (T_min, T_max),
            "Fuel: Min = %.2f, Max = %.2f" % (Y_min, Y_max)]
