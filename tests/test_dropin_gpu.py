"""The literal drop-in: the reference's own main.o, parameters.o, ibm.o,
functions.o, input.o, output.o, logs.o and utils.o linked against the B200
solver's C++ entry points (include/wf_dropin.h) instead of the reference's
solver, pde, turbulence and pressure objects (oracle/Makefile target
`dropin`).  Both programs run the same parameter file and inputs; the fields
they save must agree to the FP64 gate (1e-10 relative, per field).
"""
import glob
import os
import subprocess

import numpy as np
import pytest

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


@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFMAIN)),
                    reason="reference objects were not available when oracle/Makefile ran")
def test_reference_main_links_and_matches(tmp_path, params_from_text):
    from wildfires_b200 import configs
    case = configs.hill(Nx=33, Ny=33, Nz=16, Nt=10, NT=5, L=100.0, H=20.0, jitter=0.2, seed=3)
    P = params_from_text(configs.param_text(case.params))
    ours, _ = _run(DROPIN, case, tmp_path / "dropin")
    ref, _ = _run(REFMAIN, case, tmp_path / "reference")
    for n in (1, 2):   # saves at steps 5 and 10
        y_o, p_o = _fields(ours, P, n)
        y_r, p_r = _fields(ref, P, n)
        errs = field_errors(P, y_o, y_r)
        bad = {f: e for f, e in errs.items() if e[0] > 1e-10 or e[1] > 1e-10}
        assert not bad, (n, bad)
        assert np.max(np.abs(p_o - p_r)) <= 1e-10 * np.max(np.abs(p_r))
    # the drop-in reported through the reference's own logging
    log = open(os.path.join(ours, "log.txt")).read()
    assert "Solver time" in log
