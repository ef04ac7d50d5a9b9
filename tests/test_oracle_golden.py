"""The CPU oracle against the golden fixtures produced by the reference's own
solver sources (tests/golden/make_golden.py), and the library's parameter
parser against the reference parser's derived tables.  CPU only."""
import numpy as np
import pytest

import oracle_py as O
from conftest import field_errors, golden_names, load_golden

NAMES = golden_names()


@pytest.mark.parametrize("name", NAMES)
def test_parser_matches_reference_tables(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    np.testing.assert_array_equal(P.z(), g["z"])
    np.testing.assert_array_equal(P.nz_y(), g["nz_y"])
    np.testing.assert_array_equal(P.cut_nodes(), g["cut"])
    assert P.state_size == g["y0"].size


@pytest.mark.parametrize("name", NAMES)
def test_oracle_phi_matches_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    R = O.phi(P, g["y0"])
    for f, (linf, l2) in field_errors(P, R, g["phi"]).items():
        assert linf <= 1e-13 and l2 <= 1e-13, (f, linf, l2)


@pytest.mark.parametrize("name", [n for n in NAMES if "rk" in load_golden(n)])
def test_oracle_rk4_matches_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    y1 = O.rk(P, g["y0"])
    for f, (linf, l2) in field_errors(P, y1, g["rk"]).items():
        assert linf <= 1e-13 and l2 <= 1e-13, (f, linf, l2)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_pressure_matches_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    p, _ = O.pressure(P, g["y0"], g["y0"], g["p0"])
    scale = np.max(np.abs(g["pressure"]))
    assert np.max(np.abs(p - g["pressure"])) <= 1e-12 * scale


@pytest.mark.parametrize("name", NAMES)
def test_oracle_steps_match_reference(name, params_from_text):
    g = load_golden(name)
    P = params_from_text(g["params"])
    y, p = O.steps(P, g["y0"], g["p0"], int(g["nsteps"]))
    for f, (linf, l2) in field_errors(P, y, g["steps_y"]).items():
        assert linf <= 1e-11 and l2 <= 1e-11, (f, linf, l2)
    assert np.max(np.abs(p - g["steps_p"])) <= 1e-10 * np.max(np.abs(g["steps_p"]))


def test_cpu_fft_against_direct_dft():
    import ctypes as C
    L = C.CDLL(O.LIB)
    L.cfft_plan_create.restype = C.c_void_p
    L.cfft_plan_create.argtypes = [C.c_int]
    L.cfft_exec.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
    L.cfft_plan_destroy.argtypes = [C.c_void_p]
    rng = np.random.default_rng(0)
    for n in (1, 2, 3, 12, 17, 95, 127, 128, 159, 191, 255, 511):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        for sign in (-1, 1):
            buf = np.empty(2 * n)
            buf[0::2], buf[1::2] = x.real, x.imag
            plan = L.cfft_plan_create(n)
            L.cfft_exec(plan, buf.ctypes.data_as(C.POINTER(C.c_double)), sign)
            L.cfft_plan_destroy(plan)
            got = buf[0::2] + 1j * buf[1::2]
            ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n
            assert np.max(np.abs(got - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref))), n
