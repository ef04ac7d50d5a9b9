"""ctypes binding of the CPU oracle (liboracle.so, a restatement of the
reference time step in plain C).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None
_dp = C.POINTER(C.c_double)


def build():
    """Compile liboracle.so with oracle/Makefile (gcc, no GPU needed)."""
    r = subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.wfo_state_size.restype = C.c_size_t
        L.wfo_state_size.argtypes = [vp]
        L.wfo_phi.argtypes = [vp, _dp, _dp]
        L.wfo_time_integrate.argtypes = [vp, C.c_double, _dp, _dp]
        L.wfo_solve_pressure.restype = C.c_int
        L.wfo_solve_pressure.argtypes = [vp, _dp, _dp, _dp, _dp]
        L.wfo_project.argtypes = [vp, _dp, _dp, _dp]
        L.wfo_temperature_source.argtypes = [vp, _dp, C.c_double, _dp]
        L.wfo_step.restype = C.c_int
        L.wfo_step.argtypes = [vp, _dp, _dp, C.c_int, _dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _rec(P):
    return C.cast(C.byref(P.rec), C.c_void_p)


def phi(P, R_old):
    R_old = np.ascontiguousarray(R_old, dtype=np.float64)
    out = np.zeros_like(R_old)
    lib().wfo_phi(_rec(P), _p(R_old), _p(out))
    return out


def rk(P, y0):
    y0 = np.ascontiguousarray(y0, dtype=np.float64)
    out = np.zeros_like(y0)
    lib().wfo_time_integrate(_rec(P), 0.0, _p(y0), _p(out))
    return out


def pressure(P, y_np1, y_n, p):
    a = np.ascontiguousarray(y_np1, dtype=np.float64)
    b = np.ascontiguousarray(y_n, dtype=np.float64)
    pp = np.array(p, dtype=np.float64, copy=True)
    err = C.c_double()
    it = lib().wfo_solve_pressure(_rec(P), _p(a), _p(b), _p(pp), C.byref(err))
    return pp, it


def pressure_full(P, y_np1, y_n, p):
    """pressure() that also returns the last max-norm change: (p, solves, change)."""
    a = np.ascontiguousarray(y_np1, dtype=np.float64)
    b = np.ascontiguousarray(y_n, dtype=np.float64)
    pp = np.array(p, dtype=np.float64, copy=True)
    err = C.c_double()
    it = lib().wfo_solve_pressure(_rec(P), _p(a), _p(b), _p(pp), C.byref(err))
    return pp, it, err.value


def project(P, y_np1, y_n, p):
    y1 = np.array(y_np1, dtype=np.float64, copy=True)
    b = np.ascontiguousarray(y_n, dtype=np.float64)
    pp = np.ascontiguousarray(p, dtype=np.float64)
    lib().wfo_project(_rec(P), _p(y1), _p(b), _p(pp))
    return y1


def steps(P, y0, p0, nsteps, first=1):
    """Advance nsteps full time steps; returns (y, p)."""
    y = np.array(y0, dtype=np.float64, copy=True)
    p = np.array(p0, dtype=np.float64, copy=True)
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    Ts = y[3 * N:4 * N].copy()    # the held source is the initial temperature field
    for n in range(first, first + nsteps):
        rc = lib().wfo_step(_rec(P), _p(y), _p(p), n, _p(Ts))
        if rc != 0:
            raise RuntimeError("oracle step failed")
    return y, p
