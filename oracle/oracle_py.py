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


def timestep_reports(P, y):
    """numpy restatement of timestep_reports (src/cu/functions.cu:82-185) on a
    packed FP64 state: returns (CFL, Y_min, Y_max, T_min, T_max, first_nan),
    first_nan = None or (field, i, j, k) of the first NaN in the reference's
    scan order (i, j, k, then u, v, w, T, Y).  T and Y ranges only inside the
    fuel rectangle [Y0_x_start, Y0_x_end] x [Y0_y_start, Y0_y_end], from the
    reference's starting values (T: 1e9 / -1e9, Y: 0 / -1e9); Y is read for
    k < Nz_Y_max (:125-133), velocity maxima start at 0 (:101-103)."""
    r = P.rec
    Nx, Ny, Nz, NzY = r.Nx, r.Ny, r.Nz, r.Nz_Y_max
    N = Nx * Ny * Nz
    y = np.asarray(y, dtype=np.float64)
    u, v, w, T = (y[q * N:(q + 1) * N].reshape(Nx, Ny, Nz) for q in range(4))
    Y = np.zeros((Nx, Ny, Nz))
    Y[:, :, :NzY] = y[4 * N:4 * N + Nx * Ny * NzY].reshape(Nx, Ny, NzY)
    flags = np.stack([np.isnan(a) for a in (u, v, w, T, Y)], axis=-1)
    first = None
    if flags.any():
        q = int(np.flatnonzero(flags.reshape(-1))[0])
        first = (q % 5, q // 5 // (Ny * Nz), (q // 5 // Nz) % Ny, q // 5 % Nz)
    x = np.ctypeslib.as_array(r.x, shape=(Nx,))
    yy = np.ctypeslib.as_array(r.y, shape=(Ny,))
    zx = (r.Y0_x_start <= x) & (x <= r.Y0_x_end)
    zy = (r.Y0_y_start <= yy) & (yy <= r.Y0_y_end)
    zone = zx[:, None] & zy[None, :]
    ok = ~flags.any(axis=-1)

    def ext(a, mask, f, start):
        vals = a[mask]
        return f(np.concatenate([[start], vals])) if vals.size else start

    mu = ext(np.abs(u), ok, np.max, 0.0)
    mv = ext(np.abs(v), ok, np.max, 0.0)
    mw = ext(np.abs(w), ok, np.max, 0.0)
    zmask = zone[:, :, None] & ok
    T_min = ext(T, zmask, np.min, 1e9)
    T_max = ext(T, zmask, np.max, -1e9)
    ymask = zmask & (np.arange(Nz) < NzY)[None, None, :]
    Y_min = ext(Y, ymask, np.min, 0.0)
    Y_max = ext(Y, ymask, np.max, -1e9)
    cfl = r.dt * (mu / r.dx + mv / r.dy + mw / r.dz)
    return cfl, Y_min, Y_max, T_min, T_max, first
