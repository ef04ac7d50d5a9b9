"""Seeded synthetic workloads of the benchmark configurations.

No dataset is involved: every initial state is generated here from a seed.
Each case is a reference-format parameter file (``key = value`` lines, the
keys of src/cu/parameters.cu:78-414) plus initial fields in the reference's
raw binary layout (src/cu/input.cu:3-58), built after the parameter record is
parsed so that the grid, the terrain and the fuel tables are the solver's own.

Cases
  flat      128 x 128 x 64 flat, log wind u_r = 5 m/s, gaussian ignition,
            RK4 dt = 0.005 s, 200 steps
  hill      256 x 256 x 128 under a 10 m gaussian hill, log wind u_r = 8 m/s
            measured above the terrain, 100 m line ignition, dt = 0.003 s, 500 steps
  hills8    512 x 512 x 128, 8 seeded gaussian hills, per-column fuel
            Y ~ U(0.6, 1), wind u_r = 6 m/s at a seeded direction, 3 hot spots
            in the upwind third, dt = 0.003 s, 1000 steps
and reduced versions of each (any size) for parity tests.  Parity settings
(inert reference quirks): variable_density = 0, alpha_s = sigma_s = 0,
p_top = 0, no temperature source, Sutherland laws off, explicit Y_f.
"""
import math
import os

import numpy as np

Z0 = 0.05          # roughness length of the log wind profile (m)
T_AMB = 300.0      # ambient temperature (K)


def _fmt(v):
    if isinstance(v, str):
        return v
    if isinstance(v, (int, np.integer)):
        return "%d" % v
    return repr(float(v))


def param_text(d):
    return "".join("%s = %s\n" % (k, _fmt(v)) for k, v in d.items())


def base_params(Nx, Ny, Nz, Nt, x_max, y_max, z_max, t_max, **kw):
    d = dict(
        Nx=Nx, Ny=Ny, Nz=Nz, Nt=Nt, NT=Nt,
        x_min=0.0, x_max=x_max, y_min=0.0, y_max=y_max, z_min=0.0, z_max=z_max,
        t_min=0.0, t_max=t_max, method="RK4",
        rho_inf=1.1, C_s=0.173, T_inf=T_AMB, T_dead_nodes=T_AMB,
        Y_f=100.0, Y_h=0.5, alpha_s=0.0, sigma_s=0.0, p_top=0.0,
        variable_density=0, pressure_solver_iter=1, pressure_solver_tol=-1.0,
        t_source_start=0.0, t_source_end=0.0, topo_shape="flat",
        Y0_x_start=0.0, Y0_x_end=x_max, Y0_y_start=0.0, Y0_y_end=y_max,
        temperature_convection=1, velocity_correction_fd=0, time_step_log=1000000,
    )
    d.update(kw)
    return d


class Case:
    """A parameter dict, an optional terrain override and an initial-state builder."""

    def __init__(self, name, params, fields, topography=None, hills=None):
        self.name = name
        self.params = params
        self._fields = fields
        self._topo = topography
        # Gaussian hills of the terrain, (centre x, centre y, height, width) each:
        # the same terrain on the device by wf_set_topography_hills
        self.hills = hills

    def topography(self, P):
        return None if self._topo is None else self._topo(P)

    def fields(self, P):
        """Initial packed state y0 and pressure p0 for the parsed record P."""
        return self._fields(P)


def _grid(P):
    r = P.rec
    x = r.x_min + np.arange(r.Nx) * r.dx
    y = r.y_min + np.arange(r.Ny) * r.dy
    z = P.z()
    return x, y, z


def _topo_array(P):
    return P.topo()


def _pack(P, u, v, w, T, Y):
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    NzY = r.Nz_Y_max
    y = np.empty(4 * N + r.Nx * r.Ny * NzY)
    for q, f in enumerate((u, v, w, T)):
        y[q * N:(q + 1) * N] = f.reshape(-1)
    y[4 * N:] = Y[:, :, :NzY].reshape(-1)
    return y


def _periodic(f):
    """Make the duplicate planes i = Nx-1 and j = Ny-1 copies of planes 0."""
    f[-1, :, :] = f[0, :, :]
    f[:, -1, :] = f[:, 0, :]
    return f


def _finish(P, u, v, w, T, Y, rng=None, jitter=0.0):
    """Dead nodes, fuel above the column top, periodic planes; pack."""
    r = P.rec
    cut = P.cut_nodes()
    nzy = P.nz_y()
    k = np.arange(r.Nz)[None, None, :]
    if jitter and rng is not None:
        u = u + jitter * rng.standard_normal(u.shape)
        v = v + jitter * rng.standard_normal(v.shape)
        w = w + 0.5 * jitter * rng.standard_normal(w.shape)
        T = T + 5 * jitter * rng.standard_normal(T.shape)
    dead = k < cut[:, :, None]
    u = np.where(dead, r.u_dead_nodes, u)
    v = np.where(dead, r.v_dead_nodes, v)
    w = np.where(dead, r.w_dead_nodes, w)
    T = np.where(dead, r.T_dead_nodes, T)
    Y = np.where(k < nzy[:, :, None], Y, 0.0)
    Y = np.where(dead & (k < nzy[:, :, None]), r.Y_dead_nodes, Y)
    u, v, w, T, Y = (_periodic(np.array(a, dtype=np.float64)) for a in (u, v, w, T, Y))
    p = np.zeros((r.Nx, r.Ny, r.Nz))
    p[:, :, -1] = r.p_top
    return _pack(P, u, v, w, T, Y), p.reshape(-1)


def log_wind(height, u_r, z_r=2.0):
    h = np.maximum(height, Z0)
    return u_r * np.log(h / Z0) / math.log(z_r / Z0)


# ---- flat ------------------------------------------------------------------
def flat(Nx=128, Ny=128, Nz=64, Nt=200, dt=0.005, seed=0, jitter=0.0, **kw):
    Lx, Ly, Lz = 200.0, 200.0, 20.0
    params = base_params(Nx, Ny, Nz, Nt, Lx, Ly, Lz, Nt * dt, **kw)

    def fields(P):
        x, y, z = _grid(P)
        X, Yg, Z = np.meshgrid(x, y, z, indexing="ij")
        u = log_wind(Z, 5.0)
        v = np.zeros_like(u)
        w = np.zeros_like(u)
        # ignition centred at (50, 100) m (scaled with the box)
        xc, yc = 50.0 * Lx / 200.0, 100.0 * Ly / 200.0
        T = T_AMB + np.where(Z < 1.0, 500.0 * np.exp(-((X - xc) ** 2 + (Yg - yc) ** 2) / 18.0), 0.0)
        Y = np.ones_like(u)
        rng = np.random.default_rng(seed)
        return _finish(P, u, v, w, T, Y, rng, jitter)

    return Case("flat", params, fields)


# ---- single hill -------------------------------------------------------------
def hill(Nx=256, Ny=256, Nz=128, Nt=500, dt=0.003, seed=0, jitter=0.0, L=400.0, H=50.0, **kw):
    s = L / 400.0
    params = base_params(Nx, Ny, Nz, Nt, L, L, H, Nt * dt, topo_shape="hill",
                         hill_center_x=200.0 * s, hill_center_y=200.0 * s,
                         hill_length=60.0 * math.sqrt(2.0) * s, hill_width=60.0 * math.sqrt(2.0) * s,
                         hill_height=10.0 * H / 50.0, **kw)

    def fields(P):
        x, y, z = _grid(P)
        topo = _topo_array(P)
        X, Yg, Z = np.meshgrid(x, y, z, indexing="ij")
        hgt = Z - topo[:, :, None]
        u = log_wind(hgt, 8.0)
        v = np.zeros_like(u)
        w = np.zeros_like(u)
        line = (np.abs(Yg - 200.0 * s) <= 50.0 * s) & (hgt < 1.0)
        T = T_AMB + np.where(line, 500.0 * np.exp(-((X - 80.0 * s) ** 2) / (2 * 3.0 ** 2)), 0.0)
        Y = np.ones_like(u)
        rng = np.random.default_rng(seed)
        return _finish(P, u, v, w, T, Y, rng, jitter)

    return Case("hill", params, fields)


# ---- eight seeded hills (mixed-precision workload) ------------------------------
def hills8(Nx=512, Ny=512, Nz=128, Nt=1000, dt=0.003, seed=1234, L=800.0, H=60.0, jitter=0.0, **kw):
    # hill heights and widths are physical sizes: a smaller box (a bounded
    # sample of the workload) keeps the same terrain statistics
    params = base_params(Nx, Ny, Nz, Nt, L, L, H, Nt * dt, **kw)
    rng0 = np.random.default_rng(seed)
    hills = [(rng0.uniform(0, L), rng0.uniform(0, L), rng0.uniform(2, 15), rng0.uniform(20, 80))
             for _ in range(8)]
    theta = rng0.uniform(0, 2 * math.pi)
    spots = rng0.uniform(0, 1, size=(3, 2))
    fuel_seed = int(rng0.integers(1 << 30))

    def topography(P):
        x, y, _ = _grid(P)
        X, Yg = np.meshgrid(x, y, indexing="ij")
        h = np.zeros_like(X)
        for (cx, cy, hh, wd) in hills:
            # periodic distance so the terrain is continuous across the wrap
            dx = (X - cx + L / 2) % L - L / 2
            dy = (Yg - cy + L / 2) % L - L / 2
            h += hh * np.exp(-(dx ** 2 + dy ** 2) / (2 * wd ** 2))
        return h

    def fields(P):
        x, y, z = _grid(P)
        topo = _topo_array(P)
        X, Yg, Z = np.meshgrid(x, y, z, indexing="ij")
        hgt = Z - topo[:, :, None]
        speed = log_wind(hgt, 6.0)
        u = speed * math.cos(theta)
        v = speed * math.sin(theta)
        w = np.zeros_like(u)
        # hot spots in the upwind third along the wind direction; overlapping
        # spots take the hotter value (a sum would exceed the +500 K of one spot
        # and drive fuel cells past the RK4 stability limit of the reaction,
        # dt * Y_f * K(T) < 2.8, i.e. about 950 K at dt = 0.003 s)
        heat = np.zeros_like(u)
        ux, uy = math.cos(theta), math.sin(theta)
        for (a, b) in spots:
            along = (a / 3.0 - 0.5) * L       # upwind third of the box
            across = (b - 0.5) * L
            cx = L / 2 + along * ux - across * uy
            cy = L / 2 + along * uy + across * ux
            dx = (X - cx + L / 2) % L - L / 2
            dy = (Yg - cy + L / 2) % L - L / 2
            heat = np.maximum(heat, np.where(hgt < 1.0, 500.0 * np.exp(-(dx ** 2 + dy ** 2) / (2 * 3.0 ** 2)), 0.0))
        T = T_AMB + heat
        frng = np.random.default_rng(fuel_seed)
        Ycol = frng.uniform(0.6, 1.0, size=(P.rec.Nx, P.rec.Ny))
        Y = np.broadcast_to(Ycol[:, :, None], u.shape).copy()
        rng = np.random.default_rng(seed + 1)
        return _finish(P, u, v, w, T, Y, rng, jitter)

    return Case("hills8", params, fields, topography, hills)


# ---- ensemble members (uneven grids, varied wind, terrain, ignition, fuel) ----------
ENSEMBLE_SIZES = (96, 128, 160, 192, 256)


def scenario(Nx, Ny, Nz=64, Nt=300, dt=0.005, seed=0, dx=1.5625, z_max=19.6875, jitter=0.0, **kw):
    """One ensemble member: Nx x Ny x Nz with dx = dy = 1.5625 m and dz =
    0.3125 m, 0-4 seeded Gaussian hills (1-4 m), log wind of u_r ~ U(2, 10) m/s
    at a random direction, 1-3 hot spots (+500 K, sigma 3 m) and per-column fuel
    Y ~ U(0.5, 1)."""
    Lx, Ly = (Nx - 1) * dx, (Ny - 1) * dx
    params = base_params(Nx, Ny, Nz, Nt, Lx, Ly, z_max, Nt * dt, **kw)
    rng0 = np.random.default_rng(seed)
    nh = int(rng0.integers(0, 5))
    hills = [(rng0.uniform(0, Lx), rng0.uniform(0, Ly), rng0.uniform(1, 4), rng0.uniform(10, 40)) for _ in range(nh)]
    u_r = rng0.uniform(2, 10)
    theta = rng0.uniform(0, 2 * math.pi)
    spots = rng0.uniform(0, 1, size=(int(rng0.integers(1, 4)), 2))
    fuel_seed = int(rng0.integers(1 << 30))

    def topography(P):
        if not hills:
            return None
        x, y, _ = _grid(P)
        X, Yg = np.meshgrid(x, y, indexing="ij")
        h = np.zeros_like(X)
        for (cx, cy, hh, wd) in hills:
            ddx = (X - cx + Lx / 2) % Lx - Lx / 2
            ddy = (Yg - cy + Ly / 2) % Ly - Ly / 2
            h += hh * np.exp(-(ddx ** 2 + ddy ** 2) / (2 * wd ** 2))
        return h

    def fields(P):
        x, y, z = _grid(P)
        topo = _topo_array(P)
        X, Yg, Z = np.meshgrid(x, y, z, indexing="ij")
        hgt = Z - topo[:, :, None]
        speed = log_wind(hgt, u_r)
        u = speed * math.cos(theta)
        v = speed * math.sin(theta)
        w = np.zeros_like(u)
        heat = np.zeros_like(u)
        for (a, b) in spots:
            cx, cy = a * Lx, b * Ly
            ddx = (X - cx + Lx / 2) % Lx - Lx / 2
            ddy = (Yg - cy + Ly / 2) % Ly - Ly / 2
            heat = np.maximum(heat, np.where(hgt < 1.0, 500.0 * np.exp(-(ddx ** 2 + ddy ** 2) / (2 * 3.0 ** 2)), 0.0))
        T = T_AMB + heat
        frng = np.random.default_rng(fuel_seed)
        Ycol = frng.uniform(0.5, 1.0, size=(P.rec.Nx, P.rec.Ny))
        Y = np.broadcast_to(Ycol[:, :, None], u.shape).copy()
        rng = np.random.default_rng(seed + 1)
        return _finish(P, u, v, w, T, Y, rng, jitter)

    return Case("scenario", params, fields, topography, hills if hills else None)


def ensemble(n=64, seed=2024, sizes=ENSEMBLE_SIZES, **kw):
    """n members with Nx, Ny drawn from `sizes` (seeded)."""
    rng = np.random.default_rng(seed)
    return [scenario(int(rng.choice(sizes)), int(rng.choice(sizes)), seed=int(rng.integers(1 << 30)), **kw)
            for _ in range(n)]


CASES = {"flat": flat, "hill": hill, "hills8": hills8}


def materialize(case):
    """Parse the case's parameters with the library, apply its terrain and build
    its initial state: returns (P, y0, p0)."""
    import shutil
    import tempfile
    from . import read_parameters
    d = tempfile.mkdtemp(prefix="wf_case_")
    try:
        path = os.path.join(d, "parameters.txt")
        with open(path, "w") as f:
            f.write(param_text(case.params))
        P = read_parameters(path)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    topo = case.topography(P)
    if topo is not None:
        P.set_topography(topo)
    y0, p0 = case.fields(P)
    return P, y0, p0


def write_case(case, directory, P=None, input_subdir="in/"):
    """Write parameters.txt and the initial fields (for the reference driver).

    The parameter file points input_path at ``input_subdir`` (relative to the
    directory the reference driver program runs in).  Returns the parameter-file path."""
    from . import read_parameters
    os.makedirs(directory, exist_ok=True)
    params = dict(case.params)
    params["input_path"] = input_subdir
    ppath = os.path.join(directory, "parameters.txt")
    with open(ppath, "w") as f:
        f.write(param_text(params))
    own = P is None
    if own:
        P = read_parameters(ppath)
    topo = case.topography(P)
    if topo is not None:
        P.set_topography(topo)
        np.ascontiguousarray(topo, dtype=np.float64).tofile(os.path.join(directory, "topography.bin"))
    y0, p0 = case.fields(P)
    r = P.rec
    N = r.Nx * r.Ny * r.Nz
    ind = os.path.join(directory, input_subdir)
    os.makedirs(ind, exist_ok=True)
    for q, nm in enumerate("uvwT"):
        y0[q * N:(q + 1) * N].tofile(os.path.join(ind, nm + ".bin"))
    y0[4 * N:].tofile(os.path.join(ind, "Y.bin"))
    p0.tofile(os.path.join(ind, "p.bin"))
    return ppath, P, y0, p0
