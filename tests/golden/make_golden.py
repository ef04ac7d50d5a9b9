"""Generate the golden fixtures under tests/golden/ from the REFERENCE's own
solver (its src/cu sources compiled for the CPU by oracle/Makefile -> oracle/_ref/ref_host).

Run from the repository root in a container where the reference tree exists:

    make -C oracle ref REF=<reference tree> && python tests/golden/make_golden.py [name ...]

Each fixture <name>.npz holds the parameter file text, the reference parser's
view of the grid (z, Nz_Y, cut_nodes), the seeded initial state and the
reference outputs of
  phi      one right-hand-side evaluation  (src/cu/pde.cu:910-917)
  rk       one RK combination when method = RK4 (src/cu/solver.cu:76-93)
  pressure one pressure solve on the initial state (src/cu/pressure.cu:506-606)
  steps    Nt full time steps of solve_PDE (src/cu/solver.cu:95-265).
The reference driver reads the parameter file with the reference parser, so
the fixtures also pin this package's parser.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from wildfires_b200 import configs  # noqa: E402
import ref_runner  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def cases():
    """name -> Case; small grids that exercise every branch of the step."""
    c = {}
    c["flat_rk4"] = configs.flat(Nx=17, Ny=13, Nz=12, Nt=3, jitter=0.3, seed=1)
    c["hill_rk4"] = configs.hill(Nx=17, Ny=17, Nz=16, Nt=3, jitter=0.3, seed=2, L=40.0, H=8.0)
    # non-uniform z, RK2, forward pressure gradient, central T convection, Sutherland laws
    c["stretched_rk2"] = configs.flat(Nx=13, Ny=17, Nz=14, Nt=2, jitter=0.2, seed=3, method="RK2", z_domain=1,
                                      k_nu_grid=2.0, velocity_correction_fd=1, temperature_convection=0,
                                      sutherland_viscosity=1, sutherland_conductivity=1)
    # explicit Euler, backward pressure gradient, held temperature source
    c["source_euler"] = configs.hill(Nx=13, Ny=13, Nz=12, Nt=3, jitter=0.2, seed=4, L=30.0, H=8.0, method="Euler",
                                     velocity_correction_fd=-1, t_source_start=0.0, t_source_end=1.0)
    # variable density with a fixed number of fixed-point iterations
    c["vardens_rk4"] = configs.flat(Nx=13, Ny=13, Nz=12, Nt=2, jitter=0.2, seed=5, variable_density=1,
                                    pressure_solver_iter=3, pressure_solver_tol=-1.0)
    # more steps on a slightly larger grid (growth of rounding differences)
    c["flat_33x33x16_10"] = configs.flat(Nx=33, Ny=33, Nz=16, Nt=10, jitter=0.1, seed=6)
    # ramped temperature sources (temperature_source_delay, src/cu/functions.cu:325-380):
    # gaussian, ramp ending within the run; box, source switched off before the last step
    c["ramp_gauss_rk4"] = configs.hill(Nx=13, Ny=13, Nz=12, Nt=3, jitter=0.2, seed=7, L=30.0, H=8.0,
                                       t_source_start=2.5 * 0.003, t_source_end=10 * 0.003,
                                       T_source_shape="gaussian", T_source=800.0, TS_x_start=8.0,
                                       TS_x_end=16.0, TS_y_start=10.0, TS_y_end=20.0, TS_z_start=0.0,
                                       TS_z_end=2.0)
    c["ramp_box_euler"] = configs.flat(Nx=13, Ny=13, Nz=12, Nt=3, jitter=0.2, seed=8, method="Euler",
                                       t_source_start=1.5 * 0.005, t_source_end=2.5 * 0.005,
                                       T_source_shape="parallelepiped", T_source=700.0, TS_x_start=40.0,
                                       TS_x_end=90.0, TS_y_start=60.0, TS_y_end=140.0, TS_z_start=0.0,
                                       TS_z_end=3.0)
    return c


def main():
    if not ref_runner.available("host"):
        sys.exit("oracle/_ref/ref_host missing: run `make -C oracle ref REF=<reference tree>`")
    only = set(sys.argv[1:])   # optional: fixture names to (re)generate
    for name, case in cases().items():
        if only and name not in only:
            continue
        data = {"params": np.array(configs.param_text(case.params))}
        res = ref_runner.run(case, "phi")
        P = res["P"]
        r = P.rec
        data.update(z=P.z(), nz_y=P.nz_y(), cut=P.cut_nodes(), y0=res["y0"], p0=res["p0"], phi=res["R"])
        if case.params.get("method", "RK4") == "RK4":
            data["rk"] = ref_runner.run(case, "rk4")["y1"]
        pr = ref_runner.run(case, "pressure")
        data["pressure"] = pr["p"]
        st = ref_runner.run(case, "step")
        data["steps_y"] = st["y"]
        data["steps_p"] = st["p"]
        data["nsteps"] = np.array(r.Nt)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
        print("wrote", name, "N =", r.Nx * r.Ny * r.Nz)


if __name__ == "__main__":
    main()
