"""Generate tests/golden/ic_*.npz: the REFERENCE's own initial conditions
(initial_conditions + create_y_0, src/cu/functions.cu:187-323 and
src/cu/solver.cu:41-56) from its src/cu sources compiled for the CPU
(oracle/_ref/ref_host, driver mode `ic`).

Run from the repository root in a container where the reference tree exists:

    make -C oracle ref REF=<reference tree> && python tests/golden/make_golden_ic.py

Each fixture holds the parameter-file text, the terrain override (if any) and
the packed initial state and pressure.  Y entries the reference leaves
unwritten (above a column's fuel top, outside the fuel shapes) are zero.
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
    c = {}
    # terrain with dead nodes, gaussian initial temperature, a fuel rectangle
    # inside the domain with ramps on all four sides, non-default wind and p_top
    c["ic_hill_gauss"] = configs.hill(
        Nx=33, Ny=25, Nz=16, Nt=1, L=60.0, H=10.0, seed=7, T0_shape="gaussian", T_0=900.0,
        T0_x_start=10.0, T0_x_end=22.0, T0_y_start=18.0, T0_y_end=30.0, T0_z_start=0.0, T0_z_end=3.0,
        Y0_x_start=12.0, Y0_x_end=44.0, Y0_y_start=15.0, Y0_y_end=40.0, Y0_xa=5.0, Y0_ya=7.5, Y_h=1.3,
        u_r=4.5, z_r=2.5, alpha_u=0.21, p_top=12.5, u_dead_nodes=0.25, v_dead_nodes=-0.5,
        w_dead_nodes=0.125, T_dead_nodes=301.0, Y_dead_nodes=0.75)
    # stretched z, parallelepiped initial temperature, flat terrain
    c["ic_flat_box"] = configs.flat(
        Nx=21, Ny=17, Nz=14, Nt=1, seed=8, z_domain=1, k_nu_grid=2.0, T0_shape="parallelepiped", T_0=700.0,
        T0_x_start=40.0, T0_x_end=90.0, T0_y_start=60.0, T0_y_end=120.0, T0_z_start=0.0, T0_z_end=2.0,
        Y0_x_start=20.0, Y0_x_end=180.0, Y0_y_start=30.0, Y0_y_end=170.0, Y0_xa=12.0, Y0_ya=12.0, Y_h=0.9,
        p_top=-3.0)
    return c


def main():
    if not ref_runner.available("host"):
        sys.exit("oracle/_ref/ref_host missing: run `make -C oracle ref REF=<reference tree>`")
    for name, case in cases().items():
        res = ref_runner.run(case, "ic")
        P = res["P"]
        topo = case.topography(P)
        data = {"params": np.array(configs.param_text(case.params)), "y0": res["ic_y"], "p0": res["ic_p"]}
        if topo is not None:
            data["topography"] = np.ascontiguousarray(topo, dtype=np.float64).reshape(-1)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **data)
        r = P.rec
        print("wrote", name, "N =", r.Nx * r.Ny * r.Nz, "Nz_Y_max =", r.Nz_Y_max)


if __name__ == "__main__":
    main()
