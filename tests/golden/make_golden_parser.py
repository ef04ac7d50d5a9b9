"""Generate tests/golden/parser_records.npz: the record the REFERENCE's own
parser (read_parameters_file, src/cu/parameters.cu:11-523) builds from a set
of parameter files, through oracle/_ref/ref_host in mode `params`.

Run from the repository root in a container where the reference tree exists:

    make -C oracle ref REF=<reference tree> && python tests/golden/make_golden_parser.py

For each case the fixture holds the file text, the reference record's raw
bytes (the record layout is shared: include/wf_parameters.h) and the arrays
it points to (x, y, z, t, kx, ky, topography as FP64; cut_nodes, Nz_Y as
int32); for DOMAIN_CASES also the bytes of the files the reference's
save_domain and save_topography write (file_<name>).
tests/test_parser_golden.py compares this package's parser and writers with them.
"""
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ref_runner  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "parser_records.npz")

GRID = "Nx = 13\nNy = 11\nNz = 12\nNt = 6\nx_max = 30\ny_max = 24\nz_max = 8\nt_max = 0.03\n"

CASES = {
    # the grid only: every other member takes the reference's default
    "minimal": GRID,
    # every key of the reference's table set away from its default
    "full": GRID + """NT = 3
x_min = -2.5
y_min = 1.25
z_min = 0
t_min = 0.005
nu = 1.6e-5
mu = 1.9e-5
u_r = 6.5
z_r = 3.5
alpha_u = 0.21
alpha = 2.3e-5
T_inf = 295.5
T_0 = 812.25
T_source = 760.5
T0_shape = parallelepiped
T0_x_start = 4
T0_x_end = 9
T0_y_start = 5
T0_y_end = 15
T0_z_start = 0
T0_z_end = 1.5
Y0_x_start = 2
Y0_x_end = 26
Y0_y_start = 3
Y0_y_end = 20
Y0_xa = 1.5
Y0_ya = 2.5
Y_h = 0.75
Y_f = 120.5
C_d = 0.9
alpha_s = 0.05
sigma_s = 4500
H_C = 2.1e7
A = 1.2e9
T_act = 17500.5
T_pc = 520.5
h_c = 1.5
c_p = 1010.5
rho_inf = 1.15
U0_type = log
g = -9.79
C_s = 0.19
Pr = 0.72
p_top = 0.5
method = RK2
threads = 4
T_min = 280.5
T_max = 1600.5
Y_min = 0.01
Y_max = 0.99
topo_shape = hill
u_dead_nodes = 0.1
v_dead_nodes = 0.2
w_dead_nodes = 0.3
T_dead_nodes = 301.5
Y_dead_nodes = 0.5
hill_center_x = 14
hill_center_y = 11
hill_length = 6
hill_width = 7
hill_height = 2.5
t_source_start = 0.01
t_source_end = 0.02
T_source_shape = gaussian
delta = 0.4
k = 0.03
variable_density = 0
pressure_solver_tol = 1e-9
pressure_solver_iter = 7
pressure_solver_log = 1
z_domain = 1
k_nu_grid = 1.7
k_transition = 4
z_transition = 2.5
input_path = some/dir/
velocity_correction_fd = -1
time_step_log = 2
temperature_convection = 0
TS_x_start = 6
TS_x_end = 12
TS_y_start = 4
TS_y_end = 10
TS_z_start = 0
TS_z_end = 2
sutherland_viscosity = 1
sutherland_conductivity = 1
""",
    # line-matching rules: later lines win, only "key =" at column 0 matches,
    # values are read by sscanf (trailing text ignored, %d truncates), unknown
    # keys and comment lines are skipped
    "quirks": GRID + """C_s = 0.1
C_s = 0.25
 C_d = 7
Pr=0.9
# T_inf = 250
T_0 = 700 # ignition temperature
Nt = 8.9
method = RK4 extra words
unknown_key = 3
T_min = 250
T_minimum = 5
alpha_u = 0.3
alpha = 4e-5
z_domain = 2
k_transition = 5
z_transition = 3
""",
    # flat terrain, a save interval that does not divide Nt, two-zone z grid
    "flat_nt": GRID + """NT = 4
topo_shape = flat
z_domain = 2
k_transition = 5
z_transition = 3
""",
}
# cases whose files also go through the reference's save_domain / save_topography
# (output.cu:46-99); they need NT >= 1, which the reference divides by
DOMAIN_CASES = ("full", "flat_nt")


def main():
    if not ref_runner.available("host"):
        sys.exit("oracle/_ref/ref_host missing: run `make -C oracle ref REF=<reference tree>`")
    data = {}
    for name, text in CASES.items():
        work = tempfile.mkdtemp(prefix="wf_parser_")
        try:
            with open(os.path.join(work, "parameters.txt"), "w") as f:
                f.write(text)
            os.makedirs(os.path.join(work, "out"))
            r = subprocess.run([ref_runner.binary("host"), "params", "parameters.txt", "out"], cwd=work,
                               capture_output=True, text=True, timeout=600)
            if r.returncode != 0:
                sys.exit("reference driver failed on %s:\n%s" % (name, r.stderr[-2000:]))
            out = os.path.join(work, "out")
            data[name + "/text"] = np.array(text)
            with open(os.path.join(out, "params.bin"), "rb") as f:
                data[name + "/record"] = np.frombuffer(f.read(), dtype=np.uint8)
            for nm in ("x", "y", "z", "t", "kx", "ky", "topography"):
                data[name + "/" + nm] = np.fromfile(os.path.join(out, nm + ".bin"))
            for nm in ("cut_nodes", "Nz_Y"):
                data[name + "/" + nm] = np.fromfile(os.path.join(out, nm + ".bin"), dtype=np.int32)
            if name in DOMAIN_CASES:
                dom = os.path.join(work, "dom")
                os.makedirs(dom)
                r = subprocess.run([ref_runner.binary("host"), "domain", "parameters.txt", "dom"], cwd=work,
                                   capture_output=True, text=True, timeout=600)
                if r.returncode != 0:
                    sys.exit("reference driver (domain) failed on %s:\n%s" % (name, r.stderr[-2000:]))
                for nm in ("x", "y", "z", "t", "topography", "Nz_Y"):
                    with open(os.path.join(dom, nm + ".bin"), "rb") as f:
                        data[name + "/file_" + nm] = np.frombuffer(f.read(), dtype=np.uint8)
        finally:
            shutil.rmtree(work, ignore_errors=True)
        print("parsed", name)
    np.savez_compressed(OUT, **data)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
