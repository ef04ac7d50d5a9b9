"""ctypes mirror of the run-description record (include/wf_parameters.h).

The record is laid out exactly like the reference's ``Parameters``
(include/c/structures.h:108-259) so one record can be handed to the
reference-compatible entry points and to this package's C-ABI alike.
"""
import ctypes as C

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)


class FieldIndexes(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("u", "v", "w", "T", "Y")]


class PressureIndexes(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("ux", "vy", "wz")]


class TurbulenceIndexes(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "rho", "Tx", "Ty", "Tz", "Txx", "Tyy", "Tzz", "mu_sgs",
        "S_11", "S_12", "S_13", "S_21", "S_22", "S_23", "S_31", "S_32", "S_33",
        "div_U", "u_tau_wall")]


class LogFiles(C.Structure):
    _fields_ = [("parameters", C.c_void_p), ("log", C.c_void_p)]


def _d(*names):
    return [(n, C.c_double) for n in names]


def _i(*names):
    return [(n, C.c_int) for n in names]


def _p(*names):
    return [(n, c_double_p) for n in names]


class Parameters(C.Structure):
    _fields_ = (
        _i("Nx", "Ny", "Nz", "Nt", "NT")
        + _d("x_min", "x_max", "y_min", "y_max", "z_min", "z_max", "t_min", "t_max")
        + _d("dx", "dy", "dz", "dt")
        + _p("x", "y", "z", "t", "r", "s", "kx", "ky")
        + _d("c_p", "c_v", "rho_inf", "mu", "k", "alpha", "delta", "nu", "T_inf", "g")
        + _d("C_s", "Pr", "C_d", "alpha_s", "sigma_s")
        + _d("T_pc", "H_C", "A", "E_A", "T_act", "h_c", "Y_D", "Y_f", "T_0", "T_source", "Y_h")
        + _i("k_Y_h", "Nz_Y_max")
        + [("Nz_Y", c_int_p)]
        + _d("T_min", "T_max", "Y_min", "Y_max")
        + [("U0_type", C.c_char * 32)]
        + _d("u_z0", "d", "u_ast", "u_r", "z_r", "alpha_u")
        + [("T0_shape", C.c_char * 32)]
        + _d("T0_x_start", "T0_x_end", "T0_x_center", "T0_length",
             "T0_y_start", "T0_y_end", "T0_y_center", "T0_width",
             "T0_z_start", "T0_z_end", "T0_z_center", "T0_height")
        + _d("Y0_x_start", "Y0_x_end", "Y0_y_start", "Y0_y_end", "Y0_xa", "Y0_ya")
        + [("topo_shape", C.c_char * 32), ("topography", c_double_p)]
        + _d("hill_center_x", "hill_center_y", "hill_length", "hill_width", "hill_height")
        + [("T_source_shape", C.c_char * 32)]
        + _d("t_source_start", "t_source_end",
             "TS_x_start", "TS_x_end", "TS_x_center", "TS_length",
             "TS_y_start", "TS_y_end", "TS_y_center", "TS_width",
             "TS_z_start", "TS_z_end", "TS_z_center", "TS_height")
        + [("cut_nodes", c_int_p), ("z_ibm", c_double_p)]
        + _d("p_top", "u_dead_nodes", "v_dead_nodes", "w_dead_nodes", "T_dead_nodes", "Y_dead_nodes")
        + _i("variable_density") + _d("pressure_solver_tol") + _i("pressure_solver_iter", "pressure_solver_log")
        + [("method", C.c_char * 32), ("save_path", C.c_char * 64),
           ("input_path", C.c_char * 64), ("sim_id", C.c_char * 32)]
        + _i("n_threads", "z_domain") + _d("k_nu_grid") + _i("k_transition") + _d("z_transition")
        + _i("velocity_correction_fd", "time_step_log", "temperature_convection",
             "sutherland_viscosity", "sutherland_conductivity")
        + [("threads_per_block", C.c_size_t), ("number_of_blocks", C.c_size_t),
           ("field_indexes", FieldIndexes), ("turbulence_indexes", TurbulenceIndexes),
           ("pressure_indexes", PressureIndexes), ("log_files", LogFiles)]
    )


assert C.sizeof(Parameters) == 1400, C.sizeof(Parameters)

# Keys accepted by the parameter-file parser, with their record member and
# scanf kind, in the order the reference tests them (src/cu/parameters.cu:78-414).
PARAM_KEYS = [
    ("Nx", "Nx", "d"), ("Ny", "Ny", "d"), ("Nz", "Nz", "d"), ("Nt", "Nt", "d"), ("NT", "NT", "d"),
    ("x_min", "x_min", "f"), ("x_max", "x_max", "f"), ("y_min", "y_min", "f"), ("y_max", "y_max", "f"),
    ("z_min", "z_min", "f"), ("z_max", "z_max", "f"), ("t_min", "t_min", "f"), ("t_max", "t_max", "f"),
    ("nu", "nu", "f"), ("mu", "mu", "f"), ("u_r", "u_r", "f"), ("z_r", "z_r", "f"),
    ("alpha_u", "alpha_u", "f"), ("alpha", "alpha", "f"), ("T_inf", "T_inf", "f"), ("T_0", "T_0", "f"),
    ("T_source", "T_source", "f"), ("T0_shape", "T0_shape", "s"),
    ("T0_x_start", "T0_x_start", "f"), ("T0_x_end", "T0_x_end", "f"),
    ("T0_y_start", "T0_y_start", "f"), ("T0_y_end", "T0_y_end", "f"),
    ("T0_z_start", "T0_z_start", "f"), ("T0_z_end", "T0_z_end", "f"),
    ("Y0_x_start", "Y0_x_start", "f"), ("Y0_x_end", "Y0_x_end", "f"),
    ("Y0_y_start", "Y0_y_start", "f"), ("Y0_y_end", "Y0_y_end", "f"),
    ("Y0_xa", "Y0_xa", "f"), ("Y0_ya", "Y0_ya", "f"), ("Y_h", "Y_h", "f"), ("Y_f", "Y_f", "f"),
    ("C_d", "C_d", "f"), ("alpha_s", "alpha_s", "f"), ("sigma_s", "sigma_s", "f"), ("H_C", "H_C", "f"),
    ("A", "A", "f"), ("T_act", "T_act", "f"), ("T_pc", "T_pc", "f"), ("h_c", "h_c", "f"),
    ("c_p", "c_p", "f"), ("rho_inf", "rho_inf", "f"), ("U0_type", "U0_type", "s"),
    ("g", "g", "f"), ("C_s", "C_s", "f"), ("Pr", "Pr", "f"), ("p_top", "p_top", "f"),
    ("method", "method", "s"), ("threads", "n_threads", "d"),
    ("T_min", "T_min", "f"), ("T_max", "T_max", "f"), ("Y_min", "Y_min", "f"), ("Y_max", "Y_max", "f"),
    ("topo_shape", "topo_shape", "s"),
    ("u_dead_nodes", "u_dead_nodes", "f"), ("v_dead_nodes", "v_dead_nodes", "f"),
    ("w_dead_nodes", "w_dead_nodes", "f"), ("T_dead_nodes", "T_dead_nodes", "f"),
    ("Y_dead_nodes", "Y_dead_nodes", "f"),
    ("hill_center_x", "hill_center_x", "f"), ("hill_center_y", "hill_center_y", "f"),
    ("hill_length", "hill_length", "f"), ("hill_width", "hill_width", "f"),
    ("hill_height", "hill_height", "f"),
    ("t_source_start", "t_source_start", "f"), ("t_source_end", "t_source_end", "f"),
    ("T_source_shape", "T_source_shape", "s"), ("delta", "delta", "f"), ("k", "k", "f"),
    ("variable_density", "variable_density", "d"), ("pressure_solver_tol", "pressure_solver_tol", "f"),
    ("pressure_solver_iter", "pressure_solver_iter", "d"), ("pressure_solver_log", "pressure_solver_log", "d"),
    ("z_domain", "z_domain", "d"), ("k_nu_grid", "k_nu_grid", "f"), ("k_transition", "k_transition", "d"),
    ("z_transition", "z_transition", "f"), ("input_path", "input_path", "s"),
    ("velocity_correction_fd", "velocity_correction_fd", "d"), ("time_step_log", "time_step_log", "d"),
    ("temperature_convection", "temperature_convection", "d"),
    ("TS_x_start", "TS_x_start", "f"), ("TS_x_end", "TS_x_end", "f"),
    ("TS_y_start", "TS_y_start", "f"), ("TS_y_end", "TS_y_end", "f"),
    ("TS_z_start", "TS_z_start", "f"), ("TS_z_end", "TS_z_end", "f"),
    ("sutherland_viscosity", "sutherland_viscosity", "d"),
    ("sutherland_conductivity", "sutherland_conductivity", "d"),
]
