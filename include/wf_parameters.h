/*
 * wf_parameters.h -- the run-description record shared by the solver, the
 * parameter-file parser and every caller of the solver entry points.
 *
 * The record is passed BY VALUE to the reference's solver entry points
 * (solve_PDE, Phi, RK4, solve_pressure; reference src/cu/solver.cu:95,
 * src/cu/pde.cu:910, src/cu/solver.cu:76, src/cu/pressure.cu:506).  A caller
 * compiled against the reference header include/c/structures.h:108-259 must
 * be able to hand its record to this library unchanged, so the member list,
 * member types and member order below are fixed by that header: the record is
 * laid out byte-for-byte like the reference's `Parameters`, and the struct tag
 * `_parameters` is kept so that C++ callers link against the same mangled
 * names.  Everything else in this library is independent of that header.
 *
 * Host pointers inside the record (x, y, z, t, r, s, kx, ky, topography,
 * cut_nodes, z_ibm, Nz_Y) are owned by whoever filled the record
 * (wf_read_parameters or the reference parser) and are only read here.
 */
#ifndef WF_PARAMETERS_H
#define WF_PARAMETERS_H

#include <stddef.h>
#include <stdio.h>

/* Offsets (in elements) of the five packed fields u|v|w|T|Y in a state vector. */
typedef struct _field_indexes {
    int u, v, w, T, Y;
} FieldIndexes;

/* Offsets of the three velocity-gradient planes (unused by the solver). */
typedef struct _pressure_indexes {
    int ux, vy, wz;
} PressureIndexes;

/* Offsets of the reference's 18-field turbulence scratch layout.  This
 * library keeps no such scratch array; the offsets are carried only so the
 * record keeps its size and member order. */
typedef struct _turbulence_indexes {
    int rho;
    int Tx, Ty, Tz;
    int Txx, Tyy, Tzz;
    int mu_sgs;
    int S_11, S_12, S_13;
    int S_21, S_22, S_23;
    int S_31, S_32, S_33;
    int div_U;
    int u_tau_wall;
} TurbulenceIndexes;

/* Log files opened by the parser (parameters.txt and log.txt). */
typedef struct _log_files {
    FILE *parameters;
    FILE *log;
} LogFiles;

typedef struct _parameters {
    /* grid sizes: nodes in x, y, z; number of time steps; save interval */
    int Nx, Ny, Nz, Nt, NT;
    /* physical box and time interval */
    double x_min, x_max, y_min, y_max, z_min, z_max, t_min, t_max;
    /* uniform spacings (dz is the nominal spacing; z[] holds the real nodes) */
    double dx, dy, dz, dt;
    /* host coordinate arrays: x[Nx], y[Ny], z[Nz], t[Nt+1], r/s = FFT
     * frequency indices, kx[Nx-1]/ky[Ny-1] = angular wavenumbers */
    double *x, *y, *z, *t, *r, *s, *kx, *ky;
    /* gas properties */
    double c_p, c_v, rho_inf, mu, k, alpha, delta, nu, T_inf, g;
    /* turbulence and drag */
    double C_s, Pr, C_d, alpha_s, sigma_s;
    /* combustion */
    double T_pc, H_C, A, E_A, T_act, h_c, Y_D, Y_f, T_0, T_source, Y_h;
    int k_Y_h;
    /* fuel storage: Y is stored for k < Nz_Y_max only; Nz_Y[Nx*Ny] per column */
    int Nz_Y_max;
    int *Nz_Y;
    /* clamps applied after every step */
    double T_min, T_max, Y_min, Y_max;
    /* initial wind profile */
    char U0_type[32];
    double u_z0, d, u_ast, u_r, z_r, alpha_u;
    /* initial temperature blob */
    char T0_shape[32];
    double T0_x_start, T0_x_end, T0_x_center, T0_length;
    double T0_y_start, T0_y_end, T0_y_center, T0_width;
    double T0_z_start, T0_z_end, T0_z_center, T0_height;
    /* initial fuel box */
    double Y0_x_start, Y0_x_end, Y0_y_start, Y0_y_end, Y0_xa, Y0_ya;
    /* terrain */
    char topo_shape[32];
    double *topography;
    double hill_center_x, hill_center_y, hill_length, hill_width, hill_height;
    /* temperature source held during [t_source_start, t_source_end] */
    char T_source_shape[32];
    double t_source_start, t_source_end;
    double TS_x_start, TS_x_end, TS_x_center, TS_length;
    double TS_y_start, TS_y_end, TS_y_center, TS_width;
    double TS_z_start, TS_z_end, TS_z_center, TS_height;
    /* immersed boundary: cut node per column, height above terrain per node */
    int *cut_nodes;
    double *z_ibm;
    /* Dirichlet pressure at the top plane and the values forced below terrain */
    double p_top;
    double u_dead_nodes, v_dead_nodes, w_dead_nodes, T_dead_nodes, Y_dead_nodes;
    /* pressure solver controls */
    int variable_density;
    double pressure_solver_tol;
    int pressure_solver_iter;
    int pressure_solver_log;
    /* run bookkeeping */
    char method[32];
    char save_path[64];
    char input_path[64];
    char sim_id[32];
    int n_threads;
    /* z grid kind (0 uniform, 1 exponential, 2 two-zone) and its knobs */
    int z_domain;
    double k_nu_grid;
    int k_transition;
    double z_transition;
    /* scheme switches */
    int velocity_correction_fd;
    int time_step_log;
    int temperature_convection;
    int sutherland_viscosity;
    int sutherland_conductivity;
    size_t threads_per_block;
    size_t number_of_blocks;
    FieldIndexes field_indexes;
    TurbulenceIndexes turbulence_indexes;
    PressureIndexes pressure_indexes;
    LogFiles log_files;
} Parameters;

#endif /* WF_PARAMETERS_H */
