/*
 * wf_oracle.h -- CPU restatement (FP64) of the reference's coupled
 * atmosphere-wildfire time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the GPU kernels are compared
 * against.  It is called from tests/, from __graft_entry__.smoke() and from
 * bench.py's CPU-baseline leg, never from the product library.
 *
 * Every routine restates the arithmetic of a reference routine in plain C and
 * names the reference file:line it follows.  Layouts are the reference's:
 * state = packed [u | v | w | T | Y], u..T of N = Nx*Ny*Nz values each in
 * IDX(i,j,k) = k + Nz*(j + Ny*i); Y of Nx*Ny*Nz_Y_max values in
 * k + Nz_Y_max*(j + Ny*i).  The host arrays z, z_ibm, Nz_Y, cut_nodes, kx, ky
 * inside Parameters are used as filled by the parameter parser.
 *
 * Deliberate, documented differences from the reference (all inert for the
 * parity inputs):
 *   - the convective heat-transfer coefficient h_c is evaluated per cell from
 *     the parameter value (the reference overwrites its per-thread copy,
 *     src/cu/pde.cu:698, making the product depend on the launch shape);
 *   - Y right-hand sides above a column's fuel top are written as 0 (the
 *     reference leaves them unwritten, src/cu/pde.cu:670-675);
 *   - the periodic copy of the pressure planes i=Nx-1, j=Ny-1 uses the values
 *     of the current solve (racy in src/cu/pressure.cu:409-414);
 *   - the pressure fixed-point loop stops on a true max-norm (the reference's
 *     norm kernel races, src/cu/functions.cu:431-450).
 */
#ifndef WF_ORACLE_H
#define WF_ORACLE_H

#include "../include/wf_parameters.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of doubles in a packed state vector: 4*Nx*Ny*Nz + Nx*Ny*Nz_Y_max. */
size_t wfo_state_size(const Parameters *P);

/* One right-hand-side evaluation R_new = Phi(R_old): RHS + Smagorinsky SGS
 * terms + boundary/IBM rules (src/cu/pde.cu:910-917). */
void wfo_phi(const Parameters *P, const double *R_old, double *R_new);

/* Classic RK4 combination y_np1 = y_n + dt/6 (k1 + 2 k2 + 2 k3 + k4)
 * (src/cu/solver.cu:76-93).  method "Euler" and "RK2" follow :59 and :65. */
void wfo_time_integrate(const Parameters *P, double t_n, const double *y_n, double *y_np1);

/* Pressure Poisson solve (src/cu/pressure.cu:506-549; iterative variable
 * density loop :551-606).  p is updated in place.  Returns the number of
 * solves performed; *err receives the last max-norm change (0 when constant
 * density). */
int wfo_solve_pressure(const Parameters *P, const double *y_np1, const double *y_n,
                       double *p, double *err);

/* Projection u -= dt grad(p)/rho, state boundary rules and clamps
 * (src/cu/solver.cu:205-215; pde.cu:789-908, 14-99, 101-137). */
void wfo_project(const Parameters *P, double *y_np1, const double *y_n, const double *p);

/* Temperature source applied after projection when t_n1 <= t_source_end
 * (src/cu/solver.cu:217-223; functions.cu:325-403).  T_source_field is the
 * initial temperature field (used when t_source_start <= 0). */
void wfo_temperature_source(const Parameters *P, double *y_np1, double t_n1,
                            const double *T_source_field);

/* One full time step n -> n+1 (n >= 1 is the index of the new time level,
 * matching t[n] in solve_PDE).  y and p are updated in place. */
int wfo_step(const Parameters *P, double *y, double *p, int n, const double *T_source_field);

/* Parameter-file helpers used by the tests: fill derived arrays (x,y,z,t,kx,
 * ky, topography, cut_nodes, z_ibm, Nz_Y, offsets) of a Parameters record
 * whose scalar members are set (restates src/cu/parameters.cu:416-523 and
 * src/cu/ibm.cu:3-95).  topo may be NULL (topo_shape rules) or an explicit
 * Nx*Ny terrain height array. */
int wfo_fill_derived(Parameters *P, const double *topo);
void wfo_free_derived(Parameters *P);

#ifdef __cplusplus
}
#endif

#endif
