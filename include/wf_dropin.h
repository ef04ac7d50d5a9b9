/*
 * wf_dropin.h -- the reference's solver entry points, with C++ linkage and
 * the reference's exact signatures, implemented on the B200 solver.
 *
 * A program built against the reference (dsanmartinreyes' wildfires, src/cu)
 * links libwildfires_b200_dropin.a and libwildfires_b200.so IN PLACE OF the
 * reference objects solver.o, pde.o, turbulence.o and pressure.o; its main.o,
 * parameters.o, ibm.o, functions.o, input.o, output.o, logs.o and utils.o link
 * unchanged, and the drop-in calls back into them for what solve_PDE does
 * besides the time step (timestep_reports, log_timestep, log_message,
 * save_data, format_seconds).
 *
 * Semantics follow the reference (void return; a fatal error prints a message
 * and exits, as the reference's own checks do).  All pointers are DEVICE
 * pointers, as in the reference.  The buffer arguments the reference needs as
 * scratch (k, F, R_turbulence, gamma, a, b, c, d, l, u, y, data_in, data_out,
 * p_top_in, p_top_out, z, z_ibm, Nz_Y, cut_nodes) are accepted and not used:
 * the B200 solver keeps its own device state per parameter record.
 *
 * Precision: FP64 by default, as the reference; the environment variable
 * WF_PRECISION=fp32 selects the FP32 stencil path for solve_PDE.
 */
#ifndef WF_DROPIN_H
#define WF_DROPIN_H

#include <cuComplex.h>

#include "wf_parameters.h"

typedef cuDoubleComplex cufftDoubleComplex;

/* solver.cu:41, solver.cuh:85 -- packs host fields into the state vector
 * [u | v | w | T | Y] at the record's field offsets (Y: its first
 * Nx*Ny*Nz_Y_max values). */
void create_y_0(double *u, double *v, double *w, double *T, double *Y, double *y_0, Parameters parameters);

/* solver.cu:95, solver.cuh:149 */
void solve_PDE(double *y_n, double *p, Parameters parameters);

/* pde.cu:910 */
void Phi(double t, double *R_old, double *R_new, double *R_turbulence, double *z, double *z_ibm, int *Nz_Y,
         int *cut_nodes, Parameters parameters);

/* solver.cu:59, 65, 76 (solver.cuh:102, 120, 138) */
void euler(double t_n, double *y_n, double *y_np1, double *F, double *U_turbulence, double *z, double *z_ibm,
           int *Nz_Y, int *cut_nodes, double dt, int size, Parameters parameters);
void RK2(double t_n, double *y_n, double *y_np1, double *k, double *F, double *U_turbulence, double *z,
         double *z_ibm, int *Nz_Y, int *cut_nodes, double dt, int size, Parameters parameters);
void RK4(double t_n, double *y_n, double *y_np1, double *k, double *F, double *U_turbulence, double *z,
         double *z_ibm, int *Nz_Y, int *cut_nodes, double dt, int size, Parameters parameters);

/* pressure.cu:506, 551 (pressure.cuh:80, 82) */
void solve_pressure(double *y_np1, double *y_n, double *p, double *z, double *gamma, double *a, double *b,
                    double *c, cufftDoubleComplex *d, cufftDoubleComplex *l, cufftDoubleComplex *u,
                    cufftDoubleComplex *y, cufftDoubleComplex *data_in, cufftDoubleComplex *data_out,
                    cufftDoubleComplex *p_top_in, cufftDoubleComplex *p_top_out, int *Nz_Y,
                    Parameters parameters);
void solve_pressure_iterative(double *y_np1, double *y_n, double *p, double *z, double *gamma, double *a,
                              double *b, double *c, cufftDoubleComplex *d, cufftDoubleComplex *l,
                              cufftDoubleComplex *u, cufftDoubleComplex *y, cufftDoubleComplex *data_in,
                              cufftDoubleComplex *data_out, cufftDoubleComplex *p_top_in,
                              cufftDoubleComplex *p_top_out, int *Nz_Y, Parameters parameters, double *error,
                              int *max_iter);

#endif
