// dropin.cu -- the reference's solver entry points (include/wf_dropin.h) on
// the B200 solver's C-ABI.  Built into libwildfires_b200_dropin.a, separate
// from libwildfires_b200.so because it calls back into reference objects the
// caller links (output.o, logs.o, functions.o, utils.o).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <vector>

#include <cuda_runtime.h>

#include "wf_dropin.h"
#include "wildfires_b200.h"

// Defined by the caller's reference objects (logs.cu, utils.cu).
void log_timestep(Parameters parameters, int n, double t_n, double step_time, double CFL, double T_min,
                  double T_max, double Y_min, double Y_max);
void log_message(Parameters parameters, const char *message);
void format_seconds(double seconds, char *formatted_time);

namespace {

[[noreturn]] void fatal(const char *where)
{
    fprintf(stderr, "%s: %s\n", where, wf_last_error());
    exit(1);
}

void check_status(wf_status s, const char *where)
{
    if (s != WF_OK) fatal(where);
}

void check_cuda(cudaError_t e, const char *where)
{
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: %s\n", where, cudaGetErrorString(e));
        exit(1);
    }
}

// The operator entries keep one FP64 context for the last parameter record
// they saw (the reference passes the record by value on every call).  Its work
// goes on the legacy default stream, where the reference launches its kernels,
// so it is ordered with the caller's own default-stream work; the operators
// take the caller's device buffers directly (no host copies).
struct OperatorContext {
    wf_ctx *ctx = nullptr;
    Parameters key;
} g_op;

wf_ctx *context_for(const Parameters &P)
{
    if (g_op.ctx && memcmp(&g_op.key, &P, sizeof(Parameters)) == 0) return g_op.ctx;
    if (g_op.ctx) wf_destroy(g_op.ctx);
    g_op.ctx = nullptr;
    check_status(wf_create(&P, WF_FP64, &g_op.ctx), "wf_create");
    check_status(wf_set_stream(g_op.ctx, (void *)cudaStreamLegacy), "wf_set_stream");
    g_op.key = P;
    return g_op.ctx;
}

void to_host(std::vector<double> &h, const double *d, size_t n)
{
    h.resize(n);
    check_cuda(cudaMemcpy(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost), "device-to-host copy");
}

void to_device(double *d, const std::vector<double> &h)
{
    check_cuda(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice), "host-to-device copy");
}

// RK stages with the method of the entry point called, whatever the record says.
void rk_with(const char *method, double *y_n, double *y_np1, Parameters parameters)
{
    Parameters q = parameters;
    memset(q.method, 0, sizeof(q.method));
    strncpy(q.method, method, sizeof(q.method) - 1);
    check_status(wf_rk_device(context_for(q), y_n, y_np1), method);
}

void pressure_with(double *y_np1, double *y_n, double *p, const Parameters &q, double *error, int *max_iter)
{
    wf_ctx *c = context_for(q);
    check_status(wf_pressure_device(c, y_np1, y_n, p), "solve_pressure");
    if (error || max_iter) check_status(wf_pressure_report(c, error, max_iter), "solve_pressure_iterative");
}

double seconds_between(const timeval &a, const timeval &b)
{
    return ((b.tv_sec - a.tv_sec) * 1000000.0 + (b.tv_usec - a.tv_usec)) / 1.e6;
}

}  // namespace

void create_y_0(double *u, double *v, double *w, double *T, double *Y, double *y_0, Parameters parameters)
{
    const size_t N = (size_t)parameters.Nx * parameters.Ny * parameters.Nz;
    const size_t NY = (size_t)parameters.Nx * parameters.Ny * parameters.Nz_Y_max;
    const FieldIndexes &f = parameters.field_indexes;
    memcpy(y_0 + f.u, u, N * sizeof(double));
    memcpy(y_0 + f.v, v, N * sizeof(double));
    memcpy(y_0 + f.w, w, N * sizeof(double));
    memcpy(y_0 + f.T, T, N * sizeof(double));
    memcpy(y_0 + f.Y, Y, (NY < N ? NY : N) * sizeof(double));
}

void Phi(double t, double *R_old, double *R_new, double *, double *, double *, int *, int *, Parameters parameters)
{
    (void)t;   // the right-hand side has no explicit time dependence (pde.cu:139-787)
    check_status(wf_phi_device(context_for(parameters), R_old, R_new), "Phi");
}

void euler(double, double *y_n, double *y_np1, double *, double *, double *, double *, int *, int *, double, int,
           Parameters parameters)
{
    rk_with("Euler", y_n, y_np1, parameters);
}

void RK2(double, double *y_n, double *y_np1, double *, double *, double *, double *, double *, int *, int *, double,
         int, Parameters parameters)
{
    rk_with("RK2", y_n, y_np1, parameters);
}

void RK4(double, double *y_n, double *y_np1, double *, double *, double *, double *, double *, int *, int *, double,
         int, Parameters parameters)
{
    rk_with("RK4", y_n, y_np1, parameters);
}

void solve_pressure(double *y_np1, double *y_n, double *p, double *, double *, double *, double *, double *,
                    cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *,
                    cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *, int *,
                    Parameters parameters)
{
    // exactly one solve, as the reference's solve_pressure (pressure.cu:506-549)
    Parameters q = parameters;
    q.pressure_solver_iter = 1;
    q.pressure_solver_tol = -1.0;
    pressure_with(y_np1, y_n, p, q, nullptr, nullptr);
}

void solve_pressure_iterative(double *y_np1, double *y_n, double *p, double *, double *, double *, double *,
                              double *, cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *,
                              cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *, cufftDoubleComplex *,
                              cufftDoubleComplex *, int *, Parameters parameters, double *error, int *max_iter)
{
    double e = 0.0;
    int m = 0;
    pressure_with(y_np1, y_n, p, parameters, &e, &m);
    if (parameters.pressure_solver_log == 1) {
        char msg[128];
        snprintf(msg, sizeof(msg), "Pressure solver: Error = %e, iterations = %d", e, m);
        log_message(parameters, msg);
    }
    if (error) *error = e;
    if (max_iter) *max_iter = m;
}

// The time loop of solver.cu:95-265: Nt steps; every NT steps and at the last
// one the state is reported, logged and saved.  The report is the reference's
// timestep_reports computed on the device (wf_timestep_reports: only the
// report crosses to the host) and logged through the reference's own
// log_timestep / log_message, including its NaN message and exit; the save is
// an asynchronous dump in save_data's format (wf_dump_async), written by a
// host thread while the next steps run.  y_n and p hold the final state on
// return.
void solve_PDE(double *y_n, double *p, Parameters parameters)
{
    const char *env = getenv("WF_PRECISION");
    const int prec = (env && strcmp(env, "fp32") == 0) ? WF_FP32_STENCIL : WF_FP64;
    wf_ctx *c = nullptr;
    check_status(wf_create(&parameters, prec, &c), "wf_create");
    const size_t S = wf_state_size(&parameters), N = (size_t)parameters.Nx * parameters.Ny * parameters.Nz;
    std::vector<double> yh, ph;
    to_host(yh, y_n, S);
    to_host(ph, p, N);
    check_status(wf_upload_state(c, yh.data(), ph.data()), "wf_upload_state");

    const int Nt = parameters.Nt, NT = parameters.NT > 0 ? parameters.NT : Nt;
    const int log_every = parameters.time_step_log > 0 ? parameters.time_step_log : Nt + 1;
    double cum_step_time = 0.0, CFL = 0.0, T_min = 1e9, T_max = -1e9, Y_min = 1e9, Y_max = -1e9;
    timeval start_solver, end_solver, t0, t1;
    gettimeofday(&start_solver, nullptr);
    for (int n = 1; n <= Nt; n++) {
        gettimeofday(&t0, nullptr);
        check_status(wf_step(c, 1), "wf_step");
        check_status(wf_synchronize(c), "wf_step");
        gettimeofday(&t1, nullptr);
        const double step_time = seconds_between(t0, t1);
        cum_step_time += step_time;
        if (n % log_every == 0) printf("Time step: %d, Average time: %lf s\n", n, cum_step_time / n);
        if (n % NT == 0 || n == Nt) {
            wf_report rep;
            check_status(wf_timestep_reports(c, &rep), "wf_timestep_reports");
            if (rep.nan_field >= 0) {
                // the message and exit of timestep_reports (functions.cu:137-166)
                const char names[] = "uvwTY";
                char message[256];
                snprintf(message, sizeof(message),
                         "NaN value found in %c(%f, %f, %f, %f) in node (%d, %d, %d) at timestep %d (%d). Exiting...",
                         names[rep.nan_field], parameters.x[rep.nan_i], parameters.y[rep.nan_j],
                         parameters.z[rep.nan_k], parameters.t[n], rep.nan_i, rep.nan_j, rep.nan_k, n, n / NT);
                log_message(parameters, message);
                wf_dump_wait(c);
                exit(1);
            }
            CFL = rep.cfl;
            T_min = rep.T_min;
            T_max = rep.T_max;
            Y_min = rep.Y_min;
            Y_max = rep.Y_max;
            log_timestep(parameters, n, parameters.t[n], step_time, CFL, T_min, T_max, Y_min, Y_max);
            if (parameters.variable_density == 1) {
                double e = 0.0;
                int m = 0;
                check_status(wf_pressure_report(c, &e, &m), "wf_pressure_report");
                char msg[128];
                snprintf(msg, sizeof(msg), "Pressure solver: Error = %e, iterations = %d", e, m);
                log_message(parameters, msg);
            }
            check_status(wf_dump_async(c, parameters.save_path, n / NT), "wf_dump_async");
            printf("\n");
        }
    }
    gettimeofday(&end_solver, nullptr);
    char formatted[64], msg[128];
    format_seconds(seconds_between(start_solver, end_solver), formatted);
    snprintf(msg, sizeof(msg), "\nSolver time: %s", formatted);
    log_message(parameters, msg);
    check_status(wf_dump_wait(c), "wf_dump_wait");
    check_status(wf_download_state(c, yh.data(), ph.data()), "wf_download_state");
    to_device(y_n, yh);
    to_device(p, ph);
    wf_destroy(c);
}
