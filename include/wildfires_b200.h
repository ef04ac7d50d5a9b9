/*
 * wildfires_b200.h -- C-ABI of the B200 coupled atmosphere-wildfire solver.
 *
 * The solver advances the state of the reference model (dsanmartinreyes'
 * wildfires, src/cu) by RK time steps on one NVIDIA B200 with hand-written
 * sm_100a kernels: one fused right-hand-side pass per RK stage, an FP64
 * FFT(x,y) + tridiagonal(z) pressure Poisson solve, and a fused projection /
 * boundary / clamp pass.  All entry points return a wf_status (never exit or
 * assert); a human-readable message for the last failure on the calling host
 * thread is available from wf_last_error().
 *
 * Data conventions are the reference's: a packed state vector holds
 * [u | v | w | T | Y], u..T as Nx*Ny*Nz FP64 values in IDX(i,j,k) =
 * k + Nz*(j + Ny*i) (z fastest; reference include/cu/utils.cuh:18-20), then Y as
 * Nx*Ny*Nz_Y_max values in k + Nz_Y_max*(j + Ny*i).  Pressure p is Nx*Ny*Nz
 * FP64 in the same layout.  The planes i = Nx-1 and j = Ny-1 duplicate planes
 * 0 (period Nx-1, Ny-1).
 *
 * The reference-compatible C++ entry points (solve_PDE, Phi, RK4,
 * solve_pressure, solve_pressure_iterative) are declared in wf_dropin.h.
 */
#ifndef WILDFIRES_B200_H
#define WILDFIRES_B200_H

#include <stddef.h>

#include "wf_parameters.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum wf_status {
    WF_OK = 0,
    WF_ERR_ARG = 1,          /* invalid argument or unsupported configuration */
    WF_ERR_CUDA = 2,         /* CUDA runtime error (message in wf_last_error) */
    WF_ERR_IO = 3,           /* file missing, unreadable or of the wrong size */
    WF_ERR_PARSE = 4,        /* parameter file could not be parsed */
    WF_ERR_OOM = 5,          /* device or host allocation failed */
    WF_ERR_NAN = 6,          /* a NaN was found in the state (diagnostics) */
    WF_ERR_NO_DEVICE = 7     /* no CUDA device of compute capability 10.0 */
} wf_status;

typedef enum wf_precision {
    WF_FP64 = 0,             /* every field and operator in FP64 */
    WF_FP32_STENCIL = 1      /* u,v,w,T,Y stored and advanced in FP32; pressure,
                                divergence and diagnostics in FP64 */
} wf_precision;

typedef struct wf_ctx wf_ctx;

/* Global diagnostics of the current state, reduced on the GPU in FP64. */
typedef struct wf_diag {
    double mass;             /* sum rho dV over interior cells, rho = T_inf rho_inf / T */
    double energy;           /* sum rho c_p T dV */
    double fuel;             /* sum Y dV over stored fuel cells (k < Nz_Y(i,j)) */
    double fuel_consumed;    /* initial fuel minus fuel (since the last upload) */
    double max_abs_u, max_abs_v, max_abs_w;
    double cfl;              /* dt (max|u|/dx + max|v|/dy + max|w|/dz), functions.cu:180 */
    double T_min, T_max;     /* over all cells */
    double Y_min, Y_max;     /* over stored fuel cells */
    long long nan_count;     /* NaN values found in u, v, w, T, Y */
} wf_diag;

/* The reference's per-checkpoint report (timestep_reports, functions.cu:82-185),
 * with its conventions: T and Y ranges only inside the fuel rectangle
 * [Y0_x_start, Y0_x_end] x [Y0_y_start, Y0_y_end], starting from T_min = 1e9,
 * T_max = -1e9, Y_min = 0, Y_max = -1e9; Y read for every k < Nz_Y_max.
 * nan_field is -1, or the field (0 u, 1 v, 2 w, 3 T, 4 Y) of the first NaN in
 * the reference's scan order (i, j, k, then u, v, w, T, Y) at node
 * (nan_i, nan_j, nan_k). */
typedef struct wf_report {
    double cfl;              /* dt (max|u|/dx + max|v|/dy + max|w|/dz) over all cells */
    double Y_min, Y_max, T_min, T_max;
    int nan_field, nan_i, nan_j, nan_k;
} wf_report;

/* ---- parameters --------------------------------------------------------- */

/* Parse a `key = value` parameter file with the reference's rules
 * (src/cu/parameters.cu:39-415: defaults, prefix match, later lines override,
 * unknown keys ignored) and fill the derived arrays (grid, time, wavenumbers,
 * terrain, immersed-boundary tables; parameters.cu:416-523, ibm.cu:3-95).
 * Unlike the reference it creates no output directory and opens no log file.
 * Release with wf_free_parameters. */
wf_status wf_read_parameters(const char *path, Parameters *out);

/* Release the host arrays allocated by wf_read_parameters / wf_set_topography. */
void wf_free_parameters(Parameters *p);

/* Replace the terrain by an explicit Nx*Ny height field (j fastest) and
 * recompute cut_nodes, Nz_Y, Nz_Y_max, z_ibm (ibm.cu:57-95).  Changes the
 * packed-state size when Nz_Y_max changes. */
wf_status wf_set_topography(Parameters *p, const double *topo);

/* The immersed-boundary tables of the record's current topography (cut nodes,
 * Nz_Y, Nz_Y_max, z_ibm; ibm_parameters, ibm.cu:57-95) computed on the current
 * CUDA device and written back into the record's host arrays, bit-identical to
 * wf_set_topography's host computation.  The host arrays stay the record
 * callers may edit afterwards. */
wf_status wf_ibm_parameters_device(Parameters *p);

/* Replace the terrain by n Gaussian hills, hills[4 q .. 4 q + 3] = centre x,
 * centre y, height, width: topography(x, y) = sum_q height exp(-(dx^2 + dy^2)
 * / (2 width^2)), dx and dy the periodic distances to the centre (periods
 * x_max - x_min and y_max - y_min), summed in the order given; evaluated on
 * the current CUDA device with the immersed-boundary tables, both written back
 * into the record.  The seeded multi-hill terrain of the benchmark workloads;
 * the reference's terrains are flat and one hill (simple_hill, ibm.cu:13-28). */
wf_status wf_set_topography_hills(Parameters *p, int n, const double *hills);

/* Number of FP64 values in a packed state vector: 4*Nx*Ny*Nz + Nx*Ny*Nz_Y_max. */
size_t wf_state_size(const Parameters *p);

/* Read an initial state from `<dir>u.bin, v.bin, w.bin, T.bin, Y.bin, p.bin`
 * (input.cu:3-58) into a packed host state y (wf_state_size values) and p
 * (Nx*Ny*Nz values). */
wf_status wf_load_fields(const Parameters *p, const char *dir, double *y, double *pr);

/* Write a packed host state and p as `<dir>u.bin.<n>` ... `p.bin.<n>` in the
 * reference's raw FP64 format (output.cu:3-44). */
wf_status wf_save_fields(const Parameters *p, const char *dir, int n, const double *y, const double *pr);

/* save_domain (output.cu:46-81): `<dir>x.bin`, `y.bin`, `z.bin` (FP64 grid
 * coordinates) and `t.bin` (the times of the saved steps, n % NT == 0 or
 * n == Nt, for n = 0..Nt). */
wf_status wf_save_domain(const Parameters *p, const char *dir);

/* save_topography (output.cu:83-99): `<dir>topography.bin` (FP64, Nx*Ny, j
 * fastest) and `<dir>Nz_Y.bin` (int32, Nx*Ny). */
wf_status wf_save_topography(const Parameters *p, const char *dir);

/* ---- solver context ----------------------------------------------------- */

/* Create a solver on the current CUDA device for the given record (copied;
 * the record's host arrays are read once).  Allocates all device memory the
 * time loop needs; nothing is allocated afterwards. */
wf_status wf_create(const Parameters *p, int precision, wf_ctx **out);
wf_status wf_destroy(wf_ctx *ctx);

/* Upload a packed FP64 host state and p (the time level becomes 0). */
wf_status wf_upload_state(wf_ctx *ctx, const double *y, const double *pr);

/* The same upload, returning once the state is on the device while p's copy
 * continues on a stream of its own: the next wf_step waits for it only before
 * its pressure solve (which reads p's top plane), so the copy overlaps the RK
 * stages; every other call that reads or writes p (download, dumps, pressure
 * operators, wf_device_state, wf_synchronize) first waits for it.  The host
 * buffer pr must stay unchanged until the following step has completed or one
 * of those calls has returned.  Counterpart of the reference's host-to-device
 * copies before solve_PDE (main.cu:71-72), which block. */
wf_status wf_upload_state_async(wf_ctx *ctx, const double *y, const double *pr);
/* Download the current packed state and p as FP64. */
wf_status wf_download_state(wf_ctx *ctx, double *y, double *pr);

/* The reference's initial conditions (initial_conditions + create_y_0,
 * functions.cu:187-323, solver.cu:41-56) generated on the device straight
 * into the context's state and p: no host fields, no upload.  The time level
 * becomes 0.  T0_shape must be "gaussian" or "parallelepiped" (the reference
 * leaves T unset otherwise); Y entries the reference leaves unwritten are 0. */
wf_status wf_initial_conditions(wf_ctx *ctx);

/* Advance nsteps time steps (RK stages, pressure solve, projection, boundary
 * rules, clamps, temperature source).  Enqueued on the context's stream; the
 * first call records the step into a CUDA graph that later calls replay. */
wf_status wf_step(wf_ctx *ctx, int nsteps);
wf_status wf_synchronize(wf_ctx *ctx);

/* Tile shape of the fused stage pass: TI x TJ columns of 8 planes, processed
 * by `threads` threads per block.  The first wf_step of a context picks it:
 * WF_STAGE_TILE=TIxTJ[/threads] in the environment forces one, otherwise each
 * compiled form (FP32: 8x16/512, 8x16/384, 8x8/256; FP64: 8x8/512, 8x8/256) is timed on
 * the context's own grid and state and the fastest is kept.  All forms give
 * bit-identical results.  wf_set_stage_tile forces a form (threads <= 0: the
 * first with that TI x TJ; call it before stepping; WF_ERR_ARG for a form that
 * is not compiled).  threads may be NULL in wf_stage_tile.  The tiling is a
 * property of this implementation; the reference has no counterpart. */
wf_status wf_stage_tile(const wf_ctx *ctx, int *ti, int *tj, int *threads);
wf_status wf_set_stage_tile(wf_ctx *ctx, int ti, int tj, int threads);

/* Current time level n and time t[n]. */
wf_status wf_time(const wf_ctx *ctx, int *n, double *t);

/* FP64 diagnostics of the current state. */
wf_status wf_diagnostics(wf_ctx *ctx, wf_diag *out);

/* timestep_reports (functions.cu:82-185) of the current state, reduced on the
 * device: only the report crosses to the host, not the state.  The reference
 * logs the first NaN and exits; this call reports it (see wf_report) and
 * returns WF_OK. */
wf_status wf_timestep_reports(wf_ctx *ctx, wf_report *out);

/* Asynchronous checkpoint of the current state and p as `<dir>u.bin.<n>` ...
 * `<dir>p.bin.<n>` in the format of save_data (output.cu:3-44; FP64, also for
 * the FP32 stencil state).  Enqueues one device-to-device snapshot on the
 * context's stream and returns; the copy to pinned host memory and the file
 * writes run in the background while later steps run (solver.cu:248-250 copies
 * and writes before continuing).  Two host buffers: a dump issued while two are
 * still being written waits for the older one.  The first call allocates the
 * snapshot (state + p in FP64) and the two pinned host buffers; they are kept
 * until wf_destroy.  Write errors are returned by the next wf_dump_wait. */
wf_status wf_dump_async(wf_ctx *ctx, const char *dir, int n);

/* Wait until every dump of the context is written; returns the first error of
 * those writes, or WF_OK. */
wf_status wf_dump_wait(wf_ctx *ctx);

/* Device pointers of the current state (precision-dependent element type:
 * double for WF_FP64, float for WF_FP32_STENCIL) and of p (double).  Valid
 * until the next wf_step. */
wf_status wf_device_state(wf_ctx *ctx, void **y, double **pr);
/* The CUDA stream (cudaStream_t) the context enqueues on. */
void *wf_stream(wf_ctx *ctx);
/* Enqueue the context's work on the caller's stream (a cudaStream_t; NULL:
 * the context's own stream again), so that it orders with the caller's own
 * kernels without host synchronisation.  Work already enqueued on the previous
 * stream comes first.  Step graphs are still captured on the context's own
 * stream and launched on this one, so any stream may be given, the legacy
 * default stream (cudaStreamLegacy) included.  Not for ensemble members
 * (WF_ERR_ARG).  The reference runs everything on the default stream and
 * synchronises after every launch (solver.cu:178-265). */
wf_status wf_set_stream(wf_ctx *ctx, void *stream);

/* ---- learned subgrid closure (no reference counterpart) ------------------- */

/* The Smagorinsky eddy viscosity mu_sgs = rho C_s^2 Delta^2 |S| (pde.cu:745)
 * or a learned local coefficient in place of C_s^2: an MLP 12 -> 64 -> 64 -> 1
 * (GELU, softplus output) of the resolved strain rate, vorticity and grad T,
 * evaluated for every cell before each RK stage on BF16 tensor cores with
 * FP32 accumulation. */
#define WF_CLOSURE_SMAGORINSKY 0
#define WF_CLOSURE_MLP 1
/* Number of floats in a closure parameter vector: W1[64][12], b1[64],
 * W2[64][64], b2[64], W3[64], b3, then 12 feature scales. */
int wf_closure_param_count(void);
/* Select the closure of a context; params (host, wf_closure_param_count()
 * floats) is copied.  WF_CLOSURE_SMAGORINSKY ignores params. */
wf_status wf_set_closure(wf_ctx *ctx, int kind, const float *params);
/* The learned coefficient of every cell of a packed host state (N values). */
wf_status wf_closure_coefficients(wf_ctx *ctx, const double *y, double *coef);
/* The learned coefficient softplus(MLP(x)) of n rows of the 12 raw features
 * (strain rate, vorticity, grad T in the closure's feature order, before the
 * per-feature scales of params), evaluated on the current device by the same
 * BF16 tensor-core kernel the solver runs before each stage; host buffers
 * (features: n x 12 row-major, out: n values).  For evaluating a network on
 * data other than a solver state. */
wf_status wf_closure_predict(const float *params, const float *features, size_t n, float *out);
/* Polls of each bounded tensor-core completion wait of the context's closure
 * inference (default 4194304).  When a wait runs out the kernel gives the
 * matrix operations in flight their full drain limit, frees its tensor memory
 * and raises an error flag; the next wf_synchronize or wf_closure_coefficients
 * returns WF_ERR_CUDA once and clears it.  A small limit exercises that path. */
wf_status wf_set_closure_wait_limit(wf_ctx *ctx, int polls);
/* Training on the current device with the library's own kernels.  x: n x 12
 * normalised features (row-major), y: n target coefficients.  Loss: mean
 * squared error of softplus(MLP(x)) against y. */
wf_status wf_mlp_loss_grad(const float *theta, const float *x, const float *y, size_t n, double *loss, float *grad);
/* steps Adam steps (lr, beta 0.9 / 0.999) on minibatches of a seeded
 * permutation per epoch; theta is updated in place (feature scales kept);
 * loss_history (steps values, may be NULL) receives each batch's loss. */
wf_status wf_mlp_train(float *theta, const float *x, const float *y, size_t n, int steps, int batch, float lr,
                       unsigned long long seed, double *loss_history);

/* ---- ensembles of independent members ------------------------------------ */

/* An ensemble steps independent members (their own grids, terrain, wind,
 * ignition, fuel) together: each ensemble step is one CUDA graph whose
 * branches are the members' steps, run concurrently on the GPU.  There is no
 * reference counterpart (the reference runs one scenario per process). */
typedef struct wf_ensemble wf_ensemble;

/* Create one member context per record of members[0 .. n_members). */
wf_status wf_ensemble_create(const Parameters *members, int n_members, int precision, wf_ensemble **out);
wf_status wf_ensemble_destroy(wf_ensemble *e);
int wf_ensemble_size(const wf_ensemble *e);
/* The CUDA stream (cudaStream_t) an ensemble step is launched on: work
 * recorded on it after wf_ensemble_step follows every member's step. */
void *wf_ensemble_stream(wf_ensemble *e);
/* Member i as a context: upload, download and diagnose it with the wf_ctx
 * calls; owned by the ensemble (do not destroy it). */
wf_ctx *wf_ensemble_member(wf_ensemble *e, int i);
/* Advance every member nsteps steps. */
wf_status wf_ensemble_step(wf_ensemble *e, int nsteps);
wf_status wf_ensemble_synchronize(wf_ensemble *e);

/* ---- operator-level entry points (used by the parity tests) ------------- */

/* One right-hand-side evaluation R_new = Phi(R_old) on host buffers (packed
 * state layout) -- RHS, SGS terms and boundary rules (pde.cu:910-917). */
wf_status wf_phi(wf_ctx *ctx, const double *R_old, double *R_new);

/* One pressure solve on host buffers: p is read (top plane, and the previous
 * iterate for variable density) and overwritten (pressure.cu:506-606).
 * Returns the number of solves in *iters (may be NULL). */
wf_status wf_pressure(wf_ctx *ctx, const double *y_np1, const double *y_n, double *pr, int *iters);

/* The RK stages of one step without the pressure solve and the projection
 * (RK4 / RK2 / euler, solver.cu:59-93): y_np1 from y_n on host buffers. */
wf_status wf_rk(wf_ctx *ctx, const double *y_n, double *y_np1);

/* The same three operators on DEVICE buffers (packed FP64 state and FP64 p in
 * the reference's layout), enqueued on the context's stream with no host copy
 * and no host synchronisation: what the reference's own Phi, RK4 and
 * solve_pressure do with the device pointers they are given (pde.cu:910-917,
 * solver.cu:76-93, pressure.cu:506-549).  wf_pressure_device writes p in place;
 * its iteration count is read by wf_pressure_report. */
wf_status wf_phi_device(wf_ctx *ctx, const double *R_old, double *R_new);
wf_status wf_rk_device(wf_ctx *ctx, const double *y_n, double *y_np1);
wf_status wf_pressure_device(wf_ctx *ctx, const double *y_np1, const double *y_n, double *pr);

/* What solve_pressure_iterative reports after the last wf_pressure or step
 * (pressure.cu:596-597): the max-norm change of the last iterate and the
 * iteration count in the reference's convention (the index of the converged
 * iterate, or pressure_solver_iter).  The variable-density loop runs on the
 * device; this call waits for the context's stream and reads its record. */
wf_status wf_pressure_report(const wf_ctx *ctx, double *error, int *max_iter);

/* The operator-level entries above use the context's state buffers as
 * scratch: after them, upload a state before calling wf_step again. */

/* Number of kernel launches one wf_step(ctx, 1) enqueues. */
int wf_launches_per_step(const wf_ctx *ctx);

/* Kinds of kernels in a step, for wf_profile_phases. */
#define WF_NPHASES 9
/* Advance nsteps steps with the kernels launched one by one (no graph) and a
 * CUDA event recorded after each kernel on the context's stream.  For every
 * kernel kind q < WF_NPHASES, ms[q] receives the summed device time and
 * launches[q] the number of launches.  Variable density: pressure_solver_iter
 * solves per step without the tolerance test, the per-step part of the source
 * counted in the first solve's source kernel.  Returns WF_OK or an error
 * status. */
wf_status wf_profile_phases(wf_ctx *ctx, int nsteps, double *ms, int *launches);
/* Name of kernel kind q ("stage_fused", "p_fftx_fwd", ...), or NULL. */
const char *wf_phase_name(int q);

/* ---- pressure solve without device allocation --------------------------- */

/* One FP64 constant-density pressure solve on DEVICE buffers that performs no
 * device memory allocation.  This entry point has no counterpart in the
 * reference; it exists for callers that cannot call cudaMalloc -- code running
 * inside a framework that owns all device memory through its own pool, code
 * with a device-memory budget fixed in advance, or code that must not pay for
 * an allocation on its time-critical path.
 *
 * y_np1: packed FP64 state on the device (u, v, w are read); p: Nx*Ny*Nz FP64
 * pressure on the device, read (top plane) and overwritten exactly as by
 * wf_pressure.  stream: a cudaStream_t (NULL for the legacy default stream).
 *
 * All scratch -- the half-spectrum buffer, FFT and tridiagonal tables, grid --
 * lives in one fixed device array of 64 MiB inside this library; every device
 * that loads the library holds that array until the process exits.  The
 * half-spectrum buffer dominates: Nz*(Nx-1)*((Ny-1)/2+1) 16-byte cells, so a
 * 128 x 128 x 64 grid needs 8 MiB, 257 x 257 x 64 needs 33 MiB, and
 * 512 x 512 x 128 does not fit; grids that do not fit are rejected with
 * WF_ERR_ARG and a message naming the size, before any CUDA call.  Only
 * variable_density = 0 is accepted.  The first call on a device looks up the
 * array's device address and configures the kernels; make that first call
 * before any stream capture.  The FFT, wavenumber and tridiagonal tables stay
 * in the array from one call to the next: a call on the same grid as the
 * previous call on that device (same Nx, Ny, Nz, z, kx, ky) only enqueues the
 * solve and returns; a call on another grid first rebuilds the tables on the
 * host, copies them into the array and waits for that copy on the stream.
 * Every call on a device shares the one array and keeps what the previous
 * call left in it, so calls whose GPU work overlaps race -- on one stream or
 * several, from one host thread or several; issue them one after another.
 * The host side of concurrent calls (set-up, table rebuild) is serialised by a
 * lock.  Nothing in the array needs to start at zero: each call writes every
 * element it reads before reading it. */
wf_status wf_pressure_noalloc(const Parameters *p, const double *y_np1, double *pr, void *stream);

/* Failure injection for tests of the error paths: after `after` more device
 * allocations by contexts (wf_create, wf_set_closure, dumps) succeed, the
 * next one is refused with WF_ERR_OOM as if the device were full; then
 * injection switches itself off.  Negative: off.  No counterpart in the
 * reference (it asserts on CUDA errors, utils.cuh:124-130). */
void wf_inject_allocation_failure(int after);

const char *wf_status_string(wf_status s);
const char *wf_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
