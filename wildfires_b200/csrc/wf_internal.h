// wf_internal.h -- definitions shared by the host code and the CUDA kernels of
// the B200 solver.  Not part of the public interface.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "../../include/wildfires_b200.h"

namespace wf {

// Records a formatted message for wf_last_error() on this host thread.
void set_error(const char *fmt, ...);

// NVTX range around a host entry point, for timelines of profilers (no effect
// unless a tool is attached).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

#define WF_TRY_CUDA(call)                                                                  \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            ::wf::set_error("%s:%d: %s failed: %s", __FILE__, __LINE__, #call,             \
                            cudaGetErrorString(e_));                                       \
            return WF_ERR_CUDA;                                                            \
        }                                                                                  \
    } while (0)

// Per-k z-stencil weights on the non-uniform grid, one row of Nz doubles per
// entry.  They are the reference's finite-difference formulas with the
// division folded into a weight (src/cu/pde.cu:363-576, turbulence.cu:344-427).
enum ZCoef {
    ZF0, ZF1, ZF2,          // forward 1st derivative at k: weights of k, k+1, k+2  (k <= Nz-3)
    ZB0, ZB1, ZB2,          // backward 1st derivative at k: weights of k-2, k-1, k (k >= 2)
    ZC,                     // 1 / (dz_{k-1} + dz_k)                                (0 < k < Nz-1)
    ZCM, ZC0, ZCP,          // central 2nd derivative: weights of k-1, k, k+1       (0 < k < Nz-1)
    ZFF0, ZFF1, ZFF2, ZFF3, // forward 2nd derivative at k = 0: weights of 0..3
    ZBB0, ZBB1, ZBB2, ZBB3, // backward 2nd derivative at k = Nz-1: weights of Nz-4..Nz-1
    ZDZ,                    // dz_k = z[k+1]-z[k] (k < Nz-1), z[k]-z[k-1] at the top
    ZDELTA2,                // (C_s (dx dy dz_k)^(1/3))^2, the Smagorinsky length squared
    ZCOUNT
};

// Scalars of the model used on the device (reference Parameters members).
struct Phys {
    double dx, dy, dt;
    double mu, kT, Y_f, H_C, A, T_act, T_pc, h_c, alpha_s, sigma_s;
    double T_inf, c_p, rho_inf, C_d, g, delta, Pr;
    double T_min, T_max, Y_min, Y_max;
    double u_dead, v_dead, w_dead, T_dead, Y_dead;
    int temperature_convection, sutherland_viscosity, sutherland_conductivity;
    int variable_density, velocity_correction_fd;
    // top-plane extrapolation f_{Nz-1} = top_w1 f_{Nz-2} - top_w2 f_{Nz-3} (FP32 projection path)
    double top_w1, top_w2;
};

// Model scalars in the stencil precision R, derived once on the host from
// Phys so kernels do no double->R conversions.
template <class R> struct PhysR {
    R inv2dx, inv2dy, invdx2, invdy2;   // 1/(2 dx), 1/(2 dy), 1/dx^2, 1/dy^2
    R Trho;                             // T_inf rho_inf (rho = Trho / T)
    R mu, kT, Y_f, H_C, A, T_act, T_pc, h_c, alpha_s, sigma_s;
    R T_inf, c_p, rho_inf, cd, g, c12, c4, Pr, inv_avd;
    R T_min, T_max, Y_min, Y_max;
    R mu_Trho, inv_Trho_cp, H_C_cp;     // mu/(T_inf rho_inf), 1/(T_inf rho_inf c_p), H_C/c_p
};

// Per-k row of z-stencil weights in the stencil precision (branch-free
// interior stencils; one row per k, KROW entries).
enum KRow {
    RKM = 0,    // 5 weights (k-2..k+2) of the upwind derivative "from below"
    RKP = 5,    // 5 weights (k-2..k+2) of the upwind derivative "from above"
    RD1 = 10,   // 1/(dz_{k-1} + dz_k): central first derivative (f_{k+1} - f_{k-1}) * RD1
    RD2 = 11,   // 3 weights (k-1..k+1) of the central second derivative
    RDZ = 14,   // dz_k
    RDEL2 = 15, // Smagorinsky length squared
    RZ = 16,    // z_k
    RDD2 = 17,  // (dx dy dz_k)^(2/3): the filter width squared (learned closure)
    KROW = 20
};

// Grid geometry and immersed-boundary tables (device pointers).
struct Geom {
    int Nx, Ny, Nz, NzY;        // NzY = Nz_Y_max
    int N;                      // Nx*Ny*Nz
    int NY;                     // Nx*Ny*NzY
    const double *z;            // [Nz]
    const double *zc;           // [ZCOUNT][Nz]
    const double *topo;         // [Nx*Ny] terrain height (z_ibm = max(z_k - topo, 0))
    const int *nzy;             // [Nx*Ny] fuel-storage height per column
    const int *cut;             // [Nx*Ny] cut node per column
};

// Per-column values the boundary pass needs from the stage pass:
// T,Y at cut+1, cut+2 (4) and u,v,w,T at Nz-2, Nz-3 (8).
constexpr int kBcSlots = 12;

template <class R>
struct StageArgs {
    Geom g;
    Phys ph;
    PhysR<R> pr;
    const R *krow;   // [Nz][KROW] z-stencil weights in precision R
    const R *X;      // stage input state (packed)
    const R *yn;     // state at the start of the step (packed)
    R *acc;          // RK accumulator of k-values (packed)
    R *Xout;         // next stage input, or y_{n+1} after the last stage
    R *utau;         // [Nx*Ny] wall friction velocity from the k = 0 plane
    R *bc;           // [Nx*Ny][kBcSlots]
    double a_next;   // c_{s+1} dt of the next stage input, or dt/6 after the last stage
    double a_prev;   // Euler/RK2 weights (see stage.cu)
    int method;      // 0 Euler, 1 RK2, 2 RK4, 3 = store k_s itself (operator tests)
    int stage;       // 1-based stage index
    // learned closure (closure.cu): when coef is set, mu_sgs = rho coef Delta^2 |S|
    R *coef;               // [N] coefficient of the stage input, written before the stage
    const float *theta;    // closure parameters on the device
    int *closure_err;      // set by the closure kernel when a tensor-core wait times out
    int closure_wait;      // polls of each tensor-core completion wait
    const int *bcfix;      // columns whose cut node or top the fused pass leaves to k_stage_bc
    int nbcfix;
    int tile;              // tile shape of the fused pass (index into the compiled shapes)
    // FP32: host copies of the TMA tensor maps (CUtensorMap) of X for the tile
    // boxes of 16-column and 8-column tiles, or nullptr (tiles loaded by cp.async)
    const void *tmap[2];
    // FP32: host copies of the tensor maps of yn and acc for the boxes of the tile's
    // own cells (16- and 8-column tiles), or nullptr: the stage kernel prefetches
    // its RK operands into L2 with them while it loads and evaluates its tile
    const void *pmap_yn[2], *pmap_acc[2];
    int *kerr;             // set by a stage kernel whose bounded wait for its tile gave up
};

// Learned closure (closure.cu).
int closure_param_count();
constexpr int kClosureWaitLimit = 1 << 22;   // polls of a tensor-core completion wait before it gives up
template <class R>
cudaError_t launch_closure_coef_tc(const R *X, const Geom &g, double dx, double dy, const float *theta, R *coef,
                                   int *err, cudaStream_t s, int wait_limit = kClosureWaitLimit);
// the network on n rows of 12 raw features (feat, device) -> out[n] (device)
cudaError_t launch_closure_predict(const float *theta, const float *feat, size_t n, float *out, int *err,
                                   cudaStream_t s, int wait_limit = kClosureWaitLimit);
cudaError_t launch_mlp_grad(const float *theta, const float *xs, const float *ys, const int *idx, int n, float *grad,
                            double *loss, cudaStream_t s);
cudaError_t launch_adam(float *theta, float *m, float *v, const float *g, int step, float lr, cudaStream_t s);

// Launch helpers implemented in the .cu files.
// ev (optional): one event recorded after each of the 3 kernels, for profiling.
template <class R> cudaError_t launch_stage(const StageArgs<R> &a, cudaStream_t s, cudaEvent_t *ev = nullptr);
template <class R> cudaError_t stage_set_attributes();
int stage_tile_planes(int precision);   // z planes of a fused-stage tile
// TMA tensor map (CUtensorMap) of a packed FP32 state for the FP32 tile box of
// a TI x TJ tile (dims k, j, i, field = Nz, Ny, Nx, 4; box 16 x TJ+4 x TI+4 x 4,
// 64-byte swizzle); false when the grid cannot be described (column length not a
// multiple of 4) or the driver call fails.  encode_fn: cuTensorMapEncodeTiled.
bool stage_tensor_map(void *out, const float *X, int Nx, int Ny, int Nz, int TI, int TJ, void *encode_fn);
// map of the same buffer for boxes of a tile's own cells (8 planes x TJ x TI x 4 fields)
bool stage_cell_map(void *out, const float *X, int Nx, int Ny, int Nz, int TI, int TJ, void *encode_fn);
// Tile shapes compiled for the fused pass (all with the same z planes, so the
// boundary-column list does not depend on the choice): count and TI x TJ.
int stage_tile_count(int precision);
void stage_tile_shape(int precision, int idx, int *ti, int *tj, int *nt = nullptr);

template <class R>
struct ProjectArgs {
    Geom g;
    Phys ph;
    R *y;                  // y_{n+1} (packed), updated in place
    const R *yn;           // y_n (packed), density for variable density
    const double *p;       // pressure [N]
    const R *Tsrc;         // initial temperature field or nullptr
    int source_mode;       // 0 none, 1 hold initial field, 2 ramped shape
    double t_n1;           // time of the new level (ramped source)
    double src_scale;      // ramp factor t/t_source_start (ramped source)
    const double *xg, *yg; // coordinates (ramped source)
    double TS[12];         // source box/gaussian parameters (ramped source)
    int TS_gauss;
    double T_source;
    // FP32 path constants, set by launch_project: 0.5/dx, 0.5/dy, dt/rho_inf, dt/(T_inf rho_inf)
    double hx, hy, s_rho0, s_rhoT;
};
template <class R> cudaError_t launch_project(const ProjectArgs<R> &a, cudaStream_t s);

// ---- pressure -------------------------------------------------------------
// FFT descriptor for one transform length, tables in device memory.
struct FftDesc {
    int n;                  // transform length
    int m;                  // inner power-of-two length: n, or the Bluestein length >= 2n-1
    int L;                  // log2(m)
    int bluestein;          // n is not a power of two
    const double2 *tw;      // exp(-2 pi i j / m), j < m
    const double2 *chirp;   // Bluestein: exp(-i pi j^2 / n), j < n
    const double2 *filt;    // Bluestein: FFT_m of the conjugate chirp filter
    int pr;                 // 1: prime-factor + Rader plan of length n (fft_pr.cuh); tw, chirp, filt unused
    const double2 *prb;     // Rader: DFT of the root-power filter / (P-1), (j1, j2) order
    const int *prmap;       // Rader: input slot map [P] and output index map [P-1]
    int pr_e1;              // Rader: CRT weight of the N1 residue
    const int *prslot;      // Rader: [n] shared-memory slot of input j, [n] slot of output k (slotted run)
};
// Prime-factor + Rader plan compiled for length n: f = {N1, P, F1, F2, F3} with
// n = N1 P, P prime, P - 1 = F1 F2 F3.  False for every other length.
bool poisson_pr_plan(int n, int f[5]);
// Line layout of that plan: sub-line stride SS and the B1 / B3 unit count UB.
bool poisson_pr_layout(int n, int *ss, int *ub);

template <class R>
struct PoissonArgs {
    Geom g;
    Phys ph;
    const R *y1;            // y_{n+1} (packed) -- velocity, T, Y
    const R *yn;            // y_n (packed) -- density for variable density
    double *p;              // pressure [N], read (top plane, previous iterate) and written
    double2 *G;             // spectral buffer [(Nz-1)+1][Nx-1][h1], s fastest
    const double *kx2;      // [Nx-1] kx^2
    const double *ky2;      // [Ny-1] ky^2
    FftDesc fx, fy;         // x: length Nx-1, y: length Ny-1
    int h1;                 // (Ny-1)/2 + 1
    // variable density: the parts of the source that do not depend on p, per
    // cell (written once per step by launch_vd_base, then read by every solve of
    // the fixed point), or nullptr (each solve evaluates the whole source); and
    // the z weights of the source per plane ([Nz][kVdz]: f0, f1, f2, c, s0..s3, dz)
    double *s0;
    R *g3;                  // with s0: grad(rho_n)/rho_n per cell, [3][N] (x, y, z components)
    const double *vdz;
};
constexpr int kVdz = 9;
template <class R> cudaError_t launch_vd_base(const PoissonArgs<R> &a, cudaStream_t s);
// z weights of the variable-density source for every plane (host, [Nz][kVdz])
void vd_z_table(const double *z, int Nz, double *out);
// zt: tridiagonal constants per k (layout documented at k_p_tridiag).
// ev (optional): one event recorded after each of the 5 kernels, for profiling.
template <class R>
cudaError_t launch_poisson_impl(const PoissonArgs<R> &a, const double *zt, cudaStream_t s, cudaEvent_t *ev = nullptr);
template <class R> cudaError_t poisson_set_attributes();
constexpr int kMaxFftLength = 2048;     // longest supported x or y transform
constexpr int kMaxZUnknowns = 511;      // longest tridiagonal system (Nz-1): the projection runs one
                                        // thread per cell of a column, at most 512

// Grid-wide FP64 reductions for the diagnostics and the pressure fixed point.
template <class R>
cudaError_t launch_diag(const Geom &g, const Phys &ph, const R *y, const R *y0fuel_ref, double *out, cudaStream_t s);

// Reference-style checkpoint report (functions.cu:82-185): scratch[0..6] =
// max|u|, max|v|, max|w|, -T_min, T_max, -Y_min, Y_max (fuel rectangle for T
// and Y), scratch[7] = first NaN key ((i Ny + j) Nz + k) * 5 + field as bits, or ~0.
size_t report_scratch_bytes();
template <class R>
cudaError_t launch_report(const Geom &g, const R *y, const double *xg, const double *yg, const double rect[4],
                          double *scratch, cudaStream_t s);

// Initial conditions on the device (setup.cu; functions.cu:187-323).
struct IcArgs {
    double u_r, z_r, alpha_u;                   // power-law wind
    int T_shape;                                // 0 gaussian, 1 parallelepiped
    double T_0, T_inf, x0, y0, z0, sx, sy, sz;  // gaussian centre and widths
    double Tx0, Tx1, Ty0, Ty1, Tz0, Tz1;        // parallelepiped
    double Yx0, Yx1, Yy0, Yy1, xa, ya, Y_h;     // fuel rectangle and ramps
    double p_top;
    double dead[5];                             // u, v, w, T, Y on dead nodes
};
template <class R>
cudaError_t launch_initial_conditions(const Geom &g, const IcArgs &a, const double *xg, const double *yg, R *state,
                                      double *p, cudaStream_t s);

// Asynchronous double-buffered field dumps (dump.cu).
struct Dumper;
Dumper *dumper_create(int device, const Parameters &P, size_t S, size_t N);
wf_status dumper_enqueue(Dumper *d, cudaStream_t s, const void *state, bool fp32, const double *p, const char *dir,
                         int n);
wf_status dumper_wait(Dumper *d);
void dumper_destroy(Dumper *d);
// Device record of the variable-density pressure fixed point (one per context):
// red accumulates max |p - p_prev| of the running iteration as the bits of a
// non-negative double; h is the change of the last finished iteration, m the
// iterations finished, done whether the last one met the tolerance.
struct PIterRec {
    unsigned long long red;
    double h;
    int m;
    int done;
};
cudaError_t launch_piter_begin(PIterRec *rec, cudaStream_t s);
// max |p - p_prev| into rec->red, then p_prev = p (one pass over both)
cudaError_t launch_maxdiff_copy(const double *p, double *p_prev, int n, PIterRec *rec, cudaStream_t s);
// closes an iteration: h, m, done; sets the loop's condition to "another
// iteration" (not done and m < maxit)
cudaError_t launch_piter_next(PIterRec *rec, double tol, int use_tol, int maxit, cudaGraphConditionalHandle cond,
                              cudaStream_t s);

}  // namespace wf
