// stage_common.cuh -- device helpers of the stage kernels (stage.cu):
// periodic indices, the precision-dependent fast operations,
// the temperature source terms, the RK update and the column boundary rules
// (reference src/cu/pde.cu:14-99, 640-720; solver.cu:14-93).
#pragma once

#include <math.h>

#include "wf_internal.h"

namespace wf {
namespace {

__device__ __forceinline__ int wrap_p(int v, int n)
{
    // periodic index with period n = N-1 for v in [-2, 2n+1] (pde.cu:227-234)
    if (v >= n) v -= n;
    if (v >= n) v -= n;
    if (v < 0) v += n;
    return v;
}

template <class R> __device__ __forceinline__ R rmax(R a, R b) { return (a > b) ? a : b; }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return (a < b) ? a : b; }

// Square root, quotient and third.  The FP64 path keeps the reference's
// correctly rounded operations; the FP32 stencil path uses the PTX
// approximations (sqrt.approx.f32, div.approx.f32: about 1 ulp, no slow path),
// well inside its 1e-5 error budget against FP64.
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float rsqrt_(float x)
{
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double third(double a) { return a / 3.0; }
__device__ __forceinline__ float third(float a) { return a * (1.0f / 3.0f); }
__device__ __forceinline__ double rexp(double x) { return exp(x); }
__device__ __forceinline__ float rexp(float x) { return expf(x); }
__device__ __forceinline__ double rpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float rpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double rfabs(double x) { return fabs(x); }
__device__ __forceinline__ float rfabs(float x) { return fabsf(x); }

// Packed FP32 pairs (sm_100 FFMA2 / FMUL2 / FADD2): the stencil arithmetic of
// two fields in one instruction.  Each lane is rounded like the scalar form.
__device__ __forceinline__ float2 bcast(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }

// Van Driest damping f_w = 1 - exp(-z+ / A_VD).  Below the cut-off the
// exponential is smaller than half an ulp of 1 and the result is exactly 1.
__device__ __forceinline__ double van_driest(double x) { return x < -37.5 ? 1.0 : 1.0 - exp(x); }
__device__ __forceinline__ float van_driest(float x) { return x < -17.5f ? 1.0f : 1.0f - expf(x); }
template <class R> struct VanDriestCut;
template <> struct VanDriestCut<double> { static constexpr double v = 37.5; };
template <> struct VanDriestCut<float> { static constexpr float v = 17.5f; };
// Whether van_driest(x) needs its exponential: not below the cut-off and not
// x = +-0, where 1 - exp(x) is exactly 0 (NaN needs it, and stays NaN).
template <class R> __device__ __forceinline__ bool van_driest_needs_exp(R x)
{
    return !(x < -VanDriestCut<R>::v) && !(x == R(0));
}
// van_driest(x) for an x that does not need the exponential: 1 or 0.
template <class R> __device__ __forceinline__ R van_driest_exact(R x) { return x < -VanDriestCut<R>::v ? R(1) : R(0); }

// Arrhenius rate A exp(-T_act/T) H(T - T_pc) (pde.cu:665): exactly 0 below
// the phase change; a warp with no lane above it skips the exponential.
template <class R> __device__ __forceinline__ R arrhenius(const PhysR<R> &p, R T)
{
    R K_T = R(0);
    if (__any_sync(__activemask(), T > p.T_pc)) K_T = (T > p.T_pc) ? p.A * rexp(-fdiv(p.T_act, T)) : R(0);
    return K_T;
}

// Temperature source terms (pde.cu:664-711).
template <class R> struct Thermo {
    R T_RHS_tmp;  // conduction + radiation + reaction, before convection
    R nu;         // molecular kinematic viscosity (Sutherland when enabled)
    R mu;         // molecular dynamic viscosity
    R Y;          // solid fuel fraction (0 above the fuel top)
    R K_T;        // Arrhenius rate
};

template <class R>
__device__ __forceinline__ Thermo<R> thermo(const PhysR<R> &p, int suth_mu, int suth_k, R T, R T_kp1, R Yc, int k,
                                            int nzy, R Tx, R Ty, R Tz, R lap_T, R dz_k, R rho)
{
    Thermo<R> o;
    R mu = p.mu, kT = p.kT, dk = R(0);
    o.K_T = arrhenius(p, T);
    R Y = R(0), T_gas = p.T_inf, T_solid = p.T_inf;
    if (k <= nzy) {
        if (k < nzy) Y = Yc;
        else T_gas = T_kp1;
        if (Y > R(0)) T_solid = T;
        else T_gas = T;
    }
    if (suth_mu == 1) mu = R(1.716e-5) * rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(110.4)) / (T + R(110.4));
    if (suth_k == 1) {
        kT = R(0.0241) * rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(194)) / (T + R(194));
        dk = R(0.0241) * (R(1.5) * rpow(T / R(273.15), R(0.5)) * (R(273.15) + R(194)) / (T + R(194)) -
                          rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(194)) / ((T + R(194)) * (T + R(194))));
    }
    o.nu = fdiv(mu, rho);
    o.mu = mu;
    R q = fdiv(p.H_C * Y * o.K_T, p.c_p);
    if (p.alpha_s * p.sigma_s != R(0)) {
        // h_c evaluated per cell (the reference compounds its copy per thread, pde.cu:698)
        const R h_c = p.h_c * dz_k * rpow(rfabs(T_gas - T_solid) / dz_k, R(0.25));
        q = q - h_c * p.alpha_s * p.sigma_s * (T_gas - T_solid) / (p.c_p * p.T_inf * p.rho_inf / T_gas);
    }
    o.T_RHS_tmp = fdiv(dk + p.c12 * (T * T) * (Tx * Tx + Ty * Ty + Tz * Tz) + (kT + p.c4 * (T * T * T)) * lap_T,
                       rho * p.c_p) + q;
    o.Y = Y;
    return o;
}

// RK update of one value: returns the next-stage (or final) value, updates acc.
//   operator test (method 3): k_s itself;
//   Euler (solver.cu:14-21): y_n + a k;
//   RK2 (solver.cu:23-30, 65-74): acc = k1, y_n + a k1; then y_n + a (acc + k2);
//   RK4 (solver.cu:32-39, 76-93): acc = k1, then acc + 2 k2, acc + 2 k3 with
//   y_n + a k_s; last y_n + a (acc + k4).
// Written as three fused multiply-adds with coefficients of the method and
// stage (uniform over the launch, so computed once), without branches per
// value: t = k + cA acc, out = a t + cY y_n, acc' = cK k + cB acc.  Each is the
// rounding of the contracted expression above (1 and 0 coefficients are exact).
template <class R>
__device__ __forceinline__ R rk_update(int method, int stage, R kv, R yv, R &accv, R a_next)
{
    const bool kstore = method == 3;
    const bool last = (method == 1 && stage == 2) || (method == 2 && stage == 4);
    const bool first = (method == 1 || method == 2) && stage == 1;
    const R cA = last ? R(1) : R(0), cY = kstore ? R(0) : R(1), an = kstore ? R(1) : a_next;
    const R cB = first ? R(0) : R(1), cK = (method == 2 && stage > 1 && stage < 4) ? R(2) : R(1);
    const R t = fma(cA, accv, kv);
    const R out = fma(an, t, cY * yv);
    accv = fma(cK, kv, cB * accv);
    return out;
}

__device__ __forceinline__ bool stage_keeps_acc(int method, int stage)
{
    return (method == 1 && stage == 1) || (method == 2 && stage < 4);
}
__device__ __forceinline__ bool stage_reads_acc(int method, int stage)
{
    return (method == 1 && stage == 2) || (method == 2 && stage > 1);
}

// RK update of the value at offset o with k-value kv.
template <class R>
__device__ __forceinline__ void rk_cell(const StageArgs<R> &a, size_t o, R kv, bool rd, bool kp, R an)
{
    R accv = rd ? a.acc[o] : R(0);
    a.Xout[o] = rk_update(a.method, a.stage, kv, a.yn[o], accv, an);
    if (kp) a.acc[o] = accv;
}

// Whether the cut node kc and the two cells above it share a z-tile of KZ
// planes (then the fused pass completes the cut node), and the same for the
// top plane and the two below it.
__host__ __device__ __forceinline__ bool bc_cut_in_tile(int kc, int KZ) { return kc / KZ == (kc + 2) / KZ; }
__host__ __device__ __forceinline__ bool bc_top_in_tile(int Nz, int KZ) { return (Nz - 1) / KZ == (Nz - 3) / KZ; }

// Cut node of a column (pde.cu:58-77): no-slip velocity, T and Y extrapolated
// from the k-values of kc+1 and kc+2 held in the column's boundary slots.
template <class R>
__device__ __forceinline__ void bc_cut_node(const StageArgs<R> &a, int col, int kc, int nzy, bool rd, bool kp, R an)
{
    const R *bc = a.bc + (size_t)col * kBcSlots;
    const size_t N = (size_t)a.g.N, cb = (size_t)col * a.g.Nz;
    const double *z = a.g.z;
    const R A = (R)(z[kc + 1] - z[kc]), B = (R)(z[kc + 2] - z[kc + 1]);
    rk_cell(a, cb + kc, R(0), rd, kp, an);
    rk_cell(a, N + cb + kc, R(0), rd, kp, an);
    rk_cell(a, 2 * N + cb + kc, R(0), rd, kp, an);
    rk_cell(a, 3 * N + cb + kc, fdiv((A + B) * (A + B) * bc[0] - A * A * bc[1], B * (R(2) * A + B)), rd, kp, an);
    if (kc < nzy) {
        const R Y1 = (kc + 1 < nzy) ? bc[2] : R(0), Y2 = (kc + 2 < nzy) ? bc[3] : R(0);
        rk_cell(a, 4 * N + (size_t)col * a.g.NzY + kc, fdiv((A + B) * (A + B) * Y1 - A * A * Y2, B * (R(2) * A + B)),
                rd, kp, an);
    }
}

// Top plane of a column (pde.cu:79-86): second-order extrapolation from Nz-2, Nz-3.
template <class R>
__device__ __forceinline__ void bc_top(const StageArgs<R> &a, int col, bool rd, bool kp, R an)
{
    const R *bc = a.bc + (size_t)col * kBcSlots;
    const int k = a.g.Nz - 1;
    const size_t N = (size_t)a.g.N, cb = (size_t)col * a.g.Nz;
    const double *z = a.g.z;
    const R a1 = (R)(z[k] - z[k - 1]), a2 = (R)(z[k - 1] - z[k - 2]);
    const R num = (a2 + a1) * (a2 + a1), den = a2 * (a2 + R(2) * a1), a1s = a1 * a1;
#pragma unroll
    for (int f = 0; f < 4; f++) rk_cell(a, (size_t)f * N + cb + k, fdiv(num * bc[4 + f] - a1s * bc[8 + f], den), rd, kp, an);
}

}  // namespace
}  // namespace wf
