// stage.cu -- one RK stage of the coupled atmosphere-wildfire model on sm_100a.
//
// A stage evaluates k_s = Phi(X_s) (reference src/cu/pde.cu:910-917: RHS,
// Smagorinsky SGS terms, boundary/IBM rules) and folds the RK combination into
// the same pass (reference solver.cu:14-93, utils.cu:14-21), so no k-buffer is
// ever stored:
//   pass 1  k_turb_inputs : per cell, the SGS inputs that neighbours need
//                           (raw mu_sgs, strain S', divergence source) and the
//                           wall friction velocity of the k = 0 plane;
//   pass 2  k_stage_rhs   : per cell, advection + diffusion + forces + reaction
//                           + SGS divergence, then acc/X_{s+1} updates for every
//                           cell the boundary rules do not overwrite;
//   pass 3  k_stage_bc    : per column, the boundary/IBM values of k_s (cut node,
//                           top, dead nodes) and their RK updates.
// Arithmetic follows the reference expression by expression; divisions by
// grid constants are folded into precomputed weights (ZCoef).
#include <math.h>

#include "wf_internal.h"

namespace wf {

namespace {

constexpr double kSigmaSB = 5.670374419e-8;  // Stefan-Boltzmann (reference constants.h:16)
constexpr double kAVD = 26.0;                // Van Driest constant (constants.h:19)

__device__ __forceinline__ int wrap_p(int v, int n)
{
    // periodic index with period n = N-1 for v in [-2, n+2] (pde.cu:227-234)
    if (v >= n) v -= n;
    if (v >= n) v -= n;
    if (v < 0) v += n;
    return v;
}

template <class R> __device__ __forceinline__ R zcoef(const double *zc, int e, int Nz, int k)
{
    return (R)__ldg(zc + (size_t)e * Nz + k);
}

template <class R> __device__ __forceinline__ R rmax(R a, R b) { return (a > b) ? a : b; }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return (a < b) ? a : b; }

__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float rsqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double rexp(double x) { return exp(x); }
__device__ __forceinline__ float rexp(float x) { return expf(x); }
__device__ __forceinline__ double rpow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float rpow(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double rfabs(double x) { return fabs(x); }
__device__ __forceinline__ float rfabs(float x) { return fabsf(x); }

// Values of one field along the column of a cell: k-3 .. k+3 (0 outside).
template <class R> struct ZN {
    R m3, m2, m1, c, p1, p2, p3;
};

template <class R>
__device__ __forceinline__ void load_col(ZN<R> &v, const R *__restrict__ col, int k, int Nz, int reach)
{
    v.c = col[k];
    v.m1 = (k > 0) ? col[k - 1] : R(0);
    v.p1 = (k < Nz - 1) ? col[k + 1] : R(0);
    v.m2 = (k > 1) ? col[k - 2] : R(0);
    v.p2 = (k < Nz - 2) ? col[k + 2] : R(0);
    if (reach >= 3) {
        v.m3 = (k > 2) ? col[k - 3] : R(0);
        v.p3 = (k < Nz - 3) ? col[k + 3] : R(0);
    } else {
        v.m3 = R(0);
        v.p3 = R(0);
    }
}

// forward / backward one-sided first derivatives on the non-uniform z grid
template <class R> __device__ __forceinline__ R dz_f(const ZN<R> &v, const double *zc, int Nz, int k)
{
    return zcoef<R>(zc, ZF0, Nz, k) * v.c + zcoef<R>(zc, ZF1, Nz, k) * v.p1 + zcoef<R>(zc, ZF2, Nz, k) * v.p2;
}
template <class R> __device__ __forceinline__ R dz_b(const ZN<R> &v, const double *zc, int Nz, int k)
{
    return zcoef<R>(zc, ZB0, Nz, k) * v.m2 + zcoef<R>(zc, ZB1, Nz, k) * v.m1 + zcoef<R>(zc, ZB2, Nz, k) * v.c;
}
// first derivative: one-sided at the walls, central inside (pde.cu:471-576)
template <class R> __device__ __forceinline__ R dz_1(const ZN<R> &v, const double *zc, int Nz, int k)
{
    if (k == 0) return dz_f(v, zc, Nz, k);
    if (k == Nz - 1) return dz_b(v, zc, Nz, k);
    return (v.p1 - v.m1) * zcoef<R>(zc, ZC, Nz, k);
}
// second derivative (pde.cu:497-575)
template <class R> __device__ __forceinline__ R dz_2(const ZN<R> &v, const double *zc, int Nz, int k)
{
    if (k == 0)
        return zcoef<R>(zc, ZFF0, Nz, k) * v.c + zcoef<R>(zc, ZFF1, Nz, k) * v.p1 +
               zcoef<R>(zc, ZFF2, Nz, k) * v.p2 + zcoef<R>(zc, ZFF3, Nz, k) * v.p3;
    if (k == Nz - 1)
        return zcoef<R>(zc, ZBB0, Nz, k) * v.m3 + zcoef<R>(zc, ZBB1, Nz, k) * v.m2 +
               zcoef<R>(zc, ZBB2, Nz, k) * v.m1 + zcoef<R>(zc, ZBB3, Nz, k) * v.c;
    return zcoef<R>(zc, ZCM, Nz, k) * v.m1 + zcoef<R>(zc, ZC0, Nz, k) * v.c + zcoef<R>(zc, ZCP, Nz, k) * v.p1;
}
// upwind one-sided derivatives used for advection (pde.cu:355-437)
template <class R> __device__ __forceinline__ R dz_km(const ZN<R> &v, const double *zc, int Nz, int k)
{
    return (k <= 1) ? dz_f(v, zc, Nz, k) : dz_b(v, zc, Nz, k);
}
template <class R> __device__ __forceinline__ R dz_kp(const ZN<R> &v, const double *zc, int Nz, int k)
{
    return (k >= Nz - 2) ? dz_b(v, zc, Nz, k) : dz_f(v, zc, Nz, k);
}

// Temperature source terms shared by both passes (pde.cu:664-711).
template <class R> struct Thermo {
    R T_RHS_tmp;  // conduction + radiation + reaction, before convection
    R nu;         // molecular kinematic viscosity (Sutherland when enabled)
    R mu;         // molecular dynamic viscosity
    R Y;          // solid fuel fraction (0 above the fuel top)
    R K_T;        // Arrhenius rate
};

template <class R>
__device__ __forceinline__ Thermo<R> thermo(const Phys &ph, R T, R T_kp1, const R *__restrict__ Ycol, int k,
                                            int nzy, R Tx, R Ty, R Tz, R lap_T, R dz_k, R rho)
{
    Thermo<R> o;
    R mu = (R)ph.mu, kT = (R)ph.kT, dk = R(0);
    const R T_pc = (R)ph.T_pc, T_inf = (R)ph.T_inf;
    const R H_step = (T > T_pc) ? R(1) : R(0);
    o.K_T = (R)ph.A * rexp(-(R)ph.T_act / T) * H_step;
    R Y = R(0), T_gas = T_inf, T_solid = T_inf;
    if (k <= nzy) {
        if (k < nzy) Y = Ycol[k];
        else T_gas = T_kp1;
        if (Y > R(0)) T_solid = T;
        else T_gas = T;
    }
    if (ph.sutherland_viscosity == 1)
        mu = R(1.716e-5) * rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(110.4)) / (T + R(110.4));
    if (ph.sutherland_conductivity == 1) {
        kT = R(0.0241) * rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(194)) / (T + R(194));
        dk = R(0.0241) * (R(1.5) * rpow(T / R(273.15), R(0.5)) * (R(273.15) + R(194)) / (T + R(194)) -
                          rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(194)) / ((T + R(194)) * (T + R(194))));
    }
    o.nu = mu / rho;
    o.mu = mu;
    R q = (R)ph.H_C * Y * o.K_T / (R)ph.c_p;
    const R as = (R)ph.alpha_s * (R)ph.sigma_s;
    if (as != R(0)) {
        // h_c evaluated per cell (the reference compounds its copy per thread, pde.cu:698)
        const R h_c = (R)ph.h_c * dz_k * rpow(rfabs(T_gas - T_solid) / dz_k, R(0.25));
        q = q - h_c * (R)ph.alpha_s * (R)ph.sigma_s * (T_gas - T_solid) /
                    ((R)ph.c_p * T_inf * (R)ph.rho_inf / T_gas);
    }
    const R c12 = (R)(12 * kSigmaSB * ph.delta), c4 = (R)(4 * kSigmaSB * ph.delta);
    o.T_RHS_tmp = (dk + c12 * (T * T) * (Tx * Tx + Ty * Ty + Tz * Tz) + (kT + c4 * (T * T * T)) * lap_T) /
                      (rho * (R)ph.c_p) + q;
    o.Y = Y;
    return o;
}

// ---------------------------------------------------------------------------
// pass 1: SGS inputs (reference RHS kernel, pde.cu:632-772)
template <class R>
__global__ void __launch_bounds__(256) k_turb_inputs(const StageArgs<R> a)
{
    const Geom &g = a.g;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N) return;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const int k = c % Nz, col = c / Nz, j = col % Ny, i = col / Ny;
    const int ip1 = wrap_p(i + 1, Nx - 1), im1 = wrap_p(i - 1, Nx - 1);
    const int jp1 = wrap_p(j + 1, Ny - 1), jm1 = wrap_p(j - 1, Ny - 1);
    const R *__restrict__ X = a.X;
    const size_t cxp = ((size_t)ip1 * Ny + j) * Nz + k, cxm = ((size_t)im1 * Ny + j) * Nz + k;
    const size_t cyp = ((size_t)i * Ny + jp1) * Nz + k, cym = ((size_t)i * Ny + jm1) * Nz + k;
    const R inv2dx = (R)(1.0 / (2 * a.ph.dx)), inv2dy = (R)(1.0 / (2 * a.ph.dy));
    const R invdx2 = (R)(1.0 / (a.ph.dx * a.ph.dx)), invdy2 = (R)(1.0 / (a.ph.dy * a.ph.dy));
    ZN<R> U, V, W, T;
    const size_t cb = (size_t)col * Nz;
    load_col(U, X + cb, k, Nz, 2);
    load_col(V, X + N + cb, k, Nz, 2);
    load_col(W, X + 2 * (size_t)N + cb, k, Nz, 2);
    load_col(T, X + 3 * (size_t)N + cb, k, Nz, 3);
    const R ux = (X[cxp] - X[cxm]) * inv2dx, uy = (X[cyp] - X[cym]) * inv2dy;
    const R vx = (X[N + cxp] - X[N + cxm]) * inv2dx, vy = (X[N + cyp] - X[N + cym]) * inv2dy;
    const R wx = (X[2 * (size_t)N + cxp] - X[2 * (size_t)N + cxm]) * inv2dx;
    const R wy = (X[2 * (size_t)N + cyp] - X[2 * (size_t)N + cym]) * inv2dy;
    const R Txp = X[3 * (size_t)N + cxp], Txm = X[3 * (size_t)N + cxm];
    const R Typ = X[3 * (size_t)N + cyp], Tym = X[3 * (size_t)N + cym];
    const R Tx = (Txp - Txm) * inv2dx, Ty = (Typ - Tym) * inv2dy;
    const R Txx = (Txp - R(2) * T.c + Txm) * invdx2, Tyy = (Typ - R(2) * T.c + Tym) * invdy2;
    const R uz = dz_1(U, g.zc, Nz, k), vz = dz_1(V, g.zc, Nz, k), wz = dz_1(W, g.zc, Nz, k);
    const R Tz = dz_1(T, g.zc, Nz, k), Tzz = dz_2(T, g.zc, Nz, k);
    const R rho = (R)a.ph.T_inf * (R)a.ph.rho_inf / T.c;
    // modified strain S' and |S| (the reference's integer 2/3 removes the trace term)
    R *scr = a.scr;
    const R third = R(1) / R(3);
    (void)third;
    const R S11 = R(2) * ux / R(3) - (vy + wz) / R(3);
    const R S22 = R(2) * vy / R(3) - (ux + wz) / R(3);
    const R S33 = R(2) * wz / R(3) - (ux + vy) / R(3);
    const R S12 = R(0.5) * (uy + vx), S13 = R(0.5) * (uz + wx), S23 = R(0.5) * (wy + vz);
    const R mod_S = rsqrt_(R(2) * (ux * ux + vy * vy + wz * wz) + (uz + wx) * (uz + wx) + (vx + uy) * (vx + uy) +
                           (wy + vz) * (wy + vz));
    const R dz_k = zcoef<R>(g.zc, ZDZ, Nz, k);
    const R mu_sgs = rho * zcoef<R>(g.zc, ZDELTA2, Nz, k) * mod_S;
    const int nzy = __ldg(g.nzy + col);
    const R lap_T = Txx + Tyy + Tzz;
    const Thermo<R> th = thermo(a.ph, T.c, T.p1, X + 4 * (size_t)N + (size_t)col * g.NzY, k, nzy, Tx, Ty, Tz,
                                lap_T, dz_k, rho);
    scr[c] = mu_sgs;
    scr[(size_t)N + c] = S11;
    scr[2 * (size_t)N + c] = S12;
    scr[3 * (size_t)N + c] = S13;
    scr[4 * (size_t)N + c] = S22;
    scr[5 * (size_t)N + c] = S23;
    scr[6 * (size_t)N + c] = S33;
    scr[7 * (size_t)N + c] = th.nu * th.T_RHS_tmp / T.c;
    if (k == 0) {
        // wall shear from the k = 0 plane (pde.cu:767-772)
        const R a1 = th.mu * uz, a2 = th.mu * vz;
        const R tau_w = rsqrt_(a1 * a1 + a2 * a2);
        a.utau[col] = rsqrt_(tau_w / rho);
    }
}

// RK update of one value: returns the next-stage (or final) value, updates acc.
template <class R>
__device__ __forceinline__ R rk_update(int method, int stage, R kv, R yv, R &accv, R a_next)
{
    if (method == 3) return kv;                               // operator test: store k_s
    if (method == 0) return yv + a_next * kv;                 // Euler (solver.cu:14-21)
    if (method == 1) {                                        // RK2 (solver.cu:23-30, 65-74)
        if (stage == 1) { accv = kv; return yv + a_next * kv; }
        return yv + a_next * (accv + kv);
    }
    // RK4 (solver.cu:32-39, 76-93): acc = k1 + 2 k2 + 2 k3, then (acc + k4)
    if (stage == 1) { accv = kv; return yv + a_next * kv; }
    if (stage < 4) { accv = accv + R(2) * kv; return yv + a_next * kv; }
    return yv + a_next * (accv + kv);
}

__device__ __forceinline__ bool stage_keeps_acc(int method, int stage)
{
    return (method == 1 && stage == 1) || (method == 2 && stage < 4);
}
__device__ __forceinline__ bool stage_reads_acc(int method, int stage)
{
    return (method == 1 && stage == 2) || (method == 2 && stage > 1);
}

// ---------------------------------------------------------------------------
// pass 2: right-hand side + SGS divergence + RK update (pde.cu:139-787,
// turbulence.cu:255-454)
template <class R>
__global__ void __launch_bounds__(256) k_stage_rhs(const StageArgs<R> a)
{
    const Geom &g = a.g;
    const Phys &ph = a.ph;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N) return;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const int k = c % Nz, col = c / Nz, j = col % Ny, i = col / Ny;
    const int ip1 = wrap_p(i + 1, Nx - 1), im1 = wrap_p(i - 1, Nx - 1);
    const int ip2 = wrap_p(i + 2, Nx - 1), im2 = wrap_p(i - 2, Nx - 1);
    const int jp1 = wrap_p(j + 1, Ny - 1), jm1 = wrap_p(j - 1, Ny - 1);
    const int jp2 = wrap_p(j + 2, Ny - 1), jm2 = wrap_p(j - 2, Ny - 1);
    const R *__restrict__ X = a.X;
    const size_t cb = (size_t)col * Nz;
    const size_t cxp = ((size_t)ip1 * Ny + j) * Nz + k, cxm = ((size_t)im1 * Ny + j) * Nz + k;
    const size_t cxp2 = ((size_t)ip2 * Ny + j) * Nz + k, cxm2 = ((size_t)im2 * Ny + j) * Nz + k;
    const size_t cyp = ((size_t)i * Ny + jp1) * Nz + k, cym = ((size_t)i * Ny + jm1) * Nz + k;
    const size_t cyp2 = ((size_t)i * Ny + jp2) * Nz + k, cym2 = ((size_t)i * Ny + jm2) * Nz + k;
    const R dx = (R)ph.dx, dy = (R)ph.dy;
    const R inv2dx = (R)(1.0 / (2 * ph.dx)), inv2dy = (R)(1.0 / (2 * ph.dy));
    const R invdx2 = (R)(1.0 / (ph.dx * ph.dx)), invdy2 = (R)(1.0 / (ph.dy * ph.dy));
    (void)dx;
    (void)dy;
    const double *zc = g.zc;

    R kval[4];    // u, v, w, T right-hand sides
    R Tx, Ty, Tz, Txx, Tyy, Tzz, rho, nu_t;
    R Yc = R(0), kY = R(0);
    const int nzy = __ldg(g.nzy + col);
    {
        ZN<R> Z[4];
        R f0[4], fxp[4], fxm[4], fxp2[4], fxm2[4], fyp[4], fym[4], fyp2[4], fym2[4];
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const R *Xf = X + (size_t)f * N;
            load_col(Z[f], Xf + cb, k, Nz, 3);
            f0[f] = Z[f].c;
            fxp[f] = Xf[cxp]; fxm[f] = Xf[cxm]; fxp2[f] = Xf[cxp2]; fxm2[f] = Xf[cxm2];
            fyp[f] = Xf[cyp]; fym[f] = Xf[cym]; fyp2[f] = Xf[cyp2]; fym2[f] = Xf[cym2];
        }
        const R u = f0[0], v = f0[1], w = f0[2], T = f0[3];
        rho = (R)ph.T_inf * (R)ph.rho_inf / T;
        const R u_plu = rmax(u, R(0)), u_min = rmin(u, R(0));
        const R v_plu = rmax(v, R(0)), v_min = rmin(v, R(0));
        const R w_plu = rmax(w, R(0)), w_min = rmin(w, R(0));
        R adv[4], lap[4];
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const R im = (R(3) * f0[f] - R(4) * fxm[f] + fxm2[f]) * inv2dx;
            const R ip = (R(-3) * f0[f] + R(4) * fxp[f] - fxp2[f]) * inv2dx;
            const R jm = (R(3) * f0[f] - R(4) * fym[f] + fym2[f]) * inv2dy;
            const R jp = (R(-3) * f0[f] + R(4) * fyp[f] - fyp2[f]) * inv2dy;
            const R km = dz_km(Z[f], zc, Nz, k), kp = dz_kp(Z[f], zc, Nz, k);
            adv[f] = (u_plu * im + u_min * ip) + (v_plu * jm + v_min * jp) + (w_plu * km + w_min * kp);
            const R fxx = (fxp[f] - R(2) * f0[f] + fxm[f]) * invdx2;
            const R fyy = (fyp[f] - R(2) * f0[f] + fym[f]) * invdy2;
            const R fzz = dz_2(Z[f], zc, Nz, k);
            lap[f] = fxx + fyy + fzz;
            if (f == 3) { Txx = fxx; Tyy = fyy; Tzz = fzz; }
        }
        Tx = (fxp[3] - fxm[3]) * inv2dx;
        Ty = (fyp[3] - fym[3]) * inv2dy;
        Tz = dz_1(Z[3], zc, Nz, k);
        const R dz_k = zcoef<R>(zc, ZDZ, Nz, k);
        const Thermo<R> th = thermo(ph, T, Z[3].p1, X + 4 * (size_t)N + (size_t)col * g.NzY, k, nzy, Tx, Ty, Tz,
                                    lap[3], dz_k, rho);
        Yc = th.Y;
        kY = -(R)ph.Y_f * th.K_T * Yc;
        const R T_RHS = (ph.temperature_convection == 0) ? th.T_RHS_tmp - (u * Tx + v * Ty + w * Tz)
                                                          : th.T_RHS_tmp - adv[3];
        const R mod_U = rsqrt_(u * u + v * v + w * w);
        const R cd = (R)(0.5 * ph.C_d * ph.alpha_s * ph.sigma_s);
        const R F_x = -cd * Yc * mod_U * u;
        const R F_y = -cd * Yc * mod_U * v;
        const R F_z = (R)ph.g * (rho - (R)ph.rho_inf) / rho - cd * Yc * mod_U * w;
        nu_t = th.nu;
        kval[0] = th.nu * lap[0] - adv[0] + F_x;
        kval[1] = th.nu * lap[1] - adv[1] + F_y;
        kval[2] = th.nu * lap[2] - adv[2] + F_z;
        kval[3] = T_RHS;
    }
    // ---- SGS divergence with Van Driest damping (turbulence.cu:255-454) ----
    {
        const R *__restrict__ S = a.scr;
        const R nu = (R)ph.mu / rho;
        (void)nu_t;
        const R inv_avd_nu = R(1) / (R)kAVD / nu;
        const double *topo = g.topo;
        const double zk = __ldg(g.z + k);
        const R ut0 = a.utau[col];
        auto zibm = [&](int ci, int kk) -> R {
            const double h = __ldg(topo + ci);
            const double d = __ldg(g.z + kk) - h;
            return (R)(d > 0.0 ? d : 0.0);
        };
        (void)zk;
        auto fw = [&](R zi, R ut) -> R { return R(1) - rexp(-zi * ut * inv_avd_nu); };
        const int colxp = ip1 * Ny + j, colxm = im1 * Ny + j, colyp = i * Ny + jp1, colym = i * Ny + jm1;
        R mu_c = S[c];
        const R S11 = S[(size_t)N + c], S12 = S[2 * (size_t)N + c], S13 = S[3 * (size_t)N + c];
        const R S22 = S[4 * (size_t)N + c], S23 = S[5 * (size_t)N + c], S33 = S[6 * (size_t)N + c];
        R mu_xp = S[cxp], mu_xm = S[cxm], mu_yp = S[cyp], mu_ym = S[cym];
        const R f_c = fw(zibm(col, k), ut0);
        const R f_xp = fw(zibm(colxp, k), a.utau[colxp]);
        const R f_xm = fw(zibm(colxm, k), a.utau[colxm]);
        const R f_yp = fw(zibm(colyp, k), a.utau[colyp]);
        const R f_ym = fw(zibm(colym, k), a.utau[colym]);
        mu_c *= f_c * f_c;
        mu_xm *= f_xm * f_xm;
        mu_xp *= f_xp * f_xp;
        mu_ym *= f_ym * f_ym;
        mu_yp *= f_yp * f_yp;
        R mu_km1 = 0, S13_km1 = 0, S23_km1 = 0, S33_km1 = 0, dU_km1 = 0;
        R mu_kp1 = 0, S13_kp1 = 0, S23_kp1 = 0, S33_kp1 = 0, dU_kp1 = 0;
        if (k > 0) {
            const size_t m = c - 1;
            const R f = fw(zibm(col, k - 1), ut0);
            mu_km1 = S[m] * (f * f);
            S13_km1 = S[3 * (size_t)N + m]; S23_km1 = S[5 * (size_t)N + m]; S33_km1 = S[6 * (size_t)N + m];
            dU_km1 = S[7 * (size_t)N + m];
        }
        if (k < Nz - 1) {
            const size_t m = c + 1;
            const R f = fw(zibm(col, k + 1), ut0);
            mu_kp1 = S[m] * (f * f);
            S13_kp1 = S[3 * (size_t)N + m]; S23_kp1 = S[5 * (size_t)N + m]; S33_kp1 = S[6 * (size_t)N + m];
            dU_kp1 = S[7 * (size_t)N + m];
        }
        const R mu_x = (mu_xp - mu_xm) * inv2dx, mu_y = (mu_yp - mu_ym) * inv2dy;
        const R S11_x = (S[(size_t)N + cxp] - S[(size_t)N + cxm]) * inv2dx;
        const R S12_x = (S[2 * (size_t)N + cxp] - S[2 * (size_t)N + cxm]) * inv2dx;
        const R S13_x = (S[3 * (size_t)N + cxp] - S[3 * (size_t)N + cxm]) * inv2dx;
        const R S21_y = (S[2 * (size_t)N + cyp] - S[2 * (size_t)N + cym]) * inv2dy;
        const R S22_y = (S[4 * (size_t)N + cyp] - S[4 * (size_t)N + cym]) * inv2dy;
        const R S23_y = (S[5 * (size_t)N + cyp] - S[5 * (size_t)N + cym]) * inv2dy;
        const R dU_x = (S[7 * (size_t)N + cxp] - S[7 * (size_t)N + cxm]) * inv2dx;
        const R dU_y = (S[7 * (size_t)N + cyp] - S[7 * (size_t)N + cym]) * inv2dy;
        R mu_z, S31_z, S32_z, S33_z, dU_z;
        if (k == 0 || k == Nz - 1) {
            // one-sided at the walls: neighbours k+1,k+2 (bottom) or k-1,k-2 (top)
            const int k2 = (k == 0) ? k + 2 : k - 2;
            const size_t m2 = cb + k2;
            const R f = fw(zibm(col, k2), ut0);
            const R mu2 = S[m2] * (f * f);
            ZN<R> zm, z13, z23, z33, zd;
            const R dUc = S[7 * (size_t)N + c];
            if (k == 0) {
                zm = {0, 0, 0, mu_c, mu_kp1, mu2, 0};
                z13 = {0, 0, 0, S13, S13_kp1, S[3 * (size_t)N + m2], 0};
                z23 = {0, 0, 0, S23, S23_kp1, S[5 * (size_t)N + m2], 0};
                z33 = {0, 0, 0, S33, S33_kp1, S[6 * (size_t)N + m2], 0};
                zd = {0, 0, 0, dUc, dU_kp1, S[7 * (size_t)N + m2], 0};
                mu_z = dz_f(zm, zc, Nz, k); S31_z = dz_f(z13, zc, Nz, k); S32_z = dz_f(z23, zc, Nz, k);
                S33_z = dz_f(z33, zc, Nz, k); dU_z = dz_f(zd, zc, Nz, k);
            } else {
                zm = {0, mu2, mu_km1, mu_c, 0, 0, 0};
                z13 = {0, S[3 * (size_t)N + m2], S13_km1, S13, 0, 0, 0};
                z23 = {0, S[5 * (size_t)N + m2], S23_km1, S23, 0, 0, 0};
                z33 = {0, S[6 * (size_t)N + m2], S33_km1, S33, 0, 0, 0};
                zd = {0, S[7 * (size_t)N + m2], dU_km1, dUc, 0, 0, 0};
                mu_z = dz_b(zm, zc, Nz, k); S31_z = dz_b(z13, zc, Nz, k); S32_z = dz_b(z23, zc, Nz, k);
                S33_z = dz_b(z33, zc, Nz, k); dU_z = dz_b(zd, zc, Nz, k);
            }
        } else {
            const R wc = zcoef<R>(zc, ZC, Nz, k);
            mu_z = (mu_kp1 - mu_km1) * wc;
            S31_z = (S13_kp1 - S13_km1) * wc;
            S32_z = (S23_kp1 - S23_km1) * wc;
            S33_z = (S33_kp1 - S33_km1) * wc;
            dU_z = (dU_kp1 - dU_km1) * wc;
        }
        const R div_S_x = S11_x + S21_y + S31_z;
        const R div_S_y = S12_x + S22_y + S32_z;
        const R div_S_z = S13_x + S23_y + S33_z;
        const R inv_rho = R(1) / rho;
        const R sgs_x = R(-2) * (mu_x * S11 + mu_y * S12 + mu_z * S13 + mu_c * div_S_x) * inv_rho;
        const R sgs_y = R(-2) * (mu_x * S12 + mu_y * S22 + mu_z * S23 + mu_c * div_S_y) * inv_rho;
        const R sgs_z = R(-2) * (mu_x * S13 + mu_y * S23 + mu_z * S33 + mu_c * div_S_z) * inv_rho;
        const R sgs_q = -(mu_x * Tx + mu_y * Ty + mu_z * Tz + mu_c * (Txx + Tyy + Tzz)) / (rho * (R)ph.Pr);
        const R third = R(1) / R(3);
        (void)third;
        kval[0] += -sgs_x + dU_x / R(3);
        kval[1] += -sgs_y + dU_y / R(3);
        kval[2] += -sgs_z + dU_z / R(3);
        kval[3] -= sgs_q;
    }
    // ---- values the column boundary pass needs -----------------------------
    const int kc = __ldg(g.cut + col);
    R *bc = a.bc + (size_t)col * kBcSlots;
    if (k == kc + 1) { bc[0] = kval[3]; bc[2] = (k < nzy) ? kY : R(0); }
    if (k == kc + 2) { bc[1] = kval[3]; bc[3] = (k < nzy) ? kY : R(0); }
    if (k == Nz - 2) { bc[4] = kval[0]; bc[5] = kval[1]; bc[6] = kval[2]; bc[7] = kval[3]; }
    if (k == Nz - 3) { bc[8] = kval[0]; bc[9] = kval[1]; bc[10] = kval[2]; bc[11] = kval[3]; }
    // ---- RK update of every value the boundary rules leave alone ------------
    const bool managed = (k <= kc) || (k == Nz - 1);
    const R an = (R)a.a_next;
    const bool rd = stage_reads_acc(a.method, a.stage), kp = stage_keeps_acc(a.method, a.stage);
    if (!managed) {
#pragma unroll
        for (int f = 0; f < 4; f++) {
            const size_t o = (size_t)f * N + c;
            R accv = rd ? a.acc[o] : R(0);
            a.Xout[o] = rk_update(a.method, a.stage, kval[f], a.yn[o], accv, an);
            if (kp) a.acc[o] = accv;
        }
    }
    if (k < g.NzY) {
        // fuel above the column's fuel top is never used; its k-value is 0
        const bool ymanaged = (k <= kc) && (k < nzy);
        if (!ymanaged) {
            const size_t o = 4 * (size_t)N + (size_t)col * g.NzY + k;
            const R kv = (k < nzy) ? kY : R(0);
            R accv = rd ? a.acc[o] : R(0);
            a.Xout[o] = rk_update(a.method, a.stage, kv, a.yn[o], accv, an);
            if (kp) a.acc[o] = accv;
        }
    }
}

// ---------------------------------------------------------------------------
// pass 3: boundary/IBM k-values per column (pde.cu:14-99) and their RK update
template <class R>
__global__ void __launch_bounds__(128) k_stage_bc(const StageArgs<R> a)
{
    const Geom &g = a.g;
    const Phys &ph = a.ph;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= g.Nx * g.Ny) return;
    const int Nz = g.Nz, N = g.N;
    const int kc = __ldg(g.cut + col), nzy = __ldg(g.nzy + col);
    const R *bc = a.bc + (size_t)col * kBcSlots;
    const double *z = g.z;
    const R an = (R)a.a_next;
    const bool rd = stage_reads_acc(a.method, a.stage), kp = stage_keeps_acc(a.method, a.stage);
    auto upd = [&](size_t o, R kv) {
        R accv = rd ? a.acc[o] : R(0);
        a.Xout[o] = rk_update(a.method, a.stage, kv, a.yn[o], accv, an);
        if (kp) a.acc[o] = accv;
    };
    const size_t cb = (size_t)col * Nz;
    // cut node
    {
        const R A = (R)(z[kc + 1] - z[kc]), B = (R)(z[kc + 2] - z[kc + 1]);
        const R T1 = bc[0], T2 = bc[1];
        const R Y1 = (kc + 1 < nzy) ? bc[2] : R(0), Y2 = (kc + 2 < nzy) ? bc[3] : R(0);
        upd(cb + kc, R(0));
        upd((size_t)N + cb + kc, R(0));
        upd(2 * (size_t)N + cb + kc, R(0));
        upd(3 * (size_t)N + cb + kc, ((A + B) * (A + B) * T1 - A * A * T2) / (B * (R(2) * A + B)));
        if (kc < nzy)
            upd(4 * (size_t)N + (size_t)col * g.NzY + kc, ((A + B) * (A + B) * Y1 - A * A * Y2) / (B * (R(2) * A + B)));
    }
    // top
    {
        const int k = Nz - 1;
        const R a1 = (R)(z[k] - z[k - 1]), a2 = (R)(z[k - 1] - z[k - 2]);
        const R num = (a2 + a1) * (a2 + a1), den = a2 * (a2 + R(2) * a1), a1s = a1 * a1;
#pragma unroll
        for (int f = 0; f < 4; f++) upd((size_t)f * N + cb + k, (num * bc[4 + f] - a1s * bc[8 + f]) / den);
    }
    // dead nodes below the terrain
    for (int k = 0; k < kc; k++) {
        upd(cb + k, (R)ph.u_dead);
        upd((size_t)N + cb + k, (R)ph.v_dead);
        upd(2 * (size_t)N + cb + k, (R)ph.w_dead);
        upd(3 * (size_t)N + cb + k, (R)ph.T_dead);
        if (k < nzy) upd(4 * (size_t)N + (size_t)col * g.NzY + k, (R)ph.Y_dead);
    }
}

}  // namespace

template <class R> cudaError_t launch_stage(const StageArgs<R> &a, cudaStream_t s, cudaEvent_t *ev)
{
    const int nb = (a.g.N + 255) / 256;
    k_turb_inputs<R><<<nb, 256, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[0], s);
    k_stage_rhs<R><<<nb, 256, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[1], s);
    const int ncol = a.g.Nx * a.g.Ny;
    k_stage_bc<R><<<(ncol + 127) / 128, 128, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[2], s);
    return cudaGetLastError();
}

template cudaError_t launch_stage<double>(const StageArgs<double> &, cudaStream_t, cudaEvent_t *);
template cudaError_t launch_stage<float>(const StageArgs<float> &, cudaStream_t, cudaEvent_t *);

}  // namespace wf
