/*
 * wf_oracle.c -- CPU restatement (FP64) of the reference time step.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle of the GPU path's tests.  See wf_oracle.h for
 * the contract and the list of deliberate differences.  Every function cites
 * the reference file:line whose arithmetic it restates; expression shapes are
 * kept close to the reference so rounding stays comparable.
 */
#include "wf_oracle.h"
#include "cpu_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SIGMA_SB 5.670374419e-8   /* Stefan-Boltzmann (include/c/constants.h:16) */
#define A_VD 26.0                 /* Van Driest constant (include/c/constants.h:19) */
#define PI_D 3.14159265358979323846

#define MAXD(a, b) (((a) > (b)) ? (a) : (b))
#define MIND(a, b) (((a) < (b)) ? (a) : (b))

typedef struct {
    int Nx, Ny, Nz, NzY;
    size_t N, NY;
} Dims;

static Dims dims_of(const Parameters *P)
{
    Dims d;
    d.Nx = P->Nx; d.Ny = P->Ny; d.Nz = P->Nz; d.NzY = P->Nz_Y_max;
    d.N = (size_t)d.Nx * d.Ny * d.Nz;
    d.NY = (size_t)d.Nx * d.Ny * d.NzY;
    return d;
}

#define IX(i, j, k) ((size_t)(k) + (size_t)D.Nz * ((size_t)(j) + (size_t)D.Ny * (size_t)(i)))
#define IY(i, j, k) ((size_t)(k) + (size_t)D.NzY * ((size_t)(j) + (size_t)D.Ny * (size_t)(i)))
#define IC(i, j) ((size_t)(j) + (size_t)D.Ny * (size_t)(i))

size_t wfo_state_size(const Parameters *P)
{
    Dims D = dims_of(P);
    return 4 * D.N + D.NY;
}

/* ---- one-sided / central z stencils on the non-uniform grid -------------
 * (forms used throughout src/cu/pde.cu, e.g. :363-365, :383-385, :497-500,
 * :539-542, :568, :572) */
static inline double dz_fwd1(double f0, double f1, double f2, double a, double b)
{
    return -(2 * a + b) * f0 / (a * (a + b)) + (a + b) * f1 / (a * b) - a * f2 / (b * (a + b));
}
static inline double dz_bwd1(double fm2, double fm1, double f0, double a2, double a1)
{
    /* a2 = dz_km2, a1 = dz_km1 */
    return a1 * fm2 / (a2 * (a2 + a1)) - (a2 + a1) * fm1 / (a2 * a1) + (a2 + 2 * a1) * f0 / (a1 * (a2 + a1));
}
static inline double dz_fwd2(double f0, double f1, double f2, double f3, double a, double b, double c)
{
    /* a = dz_k, b = dz_kp1, c = dz_kp2 (src/cu/pde.cu:497-500) */
    return (6 * a + 4 * b + 2 * c) * f0 / (a * (a + b) * (a + b + c))
         - (4 * a + 4 * b + 2 * c) * f1 / (a * b * (b + c))
         + (4 * a + 2 * b + 2 * c) * f2 / (b * c * (a + b))
         - (4 * a + 2 * b) * f3 / (c * (b + c) * (a + b + c));
}
static inline double dz_bwd2(double fm3, double fm2, double fm1, double f0, double a3, double a2, double a1)
{
    /* a3 = dz_km3, a2 = dz_km2, a1 = dz_km1 (src/cu/pde.cu:539-542) */
    return -(2 * a2 + 4 * a1) * fm3 / (a3 * (a3 + a2) * (a3 + a2 + a1))
         + (2 * a3 + 2 * a2 + 4 * a1) * fm2 / (a3 * a2 * (a2 + a1))
         - (2 * a3 + 4 * a2 + 4 * a1) * fm1 / (a2 * a1 * (a3 + a2))
         + (2 * a3 + 4 * a2 + 6 * a1) * f0 / (a1 * (a2 + a1) * (a3 + a2 + a1));
}

/* Turbulence inputs produced by the RHS pass and consumed by the SGS pass.
 * The reference keeps 18 such fields in R_turbulence (src/cu/pde.cu:747-772);
 * the symmetric strain components are stored once here. */
typedef struct {
    double *rho, *Tx, *Ty, *Tz, *Txx, *Tyy, *Tzz, *mu_sgs;
    double *S11, *S12, *S13, *S22, *S23, *S33, *divU, *u_tau;
} Turb;

static int turb_alloc(Turb *t, const Dims *d)
{
    double **f[] = {&t->rho, &t->Tx, &t->Ty, &t->Tz, &t->Txx, &t->Tyy, &t->Tzz, &t->mu_sgs,
                    &t->S11, &t->S12, &t->S13, &t->S22, &t->S23, &t->S33, &t->divU};
    for (size_t q = 0; q < sizeof(f) / sizeof(f[0]); q++) {
        *f[q] = (double *)calloc(d->N, sizeof(double));
        if (!*f[q]) return -1;
    }
    t->u_tau = (double *)calloc((size_t)d->Nx * d->Ny, sizeof(double));
    return t->u_tau ? 0 : -1;
}

static void turb_free(Turb *t)
{
    double *f[] = {t->rho, t->Tx, t->Ty, t->Tz, t->Txx, t->Tyy, t->Tzz, t->mu_sgs,
                   t->S11, t->S12, t->S13, t->S22, t->S23, t->S33, t->divU, t->u_tau};
    for (size_t q = 0; q < sizeof(f) / sizeof(f[0]); q++) free(f[q]);
}

/* RHS of u, v, w, T, Y plus turbulence inputs: src/cu/pde.cu:139-787. */
static void rhs_pass(const Parameters *P, const double *Ro, double *Rn, Turb *tb)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const double dx = P->dx, dy = P->dy;
    const double *z = P->z;
    const int *Nz_Y = P->Nz_Y;
    const size_t ou = 0, ov = D.N, ow = 2 * D.N, oT = 3 * D.N, oY = 4 * D.N;

    for (int i = 0; i < Nx; i++)
    for (int j = 0; j < Ny; j++)
    for (int k = 0; k < Nz; k++) {
        double mu = P->mu, kT = P->k, dk = 0.0;
        const int im1 = (i - 1 + Nx - 1) % (Nx - 1), im2 = (i - 2 + Nx - 1) % (Nx - 1);
        const int ip1 = (i + 1) % (Nx - 1), ip2 = (i + 2) % (Nx - 1);
        const int jm1 = (j - 1 + Ny - 1) % (Ny - 1), jm2 = (j - 2 + Ny - 1) % (Ny - 1);
        const int jp1 = (j + 1) % (Ny - 1), jp2 = (j + 2) % (Ny - 1);
#define LD(o, a, b, c) Ro[(o) + IX(a, b, c)]
        const double u = LD(ou, i, j, k), v = LD(ov, i, j, k), w = LD(ow, i, j, k), T = LD(oT, i, j, k);
        const double rho = P->T_inf * P->rho_inf / T;
        double Y = 0.0;
        const double u_im1 = LD(ou, im1, j, k), v_im1 = LD(ov, im1, j, k), w_im1 = LD(ow, im1, j, k), T_im1 = LD(oT, im1, j, k);
        const double u_ip1 = LD(ou, ip1, j, k), v_ip1 = LD(ov, ip1, j, k), w_ip1 = LD(ow, ip1, j, k), T_ip1 = LD(oT, ip1, j, k);
        const double u_im2 = LD(ou, im2, j, k), v_im2 = LD(ov, im2, j, k), w_im2 = LD(ow, im2, j, k), T_im2 = LD(oT, im2, j, k);
        const double u_ip2 = LD(ou, ip2, j, k), v_ip2 = LD(ov, ip2, j, k), w_ip2 = LD(ow, ip2, j, k), T_ip2 = LD(oT, ip2, j, k);
        const double u_jm1 = LD(ou, i, jm1, k), v_jm1 = LD(ov, i, jm1, k), w_jm1 = LD(ow, i, jm1, k), T_jm1 = LD(oT, i, jm1, k);
        const double u_jp1 = LD(ou, i, jp1, k), v_jp1 = LD(ov, i, jp1, k), w_jp1 = LD(ow, i, jp1, k), T_jp1 = LD(oT, i, jp1, k);
        const double u_jm2 = LD(ou, i, jm2, k), v_jm2 = LD(ov, i, jm2, k), w_jm2 = LD(ow, i, jm2, k), T_jm2 = LD(oT, i, jm2, k);
        const double u_jp2 = LD(ou, i, jp2, k), v_jp2 = LD(ov, i, jp2, k), w_jp2 = LD(ow, i, jp2, k), T_jp2 = LD(oT, i, jp2, k);
        double u_km1 = 0, v_km1 = 0, w_km1 = 0, T_km1 = 0, u_kp1 = 0, v_kp1 = 0, w_kp1 = 0, T_kp1 = 0;
        double u_km2 = 0, v_km2 = 0, w_km2 = 0, T_km2 = 0, u_kp2 = 0, v_kp2 = 0, w_kp2 = 0, T_kp2 = 0;
        double u_km3 = 0, v_km3 = 0, w_km3 = 0, T_km3 = 0, u_kp3 = 0, v_kp3 = 0, w_kp3 = 0, T_kp3 = 0;
        if (k > 0) { u_km1 = LD(ou, i, j, k - 1); v_km1 = LD(ov, i, j, k - 1); w_km1 = LD(ow, i, j, k - 1); T_km1 = LD(oT, i, j, k - 1); }
        if (k < Nz - 1) { u_kp1 = LD(ou, i, j, k + 1); v_kp1 = LD(ov, i, j, k + 1); w_kp1 = LD(ow, i, j, k + 1); T_kp1 = LD(oT, i, j, k + 1); }
        if (k > 1) { u_km2 = LD(ou, i, j, k - 2); v_km2 = LD(ov, i, j, k - 2); w_km2 = LD(ow, i, j, k - 2); T_km2 = LD(oT, i, j, k - 2); }
        if (k < Nz - 2) { u_kp2 = LD(ou, i, j, k + 2); v_kp2 = LD(ov, i, j, k + 2); w_kp2 = LD(ow, i, j, k + 2); T_kp2 = LD(oT, i, j, k + 2); }
        if (k > 2) { u_km3 = LD(ou, i, j, k - 3); v_km3 = LD(ov, i, j, k - 3); w_km3 = LD(ow, i, j, k - 3); T_km3 = LD(oT, i, j, k - 3); }
        if (k < Nz - 3) { u_kp3 = LD(ou, i, j, k + 3); v_kp3 = LD(ov, i, j, k + 3); w_kp3 = LD(ow, i, j, k + 3); T_kp3 = LD(oT, i, j, k + 3); }
#undef LD
        /* upwind (pde.cu:332-437) */
        const double u_plu = MAXD(u, 0.0), u_min = MIND(u, 0.0);
        const double v_plu = MAXD(v, 0.0), v_min = MIND(v, 0.0);
        const double w_plu = MAXD(w, 0.0), w_min = MIND(w, 0.0);
        const double u_im = (3 * u - 4 * u_im1 + u_im2) / (2 * dx), v_im = (3 * v - 4 * v_im1 + v_im2) / (2 * dx);
        const double w_im = (3 * w - 4 * w_im1 + w_im2) / (2 * dx), T_im = (3 * T - 4 * T_im1 + T_im2) / (2 * dx);
        const double u_ip = (-3 * u + 4 * u_ip1 - u_ip2) / (2 * dx), v_ip = (-3 * v + 4 * v_ip1 - v_ip2) / (2 * dx);
        const double w_ip = (-3 * w + 4 * w_ip1 - w_ip2) / (2 * dx), T_ip = (-3 * T + 4 * T_ip1 - T_ip2) / (2 * dx);
        const double u_jm = (3 * u - 4 * u_jm1 + u_jm2) / (2 * dy), v_jm = (3 * v - 4 * v_jm1 + v_jm2) / (2 * dy);
        const double w_jm = (3 * w - 4 * w_jm1 + w_jm2) / (2 * dy), T_jm = (3 * T - 4 * T_jm1 + T_jm2) / (2 * dy);
        const double u_jp = (-3 * u + 4 * u_jp1 - u_jp2) / (2 * dy), v_jp = (-3 * v + 4 * v_jp1 - v_jp2) / (2 * dy);
        const double w_jp = (-3 * w + 4 * w_jp1 - w_jp2) / (2 * dy), T_jp = (-3 * T + 4 * T_jp1 - T_jp2) / (2 * dy);
        double u_km, v_km, w_km, T_km, u_kp, v_kp, w_kp, T_kp;
        if (k <= 1) {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            u_km = dz_fwd1(u, u_kp1, u_kp2, a, b); v_km = dz_fwd1(v, v_kp1, v_kp2, a, b);
            w_km = dz_fwd1(w, w_kp1, w_kp2, a, b); T_km = dz_fwd1(T, T_kp1, T_kp2, a, b);
        } else {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            u_km = dz_bwd1(u_km2, u_km1, u, a2, a1); v_km = dz_bwd1(v_km2, v_km1, v, a2, a1);
            w_km = dz_bwd1(w_km2, w_km1, w, a2, a1); T_km = dz_bwd1(T_km2, T_km1, T, a2, a1);
        }
        if (k >= Nz - 2) {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            u_kp = dz_bwd1(u_km2, u_km1, u, a2, a1); v_kp = dz_bwd1(v_km2, v_km1, v, a2, a1);
            w_kp = dz_bwd1(w_km2, w_km1, w, a2, a1); T_kp = dz_bwd1(T_km2, T_km1, T, a2, a1);
        } else {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            u_kp = dz_fwd1(u, u_kp1, u_kp2, a, b); v_kp = dz_fwd1(v, v_kp1, v_kp2, a, b);
            w_kp = dz_fwd1(w, w_kp1, w_kp2, a, b); T_kp = dz_fwd1(T, T_kp1, T_kp2, a, b);
        }
        const double uux = u_plu * u_im + u_min * u_ip, vuy = v_plu * u_jm + v_min * u_jp, wuz = w_plu * u_km + w_min * u_kp;
        const double uvx = u_plu * v_im + u_min * v_ip, vvy = v_plu * v_jm + v_min * v_jp, wvz = w_plu * v_km + w_min * v_kp;
        const double uwx = u_plu * w_im + u_min * w_ip, vwy = v_plu * w_jm + v_min * w_jp, wwz = w_plu * w_km + w_min * w_kp;
        const double uTx = u_plu * T_im + u_min * T_ip, vTy = v_plu * T_jm + v_min * T_jp, wTz = w_plu * T_km + w_min * T_kp;
        /* central first/second derivatives (pde.cu:453-576) */
        const double ux = (u_ip1 - u_im1) / (2 * dx), uy = (u_jp1 - u_jm1) / (2 * dy);
        const double vx = (v_ip1 - v_im1) / (2 * dx), vy = (v_jp1 - v_jm1) / (2 * dy);
        const double wx = (w_ip1 - w_im1) / (2 * dx), wy = (w_jp1 - w_jm1) / (2 * dy);
        const double Tx = (T_ip1 - T_im1) / (2.0 * dx), Ty = (T_jp1 - T_jm1) / (2.0 * dy);
        const double uxx = (u_ip1 - 2.0 * u + u_im1) / (dx * dx), uyy = (u_jp1 - 2.0 * u + u_jm1) / (dy * dy);
        const double vxx = (v_ip1 - 2.0 * v + v_im1) / (dx * dx), vyy = (v_jp1 - 2.0 * v + v_jm1) / (dy * dy);
        const double wxx = (w_ip1 - 2.0 * w + w_im1) / (dx * dx), wyy = (w_jp1 - 2.0 * w + w_jm1) / (dy * dy);
        const double Txx = (T_ip1 - 2.0 * T + T_im1) / (dx * dx), Tyy = (T_jp1 - 2.0 * T + T_jm1) / (dy * dy);
        double uz, vz, wz, Tz, uzz, vzz, wzz, Tzz;
        if (k == 0) {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1], c = z[k + 3] - z[k + 2];
            uz = dz_fwd1(u, u_kp1, u_kp2, a, b); vz = dz_fwd1(v, v_kp1, v_kp2, a, b);
            wz = dz_fwd1(w, w_kp1, w_kp2, a, b); Tz = dz_fwd1(T, T_kp1, T_kp2, a, b);
            uzz = dz_fwd2(u, u_kp1, u_kp2, u_kp3, a, b, c); vzz = dz_fwd2(v, v_kp1, v_kp2, v_kp3, a, b, c);
            wzz = dz_fwd2(w, w_kp1, w_kp2, w_kp3, a, b, c); Tzz = dz_fwd2(T, T_kp1, T_kp2, T_kp3, a, b, c);
        } else if (k == Nz - 1) {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2], a3 = z[k - 2] - z[k - 3];
            uz = dz_bwd1(u_km2, u_km1, u, a2, a1); vz = dz_bwd1(v_km2, v_km1, v, a2, a1);
            wz = dz_bwd1(w_km2, w_km1, w, a2, a1); Tz = dz_bwd1(T_km2, T_km1, T, a2, a1);
            uzz = dz_bwd2(u_km3, u_km2, u_km1, u, a3, a2, a1); vzz = dz_bwd2(v_km3, v_km2, v_km1, v, a3, a2, a1);
            wzz = dz_bwd2(w_km3, w_km2, w_km1, w, a3, a2, a1); Tzz = dz_bwd2(T_km3, T_km2, T_km1, T, a3, a2, a1);
        } else {
            const double a1 = z[k] - z[k - 1], a = z[k + 1] - z[k];
            uz = (u_kp1 - u_km1) / (a1 + a); vz = (v_kp1 - v_km1) / (a1 + a);
            wz = (w_kp1 - w_km1) / (a1 + a); Tz = (T_kp1 - T_km1) / (a1 + a);
            uzz = 2 * u_km1 / (a1 * (a1 + a)) - 2 * u / (a1 * a) + 2 * u_kp1 / (a * (a1 + a));
            vzz = 2 * v_km1 / (a1 * (a1 + a)) - 2 * v / (a1 * a) + 2 * v_kp1 / (a * (a1 + a));
            wzz = 2 * w_km1 / (a1 * (a1 + a)) - 2 * w / (a1 * a) + 2 * w_kp1 / (a * (a1 + a));
            Tzz = 2 * T_km1 / (a1 * (a1 + a)) - 2 * T / (a1 * a) + 2 * T_kp1 / (a * (a1 + a));
        }
        const double lap_u = uxx + uyy + uzz, lap_v = vxx + vyy + vzz, lap_w = wxx + wyy + wzz;
        const double lap_T = Txx + Tyy + Tzz;
        /* modified strain S' and |S| with the reference's integer 2/3 == 0
         * (pde.cu:632-646) */
        const double S_11 = 2 * ux / 3 - (vy + wz) / 3;
        const double S_22 = 2 * vy / 3 - (ux + wz) / 3;
        const double S_33 = 2 * wz / 3 - (ux + vy) / 3;
        const double S_12 = 0.5 * (uy + vx);
        const double S_13 = 0.5 * (uz + wx);
        const double S_23 = 0.5 * (wy + vz);
        const double mod_S = sqrt(2.0 * (ux * ux + vy * vy + wz * wz)
                                  + (uz + wx) * (uz + wx) + (vx + uy) * (vx + uy) + (wy + vz) * (wy + vz)
                                  - 0 * (ux + vy + wz) * (ux + vy + wz));
        const double dz_k = (k < Nz - 1) ? z[k + 1] - z[k] : z[k] - z[k - 1];
        /* fuel and reaction (pde.cu:664-688) */
        const double H_step = (T > P->T_pc) ? 1.0 : 0.0;
        const double K_T = P->A * exp(-P->T_act / T) * H_step;
        double T_gas = P->T_inf, T_solid = P->T_inf;
        const int nzy = Nz_Y[IC(i, j)];
        if (k <= nzy) {
            if (k < nzy) {
                Y = Ro[oY + IY(i, j, k)];
                Rn[oY + IY(i, j, k)] = -P->Y_f * K_T * Y;
            } else {
                T_gas = T_kp1;
            }
            if (Y > 0.0) T_solid = T;
            else T_gas = T;
        }
        if (P->sutherland_viscosity == 1)
            mu = 1.716e-5 * pow(T / 273.15, 1.5) * (273.15 + 110.4) / (T + 110.4);
        if (P->sutherland_conductivity == 1) {
            kT = 0.0241 * pow(T / 273.15, 1.5) * (273.15 + 194) / (T + 194);
            dk = 0.0241 * (1.5 * pow(T / 273.15, 0.5) * (273.15 + 194) / (T + 194)
                           - pow(T / 273.15, 1.5) * (273.15 + 194) / ((T + 194) * (T + 194)));
        }
        const double nu = mu / rho;
        /* per-cell h_c (the reference compounds it per thread, pde.cu:698) */
        const double h_c = P->h_c * dz_k * pow(fabs(T_gas - T_solid) / dz_k, 1.0 / 4.0);
        const double q = P->H_C * Y * K_T / P->c_p
                       - h_c * P->alpha_s * P->sigma_s * (T_gas - T_solid) / (P->c_p * P->T_inf * P->rho_inf / T_gas);
        const double T_RHS_tmp = (dk + 12 * SIGMA_SB * P->delta * pow(T, 2) * (Tx * Tx + Ty * Ty + Tz * Tz)
                                  + (kT + 4 * SIGMA_SB * P->delta * pow(T, 3)) * lap_T) / (rho * P->c_p) + q;
        double T_RHS;
        if (P->temperature_convection == 0) T_RHS = T_RHS_tmp - (u * Tx + v * Ty + w * Tz);
        else T_RHS = T_RHS_tmp - (uTx + vTy + wTz);
        const double mod_U = sqrt(u * u + v * v + w * w);
        const double cd = 0.5 * P->C_d * P->alpha_s * P->sigma_s;
        const double F_x = -cd * Y * mod_U * u;
        const double F_y = -cd * Y * mod_U * v;
        const double F_z = P->g * (rho - P->rho_inf) / rho - cd * Y * mod_U * w;
        const size_t c = IX(i, j, k);
        Rn[ou + c] = nu * lap_u - (uux + vuy + wuz) + F_x;
        Rn[ov + c] = nu * lap_v - (uvx + vvy + wvz) + F_y;
        Rn[ow + c] = nu * lap_w - (uwx + vwy + wwz) + F_z;
        Rn[oT + c] = T_RHS;
        const double mu_sgs = rho * pow(P->C_s * pow(dx * dy * dz_k, 1.0 / 3.0), 2.0) * mod_S;
        tb->rho[c] = rho; tb->Tx[c] = Tx; tb->Ty[c] = Ty; tb->Tz[c] = Tz;
        tb->Txx[c] = Txx; tb->Tyy[c] = Tyy; tb->Tzz[c] = Tzz; tb->mu_sgs[c] = mu_sgs;
        tb->S11[c] = S_11; tb->S12[c] = S_12; tb->S13[c] = S_13;
        tb->S22[c] = S_22; tb->S23[c] = S_23; tb->S33[c] = S_33;
        tb->divU[c] = nu * T_RHS_tmp / T;
        if (k == 0) {
            const double tau_w = sqrt(pow(mu * (uz + wx * 0), 2.0) + pow(mu * (vz + wy * 0), 2.0));
            tb->u_tau[IC(i, j)] = sqrt(tau_w / rho);
        }
    }
}

/* SGS stress divergence with Van Driest damping: src/cu/turbulence.cu:255-454. */
static void turbulence_pass(const Parameters *P, const Turb *tb, double *Rn)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const double dx = P->dx, dy = P->dy, mu = P->mu, Pr = P->Pr;
    const double *z = P->z, *z_ibm = P->z_ibm;
    for (int i = 0; i < Nx; i++)
    for (int j = 0; j < Ny; j++)
    for (int k = 0; k < Nz; k++) {
        const int im1 = (i - 1 + Nx - 1) % (Nx - 1), jm1 = (j - 1 + Ny - 1) % (Ny - 1);
        const int ip1 = (i + 1) % (Nx - 1), jp1 = (j + 1) % (Ny - 1);
        const size_t c = IX(i, j, k);
        const double rho = tb->rho[c];
        const double Tx = tb->Tx[c], Ty = tb->Ty[c], Tz = tb->Tz[c];
        const double Txx = tb->Txx[c], Tyy = tb->Tyy[c], Tzz = tb->Tzz[c];
        double mu_c = tb->mu_sgs[c];
        const double S11 = tb->S11[c], S12 = tb->S12[c], S13 = tb->S13[c];
        const double S21 = S12, S22 = tb->S22[c], S23 = tb->S23[c];
        const double S31 = S13, S32 = S23, S33 = tb->S33[c];
        const size_t xp = IX(ip1, j, k), xm = IX(im1, j, k), yp = IX(i, jp1, k), ym = IX(i, jm1, k);
        double mu_xp = tb->mu_sgs[xp], mu_xm = tb->mu_sgs[xm], mu_yp = tb->mu_sgs[yp], mu_ym = tb->mu_sgs[ym];
        const double ut0 = tb->u_tau[IC(i, j)];
        const double ut_xp = tb->u_tau[IC(ip1, j)], ut_xm = tb->u_tau[IC(im1, j)];
        const double ut_yp = tb->u_tau[IC(i, jp1)], ut_ym = tb->u_tau[IC(i, jm1)];
        const double nu = mu / rho;
        const double fw = 1 - exp(-z_ibm[c] * ut0 / A_VD / nu);
        const double fw_xp = 1 - exp(-z_ibm[xp] * ut_xp / A_VD / nu);
        const double fw_xm = 1 - exp(-z_ibm[xm] * ut_xm / A_VD / nu);
        const double fw_yp = 1 - exp(-z_ibm[yp] * ut_yp / A_VD / nu);
        const double fw_ym = 1 - exp(-z_ibm[ym] * ut_ym / A_VD / nu);
        mu_c *= fw * fw;
        mu_xm *= fw_xm * fw_xm;
        mu_xp *= fw_xp * fw_xp;
        mu_ym *= fw_ym * fw_ym;
        mu_yp *= fw_yp * fw_yp;
        double mu_km1 = 0, S31_km1 = 0, S32_km1 = 0, S33_km1 = 0, dU_km1 = 0;
        double mu_kp1 = 0, S31_kp1 = 0, S32_kp1 = 0, S33_kp1 = 0, dU_kp1 = 0;
        if (k > 0) {
            const size_t m = IX(i, j, k - 1);
            const double f = 1 - exp(-z_ibm[m] * ut0 / A_VD / nu);
            mu_km1 = tb->mu_sgs[m]; S31_km1 = tb->S13[m]; S32_km1 = tb->S23[m]; S33_km1 = tb->S33[m];
            dU_km1 = tb->divU[m];
            mu_km1 *= f * f;
        }
        if (k < Nz - 1) {
            const size_t m = IX(i, j, k + 1);
            const double f = 1 - exp(-z_ibm[m] * ut0 / A_VD / nu);
            mu_kp1 = tb->mu_sgs[m]; S31_kp1 = tb->S13[m]; S32_kp1 = tb->S23[m]; S33_kp1 = tb->S33[m];
            dU_kp1 = tb->divU[m];
            mu_kp1 *= f * f;
        }
        const double mu_x = (mu_xp - mu_xm) / (2 * dx);
        const double mu_y = (mu_yp - mu_ym) / (2 * dy);
        const double S11_x = (tb->S11[xp] - tb->S11[xm]) / (2.0 * dx);
        const double S12_x = (tb->S12[xp] - tb->S12[xm]) / (2.0 * dx);
        const double S13_x = (tb->S13[xp] - tb->S13[xm]) / (2.0 * dx);
        const double S21_y = (tb->S12[yp] - tb->S12[ym]) / (2.0 * dy);
        const double S22_y = (tb->S22[yp] - tb->S22[ym]) / (2.0 * dy);
        const double S23_y = (tb->S23[yp] - tb->S23[ym]) / (2.0 * dy);
        const double dU_x = (tb->divU[xp] - tb->divU[xm]) / (2.0 * dx);
        const double dU_y = (tb->divU[yp] - tb->divU[ym]) / (2.0 * dy);
        double mu_z, S31_z, S32_z, S33_z, dU_z;
        if (k == 0) {
            /* the reference reads an unassigned divergence at the centre and at
             * k+2 here (turbulence.cu:402); the w value this feeds is
             * overwritten by the boundary rules, so the actual values are used */
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            const size_t m = IX(i, j, k + 2);
            const double f = 1 - exp(-z_ibm[m] * ut0 / A_VD / nu);
            double mu_kp2 = tb->mu_sgs[m];
            mu_kp2 *= f * f;
            mu_z = dz_fwd1(mu_c, mu_kp1, mu_kp2, a, b);
            S31_z = dz_fwd1(S31, S31_kp1, tb->S13[m], a, b);
            S32_z = dz_fwd1(S32, S32_kp1, tb->S23[m], a, b);
            S33_z = dz_fwd1(S33, S33_kp1, tb->S33[m], a, b);
            dU_z = dz_fwd1(tb->divU[c], dU_kp1, tb->divU[m], a, b);
        } else if (k == Nz - 1) {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            const size_t m = IX(i, j, k - 2);
            const double f = 1 - exp(-z_ibm[m] * ut0 / A_VD / nu);
            double mu_km2 = tb->mu_sgs[m];
            mu_km2 *= f * f;
            mu_z = dz_bwd1(mu_km2, mu_km1, mu_c, a2, a1);
            S31_z = dz_bwd1(tb->S13[m], S31_km1, S31, a2, a1);
            S32_z = dz_bwd1(tb->S23[m], S32_km1, S32, a2, a1);
            S33_z = dz_bwd1(tb->S33[m], S33_km1, S33, a2, a1);
            dU_z = dz_bwd1(tb->divU[m], dU_km1, tb->divU[c], a2, a1);
        } else {
            const double a1 = z[k] - z[k - 1], a = z[k + 1] - z[k];
            mu_z = (mu_kp1 - mu_km1) / (a + a1);
            S31_z = (S31_kp1 - S31_km1) / (a + a1);
            S32_z = (S32_kp1 - S32_km1) / (a + a1);
            S33_z = (S33_kp1 - S33_km1) / (a + a1);
            dU_z = (dU_kp1 - dU_km1) / (a + a1);
        }
        const double div_S_x = S11_x + S21_y + S31_z;
        const double div_S_y = S12_x + S22_y + S32_z;
        const double div_S_z = S13_x + S23_y + S33_z;
        const double sgs_x = -2 * (mu_x * S11 + mu_y * S21 + mu_z * S31 + mu_c * div_S_x) / rho;
        const double sgs_y = -2 * (mu_x * S12 + mu_y * S22 + mu_z * S32 + mu_c * div_S_y) / rho;
        const double sgs_z = -2 * (mu_x * S13 + mu_y * S23 + mu_z * S33 + mu_c * div_S_z) / rho;
        const double sgs_q = -(mu_x * Tx + mu_y * Ty + mu_z * Tz + mu_c * (Txx + Tyy + Tzz)) / (rho * Pr);
        Rn[c] += -sgs_x + dU_x / 3.0;
        Rn[D.N + c] += -sgs_y + dU_y / 3.0;
        Rn[2 * D.N + c] += -sgs_z + dU_z / 3.0;
        Rn[3 * D.N + c] -= sgs_q;
    }
}

/* Boundary and immersed-boundary rules for one vector (RHS or state):
 * src/cu/pde.cu:14-99. */
static void boundary_rules(const Parameters *P, double *R)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const double *z = P->z;
    const size_t ou = 0, ov = D.N, ow = 2 * D.N, oT = 3 * D.N, oY = 4 * D.N;
    for (int i = 0; i < Nx; i++)
    for (int j = 0; j < Ny; j++) {
        const int nzy = P->Nz_Y[IC(i, j)];
        const int kc = P->cut_nodes[IC(i, j)];
        int k = kc;
        {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            const double T1 = R[oT + IX(i, j, k + 1)], T2 = R[oT + IX(i, j, k + 2)];
            const double Y1 = (k + 1 < nzy) ? R[oY + IY(i, j, k + 1)] : 0.0;
            const double Y2 = (k + 2 < nzy) ? R[oY + IY(i, j, k + 2)] : 0.0;
            R[ou + IX(i, j, k)] = 0;
            R[ov + IX(i, j, k)] = 0;
            R[ow + IX(i, j, k)] = 0;
            R[oT + IX(i, j, k)] = ((a + b) * (a + b) * T1 - a * a * T2) / (b * (2 * a + b));
            if (k < nzy)
                R[oY + IY(i, j, k)] = ((a + b) * (a + b) * Y1 - a * a * Y2) / (b * (2 * a + b));
        }
        k = Nz - 1;
        {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            const size_t m1 = IX(i, j, k - 1), m2 = IX(i, j, k - 2), c = IX(i, j, k);
            const double num = (a2 + a1) * (a2 + a1), den = a2 * (a2 + 2 * a1), a1s = a1 * a1;
            const double u1 = R[ou + m1], u2 = R[ou + m2], v1 = R[ov + m1], v2 = R[ov + m2];
            const double w1 = R[ow + m1], w2 = R[ow + m2], T1 = R[oT + m1], T2 = R[oT + m2];
            R[ou + c] = (num * u1 - a1s * u2) / den;
            R[ov + c] = (num * v1 - a1s * v2) / den;
            R[ow + c] = (num * w1 - a1s * w2) / den;
            R[oT + c] = (num * T1 - a1s * T2) / den;
        }
        for (k = 0; k < kc; k++) {
            R[ou + IX(i, j, k)] = P->u_dead_nodes;
            R[ov + IX(i, j, k)] = P->v_dead_nodes;
            R[ow + IX(i, j, k)] = P->w_dead_nodes;
            R[oT + IX(i, j, k)] = P->T_dead_nodes;
            if (k < nzy) R[oY + IY(i, j, k)] = P->Y_dead_nodes;
        }
    }
}

void wfo_phi(const Parameters *P, const double *R_old, double *R_new)
{
    const Dims D = dims_of(P);
    Turb tb;
    memset(&tb, 0, sizeof(tb));
    turb_alloc(&tb, &D);
    memset(R_new, 0, sizeof(double) * (4 * D.N + D.NY));
    rhs_pass(P, R_old, R_new, &tb);
    turbulence_pass(P, &tb, R_new);
    boundary_rules(P, R_new);
    turb_free(&tb);
}

/* src/cu/solver.cu:59-93 with utils.cu:14-21 (caxpy) */
void wfo_time_integrate(const Parameters *P, double t_n, const double *y_n, double *y_np1)
{
    (void)t_n;  /* the right-hand side does not depend on t (pde.cu:140) */
    const size_t n = wfo_state_size(P);
    const double dt = P->dt;
    if (strncmp(P->method, "Euler", 5) == 0) {
        double *F = (double *)malloc(sizeof(double) * n);
        wfo_phi(P, y_n, F);
        for (size_t q = 0; q < n; q++) y_np1[q] = y_n[q] + dt * F[q];
        free(F);
        return;
    }
    if (strncmp(P->method, "RK2", 3) == 0) {
        double *k1 = (double *)malloc(sizeof(double) * n), *k2 = (double *)malloc(sizeof(double) * n);
        double *F = (double *)malloc(sizeof(double) * n);
        wfo_phi(P, y_n, k1);
        for (size_t q = 0; q < n; q++) F[q] = y_n[q] + dt * k1[q];
        wfo_phi(P, F, k2);
        for (size_t q = 0; q < n; q++) y_np1[q] = y_n[q] + 0.5 * dt * (k1[q] + k2[q]);
        free(k1); free(k2); free(F);
        return;
    }
    double *k = (double *)malloc(sizeof(double) * 4 * n), *F = (double *)malloc(sizeof(double) * n);
    double *k1 = k, *k2 = k + n, *k3 = k + 2 * n, *k4 = k + 3 * n;
    wfo_phi(P, y_n, k1);
    for (size_t q = 0; q < n; q++) F[q] = y_n[q] + dt * 0.5 * k1[q];
    wfo_phi(P, F, k2);
    for (size_t q = 0; q < n; q++) F[q] = y_n[q] + dt * 0.5 * k2[q];
    wfo_phi(P, F, k3);
    for (size_t q = 0; q < n; q++) F[q] = y_n[q] + dt * k3[q];
    wfo_phi(P, F, k4);
    for (size_t q = 0; q < n; q++)
        y_np1[q] = y_n[q] + (dt / 6) * (k1[q] + 2 * k2[q] + 2 * k3[q] + k4[q]);
    free(k); free(F);
}

/* ---- pressure --------------------------------------------------------- */

/* Poisson right-hand side, constant density: src/cu/pressure.cu:14-101. */
static void rhs_constant(const Parameters *P, const double *U, double *f /* complex, FFT layout */)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const double *z = P->z;
    const size_t sl = (size_t)(Nx - 1) * (Ny - 1);
    for (int i = 0; i < Nx - 1; i++)
    for (int j = 0; j < Ny - 1; j++)
    for (int k = 0; k < Nz - 1; k++) {
        const int im1 = (i - 1 + Nx - 1) % (Nx - 1), jm1 = (j - 1 + Ny - 1) % (Ny - 1);
        const int ip1 = (i + 1) % (Nx - 1), jp1 = (j + 1) % (Ny - 1);
        const double u = U[IX(i, j, k)], v = U[D.N + IX(i, j, k)], w = U[2 * D.N + IX(i, j, k)];
        const double u_im1 = U[IX(im1, j, k)], u_ip1 = U[IX(ip1, j, k)];
        const double v_jm1 = U[D.N + IX(i, jm1, k)], v_jp1 = U[D.N + IX(i, jp1, k)];
        double wz;
        if (k == 0) {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            wz = dz_fwd1(w, U[2 * D.N + IX(i, j, k + 1)], U[2 * D.N + IX(i, j, k + 2)], a, b);
        } else {
            const double a1 = z[k] - z[k - 1], a = z[k + 1] - z[k];
            wz = (U[2 * D.N + IX(i, j, k + 1)] - U[2 * D.N + IX(i, j, k - 1)]) / (a + a1);
        }
        const double ux = (0.5 * (u_ip1 + u) - 0.5 * (u + u_im1)) / P->dx;
        const double vy = (0.5 * (v_jp1 + v) - 0.5 * (v + v_jm1)) / P->dy;
        const size_t o = (size_t)j + (size_t)(Ny - 1) * i + sl * k;
        f[2 * o] = P->rho_inf * (ux + vy + wz) / P->dt;
        f[2 * o + 1] = 0.0;
    }
}

/* Poisson right-hand side, variable density: src/cu/pressure.cu:103-327.
 * Cells with k = Nz-1 are not needed (not stored by the reference). */
static void rhs_variable(const Parameters *P, const double *Y1, const double *Yn, const double *p, double *f)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const double *z = P->z;
    const size_t sl = (size_t)(Nx - 1) * (Ny - 1);
    const double Ti = P->T_inf, ri = P->rho_inf;
    const size_t ou = 0, ov = D.N, ow = 2 * D.N, oT = 3 * D.N, oY = 4 * D.N;
    for (int i = 0; i < Nx - 1; i++)
    for (int j = 0; j < Ny - 1; j++)
    for (int k = 0; k < Nz - 1; k++) {
        const int im1 = (i - 1 + Nx - 1) % (Nx - 1), jm1 = (j - 1 + Ny - 1) % (Ny - 1);
        const int ip1 = (i + 1) % (Nx - 1), jp1 = (j + 1) % (Ny - 1);
        const size_t c = IX(i, j, k);
        const double u = Y1[ou + c], v = Y1[ov + c], w = Y1[ow + c], T = Y1[oT + c], pc = p[c];
        const double rho = Ti * ri / Yn[oT + c];
        const double u_im1 = Y1[ou + IX(im1, j, k)], u_ip1 = Y1[ou + IX(ip1, j, k)];
        const double v_jm1 = Y1[ov + IX(i, jm1, k)], v_jp1 = Y1[ov + IX(i, jp1, k)];
        const double T_im1 = Y1[oT + IX(im1, j, k)], T_ip1 = Y1[oT + IX(ip1, j, k)];
        const double T_jm1 = Y1[oT + IX(i, jm1, k)], T_jp1 = Y1[oT + IX(i, jp1, k)];
        const double p_im1 = p[IX(im1, j, k)], p_ip1 = p[IX(ip1, j, k)];
        const double p_jm1 = p[IX(i, jm1, k)], p_jp1 = p[IX(i, jp1, k)];
        const double r_im1 = Ti * ri / Yn[oT + IX(im1, j, k)], r_ip1 = Ti * ri / Yn[oT + IX(ip1, j, k)];
        const double r_jm1 = Ti * ri / Yn[oT + IX(i, jm1, k)], r_jp1 = Ti * ri / Yn[oT + IX(i, jp1, k)];
        const double ux = (0.5 * (u_ip1 + u) - 0.5 * (u + u_im1)) / P->dx;
        const double vy = (0.5 * (v_jp1 + v) - 0.5 * (v + v_jm1)) / P->dy;
        const double Tx = (T_ip1 - T_im1) / (2 * P->dx), Ty = (T_jp1 - T_jm1) / (2 * P->dy);
        const double Txx = (T_ip1 - 2 * T + T_im1) / (P->dx * P->dx);
        const double Tyy = (T_jp1 - 2 * T + T_jm1) / (P->dy * P->dy);
        const double rhox = (r_ip1 - r_im1) / (2 * P->dx), rhoy = (r_jp1 - r_jm1) / (2 * P->dy);
        const double px = (p_ip1 - p_im1) / (2 * P->dx), py = (p_jp1 - p_jm1) / (2 * P->dy);
        double wz, rhoz, pz, Tz, Tzz, dz_k;
        if (k == 0) {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1], cc = z[k + 3] - z[k + 2];
            dz_k = a;
            const size_t m1 = IX(i, j, k + 1), m2 = IX(i, j, k + 2), m3 = IX(i, j, k + 3);
            wz = dz_fwd1(w, Y1[ow + m1], Y1[ow + m2], a, b);
            rhoz = dz_fwd1(rho, Ti * ri / Yn[oT + m1], Ti * ri / Yn[oT + m2], a, b);
            pz = dz_fwd1(pc, p[m1], p[m2], a, b);
            Tz = dz_fwd1(T, Y1[oT + m1], Y1[oT + m2], a, b);
            /* the reference reads an unassigned T(k+3) here (pressure.cu:231);
             * f at k = 0 is never used by the solve (pressure.cu:492) */
            Tzz = dz_fwd2(T, Y1[oT + m1], Y1[oT + m2], Y1[oT + m3], a, b, cc);
        } else {
            const double a1 = z[k] - z[k - 1], a = z[k + 1] - z[k];
            dz_k = a;
            const size_t mp = IX(i, j, k + 1), mm = IX(i, j, k - 1);
            wz = (Y1[ow + mp] - Y1[ow + mm]) / (a + a1);
            rhoz = (Ti * ri / Yn[oT + mp] - Ti * ri / Yn[oT + mm]) / (a + a1);
            pz = (p[mp] - p[mm]) / (a + a1);
            Tz = (Y1[oT + mp] - Y1[oT + mm]) / (a + a1);
            Tzz = 2 * Y1[oT + mm] / (a1 * (a1 + a)) - 2 * T / (a1 * a) + 2 * Y1[oT + mp] / (a * (a1 + a));
        }
        const double lap_T = Txx + Tyy + Tzz;
        double Yc = 0.0;
        const double H_step = (T > P->T_pc) ? 1.0 : 0.0;
        const double K_T = P->A * exp(-P->T_act / T) * H_step;
        double T_gas = T;
        const double T_solid = T;
        const int nzy = P->Nz_Y[IC(i, j)];
        if (k <= nzy) {
            if (k < nzy) Yc = Y1[oY + IY(i, j, k)];
            if (Yc > 0.0) T_gas = P->T_pc + (T - P->T_pc);
            else T_gas = T;
        }
        double kT = P->k, dk = 0.0;
        if (P->sutherland_conductivity == 1) {
            kT = 0.0241 * pow(T / 273.15, 1.5) * (273.15 + 194) / (T + 194);
            dk = 0.0241 * (1.5 * pow(T / 273.15, 0.5) * (273.15 + 194) / (T + 194)
                           - pow(T / 273.15, 1.5) * (273.15 + 194) / ((T + 194) * (T + 194)));
        }
        const double h_c = P->h_c * dz_k * pow((T_gas - T_solid) / dz_k, 1.0 / 4.0);
        const double q = P->H_C * Yc * K_T / P->c_p
                       - h_c * P->alpha_s * P->sigma_s * (T_gas - T_solid) / (P->c_p * Ti * ri / T_gas);
        const double divT = (dk + 12 * SIGMA_SB * P->delta * pow(T, 2) * (Tx * Tx + Ty * Ty + Tz * Tz)
                             + (kT + 4 * SIGMA_SB * P->delta * pow(T, 3)) * lap_T) / (Ti * ri * P->c_p) + q / T;
        const size_t o = (size_t)j + (size_t)(Ny - 1) * i + sl * k;
        f[2 * o] = rho * (ux + vy + wz - divT) / P->dt + (rhox * px + rhoy * py + rhoz * pz) / rho;
        f[2 * o + 1] = 0.0;
    }
}

/* One direct solve: FFT2 per z slice, tridiagonal per wavenumber, inverse:
 * src/cu/pressure.cu:356-390 (coefficients), 473-504 (right-hand side),
 * 418-443 (Thomas), 392-416 (normalisation and periodic planes). */
static void solve_once(const Parameters *P, const double *y_np1, const double *y_n, double *p)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const int n0 = Nx - 1, n1 = Ny - 1, nk = Nz - 1;
    const size_t sl = (size_t)n0 * n1;
    const double *z = P->z;
    double *f = (double *)malloc(sizeof(double) * 2 * sl * nk);
    double *pt = (double *)malloc(sizeof(double) * 2 * sl);
    if (P->variable_density == 0) rhs_constant(P, y_np1, f);
    else rhs_variable(P, y_np1, y_n, p, f);
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++) {
            pt[2 * ((size_t)j + (size_t)n1 * i)] = p[IX(i, j, Nz - 1)];
            pt[2 * ((size_t)j + (size_t)n1 * i) + 1] = 0.0;
        }
    cfft_2d_many(n0, n1, 1, pt, pt, -1);
    cfft_2d_many(n0, n1, nk, f, f, -1);
    const double dz0 = z[1] - z[0], dz1 = z[2] - z[1];
    const double dzNm2 = z[Nz - 2] - z[Nz - 3], dzNm1 = z[Nz - 1] - z[Nz - 2];
    double *a = (double *)malloc(sizeof(double) * nk), *b = (double *)malloc(sizeof(double) * nk);
    double *cc = (double *)malloc(sizeof(double) * nk), *l = (double *)malloc(sizeof(double) * nk);
    double *uu = (double *)malloc(sizeof(double) * nk);
    double *dr = (double *)malloc(sizeof(double) * nk), *di = (double *)malloc(sizeof(double) * nk);
    for (int r = 0; r < n0; r++)
    for (int s = 0; s < n1; s++) {
        const double kk = P->kx[r] * P->kx[r] + P->ky[s] * P->ky[s];
        /* coefficients: a = sub-diagonal of row k+1, c = super-diagonal of row k */
        a[0] = 2 / (dz0 * (dz0 + dz1));
        b[0] = -1.0 / dz0;
        cc[0] = (dz0 + dz1) / (dz0 * dz1) - 0.5 * dz0 * kk - 1 / dz1;
        for (int k = 1; k < Nz - 2; k++) {
            const double dkm1 = z[k] - z[k - 1], dk = z[k + 1] - z[k], dkp1 = z[k + 2] - z[k + 1];
            a[k] = 2 / (dk * (dk + dkp1));
            cc[k] = 2 / (dk * (dkm1 + dk));
            b[k] = -(kk + 2 / (dkm1 * dk));
        }
        b[Nz - 2] = -(kk + 2 / (dzNm2 * dzNm1));
        /* right-hand side rows */
        const size_t o = (size_t)s + (size_t)n1 * r;
        dr[0] = 0.5 * dz0 * f[2 * (o + sl * 1)];
        di[0] = 0.5 * dz0 * f[2 * (o + sl * 1) + 1];
        for (int k = 1; k < Nz - 2; k++) {
            dr[k] = f[2 * (o + sl * k)];
            di[k] = f[2 * (o + sl * k) + 1];
        }
        const double cl = 2 / (dzNm1 * (dzNm2 + dzNm1));
        dr[Nz - 2] = f[2 * (o + sl * (Nz - 2))] - pt[2 * o] / cl;
        di[Nz - 2] = f[2 * (o + sl * (Nz - 2)) + 1] - pt[2 * o + 1] / cl;
        /* Thomas: LU with real factors, complex right-hand side */
        uu[0] = b[0];
        for (int k = 1; k < nk; k++) {
            l[k - 1] = a[k - 1] / uu[k - 1];
            uu[k] = b[k] - l[k - 1] * cc[k - 1];
        }
        for (int k = 1; k < nk; k++) {
            dr[k] = dr[k] - l[k - 1] * dr[k - 1];
            di[k] = di[k] - l[k - 1] * di[k - 1];
        }
        dr[nk - 1] = dr[nk - 1] / uu[nk - 1];
        di[nk - 1] = di[nk - 1] / uu[nk - 1];
        for (int k = nk - 2; k >= 0; k--) {
            dr[k] = (dr[k] - cc[k] * dr[k + 1]) / uu[k];
            di[k] = (di[k] - cc[k] * di[k + 1]) / uu[k];
        }
        for (int k = 0; k < nk; k++) {
            f[2 * (o + sl * k)] = dr[k];
            f[2 * (o + sl * k) + 1] = di[k];
        }
    }
    cfft_2d_many(n0, n1, nk, f, f, +1);
    const double norm = (double)n0 * (double)n1;
    for (int i = 0; i < n0; i++)
        for (int j = 0; j < n1; j++)
            for (int k = 0; k < nk; k++)
                p[IX(i, j, k)] = f[2 * ((size_t)j + (size_t)n1 * i + sl * k)] / norm;
    /* periodic duplicate planes take the values of this solve */
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            if (i < Nx - 1 && j < Ny - 1) continue;
            for (int k = 0; k < Nz; k++) p[IX(i, j, k)] = p[IX(i % (Nx - 1), j % (Ny - 1), k)];
        }
    free(f); free(pt); free(a); free(b); free(cc); free(l); free(uu); free(dr); free(di);
}

int wfo_solve_pressure(const Parameters *P, const double *y_np1, const double *y_n, double *p, double *err)
{
    if (P->variable_density == 0) {
        solve_once(P, y_np1, y_n, p);
        if (err) *err = 0.0;
        return 1;
    }
    const Dims D = dims_of(P);
    double *p_tmp = (double *)malloc(sizeof(double) * D.N);
    double e = 0.0;
    int m;
    for (m = 0; m < P->pressure_solver_iter; m++) {
        memcpy(p_tmp, p, sizeof(double) * D.N);
        solve_once(P, y_np1, y_n, p);
        e = 0.0;
        for (size_t q = 0; q < D.N; q++) {
            const double d = fabs(p[q] - p_tmp[q]);
            e = MAXD(e, d);
        }
        if (e <= P->pressure_solver_tol) { m++; break; }
    }
    free(p_tmp);
    if (err) *err = e;
    return m;
}

/* Projection (src/cu/pde.cu:789-908), then the boundary rules on the state
 * (pde.cu:14-99) and the clamps (pde.cu:101-137). */
void wfo_project(const Parameters *P, double *Y, const double *Yn, const double *p)
{
    const Dims D = dims_of(P);
    const int Nx = D.Nx, Ny = D.Ny, Nz = D.Nz;
    const double *z = P->z;
    const int fd = P->velocity_correction_fd;
    for (int i = 0; i < Nx; i++)
    for (int j = 0; j < Ny; j++)
    for (int k = 0; k < Nz; k++) {
        const int im1 = (i - 1 + Nx - 1) % (Nx - 1), jm1 = (j - 1 + Ny - 1) % (Ny - 1);
        const int ip1 = (i + 1) % (Nx - 1), jp1 = (j + 1) % (Ny - 1);
        const size_t c = IX(i, j, k);
        const double pc = p[c];
        double rho = P->T_inf * P->rho_inf / Yn[3 * D.N + c];
        const double px = (p[IX(ip1, j, k)] - p[IX(im1, j, k)]) / (2 * P->dx);
        const double py = (p[IX(i, jp1, k)] - p[IX(i, jm1, k)]) / (2 * P->dy);
        double pz = 0.0;
        int form; /* 0 forward, 1 backward, 2 central */
        if (fd == 0) form = (k == 0) ? 0 : (k == Nz - 1) ? 1 : 2;
        else if (fd == 1) form = (k < Nz - 2) ? 0 : 1;
        else if (fd == -1) form = (k < 2) ? 0 : 1;
        else form = -1;
        if (form == 0) {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            pz = dz_fwd1(pc, p[IX(i, j, k + 1)], p[IX(i, j, k + 2)], a, b);
        } else if (form == 1) {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            pz = dz_bwd1(p[IX(i, j, k - 2)], p[IX(i, j, k - 1)], pc, a2, a1);
        } else if (form == 2) {
            const double a1 = z[k] - z[k - 1], a = z[k + 1] - z[k];
            pz = (p[IX(i, j, k + 1)] - p[IX(i, j, k - 1)]) / (a1 + a);
        }
        if (P->variable_density == 0) rho = P->rho_inf;
        Y[c] -= P->dt * px / rho;
        Y[D.N + c] -= P->dt * py / rho;
        Y[2 * D.N + c] -= P->dt * pz / rho;
    }
    boundary_rules(P, Y);
    for (size_t c = 0; c < D.N; c++) {
        double *T = &Y[3 * D.N + c];
        if (*T < P->T_min) *T = P->T_min;
        if (*T > P->T_max) *T = P->T_max;
    }
    for (size_t c = 0; c < D.NY; c++) {
        double *y = &Y[4 * D.N + c];
        if (*y < P->Y_min) *y = P->Y_min;
        if (*y > P->Y_max) *y = P->Y_max;
    }
}

void wfo_temperature_source(const Parameters *P, double *Y, double t_n1, const double *Ts)
{
    const Dims D = dims_of(P);
    if (!(t_n1 <= P->t_source_end)) return;
    double *T = Y + 3 * D.N;
    if (P->t_source_start <= 0) {
        /* src/cu/functions.cu:382-403 */
        for (size_t c = 0; c < D.N; c++)
            if (Ts[c] > T[c]) T[c] = Ts[c];
        return;
    }
    /* src/cu/functions.cu:325-380 */
    double scale = 1.0;
    if (t_n1 <= P->t_source_start) scale = t_n1 / P->t_source_start;
    const int gauss = strcmp(P->T_source_shape, "gaussian") == 0;
    const int box = strcmp(P->T_source_shape, "parallelepiped") == 0;
    if (!gauss && !box) return;
    for (int i = 0; i < D.Nx; i++)
    for (int j = 0; j < D.Ny; j++)
    for (int k = 0; k < D.Nz; k++) {
        const double x = P->x[i], y = P->y[j], zz = P->z[k];
        double shape;
        if (gauss)
            shape = exp(-pow((x - P->TS_x_center) / P->TS_length, 2.0) - pow((y - P->TS_y_center) / P->TS_width, 2.0)
                        - pow((zz - P->TS_z_center) / P->TS_height, 2.0));
        else
            shape = (x >= P->TS_x_start && x <= P->TS_x_end && y >= P->TS_y_start && y <= P->TS_y_end
                     && zz >= P->TS_z_start && zz <= P->TS_z_end) ? 1.0 : 0.0;
        const double temp = scale * (P->T_inf + (P->T_source - P->T_inf) * shape);
        if (temp > T[IX(i, j, k)]) T[IX(i, j, k)] = temp;
    }
}

/* One step of the loop body in src/cu/solver.cu:178-265 (without I/O). */
int wfo_step(const Parameters *P, double *y, double *p, int n, const double *Ts)
{
    const size_t ns = wfo_state_size(P);
    double *y1 = (double *)malloc(sizeof(double) * ns);
    if (!y1) return -1;
    wfo_time_integrate(P, P->t ? P->t[n - 1] : 0.0, y, y1);
    double err;
    wfo_solve_pressure(P, y1, y, p, &err);
    wfo_project(P, y1, y, p);
    const double tn1 = P->t ? P->t[n] : P->t_min + n * P->dt;
    if (tn1 <= P->t_source_end) wfo_temperature_source(P, y1, tn1, Ts);
    memcpy(y, y1, sizeof(double) * ns);
    free(y1);
    return 0;
}

/* ---- derived arrays: src/cu/parameters.cu:416-523, utils.cu:32-51,
 *      functions.cu:58-80, ibm.cu:3-95 ------------------------------------ */
static void fft_freq_r(double *f, int N, double d)
{
    if (N % 2 == 0) {
        const int n = N / 2;
        for (int i = 0; i < n; i++) f[i] = i / (N * d);
        for (int i = n; i < N; i++) f[i] = (i - N) / (N * d);
    } else {
        const int n = (N - 1) / 2;
        for (int i = 0; i <= n; i++) f[i] = i / (N * d);
        for (int i = n + 1; i < N; i++) f[i] = (i - N) / (N * d);
    }
}

int wfo_fill_derived(Parameters *P, const double *topo)
{
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz, Nt = P->Nt;
    if (Nx < 4 || Ny < 4 || Nz < 4 || Nt < 1) return -1;
    P->x = (double *)malloc(sizeof(double) * Nx);
    P->y = (double *)malloc(sizeof(double) * Ny);
    P->z = (double *)malloc(sizeof(double) * Nz);
    P->t = (double *)malloc(sizeof(double) * (Nt + 1));
    P->r = (double *)malloc(sizeof(double) * (Nx - 1));
    P->s = (double *)malloc(sizeof(double) * (Ny - 1));
    P->kx = (double *)malloc(sizeof(double) * (Nx - 1));
    P->ky = (double *)malloc(sizeof(double) * (Ny - 1));
    P->cut_nodes = (int *)malloc(sizeof(int) * Nx * Ny);
    P->z_ibm = (double *)malloc(sizeof(double) * (size_t)Nx * Ny * Nz);
    P->topography = (double *)malloc(sizeof(double) * Nx * Ny);
    P->Nz_Y = (int *)malloc(sizeof(int) * Nx * Ny);
    P->dx = (P->x_max - P->x_min) / (Nx - 1);
    P->dy = (P->y_max - P->y_min) / (Ny - 1);
    P->dz = (P->z_max - P->z_min) / (Nz - 1);
    P->dt = (P->t_max - P->t_min) / Nt;
    fft_freq_r(P->r, Nx - 1, 1.0 / (Nx - 1));
    fft_freq_r(P->s, Ny - 1, 1.0 / (Ny - 1));
    for (int n = 0; n <= Nt; n++) P->t[n] = P->t_min + n * P->dt;
    for (int i = 0; i < Nx; i++) {
        P->x[i] = P->x_min + i * P->dx;
        if (i < Nx - 1) P->kx[i] = 2 * PI_D * P->r[i] / (P->x_max - P->x_min);
    }
    for (int j = 0; j < Ny; j++) {
        P->y[j] = P->y_min + j * P->dy;
        if (j < Ny - 1) P->ky[j] = 2 * PI_D * P->s[j] / (P->y_max - P->y_min);
    }
    if (P->z_domain == 0) {
        for (int k = 0; k < Nz; k++) P->z[k] = P->z_min + k * P->dz;
    } else if (P->z_domain == 1) {
        const double dz = (P->z_max - P->z_min) / (Nz - 1);
        for (int k = 0; k < Nz; k++)
            P->z[k] = (P->z_max - P->z_min) * (exp(P->k_nu_grid * k * dz / (P->z_max - P->z_min)) - 1)
                      / (exp(P->k_nu_grid) - 1) + P->z_min;
    } else if (P->z_domain == 2) {
        const double dz1 = (P->z_transition - P->z_min) / (P->k_transition - 1);
        const double dz2 = (P->z_max - P->z_transition) / (Nz - P->k_transition - 1);
        for (int k = 0; k < Nz; k++)
            P->z[k] = (k <= P->k_transition) ? P->z_min + k * dz1 : P->z_transition + (k - P->k_transition) * dz2;
    }
    P->T0_x_center = (P->T0_x_start + P->T0_x_end) / 2;
    P->T0_y_center = (P->T0_y_start + P->T0_y_end) / 2;
    P->T0_z_center = 0.0;
    P->T0_length = P->T0_x_end - P->T0_x_start;
    P->T0_width = P->T0_y_end - P->T0_y_start;
    P->T0_height = P->T0_z_end - P->T0_z_start;
    P->TS_x_center = (P->TS_x_start + P->TS_x_end) / 2.0;
    P->TS_y_center = (P->TS_y_start + P->TS_y_end) / 2.0;
    P->TS_z_center = 0.0;
    P->TS_length = P->TS_x_end - P->TS_x_start;
    P->TS_width = P->TS_y_end - P->TS_y_start;
    P->TS_height = P->TS_z_end - P->TS_z_start;
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            double h = 0.0;
            if (topo) h = topo[(size_t)j + (size_t)Ny * i];
            else if (strcmp(P->topo_shape, "hill") == 0)
                h = P->hill_height * exp(-pow((P->x[i] - P->hill_center_x) / P->hill_length, 2.0)
                                         - pow((P->y[j] - P->hill_center_y) / P->hill_width, 2.0)
                                         - pow((0 - 0) / 1.0, 2.0));
            P->topography[(size_t)j + (size_t)Ny * i] = h;
        }
    int nzy_max = 0;
    for (int i = 0; i < Nx; i++)
        for (int j = 0; j < Ny; j++) {
            const size_t cc = (size_t)j + (size_t)Ny * i;
            const double topo_h = P->topography[cc];
            P->cut_nodes[cc] = 0;
            P->Nz_Y[cc] = 0;
            for (int k = 0; k < Nz; k++) {
                const double dz = (k < Nz - 1) ? P->z[k + 1] - P->z[k] : P->z[k] - P->z[k - 1];
                if ((topo_h - dz) <= P->z[k] && P->z[k] <= topo_h) P->cut_nodes[cc] = k;
                P->z_ibm[(size_t)k + (size_t)Nz * cc] = MAXD(P->z[k] - topo_h, 0.0);
                if (P->z[k] <= topo_h + P->Y_h) P->Nz_Y[cc] = k + 1;
            }
            nzy_max = MAXD(nzy_max, P->Nz_Y[cc]);
        }
    P->Nz_Y_max = nzy_max;
    const int size = Nx * Ny * Nz;
    P->field_indexes.u = 0;
    P->field_indexes.v = size;
    P->field_indexes.w = 2 * size;
    P->field_indexes.T = 3 * size;
    P->field_indexes.Y = 4 * size;
    return 0;
}

void wfo_free_derived(Parameters *P)
{
    free(P->x); free(P->y); free(P->z); free(P->t); free(P->r); free(P->s);
    free(P->kx); free(P->ky); free(P->cut_nodes); free(P->z_ibm); free(P->topography); free(P->Nz_Y);
    P->x = P->y = P->z = P->t = P->r = P->s = P->kx = P->ky = P->z_ibm = P->topography = NULL;
    P->cut_nodes = P->Nz_Y = NULL;
}
