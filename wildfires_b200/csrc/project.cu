// project.cu -- end-of-step pass: pressure projection, boundary/IBM rules on
// the state, clamps and the temperature source, fused per column.
//
// Reference sequence (src/cu/solver.cu:205-223): velocity_correction
// (pde.cu:789-908), boundary_conditions on y_{n+1} (pde.cu:14-99), bounds
// (pde.cu:101-137), temperature_source[_delay] (functions.cu:325-403).  One
// block owns one (i,j) column and its threads run along k, the contiguous
// direction of the state, so every access of the column is coalesced.  The
// projection is computed in FP64 whatever the stencil precision.
#include <math.h>

#include "wf_internal.h"

namespace wf {

namespace {

__device__ __forceinline__ int wrap_p(int v, int n)
{
    if (v >= n) v -= n;
    if (v < 0) v += n;
    return v;
}

// One block per (i,j) column (grid Ny x Nx), one thread per cell (blockDim = Nz
// rounded up to a warp).  Every thread loads its cell once; the column's pressure, corrected
// velocity and raw T, Y go through shared memory so that the z-derivative of p
// and the boundary rules (which read the cells next to the cut node and below
// the top) need no second trip to global memory.  The pass is bound by
// instruction issue, so the FP32 path takes its constants (0.5/dx, 0.5/dy,
// dt/rho_inf, dt/(T_inf rho_inf), the top-plane weights) from the host and the
// column's (i, j) from the 2-D grid, and its instantiation is compiled for 40
// registers (12 column blocks of 128 threads per SM, almost no spills):
// 0.502 -> 0.395 ms at 512x512x128 (32 registers: 0.446 ms, 54: 0.438 ms).
template <class R>
__global__ void __launch_bounds__(512, sizeof(R) == 4 ? 3 : 0) k_project(const ProjectArgs<R> a)
{
    extern __shared__ double sh[];
    const Geom &g = a.g;
    const Phys &ph = a.ph;
    const int i = blockIdx.y, j = blockIdx.x;   // grid (Ny, Nx): no division for the column's (i, j)
    const int k = threadIdx.x;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const int col = i * Ny + j;
    const int ip1 = wrap_p(i + 1, Nx - 1), im1 = wrap_p(i - 1, Nx - 1);
    const int jp1 = wrap_p(j + 1, Ny - 1), jm1 = wrap_p(j - 1, Ny - 1);
    const size_t cb = (size_t)col * Nz;
    const size_t xp = ((size_t)ip1 * Ny + j) * Nz, xm = ((size_t)im1 * Ny + j) * Nz;
    const size_t yp = ((size_t)i * Ny + jp1) * Nz, ym = ((size_t)i * Ny + jm1) * Nz;
    const double *__restrict__ p = a.p;
    const double *__restrict__ z = g.z;
    R *__restrict__ y = a.y;
    R *__restrict__ Yc = y + 4 * (size_t)N + (size_t)col * g.NzY;
    double *sp = sh, *su = sh + Nz, *sv = su + Nz, *sw = sv + Nz, *sT = sw + Nz, *sY = sT + Nz;
    const bool live = k < Nz;
    const bool hasY = k < g.NzY;
    const int kc = __ldg(g.cut + col), nzy = __ldg(g.nzy + col);

    double pc = 0.0, pxp = 0.0, pxm = 0.0, pyp = 0.0, pym = 0.0;
    R uo = R(0), vo = R(0), wo = R(0), To = R(0), Yo = R(0);
    if (live) {
        pc = p[cb + k];
        pxp = p[xp + k];
        pxm = p[xm + k];
        pyp = p[yp + k];
        pym = p[ym + k];
        uo = y[cb + k];
        vo = y[(size_t)N + cb + k];
        wo = y[2 * (size_t)N + cb + k];
        To = y[3 * (size_t)N + cb + k];
        if (hasY) Yo = Yc[k];
        sp[k] = pc;
    }
    __syncthreads();
    // 1. u -= dt grad p / rho (pde.cu:812-907).  The FP64 path evaluates the
    //    reference's expressions; the FP32 stencil path, whose result is rounded
    //    to FP32 anyway, uses the precomputed z weights and host-computed
    //    constants (dt/rho = T_n dt/(T_inf rho_inf): no division per cell).
    R un = R(0), vn = R(0), wn = R(0);
    if (live) {
        const int fd = ph.velocity_correction_fd;
        int form;  // 0 forward, 1 backward, 2 central, -1 none
        if (fd == 0) form = (k == 0) ? 0 : (k == Nz - 1) ? 1 : 2;
        else if (fd == 1) form = (k < Nz - 2) ? 0 : 1;
        else if (fd == -1) form = (k < 2) ? 0 : 1;
        else form = -1;
        if constexpr (sizeof(R) == 4) {
            const double *zc = g.zc;
            double s_rho = a.s_rho0;
            if (ph.variable_density != 0) s_rho = a.s_rhoT * (double)a.yn[3 * (size_t)N + cb + k];
            double pz = 0.0;
            if (form == 0)
                pz = zc[ZF0 * Nz + k] * pc + zc[ZF1 * Nz + k] * sp[k + 1] + zc[ZF2 * Nz + k] * sp[k + 2];
            else if (form == 1)
                pz = zc[ZB0 * Nz + k] * sp[k - 2] + zc[ZB1 * Nz + k] * sp[k - 1] + zc[ZB2 * Nz + k] * pc;
            else if (form == 2)
                pz = (sp[k + 1] - sp[k - 1]) * zc[ZC * Nz + k];
            un = (R)((double)uo - s_rho * ((pxp - pxm) * a.hx));
            vn = (R)((double)vo - s_rho * ((pyp - pym) * a.hy));
            wn = (R)((double)wo - s_rho * pz);
        } else {
            const double px = (pxp - pxm) / (2 * ph.dx);
            const double py = (pyp - pym) / (2 * ph.dy);
            double pz = 0.0;
            if (form == 0) {
                const double A = z[k + 1] - z[k], B = z[k + 2] - z[k + 1];
                pz = -(2 * A + B) * pc / (A * (A + B)) + (A + B) * sp[k + 1] / (A * B) - A * sp[k + 2] / (B * (A + B));
            } else if (form == 1) {
                const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
                pz = a1 * sp[k - 2] / (a2 * (a2 + a1)) - (a2 + a1) * sp[k - 1] / (a2 * a1) +
                     (a2 + 2 * a1) * pc / (a1 * (a2 + a1));
            } else if (form == 2) {
                const double a1 = z[k] - z[k - 1], A = z[k + 1] - z[k];
                pz = (sp[k + 1] - sp[k - 1]) / (a1 + A);
            }
            double rho = ph.rho_inf;
            if (ph.variable_density != 0) rho = ph.T_inf * ph.rho_inf / (double)a.yn[3 * (size_t)N + cb + k];
            un = (R)((double)uo - ph.dt * px / rho);
            vn = (R)((double)vo - ph.dt * py / rho);
            wn = (R)((double)wo - ph.dt * pz / rho);
        }
        su[k] = (double)un;
        sv[k] = (double)vn;
        sw[k] = (double)wn;
        sT[k] = (double)To;
        sY[k] = hasY ? (double)Yo : 0.0;
    }
    __syncthreads();
    if (!live) return;
    // 2. boundary rules on the state (the rules applied to the right-hand side)
    R uf = un, vf = vn, wf = wn, Tf = To, Yf = Yo;
    if (k == kc) {
        const double A = z[kc + 1] - z[kc], B = z[kc + 2] - z[kc + 1];
        const double T1 = sT[kc + 1], T2 = sT[kc + 2];
        const double Y1 = (kc + 1 < nzy) ? sY[kc + 1] : 0.0;
        const double Y2 = (kc + 2 < nzy) ? sY[kc + 2] : 0.0;
        uf = R(0);
        vf = R(0);
        wf = R(0);
        Tf = (R)(((A + B) * (A + B) * T1 - A * A * T2) / (B * (2 * A + B)));
        if (kc < nzy) Yf = (R)(((A + B) * (A + B) * Y1 - A * A * Y2) / (B * (2 * A + B)));
    } else if (k == Nz - 1) {
        if constexpr (sizeof(R) == 4) {
            // the same extrapolation with host-computed weights (no divisions)
            const double w1 = ph.top_w1, w2 = ph.top_w2;
            uf = (R)(w1 * su[k - 1] - w2 * su[k - 2]);
            vf = (R)(w1 * sv[k - 1] - w2 * sv[k - 2]);
            wf = (R)(w1 * sw[k - 1] - w2 * sw[k - 2]);
            Tf = (R)(w1 * sT[k - 1] - w2 * sT[k - 2]);
        } else {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            const double num = (a2 + a1) * (a2 + a1), den = a2 * (a2 + 2 * a1), a1s = a1 * a1;
            uf = (R)((num * su[k - 1] - a1s * su[k - 2]) / den);
            vf = (R)((num * sv[k - 1] - a1s * sv[k - 2]) / den);
            wf = (R)((num * sw[k - 1] - a1s * sw[k - 2]) / den);
            Tf = (R)((num * sT[k - 1] - a1s * sT[k - 2]) / den);
        }
    } else if (k < kc) {
        uf = (R)ph.u_dead;
        vf = (R)ph.v_dead;
        wf = (R)ph.w_dead;
        Tf = (R)ph.T_dead;
        if (k < nzy) Yf = (R)ph.Y_dead;
    }
    // 3. clamps (pde.cu:116-136), then the temperature source
    if (Tf < (R)ph.T_min) Tf = (R)ph.T_min;
    if (Tf > (R)ph.T_max) Tf = (R)ph.T_max;
    if (a.source_mode == 1) {
        const R ts = a.Tsrc[cb + k];
        if (ts > Tf) Tf = ts;
    } else if (a.source_mode == 2) {
        const double xx = a.xg[i], yy = a.yg[j], zz = z[k];
        double shape;
        if (a.TS_gauss) {
            const double ex = (xx - a.TS[2]) / a.TS[3], ey = (yy - a.TS[6]) / a.TS[7], ez = (zz - a.TS[10]) / a.TS[11];
            shape = exp(-pow(ex, 2.0) - pow(ey, 2.0) - pow(ez, 2.0));
        } else {
            shape = (xx >= a.TS[0] && xx <= a.TS[1] && yy >= a.TS[4] && yy <= a.TS[5] && zz >= a.TS[8] &&
                     zz <= a.TS[9]) ? 1.0 : 0.0;
        }
        const double temp = a.src_scale * (ph.T_inf + (a.T_source - ph.T_inf) * shape);
        if (temp > (double)Tf) Tf = (R)temp;
    }
    y[cb + k] = uf;
    y[(size_t)N + cb + k] = vf;
    y[2 * (size_t)N + cb + k] = wf;
    if (Tf != To) y[3 * (size_t)N + cb + k] = Tf;
    if (hasY) {
        if (Yf < (R)ph.Y_min) Yf = (R)ph.Y_min;
        if (Yf > (R)ph.Y_max) Yf = (R)ph.Y_max;
        if (Yf != Yo) Yc[k] = Yf;
    }
}

}  // namespace

template <class R> cudaError_t launch_project(const ProjectArgs<R> &a, cudaStream_t s)
{
    const int threads = (a.g.Nz + 31) / 32 * 32;
    if (threads > 512 || a.g.Nx > 65535) return cudaErrorInvalidConfiguration;
    ProjectArgs<R> b = a;
    b.hx = 0.5 / a.ph.dx;
    b.hy = 0.5 / a.ph.dy;
    b.s_rho0 = a.ph.dt / a.ph.rho_inf;
    b.s_rhoT = a.ph.dt / (a.ph.T_inf * a.ph.rho_inf);
    k_project<R><<<dim3(a.g.Ny, a.g.Nx), threads, 6 * (size_t)a.g.Nz * sizeof(double), s>>>(b);
    return cudaGetLastError();
}

template cudaError_t launch_project<double>(const ProjectArgs<double> &, cudaStream_t);
template cudaError_t launch_project<float>(const ProjectArgs<float> &, cudaStream_t);

}  // namespace wf
