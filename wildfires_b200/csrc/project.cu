// project.cu -- end-of-step pass: pressure projection, boundary/IBM rules on
// the state, clamps and the temperature source, fused per column.
//
// Reference sequence (src/cu/solver.cu:205-223): velocity_correction
// (pde.cu:789-908), boundary_conditions on y_{n+1} (pde.cu:14-99), bounds
// (pde.cu:101-137), temperature_source[_delay] (functions.cu:325-403).  One warp
// owns one (i,j) column; lanes run along k, which is the contiguous direction
// of the state, so every access of the column is coalesced.  The projection is
// computed in FP64 whatever the stencil precision.
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

template <class R>
__global__ void __launch_bounds__(256) k_project(const ProjectArgs<R> a)
{
    const Geom &g = a.g;
    const Phys &ph = a.ph;
    const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (col >= g.Nx * g.Ny) return;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const int i = col / Ny, j = col % Ny;
    const int ip1 = wrap_p(i + 1, Nx - 1), im1 = wrap_p(i - 1, Nx - 1);
    const int jp1 = wrap_p(j + 1, Ny - 1), jm1 = wrap_p(j - 1, Ny - 1);
    const size_t cb = (size_t)col * Nz;
    const size_t xp = ((size_t)ip1 * Ny + j) * Nz, xm = ((size_t)im1 * Ny + j) * Nz;
    const size_t yp = ((size_t)i * Ny + jp1) * Nz, ym = ((size_t)i * Ny + jm1) * Nz;
    const double *__restrict__ p = a.p;
    const double *z = g.z;
    R *y = a.y;
    const int fd = ph.velocity_correction_fd;
    // 1. u -= dt grad p / rho (pde.cu:812-907)
    for (int k = lane; k < Nz; k += 32) {
        const double pc = p[cb + k];
        const double px = (p[xp + k] - p[xm + k]) / (2 * ph.dx);
        const double py = (p[yp + k] - p[ym + k]) / (2 * ph.dy);
        int form;  // 0 forward, 1 backward, 2 central, -1 none
        if (fd == 0) form = (k == 0) ? 0 : (k == Nz - 1) ? 1 : 2;
        else if (fd == 1) form = (k < Nz - 2) ? 0 : 1;
        else if (fd == -1) form = (k < 2) ? 0 : 1;
        else form = -1;
        double pz = 0.0;
        if (form == 0) {
            const double A = z[k + 1] - z[k], B = z[k + 2] - z[k + 1];
            pz = -(2 * A + B) * pc / (A * (A + B)) + (A + B) * p[cb + k + 1] / (A * B) - A * p[cb + k + 2] / (B * (A + B));
        } else if (form == 1) {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            pz = a1 * p[cb + k - 2] / (a2 * (a2 + a1)) - (a2 + a1) * p[cb + k - 1] / (a2 * a1) +
                 (a2 + 2 * a1) * pc / (a1 * (a2 + a1));
        } else if (form == 2) {
            const double a1 = z[k] - z[k - 1], A = z[k + 1] - z[k];
            pz = (p[cb + k + 1] - p[cb + k - 1]) / (a1 + A);
        }
        double rho = ph.rho_inf;
        if (ph.variable_density != 0) rho = ph.T_inf * ph.rho_inf / (double)a.yn[3 * (size_t)N + cb + k];
        y[cb + k] = (R)((double)y[cb + k] - ph.dt * px / rho);
        y[(size_t)N + cb + k] = (R)((double)y[(size_t)N + cb + k] - ph.dt * py / rho);
        y[2 * (size_t)N + cb + k] = (R)((double)y[2 * (size_t)N + cb + k] - ph.dt * pz / rho);
    }
    __syncwarp();
    // 2. boundary rules on the state (same rules as on the right-hand side)
    const int kc = __ldg(g.cut + col), nzy = __ldg(g.nzy + col);
    R *Yc = y + 4 * (size_t)N + (size_t)col * g.NzY;
    if (lane == 0) {
        const double A = z[kc + 1] - z[kc], B = z[kc + 2] - z[kc + 1];
        const double T1 = y[3 * (size_t)N + cb + kc + 1], T2 = y[3 * (size_t)N + cb + kc + 2];
        const double Y1 = (kc + 1 < nzy) ? (double)Yc[kc + 1] : 0.0;
        const double Y2 = (kc + 2 < nzy) ? (double)Yc[kc + 2] : 0.0;
        y[cb + kc] = R(0);
        y[(size_t)N + cb + kc] = R(0);
        y[2 * (size_t)N + cb + kc] = R(0);
        y[3 * (size_t)N + cb + kc] = (R)(((A + B) * (A + B) * T1 - A * A * T2) / (B * (2 * A + B)));
        if (kc < nzy) Yc[kc] = (R)(((A + B) * (A + B) * Y1 - A * A * Y2) / (B * (2 * A + B)));
    } else if (lane == 1) {
        const int k = Nz - 1;
        const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
        const double num = (a2 + a1) * (a2 + a1), den = a2 * (a2 + 2 * a1), a1s = a1 * a1;
        for (int f = 0; f < 4; f++) {
            const size_t o = (size_t)f * N + cb;
            const double v1 = y[o + k - 1], v2 = y[o + k - 2];
            y[o + k] = (R)((num * v1 - a1s * v2) / den);
        }
    }
    for (int k = lane; k < kc; k += 32) {
        y[cb + k] = (R)ph.u_dead;
        y[(size_t)N + cb + k] = (R)ph.v_dead;
        y[2 * (size_t)N + cb + k] = (R)ph.w_dead;
        y[3 * (size_t)N + cb + k] = (R)ph.T_dead;
        if (k < nzy) Yc[k] = (R)ph.Y_dead;
    }
    __syncwarp();
    // 3. clamps (pde.cu:116-136), then the temperature source
    for (int k = lane; k < Nz; k += 32) {
        R T = y[3 * (size_t)N + cb + k];
        const R T0 = T;
        if (T < (R)ph.T_min) T = (R)ph.T_min;
        if (T > (R)ph.T_max) T = (R)ph.T_max;
        if (a.source_mode == 1) {
            const R ts = a.Tsrc[cb + k];
            if (ts > T) T = ts;
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
            if (temp > (double)T) T = (R)temp;
        }
        if (T != T0) y[3 * (size_t)N + cb + k] = T;
        if (k < g.NzY) {
            R Yv = Yc[k];
            const R Y0 = Yv;
            if (Yv < (R)ph.Y_min) Yv = (R)ph.Y_min;
            if (Yv > (R)ph.Y_max) Yv = (R)ph.Y_max;
            if (Yv != Y0) Yc[k] = Yv;
        }
    }
}

}  // namespace

template <class R> cudaError_t launch_project(const ProjectArgs<R> &a, cudaStream_t s)
{
    const int ncol = a.g.Nx * a.g.Ny;
    const int threads = 256;
    const int blocks = (ncol * 32 + threads - 1) / threads;
    k_project<R><<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

template cudaError_t launch_project<double>(const ProjectArgs<double> &, cudaStream_t);
template cudaError_t launch_project<float>(const ProjectArgs<float> &, cudaStream_t);

}  // namespace wf
