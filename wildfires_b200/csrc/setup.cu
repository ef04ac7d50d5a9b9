// setup.cu -- the reference's initial conditions generated on the device.
//
// The reference builds u, v, w, T, Y and p on the host (initial_conditions,
// src/cu/functions.cu:187-323), packs them (create_y_0, solver.cu:41-56) and
// copies the packed state to the GPU (main.cu:44-73).  Here one kernel writes
// the packed state (in the context's precision) and p straight into HBM, one
// thread per cell, with the reference's expressions in FP64:
//   u = u_r (z/z_r)^alpha_u (power_law, functions.cu:18-20), v = w = 0;
//   T = T_inf + (T_0 - T_inf) * gaussian | parallelepiped (functions.cu:22-32);
//   p = p_top on the top plane, else 0;
//   Y = 1 inside the fuel rectangle up to topography + Y_h and under the four
//   linear ramps of widths Y0_xa, Y0_ya around it, for k < Nz_Y(i, j);
//   dead nodes (k < cut node) take the *_dead_nodes values (Y only below the
//   column's fuel top).
// Y entries the reference leaves unwritten (its Y array comes from malloc) are
// written as 0 here.  The products are rounded separately (no fused
// multiply-add), as the reference's host build computes them.
#include <math.h>

#include "wf_internal.h"

namespace wf {

namespace {

template <class R>
__global__ void __launch_bounds__(256) k_initial_conditions(const Geom g, const IcArgs a, const double *__restrict__ xg,
                                                            const double *__restrict__ yg, R *__restrict__ st,
                                                            double *__restrict__ p)
{
    const int N = g.N, Nz = g.Nz, Ny = g.Ny, NzY = g.NzY;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        const int k = c % Nz, col = c / Nz, j = col % Ny, i = col / Ny;
        const double x = xg[i], y = yg[j], z = g.z[k];
        double u = a.u_r * pow(z / a.z_r, a.alpha_u);
        double v = 0.0, w = 0.0;
        double shape;
        if (a.T_shape == 0)
            shape = exp(-pow((x - a.x0) / a.sx, 2.0) - pow((y - a.y0) / a.sy, 2.0) - pow((z - a.z0) / a.sz, 2.0));
        else
            shape = (x >= a.Tx0 && x <= a.Tx1 && y >= a.Ty0 && y <= a.Ty1 && z >= a.Tz0 && z <= a.Tz1) ? 1.0 : 0.0;
        double T = __dadd_rn(a.T_inf, __dmul_rn(a.T_0 - a.T_inf, shape));
        p[c] = (k == Nz - 1) ? a.p_top : 0.0;
        const int nzy = g.nzy[col], cut = g.cut[col];
        double Y = 0.0;
        if (k < nzy) {
            const double Yh = a.Y_h, xa = a.xa, ya = a.ya;
            const double z_bottom = __ddiv_rn(__dmul_rn(Yh, (y - a.Yy0) + ya), ya);
            const double z_top = __ddiv_rn(__dmul_rn(Yh, (a.Yy1 + ya) - y), ya);
            const double z_left = __ddiv_rn(__dmul_rn(Yh, (x - a.Yx0) + xa), xa);
            const double z_right = __ddiv_rn(__dmul_rn(Yh, (a.Yx1 + xa) - x), xa);
            const bool xin = a.Yx0 - xa <= x && x <= a.Yx1 + xa, yin = a.Yy0 - ya <= y && y <= a.Yy1 + ya;
            if (a.Yx0 <= x && x <= a.Yx1 && a.Yy0 <= y && y <= a.Yy1 && 0 <= z && z <= g.topo[col] + Yh)
                Y = 1.0;
            else if (a.Yy0 - ya <= y && y < a.Yy0 && xin && 0 <= z && z <= z_bottom)
                Y = 1.0;
            else if (a.Yy1 < y && y <= a.Yy1 + ya && xin && 0 <= z && z <= z_top)
                Y = 1.0;
            else if (a.Yx0 - xa <= x && x < a.Yx0 && yin && 0 <= z && z <= z_left)
                Y = 1.0;
            else if (a.Yx1 < x && x <= a.Yx1 + xa && yin && 0 <= z && z <= z_right)
                Y = 1.0;
        }
        if (k < cut) {
            u = a.dead[0];
            v = a.dead[1];
            w = a.dead[2];
            T = a.dead[3];
            if (k < nzy) Y = a.dead[4];
        }
        st[c] = (R)u;
        st[(size_t)N + c] = (R)v;
        st[2 * (size_t)N + c] = (R)w;
        st[3 * (size_t)N + c] = (R)T;
        if (k < NzY) st[4 * (size_t)N + (size_t)col * NzY + k] = (R)Y;
    }
}

}  // namespace

template <class R>
cudaError_t launch_initial_conditions(const Geom &g, const IcArgs &a, const double *xg, const double *yg, R *state,
                                      double *p, cudaStream_t s)
{
    k_initial_conditions<R><<<592, 256, 0, s>>>(g, a, xg, yg, state, p);
    return cudaGetLastError();
}
template cudaError_t launch_initial_conditions<double>(const Geom &, const IcArgs &, const double *, const double *,
                                                       double *, double *, cudaStream_t);
template cudaError_t launch_initial_conditions<float>(const Geom &, const IcArgs &, const double *, const double *,
                                                      float *, double *, cudaStream_t);

}  // namespace wf
