// terrain.cu -- terrain and immersed-boundary tables computed on the device.
//
//   k_ibm_tables   one thread per (i, j) column: cut node, fuel storage height
//                  Nz_Y and the height above terrain z_ibm of every node, with
//                  the reference's comparisons (ibm_parameters, src/cu/ibm.cu:
//                  57-95): cut node = the last k with topo - dz_k <= z_k <= topo,
//                  Nz_Y = 1 + the last k with z_k <= topo + Y_h, z_ibm =
//                  max(z_k - topo, 0); dz_k = z_{k+1} - z_k (z_k - z_{k-1} on the
//                  top plane).  Only comparisons and one subtraction per node,
//                  so the tables are bit-identical to the host computation.
//   k_hills        a terrain made of Gaussian hills h exp(-(dx^2 + dy^2) /
//                  (2 w^2)) summed in the order given, with dx, dy the
//                  periodic distances (period x_max - x_min, y_max - y_min) from
//                  the hill centre: the seeded multi-hill terrain of the
//                  benchmark workloads.
// The record's host arrays stay the contract callers may edit: both entry
// points write their results back into them.
#include <math.h>
#include <string.h>

#include "wf_internal.h"

namespace wf {

namespace {

__global__ void __launch_bounds__(128) k_ibm_tables(const double *__restrict__ topo, const double *__restrict__ z,
                                                     int ncol, int Nz, double Y_h, int *__restrict__ cut,
                                                     int *__restrict__ nzy, double *__restrict__ zibm)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    const double t = topo[c];
    int kc = 0, ny = 0;
    double *zi = zibm ? zibm + (size_t)c * Nz : nullptr;
    for (int k = 0; k < Nz; k++) {
        const double zk = z[k];
        const double dz = (k < Nz - 1) ? __dsub_rn(z[k + 1], zk) : __dsub_rn(zk, z[k - 1]);
        if (__dsub_rn(t, dz) <= zk && zk <= t) kc = k;
        if (zi) {
            const double d = __dsub_rn(zk, t);
            zi[k] = d > 0.0 ? d : 0.0;
        }
        if (zk <= __dadd_rn(t, Y_h)) ny = k + 1;
    }
    cut[c] = kc;
    nzy[c] = ny;
}

// periodic offset in [-L/2, L/2) with the floor-modulo of a floating remainder
// (the sign of the divisor), rounded operation by operation
__device__ __forceinline__ double periodic_offset(double a, double L)
{
    double r = fmod(__dadd_rn(a, 0.5 * L), L);
    if (r != 0.0 && (r < 0.0) != (L < 0.0)) r = __dadd_rn(r, L);
    return __dsub_rn(r, 0.5 * L);
}

__global__ void __launch_bounds__(128) k_hills(int Nx, int Ny, double x0, double dx, double y0, double dy, double Lx,
                                                double Ly, int n, const double *__restrict__ hills,
                                                double *__restrict__ topo)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= Nx * Ny) return;
    const int i = c / Ny, j = c % Ny;
    const double x = __dadd_rn(x0, __dmul_rn((double)i, dx)), y = __dadd_rn(y0, __dmul_rn((double)j, dy));
    double h = 0.0;
    for (int q = 0; q < n; q++) {
        const double cx = hills[4 * q], cy = hills[4 * q + 1], hh = hills[4 * q + 2], w = hills[4 * q + 3];
        const double ddx = periodic_offset(__dsub_rn(x, cx), Lx), ddy = periodic_offset(__dsub_rn(y, cy), Ly);
        const double r2 = __dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy));
        h = __dadd_rn(h, __dmul_rn(hh, exp(-r2 / __dmul_rn(2.0, __dmul_rn(w, w)))));
    }
    topo[c] = h;
}

// Device scratch of one call, released on every path.
struct Scratch {
    void *p[6] = {};
    int n = 0;
    void *get(size_t bytes)
    {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes ? bytes : 16) != cudaSuccess) return nullptr;
        p[n++] = q;
        return q;
    }
    ~Scratch()
    {
        for (int q = 0; q < n; q++) cudaFree(p[q]);
    }
};

// the IBM tables of the record's topography, computed on the device and
// written back into the record (topography already on the device in d_topo)
wf_status ibm_on_device(Parameters *P, const double *d_topo, Scratch &s)
{
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz, ncol = Nx * Ny;
    double *d_z = (double *)s.get(sizeof(double) * Nz);
    int *d_cut = (int *)s.get(sizeof(int) * ncol), *d_nzy = (int *)s.get(sizeof(int) * ncol);
    double *d_zibm = P->z_ibm ? (double *)s.get(sizeof(double) * (size_t)ncol * Nz) : nullptr;
    if (!d_z || !d_cut || !d_nzy || (P->z_ibm && !d_zibm)) {
        set_error("terrain: device allocation failed");
        return WF_ERR_OOM;
    }
    WF_TRY_CUDA(cudaMemcpy(d_z, P->z, sizeof(double) * Nz, cudaMemcpyHostToDevice));
    k_ibm_tables<<<(ncol + 127) / 128, 128>>>(d_topo, d_z, ncol, Nz, P->Y_h, d_cut, d_nzy, d_zibm);
    WF_TRY_CUDA(cudaGetLastError());
    WF_TRY_CUDA(cudaMemcpy(P->cut_nodes, d_cut, sizeof(int) * ncol, cudaMemcpyDeviceToHost));
    WF_TRY_CUDA(cudaMemcpy(P->Nz_Y, d_nzy, sizeof(int) * ncol, cudaMemcpyDeviceToHost));
    if (d_zibm) WF_TRY_CUDA(cudaMemcpy(P->z_ibm, d_zibm, sizeof(double) * (size_t)ncol * Nz, cudaMemcpyDeviceToHost));
    int m = 0;
    for (int c = 0; c < ncol; c++) m = P->Nz_Y[c] > m ? P->Nz_Y[c] : m;
    P->Nz_Y_max = m;
    return WF_OK;
}

bool usable(const Parameters *P)
{
    return P && P->Nx >= 4 && P->Ny >= 4 && P->Nz >= 4 && P->topography && P->z && P->cut_nodes && P->Nz_Y;
}

}  // namespace
}  // namespace wf

extern "C" {

wf_status wf_ibm_parameters_device(Parameters *P)
{
    using namespace wf;
    if (!usable(P)) {
        set_error("wf_ibm_parameters_device: invalid argument");
        return WF_ERR_ARG;
    }
    Scratch s;
    double *d_topo = (double *)s.get(sizeof(double) * (size_t)P->Nx * P->Ny);
    if (!d_topo) {
        set_error("wf_ibm_parameters_device: device allocation failed");
        return WF_ERR_OOM;
    }
    WF_TRY_CUDA(cudaMemcpy(d_topo, P->topography, sizeof(double) * (size_t)P->Nx * P->Ny, cudaMemcpyHostToDevice));
    return ibm_on_device(P, d_topo, s);
}

wf_status wf_set_topography_hills(Parameters *P, int n, const double *hills)
{
    using namespace wf;
    if (!usable(P) || n < 0 || (n > 0 && !hills)) {
        set_error("wf_set_topography_hills: invalid argument");
        return WF_ERR_ARG;
    }
    const int ncol = P->Nx * P->Ny;
    Scratch s;
    double *d_topo = (double *)s.get(sizeof(double) * ncol);
    double *d_hills = (double *)s.get(sizeof(double) * 4 * (n > 0 ? n : 1));
    if (!d_topo || !d_hills) {
        set_error("wf_set_topography_hills: device allocation failed");
        return WF_ERR_OOM;
    }
    if (n > 0) WF_TRY_CUDA(cudaMemcpy(d_hills, hills, sizeof(double) * 4 * n, cudaMemcpyHostToDevice));
    k_hills<<<(ncol + 127) / 128, 128>>>(P->Nx, P->Ny, P->x_min, P->dx, P->y_min, P->dy, P->x_max - P->x_min,
                                         P->y_max - P->y_min, n, d_hills, d_topo);
    WF_TRY_CUDA(cudaGetLastError());
    WF_TRY_CUDA(cudaMemcpy(P->topography, d_topo, sizeof(double) * ncol, cudaMemcpyDeviceToHost));
    return ibm_on_device(P, d_topo, s);
}

}  // extern "C"
