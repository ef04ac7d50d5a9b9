// diag.cu -- FP64 global diagnostics of a state on the GPU: mass, energy,
// fuel, velocity maxima (CFL), temperature and fuel ranges, NaN count.
//
// The reference reports CFL and T/Y ranges on the host after copying the whole
// state back (src/cu/functions.cu:82-185); it has no mass, energy or fuel
// integrals.  Here the reduction runs on the device in two deterministic
// passes (fixed block partials, then one block), so repeated calls on the same
// state give bit-identical results.
#include <math.h>

#include "wf_internal.h"

namespace wf {

namespace {

constexpr int kDiagBlocks = 592;   // 4 x 148 SMs
constexpr int kDiagThreads = 256;
// partial layout per block: 4 sums, 8 extrema, 1 count
constexpr int kSums = 4, kExt = 8;

struct Part {
    double sum[kSums];     // mass, energy, fuel, volume
    double ext[kExt];      // max|u|, max|v|, max|w|, -T_min, T_max, -Y_min, Y_max, (unused)
    double nan;
};

__device__ __forceinline__ double dmax(double a, double b) { return (b > a || b != b) ? b : a; }

template <class R>
__global__ void __launch_bounds__(kDiagThreads) k_diag_part(const Geom g, const Phys ph, const R *__restrict__ y,
                                                            Part *__restrict__ parts)
{
    const int N = g.N, Nz = g.Nz, Ny = g.Ny, Nx = g.Nx;
    double s[kSums] = {0, 0, 0, 0};
    double e[kExt];
    for (int q = 0; q < kExt; q++) e[q] = -INFINITY;
    double nan = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        const int k = c % Nz, col = c / Nz, j = col % Ny, i = col / Ny;
        const double u = y[c], v = y[(size_t)N + c], w = y[2 * (size_t)N + c], T = y[3 * (size_t)N + c];
        nan += (u != u) + (v != v) + (w != w) + (T != T);
        e[0] = dmax(e[0], fabs(u));
        e[1] = dmax(e[1], fabs(v));
        e[2] = dmax(e[2], fabs(w));
        e[3] = dmax(e[3], -T);
        e[4] = dmax(e[4], T);
        const int nzy = g.nzy[col];
        double Yv = 0.0;
        if (k < nzy) {
            Yv = y[4 * (size_t)N + (size_t)col * g.NzY + k];
            nan += (Yv != Yv);
            e[5] = dmax(e[5], -Yv);
            e[6] = dmax(e[6], Yv);
        }
        // integrals over the periodic cell set (duplicate planes excluded) above the terrain
        if (i < Nx - 1 && j < Ny - 1) {
            const double zl = g.z[k > 0 ? k - 1 : 0], zh = g.z[k < Nz - 1 ? k + 1 : Nz - 1];
            const double dV = ph.dx * ph.dy * 0.5 * (zh - zl);
            if (k >= g.cut[col]) {
                const double rho = ph.T_inf * ph.rho_inf / T;
                s[0] += rho * dV;
                s[1] += rho * ph.c_p * T * dV;
                s[3] += dV;
            }
            if (k < nzy) s[2] += Yv * dV;
        }
    }
    __shared__ double sh[kDiagThreads];
    Part out;
    for (int q = 0; q < kSums + kExt + 1; q++) {
        double v = (q < kSums) ? s[q] : (q < kSums + kExt) ? e[q - kSums] : nan;
        sh[threadIdx.x] = v;
        __syncthreads();
        for (int h = kDiagThreads / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) {
                const double o = sh[threadIdx.x + h];
                sh[threadIdx.x] = (q < kSums || q == kSums + kExt) ? sh[threadIdx.x] + o : dmax(sh[threadIdx.x], o);
            }
            __syncthreads();
        }
        if (q < kSums) out.sum[q] = sh[0];
        else if (q < kSums + kExt) out.ext[q - kSums] = sh[0];
        else out.nan = sh[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) parts[blockIdx.x] = out;
}

__global__ void k_diag_final(const Part *__restrict__ parts, int n, double *__restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Part r = parts[0];
    for (int b = 1; b < n; b++) {
        for (int q = 0; q < kSums; q++) r.sum[q] += parts[b].sum[q];
        for (int q = 0; q < kExt; q++) r.ext[q] = dmax(r.ext[q], parts[b].ext[q]);
        r.nan += parts[b].nan;
    }
    for (int q = 0; q < kSums; q++) out[q] = r.sum[q];
    for (int q = 0; q < kExt; q++) out[kSums + q] = r.ext[q];
    out[kSums + kExt] = r.nan;
}

}  // namespace

size_t diag_scratch_bytes() { return sizeof(Part) * kDiagBlocks + 16 * sizeof(double); }

template <class R>
cudaError_t launch_diag(const Geom &g, const Phys &ph, const R *y, const R *unused, double *scratch, cudaStream_t s)
{
    (void)unused;
    Part *parts = reinterpret_cast<Part *>(scratch + 16);
    k_diag_part<R><<<kDiagBlocks, kDiagThreads, 0, s>>>(g, ph, y, parts);
    k_diag_final<<<1, 32, 0, s>>>(parts, kDiagBlocks, scratch);
    return cudaGetLastError();
}
template cudaError_t launch_diag<double>(const Geom &, const Phys &, const double *, const double *, double *, cudaStream_t);
template cudaError_t launch_diag<float>(const Geom &, const Phys &, const float *, const float *, double *, cudaStream_t);

}  // namespace wf
