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

// the 13 reduced values of a Part, in its memory order: sums, extrema, NaN count
constexpr int kVals = kSums + kExt + 1;
static_assert(sizeof(Part) == kVals * sizeof(double), "Part is a plain array of doubles");
__host__ __device__ constexpr bool is_sum(int q) { return q < kSums || q == kVals - 1; }
__device__ __forceinline__ double combine(int q, double a, double b) { return is_sum(q) ? a + b : dmax(a, b); }

// Reduces v over the block (warp butterflies, then the warps in order) and
// writes the kVals results to dst.  Every thread of the block must call it.
__device__ __forceinline__ void block_reduce(double (&v)[kVals], double *dst)
{
    __shared__ double red[kDiagThreads / 32][kVals];
#pragma unroll
    for (int q = 0; q < kVals; q++)
        for (int o = 16; o > 0; o >>= 1) v[q] = combine(q, v[q], __shfl_xor_sync(0xffffffffu, v[q], o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < kVals; q++) red[warp][q] = v[q];
    }
    __syncthreads();
    if (threadIdx.x < kVals) {
        const int q = threadIdx.x;
        double r = red[0][q];
        for (int w = 1; w < kDiagThreads / 32; w++) r = combine(q, r, red[w][q]);
        dst[q] = r;
    }
}

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
    double v[kVals];
#pragma unroll
    for (int q = 0; q < kSums; q++) v[q] = s[q];
#pragma unroll
    for (int q = 0; q < kExt; q++) v[kSums + q] = e[q];
    v[kVals - 1] = nan;
    block_reduce(v, reinterpret_cast<double *>(parts + blockIdx.x));
}

// One block: thread t folds partials t, t + 256, ... in that order, then the
// block reduction (a fixed order: results are bit-reproducible).
__global__ void __launch_bounds__(kDiagThreads) k_diag_final(const Part *__restrict__ parts, int n,
                                                             double *__restrict__ out)
{
    double v[kVals];
#pragma unroll
    for (int q = 0; q < kVals; q++) v[q] = is_sum(q) ? 0.0 : -INFINITY;
    for (int b = threadIdx.x; b < n; b += kDiagThreads) {
        const double *pb = reinterpret_cast<const double *>(parts + b);
#pragma unroll
        for (int q = 0; q < kVals; q++) v[q] = combine(q, v[q], pb[q]);
    }
    block_reduce(v, out);
}

}  // namespace

size_t diag_scratch_bytes() { return sizeof(Part) * kDiagBlocks + 16 * sizeof(double); }

template <class R>
cudaError_t launch_diag(const Geom &g, const Phys &ph, const R *y, const R *unused, double *scratch, cudaStream_t s)
{
    (void)unused;
    Part *parts = reinterpret_cast<Part *>(scratch + 16);
    k_diag_part<R><<<kDiagBlocks, kDiagThreads, 0, s>>>(g, ph, y, parts);
    k_diag_final<<<1, kDiagThreads, 0, s>>>(parts, kDiagBlocks, scratch);
    return cudaGetLastError();
}
template cudaError_t launch_diag<double>(const Geom &, const Phys &, const double *, const double *, double *, cudaStream_t);
template cudaError_t launch_diag<float>(const Geom &, const Phys &, const float *, const float *, double *, cudaStream_t);

}  // namespace wf
