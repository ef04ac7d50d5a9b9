// report.cu -- the reference's per-checkpoint report on the GPU.
//
// timestep_reports (reference src/cu/functions.cu:82-185) copies the whole
// state to the host and scans it for: the velocity maxima behind the CFL
// number, the temperature range and the fuel range inside the fuel rectangle
// [Y0_x_start, Y0_x_end] x [Y0_y_start, Y0_y_end], and the first NaN in scan
// order (i, j, k; u, v, w, T, Y), at which it logs the node and exits.  Here
// the same quantities come from a two-pass device reduction (fixed block
// partials, then one block), and only a few doubles cross to the host.
// Kept as the reference has them: the fuel minimum starts at 0 and the
// maximum at -1e9, the temperature range starts at (1e9, -1e9), Y is read for
// every k < Nz_Y_max (the packed Y layout) whatever the column's own Nz_Y.
#include <math.h>

#include "wf_internal.h"

namespace wf {

namespace {

constexpr int kRepBlocks = 592;   // 4 x 148 SMs
constexpr int kRepThreads = 256;

struct RepPart {
    double ext[7];             // max|u|, max|v|, max|w|, -T_min, T_max, -Y_min, Y_max
    unsigned long long nan;    // first NaN as ((i Ny + j) Nz + k) * 5 + field, or ~0
};

// max for the non-NaN values the extrema see (a NaN stops the reference's scan)
__device__ __forceinline__ double rmax(double a, double b) { return b > a ? b : a; }

template <class R>
__global__ void __launch_bounds__(kRepThreads) k_report_part(const Geom g, const R *__restrict__ y,
                                                             const double *__restrict__ xg,
                                                             const double *__restrict__ yg, const double4 rect,
                                                             RepPart *__restrict__ parts)
{
    const int N = g.N, Nz = g.Nz, Ny = g.Ny, NzY = g.NzY;
    double e[7] = {0.0, 0.0, 0.0, -1e9, -1e9, 0.0, -1e9};   // the reference's starting values
    unsigned long long first = ~0ull;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        const int k = c % Nz, col = c / Nz, j = col % Ny, i = col / Ny;
        const double u = y[c], v = y[(size_t)N + c], w = y[2 * (size_t)N + c], T = y[3 * (size_t)N + c];
        double Yv = 0.0;
        if (k < NzY) Yv = y[4 * (size_t)N + (size_t)col * NzY + k];
        const double xi = xg[i], yj = yg[j];
        const bool zone = rect.x <= xi && xi <= rect.y && rect.z <= yj && yj <= rect.w;
        const int f = (u != u) ? 0 : (v != v) ? 1 : (w != w) ? 2 : (T != T) ? 3 : (Yv != Yv) ? 4 : -1;
        if (f >= 0) {
            const unsigned long long key = (unsigned long long)c * 5ull + (unsigned long long)f;
            first = key < first ? key : first;
            continue;
        }
        e[0] = rmax(e[0], fabs(u));
        e[1] = rmax(e[1], fabs(v));
        e[2] = rmax(e[2], fabs(w));
        if (zone) {
            e[3] = rmax(e[3], -T);
            e[4] = rmax(e[4], T);
            if (k < NzY) {
                e[5] = rmax(e[5], -Yv);
                e[6] = rmax(e[6], Yv);
            }
        }
    }
    __shared__ double sh[kRepThreads];
    __shared__ unsigned long long shk[kRepThreads];
    RepPart out;
    for (int q = 0; q < 7; q++) {
        sh[threadIdx.x] = e[q];
        __syncthreads();
        for (int h = kRepThreads / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) sh[threadIdx.x] = rmax(sh[threadIdx.x], sh[threadIdx.x + h]);
            __syncthreads();
        }
        out.ext[q] = sh[0];
        __syncthreads();
    }
    shk[threadIdx.x] = first;
    __syncthreads();
    for (int h = kRepThreads / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) shk[threadIdx.x] = min(shk[threadIdx.x], shk[threadIdx.x + h]);
        __syncthreads();
    }
    out.nan = shk[0];
    if (threadIdx.x == 0) parts[blockIdx.x] = out;
}

// One block: thread t folds partials t, t + 256, ..., then warp butterflies
// and the warps in order (maxima and the smallest key: any order gives the
// same result).
__global__ void __launch_bounds__(kRepThreads) k_report_final(const RepPart *__restrict__ parts, int n,
                                                              double *__restrict__ out)
{
    double e[7];
#pragma unroll
    for (int q = 0; q < 7; q++) e[q] = -INFINITY;
    unsigned long long key = ~0ull;
    for (int b = threadIdx.x; b < n; b += kRepThreads) {
#pragma unroll
        for (int q = 0; q < 7; q++) e[q] = rmax(e[q], parts[b].ext[q]);
        key = min(key, parts[b].nan);
    }
#pragma unroll
    for (int q = 0; q < 7; q++)
        for (int o = 16; o > 0; o >>= 1) e[q] = rmax(e[q], __shfl_xor_sync(0xffffffffu, e[q], o));
    for (int o = 16; o > 0; o >>= 1) key = min(key, __shfl_xor_sync(0xffffffffu, key, o));
    __shared__ double red[kRepThreads / 32][7];
    __shared__ unsigned long long redk[kRepThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 7; q++) red[warp][q] = e[q];
        redk[warp] = key;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        const int q = threadIdx.x;
        double r = red[0][q];
        for (int w = 1; w < kRepThreads / 32; w++) r = rmax(r, red[w][q]);
        out[q] = r;
    } else if (threadIdx.x == 7) {
        unsigned long long k = redk[0];
        for (int w = 1; w < kRepThreads / 32; w++) k = min(k, redk[w]);
        reinterpret_cast<unsigned long long *>(out)[7] = k;
    }
}

}  // namespace

size_t report_scratch_bytes() { return sizeof(RepPart) * kRepBlocks + 8 * sizeof(double); }

template <class R>
cudaError_t launch_report(const Geom &g, const R *y, const double *xg, const double *yg, const double rect[4],
                          double *scratch, cudaStream_t s)
{
    RepPart *parts = reinterpret_cast<RepPart *>(scratch + 8);
    k_report_part<R><<<kRepBlocks, kRepThreads, 0, s>>>(g, y, xg, yg, make_double4(rect[0], rect[1], rect[2], rect[3]),
                                                         parts);
    k_report_final<<<1, kRepThreads, 0, s>>>(parts, kRepBlocks, scratch);
    return cudaGetLastError();
}
template cudaError_t launch_report<double>(const Geom &, const double *, const double *, const double *,
                                           const double *, double *, cudaStream_t);
template cudaError_t launch_report<float>(const Geom &, const float *, const double *, const double *,
                                          const double *, double *, cudaStream_t);

}  // namespace wf
