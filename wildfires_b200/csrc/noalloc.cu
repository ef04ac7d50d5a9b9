// noalloc.cu -- pressure solve for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside a framework which
// owns all device memory through its own pool, code whose device-memory budget
// is fixed before it starts, or a caller that must not pay for an allocation
// (and the device-wide synchronisation it can imply) on its time-critical path.
// wf_pressure_noalloc gives them the FP64 pressure Poisson solve with every
// piece of scratch it needs -- the half-spectrum buffer, the FFT twiddle,
// chirp and filter tables, the tridiagonal constants and the grid -- placed in
// one file-scope device array of fixed size, g_noalloc_scratch below.  The
// array exists once per device that loads this library and stays allocated
// until the process exits.  Nothing else is allocated on the device.
#include <math.h>
#include <string.h>

#include "wf_internal.h"

namespace {

constexpr size_t kNoallocBytes = (size_t)64 << 20;   // 64 MiB
constexpr size_t kNoallocElems = kNoallocBytes / sizeof(double2);

static __device__ __align__(256) double2 g_noalloc_scratch[kNoallocElems];

constexpr int kMaxDevices = 64;
double2 *g_scratch_ptr[kMaxDevices];     // device address of the array, per device
bool g_ready[kMaxDevices];

// Host staging of the tables (static: no host heap either).
constexpr int kMaxM = 4096;               // longest power-of-two inner FFT length
double2 h_tw[2][kMaxM], h_chirp[2][kMaxM / 2], h_filt[2][kMaxM];
long double h_br[kMaxM], h_bi[kMaxM], h_twr[kMaxM], h_twi[kMaxM];
double h_k2[2][kMaxM / 2];
double h_zt[3 * wf::kMaxZUnknowns + 5];

const long double kPiL = 3.141592653589793238462643383279502884L;

// FFT plan of length n into the static staging tables of slot `w` (0 = x, 1 = y):
// powers of two directly, other lengths by Bluestein with m >= 2n-1.
wf::FftDesc stage_fft_tables(int n, int w)
{
    wf::FftDesc d;
    memset(&d, 0, sizeof(d));
    d.n = n;
    int m = n;
    if ((n & (n - 1)) != 0) {
        m = 1;
        while (m < 2 * n - 1) m <<= 1;
        d.bluestein = 1;
    }
    d.m = m;
    while ((1 << d.L) < m) d.L++;
    for (int j = 0; j < m; j++) {
        const long double a = -2.0L * kPiL * (long double)j / (long double)m;
        h_twr[j] = cosl(a);
        h_twi[j] = sinl(a);
        h_tw[w][j] = make_double2((double)h_twr[j], (double)h_twi[j]);
    }
    if (d.bluestein) {
        for (int j = 0; j < m; j++) h_br[j] = h_bi[j] = 0.0L;
        for (int j = 0; j < n; j++) {
            const long long jj = ((long long)j * j) % (2LL * n);
            const long double a = -kPiL * (long double)jj / (long double)n;
            const long double c = cosl(a), s = sinl(a);
            h_chirp[w][j] = make_double2((double)c, (double)s);
            h_br[j] = c;
            h_bi[j] = -s;
            if (j > 0) {
                h_br[m - j] = c;
                h_bi[m - j] = -s;
            }
        }
        for (int q = 0; q < m; q++) {
            long double sr = 0, si = 0;
            for (int j = 0; j < m; j++) {
                if (h_br[j] == 0.0L && h_bi[j] == 0.0L) continue;
                const int e = (int)(((long long)j * q) % m);
                sr += h_br[j] * h_twr[e] - h_bi[j] * h_twi[e];
                si += h_br[j] * h_twi[e] + h_bi[j] * h_twr[e];
            }
            h_filt[w][q] = make_double2((double)sr, (double)si);
        }
    }
    return d;
}

size_t units(size_t doubles) { return (doubles + 1) / 2; }   // doubles -> double2 slots

}  // namespace

extern "C" wf_status wf_pressure_noalloc(const Parameters *P, const double *y_np1, double *p, void *stream)
{
    using namespace wf;
    if (!P || !y_np1 || !p) {
        set_error("wf_pressure_noalloc: null argument");
        return WF_ERR_ARG;
    }
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz;
    if (Nx < 4 || Ny < 4 || Nz < 5 || !P->z || !P->kx || !P->ky) {
        set_error("wf_pressure_noalloc: grid %dx%dx%d or its derived arrays are not usable", Nx, Ny, Nz);
        return WF_ERR_ARG;
    }
    if (P->variable_density != 0) {
        set_error("wf_pressure_noalloc: only the constant-density solve (variable_density = 0) is available");
        return WF_ERR_ARG;
    }
    if (Nx - 1 > kMaxFftLength || Ny - 1 > kMaxFftLength || Nz - 1 > kMaxZUnknowns) {
        set_error("wf_pressure_noalloc: Nx-1, Ny-1 must be <= %d and Nz-1 <= %d", kMaxFftLength, kMaxZUnknowns);
        return WF_ERR_ARG;
    }
    int dev = 0;
    WF_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("wf_pressure_noalloc: device ordinal %d out of range", dev);
        return WF_ERR_ARG;
    }
    if (!g_ready[dev]) {
        // once per device, with that device current: the array's device address
        double2 *ptr = nullptr;
        WF_TRY_CUDA(cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch));
        WF_TRY_CUDA(poisson_set_attributes<double>());
        g_scratch_ptr[dev] = ptr;
        g_ready[dev] = true;
    }
    double2 *base = g_scratch_ptr[dev];
    cudaStream_t s = (cudaStream_t)stream;

    // layout of the scratch array (double2 slots)
    const int n0 = Nx - 1, n1 = Ny - 1, nk = Nz - 1, h1 = n1 / 2 + 1;
    const FftDesc fx = stage_fft_tables(n0, 0), fy = stage_fft_tables(n1, 1);
    const size_t nG = (size_t)Nz * n0 * h1;
    size_t off = 0;
    const size_t oG = off;       off += nG;
    const size_t oTwx = off;     off += fx.m;
    const size_t oChx = off;     off += fx.bluestein ? (size_t)n0 : 0;
    const size_t oFlx = off;     off += fx.bluestein ? (size_t)fx.m : 0;
    const size_t oTwy = off;     off += fy.m;
    const size_t oChy = off;     off += fy.bluestein ? (size_t)n1 : 0;
    const size_t oFly = off;     off += fy.bluestein ? (size_t)fy.m : 0;
    const size_t oKx = off;      off += units(n0);
    const size_t oKy = off;      off += units(n1);
    const size_t oZt = off;      off += units(3 * (size_t)nk + 5);
    const size_t oZ = off;       off += units(Nz);
    if (off > kNoallocElems) {
        set_error("wf_pressure_noalloc: a %dx%dx%d grid needs %.1f MiB of scratch, the fixed array holds %.0f MiB",
                  Nx, Ny, Nz, off * sizeof(double2) / 1048576.0, kNoallocBytes / 1048576.0);
        return WF_ERR_ARG;
    }

    // tables (tridiagonal constants follow pressure.cu:356-390, see k_p_tridiag)
    for (int i = 0; i < n0; i++) h_k2[0][i] = P->kx[i] * P->kx[i];
    for (int j = 0; j < n1; j++) h_k2[1][j] = P->ky[j] * P->ky[j];
    const double *z = P->z;
    for (int q = 0; q < 3 * nk + 5; q++) h_zt[q] = 0.0;
    for (int k = 0; k + 1 < nk; k++) {
        const double dk = z[k + 1] - z[k], dkp1 = z[k + 2] - z[k + 1];
        h_zt[k] = 2 / (dk * (dk + dkp1));
    }
    for (int k = 1; k + 1 < nk; k++) {
        const double dkm1 = z[k] - z[k - 1], dk = z[k + 1] - z[k];
        h_zt[nk + k] = 2 / (dk * (dkm1 + dk));
    }
    for (int k = 1; k < nk; k++) {
        const double dkm1 = z[k] - z[k - 1], dk = z[k + 1] - z[k];
        h_zt[2 * nk + k] = 2 / (dkm1 * dk);
    }
    const double dz0 = z[1] - z[0], dz1 = z[2] - z[1];
    const double dzNm2 = z[Nz - 2] - z[Nz - 3], dzNm1 = z[Nz - 1] - z[Nz - 2];
    h_zt[3 * nk + 0] = -1.0 / dz0;
    h_zt[3 * nk + 1] = (dz0 + dz1) / (dz0 * dz1);
    h_zt[3 * nk + 2] = 1 / dz1;
    h_zt[3 * nk + 3] = 0.5 * dz0;
    h_zt[3 * nk + 4] = 2 / (dzNm1 * (dzNm2 + dzNm1));

    auto put = [&](size_t o, const void *src, size_t bytes) -> cudaError_t {
        return cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, s);
    };
    cudaError_t e = cudaSuccess;
    if (!e) e = put(oTwx, h_tw[0], sizeof(double2) * fx.m);
    if (!e && fx.bluestein) e = put(oChx, h_chirp[0], sizeof(double2) * n0);
    if (!e && fx.bluestein) e = put(oFlx, h_filt[0], sizeof(double2) * fx.m);
    if (!e) e = put(oTwy, h_tw[1], sizeof(double2) * fy.m);
    if (!e && fy.bluestein) e = put(oChy, h_chirp[1], sizeof(double2) * n1);
    if (!e && fy.bluestein) e = put(oFly, h_filt[1], sizeof(double2) * fy.m);
    if (!e) e = put(oKx, h_k2[0], sizeof(double) * n0);
    if (!e) e = put(oKy, h_k2[1], sizeof(double) * n1);
    if (!e) e = put(oZt, h_zt, sizeof(double) * (3 * (size_t)nk + 5));
    if (!e) e = put(oZ, z, sizeof(double) * Nz);
    // the host tables are static and are refilled by the next call
    if (!e) e = cudaStreamSynchronize(s);
    if (e) {
        set_error("wf_pressure_noalloc: table upload failed: %s", cudaGetErrorString(e));
        return WF_ERR_CUDA;
    }

    PoissonArgs<double> a;
    memset(&a, 0, sizeof(a));
    a.g.Nx = Nx; a.g.Ny = Ny; a.g.Nz = Nz; a.g.NzY = P->Nz_Y_max;
    a.g.N = Nx * Ny * Nz; a.g.NY = Nx * Ny * P->Nz_Y_max;
    a.g.z = reinterpret_cast<const double *>(base + oZ);
    a.ph.dx = P->dx; a.ph.dy = P->dy; a.ph.dt = P->dt; a.ph.rho_inf = P->rho_inf;
    a.ph.variable_density = 0;
    a.y1 = y_np1;
    a.yn = y_np1;
    a.p = p;
    a.G = base + oG;
    a.kx2 = reinterpret_cast<const double *>(base + oKx);
    a.ky2 = reinterpret_cast<const double *>(base + oKy);
    a.fx = fx;
    a.fx.tw = base + oTwx;
    a.fx.chirp = fx.bluestein ? base + oChx : nullptr;
    a.fx.filt = fx.bluestein ? base + oFlx : nullptr;
    a.fy = fy;
    a.fy.tw = base + oTwy;
    a.fy.chirp = fy.bluestein ? base + oChy : nullptr;
    a.fy.filt = fy.bluestein ? base + oFly : nullptr;
    a.h1 = h1;
    e = launch_poisson_impl<double>(a, reinterpret_cast<const double *>(base + oZt), s);
    if (e) {
        set_error("wf_pressure_noalloc: %s", cudaGetErrorString(e));
        return WF_ERR_CUDA;
    }
    return WF_OK;
}
