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

#include <mutex>

#include "wf_internal.h"

namespace {

constexpr size_t kNoallocBytes = (size_t)64 << 20;   // 64 MiB
constexpr size_t kNoallocElems = kNoallocBytes / sizeof(double2);

static __device__ __align__(256) double2 g_noalloc_scratch[kNoallocElems];

constexpr int kMaxDevices = 64;
constexpr int kMaxM = 4096;               // longest power-of-two inner FFT length

// Offsets (double2 slots) of the pieces of the scratch array for one grid.
struct Layout {
    size_t G, twx, chx, flx, twy, chy, fly, kx, ky, zt, z, total;
};

// What the tables held in one device's array were built for: the grid shape
// and the grid arrays the tables depend on (z, kx, ky).
struct TableKey {
    int Nx, Ny, Nz;
    double z[wf::kMaxZUnknowns + 1];
    double kx[wf::kMaxFftLength], ky[wf::kMaxFftLength];
};

struct DeviceSlot {
    bool ready;            // array address looked up, kernels configured
    bool tables;           // `key` describes the tables in the array
    double2 *base;         // device address of g_noalloc_scratch on this device
    TableKey key;
    wf::FftDesc fx, fy;    // descriptors with device table pointers
};
DeviceSlot g_slot[kMaxDevices];

// Serialises the host side (set-up, cache check, table staging) of calls from
// different host threads; the GPU work itself is not serialised by it.
std::mutex g_lock;

// Host staging of the tables (static: no host heap either).
double2 h_tw[2][kMaxM], h_chirp[2][kMaxM / 2], h_filt[2][kMaxM];
long double h_br[kMaxM], h_bi[kMaxM], h_twr[kMaxM], h_twi[kMaxM];
double h_k2[2][kMaxM / 2];
double h_zt[3 * wf::kMaxZUnknowns + 5];

const long double kPiL = 3.141592653589793238462643383279502884L;

// inner power-of-two FFT length of a transform of length n: n itself, or the
// Bluestein length >= 2n-1
int inner_length(int n)
{
    if ((n & (n - 1)) == 0) return n;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    return m;
}

size_t units(size_t doubles) { return (doubles + 1) / 2; }   // doubles -> double2 slots

Layout layout_of(int Nx, int Ny, int Nz)
{
    const int n0 = Nx - 1, n1 = Ny - 1, nk = Nz - 1, h1 = n1 / 2 + 1;
    const int m0 = inner_length(n0), m1 = inner_length(n1);
    const bool b0 = m0 != n0, b1 = m1 != n1;
    Layout l;
    size_t off = 0;
    l.G = off;   off += (size_t)Nz * n0 * h1;
    l.twx = off; off += m0;
    l.chx = off; off += b0 ? (size_t)n0 : 0;
    l.flx = off; off += b0 ? (size_t)m0 : 0;
    l.twy = off; off += m1;
    l.chy = off; off += b1 ? (size_t)n1 : 0;
    l.fly = off; off += b1 ? (size_t)m1 : 0;
    l.kx = off;  off += units(n0);
    l.ky = off;  off += units(n1);
    l.zt = off;  off += units(3 * (size_t)nk + 5);
    l.z = off;   off += units(Nz);
    l.total = off;
    return l;
}

// FFT plan of length n into the static staging tables of slot `w` (0 = x, 1 = y):
// powers of two directly, other lengths by Bluestein with m >= 2n-1.
wf::FftDesc stage_fft_tables(int n, int w)
{
    wf::FftDesc d;
    memset(&d, 0, sizeof(d));
    d.n = n;
    d.m = inner_length(n);
    d.bluestein = d.m != n;
    const int m = d.m;
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

bool same_key(const TableKey &k, const Parameters *P)
{
    return k.Nx == P->Nx && k.Ny == P->Ny && k.Nz == P->Nz && !memcmp(k.z, P->z, sizeof(double) * P->Nz) &&
           !memcmp(k.kx, P->kx, sizeof(double) * (P->Nx - 1)) && !memcmp(k.ky, P->ky, sizeof(double) * (P->Ny - 1));
}

// Build the tables of grid P on the host and copy them into the device array
// (slot's base), then wait for the copies: the host staging tables are reused
// by the next rebuild.
wf_status build_tables(DeviceSlot &slot, const Parameters *P, const Layout &l, cudaStream_t s)
{
    using namespace wf;
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz;
    const int n0 = Nx - 1, n1 = Ny - 1, nk = Nz - 1;
    slot.tables = false;
    FftDesc fx = stage_fft_tables(n0, 0), fy = stage_fft_tables(n1, 1);
    // tridiagonal constants follow pressure.cu:356-390 (see k_p_tridiag)
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

    double2 *base = slot.base;
    auto put = [&](size_t o, const void *src, size_t bytes) -> cudaError_t {
        return cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, s);
    };
    cudaError_t e = cudaSuccess;
    if (!e) e = put(l.twx, h_tw[0], sizeof(double2) * fx.m);
    if (!e && fx.bluestein) e = put(l.chx, h_chirp[0], sizeof(double2) * n0);
    if (!e && fx.bluestein) e = put(l.flx, h_filt[0], sizeof(double2) * fx.m);
    if (!e) e = put(l.twy, h_tw[1], sizeof(double2) * fy.m);
    if (!e && fy.bluestein) e = put(l.chy, h_chirp[1], sizeof(double2) * n1);
    if (!e && fy.bluestein) e = put(l.fly, h_filt[1], sizeof(double2) * fy.m);
    if (!e) e = put(l.kx, h_k2[0], sizeof(double) * n0);
    if (!e) e = put(l.ky, h_k2[1], sizeof(double) * n1);
    if (!e) e = put(l.zt, h_zt, sizeof(double) * (3 * (size_t)nk + 5));
    if (!e) e = put(l.z, z, sizeof(double) * Nz);
    if (!e) e = cudaStreamSynchronize(s);
    if (e) {
        set_error("wf_pressure_noalloc: table upload failed: %s", cudaGetErrorString(e));
        return WF_ERR_CUDA;
    }
    fx.tw = base + l.twx;
    fx.chirp = fx.bluestein ? base + l.chx : nullptr;
    fx.filt = fx.bluestein ? base + l.flx : nullptr;
    fy.tw = base + l.twy;
    fy.chirp = fy.bluestein ? base + l.chy : nullptr;
    fy.filt = fy.bluestein ? base + l.fly : nullptr;
    slot.fx = fx;
    slot.fy = fy;
    slot.key.Nx = Nx;
    slot.key.Ny = Ny;
    slot.key.Nz = Nz;
    memcpy(slot.key.z, z, sizeof(double) * Nz);
    memcpy(slot.key.kx, P->kx, sizeof(double) * n0);
    memcpy(slot.key.ky, P->ky, sizeof(double) * n1);
    slot.tables = true;
    return WF_OK;
}

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
    // the size check needs no table and no CUDA call
    const Layout l = layout_of(Nx, Ny, Nz);
    if (l.total > kNoallocElems) {
        set_error("wf_pressure_noalloc: a %dx%dx%d grid needs %.1f MiB of scratch, the fixed array holds %.0f MiB",
                  Nx, Ny, Nz, l.total * sizeof(double2) / 1048576.0, kNoallocBytes / 1048576.0);
        return WF_ERR_ARG;
    }
    int dev = 0;
    WF_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("wf_pressure_noalloc: device ordinal %d out of range", dev);
        return WF_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    FftDesc fx, fy;
    double2 *base = nullptr;
    {
        std::lock_guard<std::mutex> hold(g_lock);
        DeviceSlot &slot = g_slot[dev];
        if (!slot.ready) {
            // once per device, with that device current: the array's device address
            double2 *ptr = nullptr;
            WF_TRY_CUDA(cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch));
            WF_TRY_CUDA(poisson_set_attributes<double>());
            slot.base = ptr;
            slot.tables = false;
            slot.ready = true;
        }
        // the tables stay in the array from one call to the next; they are
        // rebuilt (and the call waits for their upload) only when the grid changes
        if (!slot.tables || !same_key(slot.key, P)) {
            const wf_status st = build_tables(slot, P, l, s);
            if (st != WF_OK) return st;
        }
        fx = slot.fx;
        fy = slot.fy;
        base = slot.base;
    }

    PoissonArgs<double> a;
    memset(&a, 0, sizeof(a));
    a.g.Nx = Nx; a.g.Ny = Ny; a.g.Nz = Nz; a.g.NzY = P->Nz_Y_max;
    a.g.N = Nx * Ny * Nz; a.g.NY = Nx * Ny * P->Nz_Y_max;
    a.g.z = reinterpret_cast<const double *>(base + l.z);
    a.ph.dx = P->dx; a.ph.dy = P->dy; a.ph.dt = P->dt; a.ph.rho_inf = P->rho_inf;
    a.ph.variable_density = 0;
    a.y1 = y_np1;
    a.yn = y_np1;
    a.p = p;
    a.G = base + l.G;
    a.kx2 = reinterpret_cast<const double *>(base + l.kx);
    a.ky2 = reinterpret_cast<const double *>(base + l.ky);
    a.fx = fx;
    a.fy = fy;
    a.h1 = (Ny - 1) / 2 + 1;
    const cudaError_t e = launch_poisson_impl<double>(a, reinterpret_cast<const double *>(base + l.zt), s);
    if (e) {
        set_error("wf_pressure_noalloc: %s", cudaGetErrorString(e));
        return WF_ERR_CUDA;
    }
    return WF_OK;
}
