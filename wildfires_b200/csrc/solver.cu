// solver.cu -- solver context of the C-ABI: device buffers, precomputed
// tables, the per-step launch sequence and its CUDA-graph replay.
//
// One step (reference src/cu/solver.cu:178-265) is
//   RK stages       launch_stage x {1,2,4}  (stage.cu)
//   pressure solve  launch_poisson_impl      (poisson.cu), repeated for the
//                   variable-density fixed point (pressure.cu:551-606)
//   end of step     launch_project           (project.cu)
// with the state in two ping-pong buffers; nothing is allocated after wf_create.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <string>
#include <vector>

#include "wf_internal.h"

namespace wf {
size_t diag_scratch_bytes();

static thread_local char g_err[1024];

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// ---- FFT plans: power-of-two lengths directly, others by Bluestein (setup only)
const long double kPiL = 3.141592653589793238462643383279502884L;

struct HostFft {
    FftDesc d;
    std::vector<double2> tw, chirp, filt, prb;
    std::vector<int> prmap, prslot;
};

long long pow_mod(long long b, long long e, long long m)
{
    long long r = 1 % m;
    b %= m;
    for (; e > 0; e >>= 1) {
        if (e & 1) r = r * b % m;
        b = b * b % m;
    }
    return r;
}
// inverse of a modulo m (gcd(a, m) = 1, m small)
int inv_mod(int a, int m)
{
    for (int t = 0; t < m; t++)
        if ((long long)a * t % m == 1 % m) return t;
    return 0;
}
// smallest primitive root of the prime P
int primitive_root(int P)
{
    std::vector<int> fac;
    for (int r = 2, x = P - 1; x > 1; r++)
        if (x % r == 0) {
            fac.push_back(r);
            while (x % r == 0) x /= r;
        }
    for (int g = 2; g < P; g++) {
        bool ok = true;
        for (int r : fac) ok = ok && pow_mod(g, (P - 1) / r, P) != 1;
        if (ok) return g;
    }
    return 0;
}

// Tables of the prime-factor + Rader engine for n = N1 P, P - 1 = F1 F2 F3
// (layout in fft_pr.cuh, with the factors of P - 1 as (F1, M, L): (F1, 1, F2)
// for two, (F1, F2, F3) for three); the filter in long double (setup only).
void plan_pr(HostFft &h, const int f[5])
{
    const int n = h.d.n, N1 = f[0], P = f[1], F1 = f[2], Q = P - 1;
    const int M = (f[4] > 1) ? f[3] : 1, L = (f[4] > 1) ? f[4] : f[3];
    const int g = primitive_root(P), gi = (int)pow_mod(g, P - 2, P);
    const int e2 = (int)((long long)N1 * inv_mod(N1 % P, P) % n);
    h.d.pr_e1 = (N1 > 1) ? (int)((long long)P * inv_mod(P % N1, N1) % n) : 0;
    h.prmap.assign(P + Q, 0);
    for (int q1 = 0; q1 < F1; q1++)
        for (int qm = 0; qm < M; qm++)
            for (int ql = 0; ql < L; ql++) {
                const int q = (int)(((long long)(Q / F1) * q1 + (long long)(Q / M) * qm + (long long)(Q / L) * ql) % Q);
                const int slot = (q1 * M + qm) * L + ql;
                h.prmap[1 + slot] = (int)pow_mod(g, q, P);
                h.prmap[P + slot] = (int)((long long)e2 * pow_mod(gi, q, P) % n);
            }
    // B'[j] = (1/Q) sum_t exp(-2 pi i gi^t / P) exp(-2 pi i j t / Q), stored at
    // (j1, jM, jL) with j = CRT(j1 mod F1, jM mod M, jL mod L)
    std::vector<long double> br(Q), bi(Q);
    for (int t = 0; t < Q; t++) {
        const long double a = -2.0L * kPiL * (long double)pow_mod(gi, t, P) / (long double)P;
        br[t] = cosl(a);
        bi[t] = sinl(a);
    }
    auto crt_weight = [&](int F) { return F > 1 ? (Q / F) * inv_mod((Q / F) % F, F) : 0; };
    const int c1 = crt_weight(F1), cm = crt_weight(M), cl = crt_weight(L);
    h.prb.resize(Q);
    for (int j1 = 0; j1 < F1; j1++)
        for (int jm = 0; jm < M; jm++)
            for (int jl = 0; jl < L; jl++) {
                const int j = (int)(((long long)j1 * c1 + (long long)jm * cm + (long long)jl * cl) % Q);
                long double sr = 0, si = 0;
                for (int t = 0; t < Q; t++) {
                    const long double a = -2.0L * kPiL * (long double)(((long long)j * t) % Q) / (long double)Q;
                    const long double c = cosl(a), sn = sinl(a);
                    sr += br[t] * c - bi[t] * sn;
                    si += br[t] * sn + bi[t] * c;
                }
                h.prb[(j1 * M + jm) * L + jl] = make_double2((double)(sr / Q), (double)(si / Q));
            }
    // Slots of the engine's slotted run (a kernel that stages whole lines in
    // shared memory applies both permutations in its copies): input x[j] at
    // n1 SS + u for j = N1 map[u] + P n1 (mod n), the pass-A gather; output
    // X[k] at m1 UB + u (k = k1 e1 + map[P + w + M L m1], u = k1 M L + w) or,
    // for the DC terms k = k1 e1, at F1 UB + k1, the pass-B3 scatter.
    int SS = 0, UB = 0;
    if (poisson_pr_layout(n, &SS, &UB)) {
        h.prslot.assign(2 * (size_t)n, -1);
        for (int u = 0; u < P; u++)
            for (int n1 = 0; n1 < N1; n1++) h.prslot[((long long)N1 * h.prmap[u] + (long long)P * n1) % n] = n1 * SS + u;
        const int ML = M * L;
        for (int k1 = 0; k1 < N1; k1++) {
            const int kb = (int)(((long long)k1 * h.d.pr_e1) % n);
            for (int w = 0; w < ML; w++)
                for (int m1 = 0; m1 < F1; m1++)
                    h.prslot[n + (kb + h.prmap[P + w + ML * m1]) % n] = m1 * UB + k1 * ML + w;
            h.prslot[n + kb] = F1 * UB + k1;
        }
        bool full = true;
        for (int v : h.prslot) full = full && v >= 0;
        if (!full) h.prslot.clear();   // not a permutation: no slot table, and the x kernel refuses the plan
    }
    h.d.pr = 1;
}

HostFft plan_fft(int n)
{
    HostFft h;
    memset(&h.d, 0, sizeof(h.d));
    h.d.n = n;
    // WF_FFT_RADER=0 keeps such lengths on Bluestein (for comparisons)
    const char *rader = getenv("WF_FFT_RADER");
    int f[5];
    if (!(rader && rader[0] == '0') && poisson_pr_plan(n, f)) {
        plan_pr(h, f);
        return h;
    }
    if ((n & (n - 1)) == 0) {
        h.d.m = n;
    } else {
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        h.d.m = m;
        h.d.bluestein = 1;
    }
    const int m = h.d.m;
    h.d.L = 0;
    while ((1 << h.d.L) < m) h.d.L++;
    h.tw.resize(m);
    for (int j = 0; j < m; j++) {
        const long double a = -2.0L * kPiL * (long double)j / (long double)m;
        h.tw[j] = make_double2((double)cosl(a), (double)sinl(a));
    }
    if (h.d.bluestein) {
        std::vector<long double> cr(n), ci(n);
        h.chirp.resize(n);
        for (int j = 0; j < n; j++) {
            const long long jj = ((long long)j * j) % (2LL * n);
            const long double a = -kPiL * (long double)jj / (long double)n;
            cr[j] = cosl(a);
            ci[j] = sinl(a);
            h.chirp[j] = make_double2((double)cr[j], (double)ci[j]);
        }
        // b_j = conj(chirp_j) on 0..n-1 and mirrored at m-j; filt = DFT_m(b),
        // evaluated directly in long double (setup only)
        std::vector<long double> br(m, 0.0L), bi(m, 0.0L), twr(m), twi(m);
        for (int j = 0; j < n; j++) {
            br[j] = cr[j];
            bi[j] = -ci[j];
            if (j > 0) {
                br[m - j] = cr[j];
                bi[m - j] = -ci[j];
            }
        }
        for (int j = 0; j < m; j++) {
            const long double a = -2.0L * kPiL * (long double)j / (long double)m;
            twr[j] = cosl(a);
            twi[j] = sinl(a);
        }
        h.filt.resize(m);
        for (int q = 0; q < m; q++) {
            long double sr = 0, si = 0;
            for (int j = 0; j < m; j++) {
                if (br[j] == 0.0L && bi[j] == 0.0L) continue;
                const int e = (int)(((long long)j * q) % m);
                sr += br[j] * twr[e] - bi[j] * twi[e];
                si += br[j] * twi[e] + bi[j] * twr[e];
            }
            h.filt[q] = make_double2((double)sr, (double)si);
        }
    }
    return h;
}

}  // namespace
}  // namespace wf

using namespace wf;

struct wf_ctx {
    Parameters P;
    std::vector<double> hx, hy, hz, ht, hkx, hky, htopo, hzibm;
    std::vector<int> hnzy, hcut;
    int prec = 0;          // WF_FP64 / WF_FP32_STENCIL
    int method = 2;        // 0 Euler, 1 RK2, 2 RK4
    int nstages = 4;
    int device = 0;
    cudaStream_t stream = nullptr;   // the stream work is enqueued on: own, or the caller's (wf_set_stream)
    cudaStream_t own = nullptr;      // the context's own stream; graphs are captured on it
    bool member = false;             // owned by an ensemble (its stream is the ensemble's to fork and join)
    int Nx, Ny, Nz, NzY, N, NY;
    size_t S;              // packed state size (elements)
    size_t esz;            // element size of the stencil state
    std::vector<DevBuf> bufs;
    void *ybuf[2] = {nullptr, nullptr};
    int cur = 0;
    void *Xa = nullptr, *Xb = nullptr, *acc = nullptr, *utau = nullptr, *bc = nullptr;
    void *Tsrc = nullptr;
    double *p = nullptr, *p_prev = nullptr, *d_diag = nullptr;
    double *vd_s0 = nullptr, *d_vdz = nullptr;   // variable density: per-step source part, z weights
    void *vd_g3 = nullptr;                        // variable density: grad(rho_n)/rho_n, [3][N] in the stencil precision
    double2 *G = nullptr;
    double *d_z = nullptr, *d_zc = nullptr, *d_topo = nullptr, *d_kx2 = nullptr, *d_ky2 = nullptr, *d_zt = nullptr;
    double *d_x = nullptr, *d_y = nullptr;
    void *d_krow = nullptr;     // [Nz][KROW] in the stencil precision
    int *d_nzy = nullptr, *d_cut = nullptr;
    FftDesc fx, fy;
    Phys ph;
    Geom geom;
    int h1;
    int n = 0;             // current time level
    double fuel0 = 0.0;    // fuel integral at upload
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int launches = 0;
    // variable-density pressure fixed point: device record, the stream the loop
    // body is captured on, and graphs of the loop alone for steps that are not
    // replayed from a step graph (keyed by their y_{n+1}, y_n buffers)
    PIterRec *rec = nullptr;
    cudaStream_t aux = nullptr;
    struct PLoop {
        const void *y1, *yn;
        cudaGraphExec_t ge;
    } ploop[4] = {};
    int ploop_next = 0;
    int closure = 0;         // WF_CLOSURE_SMAGORINSKY / WF_CLOSURE_MLP
    int *d_bcfix = nullptr;  // columns left to k_stage_bc
    int nbcfix = 0;
    void *coef = nullptr;    // [N] learned coefficient (stencil precision)
    float *d_theta = nullptr;
    int *d_closure_err = nullptr;   // raised by the closure kernel on a timed-out tensor-core wait
    int closure_wait = kClosureWaitLimit;   // polls of each tensor-core completion wait
    double *d_rep = nullptr;        // checkpoint report scratch
    Dumper *dump = nullptr;         // asynchronous dumps (created by the first wf_dump_async)
    int tile = 0;                   // tile shape of the fused stage pass (index)
    bool tile_set = false;          // chosen by the tuner, WF_STAGE_TILE or wf_set_stage_tile
    int *d_kerr = nullptr;          // raised by a stage kernel whose bounded tile wait gave up
    // wf_upload_state_async: p is copied on `up` after the state's copy (event
    // ev_y) and completes ev_p; the step waits for ev_p just before its pressure
    // solve, every other user of p first makes the context stream wait for it
    cudaStream_t up = nullptr;
    cudaEvent_t ev_y = nullptr, ev_p = nullptr;
    bool p_pending = false;
    // FP32 uploads and downloads go through two staging buffers (G and p_prev):
    // the host copy of one chunk runs on `up` while the other is converted on
    // the context stream; ev_copy / ev_conv order the two per buffer
    cudaEvent_t ev_copy[2] = {nullptr, nullptr}, ev_conv[2] = {nullptr, nullptr};
    // FP32: TMA tensor maps (CUtensorMap, 128 bytes) of the state buffers a stage
    // reads, for the boxes of 16-column (map[0]) and 8-column (map[1]) tiles
    struct TensorMaps {
        const void *ptr = nullptr;
        alignas(64) unsigned char map[2][128];
        bool ok[2] = {false, false};
    } tmaps[4];
    int ntmaps = 0;
    // FP32: maps of y_n (either step buffer) and acc for the boxes of a tile's own
    // cells, with which the stage kernel prefetches its RK operands into L2
    TensorMaps cmaps[3];
    int ncmaps = 0;
};

namespace wfs {

wf_status finish_upload(wf_ctx *c);
wf_status tune_tiles(wf_ctx *c);

// Order the context stream after a pressure copy of wf_upload_state_async that
// may still be in flight (callers that read or write p other than the step).
wf_status settle_p(wf_ctx *c)
{
    if (c->p_pending) {
        WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, c->ev_p, 0));
        c->p_pending = false;
    }
    return WF_OK;
}

// Kernel launches of one step: per stage the optional closure inference,
// k_utau, k_stage_fused and, when some column needs it, k_stage_bc; five
// pressure kernels per solve (variable density: plus the record reset, the
// source's p-independent part and, per iteration, k_maxdiff_copy and
// k_piter_next; counted for max_iter iterations, an upper bound when the
// tolerance ends the loop early); the projection.
int launches_per_step(const wf_ctx *c)
{
    const int per_stage = 2 + (c->nbcfix > 0 ? 1 : 0) + (c->closure ? 1 : 0);
    const int maxit = c->P.pressure_solver_iter > 0 ? c->P.pressure_solver_iter : 0;
    const int pressure = (c->P.variable_density != 0) ? 1 + (maxit > 0 ? 1 : 0) + 7 * maxit : 5;
    return c->nstages * per_stage + pressure + 1;
}

// Failure injection (wf_inject_allocation_failure): the number of context
// allocations that still succeed before one is refused; negative: off.
std::atomic<int> g_alloc_budget{-1};

wf_status dev_alloc(wf_ctx *c, void **out, size_t bytes)
{
    void *p = nullptr;
    if (g_alloc_budget.load() >= 0 && g_alloc_budget.fetch_sub(1) == 0) {
        g_alloc_budget.store(-1);
        set_error("device allocation of %zu bytes failed: refused by failure injection", bytes);
        return WF_ERR_OOM;
    }
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        set_error("device allocation of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
        cudaGetLastError();
        return WF_ERR_OOM;
    }
    c->bufs.push_back(DevBuf{p, bytes});
    *out = p;
    return WF_OK;
}

template <class T> wf_status upload(wf_ctx *c, T **dst, const T *src, size_t n)
{
    wf_status s = dev_alloc(c, (void **)dst, n * sizeof(T));
    if (s) return s;
    WF_TRY_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
    return WF_OK;
}

wf_status upload_fft(wf_ctx *c, const HostFft &h, FftDesc &d)
{
    d = h.d;
    if (h.d.pr) {
        double2 *rb = nullptr;
        int *map = nullptr;
        int *slot = nullptr;
        wf_status s = upload(c, &rb, h.prb.data(), h.prb.size());
        if (!s) s = upload(c, &map, h.prmap.data(), h.prmap.size());
        if (!s && !h.prslot.empty()) s = upload(c, &slot, h.prslot.data(), h.prslot.size());
        d.prb = rb;
        d.prmap = map;
        d.prslot = slot;
        return s;
    }
    double2 *tw = nullptr, *ch = nullptr, *fl = nullptr;
    wf_status s = upload(c, &tw, h.tw.data(), h.tw.size());
    if (s) return s;
    d.tw = tw;
    if (h.d.bluestein) {
        if ((s = upload(c, &ch, h.chirp.data(), h.chirp.size()))) return s;
        if ((s = upload(c, &fl, h.filt.data(), h.filt.size()))) return s;
        d.chirp = ch;
        d.filt = fl;
    }
    return WF_OK;
}

// z-stencil weight table (see ZCoef); values of the reference's formulas.
std::vector<double> zcoef_table(const Parameters &P, const double *z)
{
    const int Nz = P.Nz;
    std::vector<double> t((size_t)ZCOUNT * Nz, 0.0);
    auto at = [&](int e, int k) -> double & { return t[(size_t)e * Nz + k]; };
    for (int k = 0; k < Nz; k++) {
        if (k <= Nz - 3) {
            const double a = z[k + 1] - z[k], b = z[k + 2] - z[k + 1];
            at(ZF0, k) = -(2 * a + b) / (a * (a + b));
            at(ZF1, k) = (a + b) / (a * b);
            at(ZF2, k) = -a / (b * (a + b));
        }
        if (k >= 2) {
            const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2];
            at(ZB0, k) = a1 / (a2 * (a2 + a1));
            at(ZB1, k) = -(a2 + a1) / (a2 * a1);
            at(ZB2, k) = (a2 + 2 * a1) / (a1 * (a2 + a1));
        }
        if (k > 0 && k < Nz - 1) {
            const double a1 = z[k] - z[k - 1], a = z[k + 1] - z[k];
            at(ZC, k) = 1.0 / (a1 + a);
            at(ZCM, k) = 2 / (a1 * (a1 + a));
            at(ZC0, k) = -2 / (a1 * a);
            at(ZCP, k) = 2 / (a * (a1 + a));
        }
        const double dzk = (k < Nz - 1) ? z[k + 1] - z[k] : z[k] - z[k - 1];
        at(ZDZ, k) = dzk;
        at(ZDELTA2, k) = pow(P.C_s * pow(P.dx * P.dy * dzk, 1.0 / 3.0), 2.0);
    }
    {
        const double a = z[1] - z[0], b = z[2] - z[1], cc = z[3] - z[2];
        at(ZFF0, 0) = (6 * a + 4 * b + 2 * cc) / (a * (a + b) * (a + b + cc));
        at(ZFF1, 0) = -(4 * a + 4 * b + 2 * cc) / (a * b * (b + cc));
        at(ZFF2, 0) = (4 * a + 2 * b + 2 * cc) / (b * cc * (a + b));
        at(ZFF3, 0) = -(4 * a + 2 * b) / (cc * (b + cc) * (a + b + cc));
    }
    {
        const int k = Nz - 1;
        const double a1 = z[k] - z[k - 1], a2 = z[k - 1] - z[k - 2], a3 = z[k - 2] - z[k - 3];
        at(ZBB0, k) = -(2 * a2 + 4 * a1) / (a3 * (a3 + a2) * (a3 + a2 + a1));
        at(ZBB1, k) = (2 * a3 + 2 * a2 + 4 * a1) / (a3 * a2 * (a2 + a1));
        at(ZBB2, k) = -(2 * a3 + 4 * a2 + 4 * a1) / (a2 * a1 * (a3 + a2));
        at(ZBB3, k) = (2 * a3 + 4 * a2 + 6 * a1) / (a1 * (a2 + a1) * (a3 + a2 + a1));
    }
    return t;
}

// Tridiagonal constants (pressure.cu:356-390; layout read by k_p_tridiag).
std::vector<double> tridiag_table(const Parameters &P, const double *z)
{
    const int Nz = P.Nz, nk = Nz - 1;
    std::vector<double> t((size_t)3 * nk + 5, 0.0);
    for (int k = 0; k + 1 < nk; k++) {
        const double dk = z[k + 1] - z[k], dkp1 = z[k + 2] - z[k + 1];
        t[k] = 2 / (dk * (dk + dkp1));                       // a[k]
    }
    for (int k = 1; k + 1 < nk; k++) {
        const double dkm1 = z[k] - z[k - 1], dk = z[k + 1] - z[k];
        t[nk + k] = 2 / (dk * (dkm1 + dk));                  // c[k]
    }
    for (int k = 1; k < nk; k++) {
        const double dkm1 = z[k] - z[k - 1], dk = z[k + 1] - z[k];
        t[2 * nk + k] = 2 / (dkm1 * dk);                     // b[k] = -(kk + D[k])
    }
    const double dz0 = z[1] - z[0], dz1 = z[2] - z[1];
    const double dzNm2 = z[Nz - 2] - z[Nz - 3], dzNm1 = z[Nz - 1] - z[Nz - 2];
    t[3 * nk + 0] = -1.0 / dz0;                              // b[0]
    t[3 * nk + 1] = (dz0 + dz1) / (dz0 * dz1);               // c[0] + 0.5 dz0 kk + 1/dz1
    t[3 * nk + 2] = 1 / dz1;
    t[3 * nk + 3] = 0.5 * dz0;
    t[3 * nk + 4] = 2 / (dzNm1 * (dzNm2 + dzNm1));           // coupling of the top row
    return t;
}

// Branch-free z-stencil rows for the fused stage kernel (see KRow).
std::vector<double> krow_table(const Parameters &P, const double *z, const std::vector<double> &zc)
{
    const int Nz = P.Nz;
    std::vector<double> t((size_t)Nz * KROW, 0.0);
    auto Z = [&](int e, int k) { return zc[(size_t)e * Nz + k]; };
    for (int k = 0; k < Nz; k++) {
        double *r = &t[(size_t)k * KROW];
        // upwind "from below": forward form at k <= 1, backward form above (pde.cu:355-395)
        if (k <= 1) { r[RKM + 2] = Z(ZF0, k); r[RKM + 3] = Z(ZF1, k); r[RKM + 4] = Z(ZF2, k); }
        else { r[RKM + 0] = Z(ZB0, k); r[RKM + 1] = Z(ZB1, k); r[RKM + 2] = Z(ZB2, k); }
        // upwind "from above": backward form at k >= Nz-2, forward form below (pde.cu:397-437)
        if (k >= Nz - 2) { r[RKP + 0] = Z(ZB0, k); r[RKP + 1] = Z(ZB1, k); r[RKP + 2] = Z(ZB2, k); }
        else { r[RKP + 2] = Z(ZF0, k); r[RKP + 3] = Z(ZF1, k); r[RKP + 4] = Z(ZF2, k); }
        r[RD1] = Z(ZC, k);
        r[RD2 + 0] = Z(ZCM, k);
        r[RD2 + 1] = Z(ZC0, k);
        r[RD2 + 2] = Z(ZCP, k);
        r[RDZ] = Z(ZDZ, k);
        r[RDEL2] = Z(ZDELTA2, k);
        r[RZ] = z[k];
        r[RDD2] = pow(P.dx * P.dy * Z(ZDZ, k), 2.0 / 3.0);
    }
    return t;
}

template <class R> PhysR<R> make_physr(const Parameters &P)
{
    constexpr double kSigmaSB = 5.670374419e-8;  // Stefan-Boltzmann (reference constants.h:16)
    PhysR<R> r;
    r.inv2dx = (R)(1.0 / (2 * P.dx));
    r.inv2dy = (R)(1.0 / (2 * P.dy));
    r.invdx2 = (R)(1.0 / (P.dx * P.dx));
    r.invdy2 = (R)(1.0 / (P.dy * P.dy));
    r.Trho = (R)P.T_inf * (R)P.rho_inf;
    r.mu = (R)P.mu; r.kT = (R)P.k; r.Y_f = (R)P.Y_f; r.H_C = (R)P.H_C; r.A = (R)P.A; r.T_act = (R)P.T_act;
    r.T_pc = (R)P.T_pc; r.h_c = (R)P.h_c; r.alpha_s = (R)P.alpha_s; r.sigma_s = (R)P.sigma_s;
    r.T_inf = (R)P.T_inf; r.c_p = (R)P.c_p; r.rho_inf = (R)P.rho_inf;
    r.cd = (R)(0.5 * P.C_d * P.alpha_s * P.sigma_s);
    r.g = (R)P.g;
    r.c12 = (R)(12 * kSigmaSB * P.delta);
    r.c4 = (R)(4 * kSigmaSB * P.delta);
    r.Pr = (R)P.Pr;
    r.inv_avd = R(1) / R(26.0);
    r.mu_Trho = (R)(P.mu / (P.T_inf * P.rho_inf));
    r.inv_Trho_cp = (R)(1.0 / (P.T_inf * P.rho_inf * P.c_p));
    r.H_C_cp = (R)(P.H_C / P.c_p);
    r.T_min = (R)P.T_min; r.T_max = (R)P.T_max; r.Y_min = (R)P.Y_min; r.Y_max = (R)P.Y_max;
    return r;
}

Phys make_phys(const Parameters &P)
{
    Phys ph;
    memset(&ph, 0, sizeof(ph));
    ph.dx = P.dx; ph.dy = P.dy; ph.dt = P.dt;
    ph.mu = P.mu; ph.kT = P.k; ph.Y_f = P.Y_f; ph.H_C = P.H_C; ph.A = P.A; ph.T_act = P.T_act;
    ph.T_pc = P.T_pc; ph.h_c = P.h_c; ph.alpha_s = P.alpha_s; ph.sigma_s = P.sigma_s;
    ph.T_inf = P.T_inf; ph.c_p = P.c_p; ph.rho_inf = P.rho_inf; ph.C_d = P.C_d; ph.g = P.g;
    ph.delta = P.delta; ph.Pr = P.Pr;
    ph.T_min = P.T_min; ph.T_max = P.T_max; ph.Y_min = P.Y_min; ph.Y_max = P.Y_max;
    ph.u_dead = P.u_dead_nodes; ph.v_dead = P.v_dead_nodes; ph.w_dead = P.w_dead_nodes;
    ph.T_dead = P.T_dead_nodes; ph.Y_dead = P.Y_dead_nodes;
    ph.temperature_convection = P.temperature_convection;
    ph.sutherland_viscosity = P.sutherland_viscosity;
    ph.sutherland_conductivity = P.sutherland_conductivity;
    ph.variable_density = P.variable_density;
    ph.velocity_correction_fd = P.velocity_correction_fd;
    if (P.z && P.Nz >= 3) {
        const int k = P.Nz - 1;
        const double a1 = P.z[k] - P.z[k - 1], a2 = P.z[k - 1] - P.z[k - 2];
        const double den = a2 * (a2 + 2 * a1);
        ph.top_w1 = (a2 + a1) * (a2 + a1) / den;
        ph.top_w2 = a1 * a1 / den;
    }
    return ph;
}

template <class R> StageArgs<R> stage_args(wf_ctx *c, const void *X, const void *yn, void *Xout, int stage)
{
    StageArgs<R> a;
    a.g = c->geom;
    a.ph = c->ph;
    a.pr = make_physr<R>(c->P);
    a.krow = (const R *)c->d_krow;
    a.X = (const R *)X;
    a.yn = (const R *)yn;
    a.acc = (R *)c->acc;
    a.Xout = (R *)Xout;
    a.utau = (R *)c->utau;
    a.bc = (R *)c->bc;
    a.method = c->method;
    a.stage = stage;
    a.a_prev = 0.0;
    a.coef = c->closure ? (R *)c->coef : nullptr;
    a.theta = c->d_theta;
    a.closure_err = c->d_closure_err;
    a.closure_wait = c->closure_wait;
    a.bcfix = c->d_bcfix;
    a.nbcfix = c->nbcfix;
    a.kerr = c->d_kerr;
    a.tmap[0] = a.tmap[1] = nullptr;
    for (int q = 0; q < c->ntmaps; q++)
        if (c->tmaps[q].ptr == X)
            for (int b = 0; b < 2; b++) a.tmap[b] = c->tmaps[q].ok[b] ? c->tmaps[q].map[b] : nullptr;
    for (int b = 0; b < 2; b++) a.pmap_yn[b] = a.pmap_acc[b] = nullptr;
    for (int q = 0; q < c->ncmaps; q++)
        for (int b = 0; b < 2; b++) {
            if (c->cmaps[q].ptr == yn) a.pmap_yn[b] = c->cmaps[q].ok[b] ? c->cmaps[q].map[b] : nullptr;
            if (c->cmaps[q].ptr == c->acc) a.pmap_acc[b] = c->cmaps[q].ok[b] ? c->cmaps[q].map[b] : nullptr;
        }
    a.tile = c->tile;
    const double dt = c->P.dt;
    if (c->method == 0) a.a_next = dt;
    else if (c->method == 1) a.a_next = (stage == 1) ? dt : 0.5 * dt;
    else a.a_next = (stage == 1 || stage == 2) ? dt * 0.5 : (stage == 3) ? dt : dt / 6;
    return a;
}

template <class R> PoissonArgs<R> poisson_args(wf_ctx *c, const void *y1, const void *yn)
{
    PoissonArgs<R> a;
    a.g = c->geom;
    a.ph = c->ph;
    a.y1 = (const R *)y1;
    a.yn = (const R *)yn;
    a.p = c->p;
    a.G = c->G;
    a.kx2 = c->d_kx2;
    a.ky2 = c->d_ky2;
    a.fx = c->fx;
    a.fy = c->fy;
    a.h1 = c->h1;
    a.s0 = nullptr;
    a.g3 = nullptr;
    a.vdz = c->d_vdz;
    return a;
}

// source mode of the step that produces time level n1 (solver.cu:217-223)
int source_mode(const wf_ctx *c, int n1, double *scale)
{
    const double t1 = c->P.t_min + n1 * c->P.dt;
    *scale = 1.0;
    if (!(t1 <= c->P.t_source_end)) return 0;
    if (c->P.t_source_start <= 0) return 1;
    if (strcmp(c->P.T_source_shape, "gaussian") != 0 && strcmp(c->P.T_source_shape, "parallelepiped") != 0) return 0;
    if (t1 <= c->P.t_source_start) *scale = t1 / c->P.t_source_start;
    return 2;
}

template <class R> wf_status enqueue_stages(wf_ctx *c, void *yn, void *y1)
{
    cudaStream_t s = c->stream;
    if (c->nstages == 1) {
        WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, yn, yn, y1, 1), s));
        return WF_OK;
    }
    if (c->nstages == 2) {
        WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, yn, yn, c->Xa, 1), s));
        WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, c->Xa, yn, y1, 2), s));
        return WF_OK;
    }
    WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, yn, yn, c->Xa, 1), s));
    WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, c->Xa, yn, c->Xb, 2), s));
    WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, c->Xb, yn, c->Xa, 3), s));
    WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, c->Xa, yn, y1, 4), s));
    return WF_OK;
}

// Capture the variable-density fixed point (pressure.cu:551-606) into the
// stream's capture: p_prev = p, reset of the device record, then a WHILE node
// whose body (captured on c->aux) is one Poisson solve, the max-norm change
// with p_prev = p, and k_piter_next, which ends the loop once the change meets
// the tolerance or maxit solves are done.
template <class R> wf_status capture_pressure_loop(wf_ctx *c, const PoissonArgs<R> &a, cudaStream_t s)
{
    const int maxit = c->P.pressure_solver_iter;
    const double tol = c->P.pressure_solver_tol;
    WF_TRY_CUDA(cudaMemcpyAsync(c->p_prev, c->p, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, s));
    WF_TRY_CUDA(launch_piter_begin(c->rec, s));
    if (maxit <= 0) return WF_OK;   // the reference's loop body does not run
    // the source's p-independent part, once for every solve of the fixed point
    PoissonArgs<R> ab = a;
    if (c->vd_s0 && c->vd_g3 && c->d_vdz) {
        ab.s0 = c->vd_s0;
        ab.g3 = (R *)c->vd_g3;
        WF_TRY_CUDA(launch_vd_base<R>(ab, s));
    }
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    WF_TRY_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive) { set_error("pressure loop: stream is not capturing"); return WF_ERR_CUDA; }
    cudaGraphConditionalHandle cond;
    WF_TRY_CUDA(cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = cond;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    WF_TRY_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
    WF_TRY_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    WF_TRY_CUDA(cudaStreamBeginCaptureToGraph(c->aux, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = launch_poisson_impl<R>(ab, c->d_zt, c->aux);
    if (!e) e = launch_maxdiff_copy(c->p, c->p_prev, c->N, c->rec, c->aux);
    if (!e) e = launch_piter_next(c->rec, tol, tol >= 0 ? 1 : 0, maxit, cond, c->aux);
    cudaGraph_t captured = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(c->aux, &captured);
    if (e || e2) {
        set_error("pressure loop body capture failed: %s", cudaGetErrorString(e ? e : e2));
        return WF_ERR_CUDA;
    }
    return WF_OK;
}

// Pressure solve of one step.  Constant density: one solve.  Variable density:
// the fixed point runs on the device (see capture_pressure_loop); inside a
// step capture it becomes part of the step graph, otherwise a graph of the loop
// alone is built once per (y1, yn) pair and launched.
template <class R> wf_status enqueue_pressure(wf_ctx *c, const void *y1, const void *yn)
{
    cudaStream_t s = c->stream;
    const PoissonArgs<R> a = poisson_args<R>(c, y1, yn);
    if (c->P.variable_density == 0) {
        WF_TRY_CUDA(launch_poisson_impl<R>(a, c->d_zt, s));
        return WF_OK;
    }
    cudaStreamCaptureStatus cs;
    WF_TRY_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusActive) return capture_pressure_loop<R>(c, a, s);
    cudaGraphExec_t ge = nullptr;
    for (auto &pl : c->ploop)
        if (pl.ge && pl.y1 == y1 && pl.yn == yn) ge = pl.ge;
    if (!ge) {
        // captured on the context's own stream, launched on the current one
        cudaGraph_t gph = nullptr;
        WF_TRY_CUDA(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
        wf_status st = capture_pressure_loop<R>(c, a, c->own);
        cudaError_t e = cudaStreamEndCapture(c->own, &gph);
        if (st) {
            if (gph) cudaGraphDestroy(gph);
            return st;
        }
        if (e != cudaSuccess) { set_error("pressure loop capture failed: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
        e = cudaGraphInstantiate(&ge, gph, 0);
        cudaGraphDestroy(gph);
        if (e != cudaSuccess) { set_error("pressure loop instantiate failed: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
        auto &slot = c->ploop[c->ploop_next];
        c->ploop_next = (c->ploop_next + 1) % 4;
        if (slot.ge) cudaGraphExecDestroy(slot.ge);
        slot = {y1, yn, ge};
    }
    WF_TRY_CUDA(cudaGraphLaunch(ge, s));
    return WF_OK;
}

// Iterations of the last variable-density pressure solve as the device record
// holds them (waits for the stream): solves done, last max-norm change, and
// the count solve_pressure_iterative reports (pressure.cu:564-600: the index of
// the breaking iteration, else max_iter).
wf_status read_piter(wf_ctx *c, int *solves, double *err, int *ref_iter)
{
    PIterRec r;
    memset(&r, 0, sizeof(r));
    if (c->P.variable_density != 0) {
        WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
        WF_TRY_CUDA(cudaMemcpy(&r, c->rec, sizeof(r), cudaMemcpyDeviceToHost));
    }
    if (solves) *solves = (c->P.variable_density != 0) ? r.m : 1;
    if (err) *err = r.h;
    if (ref_iter) *ref_iter = (c->P.variable_density == 0) ? 0 : (r.done ? r.m - 1 : c->P.pressure_solver_iter);
    return WF_OK;
}

template <class R> wf_status enqueue_step(wf_ctx *c, int cur, int n1)
{
    void *yn = c->ybuf[cur], *y1 = c->ybuf[1 - cur];
    wf_status st = enqueue_stages<R>(c, yn, y1);
    if (st) return st;
    // the pressure solve reads p's top plane: wait for an asynchronous upload of
    // p here, so that its copy overlaps the RK stages (a wait node when captured;
    // an event never recorded, or long complete, makes it a no-op)
    {
        cudaStreamCaptureStatus cs;
        WF_TRY_CUDA(cudaStreamIsCapturing(c->stream, &cs));
        WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, c->ev_p,
                                        cs == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0));
    }
    if ((st = enqueue_pressure<R>(c, y1, yn))) return st;
    ProjectArgs<R> pa;
    memset(&pa, 0, sizeof(pa));
    pa.g = c->geom;
    pa.ph = c->ph;
    pa.y = (R *)y1;
    pa.yn = (const R *)yn;
    pa.p = c->p;
    double scale;
    pa.source_mode = source_mode(c, n1, &scale);
    pa.src_scale = scale;
    pa.Tsrc = (const R *)c->Tsrc;
    if (pa.source_mode == 1 && !c->Tsrc) pa.source_mode = 0;
    pa.t_n1 = c->P.t_min + n1 * c->P.dt;
    pa.xg = c->d_x;
    pa.yg = c->d_y;
    memcpy(pa.TS, &c->P.TS_x_start, sizeof(pa.TS));
    pa.TS_gauss = strcmp(c->P.T_source_shape, "gaussian") == 0;
    pa.T_source = c->P.T_source;
    WF_TRY_CUDA(launch_project<R>(pa, c->stream));
    return WF_OK;
}

wf_status enqueue_step_any(wf_ctx *c, int cur, int n1)
{
    return c->prec == WF_FP64 ? enqueue_step<double>(c, cur, n1) : enqueue_step<float>(c, cur, n1);
}

// A step can be replayed from a graph when its launch sequence does not depend
// on the time level or on host decisions.
bool step_is_static(const wf_ctx *c, int n1)
{
    double sc;
    return source_mode(c, n1, &sc) == 0;
}

template <class R> __global__ void k_to_prec(R *dst, const double *src, size_t n)
{
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        dst[t] = (R)src[t];
}
template <class R> __global__ void k_from_prec(double *dst, const R *src, size_t n)
{
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        dst[t] = (double)src[t];
}

// host FP64 packed vector -> device buffer of the stencil precision
// Chunk length (doubles) of the FP32 staging: each of the two staging buffers
// (G and p_prev) holds one chunk.
size_t staging_chunk(const wf_ctx *c)
{
    const size_t g = (size_t)(c->Nz) * (c->Nx - 1) * c->h1 * 2;
    return g < (size_t)c->N ? g : (size_t)c->N;
}

wf_status put_state(wf_ctx *c, void *dst, const double *src)
{
    if (c->prec == WF_FP64) {
        WF_TRY_CUDA(cudaMemcpyAsync(dst, src, c->S * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        return WF_OK;
    }
    // chunks alternate between the two staging buffers: the host copy of chunk
    // i + 1 (on `up`) runs while chunk i is converted (on the context stream)
    double *stg[2] = {reinterpret_cast<double *>(c->G), c->p_prev};
    const size_t chunk = staging_chunk(c);
    // the staging buffers are free once the context stream's earlier work is done
    WF_TRY_CUDA(cudaEventRecord(c->ev_conv[0], c->stream));
    WF_TRY_CUDA(cudaEventRecord(c->ev_conv[1], c->stream));
    size_t done = 0;
    for (int i = 0; done < c->S; i++) {
        const int b = i & 1;
        const size_t nn = (c->S - done < chunk) ? c->S - done : chunk;
        WF_TRY_CUDA(cudaStreamWaitEvent(c->up, c->ev_conv[b], 0));
        WF_TRY_CUDA(cudaMemcpyAsync(stg[b], src + done, nn * sizeof(double), cudaMemcpyHostToDevice, c->up));
        WF_TRY_CUDA(cudaEventRecord(c->ev_copy[b], c->up));
        WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, c->ev_copy[b], 0));
        k_to_prec<float><<<592, 256, 0, c->stream>>>((float *)dst + done, stg[b], nn);
        WF_TRY_CUDA(cudaGetLastError());
        WF_TRY_CUDA(cudaEventRecord(c->ev_conv[b], c->stream));
        done += nn;
    }
    return WF_OK;
}

// Device state -> host FP64 (waits for the copies).  FP32: the conversion of
// chunk i + 1 (context stream) runs while chunk i is copied to the host (`up`).
wf_status get_state(wf_ctx *c, double *dst, const void *src)
{
    if (c->prec == WF_FP64) {
        WF_TRY_CUDA(cudaMemcpyAsync(dst, src, c->S * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
        return WF_OK;
    }
    double *stg[2] = {reinterpret_cast<double *>(c->G), c->p_prev};
    const size_t chunk = staging_chunk(c);
    // earlier copies out of the staging buffers (previous calls) are done
    WF_TRY_CUDA(cudaEventRecord(c->ev_copy[0], c->up));
    WF_TRY_CUDA(cudaEventRecord(c->ev_copy[1], c->up));
    size_t done = 0;
    for (int i = 0; done < c->S; i++) {
        const int b = i & 1;
        const size_t nn = (c->S - done < chunk) ? c->S - done : chunk;
        WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, c->ev_copy[b], 0));
        k_from_prec<float><<<592, 256, 0, c->stream>>>(stg[b], (const float *)src + done, nn);
        WF_TRY_CUDA(cudaGetLastError());
        WF_TRY_CUDA(cudaEventRecord(c->ev_conv[b], c->stream));
        WF_TRY_CUDA(cudaStreamWaitEvent(c->up, c->ev_conv[b], 0));
        WF_TRY_CUDA(cudaMemcpyAsync(dst + done, stg[b], nn * sizeof(double), cudaMemcpyDeviceToHost, c->up));
        WF_TRY_CUDA(cudaEventRecord(c->ev_copy[b], c->up));
        done += nn;
    }
    // the context stream's later work (which may reuse the staging buffers)
    // comes after the copies
    WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, c->ev_copy[0], 0));
    WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, c->ev_copy[1], 0));
    WF_TRY_CUDA(cudaStreamSynchronize(c->up));
    return WF_OK;
}

void drop_graphs(wf_ctx *c)
{
    for (int q = 0; q < 2; q++)
        if (c->graph[q]) {
            cudaGraphExecDestroy(c->graph[q]);
            c->graph[q] = nullptr;
        }
}

const char *kPhaseNames[WF_NPHASES] = {"stage_utau", "stage_fused", "stage_bc", "p_rhs_ffty", "p_fftx_fwd",
                                       "p_tridiag", "p_fftx_inv", "p_iffty_out", "project"};

template <class R> wf_status profile_step(wf_ctx *c, cudaEvent_t *ev, int &ne)
{
    cudaStream_t s = c->stream;
    void *yn = c->ybuf[c->cur], *y1 = c->ybuf[1 - c->cur];
    const void *ins[4], *outs[4];
    if (c->nstages == 1) { ins[0] = yn; outs[0] = y1; }
    else if (c->nstages == 2) { ins[0] = yn; outs[0] = c->Xa; ins[1] = c->Xa; outs[1] = y1; }
    else {
        ins[0] = yn; outs[0] = c->Xa; ins[1] = c->Xa; outs[1] = c->Xb;
        ins[2] = c->Xb; outs[2] = c->Xa; ins[3] = c->Xa; outs[3] = y1;
    }
    WF_TRY_CUDA(cudaEventRecord(ev[ne++], s));
    for (int st = 0; st < c->nstages; st++) {
        WF_TRY_CUDA(launch_stage<R>(stage_args<R>(c, ins[st], yn, (void *)outs[st], st + 1), s, ev + ne));
        ne += 3;
    }
    PoissonArgs<R> a = poisson_args<R>(c, y1, yn);
    const int nsolve = (c->P.variable_density == 0) ? 1 : c->P.pressure_solver_iter;
    if (nsolve > 0 && c->P.variable_density != 0 && c->vd_s0 && c->vd_g3 && c->d_vdz) {
        // as the fixed point runs: the per-step part of the source first (its
        // time lands in the first solve's source kernel), then every solve
        a.s0 = c->vd_s0;
        a.g3 = (R *)c->vd_g3;
        WF_TRY_CUDA(launch_vd_base<R>(a, s));
    }
    for (int q = 0; q < nsolve; q++) {
        WF_TRY_CUDA(launch_poisson_impl<R>(a, c->d_zt, s, ev + ne));
        ne += 5;
    }
    ProjectArgs<R> pa;
    memset(&pa, 0, sizeof(pa));
    pa.g = c->geom;
    pa.ph = c->ph;
    pa.y = (R *)y1;
    pa.yn = (const R *)yn;
    pa.p = c->p;
    WF_TRY_CUDA(launch_project<R>(pa, s));
    WF_TRY_CUDA(cudaEventRecord(ev[ne++], s));
    return WF_OK;
}

}  // namespace wfs

using namespace wfs;

// ===========================================================================
extern "C" {

const char *wf_last_error(void) { return g_err; }

const char *wf_status_string(wf_status s)
{
    switch (s) {
    case WF_OK: return "ok";
    case WF_ERR_ARG: return "invalid argument";
    case WF_ERR_CUDA: return "CUDA error";
    case WF_ERR_IO: return "I/O error";
    case WF_ERR_PARSE: return "parse error";
    case WF_ERR_OOM: return "out of memory";
    case WF_ERR_NAN: return "NaN in state";
    case WF_ERR_NO_DEVICE: return "no sm_100 device";
    }
    return "unknown status";
}

wf_status wf_create(const Parameters *P, int precision, wf_ctx **out)
{
    if (!P || !out) { set_error("wf_create: null argument"); return WF_ERR_ARG; }
    *out = nullptr;
    if (precision != WF_FP64 && precision != WF_FP32_STENCIL) { set_error("wf_create: unknown precision %d", precision); return WF_ERR_ARG; }
    const int Nx = P->Nx, Ny = P->Ny, Nz = P->Nz;
    if (Nx < 4 || Ny < 4 || Nz < 5) { set_error("wf_create: grid %dx%dx%d too small (need Nx,Ny >= 4, Nz >= 5)", Nx, Ny, Nz); return WF_ERR_ARG; }
    if (Nx - 1 > kMaxFftLength || Ny - 1 > kMaxFftLength) { set_error("wf_create: Nx-1 and Ny-1 must be <= %d", kMaxFftLength); return WF_ERR_ARG; }
    if (Nz - 1 > kMaxZUnknowns) { set_error("wf_create: Nz-1 must be <= %d", kMaxZUnknowns); return WF_ERR_ARG; }
    if ((long long)Nx * Ny * Nz * 5 > 2000000000LL) { set_error("wf_create: grid too large for 32-bit cell indices"); return WF_ERR_ARG; }
    if (!P->z || !P->Nz_Y || !P->cut_nodes || !P->kx || !P->ky || !P->topography || !P->x || !P->y) {
        set_error("wf_create: derived arrays missing (use wf_read_parameters)");
        return WF_ERR_ARG;
    }
    for (int q = 0; q < Nx * Ny; q++)
        if (P->cut_nodes[q] < 0 || P->cut_nodes[q] > Nz - 4) {
            set_error("wf_create: terrain cut node %d in column %d is above Nz-4 = %d", P->cut_nodes[q], q, Nz - 4);
            return WF_ERR_ARG;
        }
    int dev = 0, cc_major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("wf_create: no CUDA device");
        return WF_ERR_NO_DEVICE;
    }
    if (cc_major != 10) { set_error("wf_create: device %d is sm_%d0, the library is compiled for sm_100a", dev, cc_major); return WF_ERR_NO_DEVICE; }

    wf_ctx *c = new wf_ctx();
    c->P = *P;
    c->device = dev;
    c->prec = precision;
    c->Nx = Nx; c->Ny = Ny; c->Nz = Nz; c->NzY = P->Nz_Y_max;
    c->N = Nx * Ny * Nz;
    c->NY = Nx * Ny * c->NzY;
    c->S = (size_t)4 * c->N + c->NY;
    c->esz = precision == WF_FP64 ? 8 : 4;
    if (strncmp(P->method, "Euler", 5) == 0) { c->method = 0; c->nstages = 1; }
    else if (strncmp(P->method, "RK2", 3) == 0) { c->method = 1; c->nstages = 2; }
    else if (strncmp(P->method, "RK4", 3) == 0) { c->method = 2; c->nstages = 4; }
    else { delete c; set_error("wf_create: time integration method '%s' not found", P->method); return WF_ERR_ARG; }
    // host copies of the arrays the record points to
    c->hx.assign(P->x, P->x + Nx);
    c->hy.assign(P->y, P->y + Ny);
    c->hz.assign(P->z, P->z + Nz);
    c->hkx.assign(P->kx, P->kx + Nx - 1);
    c->hky.assign(P->ky, P->ky + Ny - 1);
    c->htopo.assign(P->topography, P->topography + (size_t)Nx * Ny);
    c->hnzy.assign(P->Nz_Y, P->Nz_Y + (size_t)Nx * Ny);
    c->hcut.assign(P->cut_nodes, P->cut_nodes + (size_t)Nx * Ny);
    c->P.x = c->hx.data(); c->P.y = c->hy.data(); c->P.z = c->hz.data();
    c->P.kx = c->hkx.data(); c->P.ky = c->hky.data(); c->P.topography = c->htopo.data();
    c->P.Nz_Y = c->hnzy.data(); c->P.cut_nodes = c->hcut.data();
    c->P.t = nullptr; c->P.r = nullptr; c->P.s = nullptr; c->P.z_ibm = nullptr;
    c->P.log_files.parameters = nullptr; c->P.log_files.log = nullptr;
    c->h1 = (Ny - 1) / 2 + 1;

    wf_status st = WF_OK;
    auto fail = [&](wf_status s) { wf_destroy(c); return s; };
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("wf_create: stream creation failed");
        delete c;
        return WF_ERR_CUDA;
    }
    c->stream = c->own;
    const size_t sb = c->S * c->esz;
    if ((st = dev_alloc(c, &c->ybuf[0], sb)) || (st = dev_alloc(c, &c->ybuf[1], sb))) return fail(st);
    if (c->nstages > 1) {
        if ((st = dev_alloc(c, &c->Xa, sb)) || (st = dev_alloc(c, &c->acc, sb))) return fail(st);
        if (c->nstages > 2 && (st = dev_alloc(c, &c->Xb, sb))) return fail(st);
    }
    if ((st = dev_alloc(c, &c->utau, (size_t)Nx * Ny * c->esz))) return fail(st);
    if ((st = dev_alloc(c, &c->bc, (size_t)Nx * Ny * kBcSlots * c->esz))) return fail(st);
    if ((st = dev_alloc(c, (void **)&c->p, sizeof(double) * c->N))) return fail(st);
    if ((st = dev_alloc(c, (void **)&c->p_prev, sizeof(double) * c->N))) return fail(st);
    if (P->variable_density != 0) {
        if ((st = dev_alloc(c, (void **)&c->vd_s0, sizeof(double) * c->N))) return fail(st);
        if ((st = dev_alloc(c, &c->vd_g3, 3 * (size_t)c->N * c->esz))) return fail(st);
        std::vector<double> vz((size_t)Nz * kVdz);
        vd_z_table(c->hz.data(), Nz, vz.data());
        if ((st = upload(c, &c->d_vdz, vz.data(), vz.size()))) return fail(st);
    }
    if ((st = dev_alloc(c, (void **)&c->G, sizeof(double2) * (size_t)Nz * (Nx - 1) * c->h1))) return fail(st);
    if ((st = dev_alloc(c, (void **)&c->rec, sizeof(PIterRec)))) return fail(st);
    if (cudaMemset(c->rec, 0, sizeof(PIterRec)) != cudaSuccess) {
        set_error("wf_create: clearing the pressure-loop record failed");
        return fail(WF_ERR_CUDA);
    }
    if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->up, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_y, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_p, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_copy[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_copy[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_conv[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_conv[1], cudaEventDisableTiming) != cudaSuccess) {
        set_error("wf_create: stream creation failed");
        return fail(WF_ERR_CUDA);
    }
    if ((st = dev_alloc(c, (void **)&c->d_diag, diag_scratch_bytes()))) return fail(st);
    if ((st = dev_alloc(c, (void **)&c->d_rep, report_scratch_bytes()))) return fail(st);
    // tables
    std::vector<double> zc = zcoef_table(c->P, c->hz.data()), zt = tridiag_table(c->P, c->hz.data());
    std::vector<double> kx2(Nx - 1), ky2(Ny - 1);
    for (int i = 0; i < Nx - 1; i++) kx2[i] = c->hkx[i] * c->hkx[i];
    for (int j = 0; j < Ny - 1; j++) ky2[j] = c->hky[j] * c->hky[j];
    if ((st = upload(c, &c->d_z, c->hz.data(), Nz)) || (st = upload(c, &c->d_zc, zc.data(), zc.size())) ||
        (st = upload(c, &c->d_zt, zt.data(), zt.size())) || (st = upload(c, &c->d_kx2, kx2.data(), kx2.size())) ||
        (st = upload(c, &c->d_ky2, ky2.data(), ky2.size())) || (st = upload(c, &c->d_topo, c->htopo.data(), c->htopo.size())) ||
        (st = upload(c, &c->d_nzy, c->hnzy.data(), c->hnzy.size())) || (st = upload(c, &c->d_cut, c->hcut.data(), c->hcut.size())) ||
        (st = upload(c, &c->d_x, c->hx.data(), Nx)) || (st = upload(c, &c->d_y, c->hy.data(), Ny)))
        return fail(st);
    {
        const std::vector<double> kr = krow_table(c->P, c->hz.data(), zc);
        if (precision == WF_FP64) {
            double *d = nullptr;
            if ((st = upload(c, &d, kr.data(), kr.size()))) return fail(st);
            c->d_krow = d;
        } else {
            std::vector<float> kf(kr.begin(), kr.end());
            float *d = nullptr;
            if ((st = upload(c, &d, kf.data(), kf.size()))) return fail(st);
            c->d_krow = d;
        }
    }
    const HostFft hfx = plan_fft(Nx - 1), hfy = plan_fft(Ny - 1);
    if ((st = upload_fft(c, hfx, c->fx)) || (st = upload_fft(c, hfy, c->fy))) return fail(st);
    if (P->t_source_end > P->t_min && P->t_source_start <= 0)
        if ((st = dev_alloc(c, &c->Tsrc, (size_t)c->N * c->esz))) return fail(st);
    c->geom.Nx = Nx; c->geom.Ny = Ny; c->geom.Nz = Nz; c->geom.NzY = c->NzY;
    c->geom.N = c->N; c->geom.NY = c->NY;
    c->geom.z = c->d_z; c->geom.zc = c->d_zc; c->geom.topo = c->d_topo;
    c->geom.nzy = c->d_nzy; c->geom.cut = c->d_cut;
    c->ph = make_phys(c->P);
    cudaError_t e = (precision == WF_FP64) ? poisson_set_attributes<double>() : poisson_set_attributes<float>();
    if (e == cudaSuccess) e = (precision == WF_FP64) ? stage_set_attributes<double>() : stage_set_attributes<float>();
    if (e != cudaSuccess) { set_error("wf_create: %s", cudaGetErrorString(e)); return fail(WF_ERR_CUDA); }
    {
        // columns whose cut node (or, for every column, the top plane) the
        // fused stage pass cannot complete within one z-tile
        const int KZ = stage_tile_planes(precision);
        const bool top_ok = (Nz - 1) / KZ == (Nz - 3) / KZ;
        std::vector<int> fix;
        for (int col = 0; col < Nx * Ny; col++) {
            const int kc = c->hcut[col];
            if (!top_ok || kc / KZ != (kc + 2) / KZ) fix.push_back(col);
        }
        c->nbcfix = (int)fix.size();
        if (!fix.empty() && (st = upload(c, &c->d_bcfix, fix.data(), fix.size()))) return fail(st);
    }
    e = cudaMemsetAsync(c->p, 0, sizeof(double) * c->N, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) { set_error("wf_create: %s", cudaGetErrorString(e)); return fail(WF_ERR_CUDA); }
    if ((st = dev_alloc(c, (void **)&c->d_kerr, sizeof(int)))) return fail(st);
    e = cudaMemset(c->d_kerr, 0, sizeof(int));
    if (e != cudaSuccess) { set_error("wf_create: %s", cudaGetErrorString(e)); return fail(WF_ERR_CUDA); }
    if (precision != WF_FP64 && !(getenv("WF_NO_TMA") && atoi(getenv("WF_NO_TMA")))) {
        // tensor maps for the tile loads of the FP32 stage kernel, one per state
        // buffer a stage can read; without them (column length not a multiple
        // of 4, or no driver entry point) the tiles are loaded by cp.async
        void *encode = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &encode, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            encode = nullptr;
        cudaGetLastError();
        const void *bufs[4] = {c->ybuf[0], c->ybuf[1], c->Xa, c->Xb};
        for (int b = 0; b < 4 && encode; b++) {
            if (!bufs[b]) continue;
            auto &m = c->tmaps[c->ntmaps];
            m.ok[0] = stage_tensor_map(m.map[0], (const float *)bufs[b], Nx, Ny, Nz, 8, 16, encode);
            m.ok[1] = stage_tensor_map(m.map[1], (const float *)bufs[b], Nx, Ny, Nz, 8, 8, encode);
            if (m.ok[0] || m.ok[1]) {
                m.ptr = bufs[b];
                c->ntmaps++;
            }
        }
        // the RK operands' cell boxes (WF_NO_PREFETCH=1: none, for comparisons)
        const void *cbufs[3] = {c->ybuf[0], c->ybuf[1], c->acc};
        const bool no_pf = getenv("WF_NO_PREFETCH") && atoi(getenv("WF_NO_PREFETCH"));
        for (int b = 0; b < 3 && encode && !no_pf; b++) {
            if (!cbufs[b]) continue;
            auto &m = c->cmaps[c->ncmaps];
            m.ok[0] = stage_cell_map(m.map[0], (const float *)cbufs[b], Nx, Ny, Nz, 8, 16, encode);
            m.ok[1] = stage_cell_map(m.map[1], (const float *)cbufs[b], Nx, Ny, Nz, 8, 8, encode);
            if (m.ok[0] || m.ok[1]) {
                m.ptr = cbufs[b];
                c->ncmaps++;
            }
        }
    }
    c->launches = launches_per_step(c);
    *out = c;
    return WF_OK;
}

wf_status wf_destroy(wf_ctx *c)
{
    if (!c) return WF_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    dumper_destroy(c->dump);
    drop_graphs(c);
    for (auto &pl : c->ploop)
        if (pl.ge) cudaGraphExecDestroy(pl.ge);
    for (auto &b : c->bufs) cudaFree(b.p);
    if (c->up) cudaStreamSynchronize(c->up);
    if (c->ev_y) cudaEventDestroy(c->ev_y);
    if (c->ev_p) cudaEventDestroy(c->ev_p);
    for (int b = 0; b < 2; b++) {
        if (c->ev_copy[b]) cudaEventDestroy(c->ev_copy[b]);
        if (c->ev_conv[b]) cudaEventDestroy(c->ev_conv[b]);
    }
    if (c->up) cudaStreamDestroy(c->up);
    if (c->aux) cudaStreamDestroy(c->aux);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
    return WF_OK;
}

wf_status wf_upload_state(wf_ctx *c, const double *y, const double *pr)
{
    const NvtxRange range("wf_upload_state");
    if (!c || !y || !pr) { set_error("wf_upload_state: null argument"); return WF_ERR_ARG; }
    wf_status st = settle_p(c);
    if (st) return st;
    c->cur = 0;
    c->n = 0;
    if ((st = put_state(c, c->ybuf[0], y))) return st;
    WF_TRY_CUDA(cudaMemcpyAsync(c->p, pr, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    return finish_upload(c);
}

wf_status wf_upload_state_async(wf_ctx *c, const double *y, const double *pr)
{
    const NvtxRange range("wf_upload_state_async");
    if (!c || !y || !pr) { set_error("wf_upload_state_async: null argument"); return WF_ERR_ARG; }
    wf_status st = settle_p(c);
    if (st) return st;
    c->cur = 0;
    c->n = 0;
    if ((st = put_state(c, c->ybuf[0], y))) return st;
    // p after the state on the host link, on its own stream
    WF_TRY_CUDA(cudaEventRecord(c->ev_y, c->stream));
    WF_TRY_CUDA(cudaStreamWaitEvent(c->up, c->ev_y, 0));
    WF_TRY_CUDA(cudaMemcpyAsync(c->p, pr, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->up));
    WF_TRY_CUDA(cudaEventRecord(c->ev_p, c->up));
    c->p_pending = true;
    return finish_upload(c);   // waits for the state only
}

wf_status wf_initial_conditions(wf_ctx *c)
{
    if (!c) { set_error("wf_initial_conditions: null context"); return WF_ERR_ARG; }
    if (const wf_status st0 = settle_p(c)) return st0;
    const Parameters &P = c->P;
    IcArgs a;
    memset(&a, 0, sizeof(a));
    if (strcmp(P.T0_shape, "gaussian") == 0) a.T_shape = 0;
    else if (strcmp(P.T0_shape, "parallelepiped") == 0) a.T_shape = 1;
    else {
        set_error("wf_initial_conditions: T0_shape '%s' is neither gaussian nor parallelepiped", P.T0_shape);
        return WF_ERR_ARG;
    }
    a.u_r = P.u_r; a.z_r = P.z_r; a.alpha_u = P.alpha_u;
    a.T_0 = P.T_0; a.T_inf = P.T_inf;
    a.x0 = P.T0_x_center; a.y0 = P.T0_y_center; a.z0 = P.T0_z_center;
    a.sx = P.T0_length; a.sy = P.T0_width; a.sz = P.T0_height;
    a.Tx0 = P.T0_x_start; a.Tx1 = P.T0_x_end; a.Ty0 = P.T0_y_start; a.Ty1 = P.T0_y_end;
    a.Tz0 = P.T0_z_start; a.Tz1 = P.T0_z_end;
    a.Yx0 = P.Y0_x_start; a.Yx1 = P.Y0_x_end; a.Yy0 = P.Y0_y_start; a.Yy1 = P.Y0_y_end;
    a.xa = P.Y0_xa; a.ya = P.Y0_ya; a.Y_h = P.Y_h;
    a.p_top = P.p_top;
    a.dead[0] = P.u_dead_nodes; a.dead[1] = P.v_dead_nodes; a.dead[2] = P.w_dead_nodes;
    a.dead[3] = P.T_dead_nodes; a.dead[4] = P.Y_dead_nodes;
    c->cur = 0;
    c->n = 0;
    cudaError_t e = (c->prec == WF_FP64)
                        ? launch_initial_conditions<double>(c->geom, a, c->d_x, c->d_y, (double *)c->ybuf[0], c->p,
                                                            c->stream)
                        : launch_initial_conditions<float>(c->geom, a, c->d_x, c->d_y, (float *)c->ybuf[0], c->p,
                                                           c->stream);
    if (e != cudaSuccess) { set_error("wf_initial_conditions: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    return finish_upload(c);
}

}  // extern "C"

namespace wfs {
// After a new initial state: the held temperature source, then the fuel
// integral the diagnostics report consumption against.
wf_status finish_upload(wf_ctx *c)
{
    if (c->Tsrc) {
        // the held source is the initial temperature field (solver.cu:169)
        WF_TRY_CUDA(cudaMemcpyAsync(c->Tsrc, (char *)c->ybuf[0] + (size_t)3 * c->N * c->esz, (size_t)c->N * c->esz,
                                    cudaMemcpyDeviceToDevice, c->stream));
    }
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    wf_diag d;
    const wf_status st = wf_diagnostics(c, &d);
    c->fuel0 = d.fuel;
    return st == WF_ERR_NAN ? WF_OK : st;
}

// Tile shape of the fused stage pass for this context.  WF_STAGE_TILE=TIxTJ in
// the environment forces a shape; otherwise, when more than one shape is
// compiled, each is timed on the context's own grid and current state (a
// stage that stores k_s into a scratch buffer, so the state is untouched: one
// warm-up launch, then enough launches for about 2 ms, at least 3) and the
// fastest kept.  Every shape gives
// bit-identical results: a cell's arithmetic does not depend on the tiling.
template <class R> wf_status tune_tiles_impl(wf_ctx *c)
{
    const int prec = c->prec == WF_FP64 ? 0 : 1, count = stage_tile_count(prec);
    c->tile_set = true;
    if (const char *env = getenv("WF_STAGE_TILE")) {
        int ti = 0, tj = 0, nt = 0;
        const int got = sscanf(env, "%dx%d/%d", &ti, &tj, &nt);   // TIxTJ, optionally /threads
        if (got >= 2)
            for (int q = 0; q < count; q++) {
                int a = 0, b = 0, n = 0;
                stage_tile_shape(prec, q, &a, &b, &n);
                if (a == ti && b == tj && (got < 3 || n == nt)) { c->tile = q; return WF_OK; }
            }
        set_error("WF_STAGE_TILE=%s is not a compiled tile shape", env);
        return WF_ERR_ARG;
    }
    if (count < 2) return WF_OK;
    void *in = c->ybuf[c->cur], *scratch = c->Xa ? c->Xa : c->ybuf[1 - c->cur];
    const int saved = c->method;
    c->method = 3;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        c->method = saved;
        set_error("stage tile tuning: %s", cudaGetErrorString(cudaGetLastError()));
        return WF_ERR_CUDA;
    }
    float best = 1e30f;
    int pick = 0;
    cudaError_t err = cudaSuccess;
    for (int q = 0; q < count && !err; q++) {
        c->tile = q;
        const StageArgs<R> a = stage_args<R>(c, in, in, scratch, 1);
        float ms = 0.0f;
        int reps = 1;
        for (int pass = 0; pass < 2 && !err; pass++) {   // pass 0 warms up and sizes pass 1
            err = cudaEventRecord(e0, c->stream);
            for (int r = 0; r < reps && !err; r++) err = launch_stage<R>(a, c->stream);
            if (!err) err = cudaEventRecord(e1, c->stream);
            if (!err) err = cudaEventSynchronize(e1);
            if (!err) err = cudaEventElapsedTime(&ms, e0, e1);
            if (pass == 0) reps = ms > 0.0f ? (int)fminf(fmaxf(2.0f / ms, 3.0f), 64.0f) : 3;
        }
        ms /= (float)reps;
        if (!err && ms < best) { best = ms; pick = q; }
    }
    c->method = saved;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tile = pick;
    if (err) { set_error("stage tile tuning: %s", cudaGetErrorString(err)); return WF_ERR_CUDA; }
    return WF_OK;
}

wf_status tune_tiles(wf_ctx *c)
{
    if (c->tile_set) return WF_OK;
    return c->prec == WF_FP64 ? tune_tiles_impl<double>(c) : tune_tiles_impl<float>(c);
}
}  // namespace wfs

extern "C" {

wf_status wf_download_state(wf_ctx *c, double *y, double *pr)
{
    const NvtxRange range("wf_download_state");
    if (!c || !y || !pr) { set_error("wf_download_state: null argument"); return WF_ERR_ARG; }
    wf_status st = settle_p(c);
    if (st) return st;
    st = get_state(c, y, c->ybuf[c->cur]);
    if (st) return st;
    WF_TRY_CUDA(cudaMemcpyAsync(pr, c->p, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    return WF_OK;
}

wf_status wf_step(wf_ctx *c, int nsteps)
{
    const NvtxRange range("wf_step");
    if (!c || nsteps < 0) { set_error("wf_step: invalid argument"); return WF_ERR_ARG; }
    if (nsteps > 0) {
        const wf_status st = tune_tiles(c);
        if (st) return st;
    }
    for (int q = 0; q < nsteps; q++) {
        const int n1 = c->n + 1;
        if (step_is_static(c, n1)) {
            cudaGraphExec_t &ge = c->graph[c->cur];
            if (!ge) {
                // captured on the context's own stream (a caller's stream may be
                // one that cannot be captured, such as the legacy default stream)
                // and launched on the current one
                cudaGraph_t gph = nullptr;
                const cudaStream_t user = c->stream;
                c->stream = c->own;
                WF_TRY_CUDA(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
                wf_status st = enqueue_step_any(c, c->cur, n1);
                cudaError_t e = cudaStreamEndCapture(c->own, &gph);
                c->stream = user;
                if (st) {
                    if (gph) cudaGraphDestroy(gph);
                    return st;
                }
                if (e != cudaSuccess) { set_error("wf_step: capture failed: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
                e = cudaGraphInstantiate(&ge, gph, 0);
                cudaGraphDestroy(gph);
                if (e != cudaSuccess) { set_error("wf_step: instantiate failed: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
            }
            WF_TRY_CUDA(cudaGraphLaunch(ge, c->stream));
        } else {
            wf_status st = enqueue_step_any(c, c->cur, n1);
            if (st) return st;
        }
        c->p_pending = false;   // the step waited for an asynchronous copy of p
        c->cur = 1 - c->cur;
        c->n = n1;
    }
    return WF_OK;
}

wf_status wf_synchronize(wf_ctx *c)
{
    if (!c) return WF_ERR_ARG;
    if (const wf_status st0 = settle_p(c)) return st0;
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    if (c->d_kerr) {
        int herr = 0;
        WF_TRY_CUDA(cudaMemcpy(&herr, c->d_kerr, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) {
            WF_TRY_CUDA(cudaMemset(c->d_kerr, 0, sizeof(int)));
            set_error("wf_synchronize: a stage kernel's wait for its tile load timed out");
            return WF_ERR_CUDA;
        }
    }
    if (c->closure && c->d_closure_err) {
        int herr = 0;
        WF_TRY_CUDA(cudaMemcpy(&herr, c->d_closure_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) {
            // reported once: the flag is cleared so that later calls start clean
            WF_TRY_CUDA(cudaMemset(c->d_closure_err, 0, sizeof(int)));
            set_error("wf_synchronize: a closure tensor-core completion wait timed out");
            return WF_ERR_CUDA;
        }
    }
    return WF_OK;
}

wf_status wf_time(const wf_ctx *c, int *n, double *t)
{
    if (!c) return WF_ERR_ARG;
    if (n) *n = c->n;
    if (t) *t = c->P.t_min + c->n * c->P.dt;
    return WF_OK;
}

wf_status wf_timestep_reports(wf_ctx *c, wf_report *out)
{
    const NvtxRange range("wf_timestep_reports");
    if (!c || !out) { set_error("wf_timestep_reports: null argument"); return WF_ERR_ARG; }
    const double rect[4] = {c->P.Y0_x_start, c->P.Y0_x_end, c->P.Y0_y_start, c->P.Y0_y_end};
    cudaError_t e = (c->prec == WF_FP64)
                        ? launch_report<double>(c->geom, (const double *)c->ybuf[c->cur], c->d_x, c->d_y, rect, c->d_rep,
                                                c->stream)
                        : launch_report<float>(c->geom, (const float *)c->ybuf[c->cur], c->d_x, c->d_y, rect, c->d_rep,
                                               c->stream);
    if (e != cudaSuccess) { set_error("wf_timestep_reports: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    double h[8];
    WF_TRY_CUDA(cudaMemcpyAsync(h, c->d_rep, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    // functions.cu:180, same operation order
    out->cfl = c->P.dt * (h[0] / c->P.dx + h[1] / c->P.dy + h[2] / c->P.dz);
    out->T_min = 0.0 - h[3];
    out->T_max = h[4];
    out->Y_min = 0.0 - h[5];
    out->Y_max = h[6];
    unsigned long long key;
    memcpy(&key, &h[7], sizeof(key));
    out->nan_field = out->nan_i = out->nan_j = out->nan_k = -1;
    if (key != ~0ull) {
        const unsigned long long cell = key / 5;
        out->nan_field = (int)(key % 5);
        out->nan_k = (int)(cell % (unsigned long long)c->Nz);
        out->nan_j = (int)((cell / c->Nz) % (unsigned long long)c->Ny);
        out->nan_i = (int)(cell / ((unsigned long long)c->Nz * c->Ny));
    }
    return WF_OK;
}

wf_status wf_stage_tile(const wf_ctx *c, int *ti, int *tj, int *threads)
{
    if (!c || !ti || !tj) { set_error("wf_stage_tile: null argument"); return WF_ERR_ARG; }
    stage_tile_shape(c->prec == WF_FP64 ? 0 : 1, c->tile, ti, tj, threads);
    return WF_OK;
}

wf_status wf_set_stage_tile(wf_ctx *c, int ti, int tj, int threads)
{
    if (!c) { set_error("wf_set_stage_tile: null context"); return WF_ERR_ARG; }
    const int prec = c->prec == WF_FP64 ? 0 : 1;
    for (int q = 0; q < stage_tile_count(prec); q++) {
        int a = 0, b = 0, n = 0;
        stage_tile_shape(prec, q, &a, &b, &n);
        if (a == ti && b == tj && (threads <= 0 || n == threads)) {
            c->tile = q;
            c->tile_set = true;
            drop_graphs(c);
            return WF_OK;
        }
    }
    set_error("wf_set_stage_tile: %dx%d with %d threads is not a compiled tile shape", ti, tj, threads);
    return WF_ERR_ARG;
}

wf_status wf_dump_async(wf_ctx *c, const char *dir, int n)
{
    const NvtxRange range("wf_dump_async");
    if (!c || !dir) { set_error("wf_dump_async: null argument"); return WF_ERR_ARG; }
    if (const wf_status st0 = settle_p(c)) return st0;
    if (!c->dump) c->dump = dumper_create(c->device, c->P, c->S, (size_t)c->N);
    return dumper_enqueue(c->dump, c->stream, c->ybuf[c->cur], c->prec != WF_FP64, c->p, dir, n);
}

wf_status wf_dump_wait(wf_ctx *c)
{
    if (!c) { set_error("wf_dump_wait: null context"); return WF_ERR_ARG; }
    return dumper_wait(c->dump);
}

wf_status wf_diagnostics(wf_ctx *c, wf_diag *out)
{
    const NvtxRange range("wf_diagnostics");
    if (!c || !out) return WF_ERR_ARG;
    cudaError_t e = (c->prec == WF_FP64)
                        ? launch_diag<double>(c->geom, c->ph, (const double *)c->ybuf[c->cur], nullptr, c->d_diag, c->stream)
                        : launch_diag<float>(c->geom, c->ph, (const float *)c->ybuf[c->cur], nullptr, c->d_diag, c->stream);
    if (e != cudaSuccess) { set_error("wf_diagnostics: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    double h[13];
    WF_TRY_CUDA(cudaMemcpyAsync(h, c->d_diag, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    out->mass = h[0];
    out->energy = h[1];
    out->fuel = h[2];
    out->fuel_consumed = c->fuel0 - h[2];
    out->max_abs_u = h[4];
    out->max_abs_v = h[5];
    out->max_abs_w = h[6];
    out->T_min = -h[7];
    out->T_max = h[8];
    out->Y_min = -h[9];
    out->Y_max = h[10];
    out->nan_count = (long long)h[12];
    out->cfl = c->P.dt * (h[4] / c->P.dx + h[5] / c->P.dy + h[6] / c->P.dz);
    return out->nan_count ? WF_ERR_NAN : WF_OK;
}

wf_status wf_device_state(wf_ctx *c, void **y, double **pr)
{
    if (!c) return WF_ERR_ARG;
    if (const wf_status st0 = settle_p(c)) return st0;   // work enqueued on wf_stream sees p
    if (y) *y = c->ybuf[c->cur];
    if (pr) *pr = c->p;
    return WF_OK;
}

void *wf_stream(wf_ctx *c) { return c ? (void *)c->stream : nullptr; }

int wf_launches_per_step(const wf_ctx *c) { return c ? c->launches : 0; }

const char *wf_phase_name(int q) { return (q >= 0 && q < WF_NPHASES) ? kPhaseNames[q] : nullptr; }

wf_status wf_profile_phases(wf_ctx *c, int nsteps, double *ms, int *launches)
{
    if (!c || !ms || !launches || nsteps < 1) { set_error("wf_profile_phases: invalid argument"); return WF_ERR_ARG; }
    if (const wf_status st0 = settle_p(c)) return st0;
    for (int q = 0; q < WF_NPHASES; q++) { ms[q] = 0.0; launches[q] = 0; }
    const int maxev = 2 + 3 * 4 + 5 * (c->P.pressure_solver_iter > 1 ? c->P.pressure_solver_iter : 1);
    std::vector<cudaEvent_t> ev(maxev, nullptr);
    for (auto &e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            e = nullptr;
            for (auto &d : ev)
                if (d) cudaEventDestroy(d);
            set_error("wf_profile_phases: %s", cudaGetErrorString(cudaGetLastError()));
            return WF_ERR_CUDA;
        }
    wf_status st = WF_OK;
    for (int it = 0; it < nsteps && st == WF_OK; it++) {
        int ne = 0;
        st = (c->prec == WF_FP64) ? profile_step<double>(c, ev.data(), ne) : profile_step<float>(c, ev.data(), ne);
        if (st) break;
        if (cudaEventSynchronize(ev[ne - 1]) != cudaSuccess) { set_error("wf_profile_phases: sync failed"); st = WF_ERR_CUDA; break; }
        // kinds in launch order: stages (3 each), solves (5 each), projection
        int e = 0;
        auto add = [&](int kind) {
            float t = 0.f;
            cudaEventElapsedTime(&t, ev[e], ev[e + 1]);
            ms[kind] += t;
            launches[kind] += 1;
            e++;
        };
        for (int sidx = 0; sidx < c->nstages; sidx++) { add(0); add(1); add(2); }
        while (e < ne - 2) { add(3); add(4); add(5); add(6); add(7); }
        add(8);
        c->cur = 1 - c->cur;
        c->n += 1;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return st;
}

wf_status wf_phi(wf_ctx *c, const double *R_old, double *R_new)
{
    if (!c || !R_old || !R_new) { set_error("wf_phi: null argument"); return WF_ERR_ARG; }
    void *in = c->ybuf[1 - c->cur], *outb = c->Xa ? c->Xa : c->ybuf[c->cur];
    wf_status st = put_state(c, in, R_old);
    if (st) return st;
    const int saved = c->method;
    c->method = 3;
    cudaError_t e;
    if (c->prec == WF_FP64) e = launch_stage<double>(stage_args<double>(c, in, in, outb, 1), c->stream);
    else e = launch_stage<float>(stage_args<float>(c, in, in, outb, 1), c->stream);
    c->method = saved;
    if (e != cudaSuccess) { set_error("wf_phi: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    // fuel entries above each column's fuel top are never written: zero them
    st = get_state(c, R_new, outb);
    if (st) return st;
    for (int col = 0; col < c->Nx * c->Ny; col++)
        for (int k = c->hnzy[col]; k < c->NzY; k++) R_new[(size_t)4 * c->N + (size_t)col * c->NzY + k] = 0.0;
    drop_graphs(c);
    return WF_OK;
}

wf_status wf_pressure(wf_ctx *c, const double *y_np1, const double *y_n, double *pr, int *iters)
{
    const NvtxRange range("wf_pressure");
    if (!c || !y_np1 || !y_n || !pr) { set_error("wf_pressure: null argument"); return WF_ERR_ARG; }
    if (const wf_status st0 = settle_p(c)) return st0;
    void *b1 = c->ybuf[1 - c->cur], *bn = c->Xa ? c->Xa : c->ybuf[c->cur];
    wf_status st = put_state(c, b1, y_np1);
    if (st) return st;
    if ((st = put_state(c, bn, y_n))) return st;
    WF_TRY_CUDA(cudaMemcpyAsync(c->p, pr, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->stream));
    st = (c->prec == WF_FP64) ? enqueue_pressure<double>(c, b1, bn) : enqueue_pressure<float>(c, b1, bn);
    if (st) return st;
    int it = 1;
    if ((st = read_piter(c, &it, nullptr, nullptr))) return st;
    WF_TRY_CUDA(cudaMemcpyAsync(pr, c->p, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    if (iters) *iters = it;
    drop_graphs(c);
    return WF_OK;
}

// ---- ensemble: independent members stepped together -----------------------
// One CUDA graph per ensemble step holds every member's step as a branch of
// its own (the members' streams fork from and join back to one stream), so the
// GPU runs the members' kernels concurrently and one graph launch replaces
// 18 launches per member.  Members whose step is not static (ignition source
// active) are enqueued eagerly on their own streams instead.
}  // extern "C"

struct wf_ensemble {
    std::vector<wf_ctx *> m;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int parity = 0;
};

namespace wfs {

void ensemble_drop_graphs(wf_ensemble *e)
{
    for (int q = 0; q < 2; q++)
        if (e->graph[q]) {
            cudaGraphExecDestroy(e->graph[q]);
            e->graph[q] = nullptr;
        }
}

wf_status ensemble_enqueue(wf_ensemble *e)
{
    WF_TRY_CUDA(cudaEventRecord(e->fork, e->master));
    for (size_t i = 0; i < e->m.size(); i++) {
        wf_ctx *c = e->m[i];
        WF_TRY_CUDA(cudaStreamWaitEvent(c->stream, e->fork, 0));
        wf_status st = enqueue_step_any(c, c->cur, c->n + 1);
        if (st) return st;
        WF_TRY_CUDA(cudaEventRecord(e->join[i], c->stream));
        WF_TRY_CUDA(cudaStreamWaitEvent(e->master, e->join[i], 0));
    }
    return WF_OK;
}

}  // namespace wfs

extern "C" {

wf_status wf_ensemble_create(const Parameters *members, int n_members, int precision, wf_ensemble **out)
{
    if (!members || n_members < 1 || !out) { set_error("wf_ensemble_create: invalid argument"); return WF_ERR_ARG; }
    *out = nullptr;
    wf_ensemble *e = new wf_ensemble();
    auto fail = [&](wf_status st) {
        wf_ensemble_destroy(e);
        return st;
    };
    if (cudaStreamCreateWithFlags(&e->master, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) != cudaSuccess) {
        set_error("wf_ensemble_create: stream or event creation failed");
        return fail(WF_ERR_CUDA);
    }
    for (int i = 0; i < n_members; i++) {
        wf_ctx *c = nullptr;
        wf_status st = wf_create(&members[i], precision, &c);
        if (st) return fail(st);
        c->member = true;
        e->m.push_back(c);
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            set_error("wf_ensemble_create: event creation failed");
            return fail(WF_ERR_CUDA);
        }
        e->join.push_back(ev);
    }
    *out = e;
    return WF_OK;
}

wf_status wf_ensemble_destroy(wf_ensemble *e)
{
    if (!e) return WF_OK;
    if (e->master) cudaStreamSynchronize(e->master);
    ensemble_drop_graphs(e);
    for (wf_ctx *c : e->m) wf_destroy(c);
    for (cudaEvent_t ev : e->join) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->master) cudaStreamDestroy(e->master);
    delete e;
    return WF_OK;
}

int wf_ensemble_size(const wf_ensemble *e) { return e ? (int)e->m.size() : 0; }

void *wf_ensemble_stream(wf_ensemble *e) { return e ? (void *)e->master : nullptr; }

void wf_inject_allocation_failure(int after) { g_alloc_budget.store(after < 0 ? -1 : after); }

wf_ctx *wf_ensemble_member(wf_ensemble *e, int i)
{
    return (e && i >= 0 && i < (int)e->m.size()) ? e->m[i] : nullptr;
}

wf_status wf_ensemble_step(wf_ensemble *e, int nsteps)
{
    const NvtxRange range("wf_ensemble_step");
    if (!e || nsteps < 0) { set_error("wf_ensemble_step: invalid argument"); return WF_ERR_ARG; }
    for (wf_ctx *c : e->m) {
        const wf_status st = nsteps > 0 ? tune_tiles(c) : WF_OK;
        if (st) return st;
    }
    for (int q = 0; q < nsteps; q++) {
        bool same = true, fixed = true;
        for (wf_ctx *c : e->m) {
            same = same && c->cur == e->m[0]->cur;
            fixed = fixed && step_is_static(c, c->n + 1);
        }
        if (same && fixed) {
            cudaGraphExec_t &ge = e->graph[e->m[0]->cur];
            if (!ge) {
                cudaGraph_t gph = nullptr;
                WF_TRY_CUDA(cudaStreamBeginCapture(e->master, cudaStreamCaptureModeThreadLocal));
                wf_status st = ensemble_enqueue(e);
                cudaError_t err = cudaStreamEndCapture(e->master, &gph);
                if (st) {
                    if (gph) cudaGraphDestroy(gph);
                    return st;
                }
                if (err != cudaSuccess) { set_error("wf_ensemble_step: capture failed: %s", cudaGetErrorString(err)); return WF_ERR_CUDA; }
                err = cudaGraphInstantiate(&ge, gph, 0);
                cudaGraphDestroy(gph);
                if (err != cudaSuccess) { set_error("wf_ensemble_step: instantiate failed: %s", cudaGetErrorString(err)); return WF_ERR_CUDA; }
            }
            WF_TRY_CUDA(cudaGraphLaunch(ge, e->master));
        } else {
            wf_status st = ensemble_enqueue(e);
            if (st) return st;
        }
        for (wf_ctx *c : e->m) {
            c->cur = 1 - c->cur;
            c->n += 1;
        }
    }
    return WF_OK;
}

wf_status wf_ensemble_synchronize(wf_ensemble *e)
{
    if (!e) return WF_ERR_ARG;
    WF_TRY_CUDA(cudaStreamSynchronize(e->master));
    for (wf_ctx *c : e->m) WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    return WF_OK;
}

// ---- learned closure --------------------------------------------------------
int wf_closure_param_count(void) { return closure_param_count(); }

wf_status wf_set_closure(wf_ctx *c, int kind, const float *params)
{
    if (!c || (kind != WF_CLOSURE_SMAGORINSKY && kind != WF_CLOSURE_MLP) || (kind == WF_CLOSURE_MLP && !params)) {
        set_error("wf_set_closure: invalid argument");
        return WF_ERR_ARG;
    }
    drop_graphs(c);
    if (kind == WF_CLOSURE_SMAGORINSKY) {
        c->closure = 0;
        c->launches = launches_per_step(c);
        return WF_OK;
    }
    wf_status st;
    if (!c->d_theta) {
        void *p = nullptr;
        if ((st = dev_alloc(c, &p, sizeof(float) * closure_param_count()))) return st;
        c->d_theta = (float *)p;
        if ((st = dev_alloc(c, &c->coef, c->esz * (size_t)c->N))) return st;
        if ((st = dev_alloc(c, &p, sizeof(int)))) return st;
        c->d_closure_err = (int *)p;
        WF_TRY_CUDA(cudaMemset(c->d_closure_err, 0, sizeof(int)));
    }
    WF_TRY_CUDA(cudaMemcpy(c->d_theta, params, sizeof(float) * closure_param_count(), cudaMemcpyHostToDevice));
    c->closure = 1;
    c->launches = launches_per_step(c);
    return WF_OK;
}

wf_status wf_closure_coefficients(wf_ctx *c, const double *y, double *coef)
{
    if (!c || !y || !coef) { set_error("wf_closure_coefficients: null argument"); return WF_ERR_ARG; }
    if (!c->closure) { set_error("wf_closure_coefficients: no learned closure set"); return WF_ERR_ARG; }
    void *in = c->ybuf[1 - c->cur];
    wf_status st = put_state(c, in, y);
    if (st) return st;
    WF_TRY_CUDA(cudaMemsetAsync(c->d_closure_err, 0, sizeof(int), c->stream));
    cudaError_t e = (c->prec == WF_FP64)
                        ? launch_closure_coef_tc<double>((const double *)in, c->geom, c->ph.dx, c->ph.dy, c->d_theta,
                                                         (double *)c->coef, c->d_closure_err, c->stream,
                                                         c->closure_wait)
                        : launch_closure_coef_tc<float>((const float *)in, c->geom, c->ph.dx, c->ph.dy, c->d_theta,
                                                        (float *)c->coef, c->d_closure_err, c->stream, c->closure_wait);
    if (e) { set_error("wf_closure_coefficients: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    int herr = 0;
    WF_TRY_CUDA(cudaMemcpyAsync(&herr, c->d_closure_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    if (herr) { set_error("wf_closure_coefficients: a tensor-core completion wait timed out"); return WF_ERR_CUDA; }
    if (c->prec == WF_FP64) {
        WF_TRY_CUDA(cudaMemcpyAsync(coef, c->coef, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->stream));
        WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
    } else {
        std::vector<float> h(c->N);
        WF_TRY_CUDA(cudaMemcpyAsync(h.data(), c->coef, sizeof(float) * c->N, cudaMemcpyDeviceToHost, c->stream));
        WF_TRY_CUDA(cudaStreamSynchronize(c->stream));
        for (int q = 0; q < c->N; q++) coef[q] = h[q];
    }
    drop_graphs(c);
    return WF_OK;
}

wf_status wf_set_closure_wait_limit(wf_ctx *c, int polls)
{
    if (!c || polls < 0) { set_error("wf_set_closure_wait_limit: invalid argument"); return WF_ERR_ARG; }
    drop_graphs(c);   // captured steps carry the limit
    c->closure_wait = polls;
    return WF_OK;
}

}  // extern "C"

namespace wfs {

// Device scratch of the training entry points, released on every path.
struct TrainBuffers {
    std::vector<void *> p;
    void *get(size_t bytes)
    {
        void *q = nullptr;
        if (cudaMalloc(&q, bytes ? bytes : 16) != cudaSuccess) return nullptr;
        p.push_back(q);
        return q;
    }
    ~TrainBuffers()
    {
        for (void *q : p) cudaFree(q);
    }
};

}  // namespace wfs

extern "C" {

wf_status wf_closure_predict(const float *params, const float *features, size_t n, float *out)
{
    if (!params || !features || !out || !n || n > (size_t)1 << 30) {
        set_error("wf_closure_predict: invalid argument");
        return WF_ERR_ARG;
    }
    const int np = closure_param_count();
    TrainBuffers b;
    float *dth = (float *)b.get(sizeof(float) * np), *dx = (float *)b.get(sizeof(float) * 12 * n);
    float *dout = (float *)b.get(sizeof(float) * n);
    int *derr = (int *)b.get(sizeof(int));
    if (!dth || !dx || !dout || !derr) { set_error("wf_closure_predict: device allocation failed"); return WF_ERR_OOM; }
    WF_TRY_CUDA(cudaMemcpy(dth, params, sizeof(float) * np, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(cudaMemcpy(dx, features, sizeof(float) * 12 * n, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(cudaMemset(derr, 0, sizeof(int)));
    WF_TRY_CUDA(launch_closure_predict(dth, dx, n, dout, derr, 0));
    int herr = 0;
    WF_TRY_CUDA(cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) { set_error("wf_closure_predict: a tensor-core completion wait timed out"); return WF_ERR_CUDA; }
    WF_TRY_CUDA(cudaMemcpy(out, dout, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return WF_OK;
}

wf_status wf_mlp_loss_grad(const float *theta, const float *x, const float *y, size_t n, double *loss, float *grad)
{
    if (!theta || !x || !y || !n || !loss || !grad || n > (size_t)1 << 30) {
        set_error("wf_mlp_loss_grad: invalid argument");
        return WF_ERR_ARG;
    }
    const int np = closure_param_count();
    TrainBuffers b;
    float *dth = (float *)b.get(sizeof(float) * np), *dx = (float *)b.get(sizeof(float) * 12 * n);
    float *dy = (float *)b.get(sizeof(float) * n), *dg = (float *)b.get(sizeof(float) * np);
    double *dl = (double *)b.get(sizeof(double));
    if (!dth || !dx || !dy || !dg || !dl) { set_error("wf_mlp_loss_grad: device allocation failed"); return WF_ERR_OOM; }
    WF_TRY_CUDA(cudaMemcpy(dth, theta, sizeof(float) * np, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(cudaMemcpy(dx, x, sizeof(float) * 12 * n, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(cudaMemcpy(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(launch_mlp_grad(dth, dx, dy, nullptr, (int)n, dg, dl, 0));
    WF_TRY_CUDA(cudaMemcpy(grad, dg, sizeof(float) * (np - 12), cudaMemcpyDeviceToHost));
    WF_TRY_CUDA(cudaMemcpy(loss, dl, sizeof(double), cudaMemcpyDeviceToHost));
    for (int q = np - 12; q < np; q++) grad[q] = 0.0f;   // feature scales are not trained
    return WF_OK;
}

wf_status wf_mlp_train(float *theta, const float *x, const float *y, size_t n, int steps, int batch, float lr,
                       unsigned long long seed, double *loss_history)
{
    if (!theta || !x || !y || n < 1 || steps < 1 || batch < 1 || n > (size_t)1 << 30) {
        set_error("wf_mlp_train: invalid argument");
        return WF_ERR_ARG;
    }
    if ((size_t)batch > n) batch = (int)n;
    const int np = closure_param_count();
    TrainBuffers b;
    float *dth = (float *)b.get(sizeof(float) * np), *dm = (float *)b.get(sizeof(float) * np);
    float *dv = (float *)b.get(sizeof(float) * np), *dg = (float *)b.get(sizeof(float) * np);
    float *dx = (float *)b.get(sizeof(float) * 12 * n), *dy = (float *)b.get(sizeof(float) * n);
    int *didx = (int *)b.get(sizeof(int) * (size_t)batch * steps);
    double *dl = (double *)b.get(sizeof(double) * steps);
    if (!dth || !dm || !dv || !dg || !dx || !dy || !didx || !dl) {
        set_error("wf_mlp_train: device allocation failed");
        return WF_ERR_OOM;
    }
    WF_TRY_CUDA(cudaMemcpy(dth, theta, sizeof(float) * np, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(cudaMemset(dm, 0, sizeof(float) * np));
    WF_TRY_CUDA(cudaMemset(dv, 0, sizeof(float) * np));
    WF_TRY_CUDA(cudaMemcpy(dx, x, sizeof(float) * 12 * n, cudaMemcpyHostToDevice));
    WF_TRY_CUDA(cudaMemcpy(dy, y, sizeof(float) * n, cudaMemcpyHostToDevice));
    // minibatches: a fresh seeded permutation of the samples per epoch (splitmix64)
    std::vector<int> idx((size_t)batch * steps), perm(n);
    unsigned long long s = seed;
    auto next = [&]() {
        unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    size_t pos = n;
    for (size_t q = 0; q < idx.size(); q++) {
        if (pos == n) {
            for (size_t i = 0; i < n; i++) perm[i] = (int)i;
            for (size_t i = n - 1; i > 0; i--) std::swap(perm[i], perm[next() % (i + 1)]);
            pos = 0;
        }
        idx[q] = perm[pos++];
    }
    WF_TRY_CUDA(cudaMemcpy(didx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice));
    for (int t = 0; t < steps; t++) {
        WF_TRY_CUDA(launch_mlp_grad(dth, dx, dy, didx + (size_t)t * batch, batch, dg, dl + t, 0));
        WF_TRY_CUDA(launch_adam(dth, dm, dv, dg, t + 1, lr, 0));
    }
    WF_TRY_CUDA(cudaMemcpy(theta, dth, sizeof(float) * (np - 12), cudaMemcpyDeviceToHost));
    if (loss_history) WF_TRY_CUDA(cudaMemcpy(loss_history, dl, sizeof(double) * steps, cudaMemcpyDeviceToHost));
    return WF_OK;
}

wf_status wf_pressure_report(const wf_ctx *c, double *error, int *max_iter)
{
    if (!c) { set_error("wf_pressure_report: null context"); return WF_ERR_ARG; }
    return read_piter(const_cast<wf_ctx *>(c), nullptr, error, max_iter);
}

wf_status wf_set_stream(wf_ctx *c, void *stream)
{
    if (!c) { set_error("wf_set_stream: null context"); return WF_ERR_ARG; }
    if (c->member) { set_error("wf_set_stream: an ensemble member runs on the ensemble's streams"); return WF_ERR_ARG; }
    const cudaStream_t next = stream ? (cudaStream_t)stream : c->own;
    if (next == c->stream) return WF_OK;
    // work already enqueued on the previous stream comes first
    cudaEvent_t ev = nullptr;
    WF_TRY_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, c->stream);
    if (!e) e = cudaStreamWaitEvent(next, ev, 0);
    cudaEventDestroy(ev);
    if (e) { set_error("wf_set_stream: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    c->stream = next;
    return WF_OK;
}

}  // extern "C"

namespace wfs {

// Fuel entries above each column's fuel top (k >= Nz_Y(i, j)) of a packed FP64
// state on the device, set to zero (Phi never writes them).
__global__ void k_zero_fuel_above(double *R, const int *__restrict__ nzy, int ncol, int NzY)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ncol * NzY) return;
    const int col = t / NzY, k = t % NzY;
    if (k >= nzy[col]) R[t] = 0.0;
}

// Packed FP64 device state -> stencil-precision device state, and back, on the
// context's stream (no host copy).
wf_status put_state_dev(wf_ctx *c, void *dst, const double *src)
{
    if (c->prec == WF_FP64) {
        WF_TRY_CUDA(cudaMemcpyAsync(dst, src, c->S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        return WF_OK;
    }
    k_to_prec<float><<<592, 256, 0, c->stream>>>((float *)dst, src, c->S);
    WF_TRY_CUDA(cudaGetLastError());
    return WF_OK;
}

wf_status get_state_dev(wf_ctx *c, double *dst, const void *src)
{
    if (c->prec == WF_FP64) {
        WF_TRY_CUDA(cudaMemcpyAsync(dst, src, c->S * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        return WF_OK;
    }
    k_from_prec<float><<<592, 256, 0, c->stream>>>(dst, (const float *)src, c->S);
    WF_TRY_CUDA(cudaGetLastError());
    return WF_OK;
}

}  // namespace wfs

extern "C" {

wf_status wf_phi_device(wf_ctx *c, const double *R_old, double *R_new)
{
    const NvtxRange range("wf_phi_device");
    if (!c || !R_old || !R_new) { set_error("wf_phi_device: null argument"); return WF_ERR_ARG; }
    void *in = c->ybuf[1 - c->cur], *outb = c->Xa ? c->Xa : c->ybuf[c->cur];
    wf_status st = put_state_dev(c, in, R_old);
    if (st) return st;
    const int saved = c->method;
    c->method = 3;
    cudaError_t e;
    if (c->prec == WF_FP64) e = launch_stage<double>(stage_args<double>(c, in, in, outb, 1), c->stream);
    else e = launch_stage<float>(stage_args<float>(c, in, in, outb, 1), c->stream);
    c->method = saved;
    if (e != cudaSuccess) { set_error("wf_phi_device: %s", cudaGetErrorString(e)); return WF_ERR_CUDA; }
    if ((st = get_state_dev(c, R_new, outb))) return st;
    const int ny = c->Nx * c->Ny * c->NzY;
    if (ny > 0) {
        k_zero_fuel_above<<<(ny + 255) / 256, 256, 0, c->stream>>>(R_new + (size_t)4 * c->N, c->geom.nzy,
                                                                     c->Nx * c->Ny, c->NzY);
        WF_TRY_CUDA(cudaGetLastError());
    }
    drop_graphs(c);
    return WF_OK;
}

wf_status wf_rk_device(wf_ctx *c, const double *y_n, double *y_np1)
{
    if (!c || !y_n || !y_np1) { set_error("wf_rk_device: null argument"); return WF_ERR_ARG; }
    void *yn = c->ybuf[1 - c->cur], *y1 = c->ybuf[c->cur];
    wf_status st = put_state_dev(c, yn, y_n);
    if (st) return st;
    st = (c->prec == WF_FP64) ? enqueue_stages<double>(c, yn, y1) : enqueue_stages<float>(c, yn, y1);
    if (st) return st;
    if ((st = get_state_dev(c, y_np1, y1))) return st;
    drop_graphs(c);
    return WF_OK;
}

wf_status wf_pressure_device(wf_ctx *c, const double *y_np1, const double *y_n, double *pr)
{
    const NvtxRange range("wf_pressure_device");
    if (!c || !y_np1 || !y_n || !pr) { set_error("wf_pressure_device: null argument"); return WF_ERR_ARG; }
    if (const wf_status st0 = settle_p(c)) return st0;
    void *b1 = c->ybuf[1 - c->cur], *bn = c->Xa ? c->Xa : c->ybuf[c->cur];
    wf_status st = put_state_dev(c, b1, y_np1);
    if (st) return st;
    if ((st = put_state_dev(c, bn, y_n))) return st;
    WF_TRY_CUDA(cudaMemcpyAsync(c->p, pr, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    st = (c->prec == WF_FP64) ? enqueue_pressure<double>(c, b1, bn) : enqueue_pressure<float>(c, b1, bn);
    if (st) return st;
    WF_TRY_CUDA(cudaMemcpyAsync(pr, c->p, sizeof(double) * c->N, cudaMemcpyDeviceToDevice, c->stream));
    drop_graphs(c);
    return WF_OK;
}

wf_status wf_rk(wf_ctx *c, const double *y_n, double *y_np1)
{
    if (!c || !y_n || !y_np1) { set_error("wf_rk: null argument"); return WF_ERR_ARG; }
    void *yn = c->ybuf[1 - c->cur], *y1 = c->ybuf[c->cur];
    wf_status st = put_state(c, yn, y_n);
    if (st) return st;
    st = (c->prec == WF_FP64) ? enqueue_stages<double>(c, yn, y1) : enqueue_stages<float>(c, yn, y1);
    if (st) return st;
    if ((st = get_state(c, y_np1, y1))) return st;
    drop_graphs(c);
    return WF_OK;
}

}  // extern "C"
