// poisson.cu -- FP64 pressure Poisson solve on sm_100a: FFT in x and y,
// tridiagonal solve in z per wavenumber, inverse FFT.
//
// Reference: src/cu/pressure.cu:506-549 (solve_pressure) with compute_f
// (:14-101), compute_f_density (:103-327), gammas_and_coefficients (:356-390),
// update_coefficients (:473-504), thomas_algorithm (:418-443), post_fft
// (:392-416).  The reference calls cuFFT Z2Z on real data; here every transform
// is a hand-written FP64 FFT held in shared memory (power-of-two Stockham or
// Bluestein, fft.cuh; prime factors and Rader, fft_pr.cuh), real-to-complex in
// y (two real z-slices packed into one complex line), complex in x on the half
// spectrum.  Five passes, each one kernel:
//   P1 k_p_rhs_ffty        Poisson source f (and the top-plane pressure as one
//                          extra slice) + forward FFT along y   -> G[kk][i][s]
//   P2 k_p_fftx[_pr]<fwd>  forward FFT along x                  -> G[kk][r][s]
//   P3 k_p_tridiag         Thomas along z per (r,s)             -> G[kk][r][s]
//   P4 k_p_fftx[_pr]<inv>  inverse FFT along x
//   P5 k_p_iffty_out       inverse FFT along y, normalisation, p and its
//                          periodic duplicate planes.
// Variable density adds k_vd_base once per step (the source's p-independent
// parts) ahead of the fixed point's solves.
// G is (Nz-1+1) x (Nx-1) x h1 complex doubles, s fastest, h1 = (Ny-1)/2+1.
#include <math.h>

#include <type_traits>

#include "fft.cuh"
#include "fft_pr.cuh"
#include "wf_internal.h"

namespace wf {

namespace {

constexpr double kSigmaSB = 5.670374419e-8;

// Resident blocks per SM the FFT kernels are compiled for.  Two blocks (128
// registers, a few spilled) measured faster than one block with every value of
// a radix-16 butterfly and its twiddles in registers.
#ifndef WF_FFT_MIN_BLOCKS
#define WF_FFT_MIN_BLOCKS 2
#endif
constexpr int kFftMinBlocks = WF_FFT_MIN_BLOCKS;
int g_poisson_sms = 148;   // multiprocessors of the device, read at set-up (grid of the persistent x-FFT)

using fft::cadd;
using fft::cconj;
using fft::cmul;
using fft::csub;
// Largest FFT radix per kernel: each thread of a line holds this many complex
// values per stage.  Radix 8 (no spills at 128 registers) measured faster for
// the x transforms and the inverse y transform; the source kernel, which holds
// more live values while it fills the lines, keeps radix 16.  Radix 8 needs
// M/8 threads per line, so lines of 4096 keep radix 16 (256 threads).
constexpr int kRadixRhs = 16;
constexpr int kRadixFft = 8;
template <int L, int RB> constexpr int kRad = (L >= 12) ? 16 : RB;
template <int L, int RB> __device__ __forceinline__ int padl(int i) { return fft::pad<kRad<L, RB>>(i); }

// z weights of the divergence at plane k: the one-sided weights f0, f1, f2 of
// planes 0, 1, 2 at k = 0 and the centred weight c = 1/(dz_{k-1} + dz_k) above
// (the reference's differences of pressure.cu:37-95 with the division folded
// into a weight, the values of the zc table's ZF0..ZF2 and ZC rows).
// The variable-density source also uses the second-derivative weights s0..s3
// (k = 0: planes 0..3; above: planes k-1, k, k+1) and the spacing dz of plane k
// (pressure.cu:150-262).
struct DivZ {
    double f0, f1, f2, c;
    double s0, s1, s2, s3, dz;
};
__device__ __forceinline__ DivZ div_weights(const double *z, int k)
{
    DivZ w{0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (k == 0) {
        const double A = z[1] - z[0], B = z[2] - z[1], Cc = z[3] - z[2];
        w.f0 = -(2 * A + B) / (A * (A + B));
        w.f1 = (A + B) / (A * B);
        w.f2 = -A / (B * (A + B));
        w.s0 = (6 * A + 4 * B + 2 * Cc) / (A * (A + B) * (A + B + Cc));
        w.s1 = -(4 * A + 4 * B + 2 * Cc) / (A * B * (B + Cc));
        w.s2 = (4 * A + 2 * B + 2 * Cc) / (B * Cc * (A + B));
        w.s3 = -(4 * A + 2 * B) / (Cc * (B + Cc) * (A + B + Cc));
        w.dz = A;
    } else {
        const double a1 = z[k] - z[k - 1], A = z[k + 1] - z[k];
        w.c = 1.0 / (a1 + A);
        w.s0 = 2 / (a1 * (a1 + A));
        w.s1 = -2 / (a1 * A);
        w.s2 = 2 / (A * (a1 + A));
        w.dz = A;
    }
    return w;
}

// Divergence of the intermediate velocity at (i, j, k), k < Nz-1, as the
// reference forms it (pressure.cu:37-95): periodic centred differences in x
// and y, a one-sided second-order difference at k = 0; idx = 1/dx, idy = 1/dy.
template <class R>
__device__ __forceinline__ double velocity_divergence(const PoissonArgs<R> &a, int i, int j, int k, double idx,
                                                      double idy, const DivZ &w)
{
    const Geom &g = a.g;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const int im1 = (i == 0) ? Nx - 2 : i - 1, ip1 = (i + 1 == Nx - 1) ? 0 : i + 1;
    const int jm1 = (j == 0) ? Ny - 2 : j - 1, jp1 = (j + 1 == Ny - 1) ? 0 : j + 1;
    const R *U = a.y1;
    const size_t c = ((size_t)i * Ny + j) * Nz + k;
    const size_t cxm = ((size_t)im1 * Ny + j) * Nz + k, cxp = ((size_t)ip1 * Ny + j) * Nz + k;
    const size_t cym = ((size_t)i * Ny + jm1) * Nz + k, cyp = ((size_t)i * Ny + jp1) * Nz + k;
    const double u = U[c], v = U[(size_t)N + c];
    const double u_im1 = U[cxm], u_ip1 = U[cxp];
    const double v_jm1 = U[(size_t)N + cym], v_jp1 = U[(size_t)N + cyp];
    const R *W = U + 2 * (size_t)N;
    double wz;
    if (k == 0) {
        wz = w.f0 * (double)W[c] + w.f1 * (double)W[c + 1] + w.f2 * (double)W[c + 2];
    } else {
        wz = ((double)W[c + 1] - (double)W[c - 1]) * w.c;
    }
    const double ux = (0.5 * (u_ip1 + u) - 0.5 * (u + u_im1)) * idx;
    const double vy = (0.5 * (v_jp1 + v) - 0.5 * (v + v_jm1)) * idy;
    return ux + vy + wz;
}

// Constants of the variable-density source, once per thread.
struct VdK {
    double TiRi, inv_TiRi, h2x, h2y, idx2, idy2, inv_tc, inv_dt, c12, c4, A, T_act, T_pc, HC_cp, hc, as_ss, cpT;
    int suth;
};
__device__ __forceinline__ VdK vd_constants(const Phys &ph)
{
    VdK q;
    q.TiRi = ph.T_inf * ph.rho_inf;
    q.inv_TiRi = 1.0 / q.TiRi;
    q.h2x = 1.0 / (2 * ph.dx);
    q.h2y = 1.0 / (2 * ph.dy);
    q.idx2 = 1.0 / (ph.dx * ph.dx);
    q.idy2 = 1.0 / (ph.dy * ph.dy);
    q.inv_tc = 1.0 / (q.TiRi * ph.c_p);
    q.inv_dt = 1.0 / ph.dt;
    q.c12 = 12 * kSigmaSB * ph.delta;
    q.c4 = 4 * kSigmaSB * ph.delta;
    q.A = ph.A;
    q.T_act = ph.T_act;
    q.T_pc = ph.T_pc;
    q.HC_cp = ph.H_C / ph.c_p;
    q.hc = ph.h_c;
    q.as_ss = ph.alpha_s * ph.sigma_s;
    q.cpT = ph.c_p * q.TiRi;
    q.suth = ph.sutherland_conductivity;
    return q;
}

// Variable-density Poisson source at (i, j, k), k < Nz-1, from the velocity
// divergence div (pressure.cu:103-327): f = rho_n (div u* - D_T)/dt +
// grad(rho_n).grad(p)/rho_n.  The reference's terms, with its divisions by grid
// constants folded into weights (VdK, DivZ), each difference of two densities
// T_inf rho_inf (1/T_a - 1/T_b) taken over one division, T^2 and T^3 as
// products, and the two terms that vanish exactly skipped: the Arrhenius rate
// below T_pc (the reference multiplies it by a zero step) and the convective
// solid-gas exchange when alpha_s sigma_s = 0.  vd_base is the first term and
// vd_rho_grad the factor grad(rho_n)/rho_n of the second; neither depends on p,
// so the fixed point of a step evaluates them once (k_vd_base) and each solve
// adds only grad(p) (vd_p_grad).
struct VdIdx {
    size_t c, cxm, cxp, cym, cyp;
    int col;
};
__device__ __forceinline__ VdIdx vd_index(const Geom &g, int i, int j, int k)
{
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
    const int im1 = (i == 0) ? Nx - 2 : i - 1, ip1 = (i + 1 == Nx - 1) ? 0 : i + 1;
    const int jm1 = (j == 0) ? Ny - 2 : j - 1, jp1 = (j + 1 == Ny - 1) ? 0 : j + 1;
    VdIdx x;
    x.c = ((size_t)i * Ny + j) * Nz + k;
    x.cxm = ((size_t)im1 * Ny + j) * Nz + k;
    x.cxp = ((size_t)ip1 * Ny + j) * Nz + k;
    x.cym = ((size_t)i * Ny + jm1) * Nz + k;
    x.cyp = ((size_t)i * Ny + jp1) * Nz + k;
    x.col = i * Ny + j;
    return x;
}
template <class R>
__device__ double vd_base(const PoissonArgs<R> &a, int k, const VdIdx &x, double div, const DivZ &w, const VdK &q)
{
    const Geom &g = a.g;
    const size_t N = (size_t)g.N, c = x.c;
    const R *U = a.y1;
    const R *T1 = U + 3 * N;
    const double T = T1[c];
    const double rho = q.TiRi / (double)a.yn[3 * N + c];
    const double T_im1 = T1[x.cxm], T_ip1 = T1[x.cxp], T_jm1 = T1[x.cym], T_jp1 = T1[x.cyp];
    const double Tx = (T_ip1 - T_im1) * q.h2x, Ty = (T_jp1 - T_jm1) * q.h2y;
    const double Txx = (T_ip1 - 2 * T + T_im1) * q.idx2, Tyy = (T_jp1 - 2 * T + T_jm1) * q.idy2;
    double Tz, Tzz;
    if (k == 0) {
        const double t1 = T1[c + 1], t2 = T1[c + 2], t3 = T1[c + 3];
        Tz = w.f0 * T + w.f1 * t1 + w.f2 * t2;
        Tzz = w.s0 * T + w.s1 * t1 + w.s2 * t2 + w.s3 * t3;
    } else {
        const double tp = T1[c + 1], tm = T1[c - 1];
        Tz = (tp - tm) * w.c;
        Tzz = w.s0 * tm + w.s1 * T + w.s2 * tp;
    }
    const double lap_T = Txx + Tyy + Tzz;
    const int nzy = g.nzy[x.col];
    double Yc = 0.0, T_gas = T;
    const double T_solid = T;
    if (k <= nzy) {
        if (k < nzy) Yc = (double)U[4 * N + (size_t)x.col * g.NzY + k];
        T_gas = (Yc > 0.0) ? q.T_pc + (T - q.T_pc) : T;
    }
    const double K_T = (T > q.T_pc) ? q.A * exp(-q.T_act / T) : 0.0;
    double kT = a.ph.kT, dk = 0.0;
    if (q.suth == 1) {
        const double xx = T / 273.15, sx = sqrt(xx), x15 = xx * sx, d = 1.0 / (T + 194);
        kT = 0.0241 * x15 * (273.15 + 194) * d;
        dk = 0.0241 * (1.5 * sx * (273.15 + 194) * d - x15 * (273.15 + 194) * (d * d));
    }
    double qs = q.HC_cp * Yc * K_T;
    if (q.as_ss != 0.0) {
        // (T_gas - T_solid) without abs, as the reference (pressure.cu:313)
        const double h_c = q.hc * w.dz * pow((T_gas - T_solid) / w.dz, 1.0 / 4.0);
        qs -= h_c * q.as_ss * (T_gas - T_solid) / (q.cpT / T_gas);
    }
    const double T2 = T * T;
    const double divT = (dk + q.c12 * T2 * (Tx * Tx + Ty * Ty + Tz * Tz) + (kT + q.c4 * (T2 * T)) * lap_T) * q.inv_tc +
                        qs / T;
    return rho * (div - divT) * q.inv_dt;
}
// grad(rho_n)/rho_n at the cell (p-independent)
template <class R>
__device__ __forceinline__ double3 vd_rho_grad(const PoissonArgs<R> &a, int k, const VdIdx &x, const DivZ &w, const VdK &q)
{
    const size_t N = (size_t)a.g.N, c = x.c;
    const R *Tn = a.yn + 3 * N;
    const double Tnc = Tn[c];
    // T_inf rho_inf (1/Tb - 1/Ta) = T_inf rho_inf (Ta - Tb) / (Ta Tb)
    auto drho = [&](double Ta, double Tb) { return q.TiRi * (Ta - Tb) / (Ta * Tb); };
    const double Tn_xp = Tn[x.cxp], Tn_xm = Tn[x.cxm], Tn_yp = Tn[x.cyp], Tn_ym = Tn[x.cym];
    const double rhox = drho(Tn_xm, Tn_xp) * q.h2x, rhoy = drho(Tn_ym, Tn_yp) * q.h2y;
    double rhoz;
    if (k == 0) {
        const double rho = q.TiRi / Tnc;
        const double r1 = q.TiRi / (double)Tn[c + 1], r2 = q.TiRi / (double)Tn[c + 2];
        rhoz = w.f0 * rho + w.f1 * r1 + w.f2 * r2;
    } else {
        rhoz = drho(Tn[c - 1], Tn[c + 1]) * w.c;
    }
    const double ir = Tnc * q.inv_TiRi;
    return make_double3(rhox * ir, rhoy * ir, rhoz * ir);
}
// grad(p) at the cell
__device__ __forceinline__ double3 vd_p_grad(const double *p, int k, const VdIdx &x, const DivZ &w, const VdK &q)
{
    const size_t c = x.c;
    const double px = (p[x.cxp] - p[x.cxm]) * q.h2x, py = (p[x.cyp] - p[x.cym]) * q.h2y;
    const double pz = (k == 0) ? w.f0 * p[c] + w.f1 * p[c + 1] + w.f2 * p[c + 2] : (p[c + 1] - p[c - 1]) * w.c;
    return make_double3(px, py, pz);
}

// p-independent part of the variable-density source of every cell k < Nz-1
// (once per step, before the fixed point): one block per (i, j) column, one
// thread per plane.
template <class R>
__global__ void __launch_bounds__(128) k_vd_base(const PoissonArgs<R> a)
{
    const Geom &g = a.g;
    const int i = blockIdx.y, j = blockIdx.x;
    const double idx = 1.0 / a.ph.dx, idy = 1.0 / a.ph.dy;
    const VdK q = vd_constants(a.ph);
    const size_t N = (size_t)g.N;
    for (int k = threadIdx.x; k < g.Nz - 1; k += blockDim.x) {
        const double *t = a.vdz + (size_t)k * kVdz;
        const DivZ w{t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], t[8]};
        const VdIdx x = vd_index(g, i, j, k);
        a.s0[x.c] = vd_base(a, k, x, velocity_divergence(a, i, j, k, idx, idy, w), w, q);
        const double3 gr = vd_rho_grad(a, k, x, w, q);
        a.g3[x.c] = (R)gr.x;
        a.g3[N + x.c] = (R)gr.y;
        a.g3[2 * N + x.c] = (R)gr.z;
    }
}

// Length-n DFT of the line (buf, jj): one power-of-two FFT when n = M, else
// Bluestein's chirp-z identity with two length-M FFTs,
//   X_k = c_k * IFFT_M( FFT_M(x c) * FFT_M(b) )_k,  c_j = exp(-i pi j^2 / n),
// the inverse FFT taken as conj(FFT(conj(.))).  pre(idx) supplies x[idx] for
// idx < n and post(idx, X) receives X[idx] for idx < n.  INV selects
// exp(+2 pi i jk/n), unnormalised.  pre may read buf and post may write it.
template <int L, bool INV, int RB, class Pre, class Post>
__device__ __forceinline__ void line_dft(const FftDesc &d, double2 *buf, int jj, Pre pre, Post post)
{
    if (!d.bluestein) {
        fft::run<L, kRad<L, RB>>(
            buf, jj, d.tw,
            [&](int idx) {
                const double2 v = pre(idx);
                return INV ? cconj(v) : v;
            },
            [&](int idx, double2 v) { post(idx, INV ? cconj(v) : v); });
        return;
    }
    const int n = d.n;
    const double2 *__restrict__ chirp = d.chirp;
    const double2 *__restrict__ filt = d.filt;
    fft::run<L, kRad<L, RB>>(
        buf, jj, d.tw,
        [&](int idx) {
            double2 v = make_double2(0.0, 0.0);
            if (idx < n) {
                v = pre(idx);
                if (INV) v = cconj(v);
                v = cmul(v, __ldg(chirp + idx));
            }
            return v;
        },
        [&](int idx, double2 v) { buf[padl<L, RB>(idx)] = cconj(cmul(v, __ldg(filt + idx))); });
    __syncthreads();
    constexpr double inv_m = 1.0 / (double)(1 << L);
    fft::run<L, kRad<L, RB>>(
        buf, jj, d.tw, [&](int idx) { return buf[padl<L, RB>(idx)]; },
        [&](int idx, double2 v) {
            if (idx < n) {
                v = cmul(make_double2(v.x * inv_m, -v.y * inv_m), __ldg(chirp + idx));
                post(idx, INV ? cconj(v) : v);
            }
        });
}

// Line engines.  A kernel stages LB lines of stride LS in shared memory
// (element idx of a line at pos(idx)) and transforms each with run<INV>, which
// every thread of the block calls with its line(tid) and lane(tid).
//   EngS: power-of-two Stockham, or Bluestein around it; threads of a line
//         interleave (line = tid % LB) and synchronise the block.
//   EngPR: prime-factor + Rader (fft_pr.cuh), one warp per line, no block
//         barrier inside.
template <int L, int RB>
struct EngS {
    using SH = fft::Shape<L, kRad<L, RB>>;
    static constexpr int kMinBlocks = kFftMinBlocks;
    static constexpr int LB = SH::LB, LS = SH::LS;
    static constexpr size_t smem_bytes = SH::smem_bytes;
    __device__ __forceinline__ static int line(int tid) { return tid % LB; }
    __device__ __forceinline__ static int lane(int tid) { return tid / LB; }
    __device__ __forceinline__ static int pos(int i) { return padl<L, RB>(i); }
    template <bool INV, class Pre, class Post>
    __device__ __forceinline__ static void run(const FftDesc &d, double2 *buf, int jj, Pre pre, Post post)
    {
        line_dft<L, INV, RB>(d, buf, jj, pre, post);
    }
};
template <class Plan>
struct EngPR {
    // y kernels: three blocks per SM (80 registers, a few hundred bytes spilled)
    // measured faster than two at 128 registers (source 0.465 -> 0.396 ms,
    // inverse 0.268 -> 0.246 ms at 512x512x128); the x kernel keeps two (at
    // three, 88-184 bytes spilled, it measured 2-8% slower in every form)
    static constexpr int kMinBlocks = 3;
    static constexpr int LB = Plan::LB, LS = Plan::LS;
    static constexpr size_t smem_bytes = Plan::smem_bytes;
    __device__ __forceinline__ static int line(int tid) { return tid >> 5; }
    __device__ __forceinline__ static int lane(int tid) { return tid & 31; }
    __device__ __forceinline__ static int pos(int i) { return i; }
    template <bool INV, class Pre, class Post>
    __device__ __forceinline__ static void run(const FftDesc &d, double2 *buf, int jj, Pre pre, Post post)
    {
        Plan::template run<INV>(fft::PrTables{d.prb, d.prmap, d.pr_e1}, buf, jj, pre, post);
    }
    // the same on a line stored in the plan's slot order (d.prslot)
    template <bool INV, class Pre, class Post>
    __device__ __forceinline__ static void run_slotted(const FftDesc &d, double2 *buf, int jj, Pre pre, Post post)
    {
        Plan::template run<INV, true>(fft::PrTables{d.prb, d.prmap, d.pr_e1}, buf, jj, pre, post);
    }
};

// which engine a kernel instantiation got, and the power-of-two engine's log2 length
template <class E> constexpr bool kIsPR = false;
template <class Plan> constexpr bool kIsPR<EngPR<Plan>> = true;
template <class E> constexpr int kLog2 = 0;
template <int L, int RB> constexpr int kLog2<EngS<L, RB>> = L;

// P1: source + top plane, forward FFT in y of packed slice pairs.  Block
// (pair group, i): LB complex lines, line q packs slices 2(pair0+q) (real
// part) and 2(pair0+q)+1 (imaginary part); slice nk is the top-plane pressure.
// The pair group is the fast grid index, so the blocks resident at one time
// read whole z-columns of the same x-plane of the state.
template <class E, class R>
__global__ void __launch_bounds__(256, E::kMinBlocks) k_p_rhs_ffty(const PoissonArgs<R> a)
{
    constexpr int LB = E::LB, LS = E::LS;
    extern __shared__ double2 smem[];
    const Geom &g = a.g;
    const int n0 = g.Nx - 1, n1 = g.Ny - 1, nk = g.Nz - 1, h1 = a.h1;
    const int i = blockIdx.y;
    const int pair0 = blockIdx.x * LB;
    const int nslices = nk + 1;                      // f slices + top-plane pressure
    double *Ad = reinterpret_cast<double *>(smem);
    const int total = n1 * 2 * LB;
    __shared__ DivZ s_w[2 * LB];   // z weights of the block's slices
    if (threadIdx.x < 2 * LB && 2 * pair0 + threadIdx.x < nk) s_w[threadIdx.x] = div_weights(g.z, 2 * pair0 + threadIdx.x);
    __syncthreads();
    if (a.ph.variable_density == 0) {
        // the source is the scaled divergence: SU points per thread at a
        // time, so that their loads are in flight together
        constexpr int SU = 4;
        const double idx = 1.0 / a.ph.dx, idy = 1.0 / a.ph.dy, scale = a.ph.rho_inf / a.ph.dt;
        for (int t0 = threadIdx.x; t0 < total; t0 += 256 * SU) {
            double val[SU];
#pragma unroll
            for (int r = 0; r < SU; r++) {
                const int t = t0 + 256 * r;
                const int jj = t / (2 * LB), q = t - jj * (2 * LB);
                const int kk = 2 * pair0 + q;
                val[r] = 0.0;
                if (t < total && kk < nk) val[r] = scale * velocity_divergence(a, i, jj, kk, idx, idy, s_w[q]);
                else if (t < total && kk == nk) val[r] = a.p[((size_t)i * g.Ny + jj) * g.Nz + (g.Nz - 1)];
            }
#pragma unroll
            for (int r = 0; r < SU; r++) {
                const int t = t0 + 256 * r;
                const int jj = t / (2 * LB), q = t - jj * (2 * LB);
                if (t < total) Ad[2 * ((q >> 1) * LS + E::pos(jj)) + (q & 1)] = val[r];
            }
        }
    } else {
        // variable density.  Within the fixed point (a.s0 set) each point adds
        // grad(p) . (grad(rho)/rho) to the per-step part: four points per thread
        // at a time; otherwise the whole source, two at a time
        const double idx = 1.0 / a.ph.dx, idy = 1.0 / a.ph.dy;
        const VdK vq = vd_constants(a.ph);
        auto vd_points = [&](auto su, auto fixed) {
            constexpr int SU = decltype(su)::value;
            constexpr bool FIXED = decltype(fixed)::value;   // a.s0 and a.g3 are set
            for (int t0 = threadIdx.x; t0 < total; t0 += 256 * SU) {
                double val[SU];
#pragma unroll
                for (int r = 0; r < SU; r++) {
                    const int t = t0 + 256 * r;
                    const int jj = t / (2 * LB), q = t - jj * (2 * LB);
                    const int kk = 2 * pair0 + q;
                    val[r] = 0.0;
                    if (t < total && kk < nk) {
                        const VdIdx x = vd_index(g, i, jj, kk);
                        const double3 pg = vd_p_grad(a.p, kk, x, s_w[q], vq);
                        if constexpr (FIXED) {
                            const size_t N = (size_t)g.N;
                            val[r] = a.s0[x.c] + ((double)a.g3[x.c] * pg.x + (double)a.g3[N + x.c] * pg.y +
                                                  (double)a.g3[2 * N + x.c] * pg.z);
                        } else {
                            const double3 rg = vd_rho_grad(a, kk, x, s_w[q], vq);
                            val[r] = vd_base(a, kk, x, velocity_divergence(a, i, jj, kk, idx, idy, s_w[q]), s_w[q], vq) +
                                     (rg.x * pg.x + rg.y * pg.y + rg.z * pg.z);
                        }
                    } else if (t < total && kk == nk) {
                        val[r] = a.p[((size_t)i * g.Ny + jj) * g.Nz + (g.Nz - 1)];
                    }
                }
#pragma unroll
                for (int r = 0; r < SU; r++) {
                    const int t = t0 + 256 * r;
                    const int jj = t / (2 * LB), q = t - jj * (2 * LB);
                    if (t < total) Ad[2 * ((q >> 1) * LS + E::pos(jj)) + (q & 1)] = val[r];
                }
            }
        };
        if (a.s0) vd_points(std::integral_constant<int, 4>{}, std::true_type{});
        else vd_points(std::integral_constant<int, 2>{}, std::false_type{});
    }
    __syncthreads();
    {
        const int q = E::line(threadIdx.x), jj = E::lane(threadIdx.x);
        double2 *buf = smem + q * LS;
        E::template run<false>(
            a.fy, buf, jj, [&](int idx) { return buf[E::pos(idx)]; }, [&](int idx, double2 v) { buf[E::pos(idx)] = v; });
    }
    __syncthreads();
    // split each packed transform into the two half spectra
    const int kp = min(LB, (nslices + 1) / 2 - pair0);
    for (int t = threadIdx.x; t < kp * h1; t += 256) {
        const int line = t / h1, s = t - line * h1;
        const double2 *Rb = smem + line * LS;
        const double2 Zs = Rb[E::pos(s)];
        const double2 Zc = cconj(Rb[E::pos(s == 0 ? 0 : n1 - s)]);
        const double2 Fa = make_double2(0.5 * (Zs.x + Zc.x), 0.5 * (Zs.y + Zc.y));
        const double2 Fb = make_double2(0.5 * (Zs.y - Zc.y), -0.5 * (Zs.x - Zc.x));
        const int kk0 = 2 * (pair0 + line);
        a.G[((size_t)kk0 * n0 + i) * h1 + s] = Fa;
        if (kk0 + 1 < nslices) a.G[((size_t)(kk0 + 1) * n0 + i) * h1 + s] = Fb;
    }
}

// 16-byte asynchronous copy global -> shared (cp.async, sm_80+ PTX); a
// source size of 0 writes zeros without reading.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// P2/P4: FFT along x.  A work item is LB consecutive s of one slice kk.  The
// blocks are persistent and walk the items blockIdx.x, + gridDim.x, ...: the
// lines of the next item are copied into the second shared buffer while the
// current item is transformed in place, and the last FFT stage writes the
// results straight back to G.
template <int L, bool INV>
__global__ void __launch_bounds__(256, kFftMinBlocks)
    k_p_fftx(double2 *__restrict__ G, const FftDesc fx, int n0, int h1, int nslices)
{
    using SH = fft::Shape<L, kRad<L, kRadixFft>>;
    constexpr int LB = SH::LB, LS = SH::LS;
    extern __shared__ double2 smem[];
    const int ngroups = (h1 + LB - 1) / LB;
    const int nitems = nslices * ngroups;
    const int q = threadIdx.x % LB, jj = threadIdx.x / LB;
    // lines of item `it` -> buffer B (zeros for s >= h1)
    auto fetch = [&](int it, double2 *B) {
        const int kk = it / ngroups, s0 = (it - kk * ngroups) * LB;
        const double2 *src = G + (size_t)kk * n0 * h1 + s0;
        for (int e = threadIdx.x; e < LB * n0; e += 256) {
            const int l = e % LB, idx = e / LB;
            const bool ok = s0 + l < h1;
            cp_async16(B + l * LS + padl<L, kRadixFft>(idx), src + (ok ? (size_t)idx * h1 + l : 0), ok);
        }
    };
    int item = blockIdx.x;
    if (item < nitems) fetch(item, smem);
    cp_async_commit();
    for (int t = 0; item < nitems; item += gridDim.x, t++) {
        double2 *cur = smem + (t & 1) * (LB * LS);
        const int next = item + gridDim.x;
        if (next < nitems) fetch(next, smem + ((t + 1) & 1) * (LB * LS));
        cp_async_commit();
        cp_async_wait<1>();   // this item's lines have landed (own copies) ...
        __syncthreads();      // ... and everyone else's
        const int kk = item / ngroups, s = (item - kk * ngroups) * LB + q;
        const bool act = s < h1;
        double2 *buf = cur + q * LS;
        double2 *g = G + (size_t)kk * n0 * h1 + (act ? s : 0);
        line_dft<L, INV, kRadixFft>(
            fx, buf, jj, [&](int idx) { return buf[padl<L, kRadixFft>(idx)]; },
            [&](int idx, double2 v) {
                if (act) g[(size_t)idx * h1] = v;
            });
        __syncthreads();      // buffer free before the fetch two items ahead
    }
    cp_async_wait<0>();
}

// P2/P4 with the prime-factor + Rader engine: block (s group, kk) copies LB
// lines (consecutive s, one warp each) into shared memory, each warp
// transforms its line with no block barrier, and the block writes the lines
// back.  Both copies move 128 contiguous bytes per 8 threads (LB = 8 lines of
// 16-byte values); LS = 1 (mod 8) keeps the shared-memory side conflict-free
// whatever the position within a line, so the copies also apply the engine's
// input and output permutations (fx.prslot) and the transform itself reads
// and writes its line contiguously (the slotted run).
template <class E, bool INV>
__global__ void __launch_bounds__(256, 2) k_p_fftx_pr(double2 *__restrict__ G, const FftDesc fx, int n0, int h1)
{
    constexpr int LB = E::LB, LS = E::LS;
    static_assert(LB == 8, "copies assume 8 lines of 16-byte values per 128 bytes");
    extern __shared__ double2 smem[];
    const int s0 = blockIdx.x * LB;
    const int nl = min(LB, h1 - s0);
    double2 *g = G + (size_t)blockIdx.y * n0 * h1 + s0;
    const int *__restrict__ slot = fx.prslot;
    for (int e = threadIdx.x; e < LB * n0; e += 256) {
        const int l = e % LB, idx = e / LB;
        if (l < nl) cp_async16(smem + l * LS + __ldg(slot + idx), g + (size_t)idx * h1 + l, true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const int q = E::line(threadIdx.x);
    if (q < nl) {
        double2 *buf = smem + q * LS;
        E::template run_slotted<INV>(
            fx, buf, E::lane(threadIdx.x), [&](int sl) { return buf[sl]; }, [&](int sl, double2 v) { buf[sl] = v; });
    }
    __syncthreads();
    for (int e = threadIdx.x; e < LB * n0; e += 256) {
        const int l = e % LB, idx = e / LB;
        if (l < nl) g[(size_t)idx * h1 + l] = smem[l * LS + __ldg(slot + n0 + idx)];
    }
}

// P3: tridiagonal solve in z per (r, s) (pressure.cu:356-390, 473-504, 418-443).
// zt holds per-k constants: [0..nk) a, [nk..2nk) c, [2nk..3nk) D (b = -(kk + D)),
// followed by b0, c0base, inv_dz1, half_dz0, cl.  Thomas algorithm without
// storing its forward sweep: the forward pass keeps only the modified
// diagonal u and right-hand side y at the end of every kSeg-plane segment
// (local checkpoints); the back substitution walks the segments from the top,
// recomputes each segment's u and y from the previous checkpoint and the
// original right-hand sides (still in G: a segment's solution is written only
// after it has been recomputed), then solves it.  The recomputation repeats the
// forward pass operation for operation, so the result is that of the plain
// two-sweep form, while G is read twice and written once (the two-sweep form
// also writes and re-reads the modified right-hand sides, and spills u).
constexpr int kSeg = 4;
constexpr int kMaxSeg = 128;   // nk <= kSeg * kMaxSeg = 512 planes (Nz <= 513)

__global__ void __launch_bounds__(128, 8) k_p_tridiag(double2 *__restrict__ G, const double *__restrict__ kx2,
                                                   const double *__restrict__ ky2, const double *__restrict__ zt,
                                                   int n0, int h1, int nk)
{
    const int r = blockIdx.x;
    const int s = blockIdx.y * blockDim.x + threadIdx.x;
    if (s >= h1) return;
    const double kk2 = kx2[r] + ky2[s];
    const double *za = zt, *zcc = zt + nk, *zD = zt + 2 * nk;
    const double b0 = zt[3 * nk], c0base = zt[3 * nk + 1], inv_dz1 = zt[3 * nk + 2];
    const double half_dz0 = zt[3 * nk + 3], cl = zt[3 * nk + 4];
    const double c0 = c0base - half_dz0 * kk2 - inv_dz1;   // c[0]
    const size_t stride = (size_t)n0 * h1;
    double2 *g = G + (size_t)r * h1 + s;
    // row 0 uses the source of slice 1; rows 1..nk-2 their own; the last row
    // subtracts the top pressure divided by its coupling coefficient
    const double2 pt = g[stride * nk];
    const double2 d1 = g[stride * 1];
    const double y0x = half_dz0 * d1.x, y0y = half_dz0 * d1.y;
    double cku[kMaxSeg];   // u at the last plane of each segment
    double2 cky[kMaxSeg];  // y there
    const int nseg = (nk + kSeg - 1) / kSeg;
    // one step of the forward recurrence at plane k >= 1 (u, y: values at k-1 on entry)
    auto fwd = [&](int k, double2 dk, double &u, double2 &y) {
        const double l = za[k - 1] / u;
        const double cprev = (k == 1) ? c0 : zcc[k - 1];
        const double bk = -(kk2 + zD[k]);
        u = bk - l * cprev;
        if (k == nk - 1) dk = make_double2(dk.x - pt.x / cl, dk.y - pt.y / cl);
        y = make_double2(dk.x - l * y.x, dk.y - l * y.y);
    };
    // forward pass: checkpoints only
    {
        double u = b0;
        double2 y = make_double2(y0x, y0y);
        for (int m = 0; m < nseg; m++) {
            const int kb = m * kSeg;
            double2 dv[kSeg];
#pragma unroll
            for (int q = 0; q < kSeg; q++)
                if (kb + q >= 1 && kb + q < nk) dv[q] = g[stride * (kb + q)];
#pragma unroll
            for (int q = 0; q < kSeg; q++)
                if (kb + q >= 1 && kb + q < nk) fwd(kb + q, dv[q], u, y);
            cku[m] = u;
            cky[m] = y;
        }
    }
    // back substitution, one recomputed segment at a time from the top
    double2 x = make_double2(0.0, 0.0);
    for (int m = nseg - 1; m >= 0; m--) {
        const int kb = m * kSeg;
        double u = (m == 0) ? b0 : cku[m - 1];
        double2 y = (m == 0) ? make_double2(y0x, y0y) : cky[m - 1];
        double uu[kSeg];
        double2 yy[kSeg], dv[kSeg];
#pragma unroll
        for (int q = 0; q < kSeg; q++)
            if (kb + q >= 1 && kb + q < nk) dv[q] = g[stride * (kb + q)];
#pragma unroll
        for (int q = 0; q < kSeg; q++) {
            if (kb + q >= nk) continue;
            if (kb + q >= 1) fwd(kb + q, dv[q], u, y);
            uu[q] = u;
            yy[q] = y;
        }
#pragma unroll
        for (int q = kSeg - 1; q >= 0; q--) {
            const int k = kb + q;
            if (k >= nk) continue;
            if (k == nk - 1) {
                x = make_double2(yy[q].x / uu[q], yy[q].y / uu[q]);
            } else {
                const double ck = (k == 0) ? c0 : zcc[k];
                x = make_double2((yy[q].x - ck * x.x) / uu[q], (yy[q].y - ck * x.y) / uu[q]);
            }
            g[stride * k] = x;
        }
    }
}

// P5: inverse FFT in y of packed slice pairs, normalisation, write p and the
// periodic duplicate planes (pressure.cu:392-416, deterministic here).
template <class E, class R>
__global__ void __launch_bounds__(256, E::kMinBlocks) k_p_iffty_out(const PoissonArgs<R> a)
{
    constexpr int LB = E::LB, LS = E::LS;
    extern __shared__ double2 smem[];
    const Geom &g = a.g;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
    const int n0 = Nx - 1, n1 = Ny - 1, nk = Nz - 1, h1 = a.h1;
    const int i = blockIdx.x;
    const int pair0 = blockIdx.y * LB;
    const int np = (nk + 1) / 2;
    const int kp = min(LB, np - pair0);
    const bool even = (n1 % 2) == 0;
    // each stored half-spectrum value ss fills position ss and its mirror
    // n1 - ss (conjugates) of the packed line; SU values per thread at a time
    // so that their loads are in flight together
    constexpr int SU = 4;
    const int total = LB * h1;
    for (int t0 = threadIdx.x; t0 < total; t0 += 256 * SU) {
        double2 Fa[SU], Fb[SU];
#pragma unroll
        for (int r = 0; r < SU; r++) {
            const int t = t0 + 256 * r;
            const int line = t / h1, ss = t - line * h1;
            const int kk0 = 2 * (pair0 + line), kk1 = kk0 + 1;
            Fa[r] = Fb[r] = make_double2(0.0, 0.0);
            if (t < total && line < kp) {
                Fa[r] = a.G[((size_t)kk0 * n0 + i) * h1 + ss];
                if (kk1 < nk) Fb[r] = a.G[((size_t)kk1 * n0 + i) * h1 + ss];
            }
        }
#pragma unroll
        for (int r = 0; r < SU; r++) {
            const int t = t0 + 256 * r;
            const int line = t / h1, ss = t - line * h1;
            if (t < total) {
                double2 fa = Fa[r], fb = Fb[r];
                if (ss == 0 || (even && ss == n1 / 2)) {
                    fa.y = 0.0;
                    fb.y = 0.0;
                }
                smem[line * LS + E::pos(ss)] = make_double2(fa.x - fb.y, fa.y + fb.x);
                if (ss >= 1 && ss <= n1 - h1) {
                    fa.y = -fa.y;
                    fb.y = -fb.y;
                    smem[line * LS + E::pos(n1 - ss)] = make_double2(fa.x - fb.y, fa.y + fb.x);
                }
            }
        }
    }
    __syncthreads();
    {
        const int q = E::line(threadIdx.x), jj = E::lane(threadIdx.x);
        double2 *buf = smem + q * LS;
        E::template run<true>(
            a.fy, buf, jj, [&](int idx) { return buf[E::pos(idx)]; }, [&](int idx, double2 v) { buf[E::pos(idx)] = v; });
    }
    __syncthreads();
    const double norm = (double)n0 * (double)n1;
    const int ns = 2 * kp;
    double *p = a.p;
    for (int t = threadIdx.x; t < n1 * ns; t += 256) {
        const int jj = t / ns, q = t - jj * ns;
        const int kk = 2 * pair0 + q;
        if (kk >= nk) continue;
        const double2 zv = smem[(q >> 1) * LS + E::pos(jj)];
        const double val = ((q & 1) ? zv.y : zv.x) / norm;
        p[((size_t)i * Ny + jj) * Nz + kk] = val;
        if (jj == 0) p[((size_t)i * Ny + (Ny - 1)) * Nz + kk] = val;
        if (i == 0) {
            p[((size_t)(Nx - 1) * Ny + jj) * Nz + kk] = val;
            if (jj == 0) p[((size_t)(Nx - 1) * Ny + (Ny - 1)) * Nz + kk] = val;
        }
    }
    // duplicate planes of the (fixed) top plane
    if (blockIdx.y == gridDim.y - 1) {
        const int k = Nz - 1;
        if (threadIdx.x == 0) p[((size_t)i * Ny + (Ny - 1)) * Nz + k] = p[((size_t)i * Ny + 0) * Nz + k];
        if (i == 0)
            for (int jj = threadIdx.x; jj < Ny; jj += blockDim.x)
                p[((size_t)(Nx - 1) * Ny + jj) * Nz + k] = p[((size_t)0 * Ny + (jj % (Ny - 1))) * Nz + k];
    }
}

// ---- launch: one kernel instantiation per line engine ----------------------
constexpr int kMinL = 2, kMaxL = 12;

// Prime-factor + Rader plans compiled in: n = N1 * P, P - 1 = F1 * F2 * F3.
// The x and y lengths of the workloads: 511 (512-point grids), 255 (256), 191
// (192), 159 (160), 127 (128) and 95 (96).
template <class... Pl> struct PlanList {};
using PrPlans = PlanList<fft::PrPlan<7, 73, 8, 9>, fft::PrPlan<15, 17, 16, 1>, fft::PrPlan<1, 191, 2, 5, 19>,
                         fft::PrPlan<3, 53, 4, 13>, fft::PrPlan<1, 127, 2, 7, 9>, fft::PrPlan<5, 19, 2, 9>>;

template <class Op, class... Pl, class... A>
cudaError_t by_plan(PlanList<Pl...>, int n, A &...args)
{
    cudaError_t e = cudaErrorInvalidValue;
    (void)((n == Pl::n ? (e = Op::template go<EngPR<Pl>>(args...), true) : false) || ...);
    return e;
}

// Engine of a descriptor: a Rader plan when the descriptor carries one (its
// length is then one of the plans above), else the power-of-two engine of
// inner length 2^L with largest radix RB.
template <class Op, int RB, class... A>
cudaError_t by_engine(const FftDesc &d, A &...args)
{
    if (d.pr) return by_plan<Op>(PrPlans{}, d.n, args...);
    switch (d.L) {
    case 2: return Op::template go<EngS<2, RB>>(args...);
    case 3: return Op::template go<EngS<3, RB>>(args...);
    case 4: return Op::template go<EngS<4, RB>>(args...);
    case 5: return Op::template go<EngS<5, RB>>(args...);
    case 6: return Op::template go<EngS<6, RB>>(args...);
    case 7: return Op::template go<EngS<7, RB>>(args...);
    case 8: return Op::template go<EngS<8, RB>>(args...);
    case 9: return Op::template go<EngS<9, RB>>(args...);
    case 10: return Op::template go<EngS<10, RB>>(args...);
    case 11: return Op::template go<EngS<11, RB>>(args...);
    case 12: return Op::template go<EngS<12, RB>>(args...);
    default: return cudaErrorInvalidValue;
    }
}

template <class R>
struct LaunchP1 {
    template <class E> static cudaError_t go(const PoissonArgs<R> &a, cudaStream_t &s)
    {
        const int np = (a.g.Nz - 1 + 2) / 2;
        k_p_rhs_ffty<E, R><<<dim3((np + E::LB - 1) / E::LB, a.g.Nx - 1), 256, E::smem_bytes, s>>>(a);
        return cudaSuccess;
    }
};
template <class R>
struct LaunchP5 {
    template <class E> static cudaError_t go(const PoissonArgs<R> &a, cudaStream_t &s)
    {
        const int np = (a.g.Nz - 1 + 1) / 2;
        k_p_iffty_out<E, R><<<dim3(a.g.Nx - 1, (np + E::LB - 1) / E::LB), 256, E::smem_bytes, s>>>(a);
        return cudaSuccess;
    }
};
template <bool INV>
struct LaunchFx {
    template <class E> static cudaError_t go(double2 *const &G, const FftDesc &fx, const int &nslices, const int &n0,
                                           const int &h1, cudaStream_t &s)
    {
        if constexpr (kIsPR<E>) {
            if (!fx.prslot) return cudaErrorInvalidValue;   // every compiled plan has its slot table
            k_p_fftx_pr<E, INV><<<dim3((h1 + E::LB - 1) / E::LB, nslices), 256, E::smem_bytes, s>>>(G, fx, n0, h1);
        } else {
            constexpr int L = kLog2<E>;
            const int nitems = nslices * ((h1 + E::LB - 1) / E::LB);
            const int blocks = min(nitems, kFftMinBlocks * g_poisson_sms);
            k_p_fftx<L, INV><<<blocks, 256, 2 * E::smem_bytes, s>>>(G, fx, n0, h1, nslices);
        }
        return cudaSuccess;
    }
};

template <class R, class E, class EF>
cudaError_t set_engine_attributes()
{
    const int b1 = (int)E::smem_bytes, b = (int)EF::smem_bytes;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_p_rhs_ffty<E, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, b1))) return e;
    if ((e = cudaFuncSetAttribute(k_p_iffty_out<EF, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
    return cudaSuccess;
}
template <class R, int L>
cudaError_t set_attributes_for()
{
    using E = EngS<L, kRadixRhs>;
    using EF = EngS<L, kRadixFft>;
    const int bx = 2 * (int)EF::smem_bytes;   // the persistent x kernel holds two item buffers
    cudaError_t e;
    if ((e = set_engine_attributes<R, E, EF>())) return e;
    if ((e = cudaFuncSetAttribute(k_p_fftx<L, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bx))) return e;
    if ((e = cudaFuncSetAttribute(k_p_fftx<L, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bx))) return e;
    if constexpr (L < kMaxL) return set_attributes_for<R, L + 1>();
    return cudaSuccess;
}
template <class R, class Plan>
cudaError_t set_pr_attributes()
{
    using E = EngPR<Plan>;
    const int b = (int)E::smem_bytes;
    cudaError_t e;
    if ((e = set_engine_attributes<R, E, E>())) return e;
    if ((e = cudaFuncSetAttribute(k_p_fftx_pr<E, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
    if ((e = cudaFuncSetAttribute(k_p_fftx_pr<E, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
    return cudaSuccess;
}
template <class R, class... Pl>
cudaError_t set_pr_attributes_all(PlanList<Pl...>)
{
    cudaError_t e = cudaSuccess;
    (void)(((e = set_pr_attributes<R, Pl>()) != cudaSuccess) || ...);
    return e;
}
template <class... Pl>
bool pr_plan_of(PlanList<Pl...>, int n, int f[5])
{
    return ((n == Pl::n ? (f[0] = Pl::N1, f[1] = Pl::P, f[2] = Pl::F1, f[3] = Pl::F2, f[4] = Pl::F3, true) : false) ||
            ...);
}

}  // namespace

bool poisson_pr_plan(int n, int f[5]) { return pr_plan_of(PrPlans{}, n, f); }

template <class... Pl> bool pr_layout_of(PlanList<Pl...>, int n, int *ss, int *ub)
{
    return ((n == Pl::n ? (*ss = Pl::SS, *ub = Pl::UB, true) : false) || ...);
}
bool poisson_pr_layout(int n, int *ss, int *ub) { return pr_layout_of(PrPlans{}, n, ss, ub); }

template <class R> cudaError_t poisson_set_attributes()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&g_poisson_sms, cudaDevAttrMultiProcessorCount, dev);
    if (!e) e = set_attributes_for<R, kMinL>();
    if (!e) e = set_pr_attributes_all<R>(PrPlans{});
    return e;
}
template cudaError_t poisson_set_attributes<double>();
template cudaError_t poisson_set_attributes<float>();

template <class R>
cudaError_t launch_poisson_impl(const PoissonArgs<R> &a, const double *zt, cudaStream_t s, cudaEvent_t *ev)
{
    int n0 = a.g.Nx - 1, nk = a.g.Nz - 1, h1 = a.h1;
    cudaError_t e;
    if ((e = by_engine<LaunchP1<R>, kRadixRhs>(a.fy, a, s))) return e;
    if (ev) cudaEventRecord(ev[0], s);
    int ns = nk + 1;
    double2 *G = a.G;
    if ((e = by_engine<LaunchFx<false>, kRadixFft>(a.fx, G, a.fx, ns, n0, h1, s))) return e;
    if (ev) cudaEventRecord(ev[1], s);
    if (nk > kSeg * kMaxSeg) return cudaErrorInvalidValue;
    k_p_tridiag<<<dim3(n0, (h1 + 127) / 128), 128, 0, s>>>(a.G, a.kx2, a.ky2, zt, n0, h1, nk);
    if (ev) cudaEventRecord(ev[2], s);
    ns = nk;
    if ((e = by_engine<LaunchFx<true>, kRadixFft>(a.fx, G, a.fx, ns, n0, h1, s))) return e;
    if (ev) cudaEventRecord(ev[3], s);
    if ((e = by_engine<LaunchP5<R>, kRadixFft>(a.fy, a, s))) return e;
    if (ev) cudaEventRecord(ev[4], s);
    return cudaGetLastError();
}
template cudaError_t launch_poisson_impl<double>(const PoissonArgs<double> &, const double *, cudaStream_t, cudaEvent_t *);
template cudaError_t launch_poisson_impl<float>(const PoissonArgs<float> &, const double *, cudaStream_t, cudaEvent_t *);

template <class R> cudaError_t launch_vd_base(const PoissonArgs<R> &a, cudaStream_t s)
{
    if (!a.s0 || !a.g3 || !a.vdz || a.g.Nx > 65535) return cudaErrorInvalidValue;
    k_vd_base<R><<<dim3(a.g.Ny, a.g.Nx), 128, 0, s>>>(a);
    return cudaGetLastError();
}
template cudaError_t launch_vd_base<double>(const PoissonArgs<double> &, cudaStream_t);
template cudaError_t launch_vd_base<float>(const PoissonArgs<float> &, cudaStream_t);

void vd_z_table(const double *z, int Nz, double *out)
{
    for (int k = 0; k < Nz; k++) {
        double *w = out + (size_t)k * kVdz;
        for (int e = 0; e < kVdz; e++) w[e] = 0.0;
        if (k == 0 && Nz >= 4) {
            const double A = z[1] - z[0], B = z[2] - z[1], Cc = z[3] - z[2];
            w[0] = -(2 * A + B) / (A * (A + B));
            w[1] = (A + B) / (A * B);
            w[2] = -A / (B * (A + B));
            w[4] = (6 * A + 4 * B + 2 * Cc) / (A * (A + B) * (A + B + Cc));
            w[5] = -(4 * A + 4 * B + 2 * Cc) / (A * B * (B + Cc));
            w[6] = (4 * A + 2 * B + 2 * Cc) / (B * Cc * (A + B));
            w[7] = -(4 * A + 2 * B) / (Cc * (B + Cc) * (A + B + Cc));
            w[8] = A;
        } else if (k > 0 && k + 1 < Nz) {
            const double a1 = z[k] - z[k - 1], A = z[k + 1] - z[k];
            w[3] = 1.0 / (a1 + A);
            w[4] = 2 / (a1 * (a1 + A));
            w[5] = -2 / (a1 * A);
            w[6] = 2 / (A * (a1 + A));
            w[8] = A;
        }
    }
}

// ---- variable-density fixed point, driven on the device ------------------
// The loop (pressure.cu:551-606) runs as a CUDA graph WHILE node: its body is
// one Poisson solve, k_maxdiff_copy and k_piter_next, which sets the node's
// condition, so no iteration waits for the host.
namespace {
__global__ void k_piter_begin(PIterRec *r)
{
    r->red = 0ull;
    r->h = 0.0;
    r->m = 0;
    r->done = 0;
}

__global__ void __launch_bounds__(256) k_maxdiff_copy(const double *__restrict__ a, double *__restrict__ b, int n,
                                                       unsigned long long *out)
{
    double m = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const double av = a[t];
        const double d = fabs(av - b[t]);
        m = (d > m || d != d) ? d : m;
        b[t] = av;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, m, o);
        m = (v > m || v != v) ? v : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_piter_next(PIterRec *r, double tol, int use_tol, int maxit, cudaGraphConditionalHandle cond)
{
    const double h = __longlong_as_double((long long)r->red);
    r->red = 0ull;
    r->h = h;
    const int m = r->m + 1;
    r->m = m;
    const int done = use_tol && h <= tol;   // NaN never meets the tolerance
    r->done = done;
    cudaGraphSetConditional(cond, (!done && m < maxit) ? 1u : 0u);
}
}  // namespace

cudaError_t launch_piter_begin(PIterRec *rec, cudaStream_t s)
{
    k_piter_begin<<<1, 1, 0, s>>>(rec);
    return cudaGetLastError();
}

cudaError_t launch_maxdiff_copy(const double *p, double *p_prev, int n, PIterRec *rec, cudaStream_t s)
{
    k_maxdiff_copy<<<4 * g_poisson_sms, 256, 0, s>>>(p, p_prev, n, &rec->red);
    return cudaGetLastError();
}

cudaError_t launch_piter_next(PIterRec *rec, double tol, int use_tol, int maxit, cudaGraphConditionalHandle cond,
                              cudaStream_t s)
{
    k_piter_next<<<1, 1, 0, s>>>(rec, tol, use_tol, maxit, cond);
    return cudaGetLastError();
}

}  // namespace wf
