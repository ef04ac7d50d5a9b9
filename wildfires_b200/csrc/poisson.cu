// poisson.cu -- FP64 pressure Poisson solve on sm_100a: FFT in x and y,
// tridiagonal solve in z per wavenumber, inverse FFT.
//
// Reference: src/cu/pressure.cu:506-549 (solve_pressure) with compute_f
// (:14-101), compute_f_density (:103-327), gammas_and_coefficients (:356-390),
// update_coefficients (:473-504), thomas_algorithm (:418-443), post_fft
// (:392-416).  The reference calls cuFFT Z2Z on real data; here every transform
// is a hand-written FP64 FFT held in shared memory, real-to-complex in y (two
// real z-slices packed into one complex line), complex in x on the half
// spectrum.  Five passes, each one kernel:
//   P1 k_p_rhs_ffty   Poisson source f (and the top-plane pressure as one extra
//                     slice) + forward FFT along y        -> G[kk][i][s]
//   P2 k_p_fftx<fwd>  forward FFT along x                 -> G[kk][r][s]
//   P3 k_p_tridiag    Thomas along z per (r,s)            -> G[kk][r][s]
//   P4 k_p_fftx<inv>  inverse FFT along x
//   P5 k_p_iffty_out  inverse FFT along y, normalisation, p and its periodic
//                     duplicate planes.
// G is (Nz-1+1) x (Nx-1) x h1 complex doubles, s fastest, h1 = (Ny-1)/2+1.
#include <math.h>

#include "wf_internal.h"

namespace wf {

namespace {

constexpr double kSigmaSB = 5.670374419e-8;

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// Forward radix-4 DFT of (a0, a1, a2, a3) in natural output order.
__device__ __forceinline__ void bfly4(double2 &a0, double2 &a1, double2 &a2, double2 &a3)
{
    const double2 s0 = cadd(a0, a2), d0 = csub(a0, a2);
    const double2 s1 = cadd(a1, a3), d1 = csub(a1, a3);
    const double2 md1 = make_double2(d1.y, -d1.x);   // -i * d1
    a0 = cadd(s0, s1);
    a2 = csub(s0, s1);
    a1 = cadd(d0, md1);
    a3 = csub(d0, md1);
}

// Forward Stockham FFT of length M = 2^L (radix-4 stages, one radix-2 stage
// when L is odd) on nl lines held in place in shared memory (data[l*M + j]).
// Blocks have 256 threads; lines go in groups of 1024/M so that every thread
// owns B4 radix-4 (or B2 radix-2) butterflies per stage, kept in registers
// between the loads and the stores of the stage.  All index arithmetic is
// shifts and masks.  tw[j] = exp(-2 pi i j / M).
template <int L>
__device__ void fft_pow2(double2 *data, int nl, const double2 *__restrict__ tw)
{
    constexpr int M = 1 << L;
    constexpr int Q = M / 4;
    constexpr int GL = (M >= 1024) ? 1 : 1024 / M;
    constexpr int B4 = (M > 1024) ? M / 1024 : 1;
    constexpr int B2 = (GL * M / 2 + 255) / 256;
    for (int l0 = 0; l0 < nl; l0 += GL) {
        const int ng = min(GL, nl - l0);
        double2 *base = data + (size_t)l0 * M;
#pragma unroll
        for (int st = 0; st < L / 2; st++) {
            const int lns = 2 * st;
            double2 v[B4][4];
            int jb[B4];
            double2 *xl[B4];
#pragma unroll
            for (int b = 0; b < B4; b++) {
                const int t = threadIdx.x + b * 256;
                jb[b] = -1;
                if (t < ng * Q) {
                    jb[b] = t & (Q - 1);
                    xl[b] = base + (size_t)(t / Q) * M;
#pragma unroll
                    for (int r = 0; r < 4; r++) v[b][r] = xl[b][jb[b] + r * Q];
                }
            }
            __syncthreads();
#pragma unroll
            for (int b = 0; b < B4; b++) {
                if (jb[b] < 0) continue;
                const int j = jb[b], k = j & ((1 << lns) - 1);
                if (st > 0) {
                    const int tsh = L - 2 - lns;
                    v[b][1] = cmul(v[b][1], __ldg(tw + ((1 * k) << tsh)));
                    v[b][2] = cmul(v[b][2], __ldg(tw + ((2 * k) << tsh)));
                    v[b][3] = cmul(v[b][3], __ldg(tw + ((3 * k) << tsh)));
                }
                bfly4(v[b][0], v[b][1], v[b][2], v[b][3]);
                const int o = ((j >> lns) << (lns + 2)) + k;
#pragma unroll
                for (int r = 0; r < 4; r++) xl[b][o + (r << lns)] = v[b][r];
            }
            __syncthreads();
        }
        if (L & 1) {
            // final radix-2 stage: Ns = M/2, twiddle exp(-2 pi i j / M)
            double2 v[B2][2];
            int jb[B2];
            double2 *xl[B2];
#pragma unroll
            for (int b = 0; b < B2; b++) {
                const int t = threadIdx.x + b * 256;
                jb[b] = -1;
                if (t < ng * (M / 2)) {
                    jb[b] = t & (M / 2 - 1);
                    xl[b] = base + (size_t)(t / (M / 2)) * M;
                    v[b][0] = xl[b][jb[b]];
                    v[b][1] = xl[b][jb[b] + M / 2];
                }
            }
            __syncthreads();
#pragma unroll
            for (int b = 0; b < B2; b++) {
                if (jb[b] < 0) continue;
                const double2 w = cmul(v[b][1], __ldg(tw + jb[b]));
                xl[b][jb[b]] = cadd(v[b][0], w);
                xl[b][jb[b] + M / 2] = csub(v[b][0], w);
            }
            __syncthreads();
        }
    }
}

// Length-n DFT of nl lines held in place in A ([nl][m], first n entries valid;
// m = 2^L).  inverse selects exp(+2 pi i ...), unnormalised.  Lengths that are
// not powers of two go through Bluestein's chirp-z identity
//   X_k = c_k * IFFT_m( FFT_m(x c) * FFT_m(b) )_k,  c_j = exp(-i pi j^2 / n).
template <int L>
__device__ void fft_line_set(const FftDesc &d, double2 *A, int nl, bool inverse)
{
    constexpr int M = 1 << L;
    const int n = d.n;
    if (!d.bluestein) {
        if (inverse) {
            for (int t = threadIdx.x; t < nl * M; t += blockDim.x) A[t].y = -A[t].y;
            __syncthreads();
        }
        fft_pow2<L>(A, nl, d.tw);
        if (inverse) {
            for (int t = threadIdx.x; t < nl * M; t += blockDim.x) A[t].y = -A[t].y;
            __syncthreads();
        }
        return;
    }
    for (int t = threadIdx.x; t < nl * M; t += blockDim.x) {
        const int j = t & (M - 1);
        double2 v = A[t];
        if (inverse) v.y = -v.y;
        A[t] = (j < n) ? cmul(v, __ldg(d.chirp + j)) : make_double2(0.0, 0.0);
    }
    __syncthreads();
    fft_pow2<L>(A, nl, d.tw);
    for (int t = threadIdx.x; t < nl * M; t += blockDim.x)
        A[t] = cconj(cmul(A[t], __ldg(d.filt + (t & (M - 1)))));   // conj: IFFT via FFT
    __syncthreads();
    fft_pow2<L>(A, nl, d.tw);
    const double inv_m = 1.0 / (double)M;
    for (int t = threadIdx.x; t < nl * M; t += blockDim.x) {
        const int j = t & (M - 1);
        if (j < n) {
            double2 v = cconj(A[t]);
            v.x *= inv_m;
            v.y *= inv_m;
            v = cmul(v, __ldg(d.chirp + j));
            if (inverse) v.y = -v.y;
            A[t] = v;
        }
    }
    __syncthreads();
}

__device__ void fft_lines(const FftDesc &d, double2 *A, int nl, bool inverse)
{
    switch (d.L) {
    case 2: fft_line_set<2>(d, A, nl, inverse); break;
    case 3: fft_line_set<3>(d, A, nl, inverse); break;
    case 4: fft_line_set<4>(d, A, nl, inverse); break;
    case 5: fft_line_set<5>(d, A, nl, inverse); break;
    case 6: fft_line_set<6>(d, A, nl, inverse); break;
    case 7: fft_line_set<7>(d, A, nl, inverse); break;
    case 8: fft_line_set<8>(d, A, nl, inverse); break;
    case 9: fft_line_set<9>(d, A, nl, inverse); break;
    case 10: fft_line_set<10>(d, A, nl, inverse); break;
    case 11: fft_line_set<11>(d, A, nl, inverse); break;
    case 12: fft_line_set<12>(d, A, nl, inverse); break;
    default: break;
    }
}

// Poisson source at (i, j, k), k < Nz-1 (pressure.cu:37-95 and 150-321).
template <class R>
__device__ double poisson_source(const PoissonArgs<R> &a, int i, int j, int k)
{
    const Geom &g = a.g;
    const Phys &ph = a.ph;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const int im1 = (i == 0) ? Nx - 2 : i - 1, ip1 = (i + 1 == Nx - 1) ? 0 : i + 1;
    const int jm1 = (j == 0) ? Ny - 2 : j - 1, jp1 = (j + 1 == Ny - 1) ? 0 : j + 1;
    const R *U = a.y1;
    const size_t c = ((size_t)i * Ny + j) * Nz + k;
    const size_t cxm = ((size_t)im1 * Ny + j) * Nz + k, cxp = ((size_t)ip1 * Ny + j) * Nz + k;
    const size_t cym = ((size_t)i * Ny + jm1) * Nz + k, cyp = ((size_t)i * Ny + jp1) * Nz + k;
    const double *z = g.z;
    const double u = U[c], v = U[(size_t)N + c];
    const double u_im1 = U[cxm], u_ip1 = U[cxp];
    const double v_jm1 = U[(size_t)N + cym], v_jp1 = U[(size_t)N + cyp];
    const R *W = U + 2 * (size_t)N;
    double wz;
    double dzk_f = 0, dzkp1_f = 0, dzkp2_f = 0, dzkm1_c = 0, dzk_c = 0;
    if (k == 0) {
        dzk_f = z[1] - z[0];
        dzkp1_f = z[2] - z[1];
        dzkp2_f = z[3] - z[2];
        const double A = dzk_f, B = dzkp1_f;
        wz = -(2 * A + B) * (double)W[c] / (A * (A + B)) + (A + B) * (double)W[c + 1] / (A * B) -
             A * (double)W[c + 2] / (B * (A + B));
    } else {
        dzkm1_c = z[k] - z[k - 1];
        dzk_c = z[k + 1] - z[k];
        wz = ((double)W[c + 1] - (double)W[c - 1]) / (dzk_c + dzkm1_c);
    }
    const double ux = (0.5 * (u_ip1 + u) - 0.5 * (u + u_im1)) / ph.dx;
    const double vy = (0.5 * (v_jp1 + v) - 0.5 * (v + v_jm1)) / ph.dy;
    if (ph.variable_density == 0) return ph.rho_inf * (ux + vy + wz) / ph.dt;
    // variable density: f = rho_n (div u* - D_T)/dt + grad(rho).grad(p)/rho
    const R *T1 = U + 3 * (size_t)N;
    const R *Tn = a.yn + 3 * (size_t)N;
    const double *p = a.p;
    const double Ti = ph.T_inf, ri = ph.rho_inf;
    const double T = T1[c];
    const double rho = Ti * ri / (double)Tn[c];
    const double T_im1 = T1[cxm], T_ip1 = T1[cxp], T_jm1 = T1[cym], T_jp1 = T1[cyp];
    const double Tx = (T_ip1 - T_im1) / (2 * ph.dx), Ty = (T_jp1 - T_jm1) / (2 * ph.dy);
    const double Txx = (T_ip1 - 2 * T + T_im1) / (ph.dx * ph.dx), Tyy = (T_jp1 - 2 * T + T_jm1) / (ph.dy * ph.dy);
    const double rhox = (Ti * ri / (double)Tn[cxp] - Ti * ri / (double)Tn[cxm]) / (2 * ph.dx);
    const double rhoy = (Ti * ri / (double)Tn[cyp] - Ti * ri / (double)Tn[cym]) / (2 * ph.dy);
    const double px = (p[cxp] - p[cxm]) / (2 * ph.dx), py = (p[cyp] - p[cym]) / (2 * ph.dy);
    double rhoz, pz, Tz, Tzz, dz_k;
    if (k == 0) {
        const double A = dzk_f, B = dzkp1_f, Cc = dzkp2_f;
        dz_k = A;
        const double r1 = Ti * ri / (double)Tn[c + 1], r2 = Ti * ri / (double)Tn[c + 2];
        rhoz = -(2 * A + B) * rho / (A * (A + B)) + (A + B) * r1 / (A * B) - A * r2 / (B * (A + B));
        pz = -(2 * A + B) * p[c] / (A * (A + B)) + (A + B) * p[c + 1] / (A * B) - A * p[c + 2] / (B * (A + B));
        const double t1 = T1[c + 1], t2 = T1[c + 2], t3 = T1[c + 3];
        Tz = -(2 * A + B) * T / (A * (A + B)) + (A + B) * t1 / (A * B) - A * t2 / (B * (A + B));
        Tzz = (6 * A + 4 * B + 2 * Cc) * T / (A * (A + B) * (A + B + Cc)) -
              (4 * A + 4 * B + 2 * Cc) * t1 / (A * B * (B + Cc)) + (4 * A + 2 * B + 2 * Cc) * t2 / (B * Cc * (A + B)) -
              (4 * A + 2 * B) * t3 / (Cc * (B + Cc) * (A + B + Cc));
    } else {
        const double a1 = dzkm1_c, A = dzk_c;
        dz_k = A;
        rhoz = (Ti * ri / (double)Tn[c + 1] - Ti * ri / (double)Tn[c - 1]) / (A + a1);
        pz = (p[c + 1] - p[c - 1]) / (A + a1);
        const double tp = T1[c + 1], tm = T1[c - 1];
        Tz = (tp - tm) / (A + a1);
        Tzz = 2 * tm / (a1 * (a1 + A)) - 2 * T / (a1 * A) + 2 * tp / (A * (a1 + A));
    }
    const double lap_T = Txx + Tyy + Tzz;
    const int col = i * Ny + j;
    const int nzy = g.nzy[col];
    double Yc = 0.0, T_gas = T;
    const double T_solid = T;
    if (k <= nzy) {
        if (k < nzy) Yc = (double)U[4 * (size_t)N + (size_t)col * g.NzY + k];
        T_gas = (Yc > 0.0) ? ph.T_pc + (T - ph.T_pc) : T;
    }
    const double H_step = (T > ph.T_pc) ? 1.0 : 0.0;
    const double K_T = ph.A * exp(-ph.T_act / T) * H_step;
    double kT = ph.kT, dk = 0.0;
    if (ph.sutherland_conductivity == 1) {
        kT = 0.0241 * pow(T / 273.15, 1.5) * (273.15 + 194) / (T + 194);
        dk = 0.0241 * (1.5 * pow(T / 273.15, 0.5) * (273.15 + 194) / (T + 194) -
                       pow(T / 273.15, 1.5) * (273.15 + 194) / ((T + 194) * (T + 194)));
    }
    // (T_gas - T_solid) without abs, as the reference (pressure.cu:313)
    const double h_c = ph.h_c * dz_k * pow((T_gas - T_solid) / dz_k, 1.0 / 4.0);
    const double q = ph.H_C * Yc * K_T / ph.c_p -
                     h_c * ph.alpha_s * ph.sigma_s * (T_gas - T_solid) / (ph.c_p * Ti * ri / T_gas);
    const double divT = (dk + 12 * kSigmaSB * ph.delta * pow(T, 2) * (Tx * Tx + Ty * Ty + Tz * Tz) +
                         (kT + 4 * kSigmaSB * ph.delta * pow(T, 3)) * lap_T) / (Ti * ri * ph.c_p) + q / T;
    return rho * (ux + vy + wz - divT) / ph.dt + (rhox * px + rhoy * py + rhoz * pz) / rho;
}

// P1: source + top plane, forward FFT in y of packed slice pairs.
template <class R>
__global__ void __launch_bounds__(256) k_p_rhs_ffty(const PoissonArgs<R> a, int KP)
{
    extern __shared__ double2 smem[];
    const Geom &g = a.g;
    const int n0 = g.Nx - 1, n1 = g.Ny - 1, nk = g.Nz - 1, h1 = a.h1;
    const int m1 = a.fy.m;
    const int i = blockIdx.x;
    const int pair0 = blockIdx.y * KP;
    const int nslices = nk + 1;                      // f slices + top-plane pressure
    const int np = (nslices + 1) / 2;
    const int kp = min(KP, np - pair0);
    double2 *A = smem;
    double *Ad = reinterpret_cast<double *>(A);
    const int ns = 2 * kp;
    for (int t = threadIdx.x; t < n1 * ns; t += blockDim.x) {
        const int jj = t / ns, q = t - jj * ns;
        const int kk = 2 * pair0 + q;
        double val = 0.0;
        if (kk < nk) val = poisson_source(a, i, jj, kk);
        else if (kk == nk) val = a.p[((size_t)i * g.Ny + jj) * g.Nz + (g.Nz - 1)];
        Ad[2 * ((size_t)(q >> 1) * m1 + jj) + (q & 1)] = val;
    }
    __syncthreads();
    fft_lines(a.fy, A, kp, false);
    const double2 *Rb = A;
    // split the packed transform into the two half spectra
    for (int t = threadIdx.x; t < kp * h1; t += blockDim.x) {
        const int line = t / h1, s = t - line * h1;
        const double2 Zs = Rb[(size_t)line * m1 + s];
        const double2 Zc = cconj(Rb[(size_t)line * m1 + (s == 0 ? 0 : n1 - s)]);
        const double2 Fa = make_double2(0.5 * (Zs.x + Zc.x), 0.5 * (Zs.y + Zc.y));
        const double2 Fb = make_double2(0.5 * (Zs.y - Zc.y), -0.5 * (Zs.x - Zc.x));
        const int kk0 = 2 * (pair0 + line);
        a.G[((size_t)kk0 * n0 + i) * h1 + s] = Fa;
        if (kk0 + 1 < nslices) a.G[((size_t)(kk0 + 1) * n0 + i) * h1 + s] = Fb;
    }
}

// P2/P4: FFT along x of slices [0, nslices), SC consecutive s per block.
template <bool INV>
__global__ void __launch_bounds__(256) k_p_fftx(double2 *__restrict__ G, FftDesc fx, int n0, int h1, int SC)
{
    extern __shared__ double2 smem[];
    const int m0 = fx.m;
    const int kk = blockIdx.x;
    const int s0 = blockIdx.y * SC;
    const int sc = min(SC, h1 - s0);
    double2 *A = smem;
    double2 *Gs = G + (size_t)kk * n0 * h1;
    for (int t = threadIdx.x; t < n0 * sc; t += blockDim.x) {
        const int r = t / sc, q = t - r * sc;
        A[(size_t)q * m0 + r] = Gs[(size_t)r * h1 + s0 + q];
    }
    __syncthreads();
    fft_lines(fx, A, sc, INV);
    const double2 *Rb = A;
    for (int t = threadIdx.x; t < n0 * sc; t += blockDim.x) {
        const int r = t / sc, q = t - r * sc;
        Gs[(size_t)r * h1 + s0 + q] = Rb[(size_t)q * m0 + r];
    }
}

// P3: tridiagonal solve in z per (r, s) (pressure.cu:356-390, 473-504, 418-443).
// zt holds per-k constants: [0..nk) a, [nk..2nk) c, [2nk..3nk) D (b = -(kk + D)),
// followed by b0, c0base, inv_dz1, half_dz0, cl.
__global__ void __launch_bounds__(128) k_p_tridiag(double2 *__restrict__ G, const double *__restrict__ kx2,
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
    const size_t stride = (size_t)n0 * h1;
    double2 *g = G + (size_t)r * h1 + s;
    double uk[256];
    // row 0 uses the source of slice 1; rows 1..nk-2 their own; the last row
    // subtracts the top pressure divided by its coupling coefficient
    double2 d0 = g[stride * 1];
    double2 y = make_double2(half_dz0 * d0.x, half_dz0 * d0.y);
    double u = b0;
    uk[0] = u;
    double cprev = c0base - half_dz0 * kk2 - inv_dz1;   // c[0]
    g[0] = y;
    for (int k = 1; k < nk; k++) {
        const double l = za[k - 1] / u;
        const double bk = -(kk2 + zD[k]);
        u = bk - l * cprev;
        uk[k & 255] = u;
        double2 dk = g[stride * k];
        if (k == nk - 1) {
            const double2 pt = g[stride * nk];
            dk = make_double2(dk.x - pt.x / cl, dk.y - pt.y / cl);
        }
        y = make_double2(dk.x - l * y.x, dk.y - l * y.y);
        g[stride * k] = y;
        cprev = zcc[k];
    }
    double2 x = make_double2(y.x / u, y.y / u);
    g[stride * (nk - 1)] = x;
    for (int k = nk - 2; k >= 0; k--) {
        const double ck = (k == 0) ? (c0base - half_dz0 * kk2 - inv_dz1) : zcc[k];
        const double2 yk = g[stride * k];
        const double uu = uk[k & 255];
        x = make_double2((yk.x - ck * x.x) / uu, (yk.y - ck * x.y) / uu);
        g[stride * k] = x;
    }
}

// P5: inverse FFT in y of packed slice pairs, normalisation, write p and the
// periodic duplicate planes (pressure.cu:392-416, deterministic here).
template <class R>
__global__ void __launch_bounds__(256) k_p_iffty_out(const PoissonArgs<R> a, int KP)
{
    extern __shared__ double2 smem[];
    const Geom &g = a.g;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
    const int n0 = Nx - 1, n1 = Ny - 1, nk = Nz - 1, h1 = a.h1;
    const int m1 = a.fy.m;
    const int i = blockIdx.x;
    const int pair0 = blockIdx.y * KP;
    const int np = (nk + 1) / 2;
    const int kp = min(KP, np - pair0);
    double2 *A = smem;
    const bool even = (n1 % 2) == 0;
    for (int t = threadIdx.x; t < kp * n1; t += blockDim.x) {
        const int line = t / n1, s = t - line * n1;
        const int kk0 = 2 * (pair0 + line), kk1 = kk0 + 1;
        const int ss = (s < h1) ? s : n1 - s;
        double2 Fa = a.G[((size_t)kk0 * n0 + i) * h1 + ss];
        double2 Fb = (kk1 < nk) ? a.G[((size_t)kk1 * n0 + i) * h1 + ss] : make_double2(0.0, 0.0);
        if (ss == 0 || (even && ss == n1 / 2)) {
            Fa.y = 0.0;
            Fb.y = 0.0;
        }
        if (s >= h1) {
            Fa.y = -Fa.y;
            Fb.y = -Fb.y;
        }
        A[(size_t)line * m1 + s] = make_double2(Fa.x - Fb.y, Fa.y + Fb.x);
    }
    __syncthreads();
    fft_lines(a.fy, A, kp, true);
    const double2 *Rb = A;
    const double norm = (double)n0 * (double)n1;
    const int ns = 2 * kp;
    double *p = a.p;
    for (int t = threadIdx.x; t < n1 * ns; t += blockDim.x) {
        const int jj = t / ns, q = t - jj * ns;
        const int kk = 2 * pair0 + q;
        if (kk >= nk) continue;
        const double2 zv = Rb[(size_t)(q >> 1) * m1 + jj];
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

}  // namespace

int poisson_pairs_per_block(int m) { return max(1, min(16, 6144 / m)); }
int poisson_lines_per_block(int m) { return max(1, min(16, 6144 / m)); }

template <class R> cudaError_t poisson_set_attributes()
{
    const int maxsm = 200 * 1024;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_p_rhs_ffty<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_p_iffty_out<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    if ((e = cudaFuncSetAttribute(k_p_fftx<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm))) return e;
    return cudaFuncSetAttribute(k_p_fftx<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm);
}
template cudaError_t poisson_set_attributes<double>();
template cudaError_t poisson_set_attributes<float>();

// zt: tridiagonal constants (see k_p_tridiag); passed through the G pointer's
// companion allocation by the caller.
template <class R>
cudaError_t launch_poisson_impl(const PoissonArgs<R> &a, const double *zt, cudaStream_t s, cudaEvent_t *ev)
{
    const int n0 = a.g.Nx - 1, nk = a.g.Nz - 1, h1 = a.h1;
    const int KP = poisson_pairs_per_block(a.fy.m);
    const int SC = poisson_lines_per_block(a.fx.m);
    const int np1 = (nk + 1 + 1) / 2;
    dim3 g1(n0, (np1 + KP - 1) / KP);
    k_p_rhs_ffty<R><<<g1, 256, (size_t)KP * a.fy.m * sizeof(double2), s>>>(a, KP);
    if (ev) cudaEventRecord(ev[0], s);
    dim3 g2(nk + 1, (h1 + SC - 1) / SC);
    k_p_fftx<false><<<g2, 256, (size_t)SC * a.fx.m * sizeof(double2), s>>>(a.G, a.fx, n0, h1, SC);
    if (ev) cudaEventRecord(ev[1], s);
    dim3 g3(n0, (h1 + 127) / 128);
    k_p_tridiag<<<g3, 128, 0, s>>>(a.G, a.kx2, a.ky2, zt, n0, h1, nk);
    if (ev) cudaEventRecord(ev[2], s);
    dim3 g4(nk, (h1 + SC - 1) / SC);
    k_p_fftx<true><<<g4, 256, (size_t)SC * a.fx.m * sizeof(double2), s>>>(a.G, a.fx, n0, h1, SC);
    if (ev) cudaEventRecord(ev[3], s);
    const int np5 = (nk + 1) / 2;
    dim3 g5(n0, (np5 + KP - 1) / KP);
    k_p_iffty_out<R><<<g5, 256, (size_t)KP * a.fy.m * sizeof(double2), s>>>(a, KP);
    if (ev) cudaEventRecord(ev[4], s);
    return cudaGetLastError();
}
template cudaError_t launch_poisson_impl<double>(const PoissonArgs<double> &, const double *, cudaStream_t, cudaEvent_t *);
template cudaError_t launch_poisson_impl<float>(const PoissonArgs<float> &, const double *, cudaStream_t, cudaEvent_t *);

// ---- max |a - b| reduction (pressure fixed point) ------------------------
namespace {
__global__ void __launch_bounds__(256) k_maxdiff(const double *__restrict__ a, const double *__restrict__ b, int n,
                                                  unsigned long long *out)
{
    double m = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const double d = fabs(a[t] - b[t]);
        m = (d > m || d != d) ? d : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const double v = __shfl_xor_sync(0xffffffffu, m, o);
        m = (v > m || v != v) ? v : m;
    }
    // non-negative doubles order like their bit patterns; NaN sorts above inf
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
}  // namespace

cudaError_t launch_maxdiff(const double *a, const double *b, int n, double *out, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
    if (e) return e;
    k_maxdiff<<<592, 256, 0, s>>>(a, b, n, reinterpret_cast<unsigned long long *>(out));
    return cudaGetLastError();
}

}  // namespace wf
