// fft_pr.cuh -- FP64 complex DFT lines of length n = N1 * P in shared memory
// by the prime-factor (Good-Thomas) split and Rader's algorithm, one warp per
// line.  This is the engine for lengths such as 511 = 7 * 73, which a
// power-of-two FFT reaches only through Bluestein's chirp-z identity (two
// FFTs of 1024 points per line).
//
// Plan: N1 odd (1 allowed), P an odd prime not dividing N1, P - 1 = F1 * F2 * F3
// with F1 a power of two (2 ... 16) and F2, F3 odd and coprime (F3 = 1 allowed,
// then F2 = 1 allowed).
//
//   Good-Thomas: x[(P n1 + N1 n2) mod n] -> X[k], k = k1 (mod N1), k = k2 (mod P):
//     Y[k1][n2] = sum_n1 W_N1^(n1 k1) x[P n1 + N1 n2]       (pass A, DFT_N1)
//     X[k1][k2] = sum_n2 W_P^(n2 k2) Y[k1][n2]               (passes B1-B3)
//   Rader with a primitive root g of P, for each k1 (a = Y[k1][.]):
//     X[g^-m] = a[0] + sum_q u[q] b[m - q],  u[q] = a[g^q], b[t] = W_P^(g^-t),
//     X[0]    = a[0] + sum_q u[q],
//   the cyclic convolution of length P - 1 taken as
//     c = IDFT_unnorm(DFT(u) * B'),  B' = DFT(b) / (P - 1),
//   with a[0] added to the DC term before the inverse transform.  DFT and
//   IDFT of length Q = P - 1 are Good-Thomas again over the factors of Q,
//   written here (F1, M, L): (F1, 1, F2) for two factors, (F1, F2, F3) for
//   three.  Input q = (Q/F1 q1 + Q/M qM + Q/L qL) mod Q, output index by CRT.
//
// Passes (each unit's values in registers, one __syncwarp between passes):
//   A   P units (one per n2):            DFT_N1, write the Rader layout
//   B1  N1*M*L units (k1, qM, qL):       DFT_F1 over q1, in place
//   B2a N1*F1*L units (k1, j1, qL):      DFT_M over qM, in place (M > 1)
//   B2  N1*F1*M units (k1, j1, jM):      DFT_L over qL, * B', IDFT_L, in place
//   B2b N1*F1*L units (k1, j1, mL):      IDFT_M over jM, in place (M > 1)
//   B3  N1*M*L units (k1, mM, mL):       IDFT_F1 over j1 -> X[k1][g^-m], post
//
// Rader layout of sub-line k1 (stride SS): slot 0 holds a[0] (then X[k1][0]),
// slot 1 + (q1 M + qM) L + qL holds u at q.  Within B1, B2a, B2b and B3 a
// warp's consecutive lanes read consecutive slots; in B2 they read slots L apart
// (L odd); SS = M L (mod 8) keeps the sub-line boundaries conflict free too.
//
// Tables (device, per length): rb[(j1 M + jM) L + jL] = B'[CRT(j1, jM, jL)];
// map[u] = n2 held by Rader slot u (u < P); map[P + (m1 M + mM) L + mL] =
// (e2 * g^-m) mod n, m the output index of (m1, mM, mL), e2 = N1 (N1^-1 mod P);
// and e1 = P (P^-1 mod N1) mod n, the CRT weight of k1.
//
// Trigonometric constants of the odd DFTs are compile-time values of a Taylor
// series about pi/2 (16 terms, |phi| <= pi/2: error a few units in the last
// place), so every coefficient is an immediate operand.
#pragma once

#include <utility>

#include "fft.cuh"

namespace wf {
namespace fft {

constexpr double kPiD = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr double taylor_sin(double x)
{
    double term = x, sum = x;
    for (int k = 1; k < 16; k++) {
        term *= -x * x / (double)((2 * k) * (2 * k + 1));
        sum += term;
    }
    return sum;
}
__host__ __device__ constexpr double taylor_cos(double x)
{
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 16; k++) {
        term *= -x * x / (double)((2 * k - 1) * (2 * k));
        sum += term;
    }
    return sum;
}
// cos and sin of 2 pi t / R for any integer t
__host__ __device__ constexpr double trig_cos(int R, int t)
{
    t %= R;
    if (t < 0) t += R;
    if (2 * t > R) t = R - t;   // cos is even
    const double phi = 2.0 * kPiD * (double)t / (double)R - 0.5 * kPiD;
    return -taylor_sin(phi);
}
__host__ __device__ constexpr double trig_sin(int R, int t)
{
    t %= R;
    if (t < 0) t += R;
    double sg = 1.0;
    if (2 * t > R) {
        t = R - t;
        sg = -1.0;
    }
    const double phi = 2.0 * kPiD * (double)t / (double)R - 0.5 * kPiD;
    return sg * taylor_cos(phi);
}
template <int R, int T> constexpr double kCosT = trig_cos(R, T);
template <int R, int T> constexpr double kSinT = trig_sin(R, T);

// One output pair (K, R-K) of an odd-length DFT from the pair sums s and
// differences d: X_K = x0 + sum_n cos(2 pi nK/R) s_n - i sum_n sin(2 pi nK/R) d_n.
template <int R, int K, int... N>
__device__ __forceinline__ void odd_pair(double2 (&v)[R], const double2 x0, const double2 (&s)[(R - 1) / 2],
                                         const double2 (&d)[(R - 1) / 2], std::integer_sequence<int, N...>)
{
    double ax = x0.x, ay = x0.y, bx = 0.0, by = 0.0;
    ((ax = fma(kCosT<R, (N + 1) * K>, s[N].x, ax), ay = fma(kCosT<R, (N + 1) * K>, s[N].y, ay),
      bx = fma(kSinT<R, (N + 1) * K>, d[N].x, bx), by = fma(kSinT<R, (N + 1) * K>, d[N].y, by)),
     ...);
    v[K] = make_double2(ax + by, ay - bx);
    v[R - K] = make_double2(ax - by, ay + bx);
}
template <int R, int... K>
__device__ __forceinline__ void odd_pairs(double2 (&v)[R], const double2 x0, const double2 (&s)[(R - 1) / 2],
                                          const double2 (&d)[(R - 1) / 2], std::integer_sequence<int, K...>)
{
    (odd_pair<R, K + 1>(v, x0, s, d, std::make_integer_sequence<int, (R - 1) / 2>{}), ...);
}

// In-place forward DFT of odd length R (R = 1: nothing), natural output order.
template <int R>
__device__ __forceinline__ void dft_odd(double2 (&v)[R])
{
    if constexpr (R > 1) {
        constexpr int H = (R - 1) / 2;
        double2 s[H], d[H];
        double2 sum = v[0];
#pragma unroll
        for (int n = 1; n <= H; n++) {
            s[n - 1] = cadd(v[n], v[R - n]);
            d[n - 1] = csub(v[n], v[R - n]);
            sum = cadd(sum, s[n - 1]);
        }
        const double2 x0 = v[0];
        odd_pairs<R>(v, x0, s, d, std::make_integer_sequence<int, H>{});
        v[0] = sum;
    }
}

// In-place forward DFT of power-of-two length R (2 ... 16), natural output order.
template <int R>
__device__ __forceinline__ void dft_pow2(double2 (&v)[R])
{
    dft<R>(v);
    if constexpr (R == 16) {
        double2 t[16];
#pragma unroll
        for (int r = 0; r < 16; r++) t[r] = v[out_slot<16>(r)];
#pragma unroll
        for (int r = 0; r < 16; r++) v[r] = t[r];
    }
}

// Tables of one length (see the file comment).
struct PrTables {
    const double2 *rb;
    const int *map;
    int e1;
};

template <int N1_, int P_, int F1_, int F2_, int F3_ = 1>
struct PrPlan {
    static constexpr int N1 = N1_, P = P_, F1 = F1_, F2 = F2_, F3 = F3_;
    static constexpr int n = N1 * P;
    static constexpr int M = (F3 > 1) ? F2 : 1, L = (F3 > 1) ? F3 : F2;   // middle, innermost factor
    static_assert(N1 % 2 == 1 && P % 2 == 1 && F2 % 2 == 1 && F3 % 2 == 1, "odd factors");
    static_assert(F1 == 2 || F1 == 4 || F1 == 8 || F1 == 16, "power-of-two factor");
    static_assert(F1 * F2 * F3 == P - 1, "Rader length");
    static_assert(N1 == 1 || N1 % P != 0, "coprime factors");
    static constexpr int gcd(int a, int b) { return b == 0 ? a : gcd(b, a % b); }
    static_assert(F3 == 1 || (F2 > 1 && gcd(F2, F3) == 1), "coprime odd factors");
    // sub-line stride: >= P, = M L (mod 8)
    static constexpr int SS = P + (((M * L - P) % 8) + 8) % 8;
    static constexpr int LB = 8;                              // lines (warps) per 256-thread block
    static constexpr int LS0 = (n > N1 * SS) ? n : N1 * SS;
    static constexpr int LS = LS0 + ((1 - LS0 % 8) + 8) % 8;   // line stride = 1 (mod 8)
    static constexpr size_t smem_bytes = (size_t)LB * LS * 16;
    static constexpr int RA = (P + 31) / 32;                  // rounds of pass A
    static constexpr int UB = N1 * M * L;                     // units of B1 and B3
    static constexpr int RB = (UB + 31) / 32;
    static constexpr int UC = N1 * F1 * M;                    // units of B2
    static constexpr int RC = (UC + 31) / 32;
    static constexpr int UD = N1 * F1 * L;                    // units of B2a, B2b
    static constexpr int RD = (UD + 31) / 32;

    // Forward DFT (INV: exp(+2 pi i jk/n), unnormalised) of the line at buf,
    // by the 32 lanes of one warp.  pre(idx) supplies x[idx] (idx < n) and is
    // called before the first write to buf; post(idx, X) receives X[idx] after
    // the last read of buf, so pre may read and post may write buf.  SLOT: pre
    // and post take the slots of the plan's slot table instead (input x[j] at
    // n1 SS + u, output X[k] at m1 UB + u or F1 UB + k1), which a warp's lanes
    // visit contiguously: a caller that stores its line in that order in shared
    // memory (the permutations moved into its copies) reads and writes it
    // without bank conflicts.
    template <bool INV, bool SLOT = false, class Pre, class Post>
    __device__ __forceinline__ static void run(const PrTables &t, double2 *buf, int lane, Pre pre, Post post)
    {
        // pass A.  Slotted, a lane reads and writes the same slots (j SS + u for
        // its u), so it transforms one round at a time; in the plain run its
        // writes may land on inputs other lanes have yet to read, so all reads
        // come first.
        if constexpr (SLOT) {
#pragma unroll
            for (int r = 0; r < RA; r++) {
                const int u = lane + 32 * r;
                if (u < P) {
                    double2 v[N1];
#pragma unroll
                    for (int n1 = 0; n1 < N1; n1++) {
                        v[n1] = pre(n1 * SS + u);
                        if (INV) v[n1].y = -v[n1].y;
                    }
                    dft_odd<N1>(v);
#pragma unroll
                    for (int k1 = 0; k1 < N1; k1++) buf[k1 * SS + u] = v[k1];
                }
            }
            __syncwarp();
        } else {
            double2 v[RA][N1];
#pragma unroll
            for (int r = 0; r < RA; r++) {
                const int u = lane + 32 * r;
                if (u < P) {
                    const int base = N1 * __ldg(t.map + u);
#pragma unroll
                    for (int n1 = 0; n1 < N1; n1++) {
                        int idx = base + P * n1;
                        if (idx >= n) idx -= n;
                        v[r][n1] = pre(idx);
                        if (INV) v[r][n1].y = -v[r][n1].y;
                    }
                }
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < RA; r++) {
                const int u = lane + 32 * r;
                if (u < P) {
                    dft_odd<N1>(v[r]);
#pragma unroll
                    for (int k1 = 0; k1 < N1; k1++) buf[k1 * SS + u] = v[r][k1];
                }
            }
            __syncwarp();
        }
        // pass B1: DFT_F1 over q1 (slot stride M L)
#pragma unroll
        for (int r = 0; r < RB; r++) {
            const int u = lane + 32 * r;
            if (u < UB) {
                const int k1 = u / (M * L), w = u - k1 * (M * L);
                double2 *b = buf + k1 * SS + 1 + w;
                double2 v[F1];
#pragma unroll
                for (int q1 = 0; q1 < F1; q1++) v[q1] = b[M * L * q1];
                dft_pow2<F1>(v);
#pragma unroll
                for (int j1 = 0; j1 < F1; j1++) b[M * L * j1] = v[j1];
            }
        }
        __syncwarp();
        // pass B2a: DFT_M over qM (slot stride L)
        if constexpr (M > 1) {
#pragma unroll
            for (int r = 0; r < RD; r++) {
                const int u = lane + 32 * r;
                if (u < UD) {
                    const int k1 = u / (F1 * L), w = u - k1 * (F1 * L), j1 = w / L, qL = w - j1 * L;
                    double2 *b = buf + k1 * SS + 1 + j1 * M * L + qL;
                    double2 v[M];
#pragma unroll
                    for (int q = 0; q < M; q++) v[q] = b[L * q];
                    dft_odd<M>(v);
#pragma unroll
                    for (int q = 0; q < M; q++) b[L * q] = v[q];
                }
            }
            __syncwarp();
        }
        // pass B2: DFT_L over qL, pointwise product with B', IDFT_L
#pragma unroll
        for (int r = 0; r < RC; r++) {
            const int u = lane + 32 * r;
            if (u < UC) {
                const int k1 = u / (F1 * M), jj = u - k1 * (F1 * M);   // jj = j1 M + jM
                double2 *b = buf + k1 * SS + 1 + L * jj;
                double2 v[L];
#pragma unroll
                for (int q = 0; q < L; q++) v[q] = b[q];
                dft_odd<L>(v);
                double2 a0 = make_double2(0.0, 0.0);
                if (jj == 0) {
                    a0 = buf[k1 * SS];
                    buf[k1 * SS] = cadd(a0, v[0]);   // X[k1][0]
                }
                const double2 *w = t.rb + L * jj;
#pragma unroll
                for (int q = 0; q < L; q++) v[q] = cmul(v[q], __ldg(w + q));
                v[0] = cadd(v[0], a0);
                // IDFT = conj(DFT(conj(.)))
#pragma unroll
                for (int q = 0; q < L; q++) v[q].y = -v[q].y;
                dft_odd<L>(v);
#pragma unroll
                for (int q = 0; q < L; q++) b[q] = make_double2(v[q].x, -v[q].y);
            }
        }
        __syncwarp();
        // pass B2b: IDFT_M over jM
        if constexpr (M > 1) {
#pragma unroll
            for (int r = 0; r < RD; r++) {
                const int u = lane + 32 * r;
                if (u < UD) {
                    const int k1 = u / (F1 * L), w = u - k1 * (F1 * L), j1 = w / L, mL = w - j1 * L;
                    double2 *b = buf + k1 * SS + 1 + j1 * M * L + mL;
                    double2 v[M];
#pragma unroll
                    for (int q = 0; q < M; q++) v[q] = make_double2(b[L * q].x, -b[L * q].y);
                    dft_odd<M>(v);
#pragma unroll
                    for (int q = 0; q < M; q++) b[L * q] = make_double2(v[q].x, -v[q].y);
                }
            }
            __syncwarp();
        }
        // pass B3: IDFT_F1 over j1, outputs
        {
            double2 v[RB][F1], x0[RB];
#pragma unroll
            for (int r = 0; r < RB; r++) {
                const int u = lane + 32 * r;
                if (u < UB) {
                    const int k1 = u / (M * L), w = u - k1 * (M * L);
                    const double2 *b = buf + k1 * SS + 1 + w;
#pragma unroll
                    for (int j1 = 0; j1 < F1; j1++) v[r][j1] = b[M * L * j1];
                    if (w == 0) x0[r] = buf[k1 * SS];
                }
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < RB; r++) {
                const int u = lane + 32 * r;
                if (u < UB) {
                    const int k1 = u / (M * L), w = u - k1 * (M * L);
                    const int kb = (k1 * t.e1) % n;
#pragma unroll
                    for (int j1 = 0; j1 < F1; j1++) v[r][j1].y = -v[r][j1].y;
                    dft_pow2<F1>(v[r]);
                    const int *km = t.map + P + w;
#pragma unroll
                    for (int m1 = 0; m1 < F1; m1++) {
                        int idx;
                        if constexpr (SLOT) {
                            idx = m1 * UB + u;
                        } else {
                            idx = kb + __ldg(km + M * L * m1);
                            if (idx >= n) idx -= n;
                        }
                        // conj of the IDFT trick, and of the inverse transform
                        const double2 x = v[r][m1];
                        post(idx, INV ? x : make_double2(x.x, -x.y));
                    }
                    if (w == 0) {
                        const double2 x = x0[r];
                        post(SLOT ? F1 * UB + k1 : kb, INV ? make_double2(x.x, -x.y) : x);
                    }
                }
            }
        }
    }
};

}  // namespace fft
}  // namespace wf
