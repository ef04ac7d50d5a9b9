// fft.cuh -- batched FP64 complex FFT lines in shared memory for sm_100a.
//
// A block of 256 threads transforms LB lines of length M = 2^L at once.  With
// largest radix RM (8 or 16), each line belongs to T = M/RM threads (T = 1 for
// M < RM); thread (q, jj) with q = tid % LB (the line) and jj = tid / LB holds
// RM complex values in registers per stage.  The transform is a Stockham
// auto-sort FFT with radix-RM stages and one final smaller power-of-two stage
// when L is not a multiple of log2(RM): a 1024-point line takes three passes
// through shared memory at radix 16, four at radix 8 (with half the registers).
//
// Shared-memory layout: element i of line q sits at q*LS + pad(i) with
// pad(i) = i + i/RM (one spare slot per RM).  The padding makes the stride-RM
// Stockham writes of the first stage conflict-free; the line stride LS is
// chosen so that the 8 lanes of one 128-byte shared-memory phase (8 lines at
// the same position when LB >= 8, otherwise LB lines x 8/LB positions) fall in
// 8 different 16-byte bank groups.
//
// Input enters through a functor pre(idx) -> double2 (global memory, shared
// memory, or a fused pointwise product) and output leaves through
// post(idx, value), so the Bluestein chirp products, the x-pass global loads
// and stores and the Hermitian packing are fused into the first and last
// stages.  tw[j] = exp(-2 pi i j / M).  All transforms are forward
// (exp(-2 pi i jk/M)); inverse ones conjugate on the way in and out.
#pragma once

#include <cuda_runtime.h>

namespace wf {
namespace fft {

// RM: the largest radix (8 or 16); each thread holds RM complex values per stage.
template <int L, int RM = 16>
struct Shape {
    static constexpr int M = 1 << L;
    static constexpr int T = (M >= RM) ? M / RM : 1;       // threads per line
    static constexpr int LB = 256 / T;                     // lines per block
    static constexpr int MP = M + M / RM;                  // padded line length
    static constexpr int C = (LB >= 8) ? 1 : 8 / LB;       // wanted LS mod 8
    static constexpr int LS = MP + (((C % 8) - (MP % 8)) + 8) % 8;
    static constexpr size_t smem_bytes = (size_t)LB * LS * 16;
};

// padded position of element i: one spare slot after every RM elements
template <int RM = 16> __device__ __forceinline__ int pad(int i) { return i + (RM == 16 ? (i >> 4) : (i >> 3)); }

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }   // * (-i)

// cos(pi/8), sin(pi/8), sqrt(1/2)
constexpr double kC8 = 0.92387953251128675613;
constexpr double kS8 = 0.38268343236508977173;
constexpr double kH = 0.70710678118654752440;

// a * exp(-2 pi i m / 16) for the exponents the 4x4 split uses
template <int E>
__device__ __forceinline__ double2 w16(double2 a)
{
    if constexpr (E == 0) return a;
    else if constexpr (E == 1) return make_double2(a.x * kC8 + a.y * kS8, a.y * kC8 - a.x * kS8);
    else if constexpr (E == 2) return make_double2(kH * (a.x + a.y), kH * (a.y - a.x));
    else if constexpr (E == 3) return make_double2(a.x * kS8 + a.y * kC8, a.y * kS8 - a.x * kC8);
    else if constexpr (E == 4) return mul_mi(a);
    else if constexpr (E == 6) return make_double2(kH * (a.y - a.x), -kH * (a.x + a.y));
    else return make_double2(-a.x * kC8 - a.y * kS8, a.x * kS8 - a.y * kC8);   // E == 9
}

__device__ __forceinline__ void dft2(double2 &a0, double2 &a1)
{
    const double2 t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}

__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3)
{
    const double2 s0 = cadd(a0, a2), d0 = csub(a0, a2);
    const double2 s1 = cadd(a1, a3), d1 = mul_mi(csub(a1, a3));
    a0 = cadd(s0, s1);
    a2 = csub(s0, s1);
    a1 = cadd(d0, d1);
    a3 = csub(d0, d1);
}

// Slot of output r after dft<R>: the radix-16 transform leaves X[k1 + 4 k2]
// in slot 4 k1 + k2 (a 4x4 transpose the stores undo for free).
template <int R>
__host__ __device__ constexpr int out_slot(int r)
{
    return (R == 16) ? (((r & 3) << 2) | (r >> 2)) : r;
}

// In-place length-R forward DFT; output r lands in slot out_slot<R>(r).
template <int R>
__device__ __forceinline__ void dft(double2 (&v)[R])
{
    if constexpr (R == 2) {
        dft2(v[0], v[1]);
    } else if constexpr (R == 4) {
        dft4(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        // n = 2 n1 + n2: DFT4 over n1, twiddle W8^(n2 k1), DFT2 over n2 -> X[k1 + 4 k2]
        double2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
        double2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
        dft4(a0, a1, a2, a3);
        dft4(b0, b1, b2, b3);
        b1 = w16<2>(b1);
        b2 = mul_mi(b2);
        b3 = w16<6>(b3);
        v[0] = cadd(a0, b0); v[4] = csub(a0, b0);
        v[1] = cadd(a1, b1); v[5] = csub(a1, b1);
        v[2] = cadd(a2, b2); v[6] = csub(a2, b2);
        v[3] = cadd(a3, b3); v[7] = csub(a3, b3);
    } else {
        static_assert(R == 16, "radix");
        // n = 4 n1 + n2: DFT4 over n1 per n2, twiddle W16^(n2 k1), DFT4 over n2;
        // X[k1 + 4 k2] ends in slot 4 k1 + k2
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
        // now v[n2 + 4 k1] holds A[n2][k1]
        v[5] = w16<1>(v[5]);  v[9] = w16<2>(v[9]);   v[13] = w16<3>(v[13]);
        v[6] = w16<2>(v[6]);  v[10] = w16<4>(v[10]); v[14] = w16<6>(v[14]);
        v[7] = w16<3>(v[7]);  v[11] = w16<6>(v[11]); v[15] = w16<9>(v[15]);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    }
}

// One Stockham stage with Ns = 2^SL, followed by the remaining stages.
template <int L, int RM, int SL, bool FIRST, class Pre, class Post>
__device__ __forceinline__ void stage(double2 *buf, int jj, const double2 *__restrict__ tw, Pre &pre, Post &post)
{
    constexpr int M = 1 << L;
    constexpr int REM = L - SL;
    constexpr int LRM = (RM == 16) ? 4 : 3;
    constexpr int LR = (REM >= LRM) ? LRM : REM;
    constexpr int R = 1 << LR;
    constexpr bool LAST = (REM == LR);
    constexpr int T = Shape<L, RM>::T;
    constexpr int NB = (M / R) / T;
    constexpr int Ns = 1 << SL;
    double2 v[NB][R];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = jj + T * b;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int idx = j + r * (M / R);
            if constexpr (FIRST) v[b][r] = pre(idx);
            else v[b][r] = buf[pad<RM>(idx)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = jj + T * b;
        const int k = j & (Ns - 1);
        if constexpr (Ns > 1) {
            // twiddles w^r, w = exp(-2 pi i k / (Ns R)): powers of two from the
            // table, the rest as products of at most three of them
            constexpr int SH = L - SL - LR;
            double2 w[R];
            w[1] = __ldg(tw + (k << SH));
            if constexpr (R > 2) w[2] = __ldg(tw + ((2 * k) << SH));
            if constexpr (R > 4) w[4] = __ldg(tw + ((4 * k) << SH));
            if constexpr (R > 8) w[8] = __ldg(tw + ((8 * k) << SH));
#pragma unroll
            for (int r = 3; r < R; r++) {
                if ((r & (r - 1)) == 0) continue;
                const int hi = 1 << (31 - __clz(r));     // highest power of two in r
                w[r] = cmul(w[hi], w[r - hi]);
            }
#pragma unroll
            for (int r = 1; r < R; r++) v[b][r] = cmul(v[b][r], w[r]);
        }
        dft<R>(v[b]);
        const int base = ((j >> SL) << (SL + LR)) + k;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const int o = base + (r << SL);
            if constexpr (LAST) post(o, v[b][out_slot<R>(r)]);
            else buf[pad<RM>(o)] = v[b][out_slot<R>(r)];
        }
    }
    if constexpr (!LAST) {
        __syncthreads();
        stage<L, RM, SL + LR, false>(buf, jj, tw, pre, post);
    }
}

// Forward FFT of the line owned by (buf, jj).  Every thread of the block must
// call it (it synchronises the block).  pre is read once per element in the
// first stage after which a block barrier follows, so pre may read buf; post is
// called once per element after the last barrier, so it may write buf.
template <int L, int RM, class Pre, class Post>
__device__ __forceinline__ void run(double2 *buf, int jj, const double2 *__restrict__ tw, Pre pre, Post post)
{
    stage<L, RM, 0, true>(buf, jj, tw, pre, post);
}

}  // namespace fft
}  // namespace wf
