// closure.cu -- learned subgrid closure: a small MLP predicts the local
// coefficient c(x) that replaces C_s^2 in mu_sgs = rho c Delta^2 |S|
// (Smagorinsky: c = C_s^2, reference pde.cu:745).  No reference counterpart.
//
// Network: 12 -> 64 -> 64 -> 1, GELU (tanh form) hidden activations,
// softplus output.  Features per cell: the resolved strain rate (6), the
// vorticity (3) and grad T (3) by central differences, velocity gradients
// scaled by Delta / 1 m/s and temperature gradients by Delta / 100 K, then by
// per-feature scales learned with the weights; Delta = (dx dy dz_k)^(1/3).
//
//   k_closure_coef_tc  inference for every cell of a stage input on the
//                   5th-generation tensor cores: tcgen05.mma with BF16 operands
//                   in shared memory and FP32 accumulators in tensor memory,
//                   128 cells per CTA.  The stage kernel reads the coefficient
//                   in place of C_s^2.
//   k_mlp_grad      training: FP32 forward + backward per sample, gradients
//                   accumulated in shared memory then in global memory.
//   k_adam          Adam update of the FP32 master parameters.
//
// Parameter vector (FP32): W1[64][12], b1[64], W2[64][64], b2[64], W3[64],
// b3, then 12 feature scales.
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <cuda_bf16.h>

#include "wf_internal.h"

namespace wf {

namespace {

constexpr int NIN = 12, NH = 64;
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NH;
constexpr int NPARAM = OB3 + 1;            // 5057
constexpr int NTOTAL = NPARAM + NIN;       // + feature scales
constexpr float kGeluK = 0.7978845608028654f;   // sqrt(2/pi)

__device__ __forceinline__ float gelu(float x)
{
    return 0.5f * x * (1.0f + tanhf(kGeluK * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x)
{
    const float t = tanhf(kGeluK * (x + 0.044715f * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluK * (1.0f + 3.0f * 0.044715f * x * x);
}
// Inference form: the hardware tanh approximation (PTX tanh.approx.f32, about
// 2^-11 relative error) is well inside the BF16 rounding the hidden
// activations get anyway; training keeps tanhf (its gradients are checked to 1e-4).
__device__ __forceinline__ float tanh_approx(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// Two activations at once on the paired FP32 pipe (FMUL2 / FFMA2, each lane
// rounded like the scalar form): GELU(x) = h + h tanh(z), h = x/2,
// z = x (k + k 0.044715 x^2) -- the tanh form above with its products regrouped.
constexpr float kGeluK3 = kGeluK * 0.044715f;
__device__ __forceinline__ float2 gelu2(float2 x)
{
    const float2 a = __fmul2_rn(x, x);
    const float2 b = __ffma2_rn(a, make_float2(kGeluK3, kGeluK3), make_float2(kGeluK, kGeluK));
    const float2 z = __fmul2_rn(b, x);
    const float2 t = make_float2(tanh_approx(z.x), tanh_approx(z.y));
    const float2 h = __fmul2_rn(x, make_float2(0.5f, 0.5f));
    return __ffma2_rn(h, t, h);
}
__device__ __forceinline__ float softplus(float x) { return x > 20.0f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

__device__ __forceinline__ int wrap1(int v, int n)
{
    if (v >= n) v -= n;
    if (v < 0) v += n;
    return v;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (lower 16 bits)
    return *reinterpret_cast<const uint32_t *>(&v);
}

// The 12 raw features at cell (i, j, k) of the state X (walls: zero).
// hz = 1 / (z[k+1] - z[k-1]) and delta = (dx dy dz_k)^(1/3) of the cell's plane
// come from a per-plane table (plane_scales).
template <class R>
__device__ void cell_features(const R *__restrict__ X, const Geom &g, double dx, double dy, int i, int j, int k,
                              float hz, float delta, float (&f)[NIN])
{
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
    const size_t N = (size_t)g.N;
    if (k == 0 || k == Nz - 1) {
#pragma unroll
        for (int q = 0; q < NIN; q++) f[q] = 0.0f;
        return;
    }
    const int ip = wrap1(i + 1, Nx - 1), im = wrap1(i - 1, Nx - 1);
    const int jp = wrap1(j + 1, Ny - 1), jm = wrap1(j - 1, Ny - 1);
    const size_t c = ((size_t)i * Ny + j) * Nz + k;
    const size_t cxp = ((size_t)ip * Ny + j) * Nz + k, cxm = ((size_t)im * Ny + j) * Nz + k;
    const size_t cyp = ((size_t)i * Ny + jp) * Nz + k, cym = ((size_t)i * Ny + jm) * Nz + k;
    const float hx = (float)(0.5 / dx), hy = (float)(0.5 / dy);
    float d[4][3];   // d[field][x, y, z]
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const R *F = X + q * N;
        d[q][0] = ((float)F[cxp] - (float)F[cxm]) * hx;
        d[q][1] = ((float)F[cyp] - (float)F[cym]) * hy;
        d[q][2] = ((float)F[c + 1] - (float)F[c - 1]) * hz;
    }
    const float sv = delta, st = delta * 0.01f;   // Delta / (1 m/s), Delta / (100 K)
    f[0] = d[0][0] * sv;
    f[1] = d[1][1] * sv;
    f[2] = d[2][2] * sv;
    f[3] = 0.5f * (d[0][1] + d[1][0]) * sv;
    f[4] = 0.5f * (d[0][2] + d[2][0]) * sv;
    f[5] = 0.5f * (d[1][2] + d[2][1]) * sv;
    f[6] = (d[2][1] - d[1][2]) * sv;
    f[7] = (d[0][2] - d[2][0]) * sv;
    f[8] = (d[1][0] - d[0][1]) * sv;
    f[9] = d[3][0] * st;
    f[10] = d[3][1] * st;
    f[11] = d[3][2] * st;
}

// ---- inference on the 5th-generation tensor cores (tcgen05 + TMEM) ---------------
// One CTA of 128 threads (one warpgroup) per tile of 128 cells, persistent over
// tiles.  Thread r computes the features of cell r of the tile into the A
// operand (BF16, K-major, no swizzle: 8-row x 16-byte core matrices); one
// thread issues tcgen05.mma (M = 128, N = 64, FP32 accumulation in TMEM) for
// layer 1 (K = 16) and, after the epilogue has written GELU(h1) back as the
// next A operand, four for layer 2 (K = 64); each warp reads its 32 TMEM lanes
// (= its 32 cells) with tcgen05.ld.  Every mbarrier wait is bounded (wait_limit
// polls): on timeout the kernel raises *err, skips the rest, gives the MMA group
// in flight kDrainLimit polls to finish and still frees its TMEM.
// FEAT = false: the features of every cell of the state X (coef[cell]);
// FEAT = true: n rows of 12 raw features from feat (coef[row]).
constexpr int kTcThreads = 128, kTcCols = 128;
constexpr int kDrainLimit = 1 << 22;
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
constexpr size_t kTcA1 = 0, kTcA2 = kTcA1 + 128 * 16 * 2, kTcB1 = kTcA2 + 128 * 64 * 2, kTcB2 = kTcB1 + 64 * 16 * 2;
constexpr size_t kTcF = kTcB2 + 64 * 64 * 2;                       // fp32: b1, b2, W3, b3, scales
constexpr size_t kTcBar = kTcF + sizeof(float) * (64 + 64 + 64 + 4 + 12);
constexpr int kTcPlanes = wf::kMaxZUnknowns + 1;                    // per-plane feature scales
constexpr size_t kTcPlane = kTcBar + 16;                           // float hz[kTcPlanes], delta[kTcPlanes]
constexpr size_t kSmemTc = kTcPlane + sizeof(float) * 2 * kTcPlanes;

// byte offset of (row, k) in a K-major no-swizzle operand with K/8 core
// matrices per 8-row group (core matrix = 8 rows x 8 bf16 = 128 bytes)
__device__ __forceinline__ uint32_t tc_off(int row, int k, int kchunks)
{
    return (uint32_t)(((row >> 3) * kchunks + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    const uint32_t z = 0;
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 :
                 : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, int limit)
{
    for (int it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

// 64 FP32 accumulators of this thread's TMEM lane, columns [col, col + 64)
__device__ __forceinline__ void tc_ld64(uint32_t taddr, float (&v)[64])
{
    uint32_t r[64];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                 "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, "
                 "%35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, "
                 "%56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
                   "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
                   "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
                   "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
                   "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 64; q++) v[q] = __uint_as_float(r[q]);
}

template <class R, bool FEAT>
__global__ void __launch_bounds__(kTcThreads, 4) k_closure_coef_tc(const R *__restrict__ X, Geom g, double dx,
                                                                   double dy, const float *__restrict__ feat, size_t nfeat,
                                                                   const float *__restrict__ theta,
                                                                   R *__restrict__ coef, int *err, int wait_limit)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint32_t s_taddr;
    float *sb1 = reinterpret_cast<float *>(smem + kTcF), *sb2 = sb1 + 64, *sW3 = sb2 + 64, *sb3 = sW3 + 64;
    float *sscale = sb3 + 4;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t bar = sbase + (uint32_t)kTcBar;
    // weights -> B operands (rows = output neurons, K-major)
    for (int t = tid; t < 64 * 16; t += kTcThreads) {
        const int n = t >> 4, k = t & 15;
        *reinterpret_cast<__nv_bfloat16 *>(smem + kTcB1 + tc_off(n, k, 2)) =
            __float2bfloat16(k < NIN ? theta[OW1 + n * NIN + k] : 0.0f);
    }
    for (int t = tid; t < 64 * 64; t += kTcThreads) {
        const int n = t >> 6, k = t & 63;
        *reinterpret_cast<__nv_bfloat16 *>(smem + kTcB2 + tc_off(n, k, 8)) = __float2bfloat16(theta[OW2 + n * NH + k]);
    }
    for (int t = tid; t < 64; t += kTcThreads) {
        sb1[t] = theta[OB1 + t];
        sb2[t] = theta[OB2 + t];
        sW3[t] = theta[OW3 + t];
    }
    if (tid == 0) sb3[0] = theta[OB3];
    if (tid < NIN) sscale[tid] = theta[NPARAM + tid];
    float *shz = reinterpret_cast<float *>(smem + kTcPlane), *sdel = shz + kTcPlanes;
    if (!FEAT) {
        // per-plane feature scales: 1 / (z[k+1] - z[k-1]) and (dx dy dz_k)^(1/3)
        for (int k = tid; k < g.Nz && k < kTcPlanes; k += kTcThreads) {
            shz[k] = (k > 0 && k < g.Nz - 1) ? (float)(1.0 / (g.z[k + 1] - g.z[k - 1])) : 0.0f;
            sdel[k] = (float)cbrt(dx * dy * g.zc[ZDZ * g.Nz + k]);
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&s_taddr);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = s_taddr;
    const uint32_t lane_base = taddr + ((uint32_t)(32 * warp) << 16);
    const uint64_t dB1 = tc_desc(sbase + (uint32_t)kTcB1, 128, 256);
    const size_t N = FEAT ? nfeat : (size_t)g.N;
    const size_t ntiles = (N + 127) / 128;
    uint32_t phase = 0;
    bool ok = true;
    for (size_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const size_t cell = tile * 128 + tid;
        float f[NIN];
        if (cell < N && FEAT) {
#pragma unroll
            for (int q = 0; q < NIN; q++) f[q] = feat[cell * NIN + q];
        } else if (cell < N) {
            const int k = (int)(cell % g.Nz), j = (int)((cell / g.Nz) % g.Ny), i = (int)(cell / ((size_t)g.Nz * g.Ny));
            cell_features(X, g, dx, dy, i, j, k, shz[k], sdel[k], f);
        } else {
#pragma unroll
            for (int q = 0; q < NIN; q++) f[q] = 0.0f;
        }
        {
            uint4 lo, hi;
            lo.x = pack_bf16(f[0] * sscale[0], f[1] * sscale[1]);
            lo.y = pack_bf16(f[2] * sscale[2], f[3] * sscale[3]);
            lo.z = pack_bf16(f[4] * sscale[4], f[5] * sscale[5]);
            lo.w = pack_bf16(f[6] * sscale[6], f[7] * sscale[7]);
            hi.x = pack_bf16(f[8] * sscale[8], f[9] * sscale[9]);
            hi.y = pack_bf16(f[10] * sscale[10], f[11] * sscale[11]);
            hi.z = 0u;
            hi.w = 0u;
            *reinterpret_cast<uint4 *>(smem + kTcA1 + tc_off(tid, 0, 2)) = lo;
            *reinterpret_cast<uint4 *>(smem + kTcA1 + tc_off(tid, 8, 2)) = hi;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
            tc_mma(taddr, tc_desc(sbase + (uint32_t)kTcA1, 128, 256), dB1, 0u);
            tc_commit(bar);
        }
        ok = __syncthreads_and(tc_wait(bar, phase, wait_limit) ? 1 : 0);
        phase ^= 1u;
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float acc[64];
        tc_ld64(lane_base, acc);
        // layer-1 epilogue: GELU(h + b1) -> A operand of layer 2 (row tid)
        const float2 *sb1p = reinterpret_cast<const float2 *>(sb1);
#pragma unroll
        for (int c = 0; c < 8; c++) {
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int e = 8 * c + 2 * q;
                const float2 gv = gelu2(__fadd2_rn(make_float2(acc[e], acc[e + 1]), sb1p[e >> 1]));
                w[q] = pack_bf16(gv.x, gv.y);
            }
            *reinterpret_cast<uint4 *>(smem + kTcA2 + tc_off(tid, 8 * c, 8)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int s = 0; s < 4; s++)
                tc_mma(taddr + 64, tc_desc(sbase + (uint32_t)kTcA2 + 256u * s, 128, 1024),
                       tc_desc(sbase + (uint32_t)kTcB2 + 256u * s, 128, 1024), s > 0 ? 1u : 0u);
            tc_commit(bar);
        }
        ok = __syncthreads_and(tc_wait(bar, phase, wait_limit) ? 1 : 0);
        phase ^= 1u;
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tc_ld64(lane_base + 64, acc);
        // layer 3: W3 . GELU(h2 + b2) + b3, two partial sums on the paired pipe
        const float2 *sb2p = reinterpret_cast<const float2 *>(sb2), *sW3p = reinterpret_cast<const float2 *>(sW3);
        float2 o2 = make_float2(0.0f, 0.0f);
#pragma unroll
        for (int q = 0; q < 32; q++)
            o2 = __ffma2_rn(gelu2(__fadd2_rn(make_float2(acc[2 * q], acc[2 * q + 1]), sb2p[q])), sW3p[q], o2);
        const float o = sb3[0] + (o2.x + o2.y);
        if (cell < N) coef[cell] = (R)softplus(o);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();   // TMEM and operands free for the next tile
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok) {
        // give the MMA group in flight a bounded chance to finish before TMEM is freed
        tc_wait(bar, phase ^ 1u, kDrainLimit);
        if (tid == 0 && err) atomicExch(err, 1);
    }
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTcCols) : "memory");
}

// ---- training ------------------------------------------------------------------
constexpr int kTrainThreads = 128;

// Loss and gradient over samples [0, n): thread per sample, FP32.  grad (NPARAM)
// and loss must be zero on entry.  xs: normalised features [n][12].
__global__ void __launch_bounds__(kTrainThreads) k_mlp_grad(const float *__restrict__ theta,
                                                          const float *__restrict__ xs, const float *__restrict__ ys,
                                                          const int *__restrict__ idx, int n, float *grad,
                                                          double *loss)
{
    __shared__ float sth[NPARAM];
    __shared__ float sg[NPARAM];
    __shared__ float sloss[kTrainThreads / 32];
    for (int t = threadIdx.x; t < NPARAM; t += blockDim.x) {
        sth[t] = theta[t];
        sg[t] = 0.0f;
    }
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    float lsum = 0.0f;
    if (s < n) {
        const int q = idx ? idx[s] : s;
        float x[NIN];
#pragma unroll
        for (int i = 0; i < NIN; i++) x[i] = xs[(size_t)q * NIN + i];
        float a1[NH], h1[NH], a2[NH];
        for (int o = 0; o < NH; o++) {
            float acc = sth[OB1 + o];
#pragma unroll
            for (int i = 0; i < NIN; i++) acc += sth[OW1 + o * NIN + i] * x[i];
            a1[o] = acc;
            h1[o] = gelu(acc);
        }
        float out = sth[OB3];
        for (int o = 0; o < NH; o++) {
            float acc = sth[OB2 + o];
            for (int i = 0; i < NH; i++) acc += sth[OW2 + o * NH + i] * h1[i];
            a2[o] = acc;
            out += sth[OW3 + o] * gelu(acc);
        }
        const float c = softplus(out);
        const float r = c - ys[q];
        lsum = r * r;
        const float g_o = 2.0f * r / (float)n * sigmoid(out);
        atomicAdd(&sg[OB3], g_o);
        float g_h1[NH];
        for (int i = 0; i < NH; i++) g_h1[i] = 0.0f;
        for (int o = 0; o < NH; o++) {
            atomicAdd(&sg[OW3 + o], g_o * gelu(a2[o]));
            const float g_a2 = g_o * sth[OW3 + o] * gelu_grad(a2[o]);
            atomicAdd(&sg[OB2 + o], g_a2);
            for (int i = 0; i < NH; i++) {
                atomicAdd(&sg[OW2 + o * NH + i], g_a2 * h1[i]);
                g_h1[i] += g_a2 * sth[OW2 + o * NH + i];
            }
        }
        for (int o = 0; o < NH; o++) {
            const float g_a1 = g_h1[o] * gelu_grad(a1[o]);
            atomicAdd(&sg[OB1 + o], g_a1);
#pragma unroll
            for (int i = 0; i < NIN; i++) atomicAdd(&sg[OW1 + o * NIN + i], g_a1 * x[i]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0) sloss[threadIdx.x >> 5] = lsum;
    __syncthreads();
    for (int t = threadIdx.x; t < NPARAM; t += blockDim.x) atomicAdd(&grad[t], sg[t]);
    if (threadIdx.x == 0) {
        float b = 0.0f;
        for (int w = 0; w < kTrainThreads / 32; w++) b += sloss[w];
        atomicAdd(loss, (double)b / (double)n);
    }
}

__global__ void k_adam(float *theta, float *m, float *v, const float *g, int np, float lr, float b1, float b2,
                       float eps, float c1, float c2)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.0f - b1) * gt;
    const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    theta[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

}  // namespace

int closure_param_count() { return NTOTAL; }

template <class R, bool FEAT> cudaError_t closure_tc_attr()
{
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_closure_coef_tc<R, FEAT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSmemTc);
        if (e) return e;
        attr = true;
    }
    return cudaSuccess;
}

unsigned closure_tc_blocks(size_t n)
{
    const size_t tiles = (n + 127) / 128;
    return (unsigned)(tiles < 148 * 4 ? tiles : 148 * 4);
}

template <class R>
cudaError_t launch_closure_coef_tc(const R *X, const Geom &g, double dx, double dy, const float *theta, R *coef,
                                   int *err, cudaStream_t s, int wait_limit)
{
    cudaError_t e = closure_tc_attr<R, false>();
    if (e) return e;
    k_closure_coef_tc<R, false><<<closure_tc_blocks((size_t)g.N), kTcThreads, kSmemTc, s>>>(
        X, g, dx, dy, nullptr, 0, theta, coef, err, wait_limit);
    return cudaGetLastError();
}
template cudaError_t launch_closure_coef_tc<float>(const float *, const Geom &, double, double, const float *, float *,
                                                   int *, cudaStream_t, int);
template cudaError_t launch_closure_coef_tc<double>(const double *, const Geom &, double, double, const float *,
                                                    double *, int *, cudaStream_t, int);

cudaError_t launch_closure_predict(const float *theta, const float *feat, size_t n, float *out, int *err,
                                   cudaStream_t s, int wait_limit)
{
    cudaError_t e = closure_tc_attr<float, true>();
    if (e) return e;
    Geom g;
    memset(&g, 0, sizeof(g));
    k_closure_coef_tc<float, true><<<closure_tc_blocks(n), kTcThreads, kSmemTc, s>>>(nullptr, g, 1.0, 1.0, feat, n,
                                                                                      theta, out, err, wait_limit);
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float *theta, const float *xs, const float *ys, const int *idx, int n, float *grad,
                            double *loss, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(grad, 0, sizeof(float) * NPARAM, s);
    if (!e) e = cudaMemsetAsync(loss, 0, sizeof(double), s);
    if (e) return e;
    k_mlp_grad<<<(n + kTrainThreads - 1) / kTrainThreads, kTrainThreads, 0, s>>>(theta, xs, ys, idx, n, grad, loss);
    return cudaGetLastError();
}

cudaError_t launch_adam(float *theta, float *m, float *v, const float *g, int step, float lr, cudaStream_t s)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    k_adam<<<(NPARAM + 255) / 256, 256, 0, s>>>(theta, m, v, g, NPARAM, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}

}  // namespace wf
