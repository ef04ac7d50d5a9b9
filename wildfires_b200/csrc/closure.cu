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
//   k_closure_coef  inference for every cell of a stage input: BF16 weights
//                   and activations on the tensor cores (mma.sync m16n8k16,
//                   FP32 accumulation), 32 cells per warp.  The stage kernel
//                   reads the coefficient in place of C_s^2.
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
__device__ __forceinline__ float softplus(float x) { return x > 20.0f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

__device__ __forceinline__ int wrap1(int v, int n)
{
    if (v >= n) v -= n;
    if (v < 0) v += n;
    return v;
}

// ---- inference ---------------------------------------------------------------
// Shared memory (bytes): W1 as [64][24] bf16 (k padded 12 -> 16, row stride
// 24 for conflict-free fragment loads), W2 [64][72] bf16, W3, b1, b2, b3,
// scales (fp32), and per warp a 32 x 24 bf16 feature tile.
constexpr int W1S = 24, W2S = 72, XS = 24;
constexpr int kClosureThreads = 256;
constexpr size_t kSmemW1 = 0;
constexpr size_t kSmemW2 = kSmemW1 + sizeof(__nv_bfloat16) * NH * W1S;
constexpr size_t kSmemF = kSmemW2 + sizeof(__nv_bfloat16) * NH * W2S;
constexpr size_t kSmemX = kSmemF + sizeof(float) * (NH + NH + NH + 1 + NIN + 3);
constexpr size_t kSmemClosure = kSmemX + sizeof(__nv_bfloat16) * (kClosureThreads / 32) * 32 * XS;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x = lo (lower 16 bits)
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// The 12 raw features at cell (i, j, k) of the state X (walls: zero).
template <class R>
__device__ void cell_features(const R *__restrict__ X, const Geom &g, double dx, double dy, int i, int j, int k,
                              float (&f)[NIN])
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
    const double *z = g.z;
    const float hx = (float)(0.5 / dx), hy = (float)(0.5 / dy);
    const float hz = (float)(1.0 / (z[k + 1] - z[k - 1]));
    float d[4][3];   // d[field][x, y, z]
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const R *F = X + q * N;
        d[q][0] = ((float)F[cxp] - (float)F[cxm]) * hx;
        d[q][1] = ((float)F[cyp] - (float)F[cym]) * hy;
        d[q][2] = ((float)F[c + 1] - (float)F[c - 1]) * hz;
    }
    const float delta = (float)cbrt(dx * dy * g.zc[ZDZ * Nz + k]);
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

template <class R>
__global__ void __launch_bounds__(kClosureThreads) k_closure_coef(const R *__restrict__ X, Geom g, double dx,
                                                                  double dy, const float *__restrict__ theta,
                                                                  R *__restrict__ coef)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16 *sW1 = reinterpret_cast<__nv_bfloat16 *>(smem + kSmemW1);
    __nv_bfloat16 *sW2 = reinterpret_cast<__nv_bfloat16 *>(smem + kSmemW2);
    float *sb1 = reinterpret_cast<float *>(smem + kSmemF), *sb2 = sb1 + NH, *sW3 = sb2 + NH, *sb3 = sW3 + NH;
    float *sscale = sb3 + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16 *sX = reinterpret_cast<__nv_bfloat16 *>(smem + kSmemX) + warp * 32 * XS;
    for (int t = threadIdx.x; t < NH * W1S; t += blockDim.x) {
        const int n = t / W1S, kk = t % W1S;
        sW1[t] = __float2bfloat16(kk < NIN ? theta[OW1 + n * NIN + kk] : 0.0f);
    }
    for (int t = threadIdx.x; t < NH * W2S; t += blockDim.x) {
        const int n = t / W2S, kk = t % W2S;
        sW2[t] = __float2bfloat16(kk < NH ? theta[OW2 + n * NH + kk] : 0.0f);
    }
    for (int t = threadIdx.x; t < NH; t += blockDim.x) {
        sb1[t] = theta[OB1 + t];
        sb2[t] = theta[OB2 + t];
        sW3[t] = theta[OW3 + t];
    }
    if (threadIdx.x == 0) sb3[0] = theta[OB3];
    if (threadIdx.x < NIN) sscale[threadIdx.x] = theta[NPARAM + threadIdx.x];
    __syncthreads();

    const int gid = lane >> 2, tig = lane & 3;
    const size_t N = (size_t)g.N;
    const size_t ngroups = (N + 31) / 32;
    for (size_t grp = blockIdx.x * (size_t)(blockDim.x / 32) + warp; grp < ngroups;
         grp += (size_t)gridDim.x * (blockDim.x / 32)) {
        // features of cell grp*32 + lane -> row `lane` of the warp's tile
        const size_t cell = grp * 32 + lane;
        float f[NIN];
        if (cell < N) {
            const int k = (int)(cell % g.Nz), j = (int)((cell / g.Nz) % g.Ny), i = (int)(cell / ((size_t)g.Nz * g.Ny));
            cell_features(X, g, dx, dy, i, j, k, f);
        } else {
#pragma unroll
            for (int q = 0; q < NIN; q++) f[q] = 0.0f;
        }
#pragma unroll
        for (int q = 0; q < NIN; q += 2)
            *reinterpret_cast<uint32_t *>(&sX[lane * XS + q]) = pack_bf16(f[q] * sscale[q], f[q + 1] * sscale[q + 1]);
        *reinterpret_cast<uint32_t *>(&sX[lane * XS + 12]) = 0u;
        *reinterpret_cast<uint32_t *>(&sX[lane * XS + 14]) = 0u;
        __syncwarp();
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const __nv_bfloat16 *A = sX + half * 16 * XS;
            const uint32_t a0 = *reinterpret_cast<const uint32_t *>(&A[gid * XS + 2 * tig]);
            const uint32_t a1 = *reinterpret_cast<const uint32_t *>(&A[(gid + 8) * XS + 2 * tig]);
            const uint32_t a2 = *reinterpret_cast<const uint32_t *>(&A[gid * XS + 2 * tig + 8]);
            const uint32_t a3 = *reinterpret_cast<const uint32_t *>(&A[(gid + 8) * XS + 2 * tig + 8]);
            // layer 1: 16 x 64 = A (16 x 16) W1^T
            float h[8][4];
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                h[nt][0] = h[nt][1] = h[nt][2] = h[nt][3] = 0.0f;
                const __nv_bfloat16 *Brow = sW1 + (8 * nt + gid) * W1S;
                mma_bf16(h[nt], a0, a1, a2, a3, *reinterpret_cast<const uint32_t *>(&Brow[2 * tig]),
                         *reinterpret_cast<const uint32_t *>(&Brow[2 * tig + 8]));
                const int n0 = 8 * nt + 2 * tig;
                h[nt][0] = gelu(h[nt][0] + sb1[n0]);
                h[nt][1] = gelu(h[nt][1] + sb1[n0 + 1]);
                h[nt][2] = gelu(h[nt][2] + sb1[n0]);
                h[nt][3] = gelu(h[nt][3] + sb1[n0 + 1]);
            }
            // layer 2: the layer-1 accumulators are the A fragments (k-step s = n-tiles 2s, 2s+1)
            float o[8][4];
#pragma unroll
            for (int nt = 0; nt < 8; nt++) o[nt][0] = o[nt][1] = o[nt][2] = o[nt][3] = 0.0f;
#pragma unroll
            for (int s = 0; s < 4; s++) {
                const uint32_t b0 = pack_bf16(h[2 * s][0], h[2 * s][1]), b1 = pack_bf16(h[2 * s][2], h[2 * s][3]);
                const uint32_t b2 = pack_bf16(h[2 * s + 1][0], h[2 * s + 1][1]);
                const uint32_t b3 = pack_bf16(h[2 * s + 1][2], h[2 * s + 1][3]);
#pragma unroll
                for (int nt = 0; nt < 8; nt++) {
                    const __nv_bfloat16 *Brow = sW2 + (8 * nt + gid) * W2S + 16 * s;
                    mma_bf16(o[nt], b0, b1, b2, b3, *reinterpret_cast<const uint32_t *>(&Brow[2 * tig]),
                             *reinterpret_cast<const uint32_t *>(&Brow[2 * tig + 8]));
                }
            }
            // layer 3: per-row dot with W3 over this thread's 16 columns, then the 4 threads of the row
            float r0 = 0.0f, r1 = 0.0f;
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const int n0 = 8 * nt + 2 * tig;
                r0 += gelu(o[nt][0] + sb2[n0]) * sW3[n0] + gelu(o[nt][1] + sb2[n0 + 1]) * sW3[n0 + 1];
                r1 += gelu(o[nt][2] + sb2[n0]) * sW3[n0] + gelu(o[nt][3] + sb2[n0 + 1]) * sW3[n0 + 1];
            }
            r0 += __shfl_xor_sync(0xffffffffu, r0, 1);
            r0 += __shfl_xor_sync(0xffffffffu, r0, 2);
            r1 += __shfl_xor_sync(0xffffffffu, r1, 1);
            r1 += __shfl_xor_sync(0xffffffffu, r1, 2);
            if (tig == 0) {
                const size_t c0 = grp * 32 + half * 16 + gid, c1 = c0 + 8;
                if (c0 < N) coef[c0] = (R)softplus(r0 + sb3[0]);
                if (c1 < N) coef[c1] = (R)softplus(r1 + sb3[0]);
            }
        }
        __syncwarp();
    }
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

template <class R>
cudaError_t launch_closure_coef(const R *X, const Geom &g, double dx, double dy, const float *theta, R *coef,
                                cudaStream_t s)
{
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_closure_coef<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kSmemClosure);
        if (e) return e;
        attr = true;
    }
    const size_t groups = ((size_t)g.N + 31) / 32;
    size_t blocks = (groups + (kClosureThreads / 32) - 1) / (kClosureThreads / 32);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_closure_coef<R><<<(unsigned)blocks, kClosureThreads, kSmemClosure, s>>>(X, g, dx, dy, theta, coef);
    return cudaGetLastError();
}
template cudaError_t launch_closure_coef<float>(const float *, const Geom &, double, double, const float *, float *,
                                                cudaStream_t);
template cudaError_t launch_closure_coef<double>(const double *, const Geom &, double, double, const float *,
                                                 double *, cudaStream_t);

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
