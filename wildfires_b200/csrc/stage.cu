// stage.cu -- one RK stage of the coupled atmosphere-wildfire model on sm_100a.
//
// A stage evaluates k_s = Phi(X_s) (reference src/cu/pde.cu:910-917: RHS,
// Smagorinsky SGS terms, boundary/IBM rules) and folds the RK combination into
// the same pass (reference solver.cu:14-93, utils.cu:14-21), so no k-buffer is
// ever stored:
//   k_utau        : per column, wall friction velocity from the k = 0 plane;
//   k_stage_fused : per tile of cells in shared memory, the SGS inputs on the
//                   tile and its halo, then advection + diffusion + forces +
//                   reaction + SGS divergence and the acc / X_{s+1} updates of
//                   every cell the boundary rules do not overwrite;
//   k_stage_bc    : per column, the boundary/IBM values of k_s (cut node, top,
//                   dead nodes) and their RK updates.
// The right-hand side of cells on the walls (k = 0, k = Nz-1) and below the
// cut node is never used by the reference (boundary_conditions overwrites it,
// pde.cu:58-97), so the fused pass evaluates interior stencils only.
// Arithmetic follows the reference expression by expression; divisions by
// grid constants are folded into precomputed weights (ZCoef, KRow).
#include <cuda.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "stage_common.cuh"

namespace wf {

namespace {

// ---------------------------------------------------------------------------
// wall friction velocity of every column from its k = 0 plane
// (pde.cu:767-772: tau_w = sqrt((mu uz)^2 + (mu vz)^2), u_tau = sqrt(tau_w/rho))
template <class R>
__global__ void __launch_bounds__(128) k_utau(const StageArgs<R> a)
{
    const Geom &g = a.g;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= g.Nx * g.Ny) return;
    const int Nz = g.Nz, N = g.N;
    const R *X = a.X + (size_t)col * Nz;
    const R w0 = (R)g.zc[ZF0 * Nz], w1 = (R)g.zc[ZF1 * Nz], w2 = (R)g.zc[ZF2 * Nz];
    const R uz = w0 * X[0] + w1 * X[1] + w2 * X[2];
    const R vz = w0 * X[N] + w1 * X[N + 1] + w2 * X[N + 2];
    const R T = X[3 * (size_t)N];
    const R rho = fdiv(a.pr.Trho, T);
    R mu = a.pr.mu;
    if (a.ph.sutherland_viscosity == 1)
        mu = R(1.716e-5) * rpow(T / R(273.15), R(1.5)) * (R(273.15) + R(110.4)) / (T + R(110.4));
    const R a1 = mu * uz, a2 = mu * vz;
    const R tau_w = rsqrt_(a1 * a1 + a2 * a2);
    a.utau[col] = rsqrt_(fdiv(tau_w, rho));
}

// Shared-memory tile of one stage: TI x TJ x KZ cells, state halo 2 (4 fields)
// and SGS-input halo 1 (8 fields).  Offsets are relative to the tile origin;
// (ii, jj, kk) in [-2, T+1] for the state and [-1, T] for the rest.  Both
// arrays are stored j-fastest with a row stride of TJ+4: a warp covering
// 8 consecutive k x 4 consecutive j then touches 32 distinct banks (FP32).
// In FP32 the state is stored as two arrays of pairs, (u, v) and (w, T), so
// one 8-byte load brings two fields and the pair arithmetic runs on FFMA2;
// each half-warp (4 k x 4 j) of an 8-byte load then covers the 16 bank pairs.
// The fuel fraction is read from global memory where a column has fuel.
template <class R, int TI, int TJ, int KZ> struct Tile {
    static constexpr int SI = TI + 4, SJ = TJ + 4, SK = KZ + 4, SR = SI * SJ * SK;
    static constexpr int GI = TI + 2, GJ = TJ + 2, GK = KZ + 2, GJP = SJ, GR = GI * GK * GJP;
    static constexpr bool PAIRED = sizeof(R) == 4;
    static constexpr int NCOL = GI * GJ, CELLS = TI * TJ * KZ;
    static constexpr size_t up16(size_t b) { return (b + 15) / 16 * 16; }
    static constexpr size_t O_KR = up16(sizeof(R) * 4 * (size_t)SR);
    static constexpr size_t O_TOPO = O_KR + up16(sizeof(R) * (size_t)GK * KROW);
    static constexpr size_t O_UT = O_TOPO + up16(sizeof(double) * (size_t)NCOL);
    static constexpr size_t O_NZY = O_UT + up16(sizeof(R) * (size_t)NCOL);
    static constexpr size_t O_CUT = O_NZY + up16(sizeof(int) * (size_t)NCOL);
    static constexpr size_t O_MISC = O_CUT + up16(sizeof(int) * (size_t)NCOL);   // mbarrier, flags
    // the SGS buffer doubles as the staging area of the TMA box (512-byte aligned: 64-byte swizzle)
    static constexpr size_t BUF = (O_MISC + 32 + 1023) / 1024 * 1024;
    static constexpr size_t BOX = sizeof(float) * 4 * (size_t)SI * SJ * 16;   // one box, FP32 path
    static constexpr size_t bytes() { return BUF + up16(sizeof(R) * 8 * (size_t)GR); }
    R *st;         // [4][SR]  u, v, w, T
    R *kr;         // [GK][KROW] z-stencil rows for k0-1 .. k0+KZ
    double *ctopo; // [NCOL]   terrain height of the halo-1 columns
    R *cut_;       // [NCOL]   wall friction velocity of the halo-1 columns
    int *cnzy, *ccut;
    R *gs;         // [8][GR]  mu_sgs, S11, S12, S13, S22, S23, S33, divU (shared by both buffers)
    __device__ void bind(unsigned char *buf, R *sgs)
    {
        st = reinterpret_cast<R *>(buf);
        kr = reinterpret_cast<R *>(buf + O_KR);
        ctopo = reinterpret_cast<double *>(buf + O_TOPO);
        cut_ = reinterpret_cast<R *>(buf + O_UT);
        cnzy = reinterpret_cast<int *>(buf + O_NZY);
        ccut = reinterpret_cast<int *>(buf + O_CUT);
        gs = sgs;
    }
    __device__ static int s(int ii, int jj, int kk) { return ((ii + 2) * SK + (kk + 2)) * SJ + (jj + 2); }
    __device__ static int q(int ii, int jj, int kk) { return ((ii + 1) * GK + (kk + 1)) * GJP + (jj + 1); }
    __device__ static int cq(int ii, int jj) { return (ii + 1) * GJ + (jj + 1); }
    // position of field f at tile offset sidx: pairs (u, v), (w, T) in FP32, planar in FP64
    __device__ static int so(int f, int sidx) { return PAIRED ? (f >> 1) * 2 * SR + 2 * sidx + (f & 1) : f * SR + sidx; }
    __device__ R &S(int f, int ii, int jj, int kk) { return st[so(f, s(ii, jj, kk))]; }
    // pair pr (0: u, v; 1: w, T), FP32 only
    __device__ float2 P(int pr, int ii, int jj, int kk) const
    {
        return reinterpret_cast<const float2 *>(st)[pr * SR + s(ii, jj, kk)];
    }
    __device__ R &G(int f, int ii, int jj, int kk) { return gs[f * GR + q(ii, jj, kk)]; }
    __device__ R K(int kk, int e) const { return kr[(kk + 1) * KROW + e]; }
};

// Asynchronous global -> shared copies (cp.async, sm_80+ PTX).  src_bytes 0
// writes zeros without reading, which gives the tile its zero halo in z.
template <int B>
__device__ __forceinline__ void cp_async(void *dst, const void *src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(d), "l"(src), "n"(B), "r"(valid ? B : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Issue the copies of one tile's inputs into buffer t (one commit group).
// Periodic in x and y (period N-1), zero outside 0..Nz-1 in z.
template <class R, class TL, int NT>
__device__ __forceinline__ void issue_tile(const StageArgs<R> &a, TL &t, int i0, int j0, int k0, bool state)
{
    const Geom &g = a.g;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const R *__restrict__ X = a.X;
    for (int c = threadIdx.x; c < TL::NCOL; c += NT) {
        const int jj = c % TL::GJ - 1, ii = c / TL::GJ - 1;
        const int gi = i0 + ii, gj = j0 + jj;
        const bool ok = gi <= Nx && gj <= Ny;
        const int col = ok ? wrap_p(gi, Nx - 1) * Ny + wrap_p(gj, Ny - 1) : 0;
        cp_async<8>(t.ctopo + c, g.topo + col, ok);
        cp_async<sizeof(R)>(t.cut_ + c, a.utau + col, ok);
        cp_async<4>(t.cnzy + c, g.nzy + col, ok);
        cp_async<4>(t.ccut + c, g.cut + col, ok);
    }
    for (int c = threadIdx.x; c < TL::GK * KROW; c += NT) {
        const int gk = k0 - 1 + c / KROW;
        const bool ok = gk >= 0 && gk < Nz;
        cp_async<sizeof(R)>(t.kr + c, a.krow + (ok ? (size_t)gk * KROW + c % KROW : 0), ok);
    }
    if (!state) {
        // the stage input arrives as a TMA box (see k_stage_fused)
    } else if constexpr (TL::PAIRED && TL::SK * TL::SJ <= NT) {
        // FP32 tile: thread (k, j) of the SK x SJ cross-section walks the SI
        // planes in i, so the k/j arithmetic and the j wrap happen once per
        // thread (lanes k fastest: global reads stay coalesced along k).  With
        // twice the threads, two threads share a (k, j), half the planes each.
        constexpr int KJ = TL::SK * TL::SJ, NSPLIT = (NT >= 2 * KJ && TL::SI % 2 == 0) ? 2 : 1;
        if (threadIdx.x < KJ * NSPLIT) {
            const int kj = threadIdx.x % KJ, part = threadIdx.x / KJ;
            const int kk = kj % TL::SK - 2, jj = kj / TL::SK - 2;
            const int gk = k0 + kk, gj = j0 + jj;
            const bool okjk = gk >= 0 && gk < Nz && gj <= Ny + 1;
            const size_t cj = okjk ? (size_t)wrap_p(gj, Ny - 1) * Nz + gk : 0;
            const size_t plane = (size_t)Ny * Nz;
            const int ii0 = -2 + part * (TL::SI / NSPLIT);
#pragma unroll 2
            for (int ii = ii0; ii < ii0 + TL::SI / NSPLIT; ii++) {
                const int gi = i0 + ii;
                const bool ok = okjk && gi <= Nx + 1;
                const size_t o = ok ? (size_t)wrap_p(gi, Nx - 1) * plane + cj : 0;
                const int sidx = TL::s(ii, jj, kk);
#pragma unroll
                for (int f = 0; f < 4; f++) cp_async<sizeof(R)>(t.st + TL::so(f, sidx), X + (size_t)f * N + o, ok);
            }
        }
    } else {
        for (int c = threadIdx.x; c < TL::SR; c += NT) {
            const int kk = c % TL::SK - 2, jj = (c / TL::SK) % TL::SJ - 2, ii = c / (TL::SK * TL::SJ) - 2;
            const int gk = k0 + kk;
            const bool ok = gk >= 0 && gk < Nz && i0 + ii <= Nx + 1 && j0 + jj <= Ny + 1;
            const size_t o = ok ? ((size_t)wrap_p(i0 + ii, Nx - 1) * Ny + wrap_p(j0 + jj, Ny - 1)) * Nz + gk : 0;
#pragma unroll
            for (int f = 0; f < 4; f++)
                cp_async<sizeof(R)>(t.st + TL::so(f, TL::s(ii, jj, kk)), X + (size_t)f * N + o, ok);
        }
    }
    cp_async_commit();
}

// Bounded wait on an mbarrier phase (false when the limit ran out).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit)
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
constexpr int kTmaWaitLimit = 1 << 20;   // polls before a tile load is given up (about a second)

// FP32 tile from the TMA box: the box holds u, v, w, T (outermost) x SI x SJ
// columns x 16 planes (k0-4 .. k0+11), one 64-byte row per column with the
// 64-byte swizzle (16-byte chunk c of row r at chunk c ^ ((r >> 1) & 3)), so
// the four chunk loads of consecutive columns hit distinct banks.  One thread
// per (pair, column) writes the column's planes k0-2 .. k0+9 as (u, v) or
// (w, T) pairs into the tile.
template <class TL, int NT>
__device__ __forceinline__ void repack_box(TL &t, const unsigned char *stg)
{
    for (int c = threadIdx.x; c < 2 * TL::SI * TL::SJ; c += NT) {
        const int jj = c % TL::SJ, r = c / TL::SJ, ii = r % TL::SI, pr = r / TL::SI;
        const int ra = ((2 * pr) * TL::SI + ii) * TL::SJ + jj, rb = ra + TL::SI * TL::SJ;
        float va[16], vb[16];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float4 x = *reinterpret_cast<const float4 *>(stg + ra * 64 + ((q ^ ((ra >> 1) & 3)) << 4));
            const float4 y = *reinterpret_cast<const float4 *>(stg + rb * 64 + ((q ^ ((rb >> 1) & 3)) << 4));
            va[4 * q] = x.x; va[4 * q + 1] = x.y; va[4 * q + 2] = x.z; va[4 * q + 3] = x.w;
            vb[4 * q] = y.x; vb[4 * q + 1] = y.y; vb[4 * q + 2] = y.z; vb[4 * q + 3] = y.w;
        }
        float2 *dst = reinterpret_cast<float2 *>(t.st) + pr * TL::SR + ii * TL::SK * TL::SJ + jj;
#pragma unroll
        for (int kk = 0; kk < TL::SK; kk++) dst[kk * TL::SJ] = make_float2(va[kk + 2], vb[kk + 2]);
    }
}

// upwind derivative from 5 weights (zero weights leave the sum unchanged)
template <class R> __device__ __forceinline__ R dz5(const R *w, R m2, R m1, R c, R p1, R p2)
{
    return w[0] * m2 + w[1] * m1 + w[2] * c + w[3] * p1 + w[4] * p2;
}

// One RK stage over TI x TJ x KZ tiles (reference RHS pde.cu:139-787,
// turbulence.cu:255-454, RK combination solver.cu:14-93).  One tile per block
// (the grid is the tile count); two blocks per SM in FP32, so one block's tile
// loads overlap the other's arithmetic.  Per tile:
//   1. column tables, z rows, stage input with halo 2 -> shared memory
//      (cp.async; the fuel fraction is read from global memory where needed)
//   2. SGS inputs (raw mu_sgs, strain S', divergence source) on the tile and
//      its halo 1 -> shared memory
//   3. per tile cell: advection, diffusion, forces, reaction, SGS divergence,
//      RK update.  Cells the boundary rules overwrite (k <= cut node, top) are
//      left to k_stage_bc; the values it needs are stored in a.bc.
template <class R, int TI, int TJ, int KZ, int NT>
__global__ void __launch_bounds__(NT, sizeof(R) != 4 ? 1 : NT > 256 ? 2 : (TI * TJ <= 64 ? 3 : 2))
    k_stage_fused(const StageArgs<R> a, const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap pyn,
                  const __grid_constant__ CUtensorMap pacc, int use_tma, int use_pf, int ntk, int ntj, int nti)
{
    using TL = Tile<R, TI, TJ, KZ>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *sgs = reinterpret_cast<R *>(smem_raw + TL::BUF);
    R *s_vd = reinterpret_cast<R *>(smem_raw + TL::O_MISC);
    int *s_fail = reinterpret_cast<int *>(smem_raw + TL::O_MISC + 8);
    int *s_vd_zero = reinterpret_cast<int *>(smem_raw + TL::O_MISC + 12);
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(smem_raw + TL::O_MISC + 16);
    const Geom &g = a.g;
    const PhysR<R> &p = a.pr;
    const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz, N = g.N;
    const R *__restrict__ X = a.X;
    const int ntiles = ntk * ntj * nti;
    const int tile = blockIdx.x;   // one tile per block
    if (tile >= ntiles) return;
    {
        TL t;
        t.bind(smem_raw, sgs);
        const int k0 = (tile % ntk) * KZ, j0 = ((tile / ntk) % ntj) * TJ, i0 = (tile / (ntk * ntj)) * TI;
        // FP32 tiles whose halo stays inside the stored planes 0..N-2 (no periodic
        // wrap) arrive as one TMA box of u, v, w, T; the others by cp.async
        bool tma = false;
        if constexpr (TL::PAIRED)
            tma = use_tma && i0 >= 2 && i0 + TI + 1 <= Nx - 2 && j0 >= 2 && j0 + TJ + 1 <= Ny - 2 &&
                  (((uint32_t)__cvta_generic_to_shared(sgs)) & 511u) == 0;
        if (threadIdx.x == 0) {
            *s_fail = 0;
            if (tma) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
        }
        __syncthreads();   // barrier initialised before anyone waits on it
        if (tma && threadIdx.x == 0) {
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"((uint32_t)TL::BOX)
                         : "memory");
            asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
                         "[%0], [%1, {%2, %3, %4, %5}], [%6];"
                         :
                         : "r"((uint32_t)__cvta_generic_to_shared(sgs)), "l"(reinterpret_cast<uint64_t>(&tmap)),
                           "r"(k0 - 4), "r"(j0 - 2), "r"(i0 - 2), "r"(0), "r"(bar)
                         : "memory");
        }
        // RK operands of the tile's cells (yn, and acc when this stage reads it)
        // into L2 while the tile loads and phase 2 runs: phase 3 then finds
        // them there instead of waiting on DRAM.  A prefetch has no completion
        // to wait for and ignores coordinates outside the buffer.
        if (use_pf && threadIdx.x == 32) {
            asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];"
                         :
                         : "l"(reinterpret_cast<uint64_t>(&pyn)), "r"(k0), "r"(j0), "r"(i0), "r"(0)
                         : "memory");
            if (stage_reads_acc(a.method, a.stage))
                asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];"
                             :
                             : "l"(reinterpret_cast<uint64_t>(&pacc)), "r"(k0), "r"(j0), "r"(i0), "r"(0)
                             : "memory");
        }
        issue_tile<R, TL, NT>(a, t, i0, j0, k0, !tma);
        cp_async_wait<0>();
        if (tma) {
            if (!mbar_wait(bar, 0, kTmaWaitLimit)) *s_fail = 1;
            else repack_box<TL, NT>(t, reinterpret_cast<const unsigned char *>(sgs));
        }
        __syncthreads();
        if (*s_fail) {
            // the box did not arrive in time: flag it, give the copy a bounded
            // chance to land (it writes this block's shared memory), leave the tile
            if (threadIdx.x == 0) {
                if (a.kerr) atomicExch(a.kerr, 1);
                mbar_wait(bar, 0, kTmaWaitLimit);
            }
            __syncthreads();
            return;
        }

        const int smu = a.ph.sutherland_viscosity, sk = a.ph.sutherland_conductivity;
        // FP32 path without Sutherland laws or convective exchange: the
        // divergence source nu T_RHS / T reduces to mu/(T_inf rho_inf) T_RHS
        const bool lean = sizeof(R) == 4 && smu != 1 && sk != 1 && !(p.alpha_s * p.sigma_s != R(0));

        // Lower bound over the tile of z_ibm u_tau / A_vd, taken over the
        // columns with wall friction: when it exceeds the cut-off times nu,
        // every Van Driest factor of those columns is exactly 1, and every
        // factor of a column without friction (u_tau = 0, as over the hills)
        // is 1 - exp(-0) = 0 at any height.
        R &s_vd_bound = *s_vd;
        if (threadIdx.x < 32) {
            const R zlow = (k0 > 0) ? t.K(-1, RZ) : R(0);
            R hmax = R(-1e30), umin = R(1e30);
            bool zero = false;
            for (int c = threadIdx.x; c < TL::NCOL; c += 32) {
                const R ut = t.cut_[c];
                if (ut == R(0)) {
                    zero = true;
                } else {
                    hmax = rmax(hmax, (R)t.ctopo[c]);
                    umin = rmin(umin, ut);
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                hmax = rmax(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
                umin = rmin(umin, __shfl_xor_sync(0xffffffffu, umin, o));
            }
            zero = __any_sync(0xffffffffu, zero);
            if (threadIdx.x == 0) {
                s_vd_bound = rmax(zlow - hmax, R(0)) * rmax(umin, R(0)) * p.inv_avd;
                *s_vd_zero = zero;
            }
        }

        // ---- 2. SGS inputs on the tile and its halo 1 (pde.cu:632-765).  Needed
        //        set: tile columns on k0-1 .. k0+KZ, side columns on k0 .. k0+KZ-1.
        //        Enumerated so that each warp covers 8 consecutive k x 4 j where
        //        it can: tile columns k0-1..k0+6, tile columns k0+7..k0+8,
        //        x-side columns, y-side columns.
        //        In the 8-plane groups the lanes of a warp are 4 j (fastest) x 8 k.
        static_assert(KZ == 8 && TJ % 4 == 0 && NT % 32 == 0, "phase-2/3 enumeration: 8 planes, 4-column lane groups");
        constexpr int NA1 = TI * TJ * 8, NA2 = TI * TJ * 2, NB = 2 * TJ * KZ, NC = TI * 2 * KZ;
        static_assert(NA1 % 32 == 0 && NA2 % 32 == 0, "warp-aligned groups");
        for (int c = threadIdx.x; c < NA1 + NA2 + NB + NC; c += NT) {
            int ii, jj, kk;
            if (c < NA1) {
                kk = ((c & 31) >> 2) - 1;
                jj = ((c >> 5) % (TJ / 4)) * 4 + (c & 3);
                ii = (c >> 5) / (TJ / 4);
            } else if (c < NA1 + NA2) {
                const int d = c - NA1;
                jj = d % TJ;
                kk = 7 + (d / TJ) % 2;
                ii = d / (2 * TJ);
            } else if (c < NA1 + NA2 + NB) {
                const int d = c - NA1 - NA2;
                kk = (d & 31) >> 2;
                jj = ((d >> 5) % (TJ / 4)) * 4 + (d & 3);
                ii = ((d >> 5) / (TJ / 4)) ? TI : -1;
            } else {
                const int d = c - NA1 - NA2 - NB;
                kk = d % KZ;
                jj = ((d / KZ) % 2) ? TJ : -1;
                ii = d / (2 * KZ);
            }
            const int gk = k0 + kk;
            if (gk < 0 || gk >= Nz || i0 + ii > Nx || j0 + jj > Ny) continue;
            R ux, uy, uz, vx, vy, vz, wx, wy, wz, Tc, Tx, Ty, Tz, Txx, Tyy, Tzz;
            bool zdone = false;
            if constexpr (TL::PAIRED) {
                const float2 UVxp = t.P(0, ii + 1, jj, kk), UVxm = t.P(0, ii - 1, jj, kk);
                const float2 UVyp = t.P(0, ii, jj + 1, kk), UVym = t.P(0, ii, jj - 1, kk);
                const float2 WTxp = t.P(1, ii + 1, jj, kk), WTxm = t.P(1, ii - 1, jj, kk);
                const float2 WTyp = t.P(1, ii, jj + 1, kk), WTym = t.P(1, ii, jj - 1, kk);
                const float2 i2x = bcast(p.inv2dx), i2y = bcast(p.inv2dy);
                const float2 dUVx = mul2(sub2(UVxp, UVxm), i2x), dUVy = mul2(sub2(UVyp, UVym), i2y);
                const float2 dWTx = mul2(sub2(WTxp, WTxm), i2x), dWTy = mul2(sub2(WTyp, WTym), i2y);
                ux = dUVx.x; vx = dUVx.y; wx = dWTx.x; Tx = dWTx.y;
                uy = dUVy.x; vy = dUVy.y; wy = dWTy.x; Ty = dWTy.y;
                Tc = t.P(1, ii, jj, kk).y;
                Txx = (WTxp.y - R(2) * Tc + WTxm.y) * p.invdx2;
                Tyy = (WTyp.y - R(2) * Tc + WTym.y) * p.invdy2;
                if (gk > 0 && gk < Nz - 1) {
                    const float2 UVzp = t.P(0, ii, jj, kk + 1), UVzm = t.P(0, ii, jj, kk - 1);
                    const float2 WTzp = t.P(1, ii, jj, kk + 1), WTzm = t.P(1, ii, jj, kk - 1);
                    const float2 wc = bcast(t.K(kk, RD1));
                    const float2 dUVz = mul2(sub2(UVzp, UVzm), wc), dWTz = mul2(sub2(WTzp, WTzm), wc);
                    uz = dUVz.x; vz = dUVz.y; wz = dWTz.x; Tz = dWTz.y;
                    Tzz = t.K(kk, RD2) * WTzm.y + t.K(kk, RD2 + 1) * Tc + t.K(kk, RD2 + 2) * WTzp.y;
                    zdone = true;
                }
            } else {
                Tc = t.S(3, ii, jj, kk);
                ux = (t.S(0, ii + 1, jj, kk) - t.S(0, ii - 1, jj, kk)) * p.inv2dx;
                uy = (t.S(0, ii, jj + 1, kk) - t.S(0, ii, jj - 1, kk)) * p.inv2dy;
                vx = (t.S(1, ii + 1, jj, kk) - t.S(1, ii - 1, jj, kk)) * p.inv2dx;
                vy = (t.S(1, ii, jj + 1, kk) - t.S(1, ii, jj - 1, kk)) * p.inv2dy;
                wx = (t.S(2, ii + 1, jj, kk) - t.S(2, ii - 1, jj, kk)) * p.inv2dx;
                wy = (t.S(2, ii, jj + 1, kk) - t.S(2, ii, jj - 1, kk)) * p.inv2dy;
                const R Txp = t.S(3, ii + 1, jj, kk), Txm = t.S(3, ii - 1, jj, kk);
                const R Typ = t.S(3, ii, jj + 1, kk), Tym = t.S(3, ii, jj - 1, kk);
                Tx = (Txp - Txm) * p.inv2dx;
                Ty = (Typ - Tym) * p.inv2dy;
                Txx = (Txp - R(2) * Tc + Txm) * p.invdx2;
                Tyy = (Typ - R(2) * Tc + Tym) * p.invdy2;
                if (gk > 0 && gk < Nz - 1) {
                    const R wc = t.K(kk, RD1);
                    uz = (t.S(0, ii, jj, kk + 1) - t.S(0, ii, jj, kk - 1)) * wc;
                    vz = (t.S(1, ii, jj, kk + 1) - t.S(1, ii, jj, kk - 1)) * wc;
                    wz = (t.S(2, ii, jj, kk + 1) - t.S(2, ii, jj, kk - 1)) * wc;
                    Tz = (t.S(3, ii, jj, kk + 1) - t.S(3, ii, jj, kk - 1)) * wc;
                    Tzz = t.K(kk, RD2) * t.S(3, ii, jj, kk - 1) + t.K(kk, RD2 + 1) * Tc + t.K(kk, RD2 + 2) * t.S(3, ii, jj, kk + 1);
                    zdone = true;
                }
            }
            if (!zdone) {
                // walls: one-sided stencils from the double table (planes k = 0 and Nz-1 only)
                const double *zc = g.zc;
                const bool bot = (gk == 0);
                auto d1 = [&](int f) -> R {
                    if (bot)
                        return (R)zc[ZF0 * Nz] * t.S(f, ii, jj, kk) + (R)zc[ZF1 * Nz] * t.S(f, ii, jj, kk + 1) +
                               (R)zc[ZF2 * Nz] * t.S(f, ii, jj, kk + 2);
                    return (R)zc[ZB0 * Nz + gk] * t.S(f, ii, jj, kk - 2) + (R)zc[ZB1 * Nz + gk] * t.S(f, ii, jj, kk - 1) +
                           (R)zc[ZB2 * Nz + gk] * t.S(f, ii, jj, kk);
                };
                uz = d1(0);
                vz = d1(1);
                wz = d1(2);
                Tz = d1(3);
                // the backward 4-point form needs k-3, inside the tile unless the
                // top plane is alone in its tile (then no cell of this tile needs it)
                const R m3 = (kk >= 1) ? t.S(3, ii, jj, kk - 3) : R(0), p3 = (kk <= KZ - 2) ? t.S(3, ii, jj, kk + 3) : R(0);
                Tzz = bot ? (R)zc[ZFF0 * Nz] * Tc + (R)zc[ZFF1 * Nz] * t.S(3, ii, jj, kk + 1) +
                                (R)zc[ZFF2 * Nz] * t.S(3, ii, jj, kk + 2) + (R)zc[ZFF3 * Nz] * p3
                          : (R)zc[ZBB0 * Nz + gk] * m3 + (R)zc[ZBB1 * Nz + gk] * t.S(3, ii, jj, kk - 2) +
                                (R)zc[ZBB2 * Nz + gk] * t.S(3, ii, jj, kk - 1) + (R)zc[ZBB3 * Nz + gk] * Tc;
            }
            const R rho = fdiv(p.Trho, Tc);
            const R S11 = third(R(2) * ux) - third(vy + wz);
            const R S22 = third(R(2) * vy) - third(ux + wz);
            const R S33 = third(R(2) * wz) - third(ux + vy);
            const R mod_S = rsqrt_(R(2) * (ux * ux + vy * vy + wz * wz) + (uz + wx) * (uz + wx) + (vx + uy) * (vx + uy) +
                                   (wy + vz) * (wy + vz));
            const int nzy = t.cnzy[TL::cq(ii, jj)];
            // fuel fraction of the stage input (used only below the column's fuel top)
            const R Yq = (gk < nzy) ? X[4 * (size_t)N + (size_t)(wrap_p(i0 + ii, Nx - 1) * Ny + wrap_p(j0 + jj, Ny - 1)) * g.NzY + gk]
                                    : R(0);
            R g7;
            if (lean) {
                const R K_T = arrhenius(p, Tc);
                const R Yv = (gk < nzy) ? Yq : R(0);
                const R T2 = Tc * Tc;
                g7 = p.mu_Trho * ((p.c12 * T2 * (Tx * Tx + Ty * Ty + Tz * Tz) + (p.kT + p.c4 * (T2 * Tc)) * (Txx + Tyy + Tzz)) *
                                      (Tc * p.inv_Trho_cp) +
                                  p.H_C_cp * Yv * K_T);
            } else {
                const Thermo<R> th = thermo(p, smu, sk, Tc, t.S(3, ii, jj, kk + 1), Yq, gk, nzy, Tx, Ty, Tz,
                                            Txx + Tyy + Tzz, t.K(kk, RDZ), rho);
                g7 = fdiv(th.nu * th.T_RHS_tmp, Tc);
            }
            if (a.coef) {
                // learned closure: the coefficient of this point replaces C_s^2
                const R cq = a.coef[((size_t)wrap_p(i0 + ii, Nx - 1) * Ny + wrap_p(j0 + jj, Ny - 1)) * Nz + gk];
                t.G(0, ii, jj, kk) = rho * (t.K(kk, RDD2) * cq) * mod_S;
            } else {
                t.G(0, ii, jj, kk) = rho * t.K(kk, RDEL2) * mod_S;
            }
            t.G(1, ii, jj, kk) = S11;
            t.G(2, ii, jj, kk) = R(0.5) * (uy + vx);
            t.G(3, ii, jj, kk) = R(0.5) * (uz + wx);
            t.G(4, ii, jj, kk) = S22;
            t.G(5, ii, jj, kk) = R(0.5) * (wy + vz);
            t.G(6, ii, jj, kk) = S33;
            t.G(7, ii, jj, kk) = g7;
        }
        __syncthreads();

        // ---- 3. right-hand side, SGS divergence, RK update per tile cell
        const R an = (R)a.a_next;
        const bool rd = stage_reads_acc(a.method, a.stage), kp = stage_keeps_acc(a.method, a.stage);
        for (int c = threadIdx.x; c < TL::CELLS; c += NT) {
            // lanes: 4 j (fastest) x 8 k, as in phase 2
            const int kk = (c & 31) >> 2, jj = ((c >> 5) % (TJ / 4)) * 4 + (c & 3), ii = (c >> 5) / (TJ / 4);
            const int gi = i0 + ii, gj = j0 + jj, gk = k0 + kk;
            if (gi >= Nx || gj >= Ny || gk >= Nz) continue;
            const int col = gi * Ny + gj;
            const int cc = TL::cq(ii, jj);
            const int kc = t.ccut[cc], nzy = t.cnzy[cc];
            const size_t cg = (size_t)col * Nz + gk;
            if (gk < kc) {
                // dead node below the terrain: the boundary rules fix its k-values (pde.cu:88-97)
                const double dv[4] = {a.ph.u_dead, a.ph.v_dead, a.ph.w_dead, a.ph.T_dead};
#pragma unroll
                for (int f = 0; f < 4; f++) rk_cell(a, (size_t)f * N + cg, (R)dv[f], rd, kp, an);
                if (gk < g.NzY)
                    rk_cell(a, 4 * (size_t)N + (size_t)col * g.NzY + gk, (gk < nzy) ? (R)a.ph.Y_dead : R(0), rd, kp, an);
                continue;
            }
            const bool live = (gk > kc) && (gk < Nz - 1);                 // not overwritten by the boundary rules
            const bool ylive = (gk < g.NzY) && !(gk <= kc && gk < nzy);   // fuel value this pass updates
            if (!live && !ylive) continue;
            // start the RK operand loads early
            R ynv[4], accv[4];
            if (live) {
    #pragma unroll
                for (int f = 0; f < 4; f++) {
                    ynv[f] = a.yn[(size_t)f * N + cg];
                    accv[f] = rd ? a.acc[(size_t)f * N + cg] : R(0);
                }
            }
            const size_t oY = 4 * (size_t)N + (size_t)col * g.NzY + gk;
            R ynY = R(0), accY = R(0);
            if (ylive) {
                ynY = a.yn[oY];
                accY = rd ? a.acc[oY] : R(0);
            }
            R kY = R(0);
            // fuel fraction of the stage input (used only below the column's fuel top)
            const R Yx = (gk < nzy) ? X[4 * (size_t)N + (size_t)col * g.NzY + gk] : R(0);
            if (live) {
                const R *kmw = &t.kr[(kk + 1) * KROW + RKM], *kpw = &t.kr[(kk + 1) * KROW + RKP];
                const R d2m = t.K(kk, RD2), d20 = t.K(kk, RD2 + 1), d2p = t.K(kk, RD2 + 2);
                R u, v, w, T;
                R advU, advV, advW, advT, lapU, lapV, lapW, lapT, Tx, Ty, Tz;
                if constexpr (TL::PAIRED) {
                    const float2 UV = t.P(0, ii, jj, kk), WT = t.P(1, ii, jj, kk);
                    u = UV.x; v = UV.y; w = WT.x; T = WT.y;
                    // The upwind advection of a field is a weighted sum of its 13
                    // stencil values and the Laplacian one of 7: with a = max(u,0)/(2dx)
                    // and b = min(u,0)/(2dx), u+ (3f - 4f_{i-1} + f_{i-2})/(2dx) +
                    // u- (-3f + 4f_{i+1} - f_{i+2})/(2dx) has weights 3(a-b), -4a, a, 4b, -b;
                    // in z the two 5-point rows combine as w+ kmw + w- kpw.
                    const R ax = rmax(u, R(0)) * p.inv2dx, bx = rmin(u, R(0)) * p.inv2dx;
                    const R ay = rmax(v, R(0)) * p.inv2dy, by = rmin(v, R(0)) * p.inv2dy;
                    const R wp = rmax(w, R(0)), wm = rmin(w, R(0));
                    const float2 Cxm = bcast(R(-4) * ax), Cxm2 = bcast(ax), Cxp = bcast(R(4) * bx), Cxp2 = bcast(-bx);
                    const float2 Cym = bcast(R(-4) * ay), Cym2 = bcast(ay), Cyp = bcast(R(4) * by), Cyp2 = bcast(-by);
                    const float2 Cz0 = bcast(wp * kmw[0] + wm * kpw[0]), Cz1 = bcast(wp * kmw[1] + wm * kpw[1]);
                    const float2 Cz3 = bcast(wp * kmw[3] + wm * kpw[3]), Cz4 = bcast(wp * kmw[4] + wm * kpw[4]);
                    const float2 C0 = bcast(R(3) * (ax - bx) + R(3) * (ay - by) + (wp * kmw[2] + wm * kpw[2]));
                    const float2 Lx = bcast(p.invdx2), Ly = bcast(p.invdy2), Lzm = bcast(d2m), Lzp = bcast(d2p);
                    const float2 L0 = bcast(d20 - R(2) * p.invdx2 - R(2) * p.invdy2);
                    const float2 i2x = bcast(p.inv2dx), i2y = bcast(p.inv2dy), i2z = bcast(t.K(kk, RD1));
                    auto adv_lap2 = [&](int pr, float2 f0, float2 &adv, float2 &lap, float2 &gx, float2 &gy, float2 &gz) {
                        const float2 xm = t.P(pr, ii - 1, jj, kk), xp = t.P(pr, ii + 1, jj, kk);
                        const float2 xm2 = t.P(pr, ii - 2, jj, kk), xp2 = t.P(pr, ii + 2, jj, kk);
                        const float2 ym = t.P(pr, ii, jj - 1, kk), yp = t.P(pr, ii, jj + 1, kk);
                        const float2 ym2 = t.P(pr, ii, jj - 2, kk), yp2 = t.P(pr, ii, jj + 2, kk);
                        const float2 zm2 = t.P(pr, ii, jj, kk - 2), zm = t.P(pr, ii, jj, kk - 1);
                        const float2 zp = t.P(pr, ii, jj, kk + 1), zp2 = t.P(pr, ii, jj, kk + 2);
                        float2 s0 = mul2(C0, f0);
                        s0 = fma2(Cxm, xm, s0);
                        s0 = fma2(Cxm2, xm2, s0);
                        s0 = fma2(Cxp, xp, s0);
                        s0 = fma2(Cxp2, xp2, s0);
                        s0 = fma2(Cym, ym, s0);
                        s0 = fma2(Cym2, ym2, s0);
                        s0 = fma2(Cyp, yp, s0);
                        s0 = fma2(Cyp2, yp2, s0);
                        s0 = fma2(Cz0, zm2, s0);
                        s0 = fma2(Cz1, zm, s0);
                        s0 = fma2(Cz3, zp, s0);
                        adv = fma2(Cz4, zp2, s0);
                        float2 l0 = mul2(L0, f0);
                        l0 = fma2(Lx, add2(xp, xm), l0);
                        l0 = fma2(Ly, add2(yp, ym), l0);
                        l0 = fma2(Lzm, zm, l0);
                        lap = fma2(Lzp, zp, l0);
                        gx = mul2(sub2(xp, xm), i2x);
                        gy = mul2(sub2(yp, ym), i2y);
                        gz = mul2(sub2(zp, zm), i2z);
                    };
                    float2 aUV, lUV, aWT, lWT, gx, gy, gz;
                    adv_lap2(0, UV, aUV, lUV, gx, gy, gz);
                    adv_lap2(1, WT, aWT, lWT, gx, gy, gz);
                    advU = aUV.x; advV = aUV.y; advW = aWT.x; advT = aWT.y;
                    lapU = lUV.x; lapV = lUV.y; lapW = lWT.x; lapT = lWT.y;
                    Tx = gx.y; Ty = gy.y; Tz = gz.y;
                } else {
                    u = t.S(0, ii, jj, kk); v = t.S(1, ii, jj, kk); w = t.S(2, ii, jj, kk); T = t.S(3, ii, jj, kk);
                    const R u_plu = rmax(u, R(0)), u_min = rmin(u, R(0));
                    const R v_plu = rmax(v, R(0)), v_min = rmin(v, R(0));
                    const R w_plu = rmax(w, R(0)), w_min = rmin(w, R(0));
                    // advection (upwind) and Laplacian of one field from the shared tile
                    auto adv_lap = [&](int f, R f0, R &adv, R &lap, R &fx, R &fy, R &fz) {
                        const R xm = t.S(f, ii - 1, jj, kk), xp = t.S(f, ii + 1, jj, kk);
                        const R xm2 = t.S(f, ii - 2, jj, kk), xp2 = t.S(f, ii + 2, jj, kk);
                        const R ym = t.S(f, ii, jj - 1, kk), yp = t.S(f, ii, jj + 1, kk);
                        const R ym2 = t.S(f, ii, jj - 2, kk), yp2 = t.S(f, ii, jj + 2, kk);
                        const R zm2 = t.S(f, ii, jj, kk - 2), zm = t.S(f, ii, jj, kk - 1);
                        const R zp = t.S(f, ii, jj, kk + 1), zp2 = t.S(f, ii, jj, kk + 2);
                        const R im = (R(3) * f0 - R(4) * xm + xm2) * p.inv2dx;
                        const R ip = (R(-3) * f0 + R(4) * xp - xp2) * p.inv2dx;
                        const R jm = (R(3) * f0 - R(4) * ym + ym2) * p.inv2dy;
                        const R jp = (R(-3) * f0 + R(4) * yp - yp2) * p.inv2dy;
                        const R km = dz5(kmw, zm2, zm, f0, zp, zp2), kpv = dz5(kpw, zm2, zm, f0, zp, zp2);
                        adv = (u_plu * im + u_min * ip) + (v_plu * jm + v_min * jp) + (w_plu * km + w_min * kpv);
                        const R fxx = (xp - R(2) * f0 + xm) * p.invdx2;
                        const R fyy = (yp - R(2) * f0 + ym) * p.invdy2;
                        const R fzz = d2m * zm + d20 * f0 + d2p * zp;
                        lap = fxx + fyy + fzz;
                        fx = (xp - xm) * p.inv2dx;
                        fy = (yp - ym) * p.inv2dy;
                        fz = (zp - zm) * t.K(kk, RD1);
                    };
                    R fx, fy, fz;
                    adv_lap(3, T, advT, lapT, Tx, Ty, Tz);
                    adv_lap(0, u, advU, lapU, fx, fy, fz);
                    adv_lap(1, v, advV, lapV, fx, fy, fz);
                    adv_lap(2, w, advW, lapW, fx, fy, fz);
                }
                const R rho = fdiv(p.Trho, T);
                const Thermo<R> th = thermo(p, smu, sk, T, t.S(3, ii, jj, kk + 1), Yx, gk, nzy, Tx,
                                            Ty, Tz, lapT, t.K(kk, RDZ), rho);
                kY = -p.Y_f * th.K_T * th.Y;
                R kval[4];
                kval[3] = (a.ph.temperature_convection == 0) ? th.T_RHS_tmp - (u * Tx + v * Ty + w * Tz)
                                                             : th.T_RHS_tmp - advT;
                const R mod_U = rsqrt_(u * u + v * v + w * w);
                kval[0] = th.nu * lapU - advU + (-p.cd * th.Y * mod_U * u);
                kval[1] = th.nu * lapV - advV + (-p.cd * th.Y * mod_U * v);
                kval[2] = th.nu * lapW - advW + (fdiv(p.g * (rho - p.rho_inf), rho) - p.cd * th.Y * mod_U * w);
                // ---- SGS divergence with Van Driest damping (turbulence.cu:255-454)
                {
                    const R nu = fdiv(p.mu, rho);
                    const R inv_avd_nu = fdiv(p.inv_avd, nu);
                    const R zk = t.K(kk, RZ);
                    auto zibm = [&](int q, R zz) -> R {
                        const R d = zz - (R)t.ctopo[q];
                        return d > R(0) ? d : R(0);
                    };
                    const int qxp = TL::cq(ii + 1, jj), qxm = TL::cq(ii - 1, jj);
                    const int qyp = TL::cq(ii, jj + 1), qym = TL::cq(ii, jj - 1);
                    R mu_c = t.G(0, ii, jj, kk);
                    R mu_xp = t.G(0, ii + 1, jj, kk), mu_xm = t.G(0, ii - 1, jj, kk);
                    R mu_yp = t.G(0, ii, jj + 1, kk), mu_ym = t.G(0, ii, jj - 1, kk);
                    R mu_kp = t.G(0, ii, jj, kk + 1), mu_km = t.G(0, ii, jj, kk - 1);
                    // Van Driest factors; where the bound shows them all to be
                    // exactly 1 the products would not change mu
                    if (s_vd_bound > VanDriestCut<R>::v * R(1.001) * nu) {
                        if (*s_vd_zero) {
                            // columns without friction: the factor of -z_ibm * 0 * inv_avd_nu,
                            // 1 - exp(-0) = 0 (NaN when 1/nu is not finite, as there)
                            const R f0 = R(0) * inv_avd_nu, f00 = f0 * f0;
                            if (t.cut_[cc] == R(0)) {
                                mu_c *= f00;
                                mu_kp *= f00;
                                mu_km *= f00;
                            }
                            if (t.cut_[qxp] == R(0)) mu_xp *= f00;
                            if (t.cut_[qxm] == R(0)) mu_xm *= f00;
                            if (t.cut_[qyp] == R(0)) mu_yp *= f00;
                            if (t.cut_[qym] == R(0)) mu_ym *= f00;
                        }
                    } else {
                        const R ut0 = t.cut_[cc];
                        R fc = -zibm(cc, zk) * ut0 * inv_avd_nu;
                        R fxp_ = -zibm(qxp, zk) * t.cut_[qxp] * inv_avd_nu;
                        R fxm_ = -zibm(qxm, zk) * t.cut_[qxm] * inv_avd_nu;
                        R fyp_ = -zibm(qyp, zk) * t.cut_[qyp] * inv_avd_nu;
                        R fym_ = -zibm(qym, zk) * t.cut_[qym] * inv_avd_nu;
                        R fkm = -zibm(cc, t.K(kk - 1, RZ)) * ut0 * inv_avd_nu;
                        R fkp = -zibm(cc, t.K(kk + 1, RZ)) * ut0 * inv_avd_nu;
                        // A factor is exactly 1 below the cut-off and exactly 0
                        // where -z+/A is 0 (no height above the terrain, or a
                        // column without wall friction, as over the hills): only
                        // a cell with another argument evaluates the exponentials.
                        if (van_driest_needs_exp(fc) || van_driest_needs_exp(fxp_) || van_driest_needs_exp(fxm_) ||
                            van_driest_needs_exp(fyp_) || van_driest_needs_exp(fym_) || van_driest_needs_exp(fkm) ||
                            van_driest_needs_exp(fkp)) {
                            fc = van_driest(fc);
                            fxp_ = van_driest(fxp_);
                            fxm_ = van_driest(fxm_);
                            fyp_ = van_driest(fyp_);
                            fym_ = van_driest(fym_);
                            fkm = van_driest(fkm);
                            fkp = van_driest(fkp);
                        } else {
                            fc = van_driest_exact(fc);
                            fxp_ = van_driest_exact(fxp_);
                            fxm_ = van_driest_exact(fxm_);
                            fyp_ = van_driest_exact(fyp_);
                            fym_ = van_driest_exact(fym_);
                            fkm = van_driest_exact(fkm);
                            fkp = van_driest_exact(fkp);
                        }
                        mu_c *= fc * fc;
                        mu_xp *= fxp_ * fxp_;
                        mu_xm *= fxm_ * fxm_;
                        mu_yp *= fyp_ * fyp_;
                        mu_ym *= fym_ * fym_;
                        mu_kp *= fkp * fkp;
                        mu_km *= fkm * fkm;
                    }
                    const R S11 = t.G(1, ii, jj, kk), S12 = t.G(2, ii, jj, kk), S13 = t.G(3, ii, jj, kk);
                    const R S22 = t.G(4, ii, jj, kk), S23 = t.G(5, ii, jj, kk), S33 = t.G(6, ii, jj, kk);
                    const R wc = t.K(kk, RD1);
                    const R mu_x = (mu_xp - mu_xm) * p.inv2dx, mu_y = (mu_yp - mu_ym) * p.inv2dy, mu_z = (mu_kp - mu_km) * wc;
                    const R S11_x = (t.G(1, ii + 1, jj, kk) - t.G(1, ii - 1, jj, kk)) * p.inv2dx;
                    const R S12_x = (t.G(2, ii + 1, jj, kk) - t.G(2, ii - 1, jj, kk)) * p.inv2dx;
                    const R S13_x = (t.G(3, ii + 1, jj, kk) - t.G(3, ii - 1, jj, kk)) * p.inv2dx;
                    const R S21_y = (t.G(2, ii, jj + 1, kk) - t.G(2, ii, jj - 1, kk)) * p.inv2dy;
                    const R S22_y = (t.G(4, ii, jj + 1, kk) - t.G(4, ii, jj - 1, kk)) * p.inv2dy;
                    const R S23_y = (t.G(5, ii, jj + 1, kk) - t.G(5, ii, jj - 1, kk)) * p.inv2dy;
                    const R S31_z = (t.G(3, ii, jj, kk + 1) - t.G(3, ii, jj, kk - 1)) * wc;
                    const R S32_z = (t.G(5, ii, jj, kk + 1) - t.G(5, ii, jj, kk - 1)) * wc;
                    const R S33_z = (t.G(6, ii, jj, kk + 1) - t.G(6, ii, jj, kk - 1)) * wc;
                    const R dU_x = (t.G(7, ii + 1, jj, kk) - t.G(7, ii - 1, jj, kk)) * p.inv2dx;
                    const R dU_y = (t.G(7, ii, jj + 1, kk) - t.G(7, ii, jj - 1, kk)) * p.inv2dy;
                    const R dU_z = (t.G(7, ii, jj, kk + 1) - t.G(7, ii, jj, kk - 1)) * wc;
                    const R div_S_x = S11_x + S21_y + S31_z;
                    const R div_S_y = S12_x + S22_y + S32_z;
                    const R div_S_z = S13_x + S23_y + S33_z;
                    const R inv_rho = fdiv(R(1), rho);
                    const R sgs_x = R(-2) * (mu_x * S11 + mu_y * S12 + mu_z * S13 + mu_c * div_S_x) * inv_rho;
                    const R sgs_y = R(-2) * (mu_x * S12 + mu_y * S22 + mu_z * S23 + mu_c * div_S_y) * inv_rho;
                    const R sgs_z = R(-2) * (mu_x * S13 + mu_y * S23 + mu_z * S33 + mu_c * div_S_z) * inv_rho;
                    const R sgs_q = -fdiv(mu_x * Tx + mu_y * Ty + mu_z * Tz + mu_c * lapT, rho * p.Pr);
                    kval[0] += -sgs_x + third(dU_x);
                    kval[1] += -sgs_y + third(dU_y);
                    kval[2] += -sgs_z + third(dU_z);
                    kval[3] -= sgs_q;
                }
                // values the column boundary pass needs
                R *bcs = a.bc + (size_t)col * kBcSlots;
                if (gk == kc + 1) { bcs[0] = kval[3]; bcs[2] = (gk < nzy) ? kY : R(0); }
                if (gk == kc + 2) { bcs[1] = kval[3]; bcs[3] = (gk < nzy) ? kY : R(0); }
                if (gk == Nz - 2) { bcs[4] = kval[0]; bcs[5] = kval[1]; bcs[6] = kval[2]; bcs[7] = kval[3]; }
                if (gk == Nz - 3) { bcs[8] = kval[0]; bcs[9] = kval[1]; bcs[10] = kval[2]; bcs[11] = kval[3]; }
    #pragma unroll
                for (int f = 0; f < 4; f++) {
                    const size_t o = (size_t)f * N + cg;
                    a.Xout[o] = rk_update(a.method, a.stage, kval[f], ynv[f], accv[f], an);
                    if (kp) a.acc[o] = accv[f];
                }
            } else if (gk < nzy) {
                // fuel cell whose velocity and temperature the boundary rules set (top plane)
                const R T = t.S(3, ii, jj, kk);
                const R K_T = arrhenius(p, T);
                kY = -p.Y_f * K_T * Yx;
            }
            if (ylive) {
                const R kv = (gk < nzy) ? kY : R(0);
                a.Xout[oY] = rk_update(a.method, a.stage, kv, ynY, accY, an);
                if (kp) a.acc[oY] = accY;
            }
        }
        __syncthreads();
        // ---- 4. cut node and top of the tile's columns, where the two cells
        //        they extrapolate from are in this tile (their k-values were
        //        stored to a.bc above); the other columns go to k_stage_bc.
        for (int q = threadIdx.x; q < TI * TJ; q += NT) {
            const int ii = q / TJ, jj = q % TJ;
            const int gi = i0 + ii, gj = j0 + jj;
            if (gi >= Nx || gj >= Ny) continue;
            const int col = gi * Ny + gj;
            const int kc = t.ccut[TL::cq(ii, jj)], nzy = t.cnzy[TL::cq(ii, jj)];
            if (kc >= k0 && kc < k0 + KZ && bc_cut_in_tile(kc, KZ)) bc_cut_node(a, col, kc, nzy, rd, kp, an);
            if (Nz - 1 >= k0 && Nz - 1 < k0 + KZ && bc_top_in_tile(Nz, KZ)) bc_top(a, col, rd, kp, an);
        }
    }
}


// ---------------------------------------------------------------------------
// Boundary values the fused pass could not complete (pde.cu:14-99): the cut
// node of the listed columns whose kc+1 / kc+2 lie in the next z-tile, and the
// top plane when Nz-3 and Nz-1 lie in different z-tiles.  One thread per
// listed column; the k-values come from the boundary slots.
template <class R>
__global__ void __launch_bounds__(128) k_stage_bc(const StageArgs<R> a, int KZ)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= a.nbcfix) return;
    const int col = a.bcfix[q];
    const int kc = __ldg(a.g.cut + col), nzy = __ldg(a.g.nzy + col);
    const R an = (R)a.a_next;
    const bool rd = stage_reads_acc(a.method, a.stage), kp = stage_keeps_acc(a.method, a.stage);
    if (!bc_cut_in_tile(kc, KZ)) bc_cut_node(a, col, kc, nzy, rd, kp, an);
    if (!bc_top_in_tile(a.g.Nz, KZ)) bc_top(a, col, rd, kp, an);
}

}  // namespace

// Tile shapes of the fused pass: TI x TJ columns of KZ = 8 planes, NT threads.
// FP32 compiles three block forms, all at 24 or 32 warps per SM: 8x16 columns
// with 512 threads (two blocks, 64 registers) or 384 threads (two blocks, 80
// registers), and 8x8 columns with 256 threads (three blocks, 80 registers;
// more halo work per cell).  The per-context tuner in solver.cu times them on
// the context's own grid.  (Measured and dropped: 8x16 with 256 threads at 118
// registers, 16 warps per SM, 3-4% slower; 4x16 and 4x8 tiles.)  FP64: 8x8
// columns with 512 threads (one block, 124 registers, 16 warps: 8.20 -> 6.09 ms
// per launch at 512x512x128) or 256 threads (200 registers, 8 warps).
template <class R, int TI_, int TJ_, int NT_ = 256> struct StageShape {
    static constexpr int TI = TI_, TJ = TJ_, KZ = 8, NT = NT_;
    using TL = Tile<R, TI, TJ, KZ>;
    static size_t smem() { return TL::bytes(); }
};
template <class R> struct StageShapes;
template <> struct StageShapes<float> {
    static constexpr int count = 3;
    static constexpr int ti[3] = {8, 8, 8}, tj[3] = {16, 16, 8}, nt[3] = {512, 384, 256};
};
template <> struct StageShapes<double> {
    static constexpr int count = 2;
    static constexpr int ti[2] = {8, 8}, tj[2] = {8, 8}, nt[2] = {512, 256};
};

// the shape with index idx, as a type, for f(Shape)
template <class R, class F> cudaError_t with_shape(int idx, F f)
{
    if constexpr (sizeof(R) == 4) {
        switch (idx) {
        case 0: return f(StageShape<R, 8, 16, 512>());
        case 1: return f(StageShape<R, 8, 16, 384>());
        case 2: return f(StageShape<R, 8, 8>());
        default: return cudaErrorInvalidValue;
        }
    } else {
        switch (idx) {
        case 0: return f(StageShape<R, 8, 8, 512>());
        case 1: return f(StageShape<R, 8, 8>());
        default: return cudaErrorInvalidValue;
        }
    }
}

int g_stage_sms = 0;   // multiprocessors of the device, read at set-up

template <class R> cudaError_t stage_set_attributes()
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (!e) e = cudaDeviceGetAttribute(&g_stage_sms, cudaDevAttrMultiProcessorCount, dev);
    for (int q = 0; !e && q < StageShapes<R>::count; q++)
        e = with_shape<R>(q, [](auto sh) {
            using SH = decltype(sh);
            return cudaFuncSetAttribute(k_stage_fused<R, SH::TI, SH::TJ, SH::KZ, SH::NT>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SH::smem());
        });
    return e;
}
template cudaError_t stage_set_attributes<double>();
template cudaError_t stage_set_attributes<float>();

template <class R> cudaError_t launch_stage(const StageArgs<R> &a, cudaStream_t s, cudaEvent_t *ev)
{
    const int ncol = a.g.Nx * a.g.Ny;
    if (a.coef) {
        cudaError_t e = launch_closure_coef_tc<R>(a.X, a.g, a.ph.dx, a.ph.dy, a.theta, a.coef, a.closure_err, s,
                                                  a.closure_wait);
        if (e) return e;
    }
    k_utau<R><<<(ncol + 127) / 128, 128, 0, s>>>(a);
    if (ev) cudaEventRecord(ev[0], s);
    cudaError_t e = with_shape<R>(a.tile, [&](auto sh) {
        using SH = decltype(sh);
        const int ntk = (a.g.Nz + SH::KZ - 1) / SH::KZ, ntj = (a.g.Ny + SH::TJ - 1) / SH::TJ;
        const int nti = (a.g.Nx + SH::TI - 1) / SH::TI;
        const int w = SH::TJ == 16 ? 0 : 1;
        CUtensorMap m, myn, macc;
        const void *src = (sizeof(R) == 4) ? a.tmap[w] : nullptr;
        const void *pyn = (sizeof(R) == 4) ? a.pmap_yn[w] : nullptr, *pacc = (sizeof(R) == 4) ? a.pmap_acc[w] : nullptr;
        if (src) memcpy(&m, src, sizeof(m));
        else memset(&m, 0, sizeof(m));
        const bool pf = pyn && pacc;
        if (pf) {
            memcpy(&myn, pyn, sizeof(myn));
            memcpy(&macc, pacc, sizeof(macc));
        } else {
            memset(&myn, 0, sizeof(myn));
            memset(&macc, 0, sizeof(macc));
        }
        k_stage_fused<R, SH::TI, SH::TJ, SH::KZ, SH::NT><<<ntk * ntj * nti, SH::NT, SH::smem(), s>>>(
            a, m, myn, macc, src ? 1 : 0, pf ? 1 : 0, ntk, ntj, nti);
        return cudaSuccess;
    });
    if (e) return e;
    if (ev) cudaEventRecord(ev[1], s);
    if (a.nbcfix > 0) k_stage_bc<R><<<(a.nbcfix + 127) / 128, 128, 0, s>>>(a, 8);
    if (ev) cudaEventRecord(ev[2], s);
    return cudaGetLastError();
}

int stage_tile_planes(int precision) { (void)precision; return 8; }

bool stage_tensor_map(void *out, const float *X, int Nx, int Ny, int Nz, int TI, int TJ, void *encode_fn)
{
    if (!encode_fn || Nz % 4 != 0 || (reinterpret_cast<uintptr_t>(X) & 15) != 0) return false;
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    const cuuint64_t dims[4] = {(cuuint64_t)Nz, (cuuint64_t)Ny, (cuuint64_t)Nx, 4};
    const cuuint64_t strides[3] = {(cuuint64_t)Nz * 4, (cuuint64_t)Ny * Nz * 4, (cuuint64_t)Nx * Ny * Nz * 4};
    const cuuint32_t box[4] = {16, (cuuint32_t)(TJ + 4), (cuuint32_t)(TI + 4), 4};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = reinterpret_cast<Encode>(encode_fn)(
        reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(X), dims, strides,
        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}
bool stage_cell_map(void *out, const float *X, int Nx, int Ny, int Nz, int TI, int TJ, void *encode_fn)
{
    if (!encode_fn || Nz % 4 != 0 || (reinterpret_cast<uintptr_t>(X) & 15) != 0) return false;
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    const cuuint64_t dims[4] = {(cuuint64_t)Nz, (cuuint64_t)Ny, (cuuint64_t)Nx, 4};
    const cuuint64_t strides[3] = {(cuuint64_t)Nz * 4, (cuuint64_t)Ny * Nz * 4, (cuuint64_t)Nx * Ny * Nz * 4};
    const cuuint32_t box[4] = {8, (cuuint32_t)TJ, (cuuint32_t)TI, 4};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = reinterpret_cast<Encode>(encode_fn)(
        reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(X), dims, strides,
        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}
int stage_tile_count(int precision) { return precision == 0 ? StageShapes<double>::count : StageShapes<float>::count; }
void stage_tile_shape(int precision, int idx, int *ti, int *tj, int *nt)
{
    if (precision == 0) {
        *ti = StageShapes<double>::ti[idx];
        *tj = StageShapes<double>::tj[idx];
        if (nt) *nt = StageShapes<double>::nt[idx];
    } else {
        *ti = StageShapes<float>::ti[idx];
        *tj = StageShapes<float>::tj[idx];
        if (nt) *nt = StageShapes<float>::nt[idx];
    }
}

template cudaError_t launch_stage<double>(const StageArgs<double> &, cudaStream_t, cudaEvent_t *);
template cudaError_t launch_stage<float>(const StageArgs<float> &, cudaStream_t, cudaEvent_t *);

}  // namespace wf
