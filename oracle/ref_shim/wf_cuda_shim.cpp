/*
 * wf_cuda_shim.cpp -- state of the host emulation (see wf_cuda_shim.h) and
 * the cuFFT stand-in (see include/cufft.h).  TEST INFRASTRUCTURE ONLY.
 */
#include "wf_cuda_shim.h"

#include <mutex>
#include <vector>

#include "../cpu_fft.h"
#include "include/cufft.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;
int wf_emu_parallel = 0;

namespace {
struct ShimPlan {
    int n0, n1, batch, idist, odist;
    bool live;
};
std::vector<ShimPlan> g_plans(1, ShimPlan{0, 0, 0, 0, 0, false});  /* handle 0 is never valid */
std::mutex g_mu;

cufftHandle add_plan(const ShimPlan &p)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_plans.push_back(p);
    return (cufftHandle)(g_plans.size() - 1);
}
}  // namespace

cufftResult cufftPlanMany(cufftHandle *plan, int rank, int *n, int *inembed, int istride, int idist,
                          int *onembed, int ostride, int odist, cufftType type, int batch)
{
    if (rank != 2 || type != CUFFT_Z2Z || istride != 1 || ostride != 1 || inembed || onembed)
        return CUFFT_INVALID_VALUE;
    *plan = add_plan(ShimPlan{n[0], n[1], batch, idist, odist, true});
    return CUFFT_SUCCESS;
}

cufftResult cufftPlan2d(cufftHandle *plan, int nx, int ny, cufftType type)
{
    if (type != CUFFT_Z2Z) return CUFFT_INVALID_VALUE;
    *plan = add_plan(ShimPlan{nx, ny, 1, nx * ny, nx * ny, true});
    return CUFFT_SUCCESS;
}

cufftResult cufftExecZ2Z(cufftHandle plan, cufftDoubleComplex *idata, cufftDoubleComplex *odata, int direction)
{
    ShimPlan p;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (plan <= 0 || (size_t)plan >= g_plans.size() || !g_plans[plan].live) return CUFFT_INVALID_PLAN;
        p = g_plans[plan];
    }
    if (p.idist != p.n0 * p.n1 || p.odist != p.n0 * p.n1) return CUFFT_INVALID_VALUE;
    cfft_2d_many(p.n0, p.n1, p.batch, (const double *)idata, (double *)odata, direction);
    return CUFFT_SUCCESS;
}

cufftResult cufftDestroy(cufftHandle plan)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (plan <= 0 || (size_t)plan >= g_plans.size()) return CUFFT_INVALID_PLAN;
    g_plans[plan].live = false;
    return CUFFT_SUCCESS;
}
