/*
 * wf_cuda_shim.h -- host emulation of the small CUDA runtime surface the
 * reference's kernel sources use, so those sources can be compiled by g++ and
 * run on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY.  It is force-included (g++ -include) into copies
 * of the reference's src/cu/*.cu files whose `kernel<<<B, T>>>(args)` launch
 * lines the build recipe (oracle/Makefile) rewrites to
 * `wf_emu_launch(B, T, kernel, args)`.  A launch runs every virtual thread's
 * grid-stride loop to completion, thread by thread (the order a single
 * resident wave with no overlap would give), or, when wf_emu_parallel is set,
 * distributes the virtual threads over OpenMP threads (used only for timing).
 * Device memory is host memory.
 */
#ifndef WF_CUDA_SHIM_H
#define WF_CUDA_SHIM_H

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <math.h>
#include <vector_types.h>

typedef int cudaError_t;
#define cudaSuccess 0
#define cudaErrorMemoryAllocation 2

enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3
};
enum cudaDeviceAttr { cudaDevAttrMultiProcessorCount = 16 };

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;
extern int wf_emu_parallel;

inline cudaError_t cudaMalloc(void **p, size_t n)
{
    *p = std::malloc(n ? n : 1);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
template <class T> inline cudaError_t cudaMalloc(T **p, size_t n) { return cudaMalloc((void **)p, n); }
inline cudaError_t cudaFree(void *p) { std::free(p); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { std::memmove(d, s, n); return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline const char *cudaGetErrorString(cudaError_t) { return "host emulation"; }
inline cudaError_t cudaGetDevice(int *d) { *d = 0; return cudaSuccess; }
inline cudaError_t cudaDeviceGetAttribute(int *v, cudaDeviceAttr, int) { *v = 1; return cudaSuccess; }

template <class K, class... A>
void wf_emu_launch(int blocks, int threads, K kernel, A... args)
{
    const long total = (long)blocks * (long)threads;
    if (wf_emu_parallel) {
#pragma omp parallel for schedule(dynamic, 16)
        for (long g = 0; g < total; g++) {
            gridDim = dim3((unsigned)blocks);
            blockDim = dim3((unsigned)threads);
            blockIdx.x = (unsigned)(g / threads); blockIdx.y = 0u; blockIdx.z = 0u;
            threadIdx.x = (unsigned)(g % threads); threadIdx.y = 0u; threadIdx.z = 0u;
            kernel(args...);
        }
    } else {
        gridDim = dim3((unsigned)blocks);
        blockDim = dim3((unsigned)threads);
        for (long g = 0; g < total; g++) {
            blockIdx.x = (unsigned)(g / threads); blockIdx.y = 0u; blockIdx.z = 0u;
            threadIdx.x = (unsigned)(g % threads); threadIdx.y = 0u; threadIdx.z = 0u;
            kernel(args...);
        }
    }
}

#define WF_LAUNCH(kern, blocks, threads, ...) wf_emu_launch(blocks, threads, kern, __VA_ARGS__)

#endif
