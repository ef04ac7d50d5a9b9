// dropin_device_phi.cu -- test driver for the drop-in's Phi on device buffers.
//
// TEST INFRASTRUCTURE (compiled by tests/test_boundary_gpu.py): reads a
// parameter file with wf_read_parameters and a packed FP64 state (raw doubles),
// copies the state to the device, calls the reference-signature Phi of
// include/wf_dropin.h on device buffers (one warm-up call, then one call timed
// with CUDA events on the legacy default stream, where the drop-in enqueues),
// writes R_new to a file and prints the time of that call beside the time of
// one device-to-host copy of the state.
//
// usage: dropin_device_phi PARAMS STATE_IN R_OUT
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "wf_dropin.h"
#include "wildfires_b200.h"

// The drop-in archive refers to these callbacks of the reference's own objects
// (logs.cu, utils.cu); Phi does not call them.
void log_timestep(Parameters, int, double, double, double, double, double, double, double) {}
void log_message(Parameters, const char *) {}
void format_seconds(double, char *out) { out[0] = 0; }

int main(int argc, char **argv)
{
    if (argc < 4) return 2;
    Parameters P;
    if (wf_read_parameters(argv[1], &P) != WF_OK) { fprintf(stderr, "%s\n", wf_last_error()); return 1; }
    const size_t S = wf_state_size(&P);
    double *h = (double *)malloc(S * sizeof(double));
    FILE *f = fopen(argv[2], "rb");
    if (!f || fread(h, sizeof(double), S, f) != S) return 1;
    fclose(f);
    double *a = nullptr, *b = nullptr;
    if (cudaMalloc((void **)&a, S * sizeof(double)) || cudaMalloc((void **)&b, S * sizeof(double))) return 1;
    cudaMemcpy(a, h, S * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemset(b, 0, S * sizeof(double));
    Phi(0.0, a, b, nullptr, nullptr, nullptr, nullptr, nullptr, P);   // warm-up: context creation
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    Phi(0.0, a, b, nullptr, nullptr, nullptr, nullptr, nullptr, P);
    cudaEventRecord(e1, 0);
    cudaMemcpyAsync(h, b, S * sizeof(double), cudaMemcpyDeviceToHost, 0);
    cudaEventRecord(e2, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    float phi_ms = 0, copy_ms = 0;
    cudaEventElapsedTime(&phi_ms, e0, e1);
    cudaEventElapsedTime(&copy_ms, e1, e2);
    f = fopen(argv[3], "wb");
    if (!f || fwrite(h, sizeof(double), S, f) != S) return 1;
    fclose(f);
    printf("PHI_MS=%.4f\nCOPY_MS=%.4f\n", phi_ms, copy_ms);
    return 0;
}
