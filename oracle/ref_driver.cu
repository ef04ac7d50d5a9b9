/*
 * ref_driver.cu -- project-written driver around the REFERENCE's own solver
 * entry points (read_parameters_file, initial_conditions_input, create_y_0,
 * Phi, RK4, solve_pressure[_iterative], solve_PDE), used to produce reference
 * outputs for pinning the oracle and the GPU path.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile in two flavours, both
 * into oracle/_ref/ (never committed):
 *   ref_host  -- g++ build of the reference's src/cu sources through the host
 *                emulation in oracle/ref_shim/ (CPU; golden vectors, CPU baseline)
 *   ref_gpu   -- nvcc sm_100a build of the same unmodified sources (on a B200)
 * The reference's own main (src/cu/main.cu) is not used: this driver mirrors
 * its set-up sequence (main.cu:27-76) but reads initial conditions from
 * `input_path` only and writes results into OUTDIR.
 *
 * An optional topography.bin (Nx*Ny FP64, j fastest) in the working directory
 * replaces the terrain before the immersed-boundary tables are rebuilt with
 * the reference's ibm_parameters (ibm.cu:57-95).
 *
 * usage: ref_driver MODE PARAMS_FILE OUTDIR [parallel]
 *   MODE phi      -- one right-hand-side evaluation Phi(y0)          -> OUTDIR/R.bin
 *        rk4      -- one RK4 stage combination y1 = RK4(y0)         -> OUTDIR/y1.bin
 *        pressure -- one pressure solve with y_np1 = y_n = y0, p0   -> OUTDIR/p.bin
 *        step     -- solve_PDE for Nt steps; prints SAVE_PATH=...  (files *.bin.N)
 *        time     -- as step, also prints SECONDS=<wall time of solve_PDE>
 *        ic       -- the reference's initial_conditions + create_y_0
 *                    (functions.cu:187-323, solver.cu:41-56)          -> OUTDIR/y0.bin, p0.bin
 *                    (Y entries the reference leaves unwritten are zero here:
 *                    its main mallocs Y, and large fresh allocations read as zero)
 *        params   -- the record read_parameters_file built (raw bytes, before
 *                    this driver sets its launch sizes)              -> OUTDIR/params.bin
 *                    and its arrays x, y, z, t, kx, ky, topography   -> OUTDIR/<name>.bin
 *                    (FP64), cut_nodes, Nz_Y                         -> OUTDIR/<name>.bin (int32)
 *        domain   -- the reference's save_domain + save_topography
 *                    (output.cu:46-99) with save_path = OUTDIR/    -> x y z t topography Nz_Y .bin
 * The working directory must be writable: read_parameters_file creates
 * data/output/<timestamp>/ there (src/cu/parameters.cu:21-37).
 */
#include <sys/stat.h>
#include <sys/time.h>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "functions.cuh"
#include "input.cuh"
#include "output.cuh"
#include "parameters.cuh"
#include "pde.cuh"
#include "pressure.cuh"
#include "solver.cuh"

#ifndef WF_LAUNCH
#define WF_LAUNCH(kern, blocks, threads, ...) kern<<<blocks, threads>>>(__VA_ARGS__)
#define WF_HOST_EMULATION 0
#else
#define WF_HOST_EMULATION 1
extern int wf_emu_parallel;
#endif

static int write_bin(const char *dir, const char *name, const double *d, size_t n)
{
    char path[1024];
    snprintf(path, sizeof(path), "%s/%s", dir, name);
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    size_t w = fwrite(d, sizeof(double), n, f);
    fclose(f);
    return w == n ? 0 : -1;
}

template <class T> static T *dev_copy(const T *h, size_t n)
{
    T *d = NULL;
    cudaMalloc((void **)&d, n * sizeof(T));
    cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

static double now_s()
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s MODE PARAMS_FILE OUTDIR [parallel]\n", argv[0]);
        return 2;
    }
    const char *mode = argv[1], *outdir = argv[3];
#if WF_HOST_EMULATION
    wf_emu_parallel = (argc > 4 && strcmp(argv[4], "parallel") == 0);
#endif
    mkdir("data", 0777);
    mkdir("data/output", 0777);
    Parameters P = read_parameters_file(argv[2]);
    {
        /* optional terrain override: topography.bin (Nx*Ny FP64) in the working
         * directory replaces the parsed terrain, then the reference's own
         * immersed-boundary precompute runs again (ibm.cu:57-95) */
        FILE *tf = fopen("topography.bin", "rb");
        if (tf) {
            const size_t nt = (size_t)P.Nx * P.Ny;
            const size_t got = fread(P.topography, sizeof(double), nt, tf);
            fclose(tf);
            if (got != nt) {
                fprintf(stderr, "ref_driver: topography.bin has %zu values, expected %zu\n", got, nt);
                return 2;
            }
            ibm_parameters(&P);
        }
    }
    if (strcmp(mode, "params") == 0) {
        char path[1024];
        snprintf(path, sizeof(path), "%s/params.bin", outdir);
        FILE *f = fopen(path, "wb");
        if (!f || fwrite(&P, sizeof(P), 1, f) != 1) {
            fprintf(stderr, "ref_driver: cannot write %s\n", path);
            return 1;
        }
        fclose(f);
        const size_t nc = (size_t)P.Nx * P.Ny;
        int rc = write_bin(outdir, "x.bin", P.x, P.Nx) || write_bin(outdir, "y.bin", P.y, P.Ny) ||
                 write_bin(outdir, "z.bin", P.z, P.Nz) || write_bin(outdir, "t.bin", P.t, P.Nt + 1) ||
                 write_bin(outdir, "kx.bin", P.kx, P.Nx - 1) || write_bin(outdir, "ky.bin", P.ky, P.Ny - 1) ||
                 write_bin(outdir, "topography.bin", P.topography, nc);
        const int *ia[2] = {P.cut_nodes, P.Nz_Y};
        const char *in[2] = {"cut_nodes.bin", "Nz_Y.bin"};
        for (int q = 0; q < 2 && !rc; q++) {
            snprintf(path, sizeof(path), "%s/%s", outdir, in[q]);
            FILE *g = fopen(path, "wb");
            rc = !g || fwrite(ia[q], sizeof(int), nc, g) != nc;
            if (g) fclose(g);
        }
        return rc ? 1 : 0;
    }
    if (strcmp(mode, "domain") == 0) {
        snprintf(P.save_path, sizeof(P.save_path), "%s/", outdir);
        save_domain(P);
        save_topography(P);
        return 0;
    }
    P.threads_per_block = THREADS;
    P.number_of_blocks = BLOCKS;
    if (strcmp(mode, "ic") == 0) {
        const size_t N = (size_t)P.Nx * P.Ny * P.Nz, NY = (size_t)P.Nx * P.Ny * P.Nz_Y_max, S = 4 * N + NY;
        double *u = (double *)calloc(N, 8), *v = (double *)calloc(N, 8), *w = (double *)calloc(N, 8);
        double *T = (double *)calloc(N, 8), *p = (double *)calloc(N, 8), *Y = (double *)calloc(NY ? NY : 1, 8);
        double *y0 = (double *)calloc(S, 8);
        initial_conditions(u, v, w, T, Y, p, P);
        create_y_0(u, v, w, T, Y, y0, P);
        if (write_bin(outdir, "y0.bin", y0, S) || write_bin(outdir, "p0.bin", p, N)) {
            fprintf(stderr, "ref_driver: cannot write %s\n", outdir);
            return 1;
        }
        return 0;
    }
    if (P.input_path[0] == '\0') {
        fprintf(stderr, "ref_driver: input_path must be set\n");
        return 2;
    }
    const int Nx = P.Nx, Ny = P.Ny, Nz = P.Nz;
    const size_t N = (size_t)Nx * Ny * Nz, NY = (size_t)Nx * Ny * P.Nz_Y_max, S = 4 * N + NY;
    double *u = (double *)malloc(N * 8), *v = (double *)malloc(N * 8), *w = (double *)malloc(N * 8);
    double *T = (double *)malloc(N * 8), *p = (double *)malloc(N * 8), *Y = (double *)malloc((NY ? NY : 1) * 8);
    double *y0 = (double *)malloc(S * 8);
    initial_conditions_input(u, v, w, T, Y, p, P);
    create_y_0(u, v, w, T, Y, y0, P);
    double *y0_d = dev_copy(y0, S), *p_d = dev_copy(p, N);

    if (strcmp(mode, "step") == 0 || strcmp(mode, "time") == 0) {
        const double t0 = now_s();
        solve_PDE(y0_d, p_d, P);
        cudaDeviceSynchronize();
        const double t1 = now_s();
        printf("SAVE_PATH=%s\n", P.save_path);
        printf("SECONDS=%.6f\n", t1 - t0);
        return 0;
    }

    double *z_d = dev_copy(P.z, (size_t)Nz), *zibm_d = dev_copy(P.z_ibm, N);
    int *nzy_d = dev_copy(P.Nz_Y, (size_t)Nx * Ny), *cut_d = dev_copy(P.cut_nodes, (size_t)Nx * Ny);
    double *Rt_d = NULL;
    cudaMalloc((void **)&Rt_d, (18 * N + (size_t)Nx * Ny) * 8);
    double *out = (double *)calloc(S, 8);

    if (strcmp(mode, "phi") == 0) {
        double *Rn_d = dev_copy(out, S);   /* zero-filled: Y above the fuel top stays 0 */
        Phi(P.t[0], y0_d, Rn_d, Rt_d, z_d, zibm_d, nzy_d, cut_d, P);
        cudaDeviceSynchronize();
        cudaMemcpy(out, Rn_d, S * 8, cudaMemcpyDeviceToHost);
        return write_bin(outdir, "R.bin", out, S) ? 1 : 0;
    }
    if (strcmp(mode, "rk4") == 0) {
        double *k_d = NULL, *F_d = dev_copy(out, S), *y1_d = dev_copy(out, S);
        double *kz = (double *)calloc(4 * S, 8);
        k_d = dev_copy(kz, 4 * S);
        RK4(P.t[0], y0_d, y1_d, k_d, F_d, Rt_d, z_d, zibm_d, nzy_d, cut_d, P.dt, (int)S, P);
        cudaDeviceSynchronize();
        cudaMemcpy(out, y1_d, S * 8, cudaMemcpyDeviceToHost);
        return write_bin(outdir, "y1.bin", out, S) ? 1 : 0;
    }
    if (strcmp(mode, "pressure") == 0) {
        const size_t M = (size_t)(Nx - 1) * (Ny - 1);
        double *kx_d = dev_copy(P.kx, (size_t)Nx - 1), *ky_d = dev_copy(P.ky, (size_t)Ny - 1);
        double *gam, *a, *b, *c;
        cufftDoubleComplex *d, *l, *uu, *yy, *din, *dout, *pti, *pto;
        cudaMalloc((void **)&gam, M * (Nz - 1) * 8);
        cudaMalloc((void **)&a, M * (Nz - 2) * 8);
        cudaMalloc((void **)&b, M * (Nz - 1) * 8);
        cudaMalloc((void **)&c, M * (Nz - 2) * 8);
        cudaMalloc((void **)&d, M * (Nz - 1) * 16);
        cudaMalloc((void **)&l, M * (Nz - 2) * 16);
        cudaMalloc((void **)&uu, M * (Nz - 1) * 16);
        cudaMalloc((void **)&yy, M * (Nz - 1) * 16);
        cudaMalloc((void **)&din, M * (Nz - 1) * 16);
        cudaMalloc((void **)&dout, M * (Nz - 1) * 16);
        cudaMalloc((void **)&pti, M * 16);
        cudaMalloc((void **)&pto, M * 16);
        WF_LAUNCH(gammas_and_coefficients, BLOCKS, THREADS, kx_d, ky_d, gam, a, b, c, z_d, P);
        cudaDeviceSynchronize();
        if (P.variable_density == 0) {
            solve_pressure(y0_d, y0_d, p_d, z_d, gam, a, b, c, d, l, uu, yy, din, dout, pti, pto, nzy_d, P);
        } else {
            double err;
            int it;
            solve_pressure_iterative(y0_d, y0_d, p_d, z_d, gam, a, b, c, d, l, uu, yy, din, dout, pti, pto, nzy_d, P, &err, &it);
            printf("ITERATIONS=%d ERROR=%.17g\n", it, err);
        }
        cudaDeviceSynchronize();
        cudaMemcpy(out, p_d, N * 8, cudaMemcpyDeviceToHost);
        return write_bin(outdir, "p.bin", out, N) ? 1 : 0;
    }
    fprintf(stderr, "ref_driver: unknown mode %s\n", mode);
    return 2;
}
