/*
 * cpu_fft.h -- FP64 complex FFT of arbitrary length for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  Used by the CPU restatement of the solver
 * (wf_oracle.c) and by the cuFFT stand-in that lets the reference's own
 * kernel sources run on the host (ref_shim/).  Never linked into the product.
 *
 * Conventions follow cuFFT's Z2Z transforms as called by the reference
 * (src/cu/pressure.cu:527-540): forward = sum x_n exp(-2 pi i n k / N),
 * inverse = sum X_k exp(+2 pi i n k / N), both unnormalised.
 *
 * Algorithm: recursive mixed-radix Cooley-Tukey (decimation in time) over the
 * prime factors of N when every factor is <= 13, otherwise Bluestein's
 * chirp-z transform with a power-of-two inner transform of length >= 2N-1.
 * Twiddles and chirps are computed in long double.
 */
#ifndef WF_CPU_FFT_H
#define WF_CPU_FFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cfft_plan cfft_plan;

/* Plan a length-n transform (n >= 1). Returns NULL on allocation failure. */
cfft_plan *cfft_plan_create(int n);
void cfft_plan_destroy(cfft_plan *plan);

/* In-place transform of n interleaved complex values (re, im, re, im, ...).
 * sign = -1 forward, +1 inverse.  Thread-safe for distinct data buffers. */
void cfft_exec(const cfft_plan *plan, double *data, int sign);

/* howmany independent 2-D transforms of n0 x n1 slices (n1 fastest), each
 * slice dist = n0*n1 complex values apart, out-of-place allowed (in == out ok). */
void cfft_2d_many(int n0, int n1, int howmany, const double *in, double *out, int sign);

#ifdef __cplusplus
}
#endif

#endif
