/*
 * cpu_fft.c -- FP64 complex FFT of arbitrary length (CPU oracle helper).
 * TEST INFRASTRUCTURE ONLY; see cpu_fft.h.
 */
#include "cpu_fft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct cfft_plan {
    int n;
    int nfac;
    int fac[40];
    double *tw;          /* exp(-2 pi i j / n), j < n  (forward twiddles) */
    /* Bluestein */
    int bluestein;
    int m;               /* power-of-two inner length */
    cfft_plan *inner;
    double *chirp;       /* exp(-i pi j^2 / n), j < n (forward chirp) */
    double *filt_f;      /* FFT_m of the forward filter */
    double *filt_i;      /* FFT_m of the inverse filter */
};

static const long double PI_L = 3.141592653589793238462643383279502884L;

static int factorize(int n, int *fac)
{
    int nf = 0;
    /* radix 4 first keeps recursion shallow for powers of two */
    while (n % 4 == 0) { fac[nf++] = 4; n /= 4; }
    for (int p = 2; p * p <= n; p++)
        while (n % p == 0) { fac[nf++] = p; n /= p; }
    if (n > 1) fac[nf++] = n;
    return nf;
}

static void twiddles(double *tw, int n)
{
    for (int j = 0; j < n; j++) {
        long double a = -2.0L * PI_L * (long double)j / (long double)n;
        tw[2 * j] = (double)cosl(a);
        tw[2 * j + 1] = (double)sinl(a);
    }
}

/* Recursive DIT: out[0..n) <- DFT of in[0], in[stride], ... (n values). */
static void rec(const cfft_plan *P, const double *in, double *out, int n, int stride,
                int fi, int sign)
{
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    const int p = P->fac[fi];
    const int m = n / p;
    for (int r = 0; r < p; r++)
        rec(P, in + 2 * r * stride, out + 2 * r * m, m, stride * p, fi + 1, sign);
    const int N = P->n;
    const int step_n = N / n;   /* W_n^x = tw[x * step_n] */
    const int step_p = N / p;   /* W_p^x = tw[x * step_p] */
    double tr[64], ti[64];
    double *br = (p > 64) ? (double *)malloc(sizeof(double) * 2 * p) : NULL;
    double *xr = br ? br : tr;
    double *xi = br ? br + p : ti;
    for (int k = 0; k < m; k++) {
        for (int r = 0; r < p; r++) {
            const double yr = out[2 * (r * m + k)], yi = out[2 * (r * m + k) + 1];
            const long long e = ((long long)r * k * step_n) % N;
            const double c = P->tw[2 * e], s = -sign * P->tw[2 * e + 1];
            xr[r] = yr * c - yi * s;
            xi[r] = yr * s + yi * c;
        }
        for (int q = 0; q < p; q++) {
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; r++) {
                const long long e = ((long long)r * q * step_p) % N;
                const double c = P->tw[2 * e], s = -sign * P->tw[2 * e + 1];
                sr += xr[r] * c - xi[r] * s;
                si += xr[r] * s + xi[r] * c;
            }
            out[2 * (k + q * m)] = sr;
            out[2 * (k + q * m) + 1] = si;
        }
    }
    free(br);
}

static void exec_direct(const cfft_plan *P, double *data, int sign)
{
    double *tmp = (double *)malloc(sizeof(double) * 2 * P->n);
    rec(P, data, tmp, P->n, 1, 0, sign);
    memcpy(data, tmp, sizeof(double) * 2 * P->n);
    free(tmp);
}

cfft_plan *cfft_plan_create(int n)
{
    if (n < 1) return NULL;
    cfft_plan *P = (cfft_plan *)calloc(1, sizeof(cfft_plan));
    if (!P) return NULL;
    P->n = n;
    P->nfac = factorize(n, P->fac);
    int maxf = 1;
    for (int i = 0; i < P->nfac; i++) if (P->fac[i] > maxf) maxf = P->fac[i];
    P->tw = (double *)malloc(sizeof(double) * 2 * n);
    twiddles(P->tw, n);
    if (maxf > 13) {
        P->bluestein = 1;
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        P->m = m;
        P->inner = cfft_plan_create(m);
        P->chirp = (double *)malloc(sizeof(double) * 2 * n);
        for (int j = 0; j < n; j++) {
            const long long jj = ((long long)j * j) % (2LL * n);
            const long double a = -PI_L * (long double)jj / (long double)n;
            P->chirp[2 * j] = (double)cosl(a);
            P->chirp[2 * j + 1] = (double)sinl(a);
        }
        /* filter b_j = conj(chirp_j) for the forward sign, chirp_j for inverse */
        P->filt_f = (double *)calloc(2 * m, sizeof(double));
        P->filt_i = (double *)calloc(2 * m, sizeof(double));
        for (int j = 0; j < n; j++) {
            const double c = P->chirp[2 * j], s = P->chirp[2 * j + 1];
            P->filt_f[2 * j] = c;  P->filt_f[2 * j + 1] = -s;
            P->filt_i[2 * j] = c;  P->filt_i[2 * j + 1] = s;
            if (j > 0) {
                P->filt_f[2 * (m - j)] = c;  P->filt_f[2 * (m - j) + 1] = -s;
                P->filt_i[2 * (m - j)] = c;  P->filt_i[2 * (m - j) + 1] = s;
            }
        }
        cfft_exec(P->inner, P->filt_f, -1);
        cfft_exec(P->inner, P->filt_i, -1);
    }
    return P;
}

void cfft_plan_destroy(cfft_plan *P)
{
    if (!P) return;
    if (P->inner) cfft_plan_destroy(P->inner);
    free(P->tw);
    free(P->chirp);
    free(P->filt_f);
    free(P->filt_i);
    free(P);
}

static void exec_bluestein(const cfft_plan *P, double *data, int sign)
{
    const int n = P->n, m = P->m;
    double *a = (double *)calloc(2 * m, sizeof(double));
    /* chirp for this sign: forward uses chirp, inverse its conjugate */
    for (int j = 0; j < n; j++) {
        const double c = P->chirp[2 * j], s = sign < 0 ? P->chirp[2 * j + 1] : -P->chirp[2 * j + 1];
        const double xr = data[2 * j], xi = data[2 * j + 1];
        a[2 * j] = xr * c - xi * s;
        a[2 * j + 1] = xr * s + xi * c;
    }
    cfft_exec(P->inner, a, -1);
    const double *F = sign < 0 ? P->filt_f : P->filt_i;
    for (int j = 0; j < m; j++) {
        const double ar = a[2 * j], ai = a[2 * j + 1];
        a[2 * j] = ar * F[2 * j] - ai * F[2 * j + 1];
        a[2 * j + 1] = ar * F[2 * j + 1] + ai * F[2 * j];
    }
    cfft_exec(P->inner, a, +1);
    const double inv_m = 1.0 / (double)m;
    for (int k = 0; k < n; k++) {
        const double c = P->chirp[2 * k], s = sign < 0 ? P->chirp[2 * k + 1] : -P->chirp[2 * k + 1];
        const double yr = a[2 * k] * inv_m, yi = a[2 * k + 1] * inv_m;
        data[2 * k] = yr * c - yi * s;
        data[2 * k + 1] = yr * s + yi * c;
    }
    free(a);
}

void cfft_exec(const cfft_plan *P, double *data, int sign)
{
    if (P->n == 1) return;
    if (P->bluestein) exec_bluestein(P, data, sign);
    else exec_direct(P, data, sign);
}

void cfft_2d_many(int n0, int n1, int howmany, const double *in, double *out, int sign)
{
    cfft_plan *p0 = cfft_plan_create(n0);
    cfft_plan *p1 = cfft_plan_create(n1);
    const size_t slice = (size_t)n0 * n1;
    if (out != in) memcpy(out, in, sizeof(double) * 2 * slice * howmany);
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        double *col = (double *)malloc(sizeof(double) * 2 * n0);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int h = 0; h < howmany; h++) {
            double *s = out + 2 * slice * h;
            for (int a = 0; a < n0; a++) cfft_exec(p1, s + 2 * (size_t)a * n1, sign);
            for (int b = 0; b < n1; b++) {
                for (int a = 0; a < n0; a++) {
                    col[2 * a] = s[2 * ((size_t)a * n1 + b)];
                    col[2 * a + 1] = s[2 * ((size_t)a * n1 + b) + 1];
                }
                cfft_exec(p0, col, sign);
                for (int a = 0; a < n0; a++) {
                    s[2 * ((size_t)a * n1 + b)] = col[2 * a];
                    s[2 * ((size_t)a * n1 + b) + 1] = col[2 * a + 1];
                }
            }
        }
        free(col);
    }
    cfft_plan_destroy(p0);
    cfft_plan_destroy(p1);
}
