/*
 * FP64 stand-in for the subset of the FFTW3 API that the reference's image code calls
 * (src/Image.cpp: rfft, irfft, cfft; src/hsm/PSFCorr.cpp is not built).
 *
 * ORACLE-ONLY test infrastructure.  libfftw3 is not installed on this machine, so the
 * reference C++ is linked against this file to be able to run its drawImage path on the
 * CPU.  The transform is a plain recursive mixed-radix Cooley-Tukey FFT in double
 * precision (radix 2 and 3 butterflies, an O(n*p) DFT for any other prime factor p), with
 * FFTW's sign and normalisation conventions:
 *   out[k] = sum_j in[j] exp(sign * 2 pi i j k / n),  unnormalised,
 * and FFTW's half-complex array layouts for r2c / c2r, including the padded in-place
 * layout (real rows of stride 2*(n1/2+1) when in == out).
 * It is checked against numpy.fft (pocketfft, FP64) in tests/test_oracle_fft_shim.py.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

enum { KIND_C2C = 0, KIND_R2C = 1, KIND_C2R = 2 };

struct fftw_plan_s {
    int kind;
    int rank;
    int n0, n1;
    int sign;
    void *in;
    void *out;
};

static void dft_rec(const double complex *x, double complex *y, int n, int stride, int sign,
                    double complex *scratch)
{
    if (n == 1) { y[0] = x[0]; return; }
    int p = 0;
    if (n % 2 == 0) p = 2;
    else if (n % 3 == 0) p = 3;
    else {
        for (int q = 5; q * q <= n; q += 2) if (n % q == 0) { p = q; break; }
        if (p == 0) p = n;
    }
    const int m = n / p;
    if (m == 1) {
        /* direct DFT of a prime length */
        for (int k = 0; k < n; ++k) {
            double complex acc = 0;
            for (int j = 0; j < n; ++j) {
                double ang = sign * 2.0 * M_PI * (double)((long)j * k % n) / n;
                acc += x[j * stride] * (cos(ang) + I * sin(ang));
            }
            scratch[k] = acc;
        }
        memcpy(y, scratch, sizeof(double complex) * n);
        return;
    }
    /* sub-transforms of the p decimated sequences, stored contiguously in y */
    for (int r = 0; r < p; ++r)
        dft_rec(x + r * stride, y + r * m, m, stride * p, sign, scratch);
    /* combine: Y[k + q m] = sum_r W_n^{r (k + q m)} Y_r[k] */
    double complex tmp[64];
    double complex *t = (p <= 64) ? tmp : (double complex *)malloc(sizeof(double complex) * p);
    for (int k = 0; k < m; ++k) {
        for (int r = 0; r < p; ++r) {
            double ang = sign * 2.0 * M_PI * (double)r * k / n;
            t[r] = y[r * m + k] * (cos(ang) + I * sin(ang));
        }
        for (int q = 0; q < p; ++q) {
            double complex acc = 0;
            for (int r = 0; r < p; ++r) {
                double ang = sign * 2.0 * M_PI * (double)((long)r * q % p) / p;
                acc += t[r] * (cos(ang) + I * sin(ang));
            }
            scratch[k + q * m] = acc;
        }
    }
    memcpy(y, scratch, sizeof(double complex) * n);
    if (t != tmp) free(t);
}

/* One 1-d transform of n points read with stride `is` and written with stride `os`. */
static void fft1(const double complex *in, int is, double complex *out, int os, int n, int sign)
{
    double complex *x = (double complex *)malloc(sizeof(double complex) * n);
    double complex *y = (double complex *)malloc(sizeof(double complex) * n);
    double complex *s = (double complex *)malloc(sizeof(double complex) * n);
    for (int j = 0; j < n; ++j) x[j] = in[(long)j * is];
    dft_rec(x, y, n, 1, sign, s);
    for (int j = 0; j < n; ++j) out[(long)j * os] = y[j];
    free(x); free(y); free(s);
}

static fftw_plan make_plan(int kind, int rank, int n0, int n1, int sign, void *in, void *out)
{
    fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fftw_plan_s));
    p->kind = kind; p->rank = rank; p->n0 = n0; p->n1 = n1; p->sign = sign;
    p->in = in; p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{ (void)flags; return make_plan(KIND_C2C, 1, 1, n, sign, in, out); }

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags)
{ (void)flags; return make_plan(KIND_C2C, 2, n0, n1, sign, in, out); }

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags)
{ (void)flags; return make_plan(KIND_R2C, 2, n0, n1, -1, in, out); }

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags)
{ (void)flags; return make_plan(KIND_C2R, 2, n0, n1, +1, in, out); }

void fftw_destroy_plan(fftw_plan p) { free(p); }

void fftw_execute(const fftw_plan p)
{
    const int n0 = p->n0, n1 = p->n1;
    const int h1 = n1 / 2 + 1;
    if (p->kind == KIND_C2C) {
        double complex *a = (double complex *)malloc(sizeof(double complex) * (size_t)n0 * n1);
        memcpy(a, p->in, sizeof(double complex) * (size_t)n0 * n1);
        for (int r = 0; r < n0; ++r) fft1(a + (long)r * n1, 1, a + (long)r * n1, 1, n1, p->sign);
        if (p->rank == 2)
            for (int c = 0; c < n1; ++c) fft1(a + c, n1, a + c, n1, n0, p->sign);
        memcpy(p->out, a, sizeof(double complex) * (size_t)n0 * n1);
        free(a);
    } else if (p->kind == KIND_R2C) {
        const int inplace = (p->in == p->out);
        const int rs = inplace ? 2 * h1 : n1;            /* real row stride (doubles) */
        const double *x = (const double *)p->in;
        double complex *a = (double complex *)malloc(sizeof(double complex) * (size_t)n0 * n1);
        for (int r = 0; r < n0; ++r)
            for (int c = 0; c < n1; ++c) a[(long)r * n1 + c] = x[(long)r * rs + c];
        for (int r = 0; r < n0; ++r) fft1(a + (long)r * n1, 1, a + (long)r * n1, 1, n1, -1);
        for (int c = 0; c < h1; ++c) fft1(a + c, n1, a + c, n1, n0, -1);
        double complex *o = (double complex *)p->out;
        for (int r = 0; r < n0; ++r)
            for (int c = 0; c < h1; ++c) o[(long)r * h1 + c] = a[(long)r * n1 + c];
        free(a);
    } else {
        /* c2r: inverse-transform the n1/2+1 stored columns along the first axis, then
           each row along the second axis with its Hermitian extension
           row[c] = conj(row[n1 - c]) for c > n1/2, and keep the real part. */
        const int inplace = (p->in == p->out);
        const int rs = inplace ? 2 * h1 : n1;
        const double complex *k = (const double complex *)p->in;
        double complex *a = (double complex *)malloc(sizeof(double complex) * (size_t)n0 * n1);
        double complex *col = (double complex *)malloc(sizeof(double complex) * (size_t)n0 * h1);
        memcpy(col, k, sizeof(double complex) * (size_t)n0 * h1);
        for (int c = 0; c < h1; ++c) fft1(col + c, h1, col + c, h1, n0, +1);
        for (int r = 0; r < n0; ++r) {
            double complex *row = a + (long)r * n1;
            for (int c = 0; c < h1; ++c) row[c] = col[(long)r * h1 + c];
            for (int c = h1; c < n1; ++c) row[c] = conj(col[(long)r * h1 + (n1 - c)]);
            fft1(row, 1, row, 1, n1, +1);
        }
        double *x = (double *)p->out;
        for (int r = 0; r < n0; ++r)
            for (int c = 0; c < n1; ++c) x[(long)r * rs + c] = creal(a[(long)r * n1 + c]);
        free(a); free(col);
    }
}
