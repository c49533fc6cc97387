/*
 * FP64 stand-in for the subset of the FFTW3 API that the reference's image code calls
 * (src/Image.cpp: rfft, irfft, cfft; src/hsm/PSFCorr.cpp is not built).
 *
 * ORACLE-ONLY test infrastructure.  libfftw3 is not installed where the oracle is built,
 * so the reference C++ is linked against this file to run its drawImage path on the CPU.
 * The transform is an iterative mixed-radix Stockham FFT in double precision: radix-4 and
 * radix-2 passes first, then 3, then a direct pass for any other prime factor, with the
 * twiddles exp(2 pi i m / n) tabulated once per length (per thread) and exact integer
 * exponents (m = r k n / (ns p) < n).  Conventions are FFTW's:
 *   out[k] = sum_j in[j] exp(sign * 2 pi i j k / n),  unnormalised,
 * with FFTW's half-complex array layouts for r2c / c2r, including the padded in-place
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

/* exp(+2 pi i m / n) for m < n, cached per length (a few lengths per thread). */
#define TW_SLOTS 8
static __thread int tw_len[TW_SLOTS];
static __thread double complex *tw_tab[TW_SLOTS];
static __thread int tw_next;

static const double complex *twiddles(int n)
{
    for (int i = 0; i < TW_SLOTS; ++i)
        if (tw_len[i] == n && tw_tab[i]) return tw_tab[i];
    const int slot = tw_next;
    tw_next = (tw_next + 1) % TW_SLOTS;
    free(tw_tab[slot]);
    double complex *t = (double complex *)malloc(sizeof(double complex) * (size_t)n);
    for (int m = 0; m < n; ++m) {
        const double a = 2.0 * M_PI * (double)m / (double)n;
        t[m] = cos(a) + I * sin(a);
    }
    /* the quarter turns exactly */
    if (n % 4 == 0) { t[n / 4] = I; t[3 * n / 4] = -I; }
    if (n % 2 == 0) t[n / 2] = -1.0;
    t[0] = 1.0;
    tw_tab[slot] = t;
    tw_len[slot] = n;
    return t;
}

static int smallest_factor(int m)
{
    if (m % 4 == 0) return 4;
    if (m % 2 == 0) return 2;
    if (m % 3 == 0) return 3;
    for (int q = 5; q * q <= m; q += 2) if (m % q == 0) return q;
    return m;
}

/* In-place length-n DFT of x (contiguous) with scratch y (n values). */
static void fft_inplace(double complex *x, double complex *y, int n, int sign)
{
    if (n <= 1) return;
    const double complex *tw = twiddles(n);
    double complex *src = x, *dst = y;
    double complex vbuf[64], obuf[64];
    int ns = 1;
    while (ns < n) {
        const int p = smallest_factor(n / ns);
        const int nb = n / p;
        const int tstep = n / (ns * p);
        double complex *v = p <= 64 ? vbuf : (double complex *)malloc(sizeof(double complex) * p);
        double complex *o = p <= 64 ? obuf : (double complex *)malloc(sizeof(double complex) * p);
        for (int b = 0; b < nb; ++b) {
            const int k = b % ns;
            v[0] = src[b];
            for (int r = 1; r < p; ++r) {
                const double complex w = tw[(long)r * k * tstep % n];
                v[r] = src[b + r * nb] * (sign > 0 ? w : conj(w));
            }
            if (p == 2) {
                o[0] = v[0] + v[1];
                o[1] = v[0] - v[1];
            } else if (p == 4) {
                const double complex s0 = v[0] + v[2], s1 = v[0] - v[2];
                const double complex s2 = v[1] + v[3];
                const double complex d = v[1] - v[3];
                const double complex s3 = sign > 0 ? I * d : -I * d;
                o[0] = s0 + s2; o[1] = s1 + s3; o[2] = s0 - s2; o[3] = s1 - s3;
            } else {
                /* direct p-point DFT; exp(2 pi i m / p) = tw[m n / p] */
                const int step = n / p;
                for (int q = 0; q < p; ++q) {
                    double complex acc = 0;
                    for (int r = 0; r < p; ++r) {
                        const double complex w = tw[(long)((long)r * q % p) * step];
                        acc += v[r] * (sign > 0 ? w : conj(w));
                    }
                    o[q] = acc;
                }
            }
            const int base = (b / ns) * ns * p + k;
            for (int q = 0; q < p; ++q) dst[base + q * ns] = o[q];
        }
        if (v != vbuf) free(v);
        if (o != obuf) free(o);
        double complex *t = src; src = dst; dst = t;
        ns *= p;
    }
    if (src != x) memcpy(x, src, sizeof(double complex) * (size_t)n);
}

/* One 1-d transform of n points read with stride `is` and written with stride `os`. */
static void fft1(const double complex *in, int is, double complex *out, int os, int n, int sign)
{
    double complex *x = (double complex *)malloc(sizeof(double complex) * (size_t)n * 2);
    double complex *y = x + n;
    for (int j = 0; j < n; ++j) x[j] = in[(long)j * is];
    fft_inplace(x, y, n, sign);
    for (int j = 0; j < n; ++j) out[(long)j * os] = x[j];
    free(x);
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
