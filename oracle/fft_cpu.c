/*
 * fft_cpu.c -- FP64 CPU 2D real FFT for the oracle (test infrastructure only).
 *
 * Replaces FFTW3 (the reference links -lfftw3_mpi -lfftw3, Makefile:1-2; FFTW is
 * not vendored and not installed here) with a self-contained Stockham
 * radix-4/radix-2 complex FFT.  Twiddles are taken from long-double cos/sin
 * on one octant and completed by exact symmetries.
 *
 * 2D r2c (the semantics of fftw_mpi_plan_dft_r2c_2d, main.c:193, executed in
 * fft.c:13): rows are transformed two at a time as one complex FFT
 * (z = x_r + i x_{r+1}), split into the two half spectra, then every one of
 * the n1/2+1 columns gets a complex FFT of length n0.
 * 2D c2r (main.c:194, fft.c:24): columns first (complex inverse), then rows two
 * at a time; the j = 0 and j = n1/2 bins contribute only their real parts.
 */
#include "fft_cpu.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* twiddle tables, cached per length                                          */
/* ------------------------------------------------------------------------- */

#define FFTC_MAXLOG 16

static double *g_tw[FFTC_MAXLOG + 1];
static pthread_mutex_t g_tw_lock = PTHREAD_MUTEX_INITIALIZER;

static int ilog2i(int n)
{
    int l = 0;
    while ((1 << l) < n) l++;
    return ((1 << l) == n) ? l : -1;
}

/* w[k] = exp(-2 pi i k / n), k in [0, n), interleaved. */
static const double *twiddles(int n)
{
    int l = ilog2i(n);
    if (l < 0 || l > FFTC_MAXLOG) return NULL;
    pthread_mutex_lock(&g_tw_lock);
    if (!g_tw[l]) {
        double *w = (double *)malloc(sizeof(double) * 2 * (size_t)n);
        if (w) {
            int q = n / 4, e = n / 8;
            double *c = (double *)malloc(sizeof(double) * (size_t)(q + 1));
            double *s = (double *)malloc(sizeof(double) * (size_t)(q + 1));
            const long double twopi = 6.283185307179586476925286766559005768L;
            if (n >= 8) {
                for (int k = 0; k <= e; k++) {
                    long double a = twopi * (long double)k / (long double)n;
                    c[k] = (double)cosl(a);
                    s[k] = (double)sinl(a);
                }
                for (int k = e + 1; k <= q; k++) { c[k] = s[q - k]; s[k] = c[q - k]; }
            } else {
                for (int k = 0; k <= q; k++) {
                    long double a = twopi * (long double)k / (long double)n;
                    c[k] = (double)cosl(a);
                    s[k] = (double)sinl(a);
                }
                if (q >= 1) { c[q] = 0.0; s[q] = 1.0; }
            }
            for (int k = 0; k < n; k++) {
                double re, im;
                int kk = k;
                int neg = 0;
                if (kk >= n / 2) { kk -= n / 2; neg = 1; }
                if (kk <= q) { re = c[kk]; im = -s[kk]; }
                else { re = -s[kk - q]; im = -c[kk - q]; }
                if (neg) { re = -re; im = -im; }
                w[2 * k] = re;
                w[2 * k + 1] = im;
            }
            free(c);
            free(s);
            g_tw[l] = w;
        }
    }
    pthread_mutex_unlock(&g_tw_lock);
    return g_tw[l];
}

/* ------------------------------------------------------------------------- */
/* 1D Stockham autosort FFT (decimation in time), radix 4 with one radix-2    */
/* stage when log2(n) is odd.  x holds the data on entry and on exit; y is a  */
/* scratch buffer of the same size.                                           */
/* ------------------------------------------------------------------------- */

/* 0: radix-4 stages, two real rows per complex transform; 1: radix-2 stages, one
 * real row per complex transform (a second rounding order of the same DFT) */
static int g_variant = 0;
void fftc_set_variant(int v) { g_variant = v ? 1 : 0; }
int fftc_get_variant(void) { return g_variant; }

static void stockham(int n, double *x, double *y, int sign)
{
    const double *tw = twiddles(n);
    double *src = x, *dst = y;
    int Ns = 1;
    if (n <= 1) return;
    while (Ns < n) {
        int rem = n / Ns;
        int R = (g_variant == 0 && rem % 4 == 0) ? 4 : 2;
        int m = n / R;                  /* butterflies */
        int step = n / (Ns * R);        /* twiddle stride */
        for (int b = 0; b < m / Ns; b++) {
            for (int k = 0; k < Ns; k++) {
                int j = b * Ns + k;
                int obase = b * Ns * R + k;
                if (R == 4) {
                    double a0r = src[2 * (j)],         a0i = src[2 * (j) + 1];
                    double a1r = src[2 * (j + m)],     a1i = src[2 * (j + m) + 1];
                    double a2r = src[2 * (j + 2 * m)], a2i = src[2 * (j + 2 * m) + 1];
                    double a3r = src[2 * (j + 3 * m)], a3i = src[2 * (j + 3 * m) + 1];
                    if (k) {
                        int t1 = k * step, t2 = 2 * k * step, t3 = 3 * k * step;
                        /* forward uses w = exp(-i..) as stored; inverse its conjugate */
                        double w1r = tw[2 * t1], w1i = (sign > 0) ? -tw[2 * t1 + 1] : tw[2 * t1 + 1];
                        double w2r = tw[2 * t2], w2i = (sign > 0) ? -tw[2 * t2 + 1] : tw[2 * t2 + 1];
                        double w3r = tw[2 * t3], w3i = (sign > 0) ? -tw[2 * t3 + 1] : tw[2 * t3 + 1];
                        double tr;
                        tr = a1r * w1r - a1i * w1i; a1i = a1r * w1i + a1i * w1r; a1r = tr;
                        tr = a2r * w2r - a2i * w2i; a2i = a2r * w2i + a2i * w2r; a2r = tr;
                        tr = a3r * w3r - a3i * w3i; a3i = a3r * w3i + a3i * w3r; a3r = tr;
                    }
                    double t0r = a0r + a2r, t0i = a0i + a2i;
                    double t1r = a0r - a2r, t1i = a0i - a2i;
                    double t2r = a1r + a3r, t2i = a1i + a3i;
                    double t3r = a1r - a3r, t3i = a1i - a3i;
                    /* forward: X1 = t1 - i t3, X3 = t1 + i t3 ; inverse: swapped */
                    double x1r, x1i, x3r, x3i;
                    if (sign < 0) { x1r = t1r + t3i; x1i = t1i - t3r; x3r = t1r - t3i; x3i = t1i + t3r; }
                    else          { x1r = t1r - t3i; x1i = t1i + t3r; x3r = t1r + t3i; x3i = t1i - t3r; }
                    dst[2 * (obase)]              = t0r + t2r;
                    dst[2 * (obase) + 1]          = t0i + t2i;
                    dst[2 * (obase + Ns)]         = x1r;
                    dst[2 * (obase + Ns) + 1]     = x1i;
                    dst[2 * (obase + 2 * Ns)]     = t0r - t2r;
                    dst[2 * (obase + 2 * Ns) + 1] = t0i - t2i;
                    dst[2 * (obase + 3 * Ns)]     = x3r;
                    dst[2 * (obase + 3 * Ns) + 1] = x3i;
                } else {
                    double a0r = src[2 * (j)],     a0i = src[2 * (j) + 1];
                    double a1r = src[2 * (j + m)], a1i = src[2 * (j + m) + 1];
                    if (k) {
                        int t1 = k * step;
                        double w1r = tw[2 * t1];
                        double w1i = (sign > 0) ? -tw[2 * t1 + 1] : tw[2 * t1 + 1];
                        double tr = a1r * w1r - a1i * w1i;
                        a1i = a1r * w1i + a1i * w1r;
                        a1r = tr;
                    }
                    dst[2 * (obase)]          = a0r + a1r;
                    dst[2 * (obase) + 1]      = a0i + a1i;
                    dst[2 * (obase + Ns)]     = a0r - a1r;
                    dst[2 * (obase + Ns) + 1] = a0i - a1i;
                }
            }
        }
        { double *t = src; src = dst; dst = t; }
        Ns *= R;
    }
    if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

void fftc_c2c_1d(int n, double *z, int sign)
{
    double *y = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    if (!y) return;
    stockham(n, z, y, sign);
    free(y);
}

/* ------------------------------------------------------------------------- */
/* tiny pthread parallel-for                                                  */
/* ------------------------------------------------------------------------- */

static int g_threads = 1;

void fftc_set_threads(int nthreads) { g_threads = nthreads < 1 ? 1 : (nthreads > 256 ? 256 : nthreads); }
int fftc_get_threads(void) { return g_threads; }

typedef void (*range_fn)(void *ctx, int lo, int hi, double *scratch);

typedef struct {
    range_fn fn;
    void *ctx;
    int lo, hi;
    size_t scratch_doubles;
} par_job;

static void *par_worker(void *arg)
{
    par_job *j = (par_job *)arg;
    double *s = (double *)malloc(sizeof(double) * j->scratch_doubles);
    if (s) {
        j->fn(j->ctx, j->lo, j->hi, s);
        free(s);
    }
    return NULL;
}

/* Runs fn over [0, count) split in contiguous chunks of multiples of `grain`. */
static void parallel_for(range_fn fn, void *ctx, int count, int grain, size_t scratch_doubles)
{
    int nt = g_threads;
    int units = (count + grain - 1) / grain;
    if (nt > units) nt = units;
    if (nt <= 1) {
        double *s = (double *)malloc(sizeof(double) * scratch_doubles);
        if (!s) return;
        fn(ctx, 0, count, s);
        free(s);
        return;
    }
    pthread_t th[256];
    par_job jobs[256];
    int per = (units + nt - 1) / nt;
    int started = 0;
    for (int t = 0; t < nt; t++) {
        int lo = t * per * grain, hi = (t + 1) * per * grain;
        if (hi > count) hi = count;
        if (lo >= hi) break;
        jobs[t].fn = fn; jobs[t].ctx = ctx; jobs[t].lo = lo; jobs[t].hi = hi;
        jobs[t].scratch_doubles = scratch_doubles;
        if (pthread_create(&th[t], NULL, par_worker, &jobs[t]) != 0) {
            par_worker(&jobs[t]);
            th[t] = 0;
        }
        started = t + 1;
    }
    for (int t = 0; t < started; t++)
        if (th[t]) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------- */
/* 2D real transforms                                                         */
/* ------------------------------------------------------------------------- */

struct fftc_plan {
    int n0, n1;
};

fftc_plan *fftc_plan_2d(int n0, int n1)
{
    if (ilog2i(n0) < 2 || ilog2i(n1) < 2 || ilog2i(n0) > FFTC_MAXLOG || ilog2i(n1) > FFTC_MAXLOG)
        return NULL;
    fftc_plan *p = (fftc_plan *)malloc(sizeof(*p));
    if (!p) return NULL;
    p->n0 = n0;
    p->n1 = n1;
    twiddles(n0);
    twiddles(n1);
    return p;
}

void fftc_destroy(fftc_plan *p) { free(p); }

typedef struct {
    int n0, n1;
    double *data;
    int sign;
} pass_ctx;

#define COLBLK 8

/* variant 1: one real row x (n1 + 2 doubles) -> its half spectrum, in place */
static void row_r2c_single(int n1, double *x, double *z, double *y)
{
    for (int n = 0; n < n1; n++) { z[2 * n] = x[n]; z[2 * n + 1] = 0.0; }
    stockham(n1, z, y, -1);
    for (int k = 0; k <= n1 / 2; k++) { x[2 * k] = z[2 * k]; x[2 * k + 1] = z[2 * k + 1]; }
}

/* variant 1: one half spectrum -> its real row, in place (imaginary parts of the
 * k = 0 and k = n1/2 bins ignored) */
static void row_c2r_single(int n1, double *x, double *z, double *y)
{
    int h = n1 / 2;
    z[0] = x[0]; z[1] = 0.0;
    z[2 * h] = x[2 * h]; z[2 * h + 1] = 0.0;
    for (int k = 1; k < h; k++) {
        z[2 * k] = x[2 * k];            z[2 * k + 1] = x[2 * k + 1];
        z[2 * (n1 - k)] = x[2 * k];     z[2 * (n1 - k) + 1] = -x[2 * k + 1];
    }
    stockham(n1, z, y, +1);
    for (int n = 0; n < n1; n++) x[n] = z[2 * n];
}

/* rows [lo, hi) (even), forward: pack two rows, FFT, split into half spectra */
static void rows_r2c(void *vctx, int lo, int hi, double *s)
{
    pass_ctx *c = (pass_ctx *)vctx;
    int n1 = c->n1, h = n1 / 2, rs = n1 + 2;
    double *z = s, *y = s + 2 * (size_t)n1;
    if (g_variant) {
        for (int r = lo; r < hi; r++) row_r2c_single(n1, c->data + (size_t)r * rs, z, y);
        return;
    }
    for (int r = lo; r < hi; r += 2) {
        double *xa = c->data + (size_t)r * rs;
        double *xb = xa + rs;
        for (int n = 0; n < n1; n++) { z[2 * n] = xa[n]; z[2 * n + 1] = xb[n]; }
        stockham(n1, z, y, -1);
        for (int k = 0; k <= h; k++) {
            int nk = (n1 - k) & (n1 - 1);
            double zr = z[2 * k], zi = z[2 * k + 1];
            double wr = z[2 * nk], wi = z[2 * nk + 1];
            /* A = (Z[k] + conj Z[n-k]) / 2 ; B = (Z[k] - conj Z[n-k]) / (2i) */
            xa[2 * k]     = 0.5 * (zr + wr);
            xa[2 * k + 1] = 0.5 * (zi - wi);
            xb[2 * k]     = 0.5 * (zi + wi);
            xb[2 * k + 1] = 0.5 * (wr - zr);
        }
    }
}

/* rows [lo, hi) (even), inverse: Hermitian-extend two half spectra, inverse FFT */
static void rows_c2r(void *vctx, int lo, int hi, double *s)
{
    pass_ctx *c = (pass_ctx *)vctx;
    int n1 = c->n1, h = n1 / 2, rs = n1 + 2;
    double *z = s, *y = s + 2 * (size_t)n1;
    if (g_variant) {
        for (int r = lo; r < hi; r++) row_c2r_single(n1, c->data + (size_t)r * rs, z, y);
        return;
    }
    for (int r = lo; r < hi; r += 2) {
        double *xa = c->data + (size_t)r * rs;
        double *xb = xa + rs;
        /* k = 0 and k = h: real parts only (c2r convention) */
        z[0] = xa[0];
        z[1] = xb[0];
        z[2 * h] = xa[2 * h];
        z[2 * h + 1] = xb[2 * h];
        for (int k = 1; k < h; k++) {
            double ar = xa[2 * k], ai = xa[2 * k + 1];
            double br = xb[2 * k], bi = xb[2 * k + 1];
            /* Z[k] = A + iB ; Z[n-k] = conj(A) + i conj(B) */
            z[2 * k]            = ar - bi;
            z[2 * k + 1]        = ai + br;
            z[2 * (n1 - k)]     = ar + bi;
            z[2 * (n1 - k) + 1] = br - ai;
        }
        stockham(n1, z, y, +1);
        for (int n = 0; n < n1; n++) { xa[n] = z[2 * n]; xb[n] = z[2 * n + 1]; }
    }
}

/* columns [lo, hi) of the complex view: gather COLBLK columns, FFT, scatter */
static void cols_c2c(void *vctx, int lo, int hi, double *s)
{
    pass_ctx *c = (pass_ctx *)vctx;
    int n0 = c->n0, h1 = c->n1 / 2 + 1;
    double *buf = s, *y = s + 2 * (size_t)n0 * COLBLK;
    for (int k0 = lo; k0 < hi; k0 += COLBLK) {
        int nb = hi - k0 < COLBLK ? hi - k0 : COLBLK;
        for (int i = 0; i < n0; i++) {
            const double *row = c->data + 2 * ((size_t)i * h1 + k0);
            for (int b = 0; b < nb; b++) {
                buf[2 * ((size_t)b * n0 + i)]     = row[2 * b];
                buf[2 * ((size_t)b * n0 + i) + 1] = row[2 * b + 1];
            }
        }
        for (int b = 0; b < nb; b++) stockham(n0, buf + 2 * (size_t)b * n0, y, c->sign);
        for (int i = 0; i < n0; i++) {
            double *row = c->data + 2 * ((size_t)i * h1 + k0);
            for (int b = 0; b < nb; b++) {
                row[2 * b]     = buf[2 * ((size_t)b * n0 + i)];
                row[2 * b + 1] = buf[2 * ((size_t)b * n0 + i) + 1];
            }
        }
    }
}

void fftc_r2c_2d(fftc_plan *p, double *data)
{
    pass_ctx c = {p->n0, p->n1, data, -1};
    parallel_for(rows_r2c, &c, p->n0, 2, 4 * (size_t)p->n1);
    parallel_for(cols_c2c, &c, p->n1 / 2 + 1, COLBLK, 2 * (size_t)p->n0 * (COLBLK + 1));
}

void fftc_c2r_2d(fftc_plan *p, double *data)
{
    pass_ctx c = {p->n0, p->n1, data, +1};
    parallel_for(cols_c2c, &c, p->n1 / 2 + 1, COLBLK, 2 * (size_t)p->n0 * (COLBLK + 1));
    parallel_for(rows_c2r, &c, p->n0, 2, 4 * (size_t)p->n1);
}
