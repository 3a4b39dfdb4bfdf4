/*
 * chns_oracle.c -- CPU restatement of the reference's ETD2RK CHNS step.
 *
 * TEST INFRASTRUCTURE ONLY (see chns_oracle.h).  Each function names the
 * reference file:line it restates.  Operand order of every floating-point
 * expression follows the reference (C99 complex arithmetic written out on
 * re/im pairs: real*complex scales both parts; I*k*z = (-k z.im, k z.re)).
 */
#include "chns_oracle.h"
#include "fft_cpu.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXBUF 16

struct orc_ctx {
    orc_params p;
    int nx, ny, ny2;
    size_t nc;       /* complex modes nx*ny2 */
    size_t nd;       /* doubles per buffer = 2*nc = nx*(ny+2) */
    double factor_x, factor_y, dealias;
    double ksqrmax;  /* kxmax^2 + kymax^2 (functions.c:54, main.c:57-58) */
    double gamma1, gamma2, gamma3, del;
    double *kx, *ky;
    fftc_plan *plan;
    double *w, *c1, *c2;                 /* state */
    double *nlw, *nl1, *nl2;             /* N(u) of the current stage */
    double *sw, *s1, *s2;                /* saved N(u) of stage 1 (cnl_z, cnl_phi*) */
    double *muF1, *muF2;                 /* cmuF1, cmuF2 */
    double *forc;                        /* spectrum of the forcing curl (extension) */
    double *b[MAXBUF];                   /* scratch, each nd doubles */
};

/* ------------------------------------------------------------------ */
/* helpers                                                              */
/* ------------------------------------------------------------------ */

static double *alloc_buf(size_t nd) { return (double *)calloc(nd, sizeof(double)); }

#define RE(a, k) ((a)[2 * (k)])
#define IM(a, k) ((a)[2 * (k) + 1])

static inline double ksq(const orc_ctx *c, int i, int j) { return c->kx[i] * c->kx[i] + c->ky[j] * c->ky[j]; }

/* fft.c:11-14 */
static void dfft(orc_ctx *c, double *a) { fftc_r2c_2d(c->plan, a); }

/* fft.c:16-31: c2r, then scale every one of the nx*(ny+2) reals by 1/(Nx*Ny) */
static void ifft(orc_ctx *c, double *a)
{
    double scale = 1.0 / ((double)c->nx * (double)c->ny);
    fftc_c2r_2d(c->plan, a);
    for (size_t k = 0; k < c->nd; k++) a[k] *= scale;
}

static void copy(const orc_ctx *c, const double *in, double *out) { memcpy(out, in, c->nd * sizeof(double)); }

/* functions.c:47-84: the sharp cut k^2 > dealias (:74-79), or with SMOOTH_FILTER
 * (:69-72) every mode scaled by exp(-36 (k^2/k^2max)^18), applied twice with a
 * rounding after each product */
static void truncation(orc_ctx *c, double *a)
{
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            double ksqr = ksq(c, i, j);
            if (c->p.filter) {
                double pp = ksqr / c->ksqrmax;
                double f = exp(-36.0 * pow(pp, 18));
                RE(a, k) *= f; IM(a, k) *= f;
                RE(a, k) *= f; IM(a, k) *= f;
            } else if (ksqr > c->dealias) {
                RE(a, k) = 0.0; IM(a, k) = 0.0;
            }
        }
}

/* out = I * kx * in  (nonlin.c:36, surface_tension.c:57, ...) */
static void ikx(orc_ctx *c, const double *in, double *out)
{
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            double a = RE(in, k), b = IM(in, k), q = c->kx[i];
            RE(out, k) = -(q * b);
            IM(out, k) = q * a;
        }
}

/* out = I * ky * in  (nonlin.c:37, ...) */
static void iky(orc_ctx *c, const double *in, double *out)
{
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            double a = RE(in, k), b = IM(in, k), q = c->ky[j];
            RE(out, k) = -(q * b);
            IM(out, k) = q * a;
        }
}

/* velocity.c:3-44: psi = w/k^2 (0 where k^2 <= 1e-12), ux = I ky psi, uy = -I kx psi */
static void get_velocity(orc_ctx *c, const double *w, double *ux, double *uy)
{
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            double ks = ksq(c, i, j), a, b;
            if (ks > 1e-12) { a = RE(w, k) / ks; b = IM(w, k) / ks; }
            else { a = 0.0; b = 0.0; }
            RE(ux, k) = -(c->ky[j] * b);
            IM(ux, k) = c->ky[j] * a;
            RE(uy, k) = c->kx[i] * b;
            IM(uy, k) = -(c->kx[i] * a);
        }
}

/* curl.c:16-31: w = I * (kx * uy - ky * ux) */
static void curl(orc_ctx *c, const double *ux, const double *uy, double *w)
{
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            double dr = c->kx[i] * RE(uy, k) - c->ky[j] * RE(ux, k);
            double di = c->kx[i] * IM(uy, k) - c->ky[j] * IM(ux, k);
            RE(w, k) = -di;
            IM(w, k) = dr;
        }
}

static void add_to(orc_ctx *c, double *acc, const double *x)
{
    for (size_t k = 0; k < c->nd; k++) acc[k] += x[k];
}

/* loops over the physical points j < ny of the padded real layout (IDXR) */
#define FOR_REAL(c, idx) \
    for (int i_ = 0; i_ < (c)->nx; i_++) \
        for (size_t idx = (size_t)i_ * ((c)->ny + 2), e_ = idx + (c)->ny; idx < e_; idx++)

/* ------------------------------------------------------------------ */
/* nonlinear terms                                                      */
/* ------------------------------------------------------------------ */

/* chem_potential.c:12-94 (ternary; the live branch :303-315) */
static void potential(orc_ctx *c)
{
    double *t1 = c->b[0], *t2 = c->b[1];
    double g1i = 1.0 / c->gamma1, g2i = 1.0 / c->gamma2, g3i = 1.0 / c->gamma3;
    double six_lam = 6.0 * c->p.xlambda;
    double fac = 2.0 * c->del / c->p.epsilon;
    copy(c, c->c1, t1);
    copy(c, c->c2, t2);
    truncation(c, t1);
    truncation(c, t2);
    ifft(c, t1);
    ifft(c, t2);
    FOR_REAL(c, k) {
        double a = t1[k], b = t2[k], d = (1.0 - a - b);
        double abd = a * b * d;
        double f1 = a * (1.0 - a) * (1.0 - 2.0 * a);
        double f2 = b * (1.0 - b) * (1.0 - 2.0 * b);
        double f3 = d * (1.0 - d) * (1.0 - 2.0 * d);
        double G1 = c->gamma1 * f1 + six_lam * abd * b * d;
        double G2 = c->gamma2 * f2 + six_lam * abd * a * d;
        double G3 = c->gamma3 * f3 + six_lam * abd * a * b;
        double m1 = (G1 - G2) * g2i + (G1 - G3) * g3i;
        double m2 = (G2 - G1) * g1i + (G2 - G3) * g3i;
        c->muF1[k] = m1 * fac;
        c->muF2[k] = m2 * fac;
    }
    dfft(c, c->muF1);
    dfft(c, c->muF2);
}

/* nonlin.c:13-381 with surface_tension.c:13-227; result in nlw, nl1, nl2 */
static void nonlin(orc_ctx *c)
{
    const int model = c->p.model;
    double *cux = c->b[2], *cuy = c->b[3], *tcux = c->b[4], *tcuy = c->b[5];
    double *tcwz = c->b[6], *A = c->b[7], *B = c->b[8], *C = c->b[9];
    double *cnlz = c->nlw;
    const double sg = c->p.sigma, ep = c->p.epsilon, lam = c->p.lambda;

    /* -(u . grad) w  (nonlin.c:30-101) */
    ikx(c, c->w, tcux);
    iky(c, c->w, tcuy);
    get_velocity(c, c->w, cux, cuy);
    truncation(c, cux); truncation(c, cuy);
    truncation(c, tcux); truncation(c, tcuy);
    ifft(c, cux); ifft(c, tcux);
    ifft(c, cuy); ifft(c, tcuy);
    FOR_REAL(c, k) cnlz[k] = cux[k] * tcux[k] + cuy[k] * tcuy[k];
    dfft(c, cnlz);
    for (size_t k = 0; k < c->nd; k++) cnlz[k] *= (-1.0);

    if (model == 1) {
        /* surface_tension.c:19-112 */
        copy(c, c->c1, A);
        truncation(c, A);
        ifft(c, A);
        FOR_REAL(c, k) A[k] = A[k] * (1.0 - A[k]) * (1.0 - 2.0 * A[k]);
        dfft(c, A);
        {
            double s1 = 1.5 * sg * ep, s2 = 24.0 * (sg / ep);
            for (int i = 0; i < c->nx; i++)
                for (int j = 0; j < c->ny2; j++) {
                    size_t k = (size_t)i * c->ny2 + j;
                    double q = s1 * ksq(c, i, j);
                    RE(A, k) = q * RE(c->c1, k) + s2 * RE(A, k);
                    IM(A, k) = q * IM(c->c1, k) + s2 * IM(A, k);
                }
        }
        ikx(c, c->c1, tcux);
        iky(c, c->c1, tcuy);
        truncation(c, tcux); truncation(c, tcuy);
        truncation(c, A);
        ifft(c, tcux); ifft(c, tcuy); ifft(c, A);
        FOR_REAL(c, k) { tcux[k] *= A[k]; tcuy[k] *= A[k]; }
        dfft(c, tcux);
        dfft(c, tcuy);
        curl(c, tcux, tcuy, tcwz);
        add_to(c, cnlz, tcwz);

        /* Cahn-Hilliard right-hand side (nonlin.c:174-254) */
        get_velocity(c, c->w, cux, cuy);
        copy(c, cux, tcux);
        copy(c, cuy, tcuy);
        ikx(c, c->c1, A);   /* tcphi */
        iky(c, c->c1, B);   /* ncphi */
        truncation(c, A); truncation(c, B);
        truncation(c, tcux); truncation(c, tcuy);
        ifft(c, A); ifft(c, B);
        ifft(c, tcux); ifft(c, tcuy);
        FOR_REAL(c, k) c->nl1[k] = (tcux[k] * A[k] + tcuy[k] * B[k]);
        dfft(c, c->nl1);
        copy(c, c->c1, A);
        truncation(c, A);
        ifft(c, A);
        FOR_REAL(c, k) A[k] = A[k] * (1.0 - A[k]) * (1.0 - 2.0 * A[k]);
        dfft(c, A);
        {
            double s = 24.0 * (sg / ep);
            for (int i = 0; i < c->nx; i++)
                for (int j = 0; j < c->ny2; j++) {
                    size_t k = (size_t)i * c->ny2 + j;
                    double q = s * ksq(c, i, j);
                    RE(A, k) = q * RE(A, k);
                    IM(A, k) = q * IM(A, k);
                }
            for (size_t k = 0; k < c->nc; k++) {
                RE(c->nl1, k) = -RE(c->nl1, k) - lam * RE(A, k);
                IM(c->nl1, k) = -IM(c->nl1, k) - lam * IM(A, k);
            }
        }
    } else if (model == 2) {
        const double g1 = c->gamma1, g2 = c->gamma2, g3 = c->gamma3;
        /* surface_tension.c:114-225 */
        copy(c, c->muF1, A);
        copy(c, c->muF2, B);
        {
            double s1 = 0.75 * g1 * ep, s2 = 0.75 * g2 * ep;
            for (int i = 0; i < c->nx; i++)
                for (int j = 0; j < c->ny2; j++) {
                    size_t k = (size_t)i * c->ny2 + j;
                    double ks = ksq(c, i, j);
                    double q1 = s1 * ks, q2 = s2 * ks;
                    RE(A, k) += q1 * RE(c->c1, k);
                    IM(A, k) += q1 * IM(c->c1, k);
                    RE(B, k) += q2 * RE(c->c2, k);
                    IM(B, k) += q2 * IM(c->c2, k);
                }
        }
        ikx(c, c->c1, tcux);
        iky(c, c->c1, tcuy);
        truncation(c, tcux); truncation(c, tcuy);
        truncation(c, A); truncation(c, B);
        ifft(c, tcux); ifft(c, tcuy);
        ifft(c, A); ifft(c, B);
        FOR_REAL(c, k) {
            tcux[k] *= ((1.0 + (g3 / g1)) * A[k] + (g3 / g2) * B[k]);
            tcuy[k] *= ((1.0 + (g3 / g1)) * A[k] + (g3 / g2) * B[k]);
        }
        dfft(c, tcux);
        dfft(c, tcuy);
        curl(c, tcux, tcuy, tcwz);
        add_to(c, cnlz, tcwz);
        ikx(c, c->c2, tcux);
        iky(c, c->c2, tcuy);
        truncation(c, tcux); truncation(c, tcuy);
        ifft(c, tcux); ifft(c, tcuy);
        FOR_REAL(c, k) {
            tcux[k] *= ((g3 / g1) * A[k] + (1.0 + (g3 / g2)) * B[k]);
            tcuy[k] *= ((g3 / g1) * A[k] + (1.0 + (g3 / g2)) * B[k]);
        }
        dfft(c, tcux);
        dfft(c, tcuy);
        curl(c, tcux, tcuy, tcwz);
        add_to(c, cnlz, tcwz);

        /* Cahn-Hilliard right-hand sides (nonlin.c:256-377) */
        get_velocity(c, c->w, cux, cuy);
        copy(c, cux, tcux);
        copy(c, cuy, tcuy);
        truncation(c, tcux); truncation(c, tcuy);
        ifft(c, tcux); ifft(c, tcuy);
        ikx(c, c->c1, A);
        iky(c, c->c1, B);
        truncation(c, A); truncation(c, B);
        ifft(c, A); ifft(c, B);
        FOR_REAL(c, k) c->nl1[k] = A[k] * tcux[k] + B[k] * tcuy[k];
        dfft(c, c->nl1);
        ikx(c, c->c2, A);
        iky(c, c->c2, B);
        truncation(c, A); truncation(c, B);
        ifft(c, A); ifft(c, B);
        FOR_REAL(c, k) c->nl2[k] = A[k] * tcux[k] + B[k] * tcuy[k];
        dfft(c, c->nl2);
        {
            double l1 = lam / g1, l2 = lam / g2;
            for (int i = 0; i < c->nx; i++)
                for (int j = 0; j < c->ny2; j++) {
                    size_t k = (size_t)i * c->ny2 + j;
                    double ks = ksq(c, i, j);
                    double q1 = l1 * ks, q2 = l2 * ks;
                    RE(c->nl1, k) = -RE(c->nl1, k) - q1 * RE(c->muF1, k);
                    IM(c->nl1, k) = -IM(c->nl1, k) - q1 * IM(c->muF1, k);
                    RE(c->nl2, k) = -RE(c->nl2, k) - q2 * RE(c->muF2, k);
                    IM(c->nl2, k) = -IM(c->nl2, k) - q2 * IM(c->muF2, k);
                }
        }
    }
    (void)C;
    if (c->forc) add_to(c, cnlz, c->forc);
}

static void rhs(orc_ctx *c)
{
    if (c->p.model == 2) potential(c);
    nonlin(c);
}

/* ------------------------------------------------------------------ */
/* ETD2RK (etd2rk.c:14-224)                                             */
/* ------------------------------------------------------------------ */

/* (e^z - 1 - z) / z^2 for the series/expm1 coefficient mode */
static double phi2_z(double z)
{
    if (fabs(z) < 0.5) {
        double term = 0.5, sum = 0.5;
        for (int n = 1; n < 20; n++) {
            term *= z / (double)(n + 2);
            sum += term;
        }
        return sum;
    }
    return (expm1(z) - z) / (z * z);
}

/* Coefficients of mode (i, j): stage-1 decay, stage-1 and stage-2 weights for
 * omega (etd2rk.c:88-97,162-172) and for the phase field(s) (binary :102-111,
 * 177-186; ternary :117-127, 191-203). */
static void coefs(const orc_ctx *c, int i, int j, double *o)
{
    const double dt = c->p.dt, nu = c->p.nu;
    double ksqr = ksq(c, i, j);
    double cc, eta, zeta1, zeta2, beta, z1c, z2c;
    cc = -nu * ksqr;
    eta = exp(-nu * dt * ksqr);
    if (c->p.coef_mode == 0) {
        zeta1 = (fabs(cc) > 1e-12) ? (eta - 1.0) / cc : dt;
        zeta2 = (fabs(cc) > 1e-12) ? (eta - 1.0 - cc * dt) / (dt * cc * cc) : 0.5 * dt;
    } else {
        double z = cc * dt;
        zeta1 = (z != 0.0) ? dt * (expm1(z) / z) : dt;
        zeta2 = dt * phi2_z(z);
    }
    beta = 1.0; z1c = dt; z2c = 0.5 * dt;
    if (c->p.model == 1) {
        cc = -1.5 * c->p.lambda * c->p.sigma * c->p.epsilon * ksqr * ksqr;
        beta = exp(dt * cc);
        if (c->p.coef_mode == 0) {
            z1c = (fabs(cc) > 1e-12) ? (beta - 1.0) / cc : dt;
            z2c = (fabs(cc) != 0.0) ? (beta - 1.0 - cc * dt) / (dt * cc * cc) : 0.5 * dt;
        }
    } else if (c->p.model == 2) {
        cc = -0.75 * c->p.lambda * c->p.epsilon;
        cc *= ksqr * ksqr;
        beta = exp(dt * cc);
        if (c->p.coef_mode == 0) {
            if (fabs(cc) > 1e-12) {
                z1c = (beta - 1.0) / cc;
                z2c = (beta - 1.0 - cc * dt);
                z2c /= (dt * cc * cc);
            } else {
                z1c = dt;
                z2c = 0.5 * dt;
            }
        }
    }
    if (c->p.model != 0 && c->p.coef_mode != 0) {
        double z = dt * cc;
        z1c = (z != 0.0) ? dt * (expm1(z) / z) : dt;
        z2c = dt * phi2_z(z);
    }
    o[0] = eta; o[1] = zeta1; o[2] = zeta2;
    o[3] = beta; o[4] = z1c; o[5] = z2c;
}

void orc_etd_coefs(orc_ctx *c, int i, int j, double *out6) { coefs(c, i, j, out6); }

static void etd2rk(orc_ctx *c)
{
    const int model = c->p.model;
    double co[6];
    rhs(c);
    copy(c, c->nlw, c->sw);
    if (model >= 1) copy(c, c->nl1, c->s1);
    if (model == 2) copy(c, c->nl2, c->s2);
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            coefs(c, i, j, co);
            RE(c->w, k) = RE(c->w, k) * co[0] + RE(c->nlw, k) * co[1];
            IM(c->w, k) = IM(c->w, k) * co[0] + IM(c->nlw, k) * co[1];
            if (model >= 1) {
                RE(c->c1, k) = RE(c->c1, k) * co[3] + RE(c->nl1, k) * co[4];
                IM(c->c1, k) = IM(c->c1, k) * co[3] + IM(c->nl1, k) * co[4];
            }
            if (model == 2) {
                RE(c->c2, k) = RE(c->c2, k) * co[3] + RE(c->nl2, k) * co[4];
                IM(c->c2, k) = IM(c->c2, k) * co[3] + IM(c->nl2, k) * co[4];
            }
        }
    rhs(c);
    for (int i = 0; i < c->nx; i++)
        for (int j = 0; j < c->ny2; j++) {
            size_t k = (size_t)i * c->ny2 + j;
            coefs(c, i, j, co);
            RE(c->w, k) = RE(c->w, k) + (RE(c->nlw, k) - RE(c->sw, k)) * co[2];
            IM(c->w, k) = IM(c->w, k) + (IM(c->nlw, k) - IM(c->sw, k)) * co[2];
            if (model >= 1) {
                RE(c->c1, k) = RE(c->c1, k) + (RE(c->nl1, k) - RE(c->s1, k)) * co[5];
                IM(c->c1, k) = IM(c->c1, k) + (IM(c->nl1, k) - IM(c->s1, k)) * co[5];
            }
            if (model == 2) {
                RE(c->c2, k) = RE(c->c2, k) + (RE(c->nl2, k) - RE(c->s2, k)) * co[5];
                IM(c->c2, k) = IM(c->c2, k) + (IM(c->nl2, k) - IM(c->s2, k)) * co[5];
            }
        }
}

/* ------------------------------------------------------------------ */
/* public API                                                           */
/* ------------------------------------------------------------------ */

orc_ctx *orc_create(const orc_params *p, int nthreads)
{
    orc_ctx *c = (orc_ctx *)calloc(1, sizeof(*c));
    if (!c) return NULL;
    c->p = *p;
    if (c->p.dealias_div == 0.0) c->p.dealias_div = 4.0;
    c->nx = p->nx;
    c->ny = p->ny;
    c->ny2 = p->ny / 2 + 1;
    c->nc = (size_t)c->nx * c->ny2;
    c->nd = 2 * c->nc;
    c->plan = fftc_plan_2d(c->nx, c->ny);
    if (!c->plan) { free(c); return NULL; }
    fftc_set_threads(nthreads);
    /* main.c:54-55 and functions.c:11-33 */
    c->factor_x = (2 * M_PI) / p->lx;
    c->factor_y = (2 * M_PI) / p->ly;
    c->kx = (double *)malloc(sizeof(double) * c->nx);
    c->ky = (double *)malloc(sizeof(double) * c->ny2);
    for (int i = 0; i < c->nx; i++) c->kx[i] = (i <= c->nx / 2) ? c->factor_x * i : c->factor_x * (i - c->nx);
    for (int j = 0; j < c->ny2; j++) c->ky[j] = c->factor_y * j;
    {   /* functions.c:56-59: only the x extent enters the cut */
        double dax = (c->nx / c->p.dealias_div) * c->factor_x;
        c->dealias = dax * dax;
    }
    {   /* main.c:57-58, functions.c:54 */
        double kxmax = (c->nx / 2.0) * c->factor_x, kymax = (c->ny / 2.0) * c->factor_y;
        c->ksqrmax = (double)(kxmax * kxmax + kymax * kymax);
    }
    if (p->model == 2) { /* main.c:166-170 */
        c->gamma1 = (p->sigma12 - p->sigma23 + p->sigma13);
        c->gamma2 = (p->sigma12 - p->sigma13 + p->sigma23);
        c->gamma3 = (p->sigma23 - p->sigma12 + p->sigma13);
        c->del = (6.0 * c->gamma1 * c->gamma2 * c->gamma3);
        c->del /= (c->gamma1 * c->gamma2 + c->gamma1 * c->gamma3 + c->gamma2 * c->gamma3);
    }
    c->w = alloc_buf(c->nd); c->c1 = alloc_buf(c->nd); c->c2 = alloc_buf(c->nd);
    c->nlw = alloc_buf(c->nd); c->nl1 = alloc_buf(c->nd); c->nl2 = alloc_buf(c->nd);
    c->sw = alloc_buf(c->nd); c->s1 = alloc_buf(c->nd); c->s2 = alloc_buf(c->nd);
    c->muF1 = alloc_buf(c->nd); c->muF2 = alloc_buf(c->nd);
    for (int k = 0; k < 10; k++) c->b[k] = alloc_buf(c->nd);
    if (p->force_amp != 0.0) {
        /* vorticity of f = F0 sin(kf y) x-hat: -F0 kf cos(kf y), transformed like any field */
        double dy = p->ly / p->ny;
        c->forc = alloc_buf(c->nd);
        for (int i = 0; i < c->nx; i++)
            for (int j = 0; j < c->ny; j++)
                c->forc[(size_t)i * (c->ny + 2) + j] = -p->force_amp * p->force_k * cos(p->force_k * (j * dy));
        dfft(c, c->forc);
    }
    return c;
}

void orc_destroy(orc_ctx *c)
{
    if (!c) return;
    free(c->kx); free(c->ky);
    free(c->w); free(c->c1); free(c->c2);
    free(c->nlw); free(c->nl1); free(c->nl2);
    free(c->sw); free(c->s1); free(c->s2);
    free(c->muF1); free(c->muF2); free(c->forc);
    for (int k = 0; k < MAXBUF; k++) free(c->b[k]);
    fftc_destroy(c->plan);
    free(c);
}

void orc_set_state(orc_ctx *c, const double *w, const double *c1, const double *c2)
{
    memcpy(c->w, w, c->nd * sizeof(double));
    if (c->p.model >= 1 && c1) memcpy(c->c1, c1, c->nd * sizeof(double));
    if (c->p.model == 2 && c2) memcpy(c->c2, c2, c->nd * sizeof(double));
}

void orc_get_state(orc_ctx *c, double *w, double *c1, double *c2)
{
    if (w) memcpy(w, c->w, c->nd * sizeof(double));
    if (c->p.model >= 1 && c1) memcpy(c1, c->c1, c->nd * sizeof(double));
    if (c->p.model == 2 && c2) memcpy(c2, c->c2, c->nd * sizeof(double));
}

static void load_real(orc_ctx *c, const double *src, double *dst)
{
    memset(dst, 0, c->nd * sizeof(double));
    for (int i = 0; i < c->nx; i++)
        memcpy(dst + (size_t)i * (c->ny + 2), src + (size_t)i * c->ny, c->ny * sizeof(double));
}

void orc_set_phase_real(orc_ctx *c, const double *p1, const double *p2)
{
    memset(c->w, 0, c->nd * sizeof(double));       /* init.c:78-87 */
    if (c->p.model >= 1) {                          /* init.c:221-225 */
        load_real(c, p1, c->c1);
        dfft(c, c->c1);
        truncation(c, c->c1);
    }
    if (c->p.model == 2) {                          /* init.c:253-262 */
        load_real(c, p2, c->c2);
        dfft(c, c->c2);
        truncation(c, c->c2);
    }
}

void orc_step(orc_ctx *c, int n)
{
    for (int s = 0; s < n; s++) etd2rk(c);
}

void orc_rhs(orc_ctx *c, double *nw, double *nc1, double *nc2)
{
    rhs(c);
    if (nw) memcpy(nw, c->nlw, c->nd * sizeof(double));
    if (c->p.model >= 1 && nc1) memcpy(nc1, c->nl1, c->nd * sizeof(double));
    if (c->p.model == 2 && nc2) memcpy(nc2, c->nl2, c->nd * sizeof(double));
}

/* free_energy.c:3-157 (gradients NOT truncated, as in the reference) */
void orc_free_energy(orc_ctx *c, double *ebulk, double *egrad)
{
    double scale = 1.0 / ((double)c->nx * (double)c->ny);
    double ephi = 0.0, egphi = 0.0;
    double *A = c->b[0], *B = c->b[1], *X = c->b[2], *Y = c->b[3], *P = c->b[4], *Q = c->b[5];
    const double ep = c->p.epsilon;
    if (c->p.model == 1) {
        double s = 12.0 * (c->p.sigma / ep);
        copy(c, c->c1, A);
        ifft(c, A);
        FOR_REAL(c, k) {
            double v = A[k];
            double e = v * v * (1.0 - v) * (1.0 - v);
            e *= s;
            ephi += (e * scale);
        }
        ikx(c, c->c1, X);
        iky(c, c->c1, Y);
        ifft(c, X);
        ifft(c, Y);
        FOR_REAL(c, k) egphi += (X[k] * X[k] + Y[k] * Y[k]);
        egphi *= (0.75 * c->p.sigma * ep) * scale;
    } else if (c->p.model == 2) {
        const double g1 = c->gamma1, g2 = c->gamma2, g3 = c->gamma3;
        copy(c, c->c1, A);
        copy(c, c->c2, B);
        ifft(c, A);
        ifft(c, B);
        FOR_REAL(c, k) {
            double a = A[k], b = B[k], d = 1.0 - a - b;
            double e = g1 * a * a * (1.0 - a) * (1.0 - a) + g2 * b * b * (1.0 - b) * (1.0 - b)
                     + g3 * d * d * (a + b) * (a + b);
            e *= (6.0 / ep);
            ephi += (e * scale);
        }
        ikx(c, c->c1, X);
        iky(c, c->c1, Y);
        ikx(c, c->c2, P);
        iky(c, c->c2, Q);
        ifft(c, X); ifft(c, Y);
        ifft(c, P); ifft(c, Q);
        FOR_REAL(c, k) {
            double c1x = X[k], c1y = Y[k], c2x = P[k], c2y = Q[k];
            egphi += (g1 * (c1x * c1x + c1y * c1y) + g2 * (c2x * c2x + c2y * c2y)
                      + g3 * (c1x + c2x) * (c1x + c2x) + g3 * (c1y + c2y) * (c1y + c2y));
        }
        egphi *= (0.375 * ep * scale);
    }
    *ebulk = ephi;
    *egrad = egphi;
}

/* kinetic_energy.c:3-144 (phase averages are 0 when a phase is empty) */
int orc_kinetic_energy(orc_ctx *c, double *out)
{
    double scale = 1.0 / ((double)c->nx * (double)c->ny);
    double *U = c->b[0], *V = c->b[1], *A = c->b[2], *B = c->b[3];
    double eu = 0.0, e1 = 0.0, e2 = 0.0;
    long n1 = 0, n2 = 0;
    get_velocity(c, c->w, U, V);
    truncation(c, U); truncation(c, V);
    ifft(c, U); ifft(c, V);
    if (c->p.model >= 1) { copy(c, c->c1, A); truncation(c, A); ifft(c, A); }
    if (c->p.model == 2) { copy(c, c->c2, B); truncation(c, B); ifft(c, B); }
    FOR_REAL(c, k) {
        double cx = U[k], cy = V[k], px = cx, py = cy;
        eu += 0.5 * (cx * cx + cy * cy);
        if (c->p.model >= 1) {
            double h1 = (A[k] >= 0.5) ? 1.0 : 0.0;
            if (A[k] >= 0.5) n1++;
            cx *= h1; cy *= h1;
            e1 += 0.5 * (cx * cx + cy * cy);
        }
        if (c->p.model == 2) {
            double h2 = (B[k] >= 0.5) ? 1.0 : 0.0;
            if (B[k] >= 0.5) n2++;
            px *= h2; py *= h2;
            e2 += 0.5 * (px * px + py * py);
        }
    }
    eu *= scale;
    out[0] = eu;
    if (c->p.model == 0) return 1;
    out[1] = n1 ? e1 / n1 : 0.0;
    if (c->p.model == 1) return 2;
    out[2] = n2 ? e2 / n2 : 0.0;
    return 3;
}

void orc_dfft(orc_ctx *c, double *padded) { dfft(c, padded); }
void orc_ifft(orc_ctx *c, double *padded) { ifft(c, padded); }
void orc_truncation(orc_ctx *c, double *spec) { truncation(c, spec); }
