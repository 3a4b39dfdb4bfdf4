/*
 * chns_oracle.h -- CPU restatement of the reference's ETD2RK CHNS step.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this code, and only as the checker.
 *
 * It restates, with run-time parameters instead of the reference's compile-time
 * #defines, the functions of phynadia/Ternary-CHNS that make up one time step:
 * etd2rk.c, nonlin.c, surface_tension.c, chem_potential.c, velocity.c, curl.c,
 * functions.c (kxky, truncation), fft.c, plus the INIT_READ_DATA set-up of
 * init.c and the free_energy.c / kinetic_energy.c diagnostics.  Every arithmetic
 * expression keeps the reference's operand order so that, with the same FFT, it
 * reproduces the reference's compiled code (oracle/_ref) bit for bit.
 *
 * Arrays are in FFTW's layout (reference global.h:13-14): spectral fields are
 * nx x (ny/2+1) complex (interleaved doubles), row i = x wavenumber kx[i].
 */
#ifndef CHNS_ORACLE_H
#define CHNS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    int model;          /* 0 pure Navier-Stokes, 1 binary (BINARY), 2 ternary (TERNARY) */
    int nx, ny;         /* grid, powers of two */
    double lx, ly;      /* box lengths (global.h:20-21) */
    double dt, nu;      /* time step, viscosity (global.h:30-31) */
    double lambda;      /* mobility (global.h:104,132) */
    double sigma;       /* binary surface tension (global.h:102) */
    double epsilon;     /* interface width (global.h:103,131) */
    double sigma12, sigma13, sigma23, xlambda; /* ternary (global.h:127-133) */
    double dealias_div; /* cut radius = (nx / dealias_div) * 2 pi / lx; reference: 4.0 (functions.c:56) */
    int coef_mode;      /* 0: reference's direct phi-functions (etd2rk.c:88-206); 1: series/expm1 */
    double force_amp;   /* Kolmogorov forcing F0 sin(kf y) x-hat; 0 = off (not in the reference) */
    double force_k;     /* kf */
    int filter;         /* 0: the sharp cut; 1: SMOOTH_FILTER (functions.c:69-72, macro.h:15) */
} orc_params;

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const orc_params *p, int nthreads);
void orc_destroy(orc_ctx *c);

/* State in FFTW layout; c1/c2 ignored where the model has no such field. */
void orc_set_state(orc_ctx *c, const double *w, const double *c1, const double *c2);
void orc_get_state(orc_ctx *c, double *w, double *c1, double *c2);

/* init.c:221-225 / 253-262 with INIT_READ_DATA: real nx*ny fields (row-major,
 * unpadded), dfft, truncation.  omega_hat is set to zero (init.c:78-87). */
void orc_set_phase_real(orc_ctx *c, const double *p1, const double *p2);

/* n ETD2RK steps (etd2rk.c:14-224). */
void orc_step(orc_ctx *c, int n);

/* The right-hand side of one stage on the current state: potential() + nonlin(). */
void orc_rhs(orc_ctx *c, double *nw, double *nc1, double *nc2);

/* free_energy.c: bulk and gradient energy of the current state. */
void orc_free_energy(orc_ctx *c, double *ebulk, double *egrad);

/* kinetic_energy.c: out[0] = <|u|^2/2>; binary out[1] = phase KE;
 * ternary out[1], out[2].  Returns the number of values. */
int orc_kinetic_energy(orc_ctx *c, double *out);

/* fft.c on a padded nx*(ny+2) buffer: dfft (unnormalised r2c) and ifft (c2r * 1/(nx ny)). */
void orc_dfft(orc_ctx *c, double *padded);
void orc_ifft(orc_ctx *c, double *padded);
/* functions.c:47-84 on a spectral field. */
void orc_truncation(orc_ctx *c, double *spec);

/* ETD coefficient tables for inspection: for mode (i, j) writes
 * [eta_w, zeta1_w, zeta2_w, beta_c, zeta1_c, zeta2_c]. */
void orc_etd_coefs(orc_ctx *c, int i, int j, double *out6);

#ifdef __cplusplus
}
#endif
#endif
