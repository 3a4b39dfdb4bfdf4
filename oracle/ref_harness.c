/*
 * ref_harness.c -- drives the reference's OWN compiled sources (etd2rk.c,
 * nonlin.c, surface_tension.c, chem_potential.c, velocity.c, curl.c,
 * functions.c, fft.c, init.c, free_energy.c, kinetic_energy.c, global.c) as an
 * oracle.  Test infrastructure only: it is compiled by oracle/build_ref.py into
 * oracle/_ref/<config>/libref.so together with the reference files, a
 * generated global.h/macro.h carrying the configuration, and the single-rank
 * MPI / FFTW shims.
 *
 * ref_setup() restates the allocation and set-up half of main.c (main.c:37-211):
 * local sizes, the in-place r2c buffers with their complex aliases, plans,
 * wavenumbers and the ternary gamma_i / Delta (main.c:166-170).  The time loop
 * of main.c is NOT used: it calls spectrum(), which truncates the state in place
 * every navg/2 steps (spectrum.c:22-27, main.c:271), and divides by zero when
 * maxiter == nfile (main.c:52,271).
 */
#define _GNU_SOURCE
#include "global.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#define API __attribute__((visibility("default")))

void fftc_set_threads(int nthreads);

static FILE *g_fe_stream, *g_fu_stream, *g_def_stream[2];
static char *g_fe_buf, *g_fu_buf, *g_def_buf[2];
static size_t g_def_len[2];
static size_t g_fe_len, g_fu_len;

API int ref_model(void)
{
#if defined BINARY
    return 1;
#elif defined TERNARY
    return 2;
#else
    return 0;
#endif
}

API int ref_nx(void) { return Nx; }
API int ref_ny(void) { return Ny; }

/* Parameter values exactly as the compiled reference sees them. */
API double ref_param(const char *name)
{
    if (!strcmp(name, "lx")) return lx;
    if (!strcmp(name, "ly")) return ly;
    if (!strcmp(name, "dt")) return dt;
    if (!strcmp(name, "nu")) return nu;
#if defined BINARY || defined TERNARY
    if (!strcmp(name, "epsilon")) return epsilon;
    if (!strcmp(name, "lambda")) return lambda;
#endif
#if defined BINARY
    if (!strcmp(name, "sigma")) return sigma;
#endif
#if defined TERNARY
    if (!strcmp(name, "sigma12")) return sigma_12;
    if (!strcmp(name, "sigma13")) return sigma_13;
    if (!strcmp(name, "sigma23")) return sigma_23;
    if (!strcmp(name, "xlambda")) return Xlambda;
    if (!strcmp(name, "gamma1")) return gamma1;
    if (!strcmp(name, "gamma2")) return gamma2;
    if (!strcmp(name, "gamma3")) return gamma3;
    if (!strcmp(name, "del")) return del;
#endif
    return 0.0 / 0.0;
}

API int ref_setup(int nthreads)
{
    static int done = 0;
    fftc_set_threads(nthreads);
    if (done) return 0;
    done = 1;

    MPI_Init(NULL, NULL);
    fftw_mpi_init();
    MPI_Comm_rank(MPI_COMM_WORLD, &rank);
    MPI_Comm_size(MPI_COMM_WORLD, &size);
    alloc_local = fftw_mpi_local_size_2d(Nx, Ny / 2 + 1, MPI_COMM_WORLD, &local_nx, &local_x_start);

    g_fu_stream = open_memstream(&g_fu_buf, &g_fu_len);
    fu = g_fu_stream;
    navg = 1;
    factor_x = (2 * pi) / lx;
    factor_y = (2 * pi) / ly;
    kxmax = (Nx / 2.0) * factor_x;
    kymax = (Ny / 2.0) * factor_y;

    work = fftw_malloc(local_nx * Ny * sizeof(double));
    u = fftw_alloc_real(2 * alloc_local);
    ux = fftw_alloc_real(2 * alloc_local);
    uy = fftw_alloc_real(2 * alloc_local);
    wz = fftw_alloc_real(2 * alloc_local);
    tux = fftw_alloc_real(2 * alloc_local);
    tuy = fftw_alloc_real(2 * alloc_local);
    twz = fftw_alloc_real(2 * alloc_local);
    nlz = fftw_alloc_real(2 * alloc_local);
    cu = (fftw_complex *)u;
    cux = (fftw_complex *)ux;
    cuy = (fftw_complex *)uy;
    cwz = (fftw_complex *)wz;
    tcux = (fftw_complex *)tux;
    tcuy = (fftw_complex *)tuy;
    tcwz = (fftw_complex *)twz;
    cnlz = (fftw_complex *)nlz;
    cnl_z = fftw_alloc_complex(alloc_local);
    fz = (double *)tux;
    cfz = (fftw_complex *)fz;

#ifdef BINARY
    phi = fftw_alloc_real(2 * alloc_local);
    tphi = fftw_alloc_real(2 * alloc_local);
    nphi = fftw_alloc_real(2 * alloc_local);
    nlphi = fftw_alloc_real(2 * alloc_local);
    cphi = (fftw_complex *)phi;
    tcphi = (fftw_complex *)tphi;
    ncphi = (fftw_complex *)nphi;
    cnlphi = (fftw_complex *)nlphi;
    cnl_phi = fftw_alloc_complex(alloc_local);
    coeff = (sigma / epsilon) * lambda;
#endif
#ifdef TERNARY
    phi1 = fftw_alloc_real(2 * alloc_local);
    phi2 = fftw_alloc_real(2 * alloc_local);
    tphi1 = fftw_alloc_real(2 * alloc_local);
    tphi2 = fftw_alloc_real(2 * alloc_local);
    muF1 = fftw_alloc_real(2 * alloc_local);
    muF2 = fftw_alloc_real(2 * alloc_local);
    nlphi1 = fftw_alloc_real(2 * alloc_local);
    nlphi2 = fftw_alloc_real(2 * alloc_local);
    cphi1 = (fftw_complex *)phi1;
    cphi2 = (fftw_complex *)phi2;
    tcphi1 = (fftw_complex *)tphi1;
    tcphi2 = (fftw_complex *)tphi2;
    cmuF1 = (fftw_complex *)muF1;
    cmuF2 = (fftw_complex *)muF2;
    cnlphi1 = (fftw_complex *)nlphi1;
    cnlphi2 = (fftw_complex *)nlphi2;
    cnl_phi1 = fftw_alloc_complex(alloc_local);
    cnl_phi2 = fftw_alloc_complex(alloc_local);
    gamma1 = (sigma_12 - sigma_23 + sigma_13);
    gamma2 = (sigma_12 - sigma_13 + sigma_23);
    gamma3 = (sigma_23 - sigma_12 + sigma_13);
    del = (6.0 * gamma1 * gamma2 * gamma3);
    del /= (gamma1 * gamma2 + gamma1 * gamma3 + gamma2 * gamma3);
#endif
#if defined BINARY || defined TERNARY
    g_fe_stream = open_memstream(&g_fe_buf, &g_fe_len);
    fe = g_fe_stream;
#endif
    /* spectrum() and perimeter() buffers (main.c:60-63, 104-127, 130-165, 182-185).
     * main.c gives ekx / eky kxm / kym entries, but spectrum.c indexes them with
     * (int)(|kx| / dk + 0.5) up to Nx/2, past the end; here they hold Nx/2 + 1. */
    nshell = round(((double)Nx / sqrt(2.0)) + 1.0);
    kxm = round(sqrt(kxmax * kxmax));
    kym = round(sqrt(kymax * kymax));
    ek = calloc(nshell, sizeof(double));
    ensk = calloc(nshell, sizeof(double));
    ekx = calloc((kxm > Nx / 2 + 1 ? kxm : Nx / 2 + 1), sizeof(double));
    eky = calloc((kym > Ny / 2 + 1 ? kym : Ny / 2 + 1), sizeof(double));
#ifdef BINARY
    sph = calloc(nshell, sizeof(double));
    ph = fftw_malloc((local_nx + 1) * (Ny + 2) * sizeof(double));
    aph = fftw_malloc(Ny * sizeof(double));
    bph = fftw_malloc(Ny * sizeof(double));
    g_def_stream[0] = open_memstream(&g_def_buf[0], &g_def_len[0]);
    fdef = g_def_stream[0];
#endif
#ifdef TERNARY
    sph1 = calloc(nshell, sizeof(double));
    sph2 = calloc(nshell, sizeof(double));
    sp12 = calloc(nshell, sizeof(double));
    ph1 = fftw_malloc((local_nx + 1) * (Ny + 2) * sizeof(double));
    ph2 = fftw_malloc((local_nx + 1) * (Ny + 2) * sizeof(double));
    aph1 = fftw_malloc(Ny * sizeof(double));
    aph2 = fftw_malloc(Ny * sizeof(double));
    bph1 = fftw_malloc(Ny * sizeof(double));
    bph2 = fftw_malloc(Ny * sizeof(double));
    g_def_stream[0] = open_memstream(&g_def_buf[0], &g_def_len[0]);
    g_def_stream[1] = open_memstream(&g_def_buf[1], &g_def_len[1]);
    fdef1 = g_def_stream[0];
    fdef2 = g_def_stream[1];
#endif

    kx = (double *)malloc(local_nx * sizeof(double));
    ky = (double *)malloc(Ny2 * sizeof(double));
    pfor = fftw_mpi_plan_dft_r2c_2d(Nx, Ny, u, cu, MPI_COMM_WORLD, FFTW_ESTIMATE);
    pinv = fftw_mpi_plan_dft_c2r_2d(Nx, Ny, cu, u, MPI_COMM_WORLD, FFTW_ESTIMATE);
    kxky();
    init(); /* ZERO_INIT: omega_hat = 0 (init.c:89-100); phase fields come from ref_set_phase_real */
    return 0;
}

static size_t ncplx(void) { return (size_t)local_nx * Ny2; }

API void ref_set_state(const double *w, const double *c1, const double *c2)
{
    (void)c1; (void)c2;
    memcpy(cwz, w, ncplx() * sizeof(fftw_complex));
#ifdef BINARY
    memcpy(cphi, c1, ncplx() * sizeof(fftw_complex));
#elif defined TERNARY
    memcpy(cphi1, c1, ncplx() * sizeof(fftw_complex));
    memcpy(cphi2, c2, ncplx() * sizeof(fftw_complex));
#endif
}

API void ref_get_state(double *w, double *c1, double *c2)
{
    (void)c1; (void)c2;
    memcpy(w, cwz, ncplx() * sizeof(fftw_complex));
#ifdef BINARY
    memcpy(c1, cphi, ncplx() * sizeof(fftw_complex));
#elif defined TERNARY
    memcpy(c1, cphi1, ncplx() * sizeof(fftw_complex));
    memcpy(c2, cphi2, ncplx() * sizeof(fftw_complex));
#endif
}

/* Real-space phase field(s), Nx*Ny row-major without padding (the layout of
 * read_array_real, read_array.c:20-29), then init.c:221-225 / 253-262:
 * dfft followed by truncation. */
API void ref_set_phase_real(const double *p1, const double *p2)
{
    (void)p1; (void)p2;
#if defined BINARY || defined TERNARY
    for (i = 0; i < Nx; i++)
        for (j = 0; j < Ny; j++) {
#ifdef BINARY
            phi[IDXR(i, j)] = p1[(size_t)i * Ny + j];
#else
            phi1[IDXR(i, j)] = p1[(size_t)i * Ny + j];
            phi2[IDXR(i, j)] = p2[(size_t)i * Ny + j];
#endif
        }
#ifdef BINARY
    dfft(phi, cphi);
    truncation(cphi);
#else
    dfft(phi1, cphi1);
    truncation(cphi1);
    dfft(phi2, cphi2);
    truncation(cphi2);
#endif
#endif
}

/* The main-loop body minus diagnostics: t += dt; etd2rk(...)  (main.c:263-286). */
API void ref_step(int n)
{
    for (int s = 0; s < n; s++) {
        t += dt;
#ifdef BINARY
        etd2rk(cwz, cphi);
#elif defined TERNARY
        etd2rk(cwz, cphi1, cphi2);
#else
        etd2rk(cwz);
#endif
    }
}

/* The right-hand side etd2rk.c evaluates at the start of a step
 * (etd2rk.c:28 / 40-51 / 75): potential() for ternary, then nonlin(). */
API void ref_rhs(double *nw, double *nc1, double *nc2)
{
    (void)nc1; (void)nc2;
#ifdef BINARY
    nonlin(cwz, cnlz, cphi, cnlphi);
    memcpy(nc1, cnlphi, ncplx() * sizeof(fftw_complex));
#elif defined TERNARY
    potential(cphi1, cphi2, cmuF1, cmuF2);
    nonlin(cwz, cnlz, cphi1, cphi2, cnlphi1, cnlphi2);
    memcpy(nc1, cnlphi1, ncplx() * sizeof(fftw_complex));
    memcpy(nc2, cnlphi2, ncplx() * sizeof(fftw_complex));
#else
    nonlin(cwz, cnlz);
#endif
    memcpy(nw, cnlz, ncplx() * sizeof(fftw_complex));
}

static int last_line_values(FILE *s, char **buf, size_t *len, double *out, int nmax)
{
    fflush(s);
    if (!*buf || *len == 0) return 0;
    char *end = *buf + *len - 1;
    while (end > *buf && *end == '\n') end--;
    char *line = end;
    while (line > *buf && line[-1] != '\n') line--;
    int k = 0;
    char *p = line;
    while (k < nmax) {
        char *q;
        double v = strtod(p, &q);
        if (q == p) break;
        out[k++] = v;
        p = q;
    }
    return k;
}

/* Runs the reference's free_energy() on the current state and reads back the
 * line it printed ("%lf \t %.12lf \t %.12lf", free_energy.c:149). */
API int ref_free_energy(double *ephi, double *egphi)
{
#if defined BINARY || defined TERNARY
    double v[3];
#ifdef BINARY
    free_energy(cphi);
#else
    free_energy(cphi1, cphi2);
#endif
    if (last_line_values(g_fe_stream, &g_fe_buf, &g_fe_len, v, 3) != 3) return -1;
    *ephi = v[1];
    *egphi = v[2];
    return 0;
#else
    (void)ephi; (void)egphi;
    return -1;
#endif
}

/* Runs kinetic_energy() and returns the values of the line it printed
 * (kinetic_energy.c:107-139): t, eu[, eph | eph1, eph2]. */
API int ref_kinetic_energy(double *out, int nmax)
{
#ifdef BINARY
    kinetic_energy(cwz, cphi);
#elif defined TERNARY
    kinetic_energy(cwz, cphi1, cphi2);
#else
    kinetic_energy(cwz);
#endif
    return last_line_values(g_fu_stream, &g_fu_buf, &g_fu_len, out, nmax);
}

/* spectrum() (spectrum.c:3-194) on the current state, run with `workdir` as the
 * working directory (it writes spectra/spectrum.<ifile>, Xspectrum, Yspectrum
 * there).  spectrum() truncates the phase fields in place; the state is restored
 * afterwards.  out: ek, ensk, then sph (binary) or sph1, sph2, sp12 (ternary),
 * nshell values each, then ekx and eky, Nx/2 + 1 values each.  Returns nshell. */
API int ref_spectrum(const char *workdir, double *out)
{
    char here[4096];
    const size_t nb = ncplx() * sizeof(fftw_complex);
    double *keep = malloc(3 * nb);
    if (!keep || !getcwd(here, sizeof(here)) || chdir(workdir) != 0) return -1;
    mkdir("spectra", 0755);
    memcpy(keep, cwz, nb);
#ifdef BINARY
    memcpy((char *)keep + nb, cphi, nb);
    spectrum(cwz, cphi);
    memcpy(cphi, (char *)keep + nb, nb);
#elif defined TERNARY
    memcpy((char *)keep + nb, cphi1, nb);
    memcpy((char *)keep + 2 * nb, cphi2, nb);
    spectrum(cwz, cphi1, cphi2);
    memcpy(cphi1, (char *)keep + nb, nb);
    memcpy(cphi2, (char *)keep + 2 * nb, nb);
#else
    spectrum(cwz);
#endif
    memcpy(cwz, keep, nb);
    free(keep);
    if (chdir(here) != 0) return -1;
    double *o = out;
    memcpy(o, ek, nshell * sizeof(double)); o += nshell;
    memcpy(o, ensk, nshell * sizeof(double)); o += nshell;
#ifdef BINARY
    memcpy(o, sph, nshell * sizeof(double)); o += nshell;
#elif defined TERNARY
    memcpy(o, sph1, nshell * sizeof(double)); o += nshell;
    memcpy(o, sph2, nshell * sizeof(double)); o += nshell;
    memcpy(o, sp12, nshell * sizeof(double)); o += nshell;
#endif
    memcpy(o, ekx, (Nx / 2 + 1) * sizeof(double)); o += Nx / 2 + 1;
    memcpy(o, eky, (Ny / 2 + 1) * sizeof(double));
    return nshell;
}

/* perimeter() (perimeter.c:3-271) on the current state; out receives the values
 * of the line(s) it printed (t, Sp_0, Sp_t, def; one line per phase field).
 * Returns the number of values. */
API int ref_perimeter(double *out)
{
#ifdef BINARY
    perimeter(cphi);
    return last_line_values(g_def_stream[0], &g_def_buf[0], &g_def_len[0], out, 4);
#elif defined TERNARY
    perimeter(cphi1, cphi2);
    int a = last_line_values(g_def_stream[0], &g_def_buf[0], &g_def_len[0], out, 4);
    int b = last_line_values(g_def_stream[1], &g_def_buf[1], &g_def_len[1], out + 4, 4);
    return a + b;
#else
    (void)out;
    return 0;
#endif
}

/* The last line the reference printed to one of its logs (0 free_en_t.dat,
 * 1 ken_t.dat, 2 gamma.dat / gamma1.dat, 3 gamma2.dat), without the newline.
 * Returns its length, or -1. */
API int ref_last_line(int which, char *out, int cap)
{
    FILE *s[4] = {g_fe_stream, g_fu_stream, g_def_stream[0], g_def_stream[1]};
    char **b[4] = {&g_fe_buf, &g_fu_buf, &g_def_buf[0], &g_def_buf[1]};
    size_t *l[4] = {&g_fe_len, &g_fu_len, &g_def_len[0], &g_def_len[1]};
    if (which < 0 || which > 3 || !s[which]) return -1;
    fflush(s[which]);
    if (!*b[which] || *l[which] == 0) return -1;
    char *end = *b[which] + *l[which];
    while (end > *b[which] && end[-1] == '\n') end--;
    char *line = end;
    while (line > *b[which] && line[-1] != '\n') line--;
    int n = (int)(end - line);
    if (n >= cap) return -1;
    memcpy(out, line, n);
    out[n] = 0;
    return n;
}

/* Direct access to the reference's fft.c and functions.c on a caller buffer. */
API void ref_dfft(double *padded) { dfft(padded, (fftw_complex *)padded); }
API void ref_ifft(double *padded) { ifft((fftw_complex *)padded, padded); }
API void ref_truncation(double *c) { truncation((fftw_complex *)c); }
API void ref_get_velocity(const double *w, double *cx, double *cy)
{
    /* cu is a scratch buffer that no hot-path function touches */
    memcpy(cu, w, ncplx() * sizeof(fftw_complex));
    get_velocity(cu, (fftw_complex *)cx, (fftw_complex *)cy);
}
API void ref_set_time(double tt) { t = tt; }
