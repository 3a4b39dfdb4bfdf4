/*
 * etd2rk_dropin.c -- the reference's etd2rk() (etd2rk.c:14-224) with its own
 * signature, running the step on one GPU through the C ABI of include/chns.h.
 *
 * Link it in place of etd2rk.o (Makefile:6) and add libchns_b200.so to LIBS.
 * It is compiled against the reference's own global.h so that it takes the
 * configuration from the same #defines (Nx, Ny, lx, ly, nu, dt, sigma,
 * epsilon, lambda, sigma_ij, Xlambda, BINARY/TERNARY; global.h:19-45,102-143,
 * macro.h).  Semantics are those of the reference: the state arrays (cwz,
 * cphi / cphi1, cphi2, FFTW layout, local_nx x Ny2 complex) are advanced by one
 * ETD2RK step in place.  Each call copies the state to the device, steps, and
 * copies it back, so the arrays stay the single source of truth for the rest
 * of the reference (diagnostics, dumps, spectrum()).
 *
 * The GPU context is created on the first call.  The step is single-GPU: it
 * needs the whole field on one rank (MPI size 1, local_nx == Nx); otherwise, or
 * on any error, it reports and calls MPI_Abort as the reference's own failures do.
 */
#include "global.h"

#include <string.h>

/* Capture the configuration before the field names of chns_params (lx, ly, nu,
 * dt, sigma, epsilon, lambda) are freed from the reference's macros below. */
static const double cfg_lx = lx, cfg_ly = ly, cfg_nu = nu, cfg_dt = dt;
#if defined BINARY
static const double cfg_sigma = sigma, cfg_eps = epsilon, cfg_lam = lambda;
#elif defined TERNARY
static const double cfg_s12 = sigma_12, cfg_s13 = sigma_13, cfg_s23 = sigma_23, cfg_xlam = Xlambda;
static const double cfg_eps = epsilon, cfg_lam = lambda;
#endif
#undef lx
#undef ly
#undef nu
#undef dt
#undef sigma
#undef epsilon
#undef lambda

#include "chns.h"

static chns_ctx *dropin_ctx;

static void dropin_fail(const char *what, int rc)
{
    fprintf(stderr, "etd2rk (libchns_b200): %s failed: %s (%d)\n", what, chns_status_string(rc), rc);
    MPI_Abort(MPI_COMM_WORLD, 1);
}

static void dropin_init(void)
{
    chns_params p;
    int rc;
    memset(&p, 0, sizeof(p));
    if (size != 1 || local_nx != Nx || local_x_start != 0) dropin_fail("single-GPU etd2rk (needs one MPI rank)", CHNS_ERR_UNSUPPORTED);
#if defined BINARY
    p.model = CHNS_MODEL_BINARY;
    p.sigma = cfg_sigma;
    p.epsilon = cfg_eps;
    p.lambda = cfg_lam;
#elif defined TERNARY
    p.model = CHNS_MODEL_TERNARY;
    p.sigma12 = cfg_s12;
    p.sigma13 = cfg_s13;
    p.sigma23 = cfg_s23;
    p.xlambda = cfg_xlam;
    p.epsilon = cfg_eps;
    p.lambda = cfg_lam;
#else
    p.model = CHNS_MODEL_NS;
#endif
    p.precision = CHNS_FP64;
    p.nx = Nx;
    p.ny = Ny;
    p.lx = cfg_lx;
    p.ly = cfg_ly;
    p.dt = cfg_dt;
    p.nu = cfg_nu;
    p.dealias_div = 4.0;                 /* functions.c:56 */
#ifdef SMOOTH_FILTER
    p.filter = CHNS_FILTER_SMOOTH;       /* functions.c:69-72 */
#endif
    p.coef_mode = CHNS_COEF_REFERENCE;   /* etd2rk.c's own phi-function formulas */
    rc = chns_create(&p, &dropin_ctx);
    if (rc != CHNS_OK) dropin_fail("chns_create", rc);
}

/* the state arrays are uploaded and read back on every call: page-lock them once
 * (fftw_alloc_real(2 alloc_local) doubles each, main.c:75-163) */
static void dropin_pin(void *a)
{
    if (a && chns_pin_host(dropin_ctx, a, 2 * (size_t)alloc_local * sizeof(double)) != CHNS_OK)
        fprintf(stderr, "etd2rk (libchns_b200): could not page-lock a state array; transfers stay pageable\n");
}

void etd2rk(fftw_complex *cwz
#ifdef BINARY
, fftw_complex *cphi
#elif defined TERNARY
, fftw_complex *cphi1, fftw_complex *cphi2
#endif
)
{
    double *c1 = NULL, *c2 = NULL;
    int rc;
    int first = !dropin_ctx;
    if (!dropin_ctx) dropin_init();
#ifdef BINARY
    c1 = (double *)cphi;
#elif defined TERNARY
    c1 = (double *)cphi1;
    c2 = (double *)cphi2;
#endif
    if (first) {
        dropin_pin(cwz);
        dropin_pin(c1);
        dropin_pin(c2);
    }
    rc = chns_set_state(dropin_ctx, (const double *)cwz, c1, c2, CHNS_HOST);
    if (rc == CHNS_OK) rc = chns_step(dropin_ctx, 1);
    if (rc == CHNS_OK) rc = chns_get_state(dropin_ctx, (double *)cwz, c1, c2, CHNS_HOST);
    if (rc != CHNS_OK) dropin_fail("etd2rk step", rc);
}
