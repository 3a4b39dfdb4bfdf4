/*
 * chns.h -- C ABI of the B200-native ETD2RK step for 2D pseudospectral
 * Cahn-Hilliard-Navier-Stokes (binary and ternary phase-field flows).
 *
 * Drop-in boundary for phynadia/Ternary-CHNS's time step.  The reference's
 * step is   void etd2rk(fftw_complex *cwz [, *cphi | , *cphi1, *cphi2])
 * (etd2rk.c:14-20, declared unprototyped at global.h:94), which updates the
 * state in place in FFTW's spectral layout and takes every parameter from
 * compile-time #defines (global.h:19-45,102-143) and process globals.  This ABI
 * keeps the fields, the layout and the arithmetic of that step, with explicit
 * parameters and context instead of globals:
 *
 *   state arrays : nx x (ny/2+1) complex, interleaved doubles, row i = kx[i]
 *                  (IDXC(i,j) = j + Ny2*i, global.h:13), i.e. the arrays
 *                  cwz, cphi / cphi1, cphi2 of the reference.
 *   real arrays  : nx x ny doubles, row-major, row i = x (the layout of the
 *                  reference's read_array_real / write_array_real files,
 *                  read_array.c:20-29, write_array.c:29-38).
 *
 * All functions return CHNS_OK (0) or a negative status; none aborts.  A context
 * owns its device memory, tables and CUDA stream; calls on one context are
 * stream-ordered and must not be made concurrently from several threads.  The
 * literal drop-in etd2rk() with the reference's own signature is in
 * ternary-chns_b200/csrc/etd2rk_dropin.c (it is compiled against the reference's
 * global.h so that it sees the configuration macros).
 */
#ifndef CHNS_H
#define CHNS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHNS_OK 0
#define CHNS_ERR_ARG (-1)         /* bad argument or parameter */
#define CHNS_ERR_CUDA (-2)        /* a CUDA call failed */
#define CHNS_ERR_NONFINITE (-3)   /* the state holds NaN/Inf or blew up */
#define CHNS_ERR_TIMEOUT (-4)     /* a bounded device wait ran out */
#define CHNS_ERR_UNSUPPORTED (-5) /* size or option not supported */
#define CHNS_ERR_NOMEM (-6)       /* device or host allocation failed */
#define CHNS_ERR_IO (-7)          /* a file could not be read or written */

enum { CHNS_MODEL_NS = 0, CHNS_MODEL_BINARY = 1, CHNS_MODEL_TERNARY = 2 };
/* Arithmetic of a context.  FP64: every operation in double (the reference's
 * arithmetic).  FP32: transforms and point-wise work in float, ETD coefficients
 * computed in double, k = 0 modes kept in double.  FP32_STATE64: the FP32
 * right-hand side, with the state (w, c_i) carried as a pair of floats hi + lo
 * (48 significant bits) and the ETD update u + d, d = u (e - 1) + N z1 (e - 1
 * from expm1), added to the pair without rounding error; the right-hand side
 * reads hi, the float rounding of the state.  At small dt an FP32 state loses the low bits of every increment, and
 * the spinodal modes amplify that rounding: FP32_STATE64 removes this error
 * source for one more float read and write of the modes inside the truncation
 * disc per stage (the modes outside it never reach a right-hand side, so they
 * stay float).  chns_set_state / chns_get_state convert to and from the pair
 * (relative rounding <= 2^-48 per element inside the disc, 2^-24 outside). */
enum { CHNS_FP64 = 0, CHNS_FP32 = 1, CHNS_FP32_STATE64 = 2 };
/* ETD phi-function coefficients: REFERENCE evaluates etd2rk.c's direct formulas
 * (etd2rk.c:88-206, with its small-|c| branches) on the host in double, so
 * the FP64 step reproduces the reference; ACCURATE uses expm1 and a series for
 * small |c h| (more accurate than the reference for small |c h|). */
enum { CHNS_COEF_REFERENCE = 0, CHNS_COEF_ACCURATE = 1 };
enum { CHNS_HOST = 0, CHNS_DEVICE = 1 };
/* Truncation of the spectra before their inverse transforms (functions.c:47-84).
 * SHARP zeroes the modes with k^2 > ((nx/dealias_div) 2 pi/lx)^2, the reference's
 * default build.  SMOOTH is the reference built with SMOOTH_FILTER (macro.h:15,
 * functions.c:69-72): every mode is multiplied by f = exp(-36 (k^2/k^2max)^18),
 * k^2max = kxmax^2 + kymax^2, twice (one rounding per product), and nothing is
 * zeroed, so the intermediate fields of a step keep all nx/2+1 ky rows and
 * dealias_div is ignored.  f is the host's exp and pow in double, the reference's
 * own libm calls (rounded to float for the FP32 step).  SMOOTH contexts have no
 * discrete adjoint (chns_adjoint returns CHNS_ERR_UNSUPPORTED). */
enum { CHNS_FILTER_SHARP = 0, CHNS_FILTER_SMOOTH = 1 };

typedef struct chns_params {
    int model;          /* CHNS_MODEL_*: none / BINARY / TERNARY (macro.h) */
    int precision;      /* CHNS_FP64, CHNS_FP32 or CHNS_FP32_STATE64 */
    int nx, ny;         /* Nx, Ny (global.h:23-24); nx == ny, power of two, 32..4096 */
    double lx, ly;      /* box (global.h:20-21) */
    double dt, nu;      /* dt, nu (global.h:30-31) */
    double lambda;      /* mobility (global.h:104,132) */
    double sigma;       /* binary surface tension (global.h:102) */
    double epsilon;     /* interface width (global.h:103,131) */
    double sigma12, sigma13, sigma23; /* ternary sigma_ij (global.h:127-129) */
    double xlambda;     /* ternary Xlambda (global.h:133) */
    double dealias_div; /* truncation radius (nx/dealias_div)*2pi/lx; the reference's is 4 (functions.c:56) */
    int coef_mode;      /* CHNS_COEF_* */
    double force_amp;   /* Kolmogorov forcing F0 sin(kf y) x-hat on the flow; 0 = off.  Not in the reference */
    double force_k;     /* kf; kf*ly/(2 pi) must be an integer <= ny/2 */
    int filter;         /* CHNS_FILTER_*: SHARP (default) or SMOOTH (the SMOOTH_FILTER build) */
} chns_params;

typedef struct chns_ctx chns_ctx;

/* Fills p with the reference's defaults (global.h:19-45 and the BINARY /
 * TERNARY blocks :102-143) for the given model and grid n. */
void chns_default_params(chns_params *p, int model, int n);

/* Creates a context: device buffers, truncation table, ETD coefficient tables,
 * twiddles, stream.  Replaces the allocation/plan/kxky set-up of main.c:43-211. */
int chns_create(const chns_params *p, chns_ctx **out);
int chns_destroy(chns_ctx *ctx);

/* The host-side tables chns_create builds, computed without a context or a GPU
 * (no counterpart in the reference, which recomputes them inside its loops; these
 * expose the exact values the step uses so that they can be checked):
 * chns_etd_coefficients gives, for the mode (kx index i in 0..nx-1, ky index j in
 * 0..nx/2), out[0..5] = e^{-nu k^2 dt}, zeta1, zeta2 of the vorticity and
 * e^{c dt}, z1, z2 of the phase fields (etd2rk.c:88-111,117-127 / 162-186,191-203,
 * per coef_mode; NS contexts: 1, dt, dt/2), in double;
 * chns_truncation_rows fills mrow[0..nx/2] with the largest |kx index| kept in
 * each ky row by the truncation (functions.c:47-84), -1 for an empty row (every
 * row keeps nx/2 with the SMOOTH filter); chns_truncation_factor gives the factor
 * f of one product of the truncation at mode (i, j): 1 or 0 for the SHARP cut,
 * exp(-36 (k^2/k^2max)^18) for the SMOOTH filter (the mode is multiplied by it
 * twice).  Parameters are checked as by chns_create. */
int chns_etd_coefficients(const chns_params *p, int i, int j, double *out);
int chns_truncation_rows(const chns_params *p, int *mrow);
int chns_truncation_factor(const chns_params *p, int i, int j, double *f);

/* Uses `stream` (a cudaStream_t) for all later work instead of the context's own. */
int chns_set_stream(chns_ctx *ctx, void *stream);
int chns_synchronize(chns_ctx *ctx);

/* State in FFTW layout (w = cwz, c1 = cphi or cphi1, c2 = cphi2); pointers on
 * the host or the device (where = CHNS_HOST / CHNS_DEVICE).  Unused fields may
 * be NULL. */
int chns_set_state(chns_ctx *ctx, const double *w, const double *c1, const double *c2, int where);
int chns_get_state(chns_ctx *ctx, double *w, double *c1, double *c2, int where);

/* Page-locks a host array that the caller passes to chns_set_state /
 * chns_get_state on every step (the drop-in etd2rk() does this for the
 * reference's state arrays): transfers from pageable memory run at about a third
 * of the speed of page-locked ones.  The registration lasts until chns_unpin_host
 * or chns_destroy; the caller must not free the array before either.  An array
 * that is already page-locked is accepted. */
int chns_pin_host(chns_ctx *ctx, void *ptr, size_t bytes);
int chns_unpin_host(chns_ctx *ctx, void *ptr);

/* Initial phase field(s) from real nx x ny arrays: dfft + truncation, omega = 0
 * (init.c:78-87,221-225,253-262 with INIT_READ_DATA). */
int chns_set_phase_real(chns_ctx *ctx, const double *p1, const double *p2, int where);

/* nsteps ETD2RK steps on the resident state (etd2rk.c:14-224 each), replayed
 * from a CUDA graph.  Asynchronous: returns after enqueueing. */
int chns_step(chns_ctx *ctx, int nsteps);

/* Right-hand side N(u) of the current state: the output of potential() +
 * nonlin() (etd2rk.c:28 / 40-51), in FFTW layout.  The state is unchanged. */
int chns_rhs(chns_ctx *ctx, double *nw, double *nc1, double *nc2, int where);

/* fft.c on the device: dfft = unnormalised 2D r2c of a real nx x ny array into
 * FFTW layout; ifft = c2r then x 1/(nx ny) (fft.c:11-31). */
int chns_dfft(chns_ctx *ctx, const double *real, double *spec, int where);
int chns_ifft(chns_ctx *ctx, const double *spec, double *real, int where);

/* Failure detection: scans the state (and the FP32 k = 0 side channel) on the
 * device for NaN or infinite values; CHNS_ERR_NONFINITE if there are any.  The
 * reference has no such check (it aborts only through free_energy.c:151-154, which
 * chns_diagnostics mirrors).  No call of this library waits on the device for
 * another party (work is ordered by streams, events and graphs), so none can time
 * out; CHNS_ERR_TIMEOUT is reserved. */
int chns_check(chns_ctx *ctx);

/* Free energy (free_energy.c:3-157) and kinetic energy (kinetic_energy.c:3-144)
 * of the current state: out_fe[2] = {bulk, gradient}; out_ke[3] = {<|u|^2/2>,
 * phase-1 mean, phase-2 mean}. */
int chns_diagnostics(chns_ctx *ctx, double *out_fe, double *out_ke);

/* Checkpoint / resume.  The reference cannot restart bit for bit (its dumps are
 * real-space and truncated, main.c:332-359; INIT_READ_DATA reads only the phase
 * fields).  chns_save writes the context's parameters and its spectral state
 * (FFTW layout, FP64: FP32 states convert exactly and their k = 0 modes are kept in
 * double) to `path`; chns_load reads such a file into a context created with the
 * same parameters (else CHNS_ERR_ARG).  Steps after a load are bit-identical to the
 * steps the saved context would have taken. */
int chns_save(chns_ctx *ctx, const char *path);
int chns_load(chns_ctx *ctx, const char *path);

/* Shell spectra of the current state (spectrum.c:3-194), without spectrum.c's side
 * effect (it truncates the phase fields in place).  nshell = chns_spectrum_shells
 * = round(nx/sqrt(2) + 1) (main.c:60); shell (int)(|k|/dk + 0.5), dk = 2 pi / lx.
 * out receives ek and ensk (nshell each), then sph (binary) or sph1, sph2, sp12
 * (ternary) (nshell each), then ekx and eky (nx/2 + 1 each: spectrum.c indexes
 * them up to nx/2 although main.c:182-185 allocates only kxm / kym entries). */
int chns_spectrum_shells(const chns_ctx *ctx);
int chns_spectrum(chns_ctx *ctx, double *out);

/* Interface perimeter (perimeter.c:3-271) of each phase field: out[5 f + 0..4] =
 * count of cells whose +x or +y neighbour (periodic) lies on the other side of
 * c = 0.5, count of cells with c >= 0.5, Sp_0 = 2 sqrt(pi count2 dx dy),
 * Sp_t = count1 dx, def = Sp_t / Sp_0 - 1. */
int chns_perimeter(chns_ctx *ctx, double *out);

/* The reference's initial conditions (init.c) computed on the device, each with
 * the dfft and truncation init.c applies.  Vorticity (init.c:38-96):
 *   CHNS_INIT_W_ZERO           omega = 0 (ZERO_INIT, INIT_READ_DATA)
 *   CHNS_INIT_W_TAYLOR_GREEN   TG_INIT: u = amplitude (sin x cos y, -cos x sin y),
 *                              omega_hat = I (kx uy_hat - ky ux_hat), truncated
 *   CHNS_INIT_W_SHELL          neither macro (init.c:102-182): velocity modes of
 *                              amplitude uamp vk, vk^2 = k^4 e^{-2k^2} / (3 den(|k|))
 *                              nx ny (den = modes per shell), projected by the
 *                              p11/p12/p22 tensor, curl, truncation; amplitude =
 *                              uamp (global.h:44).  The reference draws two
 *                              time-seeded phases per mode but passes
 *                              I 2 pi r to the real exp() of math.h (no tgmath.h),
 *                              which takes the real part, 0: every phase factor is
 *                              exactly 1, so the field is deterministic and is
 *                              reproduced as compiled.
 * Phase fields (init.c:229-292):
 *   CHNS_INIT_C_DROP    binary: c = (1 - tanh((r - pi/4.5) / (eps/2))) / 2, r the
 *                       distance to the box centre
 *   CHNS_INIT_C_NOISE   ternary: c_i = 1/4 + 0.001 rand()/RAND_MAX, two draws per
 *                       point in row-major order after srand(seed) (the reference
 *                       uses seed = 10 + 2 rank); the C library's generator, run
 *                       on the host with a private state
 * chns_init_phase leaves omega unchanged; the other fields are replaced. */
#define CHNS_INIT_W_ZERO 0
#define CHNS_INIT_W_TAYLOR_GREEN 1
#define CHNS_INIT_W_SHELL 2
#define CHNS_INIT_C_DROP 0
#define CHNS_INIT_C_NOISE 1
int chns_init_vorticity(chns_ctx *ctx, int kind, double amplitude);
int chns_init_phase(chns_ctx *ctx, int kind, unsigned int seed);

/* Field files in the reference's format (write_array.c:18-46, read_array.c:12-40):
 * raw FP64, nx x ny, row-major with x the slow index, no header.
 * chns_write_fields writes the real-space fields of the current state as main.c's
 * dumps do: <dir>/vort/wz.<index> and <dir>/phase_field/phi.<index> (binary) or
 * phi1.<index> and phi2.<index> (ternary), creating the two folders.  truncate = 0
 * is the serial dump (main.c:233-249, ifft of the state as it is), truncate = 1 the
 * DUMP_REAL_MPI dump (main.c:334-356, truncation then ifft).
 * chns_read_phase reads the phase file(s) of INIT_READ_DATA (init.c:221-225,
 * 253-262: read, dfft, truncation; omega = 0), as chns_set_phase_real.
 * A file that cannot be opened, written or fully read gives CHNS_ERR_IO. */
int chns_write_fields(chns_ctx *ctx, const char *dir, int index, int truncate);
int chns_read_phase(chns_ctx *ctx, const char *path1, const char *path2);

/* Discrete adjoint of `nsteps` ETD2RK steps (etd2rk.c with nonlin.c /
 * surface_tension.c / chem_potential.c transposed operation by operation) from
 * the current state.  Loss at the final state, with c and grad c untruncated as in
 * free_energy.c:3-157 (loss_w = NULL: all weights 1):
 *   binary  J = w[0] E_bulk + w[1] E_grad + w[2] <|grad phi|^2>,  phi = 2c - 1
 *   ternary J = w[0] E_bulk + w[1] E_grad + w[2] <|grad c1|^2 + |grad c2|^2>
 *   pure Navier-Stokes J = w[0] <|u|^2 / 2> + w[1] <w_t^2 / 2>, of the truncated
 *           velocity (kinetic_energy.c:17-21,43-49,89) and vorticity (w[2] unused)
 * Outputs: *J; dJ/d(omega_hat_0) in g_w and dJ/d(c_hat_0) (binary) or dJ/d(c1_hat_0)
 * followed by dJ/d(c2_hat_0) (ternary) in g_c, FFTW layout (gradients with respect
 * to the stored real and imaginary parts; g_w / g_c may be NULL; g_c is not written
 * for pure Navier-Stokes); g_params = dJ/d(nu, lambda, sigma) (binary, 3 values;
 * pure Navier-Stokes: nu, 0, 0) or dJ/d(nu, lambda, sigma_12, sigma_13, sigma_23)
 * (ternary, 5 values).  The state is kept every `ckpt` steps and recomputed in
 * between; it is unchanged on return.  The buffers stay in the context: 2 x ckpt
 * segment slots (one set when two do not fit, else CHNS_ERR_NOMEM) of 26 (binary:
 * the step's states and right-hand sides, and the forward fields its transpose
 * reads), 12 (ternary) or 4 (pure Navier-Stokes) fields of n x n/2+1 complex or
 * n x n real values.  CHNS_FP32_STATE64 contexts return CHNS_ERR_UNSUPPORTED. */
int chns_adjoint(chns_ctx *ctx, int nsteps, int ckpt, const double *loss_w, double *J, double *g_w,
                 double *g_c, double *g_params, int where);

/* Ensembles.  Many independent runs (realisations with their own seeds and
 * parameters, any mix of models, grid sizes and precisions) advanced together:
 * the reference runs one configuration per mpirun, so this has no counterpart
 * there; each member is a full context (the reference's state and step), and
 * chns_ensemble_step advances all of them with one CUDA graph launch per step in
 * which every member's stage kernels form their own branch, so members that
 * are too small to fill the GPU alone run side by side.  Member i's results are
 * identical to chns_step on a lone context with the same parameters. */
typedef struct chns_ensemble chns_ensemble;
int chns_ensemble_create(const chns_params *members, int count, chns_ensemble **out);
int chns_ensemble_destroy(chns_ensemble *ens);
/* The context of member i (owned by the ensemble: use it for set_state,
 * get_state, set_phase_real and diagnostics; do not destroy it or change its
 * stream).  NULL if i is out of range. */
chns_ctx *chns_ensemble_member(chns_ensemble *ens, int i);
int chns_ensemble_size(const chns_ensemble *ens);
/* nsteps ETD2RK steps of every member; stream-ordered after earlier work on
 * each member's stream, and later work on member streams waits for it. */
int chns_ensemble_step(chns_ensemble *ens, int nsteps);
/* How chns_ensemble_step runs (no counterpart in the reference): 1 = every step
 * is one persistent kernel over all members (its CTAs take the members' stage
 * work from a queue, each item waiting only for its own member's previous
 * pass), 0 = a graph with one branch of stage kernels per member (the default,
 * faster on the benchmark's 64-member ensemble).  The persistent form needs
 * every member ternary, CHNS_FP32, n = 256, 512 or 1024 and the reference's cut
 * on a square box.  enable = 0 or 1 switches (CHNS_ERR_UNSUPPORTED if the
 * members do not allow 1), any other value only queries; returns the mode in
 * use.  Both modes give bitwise the same states.  A bounded wait of the
 * persistent kernel that runs out is returned by chns_ensemble_synchronize as
 * CHNS_ERR_TIMEOUT. */
int chns_ensemble_persistent(chns_ensemble *ens, int enable);
int chns_ensemble_synchronize(chns_ensemble *ens);

/* Kernel launches of one step (known after the first chns_step). */
int chns_launches_per_step(const chns_ctx *ctx);

/* 1 when the step's row kernels load their input tiles with TMA (contexts whose
 * tensor maps the driver encoded), 0 when they use cp.async.  A tile wait
 * that runs out (bounded, about a second) is reported by the next
 * chns_synchronize / chns_check as CHNS_ERR_TIMEOUT.  No counterpart in the
 * reference (tracing). */
int chns_tma_tiles(const chns_ctx *ctx);

/* Failure injection for tests (no counterpart in the reference): the row
 * kernels' waits for their TMA tiles poll at most `spins` times (0 = the
 * default bound) and, with skip_copies != 0, no tile copy is issued at all, so
 * every wait runs out on a barrier nothing will complete -- no copy is in
 * flight, the kernels finish, their results are garbage -- and the next
 * chns_synchronize / chns_check returns CHNS_ERR_TIMEOUT.  chns_debug_tile_waits
 * (ctx, 0, 0) restores normal operation.  CHNS_ERR_UNSUPPORTED when the context
 * has no TMA tiles (chns_tma_tiles). */
int chns_debug_tile_waits(chns_ctx *ctx, int spins, int skip_copies);

/* Autotuning hook (no reference counterpart): overrides, for contexts created
 * afterwards in this process, a launch-shape choice of the tuned tables
 * (ternary-chns_b200/csrc/chns_tuned.h).  knob CHNS_TUNE_TMA_BOX_ROWS: rows per
 * TMA box of the row kernels' tiles, a multiple of 8 in 8..256;
 * CHNS_TUNE_P1_SPLIT: 1 runs the spectral inverse pass with two CTAs per row, 0
 * with one; CHNS_TUNE_P4_GRAD: 1 keeps grad c_i in real space from the advection
 * pass for the force pass (one more device field per phase field), 0 has the force
 * pass transform it again; CHNS_TUNE_PDL: 1 launches the stage kernels as
 * programmatic dependent launches (each scheduled while the one before drains,
 * waiting on the device for its completion), 0 plainly.  value -1 restores the
 * table.  Results are bitwise the same under every choice; only the speed changes.
 * Not thread-safe: set before creating contexts. */
enum { CHNS_TUNE_TMA_BOX_ROWS = 1, CHNS_TUNE_P1_SPLIT = 2, CHNS_TUNE_P4_GRAD = 3, CHNS_TUNE_PDL = 4 };
int chns_tune_override(int knob, int value);

/* Tracing: runs `reps` steps launching the kernels one by one (not from the
 * graph) with a CUDA event recorded after each launch on the context's stream;
 * writes the mean duration of every launch of one step to ms[] and its kind to
 * kind[] (0 spectral inverse pass, 1 row advection pass, 2 spectral forward pass
 * of c, 3 row force pass, 4 spectral curl/ETD pass of w, 5 second row advection
 * pass).  Returns the number of launches per step, or a negative status.
 * The state advances by `reps` steps. */
int chns_profile_step(chns_ctx *ctx, int reps, float *ms, int *kind, int maxk);

const char *chns_status_string(int status);

/* Slab-decomposed transforms over several GPUs: fft.c:11-31 as the reference
 * runs it under FFTW-MPI (plans main.c:193-194, slabs main.c:43-46).  Rank r of
 * P holds local_nx = n / P x-rows of the real field (row stride real_stride
 * doubles, >= n; the reference's in-place rows are n + 2) and the same kx-rows
 * of the spectrum in FFTW layout (local_nx x (n/2+1) complex doubles).  A
 * transform is three local phases with an all-to-all exchange of equal blocks
 * (exchange_complex / P complex doubles per peer) between consecutive phases,
 * issued by the caller (NCCL all-to-all, or any other):
 *   dfft: chns_slab_dfft_y, exchange, chns_slab_dfft_x, exchange, chns_slab_dfft_unpack
 *   ifft: chns_slab_ifft_pack, exchange, chns_slab_ifft_x, exchange, chns_slab_ifft_y
 * dfft is unnormalised; ifft includes the reference's 1/(nx ny) and writes only
 * the n reals of each row.  Every pointer is a DEVICE pointer of this rank's
 * GPU; a phase writes its second buffer (send, spec or real) and reads its
 * first; work is enqueued on `stream` (a cudaStream_t).  n is a power of two,
 * 32 <= n <= 4096, n divisible by P with local_nx even.  FP64, as the reference.
 * chns_slab_create allocates the plan's twiddle table on the current device. */
typedef struct chns_slab chns_slab;
int chns_slab_create(int n, int nranks, int rank, chns_slab **out);
void chns_slab_destroy(chns_slab *s);
int chns_slab_sizes(const chns_slab *s, int *local_nx, int *rows_per_rank, size_t *exchange_complex);
int chns_slab_dfft_y(const chns_slab *s, const double *real, size_t real_stride, double *send, void *stream);
int chns_slab_dfft_x(const chns_slab *s, const double *recv, double *send, void *stream);
int chns_slab_dfft_unpack(const chns_slab *s, const double *recv, double *spec, void *stream);
int chns_slab_ifft_pack(const chns_slab *s, const double *spec, double *send, void *stream);
int chns_slab_ifft_x(const chns_slab *s, const double *recv, double *send, void *stream);
int chns_slab_ifft_y(const chns_slab *s, const double *recv, double *real, size_t real_stride, void *stream);

/* Largest grid of chns_dfft_noalloc. */
#define CHNS_NOALLOC_MAX_N 512

/* The reference's dfft (fft.c:11-14) for callers that cannot allocate device
 * memory.  This entry point has no counterpart in the reference: it exists for
 * code that must not call cudaMalloc when it transforms (code running inside
 * another library's allocator or memory pool, or whose device memory is handed
 * out by a host application that owns it).  It needs no context: `real` (n x n
 * doubles) and `spec` (FFTW layout, n x (n/2+1) complex doubles) are DEVICE
 * pointers the caller owns; the transform's one intermediate field lives in a
 * fixed device array of 2 x 257 x 512 complex doubles (4.2 MB) that every GPU
 * loading this library holds until exit, so n must be a power of two with
 * 32 <= n <= CHNS_NOALLOC_MAX_N (else CHNS_ERR_UNSUPPORTED).  The first call on a
 * device does a one-time set-up for that device (symbol lookup, twiddle upload,
 * loading the kernels of every supported n, then a device synchronisation so
 * that the first transform on any stream reads a complete table); make it before
 * any stream capture.  The set-up is redone after a cudaDeviceReset.  All calls
 * share the array:
 * calls that overlap on the GPU race, so order them on one stream.  Work is
 * enqueued on `stream` (a cudaStream_t, NULL = legacy default stream); the call
 * returns without waiting for it. */
int chns_dfft_noalloc(const double *real, double *spec, int n, void *stream);

#ifdef __cplusplus
}
#endif
#endif
