/*
 * fft_cpu.h -- FP64 CPU 2D real FFT used by the oracle (test infrastructure only).
 *
 * This is the transform behind the oracle's restatement of the reference's
 * fft.c (dfft/ifft, fft.c:11-31) and behind the FFTW-MPI shim that lets the
 * reference's own sources be compiled here.  It is NOT part of the product:
 * only tests, the smoke check and bench.py's CPU baseline ever run it.
 *
 * Layout is FFTW's in-place r2c layout (reference global.h:13-14):
 *   real view    : n0 rows x (n1 + 2) doubles, row-major (IDXR(i,j) = j + (n1+2) i)
 *   complex view : n0 rows x (n1/2 + 1) complex, interleaved re/im (IDXC)
 * r2c is unnormalised; c2r is unnormalised (fft.c applies the 1/(n0 n1)).
 * c2r follows FFTW's c2r convention: the imaginary parts of the j = 0 and
 * j = n1/2 bins of each row are ignored by the final 1D c2r along the row.
 */
#ifndef CHNS_ORACLE_FFT_CPU_H
#define CHNS_ORACLE_FFT_CPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fftc_plan fftc_plan;

/* n0, n1: powers of two >= 4. Returns NULL on bad sizes / OOM. */
fftc_plan *fftc_plan_2d(int n0, int n1);
void fftc_destroy(fftc_plan *p);

/* In-place on a padded buffer of n0*(n1+2) doubles. */
void fftc_r2c_2d(fftc_plan *p, double *data);
void fftc_c2r_2d(fftc_plan *p, double *data);

/* 1D complex FFT of length n (power of two), in place, unnormalised.
 * sign = -1 forward (exp(-2 pi i jk/n)), +1 inverse. */
void fftc_c2c_1d(int n, double *z, int sign);

/* Rounding order of the transforms (default 0): 0 = radix-4 stages with two real
 * rows packed into one complex transform; 1 = radix-2 stages, one real row per
 * complex transform.  Both compute the same DFT; comparing runs under the two
 * measures how much the FFT's own rounding moves a trajectory. */
void fftc_set_variant(int v);
int fftc_get_variant(void);

/* Number of host threads used for the 2D passes (default 1). */
void fftc_set_threads(int nthreads);
int fftc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
