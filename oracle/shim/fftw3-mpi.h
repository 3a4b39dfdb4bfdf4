/*
 * fftw3-mpi.h -- stand-in for FFTW3-MPI used only to compile the reference's
 * own sources into the oracle (oracle/_ref).  Test infrastructure, not product.
 *
 * One rank: fftw_mpi_local_size_2d returns the whole slab; the r2c/c2r plans run
 * the oracle's FP64 CPU FFT (oracle/fft_cpu.c) in place on FFTW's padded
 * layout, unnormalised, as the reference's fft.c:11-31 expects.
 * fftw_complex is the C99 double _Complex, as FFTW defines it when <complex.h>
 * is included first (reference global.h:7-9).
 */
#ifndef CHNS_SHIM_FFTW3_MPI_H
#define CHNS_SHIM_FFTW3_MPI_H

#include <stddef.h>
#include <complex.h>
#include <mpi.h>

typedef double _Complex fftw_complex;
typedef struct shim_fftw_plan *fftw_plan;

#define FFTW_ESTIMATE (1U << 6)

#ifdef __cplusplus
extern "C" {
#endif
void fftw_mpi_init(void);
ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start);
fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double *in, fftw_complex *out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex *in, double *out,
                                   MPI_Comm comm, unsigned flags);
void fftw_mpi_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_mpi_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
double *fftw_alloc_real(size_t n);
fftw_complex *fftw_alloc_complex(size_t n);
void fftw_free(void *p);
#ifdef __cplusplus
}
#endif
#endif
