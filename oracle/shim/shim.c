/*
 * shim.c -- single-rank MPI and FFTW3-MPI stand-ins for compiling the
 * reference's own sources into the oracle (oracle/_ref).  Test infrastructure.
 */
#include "mpi.h"
#include "fftw3-mpi.h"
#include "../fft_cpu.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static size_t dtsize(MPI_Datatype t) { return t == MPI_INT ? sizeof(int) : sizeof(double); }

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

int MPI_Abort(MPI_Comm c, int code)
{
    (void)c;
    fprintf(stderr, "oracle shim: MPI_Abort(%d) called by the reference\n", code);
    exit(code ? code : 1);
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)root; (void)c;
    if (s != MPI_IN_PLACE && s != r) memmove(r, s, (size_t)n * dtsize(t));
    return 0;
}

int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    return MPI_Reduce(s, r, n, t, op, 0, c);
}

int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rn; (void)rt; (void)root; (void)c;
    if (s != MPI_IN_PLACE && r && s != r) memmove(r, s, (size_t)sn * dtsize(st));
    return 0;
}

int MPI_Scatter(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rn; (void)rt; (void)root; (void)c;
    if (r != MPI_IN_PLACE && s && s != r) memmove(r, s, (size_t)sn * dtsize(st));
    return 0;
}

/* one-slot mailbox per tag for messages a single rank sends to itself */
#define SHIM_TAGS 64
static void *g_box[SHIM_TAGS];
static size_t g_boxn[SHIM_TAGS];

int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
    (void)c;
    if (dest == MPI_PROC_NULL) return 0;
    int k = tag & (SHIM_TAGS - 1);
    size_t bytes = (size_t)n * dtsize(t);
    free(g_box[k]);
    g_box[k] = malloc(bytes);
    if (g_box[k]) memcpy(g_box[k], b, bytes);
    g_boxn[k] = bytes;
    return 0;
}

int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)c; (void)st;
    if (src == MPI_PROC_NULL) return 0;
    int k = tag & (SHIM_TAGS - 1);
    size_t bytes = (size_t)n * dtsize(t);
    if (g_box[k]) memcpy(b, g_box[k], bytes < g_boxn[k] ? bytes : g_boxn[k]);
    return 0;
}

struct shim_mpi_file { FILE *f; };

int MPI_File_open(MPI_Comm c, const char *name, int mode, MPI_Info info, MPI_File *fh)
{
    (void)c; (void)mode; (void)info;
    *fh = (MPI_File)malloc(sizeof(struct shim_mpi_file));
    (*fh)->f = fopen(name, "wb");
    return (*fh)->f ? 0 : 1;
}

int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void *b, int n, MPI_Datatype t, MPI_Status *st)
{
    (void)st;
    if (!fh || !fh->f) return 1;
    fseek(fh->f, (long)off, SEEK_SET);
    fwrite(b, dtsize(t), (size_t)n, fh->f);
    return 0;
}

int MPI_File_close(MPI_File *fh)
{
    if (fh && *fh) {
        if ((*fh)->f) fclose((*fh)->f);
        free(*fh);
        *fh = NULL;
    }
    return 0;
}

/* ------------------------------- FFTW ----------------------------------- */

struct shim_fftw_plan {
    fftc_plan *p;
    int n0, n1, dir;
};

void fftw_mpi_init(void) {}

ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm comm,
                                 ptrdiff_t *local_n0, ptrdiff_t *local_0_start)
{
    (void)comm;
    *local_n0 = n0;
    *local_0_start = 0;
    return n0 * n1;
}

static fftw_plan mkplan(ptrdiff_t n0, ptrdiff_t n1, int dir)
{
    fftw_plan q = (fftw_plan)malloc(sizeof(*q));
    if (!q) return NULL;
    q->p = fftc_plan_2d((int)n0, (int)n1);
    q->n0 = (int)n0;
    q->n1 = (int)n1;
    q->dir = dir;
    if (!q->p) {
        fprintf(stderr, "oracle shim: unsupported FFT size %ldx%ld\n", (long)n0, (long)n1);
        exit(2);
    }
    return q;
}

fftw_plan fftw_mpi_plan_dft_r2c_2d(ptrdiff_t n0, ptrdiff_t n1, double *in, fftw_complex *out,
                                   MPI_Comm comm, unsigned flags)
{
    (void)in; (void)out; (void)comm; (void)flags;
    return mkplan(n0, n1, -1);
}

fftw_plan fftw_mpi_plan_dft_c2r_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex *in, double *out,
                                   MPI_Comm comm, unsigned flags)
{
    (void)in; (void)out; (void)comm; (void)flags;
    return mkplan(n0, n1, +1);
}

void fftw_mpi_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out)
{
    size_t nd = (size_t)p->n0 * (size_t)(p->n1 + 2);
    if ((void *)in != (void *)out) memcpy(out, in, nd * sizeof(double));
    fftc_r2c_2d(p->p, (double *)out);
}

void fftw_mpi_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out)
{
    size_t nd = (size_t)p->n0 * (size_t)(p->n1 + 2);
    if ((void *)in != (void *)out) memcpy(out, in, nd * sizeof(double));
    fftc_c2r_2d(p->p, out);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    fftc_destroy(p->p);
    free(p);
}

void *fftw_malloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    memset(p, 0, n);
    return p;
}

double *fftw_alloc_real(size_t n) { return (double *)fftw_malloc(n * sizeof(double)); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)fftw_malloc(n * sizeof(fftw_complex)); }
void fftw_free(void *p) { free(p); }
