/*
 * mpi.h -- single-rank MPI stand-in used only to compile the reference's own
 * sources into the oracle (oracle/_ref).  Test infrastructure, not product.
 *
 * Covers exactly the subset the reference calls (main.c:37-40, free_energy.c:60,
 * kinetic_energy.c:96-120, perimeter.c:54-113, spectrum.c:123-141,
 * init.c:132, read_array.c:34-35, write_array.c:27,71-77): with one rank every
 * reduction, gather and scatter is a copy, and point-to-point messages to self
 * are buffered.
 */
#ifndef CHNS_SHIM_MPI_H
#define CHNS_SHIM_MPI_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef struct shim_mpi_file *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_SUM 1
#define MPI_INFO_NULL 0
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 2
#define MPI_PROC_NULL (-1)
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Barrier(MPI_Comm c);
int MPI_Abort(MPI_Comm c, int code);
double MPI_Wtime(void);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Scatter(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_File_open(MPI_Comm c, const char *name, int mode, MPI_Info info, MPI_File *fh);
int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void *b, int n, MPI_Datatype t, MPI_Status *st);
int MPI_File_close(MPI_File *fh);
#ifdef __cplusplus
}
#endif
#endif
