/*
 * Single-rank MPI shim for building the reference C sources as a CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. The reference (MBIR_4D, PCMBIR_3D) is written
 * against MPI, which is absent from this image. One process is one rank:
 * reductions copy, point-to-point calls are never reached on a single rank
 * (every halo call in MBIR_4D/XT_MPI.c:64-80 is guarded by a rank test), and
 * the MPI-IO calls used by MBIR_4D/XT_MPIIO.c:7-59 map onto stdio.
 * Only the names, types and constants the reference uses are provided.
 */
#ifndef ORACLE_MPI_SHIM_H
#define ORACLE_MPI_SHIM_H

#include <stdio.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef struct { int count_bytes; } MPI_Status;
typedef FILE *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_FLOAT 4
#define MPI_DOUBLE 8
#define MPI_SUM 1
#define MPI_INFO_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_CREATE 4

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Wait(MPI_Request *req, MPI_Status *status);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_read_at(MPI_File fh, long offset, void *buf, int count, MPI_Datatype dt, MPI_Status *status);
int MPI_File_write_at(MPI_File fh, long offset, const void *buf, int count, MPI_Datatype dt, MPI_Status *status);
int MPI_File_close(MPI_File *fh);
int MPI_Get_count(const MPI_Status *status, MPI_Datatype dt, int *count);

#endif
