/*
 * Single-rank MPI shim (test infrastructure only). See mpi.h for scope.
 * A datatype value is its element size in bytes, so copies and file I/O
 * need no lookup table.
 */
#include <stdio.h>
#include <string.h>
#include "mpi.h"

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return 0; }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return 0; }

/* A single rank never has a neighbour, so the reference never reaches these. */
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm, MPI_Request *req)
{ (void)buf; (void)count; (void)dt; (void)dest; (void)tag; (void)comm; *req = 0; return 0; }
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int src, int tag, MPI_Comm comm, MPI_Request *req)
{ (void)buf; (void)count; (void)dt; (void)src; (void)tag; (void)comm; *req = 0; return 0; }
int MPI_Wait(MPI_Request *req, MPI_Status *status) { (void)req; (void)status; return 0; }

int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root, MPI_Comm comm)
{ (void)op; (void)root; (void)comm; memmove(recvbuf, sendbuf, (size_t)count * (size_t)dt); return 0; }
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm comm)
{ (void)op; (void)comm; memmove(recvbuf, sendbuf, (size_t)count * (size_t)dt); return 0; }
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm)
{ (void)buf; (void)count; (void)dt; (void)root; (void)comm; return 0; }

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh)
{
    (void)comm; (void)info;
    if (amode & MPI_MODE_RDONLY) {
        *fh = fopen(filename, "rb");
    } else {
        /* MPI_MODE_CREATE|MPI_MODE_WRONLY keeps existing bytes (no truncation). */
        *fh = fopen(filename, "r+b");
        if (!*fh && (amode & MPI_MODE_CREATE)) *fh = fopen(filename, "w+b");
    }
    return *fh ? 0 : 1;
}

int MPI_File_read_at(MPI_File fh, long offset, void *buf, int count, MPI_Datatype dt, MPI_Status *status)
{
    size_t n = 0;
    if (fh && fseek(fh, offset, SEEK_SET) == 0) n = fread(buf, (size_t)dt, (size_t)count, fh);
    if (status) status->count_bytes = (int)(n * (size_t)dt);
    return 0;
}

int MPI_File_write_at(MPI_File fh, long offset, const void *buf, int count, MPI_Datatype dt, MPI_Status *status)
{
    size_t n = 0;
    if (fh && fseek(fh, offset, SEEK_SET) == 0) n = fwrite(buf, (size_t)dt, (size_t)count, fh);
    if (status) status->count_bytes = (int)(n * (size_t)dt);
    return 0;
}

int MPI_File_close(MPI_File *fh)
{
    if (fh && *fh) { fclose(*fh); *fh = NULL; }
    return 0;
}

int MPI_Get_count(const MPI_Status *status, MPI_Datatype dt, int *count)
{
    *count = status ? status->count_bytes / (int)dt : MPI_UNDEFINED;
    return 0;
}
