/*
 * Single-rank stand-in for the MPI interface, used only to compile the
 * reference library (TIMBIR v0.0.2, src/MBIR_4D) as a CPU oracle on a machine
 * without an MPI installation.  It is test infrastructure: nothing in the
 * product links it.
 *
 * Semantics are those of MPI with exactly one process:
 *   - MPI_Comm_size -> 1, MPI_Comm_rank -> 0;
 *   - reductions (Reduce, Allreduce) copy the send buffer to the receive
 *     buffer, Bcast does nothing;
 *   - point-to-point calls are never reached at one rank (the reference guards
 *     them with rank > 0 / rank < size-1, src/MBIR_4D/XT_MPI.c:66-79); they
 *     are accepted and do nothing;
 *   - MPI-IO maps onto stdio; a file opened with MPI_MODE_CREATE|MPI_MODE_WRONLY
 *     is not truncated, as in MPI.
 */
#ifndef ORACLE_SINGLE_RANK_MPI_H
#define ORACLE_SINGLE_RANK_MPI_H

#include <stdio.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { long count; } MPI_Status;
typedef FILE *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_SUM 0
#define MPI_INFO_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1

static size_t oracle_mpi_type_size(MPI_Datatype t) { return (size_t)t; }

static int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static int MPI_Finalize(void) { return 0; }
static int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
static int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }

static int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, int root, MPI_Comm c)
{
	(void)o; (void)root; (void)c;
	memmove(r, s, (size_t)n * oracle_mpi_type_size(t));
	return 0;
}
static int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op o, MPI_Comm c)
{
	(void)o; (void)c;
	memmove(r, s, (size_t)n * oracle_mpi_type_size(t));
	return 0;
}
static int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c)
{
	(void)b; (void)n; (void)t; (void)root; (void)c;
	return 0;
}
static int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *q)
{
	(void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; *q = 0;
	return 0;
}
static int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *q)
{
	(void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *q = 0;
	return 0;
}
static int MPI_Wait(MPI_Request *q, MPI_Status *st) { (void)q; (void)st; return 0; }

static int MPI_File_open(MPI_Comm c, const char *name, int mode, MPI_Info info, MPI_File *fh)
{
	(void)c; (void)info;
	if (mode & MPI_MODE_RDONLY)
		*fh = fopen(name, "rb");
	else {
		*fh = fopen(name, "r+b");
		if (*fh == NULL && (mode & MPI_MODE_CREATE))
			*fh = fopen(name, "w+b");
	}
	return *fh == NULL ? 1 : 0;
}
static int MPI_File_read_at(MPI_File fh, long long off, void *buf, int n, MPI_Datatype t, MPI_Status *st)
{
	size_t got = 0;
	if (fh != NULL && fseek(fh, (long)off, SEEK_SET) == 0)
		got = fread(buf, oracle_mpi_type_size(t), (size_t)n, fh);
	if (st) st->count = (long)got;
	return 0;
}
static int MPI_File_write_at(MPI_File fh, long long off, const void *buf, int n, MPI_Datatype t, MPI_Status *st)
{
	size_t put = 0;
	if (fh != NULL && fseek(fh, (long)off, SEEK_SET) == 0)
		put = fwrite(buf, oracle_mpi_type_size(t), (size_t)n, fh);
	if (st) st->count = (long)put;
	return 0;
}
static int MPI_File_close(MPI_File *fh)
{
	if (*fh) fclose(*fh);
	*fh = NULL;
	return 0;
}
static int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n)
{
	(void)t;
	*n = (int)st->count;
	return 0;
}

#endif
