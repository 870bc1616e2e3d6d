/*
 * No-op single-rank MPI symbols for building the reference's serial functions
 * (see mpi.h beside this file).  Test infrastructure only.
 */
#include <string.h>
#include "mpi.h"

static int dtype_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_INT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_FLOAT: return 4;
    default: return 1;
    }
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Dims_create(int n, int nd, int *dims)
{
    (void)n;
    for (int i = 0; i < nd; i++) dims[i] = 1;
    return 0;
}
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
int MPI_Bcast(void *b, int n, MPI_Datatype t, int r, MPI_Comm c) { (void)b; (void)n; (void)t; (void)r; (void)c; return 0; }
int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c) { (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; return 0; }
int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Status *st) { (void)b; (void)n; (void)t; (void)s; (void)g; (void)c; (void)st; return 0; }
int MPI_Probe(int s, int g, MPI_Comm c, MPI_Status *st) { (void)s; (void)g; (void)c; if (st) st->count = 0; return 0; }
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n) { (void)t; *n = st ? st->count : 0; return 0; }
int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c, MPI_Request *q) { (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; if (q) *q = 0; return 0; }
int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Request *q) { (void)b; (void)n; (void)t; (void)s; (void)g; (void)c; if (q) *q = 0; return 0; }
int MPI_Waitall(int n, MPI_Request *q, MPI_Status *st) { (void)n; (void)q; (void)st; return 0; }
int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return 0; }
MPI_Aint MPI_Aint_diff(MPI_Aint a, MPI_Aint b) { return a - b; }
int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *d, const MPI_Datatype *t, MPI_Datatype *nt) { (void)n; (void)bl; (void)d; (void)t; *nt = MPI_BYTE; return 0; }
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Pack_size(int n, MPI_Datatype t, MPI_Comm c, int *size) { (void)c; *size = n * dtype_size(t); return 0; }
int MPI_Pack(const void *in, int n, MPI_Datatype t, void *out, int outsize, int *pos, MPI_Comm c)
{
    (void)outsize; (void)c;
    int sz = n * dtype_size(t);
    memcpy((char *)out + *pos, in, (size_t)sz);
    *pos += sz;
    return 0;
}
int MPI_Unpack(const void *in, int insize, int *pos, void *out, int n, MPI_Datatype t, MPI_Comm c)
{
    (void)insize; (void)c;
    int sz = n * dtype_size(t);
    memcpy(out, (const char *)in + *pos, (size_t)sz);
    *pos += sz;
    return 0;
}
