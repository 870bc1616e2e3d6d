/*
 * Single-process MPI stand-in used only to compile the reference's
 * MCnptColloid.c on a machine without an MPI installation.
 *
 * Test infrastructure: this header and mpistub.c let oracle/build_ref.sh build
 * the reference's serial functions (pij_GB, GBCollRod, tot_ene,
 * attempt_monte_carlo_move, ...) into oracle/_ref/ so that tests can call them
 * as the ground truth.  Every call is a no-op for a world of size 1; nothing in
 * the product links against it.
 */
#ifndef LCMC_ORACLE_MPISTUB_H
#define LCMC_ORACLE_MPISTUB_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_FLOAT 3
#define MPI_BYTE 4
#define MPI_PACKED 5
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm c, int *n);
int MPI_Comm_rank(MPI_Comm c, int *r);
int MPI_Dims_create(int n, int nd, int *dims);
int MPI_Barrier(MPI_Comm c);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st);
int MPI_Get_address(const void *p, MPI_Aint *a);
MPI_Aint MPI_Aint_diff(MPI_Aint a, MPI_Aint b);
int MPI_Type_create_struct(int n, const int *bl, const MPI_Aint *disp, const MPI_Datatype *types, MPI_Datatype *nt);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Pack_size(int count, MPI_Datatype t, MPI_Comm c, int *size);
int MPI_Pack(const void *in, int count, MPI_Datatype t, void *out, int outsize, int *pos, MPI_Comm c);
int MPI_Unpack(const void *in, int insize, int *pos, void *out, int count, MPI_Datatype t, MPI_Comm c);

#endif
