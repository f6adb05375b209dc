/*
 * Single-rank MPI stand-in used only to compile the reference's plain-C
 * hopping pair as a CPU oracle (test infrastructure, never shipped).
 *
 * The reference calls MPI for rank bookkeeping and for half-spinor face
 * exchange (lib/dirac.c:124-131, 203-228; lib/start.c:28-47). With a
 * 1x1x1x1 process grid every face exchange is skipped by the reference
 * itself (`if (plqcd_g.nprocs[mu] > 1)`), so the only calls that run are
 * Init/Comm_size/Comm_rank/Get_processor_name/Finalize. Everything here is
 * a no-op that reports one rank and success.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Op;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_THREAD_SERIALIZED 2

static inline int MPI_Init(int *c, char ***v) { (void)c; (void)v; return 0; }
static inline int MPI_Init_thread(int *c, char ***v, int r, int *p) { (void)c; (void)v; *p = r; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm c, int e) { (void)c; (void)e; return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *n) { (void)c; *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
static inline int MPI_Get_processor_name(char *s, int *len) { strcpy(s, "oracle"); *len = 6; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c, MPI_Request *r)
{ (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; *r = 0; return 0; }
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Request *r)
{ (void)b; (void)n; (void)t; (void)s; (void)g; (void)c; *r = 0; return 0; }
static inline int MPI_Wait(MPI_Request *r, MPI_Status *s) { (void)r; (void)s; return 0; }
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int g, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)d; (void)g; (void)c; return 0; }
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int g, MPI_Comm c, MPI_Status *st)
{ (void)b; (void)n; (void)t; (void)s; (void)g; (void)c; (void)st; return 0; }
static inline int MPI_Reduce(const void *a, void *b, int n, MPI_Datatype t, MPI_Op o, int r, MPI_Comm c)
{ (void)o; (void)r; (void)c; memcpy(b, a, (size_t)n * (t == MPI_DOUBLE ? sizeof(double) : sizeof(int))); return 0; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int r, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)r; (void)c; return 0; }
#endif
