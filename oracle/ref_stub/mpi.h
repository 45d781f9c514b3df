/* Single-process stand-in for <mpi.h>, written for this project so that qcu's
 * own sources can be compiled as a parity reference without an MPI install.
 * Rank 0 of a world of size 1: broadcasts are no-ops and point-to-point calls
 * are never reached because qcu only takes the MPI branches when a grid
 * dimension is larger than 1 (include/lattice_dslash.h:198-456). */
#ifndef QCU_REF_STUB_MPI_H
#define QCU_REF_STUB_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_BYTE 1
#define MPI_DOUBLE 2
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
  (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS; }
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c,
                            MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)dst; (void)tag; (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c,
                            MPI_Request *r) {
  (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Wait(MPI_Request *r, MPI_Status *s) { (void)r; (void)s; return MPI_SUCCESS; }
#endif
