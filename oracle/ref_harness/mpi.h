// Single-rank stand-in for the MPI calls the reference's parallel-output and
// restart code makes (OSHUN-1/def-Parallel.cpp).  Test infrastructure only:
// the checker runs one rank on one node, so no message is ever sent.
#ifndef OSHUN_REF_MPI_STUB_H
#define OSHUN_REF_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_FLOAT 2
#define MPI_INT 3
#define MPI_DOUBLE_COMPLEX 4
#define MPI_SUM 0
#define MPI_MAX 1
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Send(void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
#endif
