/*
 * Single-rank stand-in for <mpi.h>, used only to build the reference's own
 * RTM driver as a checker (oracle/build_ref.sh).  With one rank and a
 * 1x1x1 subdomain split the reference creates no halo requests, so every
 * point-to-point call is a no-op and the rank/size queries return 0/1.
 */
#ifndef JVREF_MPI_STUB_H
#define JVREF_MPI_STUB_H
#include <time.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Send_init(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q) { *q = 0; return 0; }
static inline int MPI_Recv_init(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *q) { *q = 0; return 0; }
static inline int MPI_Start(MPI_Request *) { return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline double MPI_Wtime(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}
#endif
