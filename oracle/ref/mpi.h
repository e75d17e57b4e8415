/*
 * Single-process stand-in for the subset of MPI that the Euler3D solver
 * executable calls.  Test infrastructure only: it lets the reference solver
 * sources be compiled into the checker binary under oracle/_ref on a machine
 * without an MPI installation.  With one rank every collective is a copy
 * from the send buffer to the receive buffer and point-to-point calls are
 * never reached (the reference only issues them between distinct ranks).
 *
 * Call sites this covers (reference tree): MPI_Init/Comm_rank/Comm_size
 * src/parallelization/MPIHandler.cpp:8-10, Gather/Send/Recv/Bcast :38-77,
 * Barrier/Sendrecv :85-265, Gather :286; Allreduce src/solver/EulerSolver.cpp:98
 * and src/solver/FlowField.cpp:52; Reduce src/mesh/Metrics.cpp:49,267,
 * include/mesh/Mesh.hpp:90, src/parser/MeshPartition.cpp:119; Wtime everywhere.
 */
#pragma once
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
	int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_DOUBLE_PRECISION 8
#define MPI_SUM 1
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) {
	*rank = 0;
	return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm, int *size) {
	*size = 1;
	return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline double MPI_Wtime(void) {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}
/* The datatype constants above are their element sizes in bytes. */
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
	if (n > 0 && s != r) memcpy(r, s, (size_t) n * (size_t) t);
	return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
	if (n > 0 && s != r) memcpy(r, s, (size_t) n * (size_t) t);
	return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) {
	if (n > 0 && s != r) memcpy(r, s, (size_t) n * (size_t) t);
	return MPI_SUCCESS;
}
/* Never reached with one rank; they report failure if they ever are. */
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 1; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 1; }
static inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int, void *, int, MPI_Datatype, int, int,
                               MPI_Comm, MPI_Status *) { return 1; }
