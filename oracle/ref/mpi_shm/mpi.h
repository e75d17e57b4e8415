/*
 * Multi-process stand-in for the subset of MPI that the Euler3D solver calls, over shared memory.
 * Test infrastructure only: it lets the reference's own multi-rank path -- partitioned meshes, the
 * halo exchange of MPIHandler::updateFlowField and the collectives of the solver loop -- run on one
 * machine without an MPI installation, so that the reference's CPU solver can be timed on N host
 * cores as its users run it (mpiexec -np N).
 *
 * MPI_Init forks the calling process into E3D_MPI_RANKS processes (default 1); rank 0 is the
 * original process.  They share one anonymous memory mapping that holds a barrier, one collective
 * slot per rank and one single-producer/single-consumer channel per ordered pair of ranks.
 * Collectives combine the slots in rank order (so a sum is the same on every rank); point-to-point
 * messages go through the channels in chunks, and MPI_Sendrecv interleaves its send and receive so
 * that two ranks exchanging large messages cannot block each other.  Every wait gives up after
 * E3D_MPI_TIMEOUT seconds (default 900) and aborts the process group with a message.
 *
 * Call sites this covers (reference tree): MPI_Init/Comm_rank/Comm_size
 * src/parallelization/MPIHandler.cpp:8-10, Gather/Send/Recv/Bcast :38-77, Barrier/Sendrecv :85-265,
 * Gather :286; Allreduce src/solver/EulerSolver.cpp:98 and src/solver/FlowField.cpp:52; Bcast
 * src/solver/EulerSolver.cpp:416; Reduce src/mesh/Metrics.cpp:49,267, include/mesh/Mesh.hpp:90,
 * src/parser/MeshPartition.cpp:119; Wtime everywhere.
 */
#pragma once

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
	int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
/* The datatype constants are their element sizes in bytes; MPI_INT is summed as int. */
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_DOUBLE_PRECISION 8
#define MPI_SUM 1
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *) 0)

#ifdef __cplusplus
extern "C" {
#endif
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm, int *rank);
int MPI_Comm_size(MPI_Comm, int *size);
int MPI_Barrier(MPI_Comm);
double MPI_Wtime(void);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm);
int MPI_Bcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm);
int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm);
int MPI_Send(const void *buf, int n, MPI_Datatype t, int dest, int tag, MPI_Comm);
int MPI_Recv(void *buf, int n, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status *);
int MPI_Sendrecv(const void *sbuf, int sn, MPI_Datatype st, int dest, int stag, void *rbuf, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm, MPI_Status *);
#ifdef __cplusplus
}
#endif
