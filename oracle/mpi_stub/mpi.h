/*
 * Serial single-rank stand-in for <mpi.h>, used only to compile the TENSUM
 * reference sources as a CPU oracle (test infrastructure, never product code).
 *
 * With one partition (NPART = 1) and one Monte-Carlo group the reference never
 * reaches a point-to-point call; every such call here aborts loudly so that a
 * configuration which would need real MPI cannot silently run.
 *
 * Collectives behave as on a communicator of size 1: Allreduce copies the
 * send buffer, Barrier and Comm_split are no-ops, Wtime is a steady clock.
 */
#ifndef TENSUM_ORACLE_MPI_STUB_H
#define TENSUM_ORACLE_MPI_STUB_H

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Group;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; int count; };

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_SUM 10
#define MPI_MIN 11
#define MPI_MAX 12
#define MPI_ANY_TAG (-1)
#define MPI_ANY_SOURCE (-2)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

static inline size_t mpi_stub_size(MPI_Datatype t) { return t == MPI_DOUBLE ? sizeof(double) : sizeof(int); }

static inline void mpi_stub_p2p(const char* fn) {
  std::fprintf(stderr, "mpi stub: %s needs more than one rank; not available in the serial oracle\n", fn);
  std::abort();
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { std::fflush(stdout); std::exit(code == 0 ? 1 : code); }
static inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm* out) { *out = 0; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  std::memmove(r, s, (size_t)n * mpi_stub_size(t));
  return 0;
}
static inline double MPI_Wtime() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { mpi_stub_p2p("MPI_Isend"); return 1; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { mpi_stub_p2p("MPI_Irecv"); return 1; }
static inline int MPI_Wait(MPI_Request*, MPI_Status*) { mpi_stub_p2p("MPI_Wait"); return 1; }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { mpi_stub_p2p("MPI_Send"); return 1; }
static inline int MPI_Ssend(const void*, int, MPI_Datatype, int, int, MPI_Comm) { mpi_stub_p2p("MPI_Ssend"); return 1; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { mpi_stub_p2p("MPI_Recv"); return 1; }
static inline int MPI_Probe(int, int, MPI_Comm, MPI_Status*) { mpi_stub_p2p("MPI_Probe"); return 1; }
static inline int MPI_Get_count(const MPI_Status*, MPI_Datatype, int*) { mpi_stub_p2p("MPI_Get_count"); return 1; }

#endif
