/*
 * Serial stand-in for <mpi.h>, enough for CoupLB/couplb_streaming.h to compile
 * on one rank (TEST INFRASTRUCTURE ONLY, used by oracle/ref_harness.cpp).
 * With one rank every MPI_Sendrecv sends to itself, so it is a copy of the
 * send buffer into the receive buffer.
 */
#ifndef COUPLB_ORACLE_MPI_STUB_H
#define COUPLB_ORACLE_MPI_STUB_H
#include <cstring>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_PROC_NULL (-1)
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_STATUS_IGNORE nullptr
inline int MPI_Sendrecv(const void* sb, int count, MPI_Datatype t, int, int,
                        void* rb, int, MPI_Datatype, int, int, MPI_Comm,
                        MPI_Status*) {
  std::memcpy(rb, sb, static_cast<size_t>(count) * static_cast<size_t>(t));
  return 0;
}
#endif
