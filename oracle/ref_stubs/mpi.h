/* Single-process stand-in for the MPI calls of the reference's generic_simple_v1
 * (MPI_Init/Finalize, rank/size of a one-rank world, MPI_Abort, MPI_Wtime).
 * TEST INFRASTRUCTURE ONLY. */
#ifndef ANB_MPI_STUB_H
#define ANB_MPI_STUB_H
#include <chrono>
#include <cstdio>
#include <cstdlib>
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::fflush(stdout); std::exit(code ? (code & 0xff ? code & 0xff : 1) : 1); }
inline double MPI_Wtime() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
#endif
