/* Single-rank stand-in for the subset of MPI that the reference CCD code calls.
 *
 * Test infrastructure only: it lets the unmodified reference sources compile and run
 * as one rank in a container without an MPI installation.  A datatype is encoded as
 * its size in bytes, every collective is a local copy from the send buffer to the
 * receive buffer (what MPI does when the communicator holds exactly one rank), and
 * Comm_size is 1.  Call sites in the reference: Chain.hpp:740,794,844, Chain.cpp:7-8,
 * 100,134,174,208, main.cpp:28-31,172,215,286,423,451,476,586,668,739.
 */
#ifndef CCD_ORACLE_MPI_STUB_H
#define CCD_ORACLE_MPI_STUB_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_SUM 0
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_LONG_LONG ((MPI_Datatype)sizeof(long long))
#define MPI_UNSIGNED ((MPI_Datatype)sizeof(unsigned))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_UNSIGNED_SHORT ((MPI_Datatype)sizeof(unsigned short))

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

static inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *out) {
  *out = count * old;
  return 0;
}
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }

/* One rank: the "reduction" of a single contribution is that contribution. */
static inline int MPI_Reduce(const void *send, void *recv, int count, MPI_Datatype t,
                             MPI_Op op, int root, MPI_Comm c) {
  (void)op; (void)root; (void)c;
  memmove(recv, send, (size_t)count * (size_t)t);
  return 0;
}
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t,
                                MPI_Op op, MPI_Comm c) {
  (void)op; (void)c;
  memmove(recv, send, (size_t)count * (size_t)t);
  return 0;
}

/* One rank: rank 0 sends its block 0 to itself. */
static inline int MPI_Alltoall(const void *send, int scount, MPI_Datatype st, void *recv,
                               int rcount, MPI_Datatype rt, MPI_Comm c) {
  (void)rcount; (void)rt; (void)c;
  memmove(recv, send, (size_t)scount * (size_t)st);
  return 0;
}
static inline int MPI_Alltoallv(const void *send, const int *scounts, const int *sdispls,
                                MPI_Datatype st, void *recv, const int *rcounts,
                                const int *rdispls, MPI_Datatype rt, MPI_Comm c) {
  (void)rcounts; (void)c;
  memmove((char *)recv + (size_t)rdispls[0] * (size_t)rt,
          (const char *)send + (size_t)sdispls[0] * (size_t)st,
          (size_t)scounts[0] * (size_t)st);
  return 0;
}
static inline int MPI_Allgatherv(const void *send, int scount, MPI_Datatype st, void *recv,
                                 const int *rcounts, const int *displs, MPI_Datatype rt,
                                 MPI_Comm c) {
  (void)rcounts; (void)c;
  memmove((char *)recv + (size_t)displs[0] * (size_t)rt, send, (size_t)scount * (size_t)st);
  return 0;
}

#endif
