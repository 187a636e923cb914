/* TEST INFRASTRUCTURE ONLY: single-process stand-in for the MPI calls the
 * reference solver makes when run as one rank.  A 1x1x1 Cartesian communicator:
 * shifts along a periodic axis return this rank (the reference then exchanges
 * its periodic halos with itself through MPI_Sendrecv, which becomes a copy),
 * shifts along other axes return MPI_PROC_NULL; reductions over one rank copy. */
#ifndef KFVM_REFSHIM_MPI_H
#define KFVM_REFSHIM_MPI_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_CHAR 4
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int kfvm_shim_mpi_size(MPI_Datatype t) {
  return t == MPI_DOUBLE ? 8 : (t == MPI_CHAR ? 1 : 4);
}
static inline int *kfvm_shim_mpi_periods(void) {
  static int periods[3] = {0, 0, 0};
  return periods;
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Cart_create(MPI_Comm, int nd, const int *, const int *periods, int,
                                  MPI_Comm *out) {
  for (int d = 0; d < nd && d < 3; d++) kfvm_shim_mpi_periods()[d] = periods[d];
  *out = MPI_COMM_WORLD;
  return 0;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int nd, int *c) {
  for (int d = 0; d < nd; d++) c[d] = 0;
  return 0;
}
static inline int MPI_Cart_shift(MPI_Comm, int dir, int, int *src, int *dst) {
  int p = kfvm_shim_mpi_periods()[dir];
  *src = p ? 0 : MPI_PROC_NULL;
  *dst = p ? 0 : MPI_PROC_NULL;
  return 0;
}
static inline int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest,
                               int, void *rbuf, int rcount, MPI_Datatype rtype, int source,
                               int, MPI_Comm, MPI_Status *) {
  if (dest == MPI_PROC_NULL || source == MPI_PROC_NULL) return 0;
  int n = scount * kfvm_shim_mpi_size(stype);
  int m = rcount * kfvm_shim_mpi_size(rtype);
  memcpy(rbuf, sbuf, (size_t)(n < m ? n : m));
  return 0;
}
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op,
                                MPI_Comm) {
  if (in != MPI_IN_PLACE && in != out) memcpy(out, in, (size_t)n * kfvm_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, int,
                             MPI_Comm) {
  if (in != MPI_IN_PLACE && in != out) memcpy(out, in, (size_t)n * kfvm_shim_mpi_size(t));
  return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

#endif
