/*
 * Single-process stand-in for the MPI subset the reference program calls,
 * so that its unmodified sources build without an MPI installation (none is
 * available on these machines).  TEST INFRASTRUCTURE ONLY: used by
 * oracle/ref/Makefile to build oracle/_ref/openstc_ref, whose outputs pin the
 * CPU oracle.  With one rank every collective is a copy and the file calls
 * map to pread/pwrite; subarray datatypes (Fortran order, the only form the
 * reference creates) are gathered / scattered element by element.
 */
#ifndef OSTC_SINGLE_RANK_MPI_H
#define OSTC_SINGLE_RANK_MPI_H

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_SUM 1
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_ORDER_FORTRAN 57
#define MPI_ORDER_C 56
#define MPI_SUCCESS 0

#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_INT32_T 5
#define MPI_INT64_T 6
#define MPI_C_BOOL 7
#define OSTC_MPI_FIRST_DERIVED 16

struct ostc_mpi_subarray {
  int ndims, order;
  int sizes[3], subsizes[3], starts[3];
  MPI_Datatype base;
};

static inline struct ostc_mpi_subarray *ostc_mpi_types(void) {
  static struct ostc_mpi_subarray table[256];
  return table;
}
static inline int *ostc_mpi_ntypes(void) {
  static int n = 0;
  return &n;
}

static inline size_t ostc_mpi_basic_size(MPI_Datatype t) {
  switch (t) {
    case MPI_CHAR: case MPI_C_BOOL: return 1;
    case MPI_INT: case MPI_FLOAT: case MPI_INT32_T: return 4;
    case MPI_DOUBLE: case MPI_INT64_T: return 8;
    default: return 0;
  }
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) {
  fflush(stdout);
  exit(code);
}
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  memmove(r, s, n * ostc_mpi_basic_size(t));
  return 0;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  memmove(r, s, n * ostc_mpi_basic_size(t));
  return 0;
}
static inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
  memmove(r, s, n * ostc_mpi_basic_size(t));
  return 0;
}
static inline int MPI_Allgatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *displs,
                                 MPI_Datatype, MPI_Comm) {
  memmove((char *)r + displs[0] * ostc_mpi_basic_size(t), s, n * ostc_mpi_basic_size(t));
  return 0;
}
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  fprintf(stderr, "single-rank MPI: point-to-point messages are not available\n");
  abort();
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  fprintf(stderr, "single-rank MPI: point-to-point messages are not available\n");
  abort();
}
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }

static inline int MPI_Type_create_subarray(int ndims, const int *sizes, const int *subsizes, const int *starts,
                                           int order, MPI_Datatype base, MPI_Datatype *out) {
  int *n = ostc_mpi_ntypes();
  if (ndims != 3 || order != MPI_ORDER_FORTRAN || *n >= 256) {
    fprintf(stderr, "single-rank MPI: unsupported subarray type\n");
    abort();
  }
  struct ostc_mpi_subarray *a = &ostc_mpi_types()[*n];
  a->ndims = ndims;
  a->order = order;
  for (int q = 0; q < 3; ++q) {
    a->sizes[q] = sizes[q];
    a->subsizes[q] = subsizes[q];
    a->starts[q] = starts[q];
  }
  a->base = base;
  *out = OSTC_MPI_FIRST_DERIVED + (*n)++;
  return 0;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return 0; }

static inline int MPI_File_open(MPI_Comm, const char *name, int amode, MPI_Info, MPI_File *fh) {
  int flags = (amode & MPI_MODE_RDONLY) ? O_RDONLY : O_WRONLY;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
  *fh = open(name, flags, 0644);
  return *fh < 0 ? 1 : 0;
}
static inline int MPI_File_close(MPI_File *fh) {
  if (*fh >= 0) close(*fh);
  *fh = -1;
  return 0;
}

/* Moves `count` items of type t between memory `mem` and the file range at
   `off`; write = 1 copies memory to file. */
static inline int ostc_mpi_file_io(MPI_File fh, MPI_Offset off, void *mem, int count, MPI_Datatype t, int write) {
  if (t < OSTC_MPI_FIRST_DERIVED) {
    const size_t n = count * ostc_mpi_basic_size(t);
    const ssize_t r = write ? pwrite(fh, mem, n, off) : pread(fh, mem, n, off);
    return r == (ssize_t)n ? 0 : 1;
  }
  const struct ostc_mpi_subarray *a = &ostc_mpi_types()[t - OSTC_MPI_FIRST_DERIVED];
  const size_t es = ostc_mpi_basic_size(a->base);
  const size_t n = (size_t)a->subsizes[0] * a->subsizes[1] * a->subsizes[2];
  char *buf = (char *)malloc(n * es);
  if (!write && pread(fh, buf, n * es, off) != (ssize_t)(n * es)) {
    free(buf);
    return 1;
  }
  size_t q = 0;
  for (int k = 0; k < a->subsizes[2]; ++k)
    for (int j = 0; j < a->subsizes[1]; ++j)
      for (int i = 0; i < a->subsizes[0]; ++i, ++q) {
        const size_t m = ((size_t)(k + a->starts[2]) * a->sizes[1] + (j + a->starts[1])) * a->sizes[0] + i +
                         a->starts[0];
        if (write) {
          memcpy(buf + q * es, (char *)mem + m * es, es);
        } else {
          memcpy((char *)mem + m * es, buf + q * es, es);
        }
      }
  int rc = 0;
  if (write) rc = pwrite(fh, buf, n * es, off) == (ssize_t)(n * es) ? 0 : 1;
  free(buf);
  return rc;
}
static inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t,
                                    MPI_Status *) {
  return ostc_mpi_file_io(fh, off, (void *)buf, count, t, 1);
}
static inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *) {
  return ostc_mpi_file_io(fh, off, buf, count, t, 0);
}

#endif
