/*
 * mpi.h -- single-rank MPI subset used only to build the reference solver for parity runs
 * (oracle/ref/build_ref.sh).  The reference links MPI for its multi-process decomposition; run as
 * one process on one GPU it only needs these calls to behave as their one-rank semantics define:
 * collectives copy, point-to-point is never reached, and MPI-IO maps onto stdio with subarray and
 * contiguous datatypes describing the memory side of a transfer.  TEST INFRASTRUCTURE ONLY.
 */
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef std::FILE *MPI_File;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

struct ostc_mpi_type {
  int kind;      // 0 basic, 1 contiguous, 2 subarray
  size_t bytes;  // basic element size
  int count;     // contiguous count
  int nd, order;
  int sizes[4], subs[4], starts[4];
  const ostc_mpi_type *old;
};
typedef const ostc_mpi_type *MPI_Datatype;

inline const ostc_mpi_type ostc_mpi_b1{0, 1, 1, 0, 0, {}, {}, {}, nullptr};
inline const ostc_mpi_type ostc_mpi_b4{0, 4, 1, 0, 0, {}, {}, {}, nullptr};
inline const ostc_mpi_type ostc_mpi_b8{0, 8, 1, 0, 0, {}, {}, {}, nullptr};

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_INFO_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)nullptr)
#define MPI_STATUSES_IGNORE ((MPI_Status *)nullptr)
#define MPI_SUCCESS 0
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_ORDER_C 0
#define MPI_ORDER_FORTRAN 1
#define MPI_MODE_CREATE 1
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_RDWR 8
#define MPI_INT (&ostc_mpi_b4)
#define MPI_INT32_T (&ostc_mpi_b4)
#define MPI_INT64_T (&ostc_mpi_b8)
#define MPI_DOUBLE (&ostc_mpi_b8)
#define MPI_FLOAT (&ostc_mpi_b4)
#define MPI_REAL (&ostc_mpi_b4)
#define MPI_CHAR (&ostc_mpi_b1)
#define MPI_BYTE (&ostc_mpi_b1)
#define MPI_OFFSET (&ostc_mpi_b8)

namespace ostc_mpi {
inline size_t data_bytes(MPI_Datatype t) {
  if (t->kind == 0) return t->bytes;
  if (t->kind == 1) return (size_t)t->count * data_bytes(t->old);
  size_t n = 1;
  for (int d = 0; d < t->nd; ++d) n *= (size_t)t->subs[d];
  return n * data_bytes(t->old);
}
inline size_t extent_bytes(MPI_Datatype t) {
  if (t->kind != 2) return data_bytes(t);
  size_t n = 1;
  for (int d = 0; d < t->nd; ++d) n *= (size_t)t->sizes[d];
  return n * extent_bytes(t->old);
}
// copies between a memory buffer laid out by type t (count instances) and a packed byte stream
inline void pack(MPI_Datatype t, int count, char *mem, char *packed, bool to_packed) {
  const size_t ext = extent_bytes(t), db = data_bytes(t);
  for (int c = 0; c < count; ++c) {
    char *m = mem + c * ext, *pk = packed + c * db;
    if (t->kind != 2) {
      if (to_packed) std::memcpy(pk, m, db);
      else std::memcpy(m, pk, db);
      continue;
    }
    const size_t eb = extent_bytes(t->old);
    long long stride[4];
    int dims[4];
    for (int d = 0; d < t->nd; ++d) dims[d] = t->order == MPI_ORDER_FORTRAN ? d : t->nd - 1 - d;
    long long st = 1;
    for (int q = 0; q < t->nd; ++q) {  // q-th fastest dimension
      stride[dims[q]] = st;
      st *= t->sizes[dims[q]];
    }
    int idx[4] = {0, 0, 0, 0};
    size_t n = 1;
    for (int d = 0; d < t->nd; ++d) n *= (size_t)t->subs[d];
    for (size_t e = 0; e < n; ++e) {
      long long off = 0;
      for (int d = 0; d < t->nd; ++d) off += (long long)(t->starts[d] + idx[d]) * stride[d];
      if (to_packed) std::memcpy(pk + e * eb, m + off * eb, eb);
      else std::memcpy(m + off * eb, pk + e * eb, eb);
      for (int q = 0; q < t->nd; ++q) {  // odometer over the sub-box, fastest dimension first
        const int d = dims[q];
        if (++idx[d] < t->subs[d]) break;
        idx[d] = 0;
      }
    }
  }
}
}  // namespace ostc_mpi

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::fflush(stdout); std::exit(code == 0 ? 1 : code); }
inline double MPI_Wtime() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != r) std::memmove(r, s, n * ostc_mpi::data_bytes(t));
  return 0;
}
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (r && s != r) std::memmove(r, s, n * ostc_mpi::data_bytes(t));
  return 0;
}
inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != r) std::memmove(r, s, n * ostc_mpi::data_bytes(t));
  return 0;
}
inline int MPI_Allgatherv(const void *s, int n, MPI_Datatype t, void *r, const int *, const int *displs,
                          MPI_Datatype rt, MPI_Comm) {
  std::memmove((char *)r + (size_t)displs[0] * ostc_mpi::data_bytes(rt), s, n * ostc_mpi::data_bytes(t));
  return 0;
}
inline int MPI_Scatter(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) {
  if (s != r) std::memmove(r, s, n * ostc_mpi::data_bytes(t));
  return 0;
}
inline int MPI_Scatterv(const void *s, const int *counts, const int *displs, MPI_Datatype t, void *r, int,
                        MPI_Datatype, int, MPI_Comm) {
  std::memmove(r, (const char *)s + (size_t)displs[0] * ostc_mpi::data_bytes(t), counts[0] * ostc_mpi::data_bytes(t));
  return 0;
}
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  std::fprintf(stderr, "single-rank MPI: point-to-point send reached\n");
  std::exit(3);
}
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  std::fprintf(stderr, "single-rank MPI: point-to-point receive reached\n");
  std::exit(3);
}
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
inline int MPI_Type_create_subarray(int nd, const int *sizes, const int *subs, const int *starts, int order,
                                    MPI_Datatype old, MPI_Datatype *nt) {
  auto *t = new ostc_mpi_type{2, 0, 1, nd, order, {}, {}, {}, old};
  for (int d = 0; d < nd; ++d) {
    t->sizes[d] = sizes[d];
    t->subs[d] = subs[d];
    t->starts[d] = starts[d];
  }
  *nt = t;
  return 0;
}
inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype *nt) {
  *nt = new ostc_mpi_type{1, 0, n, 0, 0, {}, {}, {}, old};
  return 0;
}
inline int MPI_Type_commit(MPI_Datatype *) { return 0; }
inline int MPI_Type_free(MPI_Datatype *t) {
  if (t && *t && (*t)->kind != 0) delete *t;
  if (t) *t = nullptr;
  return 0;
}
inline int MPI_File_open(MPI_Comm, const char *name, int mode, MPI_Info, MPI_File *fh) {
  if (mode & MPI_MODE_RDONLY) *fh = std::fopen(name, "rb");
  else {
    *fh = std::fopen(name, "r+b");
    if (!*fh && (mode & MPI_MODE_CREATE)) *fh = std::fopen(name, "w+b");
  }
  if (!*fh) {
    std::fprintf(stderr, "single-rank MPI: cannot open %s\n", name);
    std::exit(4);
  }
  return 0;
}
inline int MPI_File_close(MPI_File *fh) {
  if (*fh) std::fclose(*fh);
  *fh = nullptr;
  return 0;
}
inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int n, MPI_Datatype t, MPI_Status *) {
  std::vector<char> pk(n * ostc_mpi::data_bytes(t));
  std::fseek(fh, off, SEEK_SET);
  if (std::fread(pk.data(), 1, pk.size(), fh) != pk.size()) std::memset(pk.data(), 0, pk.size());
  ostc_mpi::pack(t, n, (char *)buf, pk.data(), false);
  return 0;
}
inline int MPI_File_read(MPI_File fh, void *buf, int n, MPI_Datatype t, MPI_Status *) {
  std::vector<char> pk(n * ostc_mpi::data_bytes(t));
  if (std::fread(pk.data(), 1, pk.size(), fh) != pk.size()) std::memset(pk.data(), 0, pk.size());
  ostc_mpi::pack(t, n, (char *)buf, pk.data(), false);
  return 0;
}
inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int n, MPI_Datatype t, MPI_Status *) {
  std::vector<char> pk(n * ostc_mpi::data_bytes(t));
  ostc_mpi::pack(t, n, (char *)buf, pk.data(), true);
  std::fseek(fh, off, SEEK_SET);
  std::fwrite(pk.data(), 1, pk.size(), fh);
  return 0;
}
