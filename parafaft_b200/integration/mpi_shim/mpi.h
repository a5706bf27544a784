/*
 * Single-rank stand-in for <mpi.h>, used only where no MPI is installed.
 *
 * It implements exactly the MPI calls ParaFaFT's headers make
 * (parafaft_common.hpp, parafaft_c2c.hpp, parafaft_r2c.hpp), with the
 * semantics they have on a communicator of one rank:
 *   - every communicator has size 1 and rank 0; Cartesian grids are all-ones;
 *   - collectives copy the send buffer to the receive buffer;
 *   - MPI_Alltoallw copies the committed subarray of the send side into the
 *     subarray of the receive side (the identity exchange of a one-rank
 *     pencil step, parafaft_common.hpp:442-451);
 *   - point-to-point calls are never reached at one rank (exchange_local
 *     handles nparts == 1, parafaft_c2c.hpp:581-584) and fail if called.
 * Handles are small integers / heap records, so several communicators can be
 * created and freed as ParaFaFT does.
 */
#ifndef B200_MPI_SHIM_H
#define B200_MPI_SHIM_H

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef struct B200MpiStatus {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

struct B200MpiType {
  std::size_t base;   // bytes of one base element
  int ndims;          // 0 for a base type
  int sizes[16], subsizes[16], starts[16];
  bool committed;
};
typedef B200MpiType *MPI_Datatype;

#define MPI_SUCCESS 0
#define MPI_ERR_ARG 12
#define MPI_ERR_OTHER 15
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_ORDER_C 56
#define MPI_STATUSES_IGNORE (static_cast<MPI_Status *>(nullptr))
#define MPI_STATUS_IGNORE (static_cast<MPI_Status *>(nullptr))
#define MPI_IN_PLACE (reinterpret_cast<void *>(static_cast<std::intptr_t>(-1)))
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_SUM 3
#define MPI_LOR 4

namespace b200_mpi {
inline B200MpiType *base_type(std::size_t bytes) {
  B200MpiType *t = new B200MpiType();
  t->base = bytes;
  t->ndims = 0;
  t->committed = true;
  return t;
}
inline MPI_Datatype t_int() { static MPI_Datatype t = base_type(sizeof(int)); return t; }
inline MPI_Datatype t_byte() { static MPI_Datatype t = base_type(1); return t; }
inline MPI_Datatype t_u64() { static MPI_Datatype t = base_type(8); return t; }
inline MPI_Datatype t_float() { static MPI_Datatype t = base_type(4); return t; }
inline MPI_Datatype t_double() { static MPI_Datatype t = base_type(8); return t; }
inline MPI_Datatype t_cfloat() { static MPI_Datatype t = base_type(8); return t; }
inline MPI_Datatype t_cdouble() { static MPI_Datatype t = base_type(16); return t; }
inline std::size_t extent(MPI_Datatype t) {
  if (t->ndims == 0)
    return t->base;
  std::size_t n = t->base;
  for (int i = 0; i < t->ndims; ++i)
    n *= static_cast<std::size_t>(t->sizes[i]);
  return n;
}
inline std::size_t packed(MPI_Datatype t) {
  if (t->ndims == 0)
    return t->base;
  std::size_t n = t->base;
  for (int i = 0; i < t->ndims; ++i)
    n *= static_cast<std::size_t>(t->subsizes[i]);
  return n;
}
inline int &next_comm() { static int c = 16; return c; }
inline int fail(const char *what) {
  std::fprintf(stderr, "single-rank MPI stand-in: %s is not available\n", what);
  return MPI_ERR_OTHER;
}
// Visit the byte offsets of every contiguous last-axis run of a subarray.
template <typename F> inline void for_each_run(MPI_Datatype t, F f) {
  const int nd = t->ndims;
  const std::size_t run = static_cast<std::size_t>(t->subsizes[nd - 1]) * t->base;
  std::vector<int> idx(nd, 0);
  std::size_t count = 1;
  for (int i = 0; i < nd - 1; ++i)
    count *= static_cast<std::size_t>(t->subsizes[i]);
  for (std::size_t c = 0; c < count; ++c) {
    std::size_t off = 0;
    for (int i = 0; i < nd; ++i) {
      const std::size_t pos = static_cast<std::size_t>(t->starts[i] + (i < nd - 1 ? idx[i] : 0));
      off = off * static_cast<std::size_t>(t->sizes[i]) + pos;
    }
    f(off * t->base, run);
    for (int i = nd - 2; i >= 0; --i) {
      if (++idx[i] < t->subsizes[i])
        break;
      idx[i] = 0;
    }
  }
}
} // namespace b200_mpi

#define MPI_INT (b200_mpi::t_int())
#define MPI_BYTE (b200_mpi::t_byte())
#define MPI_UINT64_T (b200_mpi::t_u64())
#define MPI_FLOAT (b200_mpi::t_float())
#define MPI_DOUBLE (b200_mpi::t_double())
#define MPI_C_FLOAT_COMPLEX (b200_mpi::t_cfloat())
#define MPI_C_DOUBLE_COMPLEX (b200_mpi::t_cdouble())

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Finalized(int *flag) { *flag = 0; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
inline int MPI_Comm_dup(MPI_Comm, MPI_Comm *out) { *out = b200_mpi::next_comm()++; return MPI_SUCCESS; }
inline int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm *out) {
  *out = b200_mpi::next_comm()++;
  return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Dims_create(int nnodes, int ndims, int dims[]) {
  if (nnodes != 1)
    return b200_mpi::fail("MPI_Dims_create with more than one rank");
  for (int i = 0; i < ndims; ++i)
    if (dims[i] == 0)
      dims[i] = 1;
  return MPI_SUCCESS;
}
inline int MPI_Cart_create(MPI_Comm, int ndims, const int dims[], const int[], int, MPI_Comm *out) {
  for (int i = 0; i < ndims; ++i)
    if (dims[i] != 1)
      return b200_mpi::fail("a Cartesian grid larger than one rank");
  *out = b200_mpi::next_comm()++;
  return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int coords[]) {
  for (int i = 0; i < maxdims; ++i)
    coords[i] = 0;
  return MPI_SUCCESS;
}
inline int MPI_Cart_sub(MPI_Comm, const int[], MPI_Comm *out) {
  *out = b200_mpi::next_comm()++;
  return MPI_SUCCESS;
}
inline int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                                    const int starts[], int order, MPI_Datatype old,
                                    MPI_Datatype *out) {
  if (ndims < 1 || ndims > 16 || order != MPI_ORDER_C || old->ndims != 0)
    return MPI_ERR_ARG;
  B200MpiType *t = new B200MpiType();
  t->base = old->base;
  t->ndims = ndims;
  for (int i = 0; i < ndims; ++i) {
    if (sizes[i] <= 0 || subsizes[i] <= 0 || starts[i] < 0 || starts[i] + subsizes[i] > sizes[i]) {
      delete t;
      return MPI_ERR_ARG;
    }
    t->sizes[i] = sizes[i];
    t->subsizes[i] = subsizes[i];
    t->starts[i] = starts[i];
  }
  t->committed = false;
  *out = t;
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *t) { (*t)->committed = true; return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *t) {
  if (*t && (*t)->ndims != 0)
    delete *t;
  *t = nullptr;
  return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE)
    std::memmove(r, s, static_cast<std::size_t>(count) * b200_mpi::extent(t));
  return MPI_SUCCESS;
}
inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE)
    std::memmove(r, s, static_cast<std::size_t>(sc) * b200_mpi::extent(st));
  return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE)
    std::memmove(r, s, static_cast<std::size_t>(sc) * b200_mpi::extent(st));
  return MPI_SUCCESS;
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
// One-rank Alltoallw: copy the send subarray into the receive subarray.
inline int MPI_Alltoallw(const void *s, const int sc[], const int sd[], const MPI_Datatype st[],
                         void *r, const int rc[], const int rd[], const MPI_Datatype rt[], MPI_Comm) {
  if (sc[0] == 0)
    return MPI_SUCCESS;
  MPI_Datatype a = st[0], b = rt[0];
  if (b200_mpi::packed(a) != b200_mpi::packed(b) || sc[0] != 1 || rc[0] != 1)
    return MPI_ERR_ARG;
  std::vector<unsigned char> tmp(b200_mpi::packed(a));
  std::size_t pos = 0;
  const unsigned char *src = static_cast<const unsigned char *>(s) + sd[0];
  unsigned char *dst = static_cast<unsigned char *>(r) + rd[0];
  if (a->ndims == 0) {
    std::memcpy(tmp.data(), src, a->base);
  } else {
    b200_mpi::for_each_run(a, [&](std::size_t off, std::size_t n) {
      std::memcpy(tmp.data() + pos, src + off, n);
      pos += n;
    });
  }
  pos = 0;
  if (b->ndims == 0) {
    std::memcpy(dst, tmp.data(), b->base);
  } else {
    b200_mpi::for_each_run(b, [&](std::size_t off, std::size_t n) {
      std::memcpy(dst + off, tmp.data() + pos, n);
      pos += n;
    });
  }
  return MPI_SUCCESS;
}
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  return b200_mpi::fail("MPI_Isend");
}
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  return b200_mpi::fail("MPI_Irecv");
}
inline int MPI_Waitall(int, MPI_Request[], MPI_Status *) { return MPI_SUCCESS; }

#endif // B200_MPI_SHIM_H
