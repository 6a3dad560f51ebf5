/*
 * Single-rank stand-in for the MPI interface used by the reference's host
 * integrator headers (env.hpp, mpi_util.hpp, config.hpp, grid.hpp,
 * mhd_halo_exchange.hpp, mhd_integrator_host.hpp).  It lets the reference's
 * own arithmetic be compiled as the CPU checker in oracle/_ref/.  TEST
 * INFRASTRUCTURE ONLY.
 *
 * Semantics with one rank:
 *   - MPI_Cart_shift returns the rank itself on a periodic axis and
 *     MPI_PROC_NULL otherwise, so the halo exchanger's periodic faces become
 *     self-messages;
 *   - MPI_Isend copies the payload into a pending-message list keyed by tag;
 *     MPI_Irecv records the destination; MPI_Waitall delivers by tag;
 *   - reductions, broadcasts and gathers copy the local value.
 * None of these calls carries arithmetic.
 */
#ifndef MISO_REF_SHIM_MPI_H
#define MISO_REF_SHIM_MPI_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef struct { int dummy; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF_CART 2
#define MPI_PROC_NULL (-2)
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_MAX_ERROR_STRING 64
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 8

#define MPI_MIN 1
#define MPI_MAX 2

namespace miso_ref_shim {
struct Pending {
  int tag;
  std::vector<char> bytes;
};
struct Recv {
  int tag;
  void *buf;
  size_t bytes;
};
inline std::vector<Pending> &sends() {
  static std::vector<Pending> v;
  return v;
}
inline std::vector<Recv> &recvs() {
  static std::vector<Recv> v;
  return v;
}
inline int &initialized() {
  static int v = 0;
  return v;
}
inline int *periods() {
  static int p[3] = {0, 0, 0};
  return p;
}
inline size_t type_size(MPI_Datatype t) {
  switch (t) {
  case MPI_CHAR: return 1;
  case MPI_INT: return sizeof(int);
  case MPI_FLOAT: return sizeof(float);
  case MPI_DOUBLE: return sizeof(double);
  }
  return 1;
}
} // namespace miso_ref_shim

inline int MPI_Initialized(int *flag) { *flag = miso_ref_shim::initialized(); return 0; }
inline int MPI_Init(int *, char ***) { miso_ref_shim::initialized() = 1; return 0; }
inline int MPI_Finalized(int *flag) { *flag = 0; return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm *out) {
  *out = MPI_COMM_WORLD;
  return 0;
}
inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return 0; }
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
inline int MPI_Error_string(int, char *s, int *len) {
  std::snprintf(s, MPI_MAX_ERROR_STRING, "shim error");
  *len = (int)std::strlen(s);
  return 0;
}
inline int MPI_Cart_create(MPI_Comm, int ndims, const int *dims, const int *periods,
                           int, MPI_Comm *cart) {
  for (int d = 0; d < ndims && d < 3; ++d) {
    if (dims[d] != 1) {
      std::fprintf(stderr, "single-rank MPI stand-in: procs per axis must be 1\n");
      std::exit(2);
    }
    miso_ref_shim::periods()[d] = periods[d];
  }
  *cart = MPI_COMM_SELF_CART;
  return 0;
}
inline int MPI_Cart_coords(MPI_Comm, int, int ndims, int *coords) {
  for (int d = 0; d < ndims; ++d) coords[d] = 0;
  return 0;
}
inline int MPI_Cart_shift(MPI_Comm, int dir, int, int *src, int *dst) {
  const int self = miso_ref_shim::periods()[dir] ? 0 : MPI_PROC_NULL;
  *src = self;
  *dst = self;
  return 0;
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype,
                      int, MPI_Comm) {
  std::memcpy(r, s, n * miso_ref_shim::type_size(t));
  return 0;
}
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  std::memcpy(r, s, n * miso_ref_shim::type_size(t));
  return 0;
}
inline int MPI_Isend(const void *buf, int n, MPI_Datatype t, int, int tag, MPI_Comm,
                     MPI_Request *req) {
  miso_ref_shim::Pending p;
  p.tag = tag;
  const size_t b = (size_t)n * miso_ref_shim::type_size(t);
  p.bytes.resize(b);
  std::memcpy(p.bytes.data(), buf, b);
  miso_ref_shim::sends().push_back(std::move(p));
  *req = 0;
  return 0;
}
inline int MPI_Irecv(void *buf, int n, MPI_Datatype t, int, int tag, MPI_Comm,
                     MPI_Request *req) {
  miso_ref_shim::recvs().push_back({tag, buf, (size_t)n * miso_ref_shim::type_size(t)});
  *req = 0;
  return 0;
}
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) {
  auto &S = miso_ref_shim::sends();
  auto &R = miso_ref_shim::recvs();
  for (auto &r : R) {
    for (size_t s = 0; s < S.size(); ++s) {
      if (S[s].tag == r.tag) {
        std::memcpy(r.buf, S[s].bytes.data(), r.bytes);
        S.erase(S.begin() + (long)s);
        break;
      }
    }
  }
  R.clear();
  return 0;
}

#endif
