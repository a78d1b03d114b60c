// Single-process implementation of the MPI subset declared in mpi.h (test
// infrastructure for building the reference solver as a one-rank checker).
#include "mpi.h"

#include <fcntl.h>
#include <sys/time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

namespace {

struct TypeDesc {
  bool used = false;
  long long size = 0;    // packed bytes
  long long extent = 0;  // bytes spanned in memory
  // flattened map: (memory offset, length) blocks, in packing order
  std::vector<std::pair<long long, long long>> blocks;
};

std::mutex g_mu;
std::vector<TypeDesc> g_types;

void init_types() {
  if (!g_types.empty()) return;
  g_types.resize(12);
  const long long sz[12] = {0, 1, 1, 4, 4, 8, 4, 4, 8, 8, 8, 4};
  for (int t = 1; t < 12; ++t) {
    g_types[t].used = true;
    g_types[t].size = g_types[t].extent = sz[t];
    g_types[t].blocks = {{0, sz[t]}};
  }
}

const TypeDesc &type_of(MPI_Datatype t) {
  std::lock_guard<std::mutex> lock(g_mu);
  init_types();
  if (t <= 0 || t >= (int)g_types.size() || !g_types[t].used) {
    std::fprintf(stderr, "mpi shim: unknown datatype %d\n", t);
    std::abort();
  }
  return g_types[t];
}

MPI_Datatype new_type(TypeDesc d) {
  std::lock_guard<std::mutex> lock(g_mu);
  init_types();
  // merge adjacent blocks
  std::vector<std::pair<long long, long long>> merged;
  for (auto &b : d.blocks) {
    if (!merged.empty() && merged.back().first + merged.back().second == b.first)
      merged.back().second += b.second;
    else
      merged.push_back(b);
  }
  d.blocks.swap(merged);
  d.used = true;
  for (size_t t = 12; t < g_types.size(); ++t)
    if (!g_types[t].used) {
      g_types[t] = std::move(d);
      return (MPI_Datatype)t;
    }
  g_types.push_back(std::move(d));
  return (MPI_Datatype)(g_types.size() - 1);
}

long long packed_bytes(int count, MPI_Datatype t) { return (long long)count * type_of(t).size; }

// memory (typed) -> packed bytes
void pack(const void *buf, int count, MPI_Datatype t, std::vector<char> &out) {
  const TypeDesc &d = type_of(t);
  out.resize((size_t)(count * d.size));
  const char *src = static_cast<const char *>(buf);
  size_t o = 0;
  for (int c = 0; c < count; ++c)
    for (auto &b : d.blocks) {
      std::memcpy(out.data() + o, src + c * d.extent + b.first, (size_t)b.second);
      o += (size_t)b.second;
    }
}

// packed bytes -> memory (typed)
void unpack(const std::vector<char> &in, void *buf, int count, MPI_Datatype t) {
  const TypeDesc &d = type_of(t);
  char *dst = static_cast<char *>(buf);
  size_t o = 0;
  for (int c = 0; c < count; ++c)
    for (auto &b : d.blocks) {
      if (o + (size_t)b.second > in.size()) return;
      std::memcpy(dst + c * d.extent + b.first, in.data() + o, (size_t)b.second);
      o += (size_t)b.second;
    }
}

void copy_typed(const void *send, int scount, MPI_Datatype stype, void *recv, MPI_Datatype rtype, int rcount) {
  if (send == MPI_IN_PLACE || send == recv) return;
  std::vector<char> tmp;
  pack(send, scount, stype, tmp);
  if ((long long)tmp.size() > packed_bytes(rcount, rtype)) tmp.resize((size_t)packed_bytes(rcount, rtype));
  unpack(tmp, recv, rcount, rtype);
}

[[noreturn]] void unsupported(const char *what) {
  std::fprintf(stderr, "mpi shim: %s is not available in a single-process run\n", what);
  std::abort();
}

}  // namespace

struct mpi_shim_file {
  int fd;
  long long pos;  // individual file pointer, bytes
};

extern "C" {

int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) {
  std::fflush(stdout);
  std::fprintf(stderr, "MPI_Abort(%d)\n", code);
  std::exit(code ? code : 1);
}
int MPI_Comm_rank(MPI_Comm, int *rank) {
  *rank = 0;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm, int *size) {
  *size = 1;
  return MPI_SUCCESS;
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
double MPI_Wtime(void) {
  timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  copy_typed(s, n, t, r, t, n);
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy_typed(s, n, t, r, t, n);
  return MPI_SUCCESS;
}
int MPI_Gather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int, MPI_Comm) {
  copy_typed(s, sc, st, r, rt, rc);
  return MPI_SUCCESS;
}
int MPI_Gatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rcs, const int *displs, MPI_Datatype rt,
                int, MPI_Comm) {
  copy_typed(s, sc, st, static_cast<char *>(r) + (long long)displs[0] * type_of(rt).extent, rt, rcs[0]);
  return MPI_SUCCESS;
}
int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, MPI_Comm) {
  copy_typed(s, sc, st, r, rt, rc);
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void *s, int sc, MPI_Datatype st, void *r, const int *rcs, const int *displs,
                   MPI_Datatype rt, MPI_Comm) {
  copy_typed(s, sc, st, static_cast<char *>(r) + (long long)displs[0] * type_of(rt).extent, rt, rcs[0]);
  return MPI_SUCCESS;
}
int MPI_Scatter(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, int, MPI_Comm) {
  if (r == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_typed(s, sc, st, r, rt, rc);
  return MPI_SUCCESS;
}
int MPI_Scatterv(const void *s, const int *scs, const int *displs, MPI_Datatype st, void *r, int rc, MPI_Datatype rt,
                 int, MPI_Comm) {
  if (r == MPI_IN_PLACE) return MPI_SUCCESS;
  copy_typed(static_cast<const char *>(s) + (long long)displs[0] * type_of(st).extent, scs[0], st, r, rt, rc);
  return MPI_SUCCESS;
}

int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { unsupported("MPI_Isend"); }
int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { unsupported("MPI_Irecv"); }
int MPI_Waitall(int count, MPI_Request *, MPI_Status *) {
  if (count > 0) unsupported("MPI_Waitall");
  return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *out) {
  const TypeDesc o = type_of(old);
  TypeDesc d;
  d.size = count * o.size;
  d.extent = count * o.extent;
  for (int c = 0; c < count; ++c)
    for (auto &b : o.blocks) d.blocks.push_back({c * o.extent + b.first, b.second});
  *out = new_type(std::move(d));
  return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[], int order,
                             MPI_Datatype old, MPI_Datatype *out) {
  const TypeDesc o = type_of(old);
  // dimension 0 is the fastest for FORTRAN order, the slowest for C order
  std::vector<long long> sz(ndims), sub(ndims), st(ndims);
  for (int d = 0; d < ndims; ++d) {
    const int s = order == MPI_ORDER_FORTRAN ? d : ndims - 1 - d;
    sz[d] = sizes[s];
    sub[d] = subsizes[s];
    st[d] = starts[s];
  }
  TypeDesc d;
  d.extent = o.extent;
  for (int k = 0; k < ndims; ++k) d.extent *= sz[k];
  long long n_sub = 1;
  for (int k = 0; k < ndims; ++k) n_sub *= sub[k];
  d.size = n_sub * o.size;
  std::vector<long long> idx(ndims, 0);
  for (long long e = 0; e < n_sub; ++e) {
    long long off = 0, stride = 1;
    for (int k = 0; k < ndims; ++k) {
      off += (st[k] + idx[k]) * stride;
      stride *= sz[k];
    }
    for (auto &b : o.blocks) d.blocks.push_back({off * o.extent + b.first, b.second});
    for (int k = 0; k < ndims; ++k) {
      if (++idx[k] < sub[k]) break;
      idx[k] = 0;
    }
  }
  *out = new_type(std::move(d));
  return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *type) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (*type >= 12 && *type < (int)g_types.size()) g_types[*type] = TypeDesc{};
  *type = MPI_DATATYPE_NULL;
  return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm, const char *name, int amode, MPI_Info, MPI_File *fh) {
  int flags = 0;
  if (amode & MPI_MODE_RDONLY) flags = O_RDONLY;
  else if (amode & MPI_MODE_WRONLY) flags = O_WRONLY;
  else flags = O_RDWR;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
  if (amode & MPI_MODE_EXCL) flags |= O_EXCL;
  const int fd = open(name, flags, 0644);
  if (fd < 0) {
    *fh = nullptr;
    return 1;
  }
  *fh = new mpi_shim_file{fd, 0};
  if (amode & MPI_MODE_APPEND) (*fh)->pos = lseek(fd, 0, SEEK_END);
  return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh) {
  if (*fh) {
    close((*fh)->fd);
    delete *fh;
  }
  *fh = nullptr;
  return MPI_SUCCESS;
}

int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type, MPI_Status *status) {
  if (!fh) unsupported("MPI_File_read_at on a file that failed to open");
  std::vector<char> tmp((size_t)packed_bytes(count, type));
  long long got = 0;
  while (got < (long long)tmp.size()) {
    const ssize_t r = pread(fh->fd, tmp.data() + got, tmp.size() - got, offset + got);
    if (r <= 0) break;
    got += r;
  }
  tmp.resize((size_t)got);
  unpack(tmp, buf, count, type);
  if (status) status->count_bytes = got;
  return MPI_SUCCESS;
}

int MPI_File_write_at(MPI_File fh, MPI_Offset offset, const void *buf, int count, MPI_Datatype type,
                      MPI_Status *status) {
  if (!fh) unsupported("MPI_File_write_at on a file that failed to open");
  std::vector<char> tmp;
  pack(buf, count, type, tmp);
  long long put = 0;
  while (put < (long long)tmp.size()) {
    const ssize_t w = pwrite(fh->fd, tmp.data() + put, tmp.size() - put, offset + put);
    if (w <= 0) break;
    put += w;
  }
  if (status) status->count_bytes = put;
  return MPI_SUCCESS;
}

int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype type, MPI_Status *status) {
  MPI_Status s{};
  MPI_File_read_at(fh, fh->pos, buf, count, type, &s);
  fh->pos += s.count_bytes;
  if (status) *status = s;
  return MPI_SUCCESS;
}

int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype type, MPI_Status *status) {
  MPI_Status s{};
  MPI_File_write_at(fh, fh->pos, buf, count, type, &s);
  fh->pos += s.count_bytes;
  if (status) *status = s;
  return MPI_SUCCESS;
}

}  // extern "C"
