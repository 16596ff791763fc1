// The halo exchange of one rank of a partitioned run, on its handle's device
// state (include/wasl_b200.h, wasl_halo_*): pack and unpack kernels over
// per-peer column lists, device buffers a caller's own transport can move,
// and an NCCL transport (send/receive with every peer in one group, and the
// CFL parts' all-reduce).
//
// The reference's halo schedule lists, per peer and in ascending order, the
// owned elements a peer imports and the ghosts imported from it
// (cpp/include/wasl/communication/halo_schedule.hpp:17-42); its MPI transport
// posts one send and one receive per peer
// (cpp/src/communication/mpi_halo_exchange.cpp).  Here the rows of all of a
// peer's columns travel as one contiguous [rows][columns] buffer.
//
// NCCL is bound at first use with dlopen (the copy already in the process,
// such as the one PyTorch loads, else the system's libnccl.so.2), so the
// library itself does not depend on it.
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "solver.hpp"

namespace wasl_b200 {
namespace {

// dst[r][i] = state[r][columns[i]] for rows x count.
__global__ void halo_pack(const double *__restrict__ state, std::int64_t ne, int rows,
                          const std::int32_t *__restrict__ columns, std::int64_t count,
                          double *__restrict__ dst) {
  const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count)
    return;
  const std::int64_t c = columns[i];
  for (int r = 0; r < rows; ++r)
    dst[r * count + i] = state[r * ne + c];
}

// state[r][columns[i]] = src[r][i].
__global__ void halo_unpack(double *__restrict__ state, std::int64_t ne, int rows,
                            const std::int32_t *__restrict__ columns, std::int64_t count,
                            const double *__restrict__ src) {
  const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count)
    return;
  const std::int64_t c = columns[i];
  for (int r = 0; r < rows; ++r)
    state[r * ne + c] = src[r * count + i];
}

// The NCCL entry points the transport uses, resolved from the loaded library.
struct Nccl {
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) comm_init_rank = nullptr;
  decltype(&ncclCommDestroy) comm_destroy = nullptr;
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclGroupStart) group_start = nullptr;
  decltype(&ncclGroupEnd) group_end = nullptr;
  decltype(&ncclAllReduce) all_reduce = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
  std::string failure;
};

const Nccl &nccl() {
  static Nccl api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!lib)
      lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) {
      api.failure = std::string("NCCL: libnccl.so.2 not found (") + dlerror() + ")";
      return;
    }
    auto bind = [&](auto &fn, const char *name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(lib, name));
      if (!fn && api.failure.empty())
        api.failure = std::string("NCCL: symbol ") + name + " missing";
    };
    bind(api.get_unique_id, "ncclGetUniqueId");
    bind(api.comm_init_rank, "ncclCommInitRank");
    bind(api.comm_destroy, "ncclCommDestroy");
    bind(api.send, "ncclSend");
    bind(api.recv, "ncclRecv");
    bind(api.group_start, "ncclGroupStart");
    bind(api.group_end, "ncclGroupEnd");
    bind(api.all_reduce, "ncclAllReduce");
    bind(api.error_string, "ncclGetErrorString");
  });
  if (!api.failure.empty())
    throw SolverError(WASL_ERR_RUNTIME, api.failure);
  return api;
}

void nccl_check(ncclResult_t rc, const char *what) {
  if (rc != ncclSuccess)
    throw SolverError(WASL_ERR_RUNTIME,
                      std::string(what) + ": " + nccl().error_string(rc));
}

unsigned blocks_of(std::int64_t n) { return static_cast<unsigned>((n + 255) / 256); }

} // namespace

struct HaloPeer {
  int rank = 0;
  std::int64_t sends = 0, recvs = 0;
  DeviceArray<std::int32_t> send_columns, recv_columns;
  DeviceArray<double> send_buffer, recv_buffer;
};

} // namespace wasl_b200

struct wasl_halo {
  wasl_gpu *handle = nullptr;
  wasl_b200::Solver *solver = nullptr;
  int rows = 0;
  std::vector<wasl_b200::HaloPeer> peers;
  std::string error;
};

namespace wasl_b200 {
Solver *solver_of(wasl_gpu *handle);
void set_handle_error(wasl_gpu *handle, const std::string &message);
} // namespace wasl_b200

namespace {

template <typename F> int halo_guarded(wasl_halo *h, F &&body) {
  if (!h)
    return WASL_ERR_ARGUMENT;
  try {
    body();
    h->error.clear();
    return WASL_OK;
  } catch (const wasl_b200::SolverError &e) {
    h->error = e.what();
    return e.status;
  } catch (const std::exception &e) {
    h->error = e.what();
    return WASL_ERR_RUNTIME;
  }
}

void copy_text(const std::string &text, char *out, size_t length) {
  if (out && length) {
    std::strncpy(out, text.c_str(), length - 1);
    out[length - 1] = '\0';
  }
}

} // namespace

extern "C" {

int wasl_halo_create(wasl_gpu *handle, int peers, const int32_t *peer_ranks,
                     const int64_t *send_counts, const int64_t *send_elements,
                     const int64_t *recv_counts, const int64_t *recv_elements, wasl_halo **halo,
                     char *error, size_t error_length) {
  using namespace wasl_b200;
  if (!halo)
    return WASL_ERR_ARGUMENT;
  *halo = nullptr;
  auto h = std::make_unique<wasl_halo>();
  const int rc = halo_guarded(h.get(), [&] {
    Solver *s = solver_of(handle);
    if (!s)
      throw SolverError(WASL_ERR_ARGUMENT, "halo: null handle");
    if (peers < 0 || (peers > 0 && (!peer_ranks || !send_counts || !recv_counts)))
      throw SolverError(WASL_ERR_ARGUMENT, "halo: invalid peer lists");
    h->handle = handle;
    h->solver = s;
    h->rows = s->variables() * s->modes();
    const std::int64_t ne = s->elements();
    std::vector<std::int64_t> order(ne);
    s->element_order(order.data());
    std::vector<std::int32_t> column(ne); // caller's element -> storage column
    for (std::int64_t i = 0; i < ne; ++i)
      column[order[i]] = static_cast<std::int32_t>(i);
    auto columns = [&](const int64_t *elements, std::int64_t count) {
      std::vector<std::int32_t> out(count);
      for (std::int64_t i = 0; i < count; ++i) {
        if (elements[i] < 0 || elements[i] >= ne)
          throw SolverError(WASL_ERR_ARGUMENT, "halo: element index outside the handle's mesh");
        out[i] = column[elements[i]];
      }
      return out;
    };
    std::int64_t sent = 0, received = 0;
    h->peers.resize(peers);
    for (int k = 0; k < peers; ++k) {
      HaloPeer &p = h->peers[k];
      p.rank = peer_ranks[k];
      p.sends = send_counts[k];
      p.recvs = recv_counts[k];
      if (p.sends < 0 || p.recvs < 0 || (p.sends && !send_elements) ||
          (p.recvs && !recv_elements))
        throw SolverError(WASL_ERR_ARGUMENT, "halo: invalid peer lists");
      p.send_columns.upload(columns(send_elements + sent, p.sends), s->stream());
      p.recv_columns.upload(columns(recv_elements + received, p.recvs), s->stream());
      p.send_buffer.resize(static_cast<std::size_t>(h->rows) * p.sends);
      p.recv_buffer.resize(static_cast<std::size_t>(h->rows) * p.recvs);
      sent += p.sends;
      received += p.recvs;
    }
    cuda_check(cudaStreamSynchronize(s->stream()), "halo setup");
  });
  if (rc != WASL_OK) {
    copy_text(h->error, error, error_length);
    return rc;
  }
  *halo = h.release();
  return WASL_OK;
}

void wasl_halo_destroy(wasl_halo *halo) { delete halo; }

const char *wasl_halo_last_error(const wasl_halo *halo) {
  return halo ? halo->error.c_str() : "null halo";
}

int wasl_halo_pack(wasl_halo *halo) {
  return halo_guarded(halo, [&] {
    wasl_b200::Solver *s = halo->solver;
    for (auto &p : halo->peers)
      if (p.sends)
        wasl_b200::halo_pack<<<wasl_b200::blocks_of(p.sends), 256, 0, s->stream()>>>(
            s->state_device(), s->elements(), halo->rows, p.send_columns.get(), p.sends,
            p.send_buffer.get());
    wasl_b200::cuda_check(cudaGetLastError(), "halo pack");
  });
}

int wasl_halo_unpack(wasl_halo *halo) {
  return halo_guarded(halo, [&] {
    wasl_b200::Solver *s = halo->solver;
    for (auto &p : halo->peers)
      if (p.recvs)
        wasl_b200::halo_unpack<<<wasl_b200::blocks_of(p.recvs), 256, 0, s->stream()>>>(
            s->state_device(), s->elements(), halo->rows, p.recv_columns.get(), p.recvs,
            p.recv_buffer.get());
    wasl_b200::cuda_check(cudaGetLastError(), "halo unpack");
  });
}

int wasl_halo_buffers(wasl_halo *halo, int peer, double **send, double **recv,
                      int64_t *send_count, int64_t *recv_count, int64_t *rows) {
  return halo_guarded(halo, [&] {
    if (peer < 0 || peer >= static_cast<int>(halo->peers.size()))
      throw wasl_b200::SolverError(WASL_ERR_ARGUMENT, "halo: peer index out of range");
    const auto &p = halo->peers[peer];
    if (send)
      *send = p.send_buffer.get();
    if (recv)
      *recv = p.recv_buffer.get();
    if (send_count)
      *send_count = p.sends;
    if (recv_count)
      *recv_count = p.recvs;
    if (rows)
      *rows = halo->rows;
  });
}

int wasl_halo_exchange_nccl(wasl_halo *halo, void *comm) {
  const int packed = wasl_halo_pack(halo);
  if (packed != WASL_OK)
    return packed;
  const int moved = halo_guarded(halo, [&] {
    const wasl_b200::Nccl &api = wasl_b200::nccl();
    if (!comm && !halo->peers.empty())
      throw wasl_b200::SolverError(WASL_ERR_ARGUMENT, "halo: null NCCL communicator");
    const cudaStream_t stream = halo->solver->stream();
    auto c = static_cast<ncclComm_t>(comm);
    wasl_b200::nccl_check(api.group_start(), "ncclGroupStart");
    for (auto &p : halo->peers) {
      if (p.sends)
        wasl_b200::nccl_check(api.send(p.send_buffer.get(), halo->rows * p.sends, ncclFloat64,
                                       p.rank, c, stream),
                              "ncclSend");
      if (p.recvs)
        wasl_b200::nccl_check(api.recv(p.recv_buffer.get(), halo->rows * p.recvs, ncclFloat64,
                                       p.rank, c, stream),
                              "ncclRecv");
    }
    wasl_b200::nccl_check(api.group_end(), "ncclGroupEnd");
  });
  if (moved != WASL_OK)
    return moved;
  return wasl_halo_unpack(halo);
}

int wasl_gpu_stable_dt_nccl(wasl_gpu *handle, void *comm, double cfl, double *dt) {
  using namespace wasl_b200;
  Solver *s = solver_of(handle);
  if (!s || !dt || !comm)
    return WASL_ERR_ARGUMENT;
  wasl_halo scratch; // carries the error message
  scratch.handle = handle;
  const int rc = halo_guarded(&scratch, [&] {
    const Nccl &api = nccl();
    double speed = 0.0, length = 0.0;
    s->cfl_parts(speed, length);
    const double parts[2] = {speed, -length}; // max of both: largest speed, smallest length
    DeviceArray<double> d(2);
    cuda_check(cudaMemcpyAsync(d.get(), parts, sizeof parts, cudaMemcpyHostToDevice,
                               s->stream()),
               "cfl parts");
    nccl_check(api.all_reduce(d.get(), d.get(), 2, ncclFloat64, ncclMax,
                              static_cast<ncclComm_t>(comm), s->stream()),
               "ncclAllReduce");
    double reduced[2];
    cuda_check(cudaMemcpyAsync(reduced, d.get(), sizeof reduced, cudaMemcpyDeviceToHost,
                               s->stream()),
               "cfl parts");
    cuda_check(cudaStreamSynchronize(s->stream()), "cfl parts");
    *dt = s->dt_from_parts(cfl, reduced[0], -reduced[1]);
  });
  if (rc != WASL_OK)
    set_handle_error(handle, scratch.error);
  return rc;
}

int wasl_nccl_unique_id(uint8_t *id) {
  if (!id)
    return WASL_ERR_ARGUMENT;
  try {
    ncclUniqueId u;
    wasl_b200::nccl_check(wasl_b200::nccl().get_unique_id(&u), "ncclGetUniqueId");
    std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
    return WASL_OK;
  } catch (const wasl_b200::SolverError &e) {
    return e.status;
  }
}

int wasl_nccl_comm_create(int ranks, const uint8_t *id, int rank, int device, void **comm,
                          char *error, size_t error_length) {
  if (!id || !comm)
    return WASL_ERR_ARGUMENT;
  *comm = nullptr;
  try {
    wasl_b200::cuda_check(cudaSetDevice(device), "cudaSetDevice");
    ncclUniqueId u;
    std::memcpy(u.internal, id, NCCL_UNIQUE_ID_BYTES);
    ncclComm_t c = nullptr;
    wasl_b200::nccl_check(wasl_b200::nccl().comm_init_rank(&c, ranks, u, rank),
                          "ncclCommInitRank");
    *comm = c;
    return WASL_OK;
  } catch (const wasl_b200::SolverError &e) {
    copy_text(e.what(), error, error_length);
    return e.status;
  }
}

void wasl_nccl_comm_destroy(void *comm) {
  if (comm) {
    try {
      wasl_b200::nccl().comm_destroy(static_cast<ncclComm_t>(comm));
    } catch (const wasl_b200::SolverError &) {
    }
  }
}

} // extern "C"
