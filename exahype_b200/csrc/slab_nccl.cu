// Slab decomposition transport over NCCL, inside the library: the
// reference's distributed step (ADERDGSolver::sendDataToNeighbour,
// exahype/solvers/ADERDGSolver.cpp:3379, ships each rank-boundary face's
// lQhbnd / lFhbnd; mergeWithNeighbourData, :3451, solves the Riemann problem
// with the received face; the time step is a MIN over ranks,
// exahype/mappings/TimeStepSizeComputation.cpp:83-109) as a sequence of
// stream-ordered operations on the slab grid's own stream:
//
//   predict (packs the two boundary face layers)
//   ncclSend send_hi -> up, send_lo -> down; ncclRecv recv_lo <- down,
//     recv_hi <- up (one NCCL group)
//   correct (faces across the slab ends read recv_lo / recv_hi)
//   ncclAllReduce MIN of the next-dt slot (the bit pattern of a positive
//     double: the integer MIN is the double MIN)
//   commit
//
// The host enqueues a whole batch of steps and then waits for it with a
// deadline; if a peer stops answering, the communicator is aborted (which
// ends the waiting NCCL kernels) and the call returns EXA_ETIMEDOUT, so no
// rank waits for ever.  NCCL is opened at run time (libnccl.so.2): the
// library loads without it, and these entry points report its absence.
// With one rank the face layers are copied on the stream (a periodic slab
// is its own neighbour) and the reduction is NCCL's one-rank all-reduce.
#include <dlfcn.h>

#include <chrono>
#include <mutex>
#include <string>
#include <thread>

#include <nccl.h>  // types only: the functions are resolved at run time

#include "exa_device.cuh"

using namespace exa;

namespace {

struct NcclApi {
  bool ok = false;
  std::string err;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

NcclApi g_nccl;
std::once_flag g_nccl_once;

template <typename F>
bool resolve(void* h, const char* name, F& fn) {
  fn = reinterpret_cast<F>(dlsym(h, name));
  return fn != nullptr;
}

void load_nccl() {
  void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    g_nccl.err = std::string("NCCL not found: ") + dlerror();
    return;
  }
  NcclApi& a = g_nccl;
  if (!(resolve(h, "ncclGetUniqueId", a.GetUniqueId) && resolve(h, "ncclCommInitRank", a.CommInitRank) &&
        resolve(h, "ncclCommDestroy", a.CommDestroy) && resolve(h, "ncclCommAbort", a.CommAbort) &&
        resolve(h, "ncclSend", a.Send) && resolve(h, "ncclRecv", a.Recv) &&
        resolve(h, "ncclAllReduce", a.AllReduce) && resolve(h, "ncclGroupStart", a.GroupStart) &&
        resolve(h, "ncclGroupEnd", a.GroupEnd) && resolve(h, "ncclGetErrorString", a.GetErrorString))) {
    a.err = "NCCL library lacks a required symbol";
    return;
  }
  a.ok = true;
}

exa_status_t need_nccl() {
  std::call_once(g_nccl_once, load_nccl);
  if (!g_nccl.ok) return set_error(EXA_ECUDA, g_nccl.err.c_str());
  return EXA_OK;
}

exa_status_t nccl_status(ncclResult_t r, const char* where) {
  if (r == ncclSuccess) return EXA_OK;
  std::string m = std::string(where) + ": " + (g_nccl.GetErrorString ? g_nccl.GetErrorString(r) : "NCCL error");
  return set_error(EXA_ECUDA, m.c_str());
}

}  // namespace

struct exa_slab_comm {
  ncclComm_t comm = nullptr;
  int rank = 0, nranks = 1;
  int device = 0;
  bool aborted = false;
};

namespace {

// the exchange of one step on the grid's stream
exa_status_t exchange(exa_aderdg_grid* g, exa_slab_comm* c, cudaStream_t st) {
  double *s_lo, *s_hi, *r_lo, *r_hi;
  size_t n = 0;
  if (exa_status_t s = exa_aderdg_grid_halo_buffers(g, &s_lo, &s_hi, &r_lo, &r_hi, &n)) return s;
  if (c->nranks == 1) {
    cudaError_t e = cudaMemcpyAsync(r_lo, s_hi, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r_hi, s_lo, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    return cuda_status(e, "slab self-exchange");
  }
  const int up = (c->rank + 1) % c->nranks, down = (c->rank + c->nranks - 1) % c->nranks;
  // per peer, NCCL matches sends and receives in issue order: the upward
  // message (send_hi) is the receiver's recv_lo, the downward one its recv_hi
  if (exa_status_t s = nccl_status(g_nccl.GroupStart(), "ncclGroupStart")) return s;
  ncclResult_t r = g_nccl.Send(s_hi, n, ncclFloat64, up, c->comm, st);
  if (r == ncclSuccess) r = g_nccl.Send(s_lo, n, ncclFloat64, down, c->comm, st);
  if (r == ncclSuccess) r = g_nccl.Recv(r_lo, n, ncclFloat64, down, c->comm, st);
  if (r == ncclSuccess) r = g_nccl.Recv(r_hi, n, ncclFloat64, up, c->comm, st);
  const ncclResult_t r2 = g_nccl.GroupEnd();
  if (r != ncclSuccess) return nccl_status(r, "slab exchange");
  return nccl_status(r2, "ncclGroupEnd");
}

exa_status_t reduce_dt(exa_aderdg_grid* g, exa_slab_comm* c, cudaStream_t st) {
  uint64_t* slot = nullptr;
  if (exa_status_t s = exa_aderdg_grid_dt_slot(g, &slot)) return s;
  return nccl_status(g_nccl.AllReduce(slot, slot, 1, ncclUint64, ncclMin, c->comm, st), "dt MIN all-reduce");
}

// waits for the grid's stream; past the deadline the communicator is
// aborted, which ends NCCL kernels waiting for a peer
exa_status_t wait_or_abort(exa_slab_comm* c, cudaStream_t st, double timeout_s) {
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ev, st);
  if (e != cudaSuccess) return cuda_status(e, "slab step event");
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    e = cudaEventQuery(ev);
    if (e != cudaErrorNotReady) break;
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el > timeout_s) {
      if (c->nranks > 1 && !c->aborted) {
        g_nccl.CommAbort(c->comm);
        c->aborted = true;
        c->comm = nullptr;
      }
      cudaEventDestroy(ev);
      return set_error(EXA_ETIMEDOUT, "slab step: a peer did not answer within the deadline; "
                                      "communicator aborted");
    }
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
  cudaEventDestroy(ev);
  return cuda_status(e, "slab step");
}

}  // namespace

extern "C" {

exa_status_t exa_nccl_unique_id(void* id) {
  if (!id) return set_error(EXA_EINVAL, "NULL id");
  if (exa_status_t s = need_nccl()) return s;
  ncclUniqueId u;
  if (exa_status_t s = nccl_status(g_nccl.GetUniqueId(&u), "ncclGetUniqueId")) return s;
  memcpy(id, &u, sizeof(u));
  return EXA_OK;
}

exa_status_t exa_slab_comm_create(const void* id, int nranks, int rank, exa_slab_comm** out) {
  if (!id || !out) return set_error(EXA_EINVAL, "NULL argument");
  if (nranks < 1 || rank < 0 || rank >= nranks) return set_error(EXA_EINVAL, "bad rank / nranks");
  if (exa_status_t s = need_nccl()) return s;
  exa_slab_comm* c = new (std::nothrow) exa_slab_comm;
  if (!c) return set_error(EXA_ENOMEM, "host allocation");
  c->rank = rank;
  c->nranks = nranks;
  cudaGetDevice(&c->device);
  ncclUniqueId u;
  memcpy(&u, id, sizeof(u));
  if (exa_status_t s = nccl_status(g_nccl.CommInitRank(&c->comm, nranks, u, rank), "ncclCommInitRank")) {
    delete c;
    return s;
  }
  *out = c;
  return EXA_OK;
}

exa_status_t exa_slab_comm_destroy(exa_slab_comm* c) {
  if (!c) return EXA_OK;
  exa_status_t s = EXA_OK;
  if (c->comm && !c->aborted) s = nccl_status(g_nccl.CommDestroy(c->comm), "ncclCommDestroy");
  delete c;
  return s;
}

exa_status_t exa_aderdg_grid_slab_prime(exa_aderdg_grid* g, exa_slab_comm* c, double timeout_s) {
  if (!g || !c) return set_error(EXA_EINVAL, "NULL argument");
  if (c->aborted) return set_error(EXA_EINVAL, "communicator was aborted");
  void* sv = nullptr;
  if (exa_status_t s = exa_aderdg_grid_stream(g, &sv)) return s;
  cudaStream_t st = (cudaStream_t)sv;
  if (grid_fixed_dt(g)) return exa_aderdg_grid_phase(g, EXA_PHASE_PRIME_COMMIT);
  if (exa_status_t s = exa_aderdg_grid_phase(g, EXA_PHASE_PRIME_LOCAL)) return s;
  if (exa_status_t s = reduce_dt(g, c, st)) return s;
  if (exa_status_t s = exa_aderdg_grid_phase(g, EXA_PHASE_PRIME_COMMIT)) return s;
  return wait_or_abort(c, st, timeout_s > 0 ? timeout_s : 60.0);
}

exa_status_t exa_aderdg_grid_slab_step(exa_aderdg_grid* g, exa_slab_comm* c, int nsteps, double timeout_s) {
  if (!g || !c) return set_error(EXA_EINVAL, "NULL argument");
  if (nsteps < 0) return set_error(EXA_EINVAL, "nsteps must be >= 0");
  if (c->aborted) return set_error(EXA_EINVAL, "communicator was aborted");
  void* sv = nullptr;
  if (exa_status_t s = exa_aderdg_grid_stream(g, &sv)) return s;
  cudaStream_t st = (cudaStream_t)sv;
  const bool fixed = grid_fixed_dt(g);
  for (int k = 0; k < nsteps; k++) {
    if (exa_status_t s = exa_aderdg_grid_phase(g, EXA_PHASE_PREDICT)) return s;
    if (exa_status_t s = exchange(g, c, st)) return s;
    if (exa_status_t s = exa_aderdg_grid_phase(g, EXA_PHASE_CORRECT)) return s;
    if (!fixed)
      if (exa_status_t s = reduce_dt(g, c, st)) return s;
    if (exa_status_t s = exa_aderdg_grid_phase(g, EXA_PHASE_COMMIT)) return s;
  }
  return wait_or_abort(c, st, (timeout_s > 0 ? timeout_s : 60.0) * (nsteps > 0 ? nsteps : 1));
}

}  // extern "C"
