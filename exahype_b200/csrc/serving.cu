// Serving engine: continuous batching of solve requests on one GPU.
//
// Requests are 2D ADER-DG solves or 2D finite-volume (Godunov / MUSCL-
// Hancock) periodic patches with a step budget.  Admission is by device
// memory footprint out of one arena (the ensemble's): a request that does
// not fit is refused with EXA_EBUSY and the caller retries after others
// finish.  Admitted requests stay resident on the device until their result
// is collected.  Every tick advances every active request (ADER-DG requests
// by one step, FV requests by up to exa_server_set_fv_steps steps):
//   * all ADER-DG requests together in the ensemble's single persistent
//     launch (one launch regardless of how many requests are active);
//   * all FV requests of one scheme together in one batched patch launch on
//     a second stream (a device table of the live patches; each CTA finds
//     its patch from its tile index), so FV work overlaps the ADER-DG
//     launch and costs two launches per tick however many patches are
//     live.
// A request that arrives while others run joins at the next tick; its
// arithmetic is independent of its neighbours (per-request dt and state),
// so its result is the same alone or in any mix.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <thread>
#include <mutex>
#include <new>
#include <vector>

#include "exa_device.cuh"

using namespace exa;

namespace {
struct Req {
  uint64_t id = 0;
  exa_request_t r{};
  // ADER-DG
  int slot = -1;
  // FV
  exa_fv_desc_t fv{};
  double* luh = nullptr;
  double* luh_new = nullptr;
  unsigned long long* dt_slot = nullptr;  // scalars: [0] dt bits, [1] time, [2] next dt bits, [3] buffer
  int par = 0;                            // buffer holding the state: 0 luh, 1 luh_new
  size_t off = 0, bytes = 0;
  long long steps_left = 0;
  long long steps_done = 0;
  bool done = false;
  bool reported = false;  // listed for exa_server_completed once
  // eviction: the state and time-step scalars on the host, no device memory
  bool evicted = false;
  std::vector<double> saved;
  exa_solve_checkpoint_t ck{};         // ADER-DG
  unsigned long long fv_scal[4] = {};  // FV: dt bits, time, next dt bits, buffer
};

size_t fv_bytes(const exa_request_t* r) {
  const int g = r->fv_scheme == 0 ? 1 : 2;
  const size_t S = (size_t)r->fv_patch + 2 * g;
  const size_t state = ((S * S * kV * 8) + 255) & ~size_t(255);
  return 2 * state + 256;
}
}  // namespace

// the live FV patches of one (scheme, planar) group as a device table
struct FVGroup {
  std::vector<FVServePatch> host;
  FVServePatch* dev = nullptr;
  int cap = 0;
  int ntiles = 0;
};

struct exa_server {
  exa_ensemble* ens = nullptr;
  cudaStream_t fv_st = nullptr;
  FVGroup groups[4];  // scheme * 2 + planar
  bool fv_dirty = true;
  int precision = 0;
  int max_requests = 0;
  uint64_t next_id = 1;
  std::map<uint64_t, Req> live;
  std::vector<uint64_t> completed;
  std::mutex mu;
  std::vector<double> st_time;
  std::vector<uint64_t> st_steps, st_picard;
  std::vector<int> st_active, st_nan;
  double evict_after_s = 0.0;  // exa_server_run preemption (<= 0: off)
  // FV steps per tick (exa_server_set_fv_steps); measured on the benchmark
  // mix at 200 req/s: 1 step p50 / p99 1.43 / 3.95 s, 2 steps 0.67 / 3.53 s,
  // 3 steps 0.44-0.49 / 3.5-3.6 s, and choosing per tick from event timings
  // (DG step time over one FV step's, 1..4) 0.59 / 4.43 s
  int fv_steps = 3;
  bool tick_dg = false;  // the launched tick has ADER-DG work (tick_launch -> tick_finish)
  // exa_server_run's result hand-out (exa_server_set_result_mode): 1 the
  // finished states are copied into a pinned staging ring on their own
  // stream while the next tick runs; 0 each is copied synchronously after
  // its tick (the GPU idles meanwhile)
  int result_mode = 1;
  cudaStream_t res_st = nullptr;
  char* stage = nullptr;  // pinned host memory
  size_t stage_cap = 0;
  size_t stage_min = size_t(256) << 20;  // exa_server_set_staging
  std::vector<cudaEvent_t> free_events;
  // host seconds of the last exa_server_run: launching ticks, waiting for
  // them, handing out results, admission and eviction
  double loop_s[4] = {0.0, 0.0, 0.0, 0.0};
};

extern "C" {

size_t exa_server_footprint(const exa_request_t* r) {
  if (!r) return 0;
  if (r->kind == EXA_REQ_ADERDG) return exa_ensemble_footprint(&r->dg);
  if (r->kind == EXA_REQ_FV) {
    if (r->fv_patch < 1) return 0;
    return fv_bytes(r);
  }
  return 0;
}

exa_status_t exa_server_create(size_t hbm_budget, int max_requests, int precision, exa_server** out) {
  if (!out || max_requests < 1) return set_error(EXA_EINVAL, "bad server arguments");
  exa_server* s = new (std::nothrow) exa_server;
  if (!s) return set_error(EXA_ENOMEM, "host allocation");
  s->precision = precision;
  s->max_requests = max_requests;
  exa_status_t st = exa_ensemble_create(precision, max_requests, hbm_budget, &s->ens);
  if (!st) st = cuda_status(cudaStreamCreateWithFlags(&s->fv_st, cudaStreamNonBlocking), "fv stream");
  if (st) {
    exa_server_destroy(s);
    return st;
  }
  // ADER-DG requests of a tick: one launch per order and phase, replayed as
  // a graph (measured: 175 req/s of the benchmark mix sustained against 150
  // with the persistent launch, whose CTAs all reserve the largest order's
  // shared memory)
  exa_ensemble_set_launch_mode(s->ens, 1);
  exa_ensemble_use_graph(s->ens, 1);

  s->st_time.resize(max_requests);
  s->st_steps.resize(max_requests);
  s->st_picard.resize(max_requests);
  s->st_active.resize(max_requests);
  s->st_nan.resize(max_requests);
  *out = s;
  return EXA_OK;
}

exa_status_t exa_server_destroy(exa_server* s) {
  if (!s) return EXA_OK;
  if (s->fv_st) {
    cudaStreamSynchronize(s->fv_st);
    cudaStreamDestroy(s->fv_st);
  }
  if (s->res_st) {
    cudaStreamSynchronize(s->res_st);
    cudaStreamDestroy(s->res_st);
  }
  for (cudaEvent_t ev : s->free_events) cudaEventDestroy(ev);
  if (s->stage) cudaFreeHost(s->stage);
  if (s->ens) exa_ensemble_destroy(s->ens);
  for (FVGroup& gr : s->groups) cudaFree(gr.dev);
  delete s;
  return EXA_OK;
}

exa_status_t exa_server_submit(exa_server* s, const exa_request_t* r, uint64_t* id) {
  if (!s || !r || !id) return set_error(EXA_EINVAL, "NULL argument");
  if (r->steps < 1) return set_error(EXA_EINVAL, "steps must be >= 1");
  std::lock_guard<std::mutex> lk(s->mu);
  if ((int)s->live.size() >= s->max_requests) return set_error(EXA_EBUSY, "request slots full");
  Req q;
  q.id = s->next_id;
  q.r = *r;
  q.steps_left = r->steps;
  if (r->kind == EXA_REQ_ADERDG) {
    int slot = -1;
    exa_status_t st = exa_ensemble_add(s->ens, &r->dg, r->steps, &slot);
    if (st) return st;  // EXA_EBUSY when the footprint does not fit
    q.slot = slot;
  } else if (r->kind == EXA_REQ_FV) {
    if (r->fv_patch < 1 || r->fv_scheme < 0 || r->fv_scheme > 1 || !(r->fv_length > 0))
      return set_error(EXA_EINVAL, "bad FV request");
    q.fv = exa_fv_desc_t{2, r->fv_patch, r->fv_scheme == 0 ? 1 : 2, kV, 0, r->dg.pde,
                         {r->fv_length, r->fv_length, 1.0}};
    q.bytes = fv_bytes(r);
    char* p = nullptr;
    if (!ens_arena_alloc(s->ens, q.bytes, &p, &q.off))
      return set_error(EXA_EBUSY, "not enough free device memory in the arena");
    const size_t S = (size_t)q.fv.patch + 2 * q.fv.ghost;
    const size_t state = ((S * S * kV * 8) + 255) & ~size_t(255);
    q.luh = (double*)p;
    q.luh_new = (double*)(p + state);
    q.dt_slot = (unsigned long long*)(p + 2 * state);
    cudaError_t e = cudaMemsetAsync(q.dt_slot, 0, 32, s->fv_st);
    exa_status_t st = e == cudaSuccess ? launch_fv_ic(q.fv, q.luh, r->dg.ic_param, r->dg.seed, r->dg.noise, s->fv_st)
                                       : cuda_status(e, "fv scalars");
    // both state buffers start as the initial state: the steps write
    // interiors only, so the ghost cells of a result are the initial ones
    // whichever buffer holds it
    if (!st)
      st = cuda_status(cudaMemcpyAsync(q.luh_new, q.luh, S * S * kV * 8, cudaMemcpyDeviceToDevice, s->fv_st),
                       "fv second buffer");
    if (!st) st = fv_patch_prime_async(q.fv, q.luh, q.dt_slot, s->fv_st);
    if (st) {
      ens_arena_free(s->ens, q.off, q.bytes);
      return st;
    }
  } else {
    return set_error(EXA_EINVAL, "unknown request kind");
  }
  s->next_id++;
  *id = q.id;
  s->live[q.id] = q;
  if (r->kind == EXA_REQ_FV) s->fv_dirty = true;
  return EXA_OK;
}

namespace {
// rebuilds the device tables of the live FV patches (after admissions and
// completions); stream-ordered after the previous tick's launches
exa_status_t rebuild_fv_groups(exa_server* s) {
  for (FVGroup& gr : s->groups) {
    gr.host.clear();
    gr.ntiles = 0;
  }
  for (auto& kv : s->live) {
    Req& q = kv.second;
    if (q.done || q.evicted || q.r.kind != EXA_REQ_FV) continue;
    FVGroup& gr = s->groups[q.r.fv_scheme * 2 + (q.fv.pde == EXA_PDE_EULER_PLANAR ? 1 : 0)];
    FVServePatch p{};
    p.buf[0] = q.luh;
    p.buf[1] = q.luh_new;
    p.slots = q.dt_slot;
    p.P = q.fv.patch;
    p.g = q.fv.ghost;
    p.hx = q.fv.dx[0] / q.fv.patch;
    p.hy = q.fv.dx[1] / q.fv.patch;
    p.tile0 = gr.ntiles;
    gr.ntiles += fv_serve_tiles(q.r.fv_scheme, q.fv.patch, &p.tiles_x);
    gr.host.push_back(p);
  }
  for (FVGroup& gr : s->groups) {
    const int np = (int)gr.host.size();
    if (np == 0) continue;
    if (np > gr.cap) {
      // the old table may still be read by the last tick's launch
      cudaError_t e = cudaStreamSynchronize(s->fv_st);
      if (e == cudaSuccess) e = cudaFree(gr.dev);
      gr.dev = nullptr;
      gr.cap = 0;
      const int cap = np > 64 ? 2 * np : 128;
      if (e == cudaSuccess) e = cudaMalloc(&gr.dev, sizeof(FVServePatch) * cap);
      if (e != cudaSuccess) return cuda_status(e, "fv serving table");
      gr.cap = cap;
    }
    cudaError_t e = cudaMemcpyAsync(gr.dev, gr.host.data(), sizeof(FVServePatch) * np, cudaMemcpyHostToDevice,
                                    s->fv_st);
    if (e != cudaSuccess) return cuda_status(e, "fv serving table upload");
  }
  s->fv_dirty = false;
  return EXA_OK;
}
}  // namespace

namespace {
// A tick in two halves: tick_launch enqueues the work (the host returns
// while the GPU runs it), tick_finish waits for it and records the
// completions.  Both with s->mu held.
exa_status_t tick_launch(exa_server* s) {
  bool any_dg = false;
  for (auto& kv : s->live)
    if (!kv.second.done && !kv.second.evicted && kv.second.r.kind == EXA_REQ_ADERDG) any_dg = true;
  s->tick_dg = any_dg;
  if (any_dg)
    if (exa_status_t st = exa_ensemble_step(s->ens, 1)) return st;
  // FV patches: several steps per tick on their own stream (they overlap
  // the ADER-DG launch, whose step is the longer one); a patch whose budget
  // runs out mid-tick leaves the table before the next of them
  for (int sub = 0; sub < s->fv_steps; sub++) {
    if (s->fv_dirty)
      if (exa_status_t st = rebuild_fv_groups(s)) return st;
    bool any_fv = false;
    for (int k = 0; k < 4; k++) {
      FVGroup& gr = s->groups[k];
      any_fv = any_fv || !gr.host.empty();
      if (exa_status_t st = fv_serve_step_async(k / 2, k % 2 == 1, gr.dev, (int)gr.host.size(), gr.ntiles, s->fv_st))
        return st;
    }
    if (!any_fv) break;
    for (auto& kv : s->live) {
      Req& q = kv.second;
      if (q.done || q.evicted || q.r.kind != EXA_REQ_FV) continue;
      q.par ^= 1;
      q.steps_done++;
      if (--q.steps_left == 0) {
        q.done = true;
        s->fv_dirty = true;
      }
    }
  }
  return EXA_OK;
}

exa_status_t tick_finish(exa_server* s, int* ncompleted) {
  const bool any_dg = s->tick_dg;
  exa_status_t st = EXA_OK;
  if (any_dg) {
    st = exa_ensemble_status(s->ens, s->st_time.data(), s->st_steps.data(), s->st_active.data(),
                             s->st_picard.data(), s->st_nan.data());
    if (st && st != EXA_ENAN) return st;
  }
  cudaError_t e = cudaStreamSynchronize(s->fv_st);
  if (e != cudaSuccess) return cuda_status(e, "fv stream");
  int n = 0;
  for (auto& kv : s->live) {
    Req& q = kv.second;
    if (q.r.kind == EXA_REQ_ADERDG && !q.done && !q.evicted && any_dg && !s->st_active[q.slot]) {
      q.done = true;
      q.steps_done = (long long)s->st_steps[q.slot];
    }
    if (q.done && !q.reported) {
      q.reported = true;
      s->completed.push_back(q.id);
      n++;
    }
  }
  if (ncompleted) *ncompleted = n;
  return st;
}
}  // namespace

exa_status_t exa_server_tick(exa_server* s, int* ncompleted) {
  if (!s) return set_error(EXA_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (exa_status_t st = tick_launch(s)) return st;
  return tick_finish(s, ncompleted);
}

exa_status_t exa_server_completed(exa_server* s, uint64_t* ids, int cap, int* n) {
  if (!s || !n || (cap > 0 && !ids)) return set_error(EXA_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  int k = 0;
  while (k < cap && !s->completed.empty()) {
    ids[k++] = s->completed.front();
    s->completed.erase(s->completed.begin());
  }
  *n = k;
  return EXA_OK;
}

size_t exa_server_result_size(exa_server* s, uint64_t id) {
  if (!s) return 0;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return 0;
  const Req& q = it->second;
  if (q.r.kind == EXA_REQ_ADERDG) {
    const int B = q.r.dg.order + 1;
    return (size_t)q.r.dg.n[0] * q.r.dg.n[1] * B * B * kV;
  }
  const size_t S = (size_t)q.fv.patch + 2 * q.fv.ghost;
  return S * S * kV;
}

exa_status_t exa_server_result(exa_server* s, uint64_t id, double* host_out, double* sim_time,
                               long long* steps_done) {
  if (!s || !host_out) return set_error(EXA_EINVAL, "NULL argument");
  const size_t n = exa_server_result_size(s, id);
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  Req& q = it->second;
  if (!q.done) return set_error(EXA_EBUSY, "request still running");
  exa_status_t st = EXA_OK;
  if (q.r.kind == EXA_REQ_ADERDG) {
    const bool failed = s->st_nan[q.slot] != 0;
    st = exa_ensemble_get_state(s->ens, q.slot, host_out);
    if (sim_time) *sim_time = s->st_time[q.slot];
    if (!st) st = exa_ensemble_remove(s->ens, q.slot);
    // a solve that produced a non-finite state stopped there (the others
    // went on): its result is returned and the request reported failed
    if (!st && failed) st = set_error(EXA_ENAN, "the solve produced a non-finite state");
  } else {
    double scal[2];
    cudaError_t e = cudaMemcpyAsync(host_out, q.par ? q.luh_new : q.luh, n * sizeof(double),
                                    cudaMemcpyDeviceToHost, s->fv_st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(scal, q.dt_slot, 16, cudaMemcpyDeviceToHost, s->fv_st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->fv_st);
    if (e != cudaSuccess) return cuda_status(e, "fv result");
    if (sim_time) *sim_time = scal[1];
    ens_arena_free(s->ens, q.off, q.bytes);
  }
  if (steps_done) *steps_done = q.steps_done;
  s->live.erase(it);
  return st;
}

// Eviction (dump and restore of a solve's device state): the
// request's state and time-step scalars move to host memory and its device
// memory returns to the arena; restore re-admits it from there.
static exa_status_t server_evict_locked(exa_server* s, Req& q) {
  if (q.done) return set_error(EXA_EINVAL, "request already finished");
  if (q.evicted) return EXA_OK;
  if (q.r.kind == EXA_REQ_ADERDG) {
    const int B = q.r.dg.order + 1;
    q.saved.resize((size_t)q.r.dg.n[0] * q.r.dg.n[1] * B * B * kV);
    if (exa_status_t st = exa_ensemble_checkpoint(s->ens, q.slot, q.saved.data(), &q.ck)) return st;
    if (exa_status_t st = exa_ensemble_remove(s->ens, q.slot)) return st;
    q.slot = -1;
  } else {
    const size_t S = (size_t)q.fv.patch + 2 * q.fv.ghost;
    q.saved.resize(S * S * kV);
    // the last tick's launches on the FV stream wrote this state
    cudaError_t e = cudaMemcpyAsync(q.saved.data(), q.par ? q.luh_new : q.luh, q.saved.size() * 8,
                                    cudaMemcpyDeviceToHost, s->fv_st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.fv_scal, q.dt_slot, 32, cudaMemcpyDeviceToHost, s->fv_st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->fv_st);
    if (e != cudaSuccess) return cuda_status(e, "fv evict");
    ens_arena_free(s->ens, q.off, q.bytes);
    q.luh = q.luh_new = nullptr;
    q.dt_slot = nullptr;
    s->fv_dirty = true;
  }
  q.evicted = true;
  return EXA_OK;
}

static exa_status_t server_restore_locked(exa_server* s, Req& q) {
  if (!q.evicted) return EXA_OK;
  if (q.r.kind == EXA_REQ_ADERDG) {
    int slot = -1;
    if (exa_status_t st = exa_ensemble_restore(s->ens, &q.r.dg, q.saved.data(), &q.ck, &slot)) return st;
    q.slot = slot;
  } else {
    char* p = nullptr;
    if (!ens_arena_alloc(s->ens, q.bytes, &p, &q.off))
      return set_error(EXA_EBUSY, "not enough free device memory in the arena");
    const size_t S = (size_t)q.fv.patch + 2 * q.fv.ghost;
    const size_t state = ((S * S * kV * 8) + 255) & ~size_t(255);
    q.luh = (double*)p;
    q.luh_new = (double*)(p + state);
    q.dt_slot = (unsigned long long*)(p + 2 * state);
    q.par = 0;  // the state goes to buffer 0
    unsigned long long scal[4] = {q.fv_scal[0], q.fv_scal[1], q.fv_scal[2], 0ULL};
    // the saved state into both buffers (as at submission, both hold the
    // same ghost cells; the next step overwrites the other's interior)
    cudaError_t e = cudaMemcpyAsync(q.luh, q.saved.data(), q.saved.size() * 8, cudaMemcpyHostToDevice, s->fv_st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(q.luh_new, q.luh, q.saved.size() * 8, cudaMemcpyDeviceToDevice, s->fv_st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(q.dt_slot, scal, 32, cudaMemcpyHostToDevice, s->fv_st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->fv_st);
    if (e != cudaSuccess) {
      ens_arena_free(s->ens, q.off, q.bytes);
      return cuda_status(e, "fv restore");
    }
    s->fv_dirty = true;
  }
  q.evicted = false;
  q.saved.clear();
  q.saved.shrink_to_fit();
  return EXA_OK;
}

exa_status_t exa_server_evict(exa_server* s, uint64_t id) {
  if (!s) return set_error(EXA_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  return server_evict_locked(s, it->second);
}

exa_status_t exa_server_restore(exa_server* s, uint64_t id) {
  if (!s) return set_error(EXA_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  return server_restore_locked(s, it->second);
}

exa_status_t exa_server_evicted(exa_server* s, uint64_t id, int* evicted) {
  if (!s || !evicted) return set_error(EXA_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  *evicted = it->second.evicted ? 1 : 0;
  return EXA_OK;
}

exa_status_t exa_server_set_fv_steps(exa_server* s, int steps) {
  if (!s || steps < 1) return set_error(EXA_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  s->fv_steps = steps;
  return EXA_OK;
}

exa_status_t exa_server_set_eviction(exa_server* s, double wait_s) {
  if (!s) return set_error(EXA_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->evict_after_s = wait_s > 0 ? wait_s : 0.0;
  return EXA_OK;
}

exa_status_t exa_server_tune(exa_server* s, int launch_mode, int use_graph) {
  if (!s) return set_error(EXA_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (exa_status_t st = exa_ensemble_set_launch_mode(s->ens, launch_mode)) return st;
  return exa_ensemble_use_graph(s->ens, use_graph);
}

exa_status_t exa_server_device_state(exa_server* s, uint64_t id, double** luh_dev) {
  if (!s || !luh_dev) return set_error(EXA_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  const Req& q = it->second;
  if (q.evicted) return set_error(EXA_EBUSY, "request evicted to host memory");
  if (q.r.kind == EXA_REQ_ADERDG) return exa_ensemble_device_state(s->ens, q.slot, luh_dev);
  *luh_dev = q.par ? q.luh_new : q.luh;
  return EXA_OK;
}

exa_status_t exa_server_info(exa_server* s, int* live_requests, long* active_dg_cells,
                             size_t* arena_free_bytes) {
  if (!s) return set_error(EXA_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (live_requests) *live_requests = (int)s->live.size();
  if (active_dg_cells) *active_dg_cells = exa_ensemble_active_cells(s->ens);
  return exa_ensemble_info(s->ens, nullptr, nullptr, arena_free_bytes);
}

namespace {
// A finished request whose state exa_server_run is copying into the pinned
// staging ring (stage + off: the state, then for FV the 16 bytes of dt and
// time) on the result stream
struct PendingResult {
  uint64_t id = 0;
  int index = 0;
  size_t off = 0;
  size_t n = 0;  // doubles of the state
  bool fv = false;
  cudaEvent_t ev = nullptr;
  double sim_time = 0.0;
  long long steps = 0;
  exa_status_t status = EXA_OK;
};

// enqueues the copy of finished request p.id's state; the tick that
// finished it has completed, and no later tick writes it (ADER-DG: the
// solve is inactive; FV: the patch has left the table)
exa_status_t result_copy_begin(exa_server* s, PendingResult& p) {
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->live.find(p.id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  const Req& q = it->second;
  const double* src = nullptr;
  if (q.r.kind == EXA_REQ_ADERDG) {
    double* d = nullptr;
    if (exa_status_t st = exa_ensemble_device_state(s->ens, q.slot, &d)) return st;
    src = d;
    p.sim_time = s->st_time[q.slot];
    p.status = s->st_nan[q.slot] ? EXA_ENAN : EXA_OK;
  } else {
    src = q.par ? q.luh_new : q.luh;
  }
  p.steps = q.steps_done;
  char* dst = s->stage + p.off;
  cudaError_t e = cudaMemcpyAsync(dst, src, p.n * sizeof(double), cudaMemcpyDeviceToHost, s->res_st);
  if (e == cudaSuccess && p.fv)
    e = cudaMemcpyAsync(dst + p.n * sizeof(double), q.dt_slot, 16, cudaMemcpyDeviceToHost, s->res_st);
  if (e == cudaSuccess) e = cudaEventRecord(p.ev, s->res_st);
  return cuda_status(e, "result copy");
}

// the copy of p has completed: the state goes to out (nullable), the
// request's device memory back to the arena
exa_status_t result_hand_out(exa_server* s, PendingResult& p, double* out) {
  if (out) std::memcpy(out, s->stage + p.off, p.n * sizeof(double));
  if (p.fv) {
    double scal[2];
    std::memcpy(scal, s->stage + p.off + p.n * sizeof(double), sizeof(scal));
    p.sim_time = scal[1];
  }
  std::lock_guard<std::mutex> lk(s->mu);
  s->free_events.push_back(p.ev);
  p.ev = nullptr;
  auto it = s->live.find(p.id);
  if (it == s->live.end()) return set_error(EXA_ENOTFOUND, "unknown request id");
  Req& q = it->second;
  exa_status_t st = EXA_OK;
  if (q.r.kind == EXA_REQ_ADERDG) st = ens_remove_finished(s->ens, q.slot);
  else ens_arena_free(s->ens, q.off, q.bytes);
  s->live.erase(it);
  return st;
}
}  // namespace

exa_status_t exa_server_set_result_mode(exa_server* s, int mode) {
  if (!s || mode < 0 || mode > 1) return set_error(EXA_EINVAL, "result mode: 0 synchronous, 1 overlapped");
  std::lock_guard<std::mutex> lk(s->mu);
  s->result_mode = mode;
  return EXA_OK;
}

exa_status_t exa_server_set_staging(exa_server* s, size_t bytes) {
  if (!s || bytes < 4096) return set_error(EXA_EINVAL, "staging capacity: at least 4096 bytes");
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->res_st) {
    const cudaError_t e = cudaStreamSynchronize(s->res_st);
    if (e != cudaSuccess) return cuda_status(e, "result stream");
  }
  if (s->stage) cudaFreeHost(s->stage);
  s->stage = nullptr;
  s->stage_cap = 0;
  s->stage_min = bytes;
  return EXA_OK;
}

exa_status_t exa_server_loop_times(exa_server* s, double* seconds4) {
  if (!s || !seconds4) return set_error(EXA_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  for (int k = 0; k < 4; k++) seconds4[k] = s->loop_s[k];
  return EXA_OK;
}

exa_status_t exa_server_run(exa_server* s, const exa_request_t* reqs, exa_request_record_t* rec, int n,
                            double time_limit_s, double* const* results, uint64_t* ticks) {
  if (!s || (n > 0 && (!reqs || !rec)) || n < 0) return set_error(EXA_EINVAL, "bad argument");
  using clock = std::chrono::steady_clock;
  const auto t0 = clock::now();
  auto now = [&]() { return std::chrono::duration<double>(clock::now() - t0).count(); };
  for (int i = 0; i < n; i++) {
    rec[i].admitted_s = -1.0;
    rec[i].completed_s = -1.0;
    rec[i].sim_time = 0.0;
    rec[i].steps_done = 0;
    rec[i].status = -1;
    rec[i].evictions = 0;
  }
  double evict_after = 0.0;
  bool overlap = true;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    evict_after = s->evict_after_s;
    overlap = s->result_mode == 1;
    if (overlap && !s->res_st) {
      const cudaError_t e = cudaStreamCreateWithFlags(&s->res_st, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_status(e, "result stream");
    }
  }
  double loop_s[4] = {0.0, 0.0, 0.0, 0.0};  // launch, wait, results, admission
  std::deque<int> queue;              // arrived, not yet admitted (arrival order)
  std::map<uint64_t, int> live;       // request id -> index (running)
  std::deque<uint64_t> evicted;       // evicted ids, in eviction order
  std::map<uint64_t, double> resident_since;
  std::vector<double> scratch;
  std::vector<uint64_t> ids(256);
  // overlapped results: copies in flight, in issue order; they occupy the
  // staging ring from pend.front().off up to head (wrapping at stage_cap)
  std::deque<PendingResult> pend;
  size_t head = 0;
  int next = 0, done = 0;
  uint64_t nt = 0;
  exa_status_t err = EXA_OK;

  // hands out the oldest copy in flight once it has completed (wait: block
  // until then)
  auto finish_front = [&](bool wait, bool* finished) -> exa_status_t {
    *finished = false;
    PendingResult& p = pend.front();
    const cudaError_t e = wait ? cudaEventSynchronize(p.ev) : cudaEventQuery(p.ev);
    if (e == cudaErrorNotReady) return EXA_OK;
    if (e != cudaSuccess) return cuda_status(e, "result copy");
    const exa_status_t rs = result_hand_out(s, p, results ? results[p.index] : nullptr);
    exa_request_record_t& r = rec[p.index];
    r.completed_s = now();
    r.sim_time = p.sim_time;
    r.steps_done = p.steps;
    r.status = rs ? rs : p.status;
    done++;
    pend.pop_front();
    *finished = true;
    return rs;
  };
  auto finish_ready = [&](bool wait) -> exa_status_t {
    while (!pend.empty()) {
      bool fin = false;
      if (exa_status_t st = finish_front(wait, &fin)) return st;
      if (!fin) break;
    }
    return EXA_OK;
  };
  // a staging range of `bytes` for the next copy, waiting for older copies
  // while the ring has no room
  auto stage_alloc = [&](size_t bytes, size_t* off) -> exa_status_t {
    bytes = (bytes + 255) & ~size_t(255);
    for (;;) {
      if (pend.empty()) {
        if (bytes > s->stage_cap) {
          std::lock_guard<std::mutex> lk(s->mu);
          if (s->stage) cudaFreeHost(s->stage);
          s->stage = nullptr;
          s->stage_cap = 0;
          const size_t cap = std::max(bytes, s->stage_min);
          const cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&s->stage), cap, cudaHostAllocDefault);
          if (e != cudaSuccess) return cuda_status(e, "result staging memory");
          s->stage_cap = cap;
        }
        *off = 0;
        head = bytes;
        return EXA_OK;
      }
      const size_t tail = pend.front().off;
      if (head > tail) {  // [tail, head) in use
        if (s->stage_cap - head >= bytes) {
          *off = head;
          head += bytes;
          return EXA_OK;
        }
        if (bytes < tail) {
          *off = 0;
          head = bytes;
          return EXA_OK;
        }
      } else if (head + bytes < tail) {  // wrapped: [tail, cap) and [0, head) in use
        *off = head;
        head += bytes;
        return EXA_OK;
      }
      bool fin = false;
      if (exa_status_t st = finish_front(true, &fin)) return st;
    }
  };

  while (done < n) {
    const double t = now();
    if (time_limit_s > 0 && t > time_limit_s) break;
    while (next < n && rec[next].arrival_s <= t) queue.push_back(next++);
    // evicted requests come back first, as soon as they fit
    for (auto it = evicted.begin(); it != evicted.end();) {
      const exa_status_t st = exa_server_restore(s, *it);
      if (st == EXA_EBUSY) {
        ++it;
        continue;
      }
      if (st) {
        err = st;
        break;
      }
      resident_since[*it] = now();
      it = evicted.erase(it);
    }
    if (err) break;
    // admission: first fit in arrival order (a request that does not fit
    // now keeps its place; smaller later ones may go first); none while an
    // evicted request waits to come back, so it cannot starve
    for (auto it = queue.begin(); evicted.empty() && it != queue.end();) {
      uint64_t id = 0;
      const exa_status_t st = exa_server_submit(s, &reqs[*it], &id);
      if (st == EXA_EBUSY) {
        ++it;
        continue;
      }
      if (st) {
        err = st;
        break;
      }
      rec[*it].admitted_s = now();
      live[id] = *it;
      resident_since[id] = rec[*it].admitted_s;
      it = queue.erase(it);
    }
    if (err) break;
    // preemption: the oldest waiting request has waited too long: evict
    // running requests resident for at least as long, largest footprint
    // first, until it is admitted
    if (evict_after > 0 && !queue.empty() && evicted.empty() && now() - rec[queue.front()].arrival_s > evict_after) {
      std::vector<std::pair<size_t, uint64_t>> cand;
      for (auto& kv : live) {
        if (now() - resident_since[kv.first] < evict_after) continue;
        cand.push_back({exa_server_footprint(&reqs[kv.second]), kv.first});
      }
      std::sort(cand.begin(), cand.end(), [](const std::pair<size_t, uint64_t>& a,
                                             const std::pair<size_t, uint64_t>& b) { return a.first > b.first; });
      const int head_req = queue.front();
      for (const auto& c : cand) {
        const exa_status_t ev = exa_server_evict(s, c.second);
        if (ev == EXA_EINVAL) continue;  // finished in the last tick: its result is collected below
        if (ev) {
          err = ev;
          break;
        }
        evicted.push_back(c.second);
        rec[live[c.second]].evictions++;
        uint64_t id = 0;
        const exa_status_t st = exa_server_submit(s, &reqs[head_req], &id);
        if (st == EXA_EBUSY) continue;
        if (st) {
          err = st;
          break;
        }
        rec[head_req].admitted_s = now();
        live[id] = head_req;
        resident_since[id] = rec[head_req].admitted_s;
        queue.pop_front();
        break;
      }
      if (err) break;
    }
    loop_s[3] += now() - t;
    if (live.empty()) {
      if (!pend.empty()) {
        const double t1 = now();
        err = finish_ready(true);
        loop_s[2] += now() - t1;
        if (err) break;
        continue;
      }
      if (next < n) {
        const double wait = rec[next].arrival_s - now();
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait < 0.01 ? wait : 0.01));
      } else if (!queue.empty()) {
        err = set_error(EXA_EBUSY, "a request does not fit into the server's memory budget even alone");
        break;
      }
      continue;
    }
    int nc = 0;
    const double t1 = now();
    exa_status_t st;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      st = tick_launch(s);
    }
    nt++;
    if (st) {
      err = st;
      break;
    }
    const double t2 = now();
    // while the GPU runs the tick: hand out the results whose copies are done
    if ((err = finish_ready(false))) break;
    const double t3 = now();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      st = tick_finish(s, &nc);
    }
    const double t4 = now();
    loop_s[0] += t2 - t1;
    loop_s[2] += t3 - t2;
    loop_s[1] += t4 - t3;
    if (st && st != EXA_ENAN) {
      err = st;
      break;
    }
    for (;;) {
      int k = 0;
      if ((err = exa_server_completed(s, ids.data(), (int)ids.size(), &k))) break;
      for (int j = 0; j < k; j++) {
        const int i = live[ids[j]];
        live.erase(ids[j]);
        resident_since.erase(ids[j]);
        if (overlap) {
          PendingResult p;
          p.id = ids[j];
          p.index = i;
          p.n = exa_server_result_size(s, ids[j]);
          p.fv = reqs[i].kind == EXA_REQ_FV;
          if ((err = stage_alloc(p.n * sizeof(double) + (p.fv ? 16 : 0), &p.off))) break;
          {
            std::lock_guard<std::mutex> lk(s->mu);
            if (!s->free_events.empty()) {
              p.ev = s->free_events.back();
              s->free_events.pop_back();
            }
          }
          if (!p.ev) {
            const cudaError_t e = cudaEventCreateWithFlags(&p.ev, cudaEventDisableTiming);
            if (e != cudaSuccess) {
              err = cuda_status(e, "result event");
              break;
            }
          }
          pend.push_back(p);
          if ((err = result_copy_begin(s, pend.back()))) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->free_events.push_back(pend.back().ev);
            pend.pop_back();
            break;
          }
          continue;
        }
        double* out = results ? results[i] : nullptr;
        if (!out) {
          scratch.resize(exa_server_result_size(s, ids[j]));
          out = scratch.data();
        }
        double simt = 0.0;
        long long steps = 0;
        const exa_status_t rs = exa_server_result(s, ids[j], out, &simt, &steps);
        if (rs && rs != EXA_ENAN) {
          err = rs;
          break;
        }
        rec[i].completed_s = now();
        rec[i].sim_time = simt;
        rec[i].steps_done = steps;
        rec[i].status = rs;
        done++;
      }
      if (err || k < (int)ids.size()) break;
    }
    loop_s[2] += now() - t4;
    if (err) break;
  }
  // copies still in flight (time limit, error): wait for them and hand
  // them out, so that no request is left half collected
  if (!pend.empty()) {
    if (s->res_st) cudaStreamSynchronize(s->res_st);
    const exa_status_t st = finish_ready(true);
    if (!err) err = st;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int k = 0; k < 4; k++) s->loop_s[k] = loop_s[k];
  }
  if (ticks) *ticks = nt;
  return err;
}

}  // extern "C"
