// C ABI of libexahype_b200: runtime helpers, per-cell drop-ins, batched
// device entry points and the uniform periodic ADER-DG grid.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <float.h>

#include "exa_device.cuh"

namespace exa {

// ------------------------------------------------------------ errors
static thread_local std::string t_last_error;
static std::atomic<uint64_t> g_launches{0};

exa_status_t set_error(exa_status_t s, const char* msg) {
  if (s != EXA_OK) t_last_error = msg ? msg : "";
  return s;
}

exa_status_t cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return EXA_OK;
  t_last_error = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return EXA_ENOMEM;
  return EXA_ECUDA;
}

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static std::atomic<int> g_tune[kTuneCount] = {};
static std::atomic<unsigned> g_tune_set{0};

int tune_get(int key, int dflt) {
  if (key < 0 || key >= kTuneCount) return dflt;
  return (g_tune_set.load() >> key) & 1u ? g_tune[key].load() : dflt;
}

double host_pnpm(int order);

static std::mutex g_tables_mu;
static bool g_tables_done[256];

exa_status_t ensure_tables() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_tables_mu);
  if (g_tables_done[dev & 255]) return EXA_OK;
  exa_status_t s;
  if ((s = upload_tables_predictor())) return s;
  if ((s = upload_tables_amr())) return s;
  if ((s = upload_tables_limiter())) return s;
  if ((s = upload_tables_predictor_mixed())) return s;
  if ((s = upload_tables_ensemble())) return s;
  if ((s = upload_tables_faces())) return s;
  if ((s = upload_tables_fv())) return s;
  if ((s = upload_tables_adjust())) return s;
  g_tables_done[dev & 255] = true;
  return EXA_OK;
}

exa_status_t check_aderdg_desc(const exa_aderdg_desc_t* d) {
  if (!d) return set_error(EXA_EINVAL, "NULL descriptor");
  if (d->dim != 2 && d->dim != 3) return set_error(EXA_EINVAL, "dim must be 2 or 3");
  if (d->order < 2 || d->order > 5) return set_error(EXA_EINVAL, "order must be in 2..5");
  if (d->nvar != kV) return set_error(EXA_EINVAL, "nvar must be 5 (Euler)");
  if (d->npar < 0 || d->npar > 1) return set_error(EXA_EINVAL, "npar must be 0 or 1");
  if (d->pde != EXA_PDE_EULER && d->pde != EXA_PDE_EULER_PLANAR)
    return set_error(EXA_EINVAL, "unknown pde");
  if (d->pde == EXA_PDE_EULER_PLANAR && d->dim != 2)
    return set_error(EXA_EINVAL, "planar Euler is a 2D PDE");
  for (int i = 0; i < d->dim; i++)
    if (!(d->dx[i] > 0.0)) return set_error(EXA_EINVAL, "dx must be positive");
  return EXA_OK;
}

static exa_status_t check_aderdg(const exa_aderdg_desc_t* d) {
  if (exa_status_t s = check_aderdg_desc(d)) return s;
  return ensure_tables();
}

static int ipow_h(int b, int e) { int r = 1; while (e-- > 0) r *= b; return r; }

// -------------------------------------------------- drop-in workspace
struct Workspace {
  double* buf = nullptr;
  size_t cap = 0;  // doubles
  std::mutex mu;
};
static Workspace g_ws[256];

static exa_status_t ws_get(size_t doubles, double** out, std::unique_lock<std::mutex>& lk) {
  int dev = 0;
  cudaGetDevice(&dev);
  Workspace& w = g_ws[dev & 255];
  lk = std::unique_lock<std::mutex>(w.mu);
  if (w.cap < doubles) {
    if (w.buf) cudaFree(w.buf);
    w.buf = nullptr;
    w.cap = 0;
    cudaError_t e = cudaMalloc(&w.buf, doubles * sizeof(double));
    if (e != cudaSuccess) return cuda_status(e, "drop-in workspace");
    w.cap = doubles;
  }
  *out = w.buf;
  return EXA_OK;
}

static size_t ws_capacity(int dev) {
  Workspace& w = g_ws[dev & 255];
  std::lock_guard<std::mutex> lk(w.mu);
  return w.cap;
}

}  // namespace exa

namespace exa {
// runs a simple batched kernel on one host cell: copies `nin` input arrays
// in, the launcher writes to the device copies, `nout` arrays come back.
struct HostArr { const void* src; void* dst; size_t n; };

template <typename F>
static exa_status_t run_one_cell(const HostArr* arrs, int narr, F launch) {
  size_t total = 0;
  for (int i = 0; i < narr; i++) total += arrs[i].n;
  std::unique_lock<std::mutex> lk;
  double* w = nullptr;
  if (exa_status_t s = ws_get(total + 1, &w, lk)) return s;
  std::vector<double*> dp(narr);
  double* p = w;
  for (int i = 0; i < narr; i++) {
    dp[i] = p;
    if (arrs[i].src) {
      cudaError_t e = cudaMemcpy(p, arrs[i].src, arrs[i].n * sizeof(double), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return cuda_status(e, "copy in");
    }
    p += arrs[i].n;
  }
  if (exa_status_t s = launch(dp.data())) return s;
  for (int i = 0; i < narr; i++)
    if (arrs[i].dst) {
      cudaError_t e = cudaMemcpy(arrs[i].dst, dp[i], arrs[i].n * sizeof(double), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) return cuda_status(e, "copy out");
    }
  return EXA_OK;
}

}  // namespace exa

using namespace exa;

// ================================================================ C ABI
extern "C" {

const char* exa_status_string(exa_status_t s) {
  switch (s) {
    case EXA_OK: return "ok";
    case EXA_EINVAL: return "invalid argument";
    case EXA_ENONCONV: return "Picard iteration did not converge";
    case EXA_ENAN: return "NaN or Inf produced";
    case EXA_ETIMEDOUT: return "device wait timed out";
    case EXA_ECUDA: return "CUDA error";
    case EXA_ENOMEM: return "out of memory";
    case EXA_EBUSY: return "busy";
    case EXA_ENOTFOUND: return "not found";
  }
  return "unknown status";
}

const char* exa_last_error_string(void) { return t_last_error.c_str(); }

int exa_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

exa_status_t exa_set_device(int device) { return cuda_status(cudaSetDevice(device), "cudaSetDevice"); }

exa_status_t exa_dropin_workspace_doubles(int device, size_t* doubles) {
  if (!doubles) return set_error(EXA_EINVAL, "NULL doubles");
  if (device < 0 || device > 255) return set_error(EXA_EINVAL, "device out of range");
  *doubles = ws_capacity(device);
  return EXA_OK;
}

exa_status_t exa_device_alloc(size_t bytes, void** ptr) {
  if (!ptr) return set_error(EXA_EINVAL, "NULL ptr");
  return cuda_status(cudaMalloc(ptr, bytes), "cudaMalloc");
}
exa_status_t exa_device_free(void* ptr) { return cuda_status(cudaFree(ptr), "cudaFree"); }
exa_status_t exa_host_alloc_pinned(size_t bytes, void** ptr) {
  if (!ptr) return set_error(EXA_EINVAL, "NULL ptr");
  return cuda_status(cudaMallocHost(ptr, bytes), "cudaMallocHost");
}
exa_status_t exa_host_free_pinned(void* ptr) { return cuda_status(cudaFreeHost(ptr), "cudaFreeHost"); }
exa_status_t exa_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
  return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream)),
                     "memcpy h2d");
}
exa_status_t exa_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
  return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)),
                     "memcpy d2h");
}
exa_status_t exa_memset_device(void* dst, int value, size_t bytes, void* stream) {
  return cuda_status(cudaMemsetAsync(dst, value, bytes, as_stream(stream)), "memset");
}
exa_status_t exa_stream_create(void** stream) {
  cudaStream_t s;
  exa_status_t r = cuda_status(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream create");
  if (r == EXA_OK) *stream = s;
  return r;
}
exa_status_t exa_stream_destroy(void* stream) {
  return cuda_status(cudaStreamDestroy(as_stream(stream)), "stream destroy");
}
exa_status_t exa_stream_synchronize(void* stream) {
  return cuda_status(cudaStreamSynchronize(as_stream(stream)), "stream sync");
}
exa_status_t exa_device_synchronize(void) { return cuda_status(cudaDeviceSynchronize(), "device sync"); }

struct ExaTimer { cudaEvent_t a, b; };
exa_status_t exa_timer_create(void** timer) {
  ExaTimer* t = new ExaTimer;
  cudaError_t e = cudaEventCreate(&t->a);
  if (e == cudaSuccess) e = cudaEventCreate(&t->b);
  if (e != cudaSuccess) { delete t; return cuda_status(e, "event create"); }
  *timer = t;
  return EXA_OK;
}
exa_status_t exa_timer_destroy(void* timer) {
  ExaTimer* t = (ExaTimer*)timer;
  cudaEventDestroy(t->a);
  cudaEventDestroy(t->b);
  delete t;
  return EXA_OK;
}
exa_status_t exa_timer_start(void* timer, void* stream) {
  return cuda_status(cudaEventRecord(((ExaTimer*)timer)->a, as_stream(stream)), "event record");
}
exa_status_t exa_timer_stop(void* timer, void* stream) {
  return cuda_status(cudaEventRecord(((ExaTimer*)timer)->b, as_stream(stream)), "event record");
}
exa_status_t exa_timer_elapsed_ms(void* timer, float* ms) {
  ExaTimer* t = (ExaTimer*)timer;
  cudaError_t e = cudaEventSynchronize(t->b);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, t->a, t->b);
  return cuda_status(e, "event elapsed");
}
uint64_t exa_launch_count(void) { return g_launches.load(); }

exa_status_t exa_tune_set(int key, int value) {
  if (key < 0 || key >= kTuneCount) return set_error(EXA_EINVAL, "unknown tuning key");
  g_tune[key].store(value);
  g_tune_set.fetch_or(1u << key);
  return EXA_OK;
}

int exa_tune_get(int key) { return tune_get(key, -1); }

// --------------------------------------------------- per-cell drop-ins
static exa_aderdg_desc_t with_dx(const exa_aderdg_desc_t* d, const double* dx) {
  exa_aderdg_desc_t r = *d;
  if (dx)
    for (int i = 0; i < d->dim; i++) r.dx[i] = dx[i];
  return r;
}

exa_status_t exa_aderdg_spaceTimePredictor(
    const exa_aderdg_desc_t* desc, double* lQhbnd, double* lFhbnd,
    double** tempSpaceTimeUnknowns, double** tempSpaceTimeFluxUnknowns,
    double* tempUnknowns, double* tempFluxUnknowns, double* tempStateSizedVectors,
    const double* luh, const double* dx, double dt, double* pointForceSources,
    int* picardIterations) {
  (void)tempStateSizedVectors;
  (void)pointForceSources;
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (!lQhbnd || !lFhbnd || !luh || !tempUnknowns || !tempFluxUnknowns)
    return set_error(EXA_EINVAL, "NULL buffer");
  const exa_aderdg_desc_t d = with_dx(desc, dx);
  const int B = d.order + 1, D = d.nvar + d.npar, V = d.nvar;
  const int nn = ipow_h(B, d.dim), nf = ipow_h(B, d.dim - 1);
  const size_t n_luh = nn * D, n_lqi = (size_t)nn * B * D, n_lfi = (size_t)nn * B * (d.dim + 1) * V;
  const size_t n_qhi = nn * D, n_fhi = (size_t)nn * (d.dim + 1) * V, n_lduh = nn * V;
  const size_t n_qb = 2 * d.dim * nf * D, n_fb = 2 * d.dim * nf * V;
  const size_t total = n_luh + n_lqi + n_lfi + n_qhi + n_fhi + n_lduh + n_qb + n_fb + 1;
  std::unique_lock<std::mutex> lk;
  double* w = nullptr;
  if (exa_status_t s = ws_get(total, &w, lk)) return s;
  double *wl = w, *wqi = wl + n_luh, *wfi = wqi + n_lqi, *wqhi = wfi + n_lfi, *wfhi = wqhi + n_qhi,
         *wdu = wfhi + n_fhi, *wqb = wdu + n_lduh, *wfb = wqb + n_qb;
  int* wit = (int*)(wfb + n_fb);
  cudaError_t e = cudaMemcpy(wl, luh, n_luh * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "copy luh");
  PredArgs a{};
  a.ncells = 1;
  a.luh = wl;
  a.dt = dt;
  a.dt_dev = nullptr;
  for (int i = 0; i < 3; i++) a.idx[i] = i < d.dim ? 1.0 / d.dx[i] : 0.0;
  a.lduh = wdu;
  a.lQhbnd = wqb;
  a.lFhbnd = wfb;
  a.iters = wit;
  a.stats = nullptr;
  a.lQi = wqi;
  a.lFi = wfi;
  a.lQhi = wqhi;
  a.lFhi = wfhi;
  a.precision = d.precision;
  if (exa_status_t s = launch_predictor(d, a, 1, 0)) return s;
  e = cudaMemcpy(lQhbnd, wqb, n_qb * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(lFhbnd, wfb, n_fb * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tempUnknowns, wqhi, n_qhi * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(tempFluxUnknowns, wfhi, n_fhi * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && tempSpaceTimeUnknowns && tempSpaceTimeUnknowns[0])
    e = cudaMemcpy(tempSpaceTimeUnknowns[0], wqi, n_lqi * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && tempSpaceTimeFluxUnknowns && tempSpaceTimeFluxUnknowns[0])
    e = cudaMemcpy(tempSpaceTimeFluxUnknowns[0], wfi, n_lfi * sizeof(double), cudaMemcpyDeviceToHost);
  int it = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&it, wit, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "copy predictor outputs");
  if (picardIterations) *picardIterations = it;
  return EXA_OK;
}

exa_status_t exa_aderdg_volumeIntegral(const exa_aderdg_desc_t* desc, double* lduh,
                                       const double* lFhi, const double* dx) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (!lduh || !lFhi) return set_error(EXA_EINVAL, "NULL buffer");
  const exa_aderdg_desc_t d = with_dx(desc, dx);
  const int B = d.order + 1, nn = ipow_h(B, d.dim);
  HostArr arr[2] = {{nullptr, lduh, (size_t)nn * d.nvar}, {lFhi, nullptr, (size_t)nn * (d.dim + 1) * d.nvar}};
  return run_one_cell(arr, 2, [&](double** p) { return launch_volume_integral(d, 1, p[0], p[1], 0); });
}

exa_status_t exa_aderdg_surfaceIntegral(const exa_aderdg_desc_t* desc, double* lduh,
                                        const double* lFhbnd, const double* dx) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (!lduh || !lFhbnd) return set_error(EXA_EINVAL, "NULL buffer");
  const exa_aderdg_desc_t d = with_dx(desc, dx);
  const int B = d.order + 1, nn = ipow_h(B, d.dim), nf = ipow_h(B, d.dim - 1);
  HostArr arr[2] = {{lduh, lduh, (size_t)nn * d.nvar}, {lFhbnd, nullptr, (size_t)2 * d.dim * nf * d.nvar}};
  return run_one_cell(arr, 2, [&](double** p) { return launch_surface_integral(d, 1, p[0], p[1], 0); });
}

exa_status_t exa_aderdg_riemannSolver(const exa_aderdg_desc_t* desc, double* FL, double* FR,
                                      const double* QL, const double* QR,
                                      double* tempFaceUnknownsArray, double** tempStateSizedVectors,
                                      double** tempStateSizedSquareMatrices, double dt,
                                      int normalNonZeroIndex, int isBoundaryFace) {
  (void)tempFaceUnknownsArray;
  (void)tempStateSizedVectors;
  (void)tempStateSizedSquareMatrices;
  (void)dt;
  (void)isBoundaryFace;
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (!FL || !FR || !QL || !QR) return set_error(EXA_EINVAL, "NULL buffer");
  if (normalNonZeroIndex < 0 || normalNonZeroIndex >= desc->dim)
    return set_error(EXA_EINVAL, "normalNonZeroIndex out of range");
  const exa_aderdg_desc_t d = *desc;
  const int B = d.order + 1, nf = ipow_h(B, d.dim - 1), D = d.nvar + d.npar;
  // Build a two-cell face-block layout: cell 0 holds QL/FL in face slot
  // 2*dir+1, cell 1 holds QR/FR in face slot 2*dir.
  const int nface = 2 * d.dim;
  std::vector<double> qb((size_t)2 * nface * nf * D, 0.0), fb((size_t)2 * nface * nf * d.nvar, 0.0);
  const int dir = normalNonZeroIndex;
  std::memcpy(&qb[((0 * nface) + 2 * dir + 1) * nf * D], QL, sizeof(double) * nf * D);
  std::memcpy(&qb[((1 * nface) + 2 * dir) * nf * D], QR, sizeof(double) * nf * D);
  std::memcpy(&fb[((0 * nface) + 2 * dir + 1) * nf * d.nvar], FL, sizeof(double) * nf * d.nvar);
  std::memcpy(&fb[((1 * nface) + 2 * dir) * nf * d.nvar], FR, sizeof(double) * nf * d.nvar);
  int idx[3] = {0, 1, dir};
  double idxd[2];
  std::memcpy(idxd, idx, sizeof(idx));  // 12 bytes of ints in 2 doubles
  HostArr arr[3] = {{qb.data(), nullptr, qb.size()}, {fb.data(), fb.data(), fb.size()}, {idxd, nullptr, 2}};
  exa_status_t st = run_one_cell(arr, 3, [&](double** p) {
    const int* ip = (const int*)p[2];
    return launch_riemann_faces(d, 1, ip, ip + 1, ip + 2, p[0], p[1], 0);
  });
  if (st) return st;
  std::memcpy(FL, &fb[((0 * nface) + 2 * dir + 1) * nf * d.nvar], sizeof(double) * nf * d.nvar);
  std::memcpy(FR, &fb[((1 * nface) + 2 * dir) * nf * d.nvar], sizeof(double) * nf * d.nvar);
  return EXA_OK;
}

exa_status_t exa_aderdg_solutionUpdate(const exa_aderdg_desc_t* desc, double* luh,
                                       const double* lduh, double dt) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (!luh || !lduh) return set_error(EXA_EINVAL, "NULL buffer");
  const exa_aderdg_desc_t d = *desc;
  const int B = d.order + 1, nn = ipow_h(B, d.dim);
  HostArr arr[2] = {{luh, luh, (size_t)nn * (d.nvar + d.npar)}, {lduh, nullptr, (size_t)nn * d.nvar}};
  return run_one_cell(arr, 2, [&](double** p) { return launch_solution_update(d, 1, p[0], p[1], dt, 0); });
}

exa_status_t exa_aderdg_stableTimeStepSize(const exa_aderdg_desc_t* desc, const double* luh,
                                           double* tempEigenvalues, const double* dx,
                                           double* dt_out) {
  (void)tempEigenvalues;
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (!luh || !dt_out) return set_error(EXA_EINVAL, "NULL buffer");
  const exa_aderdg_desc_t d = with_dx(desc, dx);
  const int B = d.order + 1, nn = ipow_h(B, d.dim);
  HostArr arr[2] = {{luh, nullptr, (size_t)nn * (d.nvar + d.npar)}, {nullptr, dt_out, 1}};
  const double factor = 0.9 * host_pnpm(d.order);
  return run_one_cell(arr, 2, [&](double** p) {
    return launch_stable_dt(d, 1, p[0], factor, p[1], nullptr, 0);
  });
}

// ------------------------------------------------ batched device API
exa_status_t exa_aderdg_predictor_vi(const exa_aderdg_desc_t* desc, long ncells, const double* luh,
                                     double dt, const double* dt_dev, double* lduh,
                                     double* lQhbnd, double* lFhbnd, int* picard_iters,
                                     uint64_t* stats, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (desc->npar != 0) return set_error(EXA_EINVAL, "batched predictor: npar must be 0");
  if (ncells < 0 || !luh || !lduh || !lQhbnd || !lFhbnd) return set_error(EXA_EINVAL, "bad argument");
  PredArgs a{};
  a.ncells = ncells;
  a.luh = luh;
  a.dt = dt;
  a.dt_dev = dt_dev;
  for (int i = 0; i < 3; i++) a.idx[i] = i < desc->dim ? 1.0 / desc->dx[i] : 0.0;
  a.lduh = lduh;
  a.lQhbnd = lQhbnd;
  a.lFhbnd = lFhbnd;
  a.iters = picard_iters;
  a.stats = (unsigned long long*)stats;
  a.precision = desc->precision;
  return launch_predictor(*desc, a, 0, as_stream(stream));
}

exa_status_t exa_aderdg_predictor_full(const exa_aderdg_desc_t* desc, long ncells, const double* luh,
                                       double dt, double* lQi, double* lFi, double* lQhi,
                                       double* lFhi, double* lduh, double* lQhbnd, double* lFhbnd,
                                       int* picard_iters, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (ncells < 0 || !luh || !lQi || !lFi || !lQhi || !lFhi || !lduh || !lQhbnd || !lFhbnd)
    return set_error(EXA_EINVAL, "bad argument");
  PredArgs a{};
  a.ncells = ncells;
  a.luh = luh;
  a.dt = dt;
  for (int i = 0; i < 3; i++) a.idx[i] = i < desc->dim ? 1.0 / desc->dx[i] : 0.0;
  a.lduh = lduh;
  a.lQhbnd = lQhbnd;
  a.lFhbnd = lFhbnd;
  a.iters = picard_iters;
  a.lQi = lQi;
  a.lFi = lFi;
  a.lQhi = lQhi;
  a.lFhi = lFhi;
  a.precision = desc->precision;
  return launch_predictor(*desc, a, 1, as_stream(stream));
}

exa_status_t exa_aderdg_volume_integral(const exa_aderdg_desc_t* desc, long ncells, double* lduh,
                                        const double* lFhi, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (ncells < 0 || !lduh || !lFhi) return set_error(EXA_EINVAL, "bad argument");
  return launch_volume_integral(*desc, ncells, lduh, lFhi, as_stream(stream));
}

exa_status_t exa_aderdg_surface_integral(const exa_aderdg_desc_t* desc, long ncells, double* lduh,
                                         const double* lFhbnd, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (ncells < 0 || !lduh || !lFhbnd) return set_error(EXA_EINVAL, "bad argument");
  return launch_surface_integral(*desc, ncells, lduh, lFhbnd, as_stream(stream));
}

exa_status_t exa_aderdg_solution_update(const exa_aderdg_desc_t* desc, long ncells, double* luh,
                                        const double* lduh, double dt, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (ncells < 0 || !luh || !lduh) return set_error(EXA_EINVAL, "bad argument");
  return launch_solution_update(*desc, ncells, luh, lduh, dt, as_stream(stream));
}

exa_status_t exa_aderdg_riemann_faces(const exa_aderdg_desc_t* desc, long nfaces, const int* left,
                                      const int* right, const int* dir, const double* lQhbnd,
                                      double* lFhbnd, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (nfaces < 0 || !left || !right || !dir || !lQhbnd || !lFhbnd)
    return set_error(EXA_EINVAL, "bad argument");
  return launch_riemann_faces(*desc, nfaces, left, right, dir, lQhbnd, lFhbnd, as_stream(stream));
}

exa_status_t exa_aderdg_stable_dt(const exa_aderdg_desc_t* desc, long ncells, const double* luh,
                                  double* dt_cell, double* dt_min, void* stream) {
  if (exa_status_t s = check_aderdg(desc)) return s;
  if (ncells < 0 || !luh) return set_error(EXA_EINVAL, "bad argument");
  cudaStream_t st = as_stream(stream);
  if (dt_min) {
    const unsigned long long inf = 0x7FF0000000000000ULL;
    cudaError_t e = cudaMemcpyAsync(dt_min, &inf, 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "dt_min init");
    e = cudaStreamSynchronize(st);  // the host source must stay alive
    if (e != cudaSuccess) return cuda_status(e, "dt_min init");
  }
  return launch_stable_dt(*desc, ncells, luh, 0.9 * host_pnpm(desc->order), dt_cell,
                          (unsigned long long*)dt_min, st);
}

// solutionAdjustment for one cell through the drop-in workspace (no
// allocation per call): luh and the center in, luh out
exa_status_t exa_aderdg_solutionAdjustment(int dim, int order, double* luh, const double* center,
                                           const double* dx, double t, double dt, const exa_adjust_t* hook) {
  if ((dim != 2 && dim != 3) || order < 1 || order > kMaxOrder || !luh || !center || !dx || !hook)
    return set_error(EXA_EINVAL, "bad argument");
  exa_aderdg_desc_t desc{};
  desc.dim = dim;
  desc.order = order;
  desc.nvar = kV;
  for (int d = 0; d < dim; d++) desc.dx[d] = dx[d];
  const size_t nn = (size_t)ipow_h(order + 1, dim) * kV;
  HostArr arr[2] = {{luh, luh, nn}, {center, nullptr, (size_t)dim}};
  return run_one_cell(arr, 2, [&](double** p) {
    exa_status_t s = exa_aderdg_solution_adjustment(&desc, 1, p[0], p[1], t, dt, hook, nullptr);
    if (s == EXA_OK) s = cuda_status(cudaDeviceSynchronize(), "solutionAdjustment");
    return s;
  });
}

exa_status_t exa_fv_rusanov(int dim, int nvar, int npar, int pde, double* fL, double* fR,
                            const double* qL, const double* qR, int normalNonZero, double* s_max) {
  if ((dim != 2 && dim != 3) || nvar != kV || npar < 0 || npar > 8 || !fL || !fR || !qL || !qR)
    return set_error(EXA_EINVAL, "bad argument");
  if (normalNonZero < 0 || normalNonZero >= dim) return set_error(EXA_EINVAL, "bad direction");
  if (exa_status_t s = ensure_tables()) return s;
  double out[kV + 1];
  HostArr arr[3] = {{qL, nullptr, (size_t)(nvar + npar)}, {qR, nullptr, (size_t)(nvar + npar)},
                    {nullptr, out, (size_t)kV + 1}};
  exa_status_t st = run_one_cell(arr, 3, [&](double** p) {
    return launch_rusanov_one(pde, normalNonZero, p[0], p[1], p[2]);
  });
  if (st) return st;
  for (int i = 0; i < nvar; i++) fL[i] = fR[i] = out[i];
  if (s_max) *s_max = out[kV];
  return EXA_OK;
}

}  // extern "C"

// ------------------------------------------------ limiter: per-cell drop-ins
// kernels::limiter::generic::c (Limiter.cpp) argument lists on HOST
// pointers for one cell, run through the batched device kernels.
extern "C" {

static long lim_points(int dim, int n) { return dim == 3 ? (long)n * n * n : (long)n * n; }

exa_status_t exa_limiter_projectOnFVLimiterSpace(int dim, const double* luh, int numberOfVariables,
                                                 int basisSize, int ghostLayerWidth, double* lim) {
  if (!luh || !lim || (dim != 2 && dim != 3) || basisSize < 2 || ghostLayerWidth < 0 || numberOfVariables < 1)
    return set_error(EXA_EINVAL, "projectOnFVLimiterSpace: bad arguments");
  const int S = 2 * basisSize - 1, SG = S + 2 * ghostLayerWidth;
  HostArr arr[2] = {{luh, nullptr, (size_t)(lim_points(dim, basisSize) * numberOfVariables)},
                    {lim, lim, (size_t)(lim_points(dim, SG) * numberOfVariables)}};
  return run_one_cell(arr, 2, [&](double** p) {
    return exa_limiter_project_on_fv(dim, basisSize - 1, numberOfVariables, ghostLayerWidth, 1, p[0], p[1],
                                     nullptr);
  });
}

exa_status_t exa_limiter_projectOnDGSpace(int dim, const double* lim, int numberOfVariables, int basisSize,
                                          int ghostLayerWidth, double* luh) {
  if (!luh || !lim || (dim != 2 && dim != 3) || basisSize < 2 || ghostLayerWidth < 0 || numberOfVariables < 1)
    return set_error(EXA_EINVAL, "projectOnDGSpace: bad arguments");
  const int S = 2 * basisSize - 1, SG = S + 2 * ghostLayerWidth;
  HostArr arr[2] = {{lim, nullptr, (size_t)(lim_points(dim, SG) * numberOfVariables)},
                    {nullptr, luh, (size_t)(lim_points(dim, basisSize) * numberOfVariables)}};
  return run_one_cell(arr, 2, [&](double** p) {
    return exa_limiter_project_on_dg(dim, basisSize - 1, numberOfVariables, ghostLayerWidth, 1, p[0], p[1],
                                     nullptr);
  });
}

exa_status_t exa_limiter_findCellLocalMinAndMax(int dim, const double* luh, int numberOfVariables,
                                                int basisSize, int numberOfObservables,
                                                double* localMinPerObservable, double* localMaxPerObservable) {
  if (!luh || !localMinPerObservable || !localMaxPerObservable || (dim != 2 && dim != 3) || basisSize < 2 ||
      numberOfObservables < 1 || numberOfObservables > numberOfVariables)
    return set_error(EXA_EINVAL, "findCellLocalMinAndMax: bad arguments");
  // the reference writes numberOfObservables values; the batched kernel
  // fills all 2 dim face blocks, of which the first is returned
  const size_t nb = (size_t)2 * dim * numberOfObservables;
  std::vector<double> mn(nb), mx(nb);
  HostArr arr[3] = {{luh, nullptr, (size_t)(lim_points(dim, basisSize) * numberOfVariables)},
                    {nullptr, mn.data(), nb},
                    {nullptr, mx.data(), nb}};
  exa_status_t s = run_one_cell(arr, 3, [&](double** p) {
    return exa_limiter_local_min_max(dim, basisSize - 1, numberOfVariables, numberOfObservables, 1, p[0], p[1], p[2],
                                     nullptr);
  });
  if (s) return s;
  std::copy_n(mn.data(), numberOfObservables, localMinPerObservable);
  std::copy_n(mx.data(), numberOfObservables, localMaxPerObservable);
  return EXA_OK;
}

exa_status_t exa_limiter_discreteMaximumPrincipleAndMinAndMaxSearch(
    int dim, const double* luh, int numberOfVariables, int basisSize, int numberOfObservables,
    double relaxationParameter, double differenceScaling, double* boundaryMinPerObservable,
    double* boundaryMaxPerObservable, int* discreteMaximumPrincipleSatisfied) {
  if (!luh || !boundaryMinPerObservable || !boundaryMaxPerObservable || !discreteMaximumPrincipleSatisfied ||
      (dim != 2 && dim != 3) || basisSize < 2 || numberOfObservables < 1 || numberOfObservables > numberOfVariables)
    return set_error(EXA_EINVAL, "discreteMaximumPrincipleAndMinAndMaxSearch: bad arguments");
  const size_t nb = (size_t)2 * dim * numberOfObservables;
  double verdict = 0.0;  // device int in a double-sized slot
  HostArr arr[4] = {{luh, nullptr, (size_t)(lim_points(dim, basisSize) * numberOfVariables)},
                    {boundaryMinPerObservable, boundaryMinPerObservable, nb},
                    {boundaryMaxPerObservable, boundaryMaxPerObservable, nb},
                    {nullptr, &verdict, 1}};
  exa_status_t s = run_one_cell(arr, 4, [&](double** p) {
    return exa_limiter_dmp(dim, basisSize - 1, numberOfVariables, numberOfObservables, 1, p[0],
                           relaxationParameter, differenceScaling, p[1], p[2], reinterpret_cast<int*>(p[3]),
                           nullptr);
  });
  if (s) return s;
  int ok = 0;
  std::memcpy(&ok, &verdict, sizeof(int));
  *discreteMaximumPrincipleSatisfied = ok;
  return EXA_OK;
}

}  // extern "C"
