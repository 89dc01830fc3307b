// 3D finite volumes on batches of patches: the reference's
//   godunov::c::solutionUpdate      (kernels/finitevolumes/godunov/c/3d/godunov.cpph:35-143)
//   musclhancock::c::solutionUpdate (kernels/finitevolumes/musclhancock/c/3d/musclhancock.cpph:50-311)
//   commons::c::stableTimeStepSize  (kernels/finitevolumes/commons/c/commons.cpph:410-455)
// with Rusanov face fluxes (riemannsolvers/c/rusanov.cpph:98-156) for the
// 3D Euler equations.  One CTA per patch: the patch with its ghost layers is
// staged in shared memory; MUSCL-Hancock first stores the half-step
// increment of every interior cell; then every interior cell evaluates its
// own six face fluxes (each interior face twice, once per side) and applies
// them in the reference's order (x faces, then y, then z; the lower face
// before the upper).  As in the reference, the contributions of the
// patch-boundary faces also reach the first ghost layer of the output, and
// the MUSCL ring cells next to the patch are not half-step evolved.
#include <cfloat>

#include "exa_device.cuh"

namespace exa {

// threads per CTA: MUSCL-Hancock's staging (117 KB for 9^3 patches) leaves
// one CTA per SM, so it runs 512 threads; Godunov fits several 256-thread CTAs
template <int SCHEME>
struct FV3Threads {
  static constexpr int value = SCHEME == 1 ? 512 : 256;
};

struct FV3Args {
  int P, g, S, D;
  double h[3];              // cell sizes
  double dt;                // used when dt_dev is null
  const double* dt_dev;
  const double* luh;        // state the fluxes are computed from
  double* out;              // luh_new (a copy of luh on entry), updated in place
  unsigned long long* max_dt;  // per patch admissible dt (atomic min), nullable
  const int* list;          // optional patch selection: list[0 .. *count)
  const int* count;
};

__device__ __forceinline__ double fv3_minmod(double a, double b) {
  if (a * b < 0.0) return 0.0;
  return fabs(a) < fabs(b) ? a : b;
}

// Rusanov flux of the face between qL and qR in direction d; returns s_max
__device__ __forceinline__ double fv3_rusanov(const double* qL, const double* qR, int d, double* f) {
  const double sL = euler_max_eig<false>(qL, d), sR = euler_max_eig<false>(qR, d);
  const double smax = fmax(sL, sR);
  double FL[3][kV], FR[3][kV];
  euler_flux<3, false>(qL, FL);
  euler_flux<3, false>(qR, FR);
#pragma unroll
  for (int i = 0; i < kV; i++) {
    double v = 0.5 * smax * (qL[i] - qR[i]);
    v += 0.5 * (FL[d][i] + FR[d][i]);
    f[i] = v;
  }
  return smax;
}

// MUSCL face value of cell (i, j, k) in direction d, side -1 (lower face,
// wL) or +1 (upper, wR): u -/+ h/2 slope, plus the half step for interior
// cells
__device__ __forceinline__ void fv3_face_value(const double* su, const double* qt, int S, int P, int g, const double* h,
                                               const double* ih, double dt, int i, int j, int k, int d, int side,
                                               double* w) {
  const int st = d == 0 ? 1 : (d == 1 ? S : S * S);
  const double* u = su + (((long)i * S + j) * S + k) * kV;
  const bool interior = i >= g && i < g + P && j >= g && j < g + P && k >= g && k < g + P;
#pragma unroll
  for (int m = 0; m < kV; m++) {
    const double sl = fv3_minmod(u[st * kV + m] - u[m], u[m] - u[-st * kV + m]) * ih[d];
    double v = side < 0 ? u[m] - 0.5 * h[d] * sl : u[m] + 0.5 * h[d] * sl;
    if (interior) v += 0.5 * dt * qt[(((long)(i - g) * P + (j - g)) * P + (k - g)) * kV + m];
    w[m] = v;
  }
}

template <int SCHEME>
__global__ void __launch_bounds__(FV3Threads<SCHEME>::value) k_fv3_patch(FV3Args a) {
  constexpr int V = kV;
  constexpr int FV3_NT = FV3Threads<SCHEME>::value;
  extern __shared__ double sm[];
  __shared__ double sred[FV3_NT / 32];
  const int P = a.P, g = a.g, S = a.S, D = a.D;
  const long S3 = (long)S * S * S;
  double* su = sm;         // [S^3][V]
  double* qt = su + S3 * V;  // [P^3][V] (MUSCL)
  const int tid = threadIdx.x;
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;
  const double cfl = SCHEME == 0 ? 0.9 : 0.99;
  // reciprocal cell sizes: multiplications instead of the reference's
  // divisions in the slopes and half-step increments
  const double ihs[3] = {1.0 / a.h[0], 1.0 / a.h[1], 1.0 / a.h[2]};
  const long npatch = a.count ? (long)*a.count : (long)gridDim.x;
  for (long e = blockIdx.x; e < npatch; e += gridDim.x) {
    const long patch = a.list ? (long)a.list[e] : e;
    const double* luh = a.luh + patch * S3 * D;
    double* out = a.out + patch * S3 * D;
    for (long i = tid; i < S3 * V; i += FV3_NT) su[i] = luh[(i / V) * D + i % V];
    __syncthreads();
    if (SCHEME == 1) {
      // half-step increment of the interior cells (musclhancock.cpph:152-205)
      for (int c = tid; c < P * P * P; c += FV3_NT) {
        const int i = g + c / (P * P), j = g + (c / P) % P, k = g + c % P;
        double Qt[V];
#pragma unroll
        for (int m = 0; m < V; m++) Qt[m] = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const int st = d == 0 ? 1 : (d == 1 ? S : S * S);
          const double* u = su + (((long)i * S + j) * S + k) * V;
          double wl[V], wr[V], F[3][V];
#pragma unroll
          for (int m = 0; m < V; m++) {
            const double sl = fv3_minmod(u[st * V + m] - u[m], u[m] - u[-st * V + m]) * ihs[d];
            wl[m] = u[m] - 0.5 * a.h[d] * sl;
            wr[m] = u[m] + 0.5 * a.h[d] * sl;
          }
          euler_flux<3, false>(wl, F);
#pragma unroll
          for (int m = 0; m < V; m++) Qt[m] += F[d][m] * ihs[d];
          euler_flux<3, false>(wr, F);
#pragma unroll
          for (int m = 0; m < V; m++) Qt[m] -= F[d][m] * ihs[d];
        }
#pragma unroll
        for (int m = 0; m < V; m++) qt[(long)c * V + m] = Qt[m];
      }
      __syncthreads();
    }
    double dtl = DBL_MAX;
    for (int c = tid; c < P * P * P; c += FV3_NT) {
      const int i = g + c / (P * P), j = g + (c / P) % P, k = g + c % P;
      double fl[3][V], fr[3][V];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int di = d == 2, dj = d == 1, dk = d == 0;
        double sl, sr;
        if (SCHEME == 0) {
          const double* uc = su + (((long)i * S + j) * S + k) * V;
          const double* ul = su + (((long)(i - di) * S + (j - dj)) * S + (k - dk)) * V;
          const double* ur = su + (((long)(i + di) * S + (j + dj)) * S + (k + dk)) * V;
          sl = fv3_rusanov(ul, uc, d, fl[d]);
          sr = fv3_rusanov(uc, ur, d, fr[d]);
        } else {
          double wa[V], wb[V];
          fv3_face_value(su, qt, S, P, g, a.h, ihs, dt, i - di, j - dj, k - dk, d, +1, wa);
          fv3_face_value(su, qt, S, P, g, a.h, ihs, dt, i, j, k, d, -1, wb);
          sl = fv3_rusanov(wa, wb, d, fl[d]);
          fv3_face_value(su, qt, S, P, g, a.h, ihs, dt, i, j, k, d, +1, wa);
          fv3_face_value(su, qt, S, P, g, a.h, ihs, dt, i + di, j + dj, k + dk, d, -1, wb);
          sr = fv3_rusanov(wa, wb, d, fr[d]);
        }
        // min of c / s over the two faces = c / max of s (division is
        // monotone): one division instead of two, the same value
        dtl = fmin(dtl, cfl / 3 * a.h[d] / fmax(sl, sr));
      }
      const double c0 = dt / a.h[0], c1 = dt / a.h[1], c2 = dt / a.h[2];
      double* o = out + (((long)i * S + j) * S + k) * D;
#pragma unroll
      for (int m = 0; m < V; m++) {
        double v = o[m];
        v += c0 * fl[0][m];
        v -= c0 * fr[0][m];
        v += c1 * fl[1][m];
        v -= c1 * fr[1][m];
        v += c2 * fl[2][m];
        v -= c2 * fr[2][m];
        o[m] = v;
      }
      // the patch-boundary faces also update the first ghost layer
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int cd = d == 0 ? k : (d == 1 ? j : i);
        const double cc = d == 0 ? c0 : (d == 1 ? c1 : c2);
        const long st = d == 0 ? 1 : (d == 1 ? S : (long)S * S);
        if (cd == g) {
          double* q = o - st * D;
#pragma unroll
          for (int m = 0; m < V; m++) q[m] -= cc * fl[d][m];
        }
        if (cd == g + P - 1) {
          double* q = o + st * D;
#pragma unroll
          for (int m = 0; m < V; m++) q[m] += cc * fr[d][m];
        }
      }
    }
    if (a.max_dt) {
      for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
      if ((tid & 31) == 0) sred[tid >> 5] = dtl;
      __syncthreads();
      if (tid == 0) {
        double m = sred[0];
        for (int w = 1; w < FV3_NT / 32; w++) m = fmin(m, sred[w]);
        atomic_min_pos_double(&a.max_dt[patch], m);
      }
    }
    __syncthreads();
  }
}

// commons::stableTimeStepSize per patch (CFL 0.9 / 3)
__global__ void k_fv3_stable_dt(int P, int g, int D, double h0, double h1, double h2, const double* luh,
                                double* dt_patch) {
  const int S = P + 2 * g;
  const long patch = blockIdx.y;
  const double* u = luh + patch * (long)S * S * S * D;
  double dtl = DBL_MAX;
  for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < (long)P * P * P; c += (long)gridDim.x * blockDim.x) {
    const int i = g + (int)(c / (P * P)), j = g + (int)((c / P) % P), k = g + (int)(c % P);
    const double* q = u + (((long)i * S + j) * S + k) * D;
    dtl = fmin(dtl, 0.9 / 3 * h0 / euler_max_eig<false>(q, 0));
    dtl = fmin(dtl, 0.9 / 3 * h1 / euler_max_eig<false>(q, 1));
    dtl = fmin(dtl, 0.9 / 3 * h2 / euler_max_eig<false>(q, 2));
  }
  for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
  if ((threadIdx.x & 31) == 0) atomic_min_pos_double((unsigned long long*)&dt_patch[patch], dtl);
}

// periodic ghost layers of every patch (corners included)
__global__ void k_fv3_ghosts(int P, int g, int D, long npatches, double* luh) {
  const int S = P + 2 * g;
  const long S3 = (long)S * S * S;
  for (long gid = (long)blockIdx.x * blockDim.x + threadIdx.x; gid < S3 * npatches;
       gid += (long)gridDim.x * blockDim.x) {
    const long patch = gid / S3;
    const long r = gid % S3;
    const int i = (int)(r / (S * S)), j = (int)((r / S) % S), k = (int)(r % S);
    const int si = g + ((i - g) % P + P) % P, sj = g + ((j - g) % P + P) % P, sk = g + ((k - g) % P + P) % P;
    if (si == i && sj == j && sk == k) continue;
    double* base = luh + patch * S3 * D;
    const double* src = base + (((long)si * S + sj) * S + sk) * D;
    double* dst = base + (((long)i * S + j) * S + k) * D;
    for (int m = 0; m < D; m++) dst[m] = src[m];
  }
}

size_t fv3_smem(int P, int g, int scheme) {
  const size_t S = P + 2 * g;
  return sizeof(double) * (S * S * S * kV + (scheme == 1 ? (size_t)P * P * P * kV : 0));
}

exa_status_t fv3_update(int scheme, int P, int g, int D, const double* h, long npatches, double* luh_new,
                        const double* luh, double dt, const double* dt_dev, double* max_dt, const int* list,
                        const int* count, cudaStream_t st) {
  const size_t smem = fv3_smem(P, g, scheme);
  if (smem > 200 * 1024) return set_error(EXA_EINVAL, "3D FV: patch too large for one CTA");
  FV3Args a{};
  a.P = P;
  a.g = g;
  a.S = P + 2 * g;
  a.D = D;
  for (int d = 0; d < 3; d++) a.h[d] = h[d];
  a.dt = dt;
  a.dt_dev = dt_dev;
  a.luh = luh;
  a.out = luh_new;
  a.max_dt = (unsigned long long*)max_dt;
  a.list = list;
  a.count = count;
  auto kern = scheme == 0 ? k_fv3_patch<0> : k_fv3_patch<1>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e, "3D FV attribute");
  long grid = npatches;
  if (count) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    grid = npatches < 4L * sms ? npatches : 4L * sms;  // CTAs loop over the listed patches
  }
  if (grid > 0x7fffffffL) return set_error(EXA_EINVAL, "3D FV: too many patches");
  kern<<<(unsigned)grid, scheme == 0 ? FV3Threads<0>::value : FV3Threads<1>::value, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv3_patch");
}

// face ghosts of the listed 3D subcell patches from the face neighbours'
// boundary layers (grid of n[0] x n[1] x n[2] cells, x fastest).  At a
// domain-boundary face (bc[d] != 0) the ghosts mirror the patch's own
// boundary layers, ghost layer k <- interior layer k counted from the face
// (FiniteVolumesSolver::mergeWithBoundaryData: boundaryLayerExtraction,
// boundaryConditions with its mirrored index K = g - 1 - k, and
// ghostLayerFillingAtBoundary, commons.cpph:502-875), the normal momentum
// negated for a reflecting wall.  Grid-stride over list entries x face
// ghosts.
__global__ void k_fv3_subcell_exchange(int P, int g, int nx, int ny, int nz, int3 bc, double* lim, const int* list,
                                       const int* count) {
  const int S = P + 2 * g;
  const long S3 = (long)S * S * S;
  const long per = 6L * g * P * P;  // face ghosts per patch
  const long total = (long)*count * per;
  for (long gid = (long)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (long)gridDim.x * blockDim.x) {
    const long patch = list[gid / per];
    int r = (int)(gid % per);
    const int f = r / (g * P * P);  // face 2 d + side
    r %= g * P * P;
    const int layer = r / (P * P), a = (r / P) % P, b = r % P;  // layer across, (a, b) along the face
    const int d = f >> 1;
    const bool up = f & 1;
    int x = (int)(patch % nx), y = (int)((patch / nx) % ny), z = (int)(patch / ((long)nx * ny));
    // destination (i, j, k) = (z, y, x) subcell in this patch, source in the neighbour
    int di[3], si[3];  // [z][y][x] coordinates
    const int ghost = up ? g + P + layer : layer;        // ghost coordinate along d
    const int src = up ? g + layer : P + layer;           // neighbour's boundary layer
    const int ax = 2 - d;                                 // coordinate index of direction d in (z, y, x)
    const int o1 = ax == 0 ? 1 : 0, o2 = ax == 2 ? 1 : 2;  // the two other coordinates
    di[ax] = ghost;
    si[ax] = src;
    di[o1] = si[o1] = g + a;
    di[o2] = si[o2] = g + b;
    int* p = d == 0 ? &x : (d == 1 ? &y : &z);
    const int n = d == 0 ? nx : (d == 1 ? ny : nz);
    const int rule = d == 0 ? bc.x : (d == 1 ? bc.y : bc.z);
    long nbp;
    if (rule != 0 && (up ? *p + 1 == n : *p == 0)) {
      nbp = patch;
      // lower y and z faces: every ghost layer repeats the layer next to the
      // face (the reference's 3D extraction reads patchBegin for every
      // layer there, commons.cpph:561 and 591)
      si[ax] = up ? g + P - 1 - layer : (d > 0 ? g : 2 * g - 1 - layer);
    } else {
      *p = up ? (*p + 1 == n ? 0 : *p + 1) : (*p == 0 ? n - 1 : *p - 1);
      nbp = ((long)z * ny + y) * nx + x;
    }
    const int flip = nbp == patch && rule == EXA_BC_REFLECT ? 1 + d : -1;
    double* dst = lim + patch * S3 * kV + (((long)di[0] * S + di[1]) * S + di[2]) * kV;
    const double* s = lim + nbp * S3 * kV + (((long)si[0] * S + si[1]) * S + si[2]) * kV;
#pragma unroll
    for (int m = 0; m < kV; m++) dst[m] = m == flip ? -s[m] : s[m];
  }
}

exa_status_t fv3_subcell_step(int scheme, int P, int g, const int* n, const double* h, double* lim, const int* list,
                              const int* count, long maxcells, const double* dt_dev, cudaStream_t st, const int* bc) {
  if ((scheme == 0 && g < 1) || (scheme == 1 && g < 2)) return set_error(EXA_EINVAL, "subcell FV: ghost layer too thin");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int3 rules = bc ? make_int3(bc[0], bc[1], bc[2]) : make_int3(0, 0, 0);
  k_fv3_subcell_exchange<<<(unsigned)(8 * sms), 256, 0, st>>>(P, g, n[0], n[1], n[2], rules, lim, list, count);
  count_launch();
  if (exa_status_t s = cuda_status(cudaGetLastError(), "k_fv3_subcell_exchange")) return s;
  // in place: each CTA stages its patch before it writes
  return fv3_update(scheme, P, g, kV, h, maxcells, lim, lim, 0.0, dt_dev, nullptr, list, count, st);
}

exa_status_t fv3_stable_dt(int P, int g, int D, const double* h, long npatches, const double* luh, double* dt_patch,
                           cudaStream_t st) {
  if (npatches > 65535) return set_error(EXA_EINVAL, "at most 65535 patches per call");
  const long cells = (long)P * P * P;
  unsigned bx = (unsigned)((cells + 255) / 256);
  if (bx > 1024) bx = 1024;
  k_fv3_stable_dt<<<dim3(bx, (unsigned)npatches), 256, 0, st>>>(P, g, D, h[0], h[1], h[2], luh, dt_patch);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv3_stable_dt");
}

exa_status_t fv3_periodic_ghosts(int P, int g, int D, long npatches, double* luh, cudaStream_t st) {
  const long S = P + 2 * g;
  const long work = S * S * S * npatches;
  long blocks = (work + 255) / 256;
  if (blocks > 65535) blocks = 65535;
  k_fv3_ghosts<<<(unsigned)blocks, 256, 0, st>>>(P, g, D, npatches, luh);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv3_ghosts");
}

}  // namespace exa
