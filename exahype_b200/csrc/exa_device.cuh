// Device-side building blocks shared by the ADER-DG and FV kernels:
// DG operator tables in constant memory, the compressible Euler PDE, and
// block/segment reductions.  sm_100a only.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "exa_internal.h"

namespace exa {

constexpr int kMaxOrder = 9;
constexpr int kV = 5;  // Euler: rho, j_x, j_y, j_z, E
constexpr double kGamma = 1.4;

// Operator tables for one order N (B = N+1 nodes on [0,1]).  All derived
// on the host in double from the generated dg_tables.h (see tables.cpp).
struct DGConst {
  double w[10];         // Gauss-Legendre weights
  double nodes[10];     // Gauss-Legendre nodes on [0,1]
  double kxi[10][10];   // Kxi[k][m]   (reference DGMatrices.h:47-52)
  double deriv[10][10]; // Kxi[p][l] / w_l  -> derivative onto node l
  double tA[10][10];    // iK1[t][n] * w_n  (Picard time contraction)
  double c0[10];        // sum_n iK1[t][n] F0[n]
  double fl[10];        // FLCoeff
  double fr[10];        // FRCoeff
  double pnpm;          // CFL safety factor of order N
};

// Every translation unit gets its own copy (internal linkage); the host
// uploads the same bytes into each (exa::upload_tables_*).
static __constant__ DGConst c_dg[kMaxOrder + 1];

// FP32 copies (rounded from the FP64 tables) for the mixed-precision Picard
// loop, so its FMAs take constant-bank operands without conversions.
struct DGConstF {
  float w[10];
  float deriv[10][10];
  float derivT[10][10];  // derivT[p][l] = deriv[l][p] (pairs of outputs adjacent)
  float tA[10][10];
};
static __constant__ DGConstF c_dgf[kMaxOrder + 1];

// ------------------------------------------------------------------ PDE
// Compressible Euler, gamma = 1.4.  PLANAR selects the "2.5D" pressure
// p = (g-1)(E - (j_x^2+j_y^2)/(2 rho)) of the reference's 2D kernel tests
// (exahype/tests/kernels/c/GenericEulerKernelTest2D.cpp:28-79); otherwise
// all three momenta enter (GenericEulerKernelTest3D.cpp:26-82).
template <bool PLANAR>
__device__ __forceinline__ double euler_pressure(const double* q, double irho) {
  const double j2 = PLANAR ? (q[1] * q[1] + q[2] * q[2])
                           : (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  return (kGamma - 1.0) * (q[4] - 0.5 * j2 * irho);
}

// Flux in DIM directions: F[d][m].
template <int DIM, bool PLANAR>
__device__ __forceinline__ void euler_flux(const double* q, double (*F)[kV]) {
  const double irho = 1.0 / q[0];
  const double p = euler_pressure<PLANAR>(q, irho);
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    const double jn = q[d + 1];
    const double ij = irho * jn;
    F[d][0] = jn;
    F[d][1] = ij * q[1];
    F[d][2] = ij * q[2];
    F[d][3] = ij * q[3];
    F[d][d + 1] += p;
    F[d][4] = ij * (q[4] + p);
  }
}

// max |lambda| in direction d: |u_n| + c  (eigenvalues u_n-c, u_n x3, u_n+c)
template <bool PLANAR>
__device__ __forceinline__ double euler_max_eig(const double* q, int d) {
  const double irho = 1.0 / q[0];
  const double p = euler_pressure<PLANAR>(q, irho);
  const double un = q[d + 1] * irho;
  const double c = sqrt(kGamma * p * irho);
  return fmax(fabs(un - c), fmax(fabs(un), fabs(un + c)));
}

// ------------------------------------------------------ async copies
// 8-byte global -> shared copy that completes asynchronously (cp.async,
// sm_80+), and the wait for all of this thread's outstanding copies.
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// ------------------------------------------------------------ reductions
// Sum over groups of G consecutive threads (G a power of two <= 32, or a
// multiple of 32).  Every thread of a group returns the bitwise identical
// sum (xor butterflies add commutative pairs; the cross-warp step is read
// by all threads in the same order).  sred needs NT/32 doubles.
template <int G>
__device__ __forceinline__ double group_sum(double v, double* sred) {
  constexpr int L = G < 32 ? G : 32;
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if constexpr (G <= 32) {
    return v;
  } else {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sred[warp] = v;
    __syncthreads();
    const int g0 = (threadIdx.x / G) * (G / 32);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < G / 32; k++) s += sred[g0 + k];
    return s;
  }
}

// group_sum with one barrier, for a loop that calls it once per iteration:
// the warp partials go to one of two slot sets chosen by the iteration's
// parity, so the next iteration's writes never meet this iteration's reads
// (every thread passes this barrier before any thread writes again).  sred
// needs 2 NT/32 doubles.  Same summation order, so the same bits as
// group_sum.
template <int G, int NT>
__device__ __forceinline__ double group_sum_1b(double v, double* sred, int parity) {
  constexpr int L = G < 32 ? G : 32;
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if constexpr (G <= 32) {
    return v;
  } else {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* slot = sred + (parity & 1) * (NT / 32);
    if (lane == 0) slot[warp] = v;
    __syncthreads();
    const int g0 = (threadIdx.x / G) * (G / 32);
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < G / 32; k++) s += slot[g0 + k];
    return s;
  }
}

template <int G>
__device__ __forceinline__ double group_min(double v, double* sred) {
  constexpr int L = G < 32 ? G : 32;
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  if constexpr (G <= 32) {
    return v;
  } else {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sred[warp] = v;
    __syncthreads();
    const int g0 = (threadIdx.x / G) * (G / 32);
    double s = sred[g0];
#pragma unroll
    for (int k = 1; k < G / 32; k++) s = fmin(s, sred[g0 + k]);
    return s;
  }
}

// atomic min on a non-negative double stored as its bit pattern
__device__ __forceinline__ void atomic_min_pos_double(unsigned long long* addr, double v) {
  if (v >= 0.0) atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

constexpr int next_pow2(int x) { int p = 1; while (p < x) p <<= 1; return p; }
constexpr int round_up(int x, int m) { return (x + m - 1) / m * m; }
constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

// Threads per cell: next power of two for small cells, whole warps above.
template <int NPC>
struct CellThreads {
  static constexpr int G = NPC <= 32 ? next_pow2(NPC) : round_up(NPC, 32);
};

}  // namespace exa
