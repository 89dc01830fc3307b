// Mixed-precision predictor body (see aderdg_predictor_mixed.cu for the
// design notes); shared by k_predictor_mixed and the ensemble kernel.
#pragma once
#include "exa_device.cuh"

namespace exa {

template <int DIM, int N>
struct MixShape {
  static constexpr int B = N + 1;
  static constexpr int V = kV;
  static constexpr int NPC = ipow(B, DIM);
  static constexpr int NF = ipow(B, DIM - 1);
  static constexpr int G = CellThreads<NPC>::G;
  static constexpr int CPB = DIM == 3 ? 1 : (128 / G > 0 ? 128 / G : 1);
  static constexpr int NT = G * CPB;
  // per cell, in doubles: max(two FP32 slice buffers, FP64 staging of the
  // time-averaged flux [DIM][NPC][V] + state [NPC][V])
  static constexpr int SLICE_F = DIM * NPC * V;  // floats per slice
  static constexpr int STAGE_D = (DIM + 1) * NPC * V;
  static constexpr int SM_CELL = SLICE_F > STAGE_D ? SLICE_F : STAGE_D;  // 2 float slices = SLICE_F doubles
  static constexpr int SM_DOUBLES = CPB * SM_CELL + NT / 32 + 1;
};

// MINB: minimum resident CTAs per SM requested from the register
// allocator (1 = unconstrained; 3 trades a small spill for occupancy).
template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void predictor_mixed_block(const PredArgs& a, long block, double* smem) {
  using S = MixShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];

  const int lc = threadIdx.x / G;
  const int s = threadIdx.x % G;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  double* sD = smem + lc * S::SM_CELL;       // FP64 staging [DIM][NPC][V] + [NPC][V]
  float* sFf = reinterpret_cast<float*>(sD);  // two FP32 slices [2][DIM][NPC][V]
  double* sQh = sD + DIM * NPC * V;
  double* sred = smem + S::CPB * S::SM_CELL;

  int sd[3];
  sd[0] = s % B;
  sd[1] = (s / B) % B;
  sd[2] = DIM == 3 ? s / (B * B) : 0;
  const int stride[3] = {1, B, B * B};

  double lu[V];
  const double* luh = a.luh + cell * (long)NPC * V;
#pragma unroll
  for (int m = 0; m < V; m++) lu[m] = active ? luh[s * V + m] : (m == 0 ? 1.0 : (m == 4 ? 2.5 : 0.0));
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;

  // base flux F0 = F(luh) and its derivative G0 (FP64, once per cell)
  double F0[DIM][V];
  euler_flux<DIM, PLANAR>(lu, F0);
  if (active)
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sD[(d * NPC + s) * V + m] = F0[d][m];
  __syncthreads();
  double G0[V];
#pragma unroll
  for (int m = 0; m < V; m++) G0[m] = 0.0;
  if (active) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const double* line = sD + (d * NPC + s - sd[d] * stride[d]) * V;
#pragma unroll
      for (int p = 0; p < B; p++) {
        const double c = T.deriv[sd[d]][p] * a.idx[d];
#pragma unroll
        for (int m = 0; m < V; m++) G0[m] += c * line[p * stride[d] * V + m];
      }
    }
  }
  __syncthreads();  // staging area is reused for the FP32 slices

  float dcf[DIM][B];
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int p = 0; p < B; p++) dcf[d][p] = active ? (float)(T.deriv[sd[d]][p] * a.idx[d]) : 0.f;

  // First Picard deviation (all time nodes share luh, so F = F0 and the
  // FP64 part of every iterate is the same):
  //   base[t] = (c0[t] - 1) luh - dt (sum_n tA[t][n]) D.F0
  // kept in FP32 (an O(dt) quantity); an iterate is dq = base - dt acc.
  float base[B][V];
#pragma unroll
  for (int t = 0; t < B; t++) {
    double tas = 0.0;
#pragma unroll
    for (int n = 0; n < B; n++) tas += T.tA[t][n];
#pragma unroll
    for (int m = 0; m < V; m++) base[t][m] = (float)((T.c0[t] - 1.0) * lu[m] - dt * tas * G0[m]);
  }
  const float dtf = (float)dt;

  float dq[B][V];
#pragma unroll
  for (int t = 0; t < B; t++)
#pragma unroll
    for (int m = 0; m < V; m++) dq[t][m] = 0.f;

  // FP64 flux of time slice n from luh + dq[n], returned as the FP32 deviation
  auto slice_flux = [&](int n, float (*dF)[V]) {
    double qq[V], F[DIM][V];
#pragma unroll
    for (int m = 0; m < V; m++) qq[m] = lu[m] + (double)dq[n][m];
    euler_flux<DIM, PLANAR>(qq, F);
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) dF[d][m] = (float)(F[d][m] - F0[d][m]);
  };

  constexpr bool kShared = S::CPB > 1;
  float fhd[DIM][V];
  int it = 0;
  bool conv = false;
  int buf = 0;  // slice buffer parity, alternates every slice
  for (int iter = 0; iter < MAXIT; iter++) {
    float acc[B][V];
#pragma unroll
    for (int t = 0; t < B; t++)
#pragma unroll
      for (int m = 0; m < V; m++) acc[t][m] = 0.f;
    float fhn[kShared ? DIM : 1][V];
    float(*fa)[V] = kShared ? fhn : fhd;
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) fa[d][m] = 0.f;

    // prologue: flux of slice 0
    {
      float dF[DIM][V];
      if (active) slice_flux(0, dF);
      else
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) dF[d][m] = 0.f;
      float* sFn = sFf + buf * S::SLICE_F;
      if (active)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) sFn[(d * NPC + s) * V + m] = dF[d][m];
      if (!conv) {
        const float wn = (float)T.w[0];
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fa[d][m] = fmaf(wn, dF[d][m], fa[d][m]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int n = 0; n < B; n++) {
      // Software pipeline: the FP64 flux chain of slice n+1 and the shared-
      // memory derivative of slice n sit between the same two barriers, so
      // they overlap.  Slice n+1 goes to the other buffer, whose slice n-1
      // every thread finished reading before the previous barrier.
      float dFn[DIM][V];
      if (n + 1 < B) {
        if (active) slice_flux(n + 1, dFn);
        else
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) dFn[d][m] = 0.f;
      }
      if (active) {
        const float* sFn = sFf + buf * S::SLICE_F;
        float Gm[V];
#pragma unroll
        for (int m = 0; m < V; m++) Gm[m] = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const float* line = sFn + (d * NPC + s - sd[d] * stride[d]) * V;
#pragma unroll
          for (int p = 0; p < B; p++) {
            const float c = dcf[d][p];
#pragma unroll
            for (int m = 0; m < V; m++) Gm[m] = fmaf(c, line[p * stride[d] * V + m], Gm[m]);
          }
        }
#pragma unroll
        for (int t = 0; t < B; t++) {
          const float ta = (float)T.tA[t][n];
#pragma unroll
          for (int m = 0; m < V; m++) acc[t][m] = fmaf(ta, Gm[m], acc[t][m]);
        }
      }
      if (n + 1 < B) {
        buf ^= 1;
        float* sFo = sFf + buf * S::SLICE_F;
        if (active)
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) sFo[(d * NPC + s) * V + m] = dFn[d][m];
        if (!conv) {
          const float wn = (float)T.w[n + 1];
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) fa[d][m] = fmaf(wn, dFn[d][m], fa[d][m]);
        }
        __syncthreads();
      }
    }
    buf ^= 1;  // the next iteration's slice 0 goes to the other buffer

    // new iterate dq = base - dt acc (FP32) and its squared increment
    float r = 0.f;
    if (active && !conv) {
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const float dqn = fmaf(-dtf, acc[t][m], base[t][m]);
          const float diff = dqn - dq[t][m];
          r = fmaf(diff, diff, r);
          dq[t][m] = dqn;
        }
      if (kShared)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fhd[d][m] = fa[d][m];
    }
    const double res = group_sum<G>((double)r, sred);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    if (__syncthreads_and(conv || !valid)) break;
  }

  // ---- FP64 outputs ------------------------------------------------------
  __syncthreads();
  double wsum = 0.0;
#pragma unroll
  for (int t = 0; t < B; t++) wsum += T.w[t];
  if (active) {
#pragma unroll
    for (int m = 0; m < V; m++) {
      double qh = lu[m] * wsum;
#pragma unroll
      for (int t = 0; t < B; t++) qh += (double)dq[t][m] * T.w[t];
      sQh[s * V + m] = qh;
    }
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sD[(d * NPC + s) * V + m] = F0[d][m] * wsum + (double)fhd[d][m];
  }
  __syncthreads();
  if (!valid) return;

  if (active) {
    double* lduh = a.lduh + cell * (long)NPC * V;
    double out[V];
#pragma unroll
    for (int m = 0; m < V; m++) out[m] = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      double us = a.idx[d];
#pragma unroll
      for (int e = 0; e < DIM; e++)
        if (e != d) us *= T.w[sd[e]];
      const double* line = sD + (d * NPC + s - sd[d] * stride[d]) * V;
#pragma unroll
      for (int p = 0; p < B; p++) {
        const double k = T.kxi[sd[d]][p];
#pragma unroll
        for (int m = 0; m < V; m++) out[m] += k * line[p * stride[d] * V + m] * us;
      }
    }
#pragma unroll
    for (int m = 0; m < V; m++) lduh[s * V + m] = out[m];
  }
  {
    constexpr int NF = S::NF;
    double* qb = a.lQhbnd + cell * (long)2 * DIM * NF * V;
    double* fb = a.lFhbnd + cell * (long)2 * DIM * NF * V;
    for (int k = s; k < 2 * DIM * NF; k += G) {
      const int f = k / NF, j = k % NF, d = f >> 1, side = f & 1;
      int base, st;
      if (DIM == 3) {
        const int ia = j / B, ib = j % B;
        if (d == 0) { base = (ia * B + ib) * B; st = 1; }
        else if (d == 1) { base = ia * B * B + ib; st = B; }
        else { base = ia * B + ib; st = B * B; }
      } else {
        if (d == 0) { base = j * B; st = 1; }
        else { base = j; st = B; }
      }
      double vq[V], vf[V];
#pragma unroll
      for (int m = 0; m < V; m++) { vq[m] = 0.0; vf[m] = 0.0; }
#pragma unroll
      for (int l = 0; l < B; l++) {
        const double c = side ? T.fr[l] : T.fl[l];
        const int node = base + l * st;
#pragma unroll
        for (int m = 0; m < V; m++) {
          vq[m] += sQh[node * V + m] * c;
          vf[m] += sD[(d * NPC + node) * V + m] * c;
        }
      }
#pragma unroll
      for (int m = 0; m < V; m++) {
        qb[(f * NF + j) * V + m] = vq[m];
        fb[(f * NF + j) * V + m] = vf[m];
      }
    }
  }
  if (s == 0) {
    if (a.iters) a.iters[cell] = it;
    if (a.stats) {
      atomicAdd(&a.stats[0], (unsigned long long)it);
      if (!conv) atomicAdd(&a.stats[1], 1ull);
    }
  }
}

}  // namespace exa
