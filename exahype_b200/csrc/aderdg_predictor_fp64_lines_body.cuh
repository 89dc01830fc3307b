// FP64 predictor + volume integral, line-owner contraction.
//
// Same operator and precision as predictor_block (aderdg_predictor_body.cuh,
// the reference's aderPicardLoopNonlinear / aderPredictorNonlinear /
// aderExtrapolatorNonlinear / volumeIntegralNonlinear), reorganised for
// shared-memory bandwidth, which bounds the node-gather form: there each
// node thread reads the 3 B flux values of its three lines for every time
// slice, so every stored double is read B times.  Here, per time slice,
//   1. node threads evaluate the flux of their node (FP64) into a slice
//      buffer;
//   2. line tasks (direction d, line c, variable m) read the B values of
//      their line once, apply the derivative matrix (uniform constants) and
//      store the B line sums into a per-iteration buffer holding every
//      slice;
// and after the last slice each node thread sums its directions (times
// 1/dx_d), applies the time matrix and forms the new iterate
// q[t] = c0[t] luh - dt sum_n tA[t][n] G[n].  Shared-memory traffic per
// node and slice: 4 DIM V doubles (flux store, line load, line-sum store,
// node load) instead of DIM V (B + 1).  The task numbering per direction is
// chosen so that every one of these accesses is free of bank conflicts for
// 3D order 4 (FP64 accesses: each half-warp hits 16 distinct 8-byte banks).
#pragma once
#include "exa_device.cuh"
#include "aderdg_predictor_mixed_body.cuh"

namespace exa {

template <int DIM, int N>
struct Fp64LineShape {
  using M = MixShape<DIM, N>;
  static constexpr int B = N + 1;
  static constexpr int V = kV;
  static constexpr int NPC = M::NPC;
  static constexpr int G = M::G;
  static constexpr int CPB = M::CPB;
  static constexpr int NT = M::NT;
  static constexpr int L = NPC / B;
  static constexpr int TPD = L * V;
  static constexpr int TPT = (TPD + G - 1) / G;
  // task numbering of direction d: 0 = line index fastest, then variable;
  // 2 = variable fastest, then line; 3 = second line coordinate, variable,
  // first line coordinate
  __host__ __device__ static constexpr int order(int d) {
    return (DIM == 3 && N == 4) ? (d == 0 ? 0 : (d == 1 ? 3 : 2)) : 0;
  }
  // doubles: flux slice [DIM][NPC][V]; line sums [DIM][B][V][NPC]
  static constexpr int F_SLICE = (DIM * NPC * V + 1) & ~1;
  static constexpr int X_SIZE = DIM * B * V * NPC;
  static constexpr int LOOP_D = 2 * F_SLICE + X_SIZE;
  static constexpr int CELL_D = ((LOOP_D > M::STAGE_D ? LOOP_D : M::STAGE_D) + 1) & ~1;
  static constexpr int SM_DOUBLES = CPB * CELL_D + 2 * (NT / 32) + 1;
};

template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void predictor_fp64_lines_block(const PredArgs& a, long block, double* smem) {
  using S = Fp64LineShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G, L = S::L, TPD = S::TPD, TPT = S::TPT;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];

  const int lc = threadIdx.x / G;
  const int s = threadIdx.x % G;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  double* sD = smem + lc * S::CELL_D;
  double* sF = sD;                  // [2][DIM][NPC][V]
  double* sX = sD + 2 * S::F_SLICE;  // [DIM][B][V][NPC]
  double* sred = smem + S::CPB * S::CELL_D;

  double lu[V];
  {
    const double* luh = a.luh + cell * (long)NPC * V;
#pragma unroll
    for (int m = 0; m < V; m++) lu[m] = active ? luh[s * V + m] : (m == 0 ? 1.0 : (m == 4 ? 2.5 : 0.0));
  }
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;

  double q[B][V];
#pragma unroll
  for (int t = 0; t < B; t++)
#pragma unroll
    for (int m = 0; m < V; m++) q[t][m] = lu[m];

  // task offsets: first point of the line in the flux slice (AoS) and in
  // the line-sum buffer
  int fbase[TPT][DIM], xbase[TPT][DIM];
  bool tv[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = s + r * G;
    tv[r] = valid && k < TPD;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      int c, m;
      if (S::order(d) == 3) {
        c = k / (B * V) + B * (k % B);
        m = (k / B) % V;
      } else if (S::order(d) == 2) {
        c = k / V;
        m = k % V;
      } else {
        c = k % L;
        m = k / L;
      }
      if (!tv[r]) c = m = 0;
      const int n0 = d == 0 ? line_node<B, 0>(c, 0) : (d == 1 ? line_node<B, 1>(c, 0) : line_node<B, 2>(c, 0));
      fbase[r][d] = (d * NPC + n0) * V + m;
      xbase[r][d] = (d * B * V + m) * NPC + n0;
    }
  }

  constexpr bool kShared = S::CPB > 1;
  double fa[DIM][V];
  double fkeep[kShared ? DIM : 1][V];
  int it = 0;
  bool conv = false;
  int buf = 0;
  for (int iter = 0; iter < MAXIT; iter++) {
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) fa[d][m] = 0.0;
    // The first iterate is luh in every time slice (the reference's
    // trivial initial guess), so iteration 0 evaluates one slice and every
    // later read of a slice's line sums takes slice 0: the same values the
    // B identical evaluations would give, bit for bit.
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (iter == 0 && n > 0) continue;
      {
        double* sFn = sF + buf * S::F_SLICE;
        if (active) {
          double F[DIM][V];
          double qq[V];
#pragma unroll
          for (int m = 0; m < V; m++) qq[m] = q[n][m];
          euler_flux<DIM, PLANAR>(qq, F);
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) {
              sFn[(d * NPC + s) * V + m] = F[d][m];
              fa[d][m] += T.w[n] * F[d][m];
              if (iter == 0)
#pragma unroll
                for (int n2 = 1; n2 < B; n2++) fa[d][m] += T.w[n2] * F[d][m];
            }
        }
      }
      __syncthreads();
      {
        const double* sFn = sF + buf * S::F_SLICE;
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          if (!tv[r]) continue;
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            const int SD = d == 0 ? 1 : (d == 1 ? B : B * B);
            double fl[B];
#pragma unroll
            for (int p = 0; p < B; p++) fl[p] = sFn[fbase[r][d] + p * SD * V];
            double* xo = sX + xbase[r][d] + n * V * NPC;
#pragma unroll
            for (int i = 0; i < B; i++) {
              double g = 0.0;
#pragma unroll
              for (int p = 0; p < B; p++) g += T.deriv[i][p] * fl[p];
              xo[i * SD] = g;
            }
          }
        }
      }
      buf ^= 1;
    }
    __syncthreads();

    double r2 = 0.0;
    if (active && !conv) {
      double acc[B][V];
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) acc[t][m] = 0.0;
#pragma unroll
      for (int n = 0; n < B; n++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const int ns = iter == 0 ? 0 : n;
          double g = 0.0;
#pragma unroll
          for (int d = 0; d < DIM; d++) g += a.idx[d] * sX[((d * B + ns) * V + m) * NPC + s];
#pragma unroll
          for (int t = 0; t < B; t++) acc[t][m] += T.tA[t][n] * g;
        }
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const double qn = T.c0[t] * lu[m] - dt * acc[t][m];
          const double dq = q[t][m] - qn;
          r2 += dq * dq;
          q[t][m] = qn;
        }
      if (kShared)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fkeep[d][m] = fa[d][m];
    }
    // one barrier per iteration for the residual; with one cell per CTA
    // every thread holds the same sum, so the exit needs no vote
    const double res = group_sum_1b<G, S::NT>(r2, sred, iter);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    if constexpr (S::CPB == 1) {
      if (conv || !valid) break;
    } else {
      if (__syncthreads_and(conv || !valid)) break;
    }
  }

  // time averages -> staging, then faces and volume integral
  __syncthreads();
  if (active) {
    double* sQh = sD;
    double* sFh = sD + NPC * V;
#pragma unroll
    for (int m = 0; m < V; m++) {
      double qh = 0.0;
#pragma unroll
      for (int t = 0; t < B; t++) qh += q[t][m] * T.w[t];
      sQh[s * V + m] = qh;
    }
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sFh[(d * NPC + s) * V + m] = kShared ? fkeep[d][m] : fa[d][m];
  }
  dg_line_outputs<DIM, N>(a, cell, s, valid, active, sD, it, conv);
}

}  // namespace exa
