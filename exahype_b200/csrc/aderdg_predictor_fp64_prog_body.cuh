// FP64 predictor + volume integral, line-owner contraction with the time
// contraction folded in slice by slice ("progressive"): one cell per CTA
// (3D) or several cells per CTA (2D), as the line-owner block.
//
// Same operator, same operations in the same order and so the same bits as
// predictor_fp64_lines_block (aderdg_predictor_fp64_lines_body.cuh); what
// changes is what stays live:
//   * the line sums of a time slice are folded into the node's time
//     accumulators (acc[t] += tA[t][n] G[n]) right after the slice, so only
//     two slices of line sums are kept (double buffer) instead of all B:
//     shared memory per cell drops from 105 KB to 60 KB (two flux slices +
//     two line-sum slices), three CTAs per SM instead of two;
//   * the time-weighted flux sum of the outputs is not carried through the
//     Picard loop: once the loop has converged (or reached 2(N+1)
//     iterations), it is evaluated from the last iteration's input iterate,
//     which is still in registers at that point (the flux of the same
//     values, summed in the same order), so no 15 accumulators live across
//     the slices.
// Time slices are pipelined with one barrier per slice: node threads store
// slice n's flux, barrier, then every thread runs the line tasks of slice n
// and the node threads fold in the line sums of slice n-1 (stored before
// that barrier).
#pragma once
#include "exa_device.cuh"
#include "aderdg_predictor_mixed_body.cuh"
#include "aderdg_predictor_fp64_lines_body.cuh"

namespace exa {

template <int DIM, int N>
struct Fp64ProgShape {
  using M = MixShape<DIM, N>;
  using LS = Fp64LineShape<DIM, N>;
  static constexpr int B = N + 1;
  static constexpr int V = kV;
  static constexpr int NPC = M::NPC;
  static constexpr int G = M::G;
  static constexpr int CPB = M::CPB;
  static constexpr int NT = M::NT;
  static constexpr int L = NPC / B;
  static constexpr int TPD = L * V;
  static constexpr int TPT = (TPD + G - 1) / G;
  // doubles: flux slice [DIM][NPC][V]; line sums of one slice [DIM][V][NPC]
  static constexpr int F_SLICE = (DIM * NPC * V + 1) & ~1;
  static constexpr int X_SLICE = (DIM * V * NPC + 1) & ~1;
  static constexpr int LOOP_D = 2 * F_SLICE + 2 * X_SLICE;
  static constexpr int CELL_D = ((LOOP_D > M::STAGE_D ? LOOP_D : M::STAGE_D) + 1) & ~1;
  static constexpr int SM_DOUBLES = CPB * CELL_D + 2 * (NT / 32) + 1;
};

template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void predictor_fp64_prog_block(const PredArgs& a, long block, double* smem) {
  using S = Fp64ProgShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G, L = S::L, TPD = S::TPD, TPT = S::TPT;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];

  constexpr bool kMulti = S::CPB > 1;  // several cells per CTA
  const int lc = kMulti ? threadIdx.x / G : 0;  // cell of the CTA
  const int s = kMulti ? threadIdx.x % G : threadIdx.x;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  double* sD = smem + lc * S::CELL_D;
  double* sF = sD;                    // [2][F_SLICE]
  double* sX = sD + 2 * S::F_SLICE;  // [2][X_SLICE]
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

  // task offsets (the numbering of predictor_fp64_lines_block, so every
  // shared access keeps its bank pattern): first point of the line in the
  // flux slice and in a line-sum slice
  int fbase[TPT][DIM], xbase[TPT][DIM];
  bool tv[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = s + r * G;
    tv[r] = valid && k < TPD;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      int c, m;
      if (S::LS::order(d) == 3) {
        c = k / (B * V) + B * (k % B);
        m = (k / B) % V;
      } else if (S::LS::order(d) == 2) {
        c = k / V;
        m = k % V;
      } else {
        c = k % L;
        m = k / L;
      }
      if (!tv[r]) c = m = 0;
      const int n0 = d == 0 ? line_node<B, 0>(c, 0) : (d == 1 ? line_node<B, 1>(c, 0) : line_node<B, 2>(c, 0));
      fbase[r][d] = (d * NPC + n0) * V + m;
      xbase[r][d] = (d * V + m) * NPC + n0;
    }
  }

  double fa[DIM][V];
  int it = 0;
  bool conv = false;
  bool done = false;  // this cell's outputs are final (several cells per CTA)
  int buf = 0;
  for (int iter = 0; iter < MAXIT; iter++) {
    double acc[B][V];
#pragma unroll
    for (int t = 0; t < B; t++)
#pragma unroll
      for (int m = 0; m < V; m++) acc[t][m] = 0.0;

    // node threads: fold the line sums of slice n (buffer X) into the time
    // accumulators; the first iteration's slices all equal slice 0, folded
    // once per slice weight as the reference's B identical evaluations
    auto consume = [&](int n, const double* X) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        double g = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) g += a.idx[d] * X[(d * V + m) * NPC + s];
        if (iter == 0) {
#pragma unroll
          for (int n2 = 0; n2 < B; n2++)
#pragma unroll
            for (int t = 0; t < B; t++) acc[t][m] += T.tA[t][n2] * g;
        } else {
#pragma unroll
          for (int t = 0; t < B; t++) acc[t][m] += T.tA[t][n] * g;
        }
      }
    };

    const int nsl = iter == 0 ? 1 : B;
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (n >= nsl) break;
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
          for (int m = 0; m < V; m++) sFn[(d * NPC + s) * V + m] = F[d][m];
      }
      __syncthreads();
      // line tasks of slice n -> line-sum buffer `buf`; the buffer `buf ^ 1`
      // holds slice n-1's line sums, stored before the barrier above
      {
        double* Xn = sX + buf * S::X_SLICE;
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          if (!tv[r]) continue;
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            const int SD = d == 0 ? 1 : (d == 1 ? B : B * B);
            double fl[B];
#pragma unroll
            for (int p = 0; p < B; p++) fl[p] = sFn[fbase[r][d] + p * SD * V];
            double* xo = Xn + xbase[r][d];
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
      if (active && n > 0) consume(n - 1, sX + (buf ^ 1) * S::X_SLICE);
      buf ^= 1;
    }
    __syncthreads();
    if (active) consume(nsl - 1, sX + (buf ^ 1) * S::X_SLICE);

    // new iterate into acc (the old one stays in q until the exit test)
    double r2 = 0.0;
    if (active && !conv) {
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          // luh re-read (read-only path, L1): ten fewer registers across
          // the slice loop
          const double qn = T.c0[t] * __ldg(a.luh + cell * (long)NPC * V + s * V + m) - dt * acc[t][m];
          const double dq = q[t][m] - qn;
          r2 += dq * dq;
          acc[t][m] = qn;
        }
    }
    const double res = group_sum_1b<G, S::NT>(r2, sred, iter);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    const bool last = conv || iter == MAXIT - 1;
    if (last && active && (!kMulti || !done)) {
      // the outputs' flux time average: the fluxes of this iteration's
      // input iterate q, weighted and summed slice by slice in order
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int m = 0; m < V; m++) fa[d][m] = 0.0;
#pragma unroll
      for (int n = 0; n < B; n++) {
        double F[DIM][V];
        double qq[V];
#pragma unroll
        for (int m = 0; m < V; m++) qq[m] = q[n][m];  // (the first iterate is luh in every slice)
        euler_flux<DIM, PLANAR>(qq, F);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fa[d][m] += T.w[n] * F[d][m];
      }
    }
    if (active && (!kMulti || !done))
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) q[t][m] = acc[t][m];
    // one cell per CTA: every thread holds its cell's sum, so the exit needs
    // no vote; several cells run until the last of them is done
    if constexpr (!kMulti) {
      if (last || !valid) break;
    } else {
      done = done || last;
      if (__syncthreads_and(done || !valid)) break;
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
      for (int m = 0; m < V; m++) sFh[(d * NPC + s) * V + m] = fa[d][m];
  }
  dg_line_outputs<DIM, N>(a, cell, s, valid, active, sD, it, conv);
}

}  // namespace exa
