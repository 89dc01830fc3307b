// Mixed-precision predictor, line-owner contraction with the time
// contraction folded in slice by slice ("progressive"): one cell per CTA
// (3D) or several cells per CTA (2D), as the line-owner block.
//
// Same operator, same FP32 operations in the same order and so the same
// bits as predictor_mixed_lines_block (aderdg_predictor_lines_body.cuh);
// what changes is what stays live:
//   * the line sums of a time slice are folded into the node's time
//     accumulators (acc[t] += tA[t][n] g[n]) right after the slice, so only
//     two slices of line sums are kept (double buffer) instead of all B:
//     shared memory per cell drops from 68 KB to 44 KB;
//   * the time-weighted flux-deviation sum of the outputs is not carried
//     through the Picard loop: once the loop has converged (or reached
//     2(N+1) iterations) it is evaluated from the last iteration's input
//     deviations, still in registers (the fluxes of the same values, summed
//     in the same order), so 15 accumulators less live across the slices.
// Time slices are pipelined with one barrier per slice: node threads store
// slice n's flux deviation, barrier, then every thread runs the line tasks
// of slice n and the node threads fold in the line sums of slice n-1
// (stored before that barrier).
#pragma once
#include "aderdg_predictor_lines_body.cuh"

namespace exa {

template <int DIM, int N>
struct MixProgShape {
  using LS = LineShape<DIM, N>;
  static constexpr int B = LS::B, V = LS::V, NPC = LS::NPC, G = LS::G, CPB = LS::CPB, NT = LS::NT;
  // one slice of line outputs, [DIM][V][x_ms(d)] floats (the line-owner
  // kernel's layout without its slice index: the same bank pattern)
  __host__ __device__ static constexpr int x1_off(int d) {
    return (d > 0 ? V * LS::x_ms(0) : 0) + (d > 1 ? V * LS::x_ms(1) : 0);
  }
  static constexpr int X_SLICE = (x1_off(DIM - 1) + V * LS::x_ms(DIM - 1) + 3) & ~3;
  __device__ static __forceinline__ int x1_addr(int d, int m, int node) { return x1_off(d) + m * LS::x_ms(d) + node; }
  static constexpr int LOOP_F = 2 * LS::F_SLICE + 2 * X_SLICE + LS::BASE_SIZE;
  static constexpr int CELL_F = ((LOOP_F > LS::STAGE_F ? LOOP_F : LS::STAGE_F) + 1) & ~1;
  static constexpr int SM_DOUBLES = CPB * CELL_F / 2 + 2 * (NT / 32) + 1;
};

__device__ __forceinline__ void f5_set(F5& x, int m, float v) {
  if (m == 0) x.a.x = v;
  else if (m == 1) x.a.y = v;
  else if (m == 2) x.b.x = v;
  else if (m == 3) x.b.y = v;
  else x.c = v;
}

template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void predictor_mixed_prog_block(const PredArgs& a, long block, double* smem) {
  using S = MixProgShape<DIM, N>;
  using LS = LineShape<DIM, N>;
  constexpr bool kMulti = S::CPB > 1;  // several cells per CTA (2D)
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G, L = LS::L, TPD = LS::TPD, TPT = LS::TPT;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];
  const DGConstF& TF = c_dgf[N];

  const int lc = kMulti ? threadIdx.x / G : 0;  // cell of the CTA
  const int s = kMulti ? threadIdx.x % G : threadIdx.x;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  float* cf = reinterpret_cast<float*>(smem) + lc * S::CELL_F;
  double* sD = reinterpret_cast<double*>(cf);  // FP64 staging (before / after the loop)
  float* sF = cf;                       // [2][F_SLICE]
  float* sX = cf + 2 * LS::F_SLICE;     // [2][X_SLICE]
  float* sB = sX + 2 * S::X_SLICE;      // [B][V][NPC]
  double* sred = smem + S::CPB * S::CELL_F / 2;

  double lu[V];
  {
    const double* luh = a.luh + cell * (long)NPC * V;
#pragma unroll
    for (int m = 0; m < V; m++) lu[m] = active ? luh[s * V + m] : (m == 0 ? 1.0 : (m == 4 ? 2.5 : 0.0));
  }
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;

  // FP64 base flux and its derivative (once per cell)
  double G0[V];
  mixed_base_derivative<DIM, N, PLANAR>(a, lu, s, valid, active, sD, G0);

  // base deviations (c0[t] - 1) luh - dt (sum_n tA[t][n]) D.F0, FP32
  if (active)
#pragma unroll
    for (int t = 0; t < B; t++) {
      double tas = 0.0;
#pragma unroll
      for (int n = 0; n < B; n++) tas += T.tA[t][n];
#pragma unroll
      for (int m = 0; m < V; m++) sB[(t * V + m) * NPC + s] = (float)((T.c0[t] - 1.0) * lu[m] - dt * tas * G0[m]);
    }
  const float dtf = (float)dt;
  float idxf[3];
#pragma unroll
  for (int d = 0; d < 3; d++) idxf[d] = (float)a.idx[d];

  // FP32 base quantities of the difference-form flux
  float r0f, m0f[3], u0f[3], H0f, h0f;
  {
    const double irho = 1.0 / lu[0];
    const double p0 = euler_pressure<PLANAR>(lu, irho);
    r0f = (float)lu[0];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      m0f[k] = (float)lu[k + 1];
      u0f[k] = (float)(lu[k + 1] * irho);
    }
    H0f = (float)(lu[4] + p0);
    h0f = (float)((lu[4] + p0) * irho);
  }

  float dq[B][V];
#pragma unroll
  for (int t = 0; t < B; t++)
#pragma unroll
    for (int m = 0; m < V; m++) dq[t][m] = 0.f;

  // flux deviation of slice n (the line-owner kernel's slice_flux)
  auto slice_flux = [&](int n, float (*dF)[V]) {
    const float* dv = dq[n];
    const float r1 = __fdividef(1.0f, r0f + dv[0]);
    float m1[3], w[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      m1[k] = m0f[k] + dv[k + 1];
      w[k] = fmaf(-u0f[k], dv[0], dv[k + 1]);
    }
    float k2 = 0.f;
#pragma unroll
    for (int k = 0; k < (PLANAR ? 2 : 3); k++) k2 = fmaf(m0f[k], w[k], fmaf(dv[k + 1], m1[k], k2));
    const float dp = (float)(kGamma - 1.0) * fmaf(-0.5f * k2, r1, dv[4]);
    const float dH = dv[4] + dp;
    const float H1 = H0f + dH;
    const float e = fmaf(-h0f, dv[0], dH);
    const float2 m1p = make_float2(m1[0], m1[1]), wp = make_float2(w[0], w[1]), r1p = make_float2(r1, r1);
#pragma unroll
    for (int j = 0; j < DIM; j++) {
      dF[j][0] = dv[j + 1];
      const float2 t = __fmul2_rn(__ffma2_rn(make_float2(m0f[j], m0f[j]), wp,
                                             __fmul2_rn(make_float2(dv[j + 1], dv[j + 1]), m1p)),
                                  r1p);
      dF[j][1] = t.x;
      dF[j][2] = t.y;
      dF[j][3] = fmaf(m0f[j], w[2], dv[j + 1] * m1[2]) * r1;
      dF[j][j + 1] += dp;
      dF[j][4] = fmaf(m0f[j], e, dv[j + 1] * H1) * r1;
    }
  };

  // this thread's tasks (the line-owner kernel's numbering and layouts)
  int fbase[TPT][DIM], xbase[TPT][DIM];
  bool tv[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = s + r * G;
    tv[r] = valid && k < TPD;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      int c = 0, m = 0;
      if (LS::order(d) == 1) {
        c = (k % B) + B * (k / (B * V));
        m = (k / B) % V;
      } else if (LS::order(d) == 2) {
        c = k / V;
        m = k % V;
      } else {
        c = k % L;
        m = k / L;
      }
      if (!tv[r]) c = m = 0;
      const int n0 = d == 0 ? line_node<B, 0>(c, 0) : (d == 1 ? line_node<B, 1>(c, 0) : line_node<B, 2>(c, 0));
      fbase[r][d] = LS::flux_addr(d, n0, m);
      xbase[r][d] = S::x1_addr(d, m, n0);
    }
  }

  float fa[DIM][V];
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int m = 0; m < V; m++) fa[d][m] = 0.f;
  int it = 0;
  bool conv = false;
  bool done = false;  // this cell's outputs are final (several cells per CTA)
  int buf = 0;
  for (int iter = 0; iter < MAXIT; iter++) {
    F5 acc[B];
#pragma unroll
    for (int t = 0; t < B; t++) acc[t] = f5_zero();

    // node threads: fold the line sums of slice n (buffer X) into the time
    // accumulators; the first iteration's slices all equal slice 0, folded
    // once per time weight as the reference's B identical evaluations
    auto consume = [&](int n, const float* X) {
      float g[V];
#pragma unroll
      for (int m = 0; m < V; m++) {
        g[m] = 0.f;
#pragma unroll
        for (int d = 0; d < DIM; d++) g[m] = fmaf(idxf[d], X[S::x1_addr(d, m, s)], g[m]);
      }
      const F5 gn{make_float2(g[0], g[1]), make_float2(g[2], g[3]), g[4]};
      if (iter == 0) {
#pragma unroll
        for (int n2 = 0; n2 < B; n2++)
#pragma unroll
          for (int t = 0; t < B; t++) f5_fma(TF.tA[t][n2], gn, acc[t]);
      } else {
#pragma unroll
        for (int t = 0; t < B; t++) f5_fma(TF.tA[t][n], gn, acc[t]);
      }
    };

    const int nsl = iter == 0 ? 1 : B;
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (n >= nsl) break;
      float* sFn = sF + buf * LS::F_SLICE;
      if (active) {
        float dF[DIM][V];
        slice_flux(n, dF);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) sFn[LS::flux_addr(d, s, m)] = dF[d][m];
      }
      __syncthreads();
      // line tasks of slice n -> line-sum buffer `buf`; buffer buf ^ 1 holds
      // slice n-1's line sums, stored before the barrier above
      {
        float* Xn = sX + buf * S::X_SLICE;
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          if (!tv[r]) continue;
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            const int SD = d == 0 ? 1 : (d == 1 ? B : B * B);
            const int FSTEP = LS::flux_vmajor(d) ? SD : SD * V;
            float fl[B];
#pragma unroll
            for (int p = 0; p < B; p++) fl[p] = sFn[fbase[r][d] + p * FSTEP];
            float* xo = Xn + xbase[r][d];
            constexpr int NP = B / 2;
            float2 gp[NP];
            float gs = 0.f;
#pragma unroll
            for (int q = 0; q < NP; q++) gp[q] = make_float2(0.f, 0.f);
#pragma unroll
            for (int p = 0; p < B; p++) {
              const float2 fp = make_float2(fl[p], fl[p]);
#pragma unroll
              for (int q = 0; q < NP; q++)
                gp[q] = __ffma2_rn(*reinterpret_cast<const float2*>(&TF.derivT[p][2 * q]), fp, gp[q]);
              if (B & 1) gs = fmaf(TF.derivT[p][B - 1], fl[p], gs);
            }
#pragma unroll
            for (int i = 0; i < B; i++) {
              const float g = (B & 1) && i == B - 1 ? gs : ((i & 1) ? gp[i / 2].y : gp[i / 2].x);
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

    // new deviations into acc (the old ones stay in dq until the exit test)
    float r2 = 0.f;
    if (active && !conv) {
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const float dqn = fmaf(-dtf, f5_get(acc[t], m), sB[(t * V + m) * NPC + s]);
          const float diff = dqn - dq[t][m];
          r2 = fmaf(diff, diff, r2);
          f5_set(acc[t], m, dqn);
        }
    }
    const double res = group_sum_1b<G, S::NT>((double)r2, sred, iter);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    const bool last = conv || iter == MAXIT - 1;
    if (last && active && (!kMulti || !done)) {
      // the outputs' time-weighted flux deviations: those of this
      // iteration's input deviations, weighted and summed slice by slice
      // (the first iterate's slices are all deviation 0)
#pragma unroll
      for (int n = 0; n < B; n++) {
        float dF[DIM][V];
        slice_flux(n, dF);
        const float wn = TF.w[n];
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fa[d][m] = fmaf(wn, dF[d][m], fa[d][m]);
      }
    }
    // (with one cell per CTA an iteration never starts converged: the loop
    // ends in the iteration that converges; several cells run until the
    // last of them is done, the others' outputs fixed)
    if (active && (!kMulti || !done))
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) dq[t][m] = f5_get(acc[t], m);
    if constexpr (!kMulti) {
      if (last || !valid) break;
    } else {
      done = done || last;
      if (__syncthreads_and(done || !valid)) break;
    }
  }

  mixed_outputs<DIM, N, PLANAR>(a, cell, s, valid, active, dq, fa, sD, it, conv);
}

}  // namespace exa
