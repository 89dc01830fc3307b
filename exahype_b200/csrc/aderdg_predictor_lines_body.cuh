// Mixed-precision predictor, line-owner contraction (same operator and
// arithmetic format as predictor_mixed_block: FP32 Picard deviations over
// an FP64 base, difference-form FP32 flux deviations, FP64 outputs).
//
// What changes is who contracts what.  In predictor_mixed_block every node
// thread gathers its 3 x B flux deviations along its three lines from
// shared memory for every time slice, so each stored value is read B times
// and the kernel is bound by shared-memory bandwidth.  Here each thread
// also owns one (line, variable) task per direction: it reads the B values
// of its line once per slice, applies the B x B derivative matrix (uniform
// constants) and stores the B outputs into a per-iteration buffer that
// holds every slice.  After the last slice each node thread sums its three
// directions and applies the time matrix.  Shared-memory traffic per Picard iteration drops from
// B^(d+1) * (d B V) loads to about 4 B^(d+1) V (flux store + line load +
// output store + node load per direction).
//
// Tasks: per direction NPC/B lines x V variables; thread k < tasks holds
// task k (line index fastest, so the lanes of a warp read distinct banks);
// cells whose task count exceeds the thread count take two tasks per thread.
#pragma once
#include "exa_device.cuh"
#include "aderdg_predictor_mixed_body.cuh"

namespace exa {

template <int DIM, int N>
struct LineShape {
  using M = MixShape<DIM, N>;
  static constexpr int B = N + 1;
  static constexpr int V = kV;
  static constexpr int NPC = M::NPC;
  static constexpr int G = M::G;
  static constexpr int CPB = M::CPB;
  static constexpr int NT = M::NT;
  static constexpr int L = NPC / B;              // lines per direction
  static constexpr int TPD = L * V;              // tasks per direction
  static constexpr int TPT = (TPD + G - 1) / G;  // tasks per thread
  // Shared-memory layouts, per direction d (in floats):
  //  * flux slice part of d: [NPC][V] (node-major) or [V][MS] (variable-
  //    major, row stride MS >= NPC);
  //  * line outputs of d: [B (slice)][V][XMS] (row stride XMS >= NPC);
  //  * task numbering of d: 0 = line fastest, then variable; 1 = first line
  //    coordinate, variable, second line coordinate; 2 = variable fastest.
  // For 3D order 4 these were chosen by an exhaustive search of the bank
  // mapping so that the node-lane stores/loads and the line-lane loads/
  // stores of every direction are free of bank conflicts (one wavefront per
  // warp access); other shapes use the plain layout.
  static constexpr bool kTuned = DIM == 3 && N == 4;
  __host__ __device__ static constexpr bool flux_vmajor(int d) { return kTuned && d < 2; }
  __host__ __device__ static constexpr int flux_ms(int d) { return kTuned ? (d == 0 ? 125 : 133) : NPC; }
  __host__ __device__ static constexpr int flux_size(int d) { return flux_vmajor(d) ? V * flux_ms(d) : NPC * V; }
  __host__ __device__ static constexpr int flux_off(int d) {
    return (d > 0 ? flux_size(0) : 0) + (d > 1 ? flux_size(1) : 0);
  }
  static constexpr int F_SLICE = (flux_off(DIM - 1) + flux_size(DIM - 1) + 3) & ~3;
  __host__ __device__ static constexpr int x_ms(int d) { return kTuned ? (d == 0 ? 125 : (d == 1 ? 133 : 141)) : NPC; }
  __host__ __device__ static constexpr int x_off(int d) {
    return (d > 0 ? B * V * x_ms(0) : 0) + (d > 1 ? B * V * x_ms(1) : 0);
  }
  static constexpr int X_SIZE = x_off(DIM - 1) + B * V * x_ms(DIM - 1);
  __host__ __device__ static constexpr int order(int d) { return kTuned ? d : 0; }
  __device__ static __forceinline__ int flux_addr(int d, int node, int m) {
    return flux_off(d) + (flux_vmajor(d) ? m * flux_ms(d) + node : node * V + m);
  }
  __device__ static __forceinline__ int x_addr(int d, int n, int m, int node) {
    return x_off(d) + (n * V + m) * x_ms(d) + node;
  }
  static constexpr int BASE_SIZE = B * V * NPC;
  static constexpr int LOOP_F = 2 * F_SLICE + X_SIZE + BASE_SIZE;
  static constexpr int STAGE_F = 2 * M::STAGE_D;  // FP64 staging (mixed_outputs), in floats
  static constexpr int CELL_F = ((LOOP_F > STAGE_F ? LOOP_F : STAGE_F) + 1) & ~1;  // keep doubles aligned
  static constexpr int SM_DOUBLES = CPB * CELL_F / 2 + 2 * (NT / 32) + 1;
};

template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void predictor_mixed_lines_block(const PredArgs& a, long block, double* smem) {
  using S = LineShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G, L = S::L, TPD = S::TPD, TPT = S::TPT;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];
  const DGConstF& TF = c_dgf[N];

  const int lc = threadIdx.x / G;
  const int s = threadIdx.x % G;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  float* cf = reinterpret_cast<float*>(smem) + lc * S::CELL_F;
  double* sD = reinterpret_cast<double*>(cf);  // FP64 staging (before / after the loop)
  float* sF = cf;                              // [2][DIM][NPC][V]
  float* sX = cf + 2 * S::F_SLICE;             // line outputs (S::x_addr)
  float* sB = sX + S::X_SIZE;                  // [B][V][NPC]
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

  // base deviations (c0[t] - 1) luh - dt (sum_n tA[t][n]) D.F0, FP32, in
  // this node's slots of sB
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

  // FP32 base quantities of the difference-form flux (see
  // predictor_mixed_block for the formulas)
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

  auto slice_flux = [&](int n, float (*dF)[V]) {
    const float* dv = dq[n];
    // fast reciprocal (about 2 ulp): every use multiplies a deviation term,
    // whose own FP32 rounding is of the same size
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
    // components 1 and 2 of each direction on the packed FP32 pipe: the
    // same multiply, fma, multiply as the scalar lines, two lanes at once
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

  // this thread's tasks: (line c, variable m) per direction, kept as the
  // shared-memory offsets of the line's first point in the flux slice
  // (fbase) and in the line-output buffer (xbase); the other points follow
  // at compile-time strides
  int fbase[TPT][DIM], xbase[TPT][DIM];
  bool tv[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = s + r * G;
    tv[r] = valid && k < TPD;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      int c = 0, m = 0;
      if (S::order(d) == 1) {  // first line coordinate, variable, second
        c = (k % B) + B * (k / (B * V));
        m = (k / B) % V;
      } else if (S::order(d) == 2) {  // variable fastest
        c = k / V;
        m = k % V;
      } else {
        c = k % L;
        m = k / L;
      }
      if (!tv[r]) c = m = 0;
      const int n0 = d == 0 ? line_node<B, 0>(c, 0) : (d == 1 ? line_node<B, 1>(c, 0) : line_node<B, 2>(c, 0));
      fbase[r][d] = S::flux_addr(d, n0, m);
      xbase[r][d] = S::x_addr(d, 0, m, n0);
    }
  }

  // time-weighted flux deviations of the last iteration; with several cells
  // per CTA a cell that converged keeps the sum of its last iteration while
  // the others continue (its fluxes are then recomputed from the final
  // iterate and must not replace it)
  constexpr bool kShared = S::CPB > 1;
  float fa[DIM][V];
  float fkeep[kShared ? DIM : 1][V];
  int it = 0;
  bool conv = false;
  int buf = 0;
  for (int iter = 0; iter < MAXIT; iter++) {
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) fa[d][m] = 0.f;

    // the first iterate is the same in every time slice (deviation 0, the
    // reference's trivial initial guess): iteration 0 evaluates slice 0 only
    // and every later read of a slice's line sums takes slice 0, the values
    // the B identical evaluations would give
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (iter == 0 && n > 0) continue;
      // node threads: flux deviation of slice n into buffer buf (whose
      // previous contents, slice n-2, every thread read before the last
      // barrier)
      {
        float dF[DIM][V];
        if (active) slice_flux(n, dF);
        float* sFn = sF + buf * S::F_SLICE;
        if (active)
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) sFn[S::flux_addr(d, s, m)] = dF[d][m];
        if (active) {
          const float wn = TF.w[n];
          const float2 wn2 = make_float2(wn, wn);
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            // (0,1) and (2,3) on the packed FP32 pipe, bitwise the scalar fmaf
            const float2 a01 = __ffma2_rn(wn2, make_float2(dF[d][0], dF[d][1]), make_float2(fa[d][0], fa[d][1]));
            const float2 a23 = __ffma2_rn(wn2, make_float2(dF[d][2], dF[d][3]), make_float2(fa[d][2], fa[d][3]));
            fa[d][0] = a01.x;
            fa[d][1] = a01.y;
            fa[d][2] = a23.x;
            fa[d][3] = a23.y;
            fa[d][4] = fmaf(wn, dF[d][4], fa[d][4]);
          }
          if (iter == 0)  // slices 1..B-1 carry the same deviation
#pragma unroll
            for (int n2 = 1; n2 < B; n2++)
#pragma unroll
              for (int d = 0; d < DIM; d++)
#pragma unroll
                for (int m = 0; m < V; m++) fa[d][m] = fmaf(TF.w[n2], dF[d][m], fa[d][m]);
        }
      }
      __syncthreads();
      // line tasks: derivative along the line (uniform constant matrix);
      // the B outputs go straight to sX [d][n][m][node] (a region disjoint
      // from the flux buffers, read by the node threads after the last slice)
      {
        const float* sFn = sF + buf * S::F_SLICE;
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          if (!tv[r]) continue;
#pragma unroll
          for (int d = 0; d < DIM; d++) {
            const int SD = d == 0 ? 1 : (d == 1 ? B : B * B);  // node stride along the line
            const int FSTEP = S::flux_vmajor(d) ? SD : SD * V;
            float fl[B];
#pragma unroll
            for (int p = 0; p < B; p++) fl[p] = sFn[fbase[r][d] + p * FSTEP];
            float* xo = sX + xbase[r][d] + n * V * S::x_ms(d);
            // outputs in pairs (i, i+1) on the packed FP32 pipe; each output
            // is the same fma chain over p as a scalar loop
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
      buf ^= 1;
    }

    __syncthreads();

    // node threads: sum of directions, time matrix, new deviation
    float r2 = 0.f;
    if (active && !conv) {
      F5 acc[B];
#pragma unroll
      for (int t = 0; t < B; t++) acc[t] = f5_zero();
#pragma unroll
      for (int n = 0; n < B; n++) {
        const int ns = iter == 0 ? 0 : n;
        float g[V];
#pragma unroll
        for (int m = 0; m < V; m++) {
          g[m] = 0.f;
#pragma unroll
          for (int d = 0; d < DIM; d++) g[m] = fmaf(idxf[d], sX[S::x_addr(d, ns, m, s)], g[m]);
        }
        const F5 gn{make_float2(g[0], g[1]), make_float2(g[2], g[3]), g[4]};
#pragma unroll
        for (int t = 0; t < B; t++) f5_fma(TF.tA[t][n], gn, acc[t]);
      }
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const float dqn = fmaf(-dtf, f5_get(acc[t], m), sB[(t * V + m) * NPC + s]);
          const float diff = dqn - dq[t][m];
          r2 = fmaf(diff, diff, r2);
          dq[t][m] = dqn;
        }
      if (kShared)
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fkeep[d][m] = fa[d][m];
    }
    // one barrier per iteration for the residual; with one cell per CTA
    // every thread holds the same sum, so the exit needs no vote
    const double res = group_sum_1b<G, S::NT>((double)r2, sred, iter);
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

  // fa holds the weighted flux-deviation sum of the last iteration (the
  // reference averages the fluxes of the last iteration's input iterate)
  mixed_outputs<DIM, N, PLANAR>(a, cell, s, valid, active, dq, kShared ? fkeep : fa, sD, it, conv);
}

}  // namespace exa
