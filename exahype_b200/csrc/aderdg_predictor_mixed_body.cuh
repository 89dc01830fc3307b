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
  // time-averaged flux [DIM][NPC][V] + state [NPC][V]).  A slice stores a
  // node's 5 values in 6 floats so that (0,1) and (2,3) load as 8-byte pairs.
  // A slice holds the flux deviations of every node and direction as
  // components 0-3 ([DIM][NPC] float4, one 16-byte load per node) followed
  // by component 4 ([DIM][NPC] float); both parts padded to 16 bytes.
  static constexpr int S4 = DIM * NPC * 4;
  static constexpr int S1 = (DIM * NPC + 3) & ~3;
  static constexpr int SLICE_F = S4 + S1;  // floats per slice, a multiple of 4
  // per-node FP32 base deviations [NPC][B][VP], live through the Picard loop
  static constexpr int VP = 6;
  static constexpr int BASE_D = NPC * B * VP / 2;
  static constexpr int STAGE_D = (2 * DIM + 1) * NPC * V;  // output staging (mixed_outputs)
  static constexpr int LOOP_D = SLICE_F + BASE_D;  // 2 float slices = SLICE_F doubles
  static constexpr int SM_CELL = ((LOOP_D > STAGE_D ? LOOP_D : STAGE_D) + 1) & ~1;  // 16-byte cells
  static constexpr int SM_DOUBLES = CPB * SM_CELL + NT / 32 + 1;
};

// Five FP32 components as two packed pairs and a single: (0,1), (2,3), 4.
// The pairs go through the sm_100 packed FP32 pipe (__ffma2_rn: two
// round-to-nearest fmaf in one instruction, bitwise equal to two fmaf).
struct F5 {
  float2 a, b;
  float c;
};

__device__ __forceinline__ F5 f5_zero() { return F5{make_float2(0.f, 0.f), make_float2(0.f, 0.f), 0.f}; }

// acc += s * x
__device__ __forceinline__ void f5_fma(float s, const F5& x, F5& acc) {
  const float2 ss = make_float2(s, s);
  acc.a = __ffma2_rn(ss, x.a, acc.a);
  acc.b = __ffma2_rn(ss, x.b, acc.b);
  acc.c = fmaf(s, x.c, acc.c);
}

// acc += s * (node values at p, 6-float stride, 8-byte aligned)
__device__ __forceinline__ void f5_fma_smem(float s, const float* p, F5& acc) {
  const float2 ss = make_float2(s, s);
  acc.a = __ffma2_rn(ss, *reinterpret_cast<const float2*>(p), acc.a);
  acc.b = __ffma2_rn(ss, *reinterpret_cast<const float2*>(p + 2), acc.b);
  acc.c = fmaf(s, p[4], acc.c);
}

// acc += s * (components 0-3 at p4 (16-byte aligned), component 4 at p1)
__device__ __forceinline__ void f5_fma_split(float s, const float* p4, const float* p1, F5& acc) {
  const float2 ss = make_float2(s, s);
  const float4 v = *reinterpret_cast<const float4*>(p4);
  acc.a = __ffma2_rn(ss, make_float2(v.x, v.y), acc.a);
  acc.b = __ffma2_rn(ss, make_float2(v.z, v.w), acc.b);
  acc.c = fmaf(s, *p1, acc.c);
}

__device__ __forceinline__ void f5_store_split(float* p4, float* p1, const F5& x) {
  *reinterpret_cast<float4*>(p4) = make_float4(x.a.x, x.a.y, x.b.x, x.b.y);
  *p1 = x.c;
}

__device__ __forceinline__ void f5_store(float* p, const F5& x) {
  *reinterpret_cast<float2*>(p) = x.a;
  *reinterpret_cast<float2*>(p + 2) = x.b;
  p[4] = x.c;
}

__device__ __forceinline__ float f5_get(const F5& x, int m) {
  return m == 0 ? x.a.x : m == 1 ? x.a.y : m == 2 ? x.b.x : m == 3 ? x.b.y : x.c;
}

// node index of point p on line c of direction d (line c: the other
// coordinates a + B b, in x, y, z order without d)
template <int B, int D>
__device__ __forceinline__ int line_node(int c, int p) {
  constexpr int SD = D == 0 ? 1 : (D == 1 ? B : B * B);
  return (c / SD) * SD * B + (c % SD) + p * SD;
}

// Derivative G0 = sum_d (1/dx_d) D_d F(luh) of a mixed-precision predictor
// cell's base flux (FP64, once per cell; every thread of the CTA calls it).
// Line tasks (direction d, line c, variable m) read the B flux values of
// their line once and store the B line sums (uniform derivative matrix);
// each node thread then weights and sums its DIM line sums.  sD: the cell's
// FP64 staging area (2 DIM NPC V doubles).  Returns G0 of node s.
template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void mixed_base_derivative(const PredArgs& a, const double* lu, int s, bool valid,
                                                      bool active, double* sD, double* G0) {
  using S = MixShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G;
  constexpr int L = NPC / B, TPD = L * V, TPT = (TPD + G - 1) / G;
  const DGConst& T = c_dg[N];
  double* sF0 = sD;                // [DIM][NPC][V]
  double* sG = sD + DIM * NPC * V;  // [DIM][NPC][V]
  if (active) {
    double F0[DIM][V];
    euler_flux<DIM, PLANAR>(lu, F0);
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sF0[(d * NPC + s) * V + m] = F0[d][m];
  }
  __syncthreads();
  if (valid) {
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      const int k = s + r * G;
      if (k >= TPD) continue;
      const int c = k % L, m = k / L;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int SD = d == 0 ? 1 : (d == 1 ? B : B * B);
        const int n0 = d == 0 ? line_node<B, 0>(c, 0) : (d == 1 ? line_node<B, 1>(c, 0) : line_node<B, 2>(c, 0));
        double f[B];
#pragma unroll
        for (int p = 0; p < B; p++) f[p] = sF0[(d * NPC + n0 + p * SD) * V + m];
#pragma unroll
        for (int i = 0; i < B; i++) {
          double g = 0.0;
#pragma unroll
          for (int p = 0; p < B; p++) g += T.deriv[i][p] * f[p];
          sG[(d * NPC + n0 + i * SD) * V + m] = g;
        }
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < V; m++) G0[m] = 0.0;
  if (active)
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) G0[m] += a.idx[d] * sG[(d * NPC + s) * V + m];
  __syncthreads();  // the staging area becomes the caller's loop buffers
}

// FP64 outputs of a mixed-precision predictor cell (every thread of the CTA
// calls it): time-averaged state Qh and flux Fh from luh, F(luh) and the FP32
// deviations of the last Picard iterate (dqv: state per time node, fdv: the
// weighted time sum of the flux deviations of the last iteration), then the
// face extrapolations into lQhbnd/lFhbnd and the volume integral into lduh
// (the reference's formulas, FP64).
//
// Both are contractions along lines, so they run as line tasks (direction
// d, line c, variable m; the same numbering as the line-owner predictor):
// a task reads the B values of Qh and Fh_d on its line once and produces
// the two face values of that line (the face node of line c is c) and the
// B line sums  sum_p Kxi[i][p] Fh_d[p]  of the volume integral, which the
// node threads weight and sum over directions.  sD: the cell's FP64 staging
// area, MixShape::STAGE_D doubles: Qh [NPC][V], Fh [DIM][NPC][V],
// volume-integral line sums [DIM][NPC][V].
template <int DIM, int N>
__device__ __forceinline__ void dg_line_outputs(const PredArgs& a, long cell, int s, bool valid, bool active,
                                                double* sD, int it, bool conv);

template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void mixed_outputs(const PredArgs& a, long cell, int s, bool valid, bool active,
                                              const float (*dqv)[kV], const float (*fdv)[kV], double* sD,
                                              int it, bool conv) {
  using S = MixShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC;
  const DGConst& T = c_dg[N];
  double* sQh = sD;            // [NPC][V]
  double* sFh = sD + NPC * V;  // [DIM][NPC][V]
  const double* luh = a.luh + cell * (long)NPC * V;
  __syncthreads();  // the caller's loop buffers overlap the staging area
  if (active) {
    double lu[V], F0[DIM][V];
#pragma unroll
    for (int m = 0; m < V; m++) lu[m] = luh[s * V + m];
    euler_flux<DIM, PLANAR>(lu, F0);
    double wsum = 0.0;
#pragma unroll
    for (int t = 0; t < B; t++) wsum += T.w[t];
#pragma unroll
    for (int m = 0; m < V; m++) {
      double qh = lu[m] * wsum;
#pragma unroll
      for (int t = 0; t < B; t++) qh += (double)dqv[t][m] * T.w[t];
      sQh[s * V + m] = qh;
    }
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sFh[(d * NPC + s) * V + m] = F0[d][m] * wsum + (double)fdv[d][m];
  }
  dg_line_outputs<DIM, N>(a, cell, s, valid, active, sD, it, conv);
}

// Face extrapolations and volume integral of a predictor cell from the
// FP64 staging area written by the caller (Qh [NPC][V], Fh [DIM][NPC][V];
// every thread of the CTA calls it after the caller's stores): see
// mixed_outputs.
template <int DIM, int N>
__device__ __forceinline__ void dg_line_outputs(const PredArgs& a, long cell, int s, bool valid, bool active,
                                                double* sD, int it, bool conv) {
  using S = MixShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G, NF = S::NF;
  constexpr int L = NPC / B, TPD = L * V, TPT = (TPD + G - 1) / G;
  const DGConst& T = c_dg[N];
  double* sQh = sD;                     // [NPC][V]
  double* sFh = sD + NPC * V;           // [DIM][NPC][V]
  double* sVI = sFh + DIM * NPC * V;    // [DIM][NPC][V]
  __syncthreads();
  if (valid) {
    double* qb = a.lQhbnd + cell * (long)2 * DIM * NF * V;
    double* fb = a.lFhbnd + cell * (long)2 * DIM * NF * V;
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      const int k = s + r * G;
      if (k >= TPD) continue;
      const int c = k % L, m = k / L;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        double q[B], f[B];
#pragma unroll
        for (int p = 0; p < B; p++) {
          const int node = d == 0 ? line_node<B, 0>(c, p) : (d == 1 ? line_node<B, 1>(c, p) : line_node<B, 2>(c, p));
          q[p] = sQh[node * V + m];
          f[p] = sFh[(d * NPC + node) * V + m];
        }
        // faces 2d (FLCoeff) and 2d+1 (FRCoeff) of line c
        double ql = 0.0, qr = 0.0, fl = 0.0, fr = 0.0;
#pragma unroll
        for (int p = 0; p < B; p++) {
          ql += q[p] * T.fl[p];
          qr += q[p] * T.fr[p];
          fl += f[p] * T.fl[p];
          fr += f[p] * T.fr[p];
        }
        qb[((2 * d) * NF + c) * V + m] = ql;
        qb[((2 * d + 1) * NF + c) * V + m] = qr;
        fb[((2 * d) * NF + c) * V + m] = fl;
        fb[((2 * d + 1) * NF + c) * V + m] = fr;
        // volume-integral line sums
#pragma unroll
        for (int i = 0; i < B; i++) {
          double v = 0.0;
#pragma unroll
          for (int p = 0; p < B; p++) v += T.kxi[i][p] * f[p];
          const int node = d == 0 ? line_node<B, 0>(c, i) : (d == 1 ? line_node<B, 1>(c, i) : line_node<B, 2>(c, i));
          sVI[(d * NPC + node) * V + m] = v;
        }
      }
    }
  }
  __syncthreads();
  if (!valid) return;
  if (active) {
    // lduh[s] = sum_d (idx_d prod_{e != d} w[s_e]) sum_p Kxi[s_d][p] Fh_d(s_d -> p)
    int sd[3];
    sd[0] = s % B;
    sd[1] = (s / B) % B;
    sd[2] = DIM == 3 ? s / (B * B) : 0;
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
#pragma unroll
      for (int m = 0; m < V; m++) out[m] += sVI[(d * NPC + s) * V + m] * us;
    }
#pragma unroll
    for (int m = 0; m < V; m++) lduh[s * V + m] = out[m];
  }
  if (s == 0) {
    if (a.iters) a.iters[cell] = it;
    if (a.stats) {
      atomicAdd(&a.stats[0], (unsigned long long)it);
      if (!conv) atomicAdd(&a.stats[1], 1ull);
    }
  }
}

template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void predictor_mixed_block(const PredArgs& a, long block, double* smem) {
  using S = MixShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, G = S::G;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];
  const DGConstF& TF = c_dgf[N];

  const int lc = threadIdx.x / G;
  const int s = threadIdx.x % G;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  double* sD = smem + lc * S::SM_CELL;       // FP64 staging [DIM][NPC][V] + [NPC][V]
  float* sFf = reinterpret_cast<float*>(sD);  // two FP32 slices (S4 + S1 floats each)
  float* sBase = reinterpret_cast<float*>(sD + S::SLICE_F) + s * B * S::VP;  // this node's [B][VP]
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
  double G0[V];
  mixed_base_derivative<DIM, N, PLANAR>(a, lu, s, valid, active, sD, G0);

  float dcf[DIM][B];
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int p = 0; p < B; p++) dcf[d][p] = active ? (float)(T.deriv[sd[d]][p] * a.idx[d]) : 0.f;

  // First Picard deviation (all time nodes share luh, so F = F0 and the
  // FP64 part of every iterate is the same):
  //   base[t] = (c0[t] - 1) luh - dt (sum_n tA[t][n]) D.F0
  // kept in FP32 (an O(dt) quantity); an iterate is dq = base - dt acc.
  // (in this thread's shared-memory slot: read once per iteration, it does
  // not need registers across the loop)
  if (active)
#pragma unroll
    for (int t = 0; t < B; t++) {
      double tas = 0.0;
#pragma unroll
      for (int n = 0; n < B; n++) tas += T.tA[t][n];
      float bv[V];
#pragma unroll
      for (int m = 0; m < V; m++) bv[m] = (float)((T.c0[t] - 1.0) * lu[m] - dt * tas * G0[m]);
      f5_store(sBase + t * S::VP, F5{make_float2(bv[0], bv[1]), make_float2(bv[2], bv[3]), bv[4]});
    }
  const float dtf = (float)dt;

  F5 dq[B];
#pragma unroll
  for (int t = 0; t < B; t++) dq[t] = f5_zero();

  // Flux deviation dF = F(luh + dq[n]) - F(luh) of time slice n, computed
  // directly in FP32 from algebraically exact difference formulas (no FP64
  // flux, no conversions inside the Picard loop).  With q1 = q0 + d,
  // rho1 = rho0 + d_rho, m1 = m0 + d_m, w = d_m - u0 d_rho, H = E + p,
  // h0 = H0 / rho0:
  //   d(m_j m_k / rho) = (m0_j w_k + d_mj m1_k) / rho1
  //   d(|m|^2 / 2 rho) = sum_k (m0_k w_k + d_mk m1_k) / (2 rho1)
  //   d(m_j H / rho)    = (m0_j (dH - h0 d_rho) + d_mj H1) / rho1
  // Every term is a product of a base quantity (FP64 rounded once to FP32)
  // and a deviation, so the FP32 rounding error is relative to dF, not to
  // F: the same accuracy as evaluating F in FP64 and rounding F - F0.
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
  auto slice_flux = [&](int n, F5* dF) {
    const float dv[V] = {dq[n].a.x, dq[n].a.y, dq[n].b.x, dq[n].b.y, dq[n].c};
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
#pragma unroll
    for (int j = 0; j < DIM; j++) {
      float f[V];
      f[0] = dv[j + 1];
#pragma unroll
      for (int k = 0; k < 3; k++) f[k + 1] = fmaf(m0f[j], w[k], dv[j + 1] * m1[k]) * r1;
      f[j + 1] += dp;
      f[4] = fmaf(m0f[j], e, dv[j + 1] * H1) * r1;
      dF[j] = F5{make_float2(f[0], f[1]), make_float2(f[2], f[3]), f[4]};
    }
  };

  constexpr bool kShared = S::CPB > 1;
  constexpr int VP = S::VP;
  F5 fhd[DIM];
  int it = 0;
  bool conv = false;
  int buf = 0;  // slice buffer parity, alternates every slice
  for (int iter = 0; iter < MAXIT; iter++) {
    F5 acc[B];
#pragma unroll
    for (int t = 0; t < B; t++) acc[t] = f5_zero();
    F5 fhn[kShared ? DIM : 1];
    F5* fa = kShared ? fhn : fhd;
#pragma unroll
    for (int d = 0; d < DIM; d++) fa[d] = f5_zero();

    // prologue: flux of slice 0
    {
      F5 dF[DIM];
      if (active) slice_flux(0, dF);
      else
#pragma unroll
        for (int d = 0; d < DIM; d++) dF[d] = f5_zero();
      float* sFn = sFf + buf * S::SLICE_F;
      if (active)
#pragma unroll
        for (int d = 0; d < DIM; d++) f5_store_split(sFn + (d * NPC + s) * 4, sFn + S::S4 + d * NPC + s, dF[d]);
      if (!conv) {
        const float wn = TF.w[0];
#pragma unroll
        for (int d = 0; d < DIM; d++) f5_fma(wn, dF[d], fa[d]);
        // the first iterate is the same in every slice (deviation 0, the
        // reference's trivial initial guess): iteration 0 evaluates slice 0
        // only and applies it for every slice, in slice order
        if (iter == 0)
#pragma unroll
          for (int n2 = 1; n2 < B; n2++)
#pragma unroll
            for (int d = 0; d < DIM; d++) f5_fma(TF.w[n2], dF[d], fa[d]);
      }
      __syncthreads();
    }
    F5 Gm0 = f5_zero();
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (iter == 0 && n > 0) {
        if (active)
#pragma unroll
          for (int t = 0; t < B; t++) f5_fma(TF.tA[t][n], Gm0, acc[t]);
        continue;
      }
      // derivative of slice n (buffer buf), then the flux of slice n+1 into
      // the other buffer, whose slice n-1 every thread finished reading
      // before the previous barrier; one barrier per slice
      if (active) {
        const float* sFn = sFf + buf * S::SLICE_F;
        F5 Gm = f5_zero();
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const int l0 = d * NPC + s - sd[d] * stride[d];
          const float* line4 = sFn + l0 * 4;
          const float* line1 = sFn + S::S4 + l0;
#pragma unroll
          for (int p = 0; p < B; p++) f5_fma_split(dcf[d][p], line4 + p * stride[d] * 4, line1 + p * stride[d], Gm);
        }
#pragma unroll
        for (int t = 0; t < B; t++) f5_fma(TF.tA[t][n], Gm, acc[t]);
        Gm0 = Gm;
      }
      if (iter == 0) continue;
      if (n + 1 < B) {
        F5 dFn[DIM];
        if (active) slice_flux(n + 1, dFn);
        else
#pragma unroll
          for (int d = 0; d < DIM; d++) dFn[d] = f5_zero();
        buf ^= 1;
        float* sFo = sFf + buf * S::SLICE_F;
        if (active)
#pragma unroll
          for (int d = 0; d < DIM; d++) f5_store_split(sFo + (d * NPC + s) * 4, sFo + S::S4 + d * NPC + s, dFn[d]);
        if (!conv) {
          const float wn = TF.w[n + 1];
#pragma unroll
          for (int d = 0; d < DIM; d++) f5_fma(wn, dFn[d], fa[d]);
        }
        __syncthreads();
      }
    }
    buf ^= 1;  // the next iteration's slice 0 goes to the other buffer

    // new iterate dq = base - dt acc (FP32) and its squared increment
    float r = 0.f;
    if (active && !conv) {
      float2 r2 = make_float2(0.f, 0.f);
      const float2 mdt = make_float2(-dtf, -dtf);
#pragma unroll
      for (int t = 0; t < B; t++) {
        const float* bt = sBase + t * VP;
        F5 dqn;
        dqn.a = __ffma2_rn(mdt, acc[t].a, *reinterpret_cast<const float2*>(bt));
        dqn.b = __ffma2_rn(mdt, acc[t].b, *reinterpret_cast<const float2*>(bt + 2));
        dqn.c = fmaf(-dtf, acc[t].c, bt[4]);
        const float2 da = make_float2(dqn.a.x - dq[t].a.x, dqn.a.y - dq[t].a.y);
        const float2 db = make_float2(dqn.b.x - dq[t].b.x, dqn.b.y - dq[t].b.y);
        const float dc = dqn.c - dq[t].c;
        r2 = __ffma2_rn(da, da, r2);
        r2 = __ffma2_rn(db, db, r2);
        r = fmaf(dc, dc, r);
        dq[t] = dqn;
      }
      r += r2.x + r2.y;
      if (kShared)
#pragma unroll
        for (int d = 0; d < DIM; d++) fhd[d] = fa[d];
    }
    const double res = group_sum<G>((double)r, sred);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    if (__syncthreads_and(conv || !valid)) break;
  }

  // ---- FP64 outputs ------------------------------------------------------
  float dqv[B][V], fdv[DIM][V];
#pragma unroll
  for (int t = 0; t < B; t++)
#pragma unroll
    for (int m = 0; m < V; m++) dqv[t][m] = f5_get(dq[t], m);
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int m = 0; m < V; m++) fdv[d][m] = f5_get(fhd[d], m);
  mixed_outputs<DIM, N, PLANAR>(a, cell, s, valid, active, dqv, fdv, sD, it, conv);
}

}  // namespace exa
