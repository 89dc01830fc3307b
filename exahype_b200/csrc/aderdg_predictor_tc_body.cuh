// Mixed-precision predictor, 3D order 4, with the Picard line derivatives
// on the tensor cores (warp-level mma.sync m16n8k8, TF32 inputs, FP32
// accumulation).
//
// Same arithmetic format as predictor_mixed_lines_block (FP32 Picard
// deviations dq = q - luh over an FP64 base, FP32 difference-form flux
// deviations dF = F(luh + dq) - F(luh), FP64 outputs); what moves is the
// contraction of each time slice's flux deviations along the lines,
// G_d[n] = (1/dx_d) D dF_d[n] (D = the nodal derivative matrix of
// spaceTimePredictorNonlinear.cpph:141-225 with the quadrature weights
// folded in).  Per direction d the slice is a 125 x 5 matrix A_d whose rows
// are (line c, variable m) and whose columns are the 5 points of the line;
// G_d = A_d (D^T / dx_d) is 8 MMA tiles of 16 rows (K and N padded from 5 to
// 8).  The node threads store dF (FP32) straight into the A_d tile layout; each warp takes two row tiles of every direction; the fragments
// of C go to a per-direction output buffer in node order, where each node
// thread sums its three directions and applies the time matrix.
//
// Precision: 3xTF32.  One TF32 product keeps 10 mantissa bits (relative
// 2^-11); that rounding noise in the Picard update lies above the
// reference's absolute stopping rule (squared update < 1e-14), so a
// single-pass TF32 contraction leaves cells iterating to the 2(N+1) cap
// (measured: 5.4 instead of 4.9 mean iterations at 81^3, 1.5e-8 relative
// state error after one step of a coarse grid).  Both operands are
// therefore split into a TF32 head and remainder and three MMAs (head x
// head, remainder x head, head x remainder) give about FP32 accuracy, with
// FP32 accumulation.
//
// Time slices are pipelined with double buffers and one barrier per slice:
// node threads write slice n's tiles, barrier, then every warp runs the MMAs
// of slice n and the node threads take the outputs of slice n-1 (written
// before that barrier).  Shared-memory row strides per direction were
// chosen by a search of the bank mapping of the node stores, fragment loads,
// fragment stores and node loads.
#pragma once
#include "exa_device.cuh"
#include "aderdg_predictor_mixed_body.cuh"

namespace exa {

struct TcShape {
  static constexpr int DIM = 3, N = 4, B = 5, V = 5, NPC = 125, NT = 128, L = 25;
  // A_d rows: order 1: r = 5 c + m; order 0: r = 25 m + c; row stride ps(d)
  __host__ __device__ static constexpr int order(int d) { return d < 2 ? 1 : 0; }
  __host__ __device__ static constexpr int ps(int d) { return d < 2 ? 12 : 9; }
  __host__ __device__ static constexpr int a_size(int d) { return 128 * ps(d); }
  __host__ __device__ static constexpr int a_off(int d) {
    return (d > 0 ? a_size(0) : 0) + (d > 1 ? a_size(1) : 0);
  }
  static constexpr int A_SIZE = 128 * 12 + 128 * 12 + 128 * 9;  // a_off(2) + a_size(2)
  // outputs of direction d: [m][node], row stride xms(d)
  __host__ __device__ static constexpr int xms(int d) { return d == 0 ? 134 : (d == 1 ? 130 : 125); }
  __host__ __device__ static constexpr int x_off(int d) {
    return (d > 0 ? V * xms(0) : 0) + (d > 1 ? V * xms(1) : 0);
  }
  static constexpr int X_SIZE = (V * (134 + 130 + 125) + 3) & ~3;  // x_off(2) + V xms(2), rounded up
  static constexpr int BASE = B * V * NPC;
  static constexpr int LOOP_F = 2 * A_SIZE + 2 * X_SIZE + BASE;
  static constexpr int STAGE_F = 2 * MixShape<3, 4>::STAGE_D;
  static constexpr int CELL_F = ((LOOP_F > STAGE_F ? LOOP_F : STAGE_F) + 3) & ~3;
  static constexpr int SM_DOUBLES = CELL_F / 2 + NT / 32 + 1;
  // (A_SIZE and X_SIZE are spelled out: a class's own constexpr functions
  // cannot be called in its member initialisers; the static_asserts after
  // the class pin them)
  // m stride of a node's values in A_d
  __host__ __device__ static constexpr int a_mstride(int d) { return order(d) ? ps(d) : L * ps(d); }
  // node stride along a line of direction d
  __host__ __device__ static constexpr int sd(int d) { return d == 0 ? 1 : (d == 1 ? 5 : 25); }
};

static_assert(TcShape::a_off(2) + TcShape::a_size(2) == TcShape::A_SIZE, "A_SIZE");
static_assert(TcShape::x_off(2) + TcShape::V * TcShape::xms(2) <= TcShape::X_SIZE, "X_SIZE");
static_assert(TcShape::SM_DOUBLES * 8 * 3 <= 227 * 1024, "3 CTAs per SM");

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// (line, position along the line) of node s in direction d
template <int D>
__device__ __forceinline__ void tc_line_coords(int s, int& c, int& p) {
  if (D == 0) {
    c = s / 5;
    p = s % 5;
  } else if (D == 1) {
    c = (s / 25) * 5 + s % 5;
    p = (s / 5) % 5;
  } else {
    c = s % 25;
    p = s / 25;
  }
}

template <int D>
__device__ __forceinline__ void tc_row_cm(int r, int& c, int& m) {
  if (TcShape::order(D)) {
    c = r / 5;
    m = r % 5;
  } else {
    c = r % 25;
    m = r / 25;
  }
}

template <bool PLANAR>
__device__ __forceinline__ void predictor_mixed_tc_block(const PredArgs& a, long block, double* smem) {
  using S = TcShape;
  constexpr int B = S::B, V = S::V, NPC = S::NPC;
  constexpr int MAXIT = 2 * (S::N + 1);
  const DGConst& T = c_dg[S::N];
  const DGConstF& TF = c_dgf[S::N];

  const int s = threadIdx.x;
  const long cell = block;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  float* cf = reinterpret_cast<float*>(smem);
  double* sD = smem;                        // FP64 staging (before / after the loop)
  float* sA = cf;                           // [2][A_SIZE]
  float* sX = cf + 2 * S::A_SIZE;           // [2][X_SIZE]
  float* sB = sX + 2 * S::X_SIZE;           // [B][V][NPC]
  double* sred = smem + S::CELL_F / 2;

  double lu[V];
  {
    const double* luh = a.luh + cell * (long)NPC * V;
#pragma unroll
    for (int m = 0; m < V; m++) lu[m] = active ? luh[s * V + m] : (m == 0 ? 1.0 : (m == 4 ? 2.5 : 0.0));
  }
  const double dt = a.dt_dev ? *a.dt_dev : a.dt;

  // FP64 base flux derivative (once per cell); ends with a barrier, after
  // which the staging area is the loop's buffers
  double G0[V];
  mixed_base_derivative<3, 4, PLANAR>(a, lu, s, valid, active, sD, G0);

  float tas_f[B];
#pragma unroll
  for (int t = 0; t < B; t++) {
    double tas = 0.0;
#pragma unroll
    for (int n = 0; n < B; n++) tas += T.tA[t][n];
    tas_f[t] = (float)tas;
    if (active)
#pragma unroll
      for (int m = 0; m < V; m++) sB[(t * V + m) * NPC + s] = (float)((T.c0[t] - 1.0) * lu[m] - dt * tas * G0[m]);
  }
  // the padding rows 125..127 of every tile enter the MMAs (their outputs
  // are discarded): keep them finite
  for (int i = s; i < 2 * 3 * 3 * 12; i += S::NT) {
    const int b = i / (3 * 3 * 12), rem = i % (3 * 3 * 12), d = rem / 36, k = rem % 36;
    const int r = 125 + k / 12, col = k % 12;
    if (col < S::ps(d)) sA[b * S::A_SIZE + S::a_off(d) + r * S::ps(d) + col] = 0.f;
  }

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
  const float dtf = (float)dt;

  // node-thread offsets of its values in the A tiles
  int afl[3];
  {
    int c, p;
    tc_line_coords<0>(s < NPC ? s : 0, c, p);
    afl[0] = S::a_off(0) + (S::order(0) ? 5 * c : c) * S::ps(0) + p;
    tc_line_coords<1>(s < NPC ? s : 0, c, p);
    afl[1] = S::a_off(1) + (S::order(1) ? 5 * c : c) * S::ps(1) + p;
    tc_line_coords<2>(s < NPC ? s : 0, c, p);
    afl[2] = S::a_off(2) + (S::order(2) ? 5 * c : c) * S::ps(2) + p;
  }

  // MMA lane constants: warp w takes row tiles 2w and 2w+1 of every
  // direction; rows rb + 16 k + 8 h (k tile, h fragment half)
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  const int rb = 32 * w + gq;
  // B fragments: B[k = p][n = i] = D[i][p] / dx_d in FP32, split into a
  // TF32 head and the TF32 rounding of the remainder (3xTF32)
  uint32_t bfr[3][2], bfl[3][2];
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const double id = a.idx[d];
    const float b0 = gq < B ? (float)(T.deriv[gq][tq] * id) : 0.f;
    const float b1 = (gq < B && tq == 0) ? (float)(T.deriv[gq][4] * id) : 0.f;
    bfr[d][0] = to_tf32(b0);
    bfr[d][1] = to_tf32(b1);
    bfl[d][0] = to_tf32(b0 - __uint_as_float(bfr[d][0]));
    bfl[d][1] = to_tf32(b1 - __uint_as_float(bfr[d][1]));
  }
  // output offsets of the C fragment rows: x_off(d) + m xms(d) + node of
  // column 2 tq; -1 marks a padding row
  int xo[3][2][2];
#pragma unroll
  for (int d = 0; d < 3; d++)
#pragma unroll
    for (int k = 0; k < 2; k++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int r = rb + 16 * k + 8 * h;
        int c, m;
        if (d == 0) tc_row_cm<0>(r, c, m);
        else if (d == 1) tc_row_cm<1>(r, c, m);
        else tc_row_cm<2>(r, c, m);
        const int node = d == 0 ? line_node<5, 0>(c, 2 * tq) : (d == 1 ? line_node<5, 1>(c, 2 * tq)
                                                                        : line_node<5, 2>(c, 2 * tq));
        xo[d][k][h] = r < NPC ? S::x_off(d) + m * S::xms(d) + node : -1;
      }

  auto slice_flux = [&](const float* dv, float (*dF)[V]) {
    const float r1 = __fdividef(1.0f, r0f + dv[0]);
    float m1[3], wv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      m1[k] = m0f[k] + dv[k + 1];
      wv[k] = fmaf(-u0f[k], dv[0], dv[k + 1]);
    }
    float k2 = 0.f;
#pragma unroll
    for (int k = 0; k < (PLANAR ? 2 : 3); k++) k2 = fmaf(m0f[k], wv[k], fmaf(dv[k + 1], m1[k], k2));
    const float dp = (float)(kGamma - 1.0) * fmaf(-0.5f * k2, r1, dv[4]);
    const float dH = dv[4] + dp;
    const float H1 = H0f + dH;
    const float e = fmaf(-h0f, dv[0], dH);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      dF[j][0] = dv[j + 1];
#pragma unroll
      for (int k = 0; k < 3; k++) dF[j][k + 1] = fmaf(m0f[j], wv[k], dv[j + 1] * m1[k]) * r1;
      dF[j][j + 1] += dp;
      dF[j][4] = fmaf(m0f[j], e, dv[j + 1] * H1) * r1;
    }
  };

  // MMAs of one slice: A tiles of buffer ab -> outputs of buffer xb
  auto mma_slice = [&](const float* __restrict__ A, float* __restrict__ X) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const float* Ar0 = A + S::a_off(d) + (rb + 16 * k) * S::ps(d);
        const float* Ar1 = Ar0 + 8 * S::ps(d);
        // A = head + remainder: the head rounded to TF32, the remainder
        // (exact in FP32) truncated to TF32 by the tensor core, an error of
        // 2^-21 of A; three products head x head, remainder x head,
        // head x remainder carry A B to about FP32 accuracy
        const float f0 = Ar0[tq], f1 = Ar1[tq];
        const float f2 = tq == 0 ? Ar0[4] : 0.f, f3 = tq == 0 ? Ar1[4] : 0.f;
        const uint32_t h0 = to_tf32(f0), h1 = to_tf32(f1), h2 = to_tf32(f2), h3 = to_tf32(f3);
        const uint32_t l0 = __float_as_uint(f0 - __uint_as_float(h0));
        const uint32_t l1 = __float_as_uint(f1 - __uint_as_float(h1));
        const uint32_t l2 = __float_as_uint(f2 - __uint_as_float(h2));
        const uint32_t l3 = __float_as_uint(f3 - __uint_as_float(h3));
        float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#define EXA_MMA_TF32(A0, A1, A2, A3, B0, B1)                                                             \
  asm volatile(                                                                                        \
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "     \
      "{%0,%1,%2,%3};"                                                                                 \
      : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)                                                         \
      : "r"(A0), "r"(A1), "r"(A2), "r"(A3), "r"(B0), "r"(B1))
        EXA_MMA_TF32(l0, l1, l2, l3, bfr[d][0], bfr[d][1]);
        EXA_MMA_TF32(h0, h1, h2, h3, bfl[d][0], bfl[d][1]);
        EXA_MMA_TF32(h0, h1, h2, h3, bfr[d][0], bfr[d][1]);
#undef EXA_MMA_TF32
        const int SD = S::sd(d);
        const int x0 = xo[d][k][0], x1 = xo[d][k][1];
        if (tq <= 2) {
          if (x0 >= 0) X[x0] = c0;
          if (x1 >= 0) X[x1] = c2;
        }
        if (tq <= 1) {
          if (x0 >= 0) X[x0 + SD] = c1;
          if (x1 >= 0) X[x1 + SD] = c3;
        }
      }
    }
  };

  float dq[B][V];
#pragma unroll
  for (int t = 0; t < B; t++)
#pragma unroll
    for (int m = 0; m < V; m++) dq[t][m] = 0.f;

  float fa[3][V];
  int it = 0;
  bool conv = false;
  for (int iter = 0; iter < MAXIT; iter++) {
#pragma unroll
    for (int d = 0; d < 3; d++)
#pragma unroll
      for (int m = 0; m < V; m++) fa[d][m] = 0.f;
    F5 acc[B];
#pragma unroll
    for (int t = 0; t < B; t++) acc[t] = f5_zero();

    // node threads: the three directions' outputs of slice n, weighted by
    // the time matrix (iteration 0: every slice equals slice 0)
    auto consume = [&](int n, const float* X) {
      float g[V];
#pragma unroll
      for (int m = 0; m < V; m++)
        g[m] = X[S::x_off(0) + m * S::xms(0) + s] + X[S::x_off(1) + m * S::xms(1) + s] +
               X[S::x_off(2) + m * S::xms(2) + s];
      const F5 gn{make_float2(g[0], g[1]), make_float2(g[2], g[3]), g[4]};
#pragma unroll
      for (int t = 0; t < B; t++) f5_fma(iter == 0 ? tas_f[t] : TF.tA[t][n], gn, acc[t]);
    };

    // the first iterate is the same in every time slice (deviation 0): the
    // first iteration evaluates slice 0 only
    const int nsl = iter == 0 ? 1 : B;
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (n >= nsl) break;
      float* An = sA + (n & 1) * S::A_SIZE;
      if (active) {
        float dF[3][V];
        slice_flux(dq[n], dF);
#pragma unroll
        for (int d = 0; d < 3; d++)
#pragma unroll
          for (int m = 0; m < V; m++)
            An[afl[d] + m * S::a_mstride(d)] = dF[d][m];
        if (iter == 0) {
#pragma unroll
          for (int d = 0; d < 3; d++)
#pragma unroll
            for (int m = 0; m < V; m++) {
              float wsum = 0.f;
#pragma unroll
              for (int n2 = 0; n2 < B; n2++) wsum += TF.w[n2];
              fa[d][m] = wsum * dF[d][m];
            }
        } else {
          const float wn = TF.w[n];
#pragma unroll
          for (int d = 0; d < 3; d++)
#pragma unroll
            for (int m = 0; m < V; m++) fa[d][m] = fmaf(wn, dF[d][m], fa[d][m]);
        }
      }
      __syncthreads();
      if (valid) mma_slice(An, sX + (n & 1) * S::X_SIZE);
      if (active && n > 0) consume(n - 1, sX + ((n - 1) & 1) * S::X_SIZE);
    }
    __syncthreads();
    if (active) consume(nsl - 1, sX + ((nsl - 1) & 1) * S::X_SIZE);

    float r2 = 0.f;
    if (active && !conv) {
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const float dqn = fmaf(-dtf, f5_get(acc[t], m), sB[(t * V + m) * NPC + s]);
          const float diff = dqn - dq[t][m];
          r2 = fmaf(diff, diff, r2);
          dq[t][m] = dqn;
        }
    }
    const double res = group_sum<S::NT>((double)r2, sred);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    if (__syncthreads_and(conv || !valid)) break;
  }

  // fa: the weighted flux-deviation sum of the last iteration (the
  // reference averages the fluxes of the last iteration's input iterate)
  mixed_outputs<3, 4, PLANAR>(a, cell, s, valid, active, dq, fa, sD, it, conv);
}

}  // namespace exa
