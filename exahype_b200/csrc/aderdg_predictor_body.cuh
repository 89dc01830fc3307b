// FP64 predictor body (see aderdg_predictor.cu for the design notes);
// shared by k_predictor and the persistent ensemble kernel.
#pragma once
#include "exa_device.cuh"

namespace exa {

template <int DIM, int N, int NPAR>
struct PredShape {
  static constexpr int B = N + 1;
  static constexpr int V = kV;
  static constexpr int D = V + NPAR;
  static constexpr int NPC = ipow(B, DIM);        // nodes per cell
  static constexpr int NF = ipow(B, DIM - 1);     // nodes per face
  static constexpr int G = CellThreads<NPC>::G;   // threads per cell
  static constexpr int CPB = DIM == 3 ? 1 : (128 / G > 0 ? 128 / G : 1);
  static constexpr int NT = G * CPB;
  // shared memory per cell: two flux-slice buffers [2][DIM][NPC][V] (the
  // second doubles as the time-averaged state [NPC][D] after the loop)
  // one flux slice, padded to keep 16-byte alignment of the second buffer
  static constexpr int SLICE_D = (DIM * NPC * V + 1) & ~1;
  static constexpr int SM_CELL = ((2 * SLICE_D > DIM * NPC * V + NPC * D ? 2 * SLICE_D
                                                                         : DIM * NPC * V + NPC * D) + 1) & ~1;
  static constexpr int SM_DOUBLES = CPB * SM_CELL + NT / 32 + 1;
};

// Body of the predictor for the CTA that owns cells [block*CPB, block*CPB+CPB)
// of the cell array described by `a`; also run by the persistent ensemble
// kernel on its work items.
template <int DIM, int N, int NPAR, bool PLANAR, int FULL>
__device__ __forceinline__ void predictor_block(const PredArgs& a, long block, double* smem) {
  using S = PredShape<DIM, N, NPAR>;
  constexpr int B = S::B, V = S::V, D = S::D, NPC = S::NPC, G = S::G;
  constexpr int MAXIT = 2 * (N + 1);
  const DGConst& T = c_dg[N];

  const int lc = threadIdx.x / G;
  const int s = threadIdx.x % G;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  const bool active = valid && s < NPC;
  double* sF = smem + lc * S::SM_CELL;      // [DIM][NPC][V]
  double* sQh = sF + DIM * NPC * V;         // [NPC][D] (after the loop)
  double* sred = smem + S::CPB * S::SM_CELL;

  // node coordinates: sd[0]=x, sd[1]=y, sd[2]=z
  int sd[3];
  sd[0] = s % B;
  sd[1] = (s / B) % B;
  sd[2] = DIM == 3 ? s / (B * B) : 0;
  int stride[3] = {1, B, B * B};

  double lu[D];
  const double* luh = a.luh + cell * (long)NPC * D;
#pragma unroll
  for (int m = 0; m < D; m++) lu[m] = active ? luh[s * D + m] : 1.0;

  const double dt = a.dt_dev ? *a.dt_dev : a.dt;

  // per-thread derivative rows, scaled by 1/dx_d
  double dc[DIM][B];
#pragma unroll
  for (int d = 0; d < DIM; d++)
#pragma unroll
    for (int p = 0; p < B; p++) dc[d][p] = active ? T.deriv[sd[d]][p] * a.idx[d] : 0.0;

  double q[B][V];
#pragma unroll
  for (int t = 0; t < B; t++)
#pragma unroll
    for (int m = 0; m < V; m++) q[t][m] = lu[m];

  double fh[DIM][V];
  int it = 0;
  bool conv = false;
  for (int iter = 0; iter < MAXIT; iter++) {
    double acc[B][V];
#pragma unroll
    for (int t = 0; t < B; t++)
#pragma unroll
      for (int m = 0; m < V; m++) acc[t][m] = 0.0;
    // time-averaged flux of this iteration; a cell that converged earlier
    // than its CTA neighbours keeps its fh (only possible when CPB > 1)
    constexpr bool kShared = S::CPB > 1;
    double fhn[kShared ? DIM : 1][V];
    double(*fa)[V] = kShared ? fhn : fh;
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) fa[d][m] = 0.0;

    // The first iterate is luh in every time slice (the reference's trivial
    // initial guess): iteration 0 evaluates slice 0 once and applies its
    // flux and derivative for every slice n2 in order, the same operations
    // on the same values as B separate evaluations.
#pragma unroll
    for (int n = 0; n < B; n++) {
      if (iter == 0 && n > 0) continue;
      const int nend = iter == 0 ? B : n + 1;
      // alternate the two slice buffers: a thread writing slice n+1 has
      // passed the barrier of slice n, which every thread reaches only after
      // it finished reading slice n-1 (the buffer being overwritten)
      double* sFn = sF + ((iter * B + n) & 1) * S::SLICE_D;
      double F[DIM][V];
      if (active) {
        double qq[5] = {q[n][0], q[n][1], q[n][2], q[n][3], q[n][4]};
        euler_flux<DIM, PLANAR>(qq, F);
      } else {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) F[d][m] = 0.0;
      }
      if (!conv)
        for (int n2 = n; n2 < nend; n2++)
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) fa[d][m] += T.w[n2] * F[d][m];
      if (active) {
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          // split slice layout: components (0,1) and (2,3) as 16-byte pairs,
          // component 4 alone, each [DIM][NPC] (conflict-free 16-byte loads)
          double2* p01 = reinterpret_cast<double2*>(sFn);
          double2* p23 = p01 + DIM * NPC;
          double* p4 = reinterpret_cast<double*>(p23 + DIM * NPC);
          p01[d * NPC + s] = make_double2(F[d][0], F[d][1]);
          p23[d * NPC + s] = make_double2(F[d][2], F[d][3]);
          p4[d * NPC + s] = F[d][4];
        }
        if (FULL && !conv) {
          double* lFi = a.lFi + cell * (long)NPC * B * (DIM + 1) * V;
          for (int n2 = n; n2 < nend; n2++) {
#pragma unroll
            for (int d = 0; d < DIM; d++)
#pragma unroll
              for (int m = 0; m < V; m++) lFi[((n2 * NPC + s) * (DIM + 1) + d) * V + m] = F[d][m];
#pragma unroll
            for (int m = 0; m < V; m++) lFi[((n2 * NPC + s) * (DIM + 1) + DIM) * V + m] = 0.0;
          }
        }
      }
      __syncthreads();
      if (active) {
        double Gm[V];
#pragma unroll
        for (int m = 0; m < V; m++) Gm[m] = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const int l0 = d * NPC + s - sd[d] * stride[d];
          const double2* p01 = reinterpret_cast<const double2*>(sFn) + l0;
          const double2* p23 = p01 + DIM * NPC;
          const double* p4 = reinterpret_cast<const double*>(reinterpret_cast<const double2*>(sFn) + 2 * DIM * NPC) + l0;
#pragma unroll
          for (int p = 0; p < B; p++) {
            const double c = dc[d][p];
            const double2 v01 = p01[p * stride[d]];
            const double2 v23 = p23[p * stride[d]];
            Gm[0] += c * v01.x;
            Gm[1] += c * v01.y;
            Gm[2] += c * v23.x;
            Gm[3] += c * v23.y;
            Gm[4] += c * p4[p * stride[d]];
          }
        }
        for (int n2 = n; n2 < nend; n2++)
#pragma unroll
          for (int t = 0; t < B; t++)
#pragma unroll
            for (int m = 0; m < V; m++) acc[t][m] += T.tA[t][n2] * Gm[m];
      }
    }

    // new iterate and squared increment
    double r = 0.0;
    if (active && !conv) {
#pragma unroll
      for (int t = 0; t < B; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          const double qn = T.c0[t] * lu[m] - dt * acc[t][m];
          const double dq = q[t][m] - qn;
          r += dq * dq;
          q[t][m] = qn;
        }
      if (kShared) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) fh[d][m] = fa[d][m];
      }
    }
    const double res = group_sum<G>(r, sred);
    if (!conv) {
      it = iter + 1;
      if (res < 1e-7 * 1e-7) conv = true;
    }
    if (__syncthreads_and(conv || !valid)) break;
  }

  // ---- outputs --------------------------------------------------------
  __syncthreads();  // last slice's derivative reads are done before reuse
  if (active) {
#pragma unroll
    for (int m = 0; m < V; m++) {
      double qh = 0.0;
#pragma unroll
      for (int t = 0; t < B; t++) qh += q[t][m] * T.w[t];
      sQh[s * D + m] = qh;
    }
#pragma unroll
    for (int m = V; m < D; m++) {
      double qh = 0.0;
#pragma unroll
      for (int t = 0; t < B; t++) qh += lu[m] * T.w[t];
      sQh[s * D + m] = qh;
    }
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sF[(d * NPC + s) * V + m] = fh[d][m];
    if (FULL) {
      double* lQi = a.lQi + cell * (long)NPC * B * D;
#pragma unroll
      for (int t = 0; t < B; t++) {
#pragma unroll
        for (int m = 0; m < V; m++) lQi[(s * B + t) * D + m] = q[t][m];
#pragma unroll
        for (int m = V; m < D; m++) lQi[(s * B + t) * D + m] = lu[m];
      }
      double* lQhi = a.lQhi + cell * (long)NPC * D;
#pragma unroll
      for (int m = 0; m < D; m++) lQhi[s * D + m] = sQh[s * D + m];
      double* lFhi = a.lFhi + cell * (long)NPC * (DIM + 1) * V;
      // reference block layouts: x [z][y][x], y [z][x][y], z [y][x][z]
      int pos[3];
      if (DIM == 3) {
        pos[0] = s;
        pos[1] = (sd[2] * B + sd[0]) * B + sd[1];
        pos[2] = (sd[1] * B + sd[0]) * B + sd[2];
      } else {
        pos[0] = s;
        pos[1] = sd[0] * B + sd[1];
        pos[2] = 0;
      }
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int m = 0; m < V; m++) lFhi[(d * NPC + pos[d]) * V + m] = fh[d][m];
#pragma unroll
      for (int m = 0; m < V; m++) lFhi[(DIM * NPC + s) * V + m] = 0.0;
    }
  }
  __syncthreads();
  if (!valid) return;

  // volume integral: lduh[s] = sum_d (W_s / w_{s_d} / dx_d) sum_p Kxi[s_d][p] Fh_d(s_d -> p)
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
      const double* line = sF + (d * NPC + s - sd[d] * stride[d]) * V;
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

  // face extrapolation: faces 2d (left, FLCoeff) and 2d+1 (right, FRCoeff)
  {
    constexpr int NF = S::NF;
    double* qb = a.lQhbnd + cell * (long)2 * DIM * NF * D;
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
      double vq[D], vf[V];
#pragma unroll
      for (int m = 0; m < D; m++) vq[m] = 0.0;
#pragma unroll
      for (int m = 0; m < V; m++) vf[m] = 0.0;
#pragma unroll
      for (int l = 0; l < B; l++) {
        const double c = side ? T.fr[l] : T.fl[l];
        const int node = base + l * st;
#pragma unroll
        for (int m = 0; m < D; m++) vq[m] += sQh[node * D + m] * c;
#pragma unroll
        for (int m = 0; m < V; m++) vf[m] += sF[(d * NPC + node) * V + m] * c;
      }
#pragma unroll
      for (int m = 0; m < D; m++) qb[(f * NF + j) * D + m] = vq[m];
#pragma unroll
      for (int m = 0; m < V; m++) fb[(f * NF + j) * V + m] = vf[m];
    }
  }

  if (s == 0) {
    const bool nonconv = !conv;
    if (a.iters) a.iters[cell] = it;
    if (a.stats) {
      atomicAdd(&a.stats[0], (unsigned long long)it);
      if (nonconv) atomicAdd(&a.stats[1], 1ull);
    }
  }
}

}  // namespace exa
