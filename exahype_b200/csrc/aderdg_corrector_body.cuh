// Corrector body (Riemann + surface integral + update + next dt, see
// aderdg_faces.cu); shared by k_corrector and the ensemble kernel.
#pragma once
#include "exa_device.cuh"

namespace exa {

template <int DIM, int N>
struct CellShape {
  static constexpr int B = N + 1;
  static constexpr int V = kV;
  static constexpr int NPC = ipow(B, DIM);
  static constexpr int NF = ipow(B, DIM - 1);
  static constexpr int NFACE = 2 * DIM;
  static constexpr int G = CellThreads<NPC>::G;
  static constexpr int CPB = DIM == 3 ? 1 : (128 / G > 0 ? 128 / G : 1);
  static constexpr int NT = G * CPB;
};

// dynamic shared memory (doubles) of one corrector CTA
template <int DIM, int N>
struct CorrShapeSmem {
  using S = CellShape<DIM, N>;
  static constexpr int value =
      S::CPB * (4 * S::NFACE * S::NF * S::V + S::NFACE * 2 * S::V + S::NFACE) + S::NT / 32 + 1;
};

// face-node index of node s on the faces normal to direction d
template <int DIM, int B>
__device__ __forceinline__ int face_node(const int* sd, int d) {
  if (DIM == 3) {
    if (d == 0) return sd[2] * B + sd[1];
    if (d == 1) return sd[2] * B + sd[0];
    return sd[1] * B + sd[0];
  }
  return d == 0 ? sd[1] : sd[0];
}

// weight of face node j (product of the GL weights of its coordinates)
template <int DIM, int B>
__device__ __forceinline__ double face_weight(const DGConst& T, int j) {
  return DIM == 3 ? T.w[j / B] * T.w[j % B] : T.w[j];
}

// ---------------------------------------------------------------- corrector
template <int DIM, int N, bool PLANAR>
__device__ __forceinline__ void corrector_block(const CorrArgs& a, long block, double* smem) {
  using S = CellShape<DIM, N>;
  constexpr int B = S::B, V = S::V, NPC = S::NPC, NF = S::NF, NFACE = S::NFACE, G = S::G;
  constexpr int FV = NFACE * NF * V;
  const DGConst& T = c_dg[N];
  const int lc = threadIdx.x / G;
  const int s = threadIdx.x % G;
  const long cell = block * S::CPB + lc;
  const bool valid = cell < a.ncells;
  double* sQo = smem + lc * (4 * FV + NFACE * 2 * V + NFACE);
  double* sQn = sQo + FV;
  double* sFo = sQn + FV;
  double* sFn = sFo + FV;
  double* sAv = sFn + FV;            // [NFACE][2 (own, neighbour)][V]
  double* sSm = sAv + NFACE * 2 * V;  // [NFACE]

  int cc[3] = {0, 0, 0};
  if (valid) {
    cc[0] = (int)(cell % a.n[0]);
    cc[1] = (int)((cell / a.n[0]) % a.n[1]);
    cc[2] = DIM == 3 ? (int)(cell / ((long)a.n[0] * a.n[1])) : 0;
  }
  // Own faces and the matching faces of the neighbours -> shared memory,
  // as asynchronous 8-byte copies (cp.async): every copy of the CTA is in
  // flight at once without holding registers.  The node's luh and lduh are
  // loaded into registers meanwhile (needed after the face phases).
  if (valid) {
    const double* qo = a.lQhbnd + cell * FV;
    const double* fo = a.lFhbnd + cell * FV;
#pragma unroll
    for (int f = 0; f < NFACE; f++) {
      // the neighbour across face f and where its matching face f^1 lives
      const int d = f >> 1;
      const bool up = f & 1;
      const double* nq;
      const double* nf;
      const bool at_end = up ? cc[d] + 1 == a.n[d] : cc[d] == 0;
      if (at_end && a.bc[d] != 0) {
        // domain boundary: the outside state is formed below from this
        // cell's own face data
        for (int r = s; r < NF * V; r += G) {
          const int k = f * NF * V + r;
          cp_async8(sQo + k, qo + k);
          cp_async8(sFo + k, fo + k);
        }
        continue;
      }
      if (d == DIM - 1 && a.halo_lo && at_end) {
        // across a slab boundary: the adjacent slab's face data
        const long lc2 = DIM == 3 ? (long)cc[1] * a.n[0] + cc[0] : cc[0];
        const double* h = (up ? a.halo_hi : a.halo_lo) + lc2 * 2 * NF * V;
        nq = h;
        nf = h + NF * V;
      } else {
        int nc[3] = {cc[0], cc[1], cc[2]};
        nc[d] = up ? (nc[d] + 1 == a.n[d] ? 0 : nc[d] + 1) : (nc[d] == 0 ? a.n[d] - 1 : nc[d] - 1);
        const long nb = DIM == 3 ? ((long)nc[2] * a.n[1] + nc[1]) * a.n[0] + nc[0]
                                 : (long)nc[1] * a.n[0] + nc[0];
        nq = a.lQhbnd + nb * FV + (f ^ 1) * NF * V;
        nf = a.lFhbnd + nb * FV + (f ^ 1) * NF * V;
      }
      for (int r = s; r < NF * V; r += G) {
        const int k = f * NF * V + r;
        cp_async8(sQo + k, qo + k);
        cp_async8(sFo + k, fo + k);
        cp_async8(sQn + k, nq + r);
        cp_async8(sFn + k, nf + r);
      }
    }
  }
  double v_lduh[V], v_luh[V];
  if (valid && s < NPC) {
    const double* lduh = a.lduh + cell * (long)NPC * V;
    const double* luh = a.luh + cell * (long)NPC * V;
#pragma unroll
    for (int m = 0; m < V; m++) {
      v_lduh[m] = lduh[s * V + m];
      v_luh[m] = luh[s * V + m];
    }
  }
  cp_async_commit_wait_all();
  __syncthreads();
  if (a.bc_any) {
    // outside states of domain-boundary faces, one thread per face node
    // faces unrolled so that d indexes cc, a.bc and a.n at compile time
    // (a runtime index would move them to local memory)
    if (valid)
#pragma unroll
      for (int f = 0; f < NFACE; f++) {
        const int d = f >> 1;
        const bool up = f & 1;
        if (a.bc[d] == 0 || !(up ? cc[d] + 1 == a.n[d] : cc[d] == 0)) continue;
        for (int j = s; j < NF; j += G) {
        const int o = (f * NF + j) * V;
        if (a.bc[d] == EXA_BC_OUTFLOW) {
#pragma unroll
          for (int m = 0; m < V; m++) {
            sQn[o + m] = sQo[o + m];
            sFn[o + m] = sFo[o + m];
          }
        } else {  // EXA_BC_REFLECT
          double qo_[V];
#pragma unroll
          for (int m = 0; m < V; m++) qo_[m] = sQo[o + m];
          qo_[d + 1] = -qo_[d + 1];
          double F[3][V];
          euler_flux<DIM, PLANAR>(qo_, F);
#pragma unroll
          for (int m = 0; m < V; m++) {
            sQn[o + m] = qo_[m];
            sFn[o + m] = F[d][m];
          }
        }
        }
      }
    __syncthreads();
  }
  // face-averaged states (riemannSolverNonlinear.cpph:52-69) and smax per
  // face (:71-81)
  if constexpr (G >= 32) {
    // one warp per face: the averages, a warp barrier, then the face's smax
    constexpr int NWC = G / 32;  // warps of this cell
    const int wc = s >> 5, lane = s & 31;
    if (valid)
      for (int f = wc; f < NFACE; f += NWC) {
        if (lane < 2 * V) {
          const int side = lane / V, m = lane % V;
          const double* Q = (side ? sQn : sQo) + f * NF * V;
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < NF; j++) acc += face_weight<DIM, B>(T, j) * Q[j * V + m];
          sAv[f * 2 * V + lane] = acc;
        }
        __syncwarp();
        if (lane == 0) {
          double qa[5], qb[5];
#pragma unroll
          for (int m = 0; m < V; m++) {
            qa[m] = sAv[(f * 2 + 0) * V + m];
            qb[m] = sAv[(f * 2 + 1) * V + m];
          }
          sSm[f] = fmax(euler_max_eig<PLANAR>(qa, f >> 1), euler_max_eig<PLANAR>(qb, f >> 1));
        }
      }
    __syncthreads();
  } else {
    if (valid) {
      for (int k = s; k < NFACE * 2 * V; k += G) {
        const int f = k / (2 * V), side = (k / V) & 1, m = k % V;
        const double* Q = (side ? sQn : sQo) + f * NF * V;
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < NF; j++) acc += face_weight<DIM, B>(T, j) * Q[j * V + m];
        sAv[k] = acc;
      }
    }
    __syncthreads();
    if (valid && s < NFACE) {
      const int f = s, d = f >> 1;
      double qa[5], qb[5];
#pragma unroll
      for (int m = 0; m < V; m++) {
        qa[m] = sAv[(f * 2 + 0) * V + m];
        qb[m] = sAv[(f * 2 + 1) * V + m];
      }
      sSm[f] = fmax(euler_max_eig<PLANAR>(qa, d), euler_max_eig<PLANAR>(qb, d));
    }
    __syncthreads();
  }
  double dtc = DBL_MAX;
  if (valid && s < NPC) {
    int sd[3];
    sd[0] = s % B;
    sd[1] = (s / B) % B;
    sd[2] = DIM == 3 ? s / (B * B) : 0;
    double* luh = a.luh + cell * (long)NPC * V;
    double v[V];
#pragma unroll
    for (int m = 0; m < V; m++) v[m] = v_lduh[m];
    // surface integral (surfaceIntegralNonlinear.cpph:21-85) of the Rusanov
    // fluxes at this node's face nodes (riemannSolverNonlinear.cpph:83-115:
    // F = (FL+FR)/2 - smax/2 (QR-QL), left = lower cell), formed here by
    // each node that applies them instead of being stored first
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      double wprod = 1.0;
#pragma unroll
      for (int e = DIM - 1; e >= 0; e--)
        if (e != d) wprod *= T.w[sd[e]];
      const double us = wprod / a.dx[d];
      const int j = face_node<DIM, B>(sd, d);
      const double cr = T.fr[sd[d]], cl = T.fl[sd[d]];
      const int kr = ((2 * d + 1) * NF + j) * V, kl = ((2 * d) * NF + j) * V;
      const double smr = sSm[2 * d + 1], sml = sSm[2 * d];
#pragma unroll
      for (int m = 0; m < V; m++) {
        // face 2d+1: this cell is the left one; face 2d: the right one
        const double FR_ = 0.5 * (sFn[kr + m] + sFo[kr + m]) - 0.5 * smr * (sQn[kr + m] - sQo[kr + m]);
        const double FL_ = 0.5 * (sFo[kl + m] + sFn[kl + m]) - 0.5 * sml * (sQo[kl + m] - sQn[kl + m]);
        v[m] -= (FR_ * cr - FL_ * cl) * us;
      }
    }
    // solution update (solutionUpdate.cpph:23-47)
    double W = 1.0;
#pragma unroll
    for (int e = DIM - 1; e >= 0; e--) W *= T.w[sd[e]];
    const double dt = *a.dt_dev;
    const double us = dt / W;
    double q[V];
    bool finite = true;
#pragma unroll
    for (int m = 0; m < V; m++) {
      q[m] = v_luh[m] + v[m] * us;
      luh[s * V + m] = q[m];
      finite = finite && isfinite(q[m]);
    }
    if (!finite && a.nan_flag) atomicOr(a.nan_flag, 1);
    // next step's stable dt at this node (stableTimeStepSize.cpph:21-61)
    if (a.dt_next) {
      double den = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++) den += euler_max_eig<PLANAR>(q, d) / a.dx[d];
      dtc = a.dt_factor / den;
    }
  }
  if (a.dt_next) {
    // minimum over the warp's lanes of this cell, then one atomic per warp
    // (per cell for cells narrower than a warp), skipped when the slot
    // already holds a smaller value (read at L2, where the atomics land;
    // the slot only decreases within a step)
    constexpr int L = G < 32 ? G : 32;
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, o));
    if (valid && (s % L) == 0 && dtc < __longlong_as_double((long long)__ldcg(a.dt_next)))
      atomic_min_pos_double(a.dt_next, dtc);
  }
}

}  // namespace exa

