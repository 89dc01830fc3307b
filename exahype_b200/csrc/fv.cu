// 2D finite-volume patch kernels (EulerFV path): first-order Godunov and
// MUSCL-Hancock with Rusanov face fluxes, FV CFL time step, periodic ghost
// fill.  Reference:
//   kernels/finitevolumes/godunov/c/2d/godunov.cpph:33-120
//   kernels/finitevolumes/musclhancock/c/2d/musclhancock.cpph:50-240
//   kernels/finitevolumes/riemannsolvers/c/rusanov.cpph:24-83
//   kernels/finitevolumes/commons/c/commons.cpph:26-67
//
// Layout: a patch is (P+2g)^2 cells, row-major [y][x][nData]; patches are
// stored back to back.  A CTA updates a TX x TY tile of interior cells; the
// tile and its halo are staged in shared memory, every face flux is
// computed once per tile, and each cell applies its four face contributions
// in the reference's order (x faces, then y faces).  The reference also
// writes the flux contributions of the patch-boundary faces into the first
// ghost layer of luh_new; that is reproduced.  HBM traffic per cell-update
// is the state read + write (80 B), halo re-reads excepted.
#include <float.h>

#include <cstring>
#include <new>
#include <utility>
#include <vector>

#include "exa_device.cuh"

namespace exa {

constexpr int FV_TX = 32, FV_TY = 8, FV_NT = FV_TX * FV_TY;

struct FVArgs {
  int P, g, S, npar;
  double hx, hy;      // cell sizes
  double dt;
  const double* dt_dev;  // when non-null, dt is read here (device-resident stepping)
  const double* luh;  // state the fluxes are computed from
  double* out;        // luh_new: updated in place (reference semantics)
  unsigned long long* max_dt;  // per patch, atomic-min bit patterns (nullable)
  unsigned long long* next_dt;  // fused steps: CFL dt of the new state (atomic min)
  // optional patch selection of k_fv_patch_small: patches list[0 .. *count)
  const int* list;
  const int* count;
  // fused steps: a grid of npx x npy patches (one patch: 1 x 1) and its
  // boundary rule per dimension (EXA_BC_*)
  int npx, npy, bcx, bcy;
};

// Periodic index of a cell coordinate of a single patch with ghost width g:
// ghost coordinates map to the interior cell a ghost fill would copy.
__device__ __forceinline__ int fv_wrap(int j, int g, int P) { return g + ((j - g) % P + P) % P; }

// Fused steps address the state as one global grid of cells: cell (X, Y),
// 0 <= X < npx P, 0 <= Y < npy P, is interior cell (X mod P, Y mod P) of
// patch (X / P, Y / P) (patch-major, x fastest, P^2 interior cells and g
// ghost layers per patch).  A stencil coordinate outside the domain folds
// back to the cell that a ghost fill would have copied there: the periodic
// image, or at a wall the mirror image (ghost k from the face <- interior
// layer k from the face; FiniteVolumesSolver::mergeWithBoundaryData,
// kernels/finitevolumes/commons/c/commons.cpph:99-340), and inside the
// domain a neighbour patch's ghost cell is that neighbour's interior cell
// (ghostLayerFilling, commons.cpph:337-405).  So a fused step reads no ghost
// cell and needs no exchange pass.
__device__ __forceinline__ int fv_fold(int X, int NX, int bc, bool& mirrored) {
  if (X >= 0 && X < NX) return X;
  if (bc == 0) return (X % NX + NX) % NX;
  mirrored = true;
  // the mirror image of a ghost layer; a coordinate further out than the
  // domain is wide (a tile or strip that overhangs a small grid) feeds only
  // cells that are not written, and is clamped so that it reads inside
  const int Y = X < 0 ? -1 - X : 2 * NX - 1 - X;
  return Y < 0 ? 0 : (Y >= NX ? NX - 1 : Y);
}

// element offset of in-domain cell (X, Y); GRID = false: one periodic
// patch (npx = npy = 1, no walls), known at compile time
template <bool GRID>
__device__ __forceinline__ long fv_cell_offset(const FVArgs& a, int X, int Y) {
  if (!GRID) return ((long)(a.g + Y) * a.S + (a.g + X)) * (kV + a.npar);
  const int px = a.npx == 1 ? 0 : X / a.P, py = a.npy == 1 ? 0 : Y / a.P;
  const long patch = (long)py * a.npx + px;
  return (patch * a.S * a.S + (long)(a.g + Y - py * a.P) * a.S + (a.g + X - px * a.P)) * (kV + a.npar);
}

// element offset of the cell read at stencil coordinate (X, Y); *flip =
// the momentum component a reflecting wall negates there, else -1
template <bool GRID>
__device__ __forceinline__ long fv_stencil_offset(const FVArgs& a, int X, int Y, int* flip) {
  bool mx = false, my = false;
  const int Xf = fv_fold(X, a.P * (GRID ? a.npx : 1), GRID ? a.bcx : 0, mx);
  const int Yf = fv_fold(Y, a.P * (GRID ? a.npy : 1), GRID ? a.bcy : 0, my);
  *flip = !GRID ? -1 : ((mx && a.bcx == EXA_BC_REFLECT) ? 1 : ((my && a.bcy == EXA_BC_REFLECT) ? 2 : -1));
  return fv_cell_offset<GRID>(a, Xf, Yf);
}

// Fused steps (FUSED = true) of a single periodic patch: the tile is loaded
// straight from the periodic interior (no ghost fill, no luh_new copy), the
// new state is luh + face contributions written once, and the new state's
// CFL dt (the commons::stableTimeStepSize rule that the next step starts
// with) is reduced into next_dt.  Ghost layers of `out` are not written.
// Per cell-update HBM traffic: one state read, one state write.


// The next step's CFL dt over the cells a warp updated: the minimum over
// its cells and both directions of 0.45 h_d / s_d (s_d the cell's largest
// |eigenvalue| in direction d, commons::stableTimeStepSize), taken as
// 0.45 h_d / (max over its cells of s_d).  The division is monotone, so
// this is the same value with two divisions per warp instead of two per
// cell; a warp without cells contributes DBL_MAX as before.  Used by the
// Godunov kernels; the MUSCL-Hancock kernels keep the per-cell form, which
// measured faster there (their registers are capped for occupancy).
struct FVNextDt {
  double sx = 0.0, sy = 0.0;
  template <bool PLANAR>
  __device__ __forceinline__ void add(const double* u) {
    sx = fmax(sx, euler_max_eig<PLANAR>(u, 0));
    sy = fmax(sy, euler_max_eig<PLANAR>(u, 1));
  }
  // every lane of the warp calls it; lane 0 reduces into slot
  __device__ __forceinline__ void commit(const FVArgs& a, unsigned long long* slot, bool lane0) {
    for (int o = 16; o > 0; o >>= 1) {
      sx = fmax(sx, __shfl_xor_sync(0xffffffffu, sx, o));
      sy = fmax(sy, __shfl_xor_sync(0xffffffffu, sy, o));
    }
    if (lane0) atomic_min_pos_double(slot, fmin(DBL_MAX, fmin(0.9 / 2 * a.hx / sx, 0.9 / 2 * a.hy / sy)));
  }
};

// Rusanov flux of the face between qL and qR in direction d
// (riemannsolvers/c/rusanov.cpph:24-83); returns s_max.
template <bool PLANAR>
__device__ __forceinline__ double rusanov(const double* qL, const double* qR, int d, double* f) {
  const double sL = euler_max_eig<PLANAR>(qL, d), sR = euler_max_eig<PLANAR>(qR, d);
  const double smax = fmax(sL, sR);
  double FL[2][kV], FR[2][kV];
  euler_flux<2, PLANAR>(qL, FL);
  euler_flux<2, PLANAR>(qR, FR);
#pragma unroll
  for (int i = 0; i < kV; i++) {
    double v = 0.5 * smax * (qL[i] - qR[i]);
    v += 0.5 * (FL[d][i] + FR[d][i]);
    f[i] = v;
  }
  return smax;
}

// ------------------------------------------------------------- Godunov
// The Rusanov flux of a face needs F_d and the largest |eigenvalue| of the
// two cells beside it; both are evaluated once per cell and direction (the
// reference's face loop evaluates them once per face side, i.e. twice per
// cell and direction) and combined per face with the reference's formula,
// so every face flux is the same value.
template <bool PLANAR>
__device__ __forceinline__ void fv_cell_flux(const double* q, int d, double* out) {
  double F[2][kV];
  euler_flux<2, PLANAR>(q, F);
#pragma unroll
  for (int m = 0; m < kV; m++) out[m] = F[d][m];
  out[kV] = euler_max_eig<PLANAR>(q, d);
}

// rusanov() from per-cell fluxes: cl/cr = [F_d(q), lambda] of the left and
// right cell
__device__ __forceinline__ double fv_face_flux(const double* qL, const double* qR, const double* cl,
                                               const double* cr, double* f) {
  const double smax = fmax(cl[kV], cr[kV]);
#pragma unroll
  for (int i = 0; i < kV; i++) {
    double v = 0.5 * smax * (qL[i] - qR[i]);
    v += 0.5 * (cl[i] + cr[i]);
    f[i] = v;
  }
  return smax;
}

// five 256-thread CTAs (42 KB each) per SM: 48 registers and the largest
// shared-memory carveout
// One FV_TX x FV_TY tile (tile column bx, row by) of patch `patch` of a.luh
// / a.out (the body of k_fv_godunov; the serving batch calls it per entry).
// Godunov step as a sweep in y (one periodic patch, or the global view of a
// patch grid): each warp owns a strip of FVS_W output columns (lane l =
// column k0 - 1 + l; lanes 0 and 31 are halo columns) and walks up FVS_H
// rows.  A lane loads its cell of the next row into registers, evaluates F_x,
// F_y and their eigenvalue bounds once, takes the left neighbour's x values
// by a warp shuffle and the row below's y values from its own registers, so
// the kernel has no shared memory and no barrier.  A cell's update is the
// tile kernel's, in the same order (x faces, bottom, then the top face once
// the row above is known), bit for bit.
constexpr int FVS_W = 30, FVS_WARPS = 4, FVS_H = 32;

template <bool PLANAR, bool GRID>
__global__ void __launch_bounds__(32 * FVS_WARPS) k_fv_godunov_sweep(FVArgs a) {
  constexpr int V = kV, C = kV + 1;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  const int NX = GRID ? a.P * a.npx : a.P, NY = GRID ? a.P * a.npy : a.P;
  const int c = (blockIdx.x * FVS_WARPS + w) * FVS_W - 1 + l;  // this lane's column
  const int j0 = blockIdx.y * FVS_H;
  const bool out_col = l >= 1 && l <= FVS_W && c < NX;
  const double dtv = *a.dt_dev;
  const double cx = dtv / a.hx, cy = dtv / a.hy;
  FVNextDt ndt;

  // cell offsets split into a column part, fixed for the lane, and a row
  // part that follows the rows as the strip walks up them (no division per
  // row inside the domain; rows beyond it fold as fv_stencil_offset does)
  const int D = kV + a.npar, S = a.S;
  int fx;
  long colc;
  {
    bool mx = false;
    const int Xf = fv_fold(c, NX, GRID ? a.bcx : 0, mx);
    fx = (GRID && mx && a.bcx == EXA_BC_REFLECT) ? 1 : -1;
    const int px = (GRID && a.npx != 1) ? Xf / a.P : 0;
    colc = (long)px * S * S + (a.g + Xf - px * a.P);
  }
  const int r0 = j0 > 0 ? j0 - 1 : 0;  // first in-domain row the strip loads
  int py = (GRID && a.npy != 1) ? r0 / a.P : 0, ky = r0 - py * a.P;
  auto row_part = [&](int r, int* fy) -> long {
    if (r >= 0 && r < NY) {  // rows load in order: r is the tracked row
      const long rc = (long)py * a.npx * S * S + (long)(a.g + ky) * S;
      if (++ky == a.P) {
        ky = 0;
        ++py;
      }
      *fy = -1;
      return rc;
    }
    bool my = false;
    const int Yf = fv_fold(r, NY, GRID ? a.bcy : 0, my);
    *fy = (GRID && my && a.bcy == EXA_BC_REFLECT) ? 2 : -1;
    const int pr = (GRID && a.npy != 1) ? Yf / a.P : 0;
    return (long)pr * a.npx * S * S + (long)(a.g + Yf - pr * a.P) * S;
  };
  auto load = [&](int r, double* q, long* rc) {
    int fy;
    *rc = row_part(r, &fy);
    const int flip = fx >= 0 ? fx : fy;
    const double* p = a.luh + (*rc + colc) * D;
#pragma unroll
    for (int m = 0; m < V; m++) q[m] = m == flip ? -p[m] : p[m];
  };
  // the row below the strip: its state and y flux record
  double up[V], cyp[C];
  long rc_up, rc_u, rc_n;
  load(j0 - 1, up, &rc_up);
  fv_cell_flux<PLANAR>(up, 1, cyp);
  double part[V];  // the row below's update without its top face
#pragma unroll
  for (int m = 0; m < V; m++) part[m] = 0.0;
  double un[V];
  load(j0, un, &rc_n);
  for (int i = 0; i <= FVS_H; i++) {
    const int r = j0 + i;
    double u[V];
#pragma unroll
    for (int m = 0; m < V; m++) u[m] = un[m];
    rc_u = rc_n;
    if (i < FVS_H) load(r + 1, un, &rc_n);  // prefetch the next row
    double cyr[C];
    fv_cell_flux<PLANAR>(u, 1, cyr);
    // the face below row r: bottom face of row r, top face of row r - 1
    double fy[V];
    fv_face_flux(up, u, cyp, cyr, fy);
    if (i > 0 && out_col && r - 1 < NY) {
      double v[V];
#pragma unroll
      for (int m = 0; m < V; m++) {
        v[m] = part[m];
        v[m] -= cy * fy[m];
      }
      double* o = a.out + (rc_up + colc) * D;  // row r - 1, in the domain
#pragma unroll
      for (int m = 0; m < V; m++) o[m] = v[m];
      ndt.add<PLANAR>(v);
    }
    if (i == FVS_H) break;
    // x faces of row r: the left one from this lane and its left neighbour,
    // the right one from the right neighbour lane
    double cxr[C];
    fv_cell_flux<PLANAR>(u, 0, cxr);
    double ul[V], cxl[C];
#pragma unroll
    for (int m = 0; m < V; m++) ul[m] = __shfl_up_sync(0xffffffffu, u[m], 1);
#pragma unroll
    for (int m = 0; m < C; m++) cxl[m] = __shfl_up_sync(0xffffffffu, cxr[m], 1);
    double fxl[V], fxr[V];
    fv_face_flux(ul, u, cxl, cxr, fxl);
#pragma unroll
    for (int m = 0; m < V; m++) fxr[m] = __shfl_down_sync(0xffffffffu, fxl[m], 1);
#pragma unroll
    for (int m = 0; m < V; m++) {
      double v = u[m];
      v += cx * fxl[m];
      v -= cx * fxr[m];
      v += cy * fy[m];
      part[m] = v;
    }
#pragma unroll
    for (int m = 0; m < V; m++) up[m] = u[m];
#pragma unroll
    for (int m = 0; m < C; m++) cyp[m] = cyr[m];
    rc_up = rc_u;
  }
  ndt.commit(a, a.next_dt, l == 0);
}

template <bool PLANAR, bool FUSED, bool GRID = false>
__device__ __forceinline__ void fv_godunov_tile(const FVArgs& a, int bx, int by, long patch) {
  constexpr int V = kV, C = kV + 1;
  constexpr int LX = FV_TX + 2, LY = FV_TY + 2;
  __shared__ double su[LY * LX * V];
  __shared__ double scx[FV_TY * LX * C];  // x: staged rows 1..TY, all columns
  __shared__ double scy[LY * FV_TX * C];  // y: all rows, staged columns 1..TX
  __shared__ double sred[FV_NT / 32];
  const int D = V + a.npar, S = a.S, pb = a.g, pe = a.g + a.P;
  const double* luh = a.luh + patch * (long)S * S * D;
  double* out = a.out + patch * (long)S * S * D;
  // FUSED: global cell coordinates of the patch grid (fv_cell_offset)
  const int k0 = (FUSED ? 0 : pb) + bx * FV_TX, j0 = (FUSED ? 0 : pb) + by * FV_TY;
  const int tid = threadIdx.x;
  for (int i = tid; i < LY * LX; i += FV_NT) {
    const int r = i / LX, c = i % LX;
    const int j = j0 - 1 + r, k = k0 - 1 + c;
    if (FUSED) {
      int flip;
      const double* q = luh + fv_stencil_offset<GRID>(a, k, j, &flip);
#pragma unroll
      for (int m = 0; m < V; m++) su[i * V + m] = m == flip ? -q[m] : q[m];
    } else if (j >= 0 && j < S && k >= 0 && k < S) {
#pragma unroll
      for (int m = 0; m < V; m++) su[i * V + m] = luh[((long)j * S + k) * D + m];
    }
  }
  __syncthreads();
  // per-cell x fluxes of the cells beside the tile's x faces (rows j < pe,
  // columns pb-1..pe) and y fluxes of the cells beside its y faces
  for (int i = tid; i < FV_TY * LX + LY * FV_TX; i += FV_NT) {
    if (i < FV_TY * LX) {
      const int r = i / LX, c = i % LX;
      const int j = j0 + r, k = k0 - 1 + c;
      if (FUSED || (j < pe && k <= pe)) fv_cell_flux<PLANAR>(&su[((r + 1) * LX + c) * V], 0, &scx[i * C]);
    } else {
      const int i2 = i - FV_TY * LX;
      const int r = i2 / FV_TX, c = i2 % FV_TX;
      const int j = j0 - 1 + r, k = k0 + c;
      if (FUSED || (j <= pe && k < pe)) fv_cell_flux<PLANAR>(&su[(r * LX + c + 1) * V], 1, &scy[i2 * C]);
    }
  }
  __syncthreads();
  const double dtv = a.dt_dev ? *a.dt_dev : a.dt;
  const double cx = dtv / a.hx, cy = dtv / a.hy;
  double dtl = DBL_MAX;
  FVNextDt ndt;
  {
    const int r = tid / FV_TX, c = tid % FV_TX;
    const int j = j0 + r, k = k0 + c;
    const bool valid = FUSED ? (j < a.P * a.npy && k < a.P * a.npx) : (j < pe && k < pe);
    double fxl[V], fxr[V], fyb[V], fyt[V];
    // output cell, addressed before the face fluxes hold their registers
    double* o = FUSED ? a.out + (valid ? fv_cell_offset<GRID>(a, k, j) : 0) : out + ((long)j * S + k) * D;
    if (valid) {
      const double* q = &su[((r + 1) * LX + c + 1) * V];
      const double sxl = fv_face_flux(q - V, q, &scx[(r * LX + c) * C], &scx[(r * LX + c + 1) * C], fxl);
      const double sxr = fv_face_flux(q, q + V, &scx[(r * LX + c + 1) * C], &scx[(r * LX + c + 2) * C], fxr);
      const double syb = fv_face_flux(q - LX * V, q, &scy[(r * FV_TX + c) * C], &scy[((r + 1) * FV_TX + c) * C], fyb);
      const double syt = fv_face_flux(q, q + LX * V, &scy[((r + 1) * FV_TX + c) * C], &scy[((r + 2) * FV_TX + c) * C], fyt);
      if (!FUSED && a.max_dt) {
        // min over faces of 0.45 h / s = 0.45 h / (max over faces of s):
        // the division is monotone, so the same value as per face
        dtl = fmin(0.9 / 2 * a.hx / fmax(sxl, sxr), 0.9 / 2 * a.hy / fmax(syb, syt));
      }
      double un[V];
#pragma unroll
      for (int m = 0; m < V; m++) {
        double u = FUSED ? q[m] : o[m];
        u += cx * fxl[m];
        u -= cx * fxr[m];
        u += cy * fyb[m];
        u -= cy * fyt[m];
        o[m] = u;
        un[m] = u;
      }
      if (FUSED) {
        ndt.add<PLANAR>(un);
      }
    }
    if (FUSED) {
      ndt.commit(a, a.next_dt, (tid & 31) == 0);
      return;
    }
    // first ghost layer, as the reference's face loops touch it
    if (valid && k0 == pb && c == 0) {
      o = out + ((long)j * S + (pb - 1)) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] -= cx * fxl[m];
    }
    if (valid && k == pe - 1) {
      double* o = out + ((long)j * S + pe) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] += cx * fxr[m];
    }
    if (valid && j0 == pb && r == 0) {
      double* o = out + ((long)(pb - 1) * S + k) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] -= cy * fyb[m];
    }
    if (valid && j == pe - 1) {
      double* o = out + ((long)pe * S + k) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] += cy * fyt[m];
    }
  }
  if (a.max_dt) {
    for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
    if ((tid & 31) == 0) sred[tid >> 5] = dtl;
    __syncthreads();
    if (tid == 0) {
      double m = sred[0];
      for (int w = 1; w < FV_NT / 32; w++) m = fmin(m, sred[w]);
      atomic_min_pos_double(&a.max_dt[patch], m);
    }
  }
}

template <bool PLANAR, bool FUSED, bool GRID = false>
__global__ void __launch_bounds__(FV_NT, 5) k_fv_godunov(FVArgs a) {
  fv_godunov_tile<PLANAR, FUSED, GRID>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// -------------------------------------------------------- MUSCL-Hancock
__device__ __forceinline__ double minmod(double a, double b) {
  if (a * b < 0.0) return 0.0;
  return fabs(a) < fabs(b) ? a : b;
}

template <bool PLANAR, bool FUSED>
__global__ void __launch_bounds__(FV_NT) k_fv_muscl(FVArgs a) {
  constexpr int V = kV;
  // staged state: cells j0-2..j0+TY+1, k0-2..k0+TX+1
  constexpr int LX = FV_TX + 4, LY = FV_TY + 4;
  // extrapolated values: x-type on rows j0..j0+TY-1 (+1 ring rows for the
  // y-face cells' evolution), cols k0-1..k0+TX; y-type similarly
  constexpr int RX = FV_TX + 2, RY = FV_TY + 2;  // ring region (tile + 1)
  extern __shared__ double sm[];
  double* su = sm;                               // LY*LX*V
  double* wLx = su + LY * LX * V;                // RY*RX*V each
  double* wRx = wLx + RY * RX * V;
  double* wLy = wRx + RY * RX * V;
  double* wRy = wLy + RY * RX * V;
  double* sfx = wRy + RY * RX * V;               // TY*(TX+1)*V
  double* sfy = sfx + FV_TY * (FV_TX + 1) * V;   // (TY+1)*TX*V
  double* sred = sfy + (FV_TY + 1) * FV_TX * V;
  const int D = V + a.npar, S = a.S, pb = a.g, pe = a.g + a.P;
  const long patch = blockIdx.z;
  const double* luh = a.luh + patch * (long)S * S * D;
  double* out = a.out + patch * (long)S * S * D;
  const int k0 = pb + blockIdx.x * FV_TX, j0 = pb + blockIdx.y * FV_TY;
  const int tid = threadIdx.x;
  const double hx = a.hx, hy = a.hy, dt = a.dt_dev ? *a.dt_dev : a.dt;
  // reciprocal cell sizes: multiplications instead of the reference's
  // divisions (an FP64 division is a long dependent chain)
  const double ihx = 1.0 / hx, ihy = 1.0 / hy;
  for (int i = tid; i < LY * LX; i += FV_NT) {
    const int r = i / LX, c = i % LX;
    int j = j0 - 2 + r, k = k0 - 2 + c;
    if (FUSED) {
      j = fv_wrap(j, pb, a.P);
      k = fv_wrap(k, pb, a.P);
    }
    if (j >= 0 && j < S && k >= 0 && k < S)
#pragma unroll
      for (int m = 0; m < V; m++) su[i * V + m] = luh[((long)j * S + k) * D + m];
  }
  __syncthreads();
  // ring cells (j, k) with j in [j0-1, j0+TY], k in [k0-1, k0+TX]
  for (int i = tid; i < RY * RX; i += FV_NT) {
    const int rr = i / RX, rc = i % RX;
    const int j = j0 - 1 + rr, k = k0 - 1 + rc;
    const double* U = &su[((rr + 1) * LX + rc + 1) * V];
    // reference slope ranges (musclhancock.cpph:79-98): x slopes for
    // j in [pb,pe), k in [pb-1,pe+1); y slopes for j in [pb-1,pe+1), k in [pb,pe)
    const bool has_x = j >= pb && j < pe && k >= pb - 1 && k < pe + 1;
    const bool has_y = j >= pb - 1 && j < pe + 1 && k >= pb && k < pe;
    const bool interior = j >= pb && j < pe && k >= pb && k < pe;
    double lx[V], rx[V], ly[V], ry[V];
#pragma unroll
    for (int m = 0; m < V; m++) { lx[m] = rx[m] = ly[m] = ry[m] = 0.0; }
    if (has_x) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        const double sl = minmod(U[V + m] - U[m], U[m] - U[-V + m]) * ihx;
        lx[m] = U[m] - 0.5 * hx * sl;
        rx[m] = U[m] + 0.5 * hx * sl;
      }
    }
    if (has_y) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        const double sl = minmod(U[LX * V + m] - U[m], U[m] - U[-LX * V + m]) * ihy;
        ly[m] = U[m] - 0.5 * hy * sl;
        ry[m] = U[m] + 0.5 * hy * sl;
      }
    }
    if (interior) {
      // half time step of the interior cells (musclhancock.cpph:126-170)
      double Qt[V];
      double F[2][V];
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] = 0.0;
      euler_flux<2, PLANAR>(lx, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] += F[0][m] * ihx;
      euler_flux<2, PLANAR>(rx, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] -= F[0][m] * ihx;
      euler_flux<2, PLANAR>(ly, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] += F[1][m] * ihy;
      euler_flux<2, PLANAR>(ry, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] -= F[1][m] * ihy;
#pragma unroll
      for (int m = 0; m < V; m++) {
        lx[m] += 0.5 * dt * Qt[m];
        rx[m] += 0.5 * dt * Qt[m];
        ly[m] += 0.5 * dt * Qt[m];
        ry[m] += 0.5 * dt * Qt[m];
      }
    }
#pragma unroll
    for (int m = 0; m < V; m++) {
      wLx[i * V + m] = lx[m];
      wRx[i * V + m] = rx[m];
      wLy[i * V + m] = ly[m];
      wRy[i * V + m] = ry[m];
    }
  }
  __syncthreads();
  double dtl = DBL_MAX;
  // x faces between ring col c (k = k0-1+c) and c+1, rows j0..j0+TY-1
  for (int i = tid; i < FV_TY * (FV_TX + 1); i += FV_NT) {
    const int r = i / (FV_TX + 1), c = i % (FV_TX + 1);
    const int j = j0 + r, k = k0 - 1 + c;  // face between k and k+1
    if (j < pe && k + 1 <= pe) {
      const int il = (r + 1) * RX + c, ir = il + 1;
      const double s = rusanov<PLANAR>(&wRx[il * V], &wLx[ir * V], 0, &sfx[i * V]);
      dtl = fmin(dtl, 0.99 / 2 * hx / s);
    }
  }
  for (int i = tid; i < (FV_TY + 1) * FV_TX; i += FV_NT) {
    const int r = i / FV_TX, c = i % FV_TX;
    const int j = j0 - 1 + r, k = k0 + c;  // face between j and j+1
    if (j + 1 <= pe && k < pe) {
      const int il = r * RX + c + 1, ir = il + RX;
      const double s = rusanov<PLANAR>(&wRy[il * V], &wLy[ir * V], 1, &sfy[i * V]);
      dtl = fmin(dtl, 0.99 / 2 * hy / s);
    }
  }
  __syncthreads();
  const double cx = dt / hx, cy = dt / hy;
  double dtn = DBL_MAX;
  {
    const int r = tid / FV_TX, c = tid % FV_TX;
    const int j = j0 + r, k = k0 + c;
    if (j < pe && k < pe) {
      double* o = out + ((long)j * S + k) * D;
      const double* uc = &su[((r + 2) * LX + c + 2) * V];
      double un[V];
#pragma unroll
      for (int m = 0; m < V; m++) {
        double u = FUSED ? uc[m] : o[m];
        u += cx * sfx[(r * (FV_TX + 1) + c) * V + m];
        u -= cx * sfx[(r * (FV_TX + 1) + c + 1) * V + m];
        u += cy * sfy[(r * FV_TX + c) * V + m];
        u -= cy * sfy[((r + 1) * FV_TX + c) * V + m];
        o[m] = u;
        un[m] = u;
      }
      if (FUSED) {
        dtn = fmin(dtn, 0.9 / 2 * a.hx / euler_max_eig<PLANAR>(un, 0));
        dtn = fmin(dtn, 0.9 / 2 * a.hy / euler_max_eig<PLANAR>(un, 1));
      }
    }
    if (FUSED) {
      for (int o = 16; o > 0; o >>= 1) dtn = fmin(dtn, __shfl_xor_sync(0xffffffffu, dtn, o));
      if ((tid & 31) == 0) atomic_min_pos_double(a.next_dt, dtn);
      return;
    }
    if (j < pe && k0 == pb && c == 0) {
      double* o = out + ((long)j * S + (pb - 1)) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] -= cx * sfx[(r * (FV_TX + 1)) * V + m];
    }
    if (j < pe && k == pe - 1) {
      double* o = out + ((long)j * S + pe) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] += cx * sfx[(r * (FV_TX + 1) + c + 1) * V + m];
    }
    if (k < pe && j0 == pb && r == 0) {
      double* o = out + ((long)(pb - 1) * S + k) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] -= cy * sfy[c * V + m];
    }
    if (k < pe && j == pe - 1) {
      double* o = out + ((long)pe * S + k) * D;
#pragma unroll
      for (int m = 0; m < V; m++) o[m] += cy * sfy[((r + 1) * FV_TX + c) * V + m];
    }
  }
  if (a.max_dt) {
    for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
    if ((tid & 31) == 0) sred[tid >> 5] = dtl;
    __syncthreads();
    if (tid == 0) {
      double m = sred[0];
      for (int w = 1; w < FV_NT / 32; w++) m = fmin(m, sred[w]);
      atomic_min_pos_double(&a.max_dt[patch], m);
    }
  }
}

constexpr size_t kMusclSmem =
    sizeof(double) * ((FV_TY + 4) * (FV_TX + 4) * kV + 4 * (FV_TY + 2) * (FV_TX + 2) * kV +
                      FV_TY * (FV_TX + 1) * kV + (FV_TY + 1) * FV_TX * kV + FV_NT / 32);

// ------------------------------------- fused steps of patches and grids
// Device-resident stepping of one periodic patch (exa_fv_grid, serving) or
// of a grid of patches (exa_fv_patchgrid): the tile and its halo are loaded
// through the global cell view (fv_stencil_offset), the MUSCL-Hancock tile
// lets every interior cell evaluate its own four face fluxes (no flux
// arrays and one barrier fewer than the tile kernels above, which lets more
// CTAs share an SM), and the new state's CFL dt is reduced in the same
// pass.  The update applies the face contributions in the reference's
// order (x faces, then y faces).  Ghost cells of the output are not
// written.
constexpr int FVP_TX = 32, FVP_TY = 8, FVP_NT = FVP_TX * FVP_TY;

template <bool PLANAR>
__device__ __forceinline__ void fv_update_store_dt(const FVArgs& a, double* out, const double* u,
                                                   const double* fxl, const double* fxr, const double* fyb,
                                                   const double* fyt, double cx, double cy, double& dtn) {
  double un[kV];
#pragma unroll
  for (int m = 0; m < kV; m++) {
    double v = u[m];
    v += cx * fxl[m];
    v -= cx * fxr[m];
    v += cy * fyb[m];
    v -= cy * fyt[m];
    out[m] = v;
    un[m] = v;
  }
  dtn = fmin(dtn, 0.9 / 2 * a.hx / euler_max_eig<PLANAR>(un, 0));
  dtn = fmin(dtn, 0.9 / 2 * a.hy / euler_max_eig<PLANAR>(un, 1));
}

// One FVP_TX x FVP_TY tile (tile column bx, row by) of a fused MUSCL-Hancock
// step over a grid of patches (one periodic patch: npx = npy = 1; the
// serving batch calls it per entry); sm: kMusclPeriodicSmem bytes of dynamic
// shared memory.
//
// The reference evolves (half step, musclhancock.cpph:79-170) only a
// patch's interior cells: the extrapolations of its ghost cells enter its
// boundary faces without the half step.  So the face between two patches
// has two different fluxes, one per side.  Here every cell of the tile's
// ring is evolved (in the global view each is interior to its own patch),
// and a cell on its patch's boundary recomputes the neighbour's plain
// extrapolation (the ghost cell's value) for that face from the staged
// state: the same values as a per-patch step after a ghost exchange.
template <bool PLANAR, bool GRID>
__device__ __forceinline__ void fv_muscl_periodic_tile(const FVArgs& a, int bx, int by, double* sm) {
  constexpr int V = kV;
  constexpr int LX = FVP_TX + 4, LY = FVP_TY + 4;   // state: cells j0-2..j0+TY+1, k0-2..k0+TX+1
  constexpr int RX = FVP_TX + 2, RY = FVP_TY + 2;   // ring: j0-1..j0+TY, k0-1..k0+TX
  double* su = sm;                 // LY*LX*V
  double* wLx = su + LY * LX * V;  // RY*RX*V each
  double* wRx = wLx + RY * RX * V;
  double* wLy = wRx + RY * RX * V;
  double* wRy = wLy + RY * RX * V;
  const int P = a.P, NX = GRID ? P * a.npx : P, NY = GRID ? P * a.npy : P;
  const int k0 = bx * FVP_TX, j0 = by * FVP_TY;  // global cell coordinates
  const int tid = threadIdx.x;
  const double hx = a.hx, hy = a.hy, dt = *a.dt_dev;
  // reciprocal cell sizes: multiplications instead of the reference's
  // divisions (an FP64 division is a long dependent chain)
  const double ihx = 1.0 / hx, ihy = 1.0 / hy;
  if constexpr (GRID) {
    // the staged block's cell offsets as a column part per staged column
    // and a row part per staged row (48 folds instead of one per cell),
    // kept in the ring buffer until the ring phase
    long* offs = reinterpret_cast<long*>(wRy + RY * RX * V);  // [LX] columns, then [LY] rows
    int* flips = reinterpret_cast<int*>(offs + LX + LY);
    int* kpos = flips + LX + LY;  // position in the patch (for in-domain columns and rows)
    const int S = a.S;
    if (tid < LX) {
      bool mx = false;
      const int Xf = fv_fold(k0 - 2 + tid, NX, a.bcx, mx);
      const int px = a.npx == 1 ? 0 : Xf / P;
      offs[tid] = (long)px * S * S + (a.g + Xf - px * P);
      flips[tid] = (mx && a.bcx == EXA_BC_REFLECT) ? 1 : -1;
      kpos[tid] = Xf - px * P;
    } else if (tid < LX + LY) {
      bool my = false;
      const int Yf = fv_fold(j0 - 2 + (tid - LX), NY, a.bcy, my);
      const int py = a.npy == 1 ? 0 : Yf / P;
      offs[tid] = (long)py * a.npx * S * S + (long)(a.g + Yf - py * P) * S;
      flips[tid] = (my && a.bcy == EXA_BC_REFLECT) ? 2 : -1;
      kpos[tid] = Yf - py * P;
    }
    __syncthreads();
    const int D = kV + a.npar;
    for (int i = tid; i < LY * LX; i += FVP_NT) {
      const int r = i / LX, c = i % LX;
      const int flip = flips[c] >= 0 ? flips[c] : flips[LX + r];
      const double* q = a.luh + (offs[c] + offs[LX + r]) * D;
#pragma unroll
      for (int m = 0; m < V; m++) su[i * V + m] = m == flip ? -q[m] : q[m];
    }
  } else {
    for (int i = tid; i < LY * LX; i += FVP_NT) {
      const int r = i / LX, c = i % LX;
      int flip;
      const double* q = a.luh + fv_stencil_offset<GRID>(a, k0 - 2 + c, j0 - 2 + r, &flip);
#pragma unroll
      for (int m = 0; m < V; m++) su[i * V + m] = m == flip ? -q[m] : q[m];
    }
  }
  __syncthreads();
  // ring cells: slopes, extrapolations and the half step.  One patch: a
  // ring cell outside the patch is its ghost (x or y extrapolation only, no
  // half step), as the reference's per-patch loops have it.  Patch grid:
  // every ring cell is evolved as the interior cell of its own patch, and
  // the face phase recomputes the ghost form on patch faces.
  for (int i = tid; i < RY * RX; i += FVP_NT) {
    const int rr = i / RX, rc = i % RX;
    const double* U = &su[((rr + 1) * LX + rc + 1) * V];
    bool has_x = true, has_y = true, interior = true;
    if (!GRID) {
      const int j = j0 - 1 + rr, k = k0 - 1 + rc;
      has_x = j >= 0 && j < P && k >= -1 && k < P + 1;
      has_y = j >= -1 && j < P + 1 && k >= 0 && k < P;
      interior = j >= 0 && j < P && k >= 0 && k < P;
    }
    double lx[V], rx[V], ly[V], ry[V];
#pragma unroll
    for (int m = 0; m < V; m++) { lx[m] = rx[m] = ly[m] = ry[m] = 0.0; }
    if (has_x) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        const double sl = minmod(U[V + m] - U[m], U[m] - U[-V + m]) * ihx;
        lx[m] = U[m] - 0.5 * hx * sl;
        rx[m] = U[m] + 0.5 * hx * sl;
      }
    }
    if (has_y) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        const double sl = minmod(U[LX * V + m] - U[m], U[m] - U[-LX * V + m]) * ihy;
        ly[m] = U[m] - 0.5 * hy * sl;
        ry[m] = U[m] + 0.5 * hy * sl;
      }
    }
    if (interior) {
      double Qt[V];
      double F[2][V];
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] = 0.0;
      euler_flux<2, PLANAR>(lx, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] += F[0][m] * ihx;
      euler_flux<2, PLANAR>(rx, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] -= F[0][m] * ihx;
      euler_flux<2, PLANAR>(ly, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] += F[1][m] * ihy;
      euler_flux<2, PLANAR>(ry, F);
#pragma unroll
      for (int m = 0; m < V; m++) Qt[m] -= F[1][m] * ihy;
#pragma unroll
      for (int m = 0; m < V; m++) {
        lx[m] += 0.5 * dt * Qt[m];
        rx[m] += 0.5 * dt * Qt[m];
        ly[m] += 0.5 * dt * Qt[m];
        ry[m] += 0.5 * dt * Qt[m];
      }
    }
#pragma unroll
    for (int m = 0; m < V; m++) {
      wLx[i * V + m] = lx[m];
      wRx[i * V + m] = rx[m];
      wLy[i * V + m] = ly[m];
      wRy[i * V + m] = ry[m];
    }
  }
  __syncthreads();
  const double cx = dt / hx, cy = dt / hy;
  double dtn = DBL_MAX;
  const int r = tid / FVP_TX, c = tid % FVP_TX;
  const int j = j0 + r, k = k0 + c;
  if (j < NY && k < NX) {
    const int ic = (r + 1) * RX + c + 1;  // this cell in the ring arrays
    const double* U = &su[((r + 2) * LX + c + 2) * V];
    int kx = k, ky = j;  // position in the patch
    double* o;
    if constexpr (GRID) {
      // the staged column c + 2 and row r + 2 are this cell's (in the domain)
      const long* offs = reinterpret_cast<const long*>(wRy + RY * RX * V);
      const int* kpos = reinterpret_cast<const int*>(offs + LX + LY) + LX + LY;
      kx = kpos[c + 2];
      ky = kpos[LX + r + 2];
      o = a.out + (offs[c + 2] + offs[LX + r + 2]) * (kV + a.npar);
    } else {
      o = a.out + fv_cell_offset<GRID>(a, k, j);
    }
    double fxl[V], fxr[V], fyb[V], fyt[V];
    if constexpr (!GRID) {
      rusanov<PLANAR>(&wRx[(ic - 1) * V], &wLx[ic * V], 0, fxl);
      rusanov<PLANAR>(&wRx[ic * V], &wLx[(ic + 1) * V], 0, fxr);
      rusanov<PLANAR>(&wRy[(ic - RX) * V], &wLy[ic * V], 1, fyb);
      rusanov<PLANAR>(&wRy[ic * V], &wLy[(ic + RX) * V], 1, fyt);
      fv_update_store_dt<PLANAR>(a, o, U, fxl, fxr, fyb, fyt, cx, cy, dtn);
    } else {
    double qa[V], qb[V];
    // x faces; across a patch boundary the outer side is the plain
    // extrapolation of the neighbour cell (its ghost image in this patch)
#pragma unroll
    for (int m = 0; m < V; m++) {
      qa[m] = wRx[(ic - 1) * V + m];
      qb[m] = wLx[ic * V + m];
    }
    if (kx == 0) {
      const double* W = U - V;
#pragma unroll
      for (int m = 0; m < V; m++) qa[m] = W[m] + 0.5 * hx * (minmod(W[V + m] - W[m], W[m] - W[-V + m]) * ihx);
    }
    rusanov<PLANAR>(qa, qb, 0, fxl);
#pragma unroll
    for (int m = 0; m < V; m++) {
      qa[m] = wRx[ic * V + m];
      qb[m] = wLx[(ic + 1) * V + m];
    }
    if (kx == P - 1) {
      const double* W = U + V;
#pragma unroll
      for (int m = 0; m < V; m++) qb[m] = W[m] - 0.5 * hx * (minmod(W[V + m] - W[m], W[m] - W[-V + m]) * ihx);
    }
    rusanov<PLANAR>(qa, qb, 0, fxr);
    // y faces
#pragma unroll
    for (int m = 0; m < V; m++) {
      qa[m] = wRy[(ic - RX) * V + m];
      qb[m] = wLy[ic * V + m];
    }
    if (ky == 0) {
      const double* W = U - LX * V;
#pragma unroll
      for (int m = 0; m < V; m++)
        qa[m] = W[m] + 0.5 * hy * (minmod(W[LX * V + m] - W[m], W[m] - W[-LX * V + m]) * ihy);
    }
    rusanov<PLANAR>(qa, qb, 1, fyb);
#pragma unroll
    for (int m = 0; m < V; m++) {
      qa[m] = wRy[ic * V + m];
      qb[m] = wLy[(ic + RX) * V + m];
    }
    if (ky == P - 1) {
      const double* W = U + LX * V;
#pragma unroll
      for (int m = 0; m < V; m++)
        qb[m] = W[m] - 0.5 * hy * (minmod(W[LX * V + m] - W[m], W[m] - W[-LX * V + m]) * ihy);
    }
    rusanov<PLANAR>(qa, qb, 1, fyt);
    fv_update_store_dt<PLANAR>(a, o, U, fxl, fxr, fyb, fyt, cx, cy, dtn);
    }
  }
  for (int o = 16; o > 0; o >>= 1) dtn = fmin(dtn, __shfl_xor_sync(0xffffffffu, dtn, o));
  if ((tid & 31) == 0) atomic_min_pos_double(a.next_dt, dtn);
}

template <bool PLANAR, bool GRID>
__global__ void __launch_bounds__(FVP_NT, 3) k_fv_muscl_periodic(FVArgs a) {
  extern __shared__ double sm[];
  fv_muscl_periodic_tile<PLANAR, GRID>(a, blockIdx.x, blockIdx.y, sm);
}

constexpr size_t kMusclPeriodicSmem =
    sizeof(double) * ((FVP_TY + 4) * (FVP_TX + 4) * kV + 4 * (FVP_TY + 2) * (FVP_TX + 2) * kV);
// the patch grid adds the staged block's offsets, flips and patch positions
constexpr size_t kMusclGridSmem = kMusclPeriodicSmem + ((FVP_TX + 4) + (FVP_TY + 4)) * (8 + 4 + 4);

// --------------------------------------------------------- stable dt
template <bool PLANAR>
__global__ void k_fv_stable_dt(FVArgs a, double* dt_patch, int one_slot) {
  const int D = kV + a.npar, S = a.S, P = a.P, g = a.g;
  const long patch = blockIdx.y;
  const double* luh = a.luh + patch * (long)S * S * D;
  double dtl = DBL_MAX;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (long)P * P; i += (long)gridDim.x * blockDim.x) {
    const int j = g + (int)(i / P), k = g + (int)(i % P);
    const double* q = luh + ((long)j * S + k) * D;
    dtl = fmin(dtl, 0.9 / 2 * a.hx / euler_max_eig<PLANAR>(q, 0));
    dtl = fmin(dtl, 0.9 / 2 * a.hy / euler_max_eig<PLANAR>(q, 1));
  }
  for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
  if ((threadIdx.x & 31) == 0)
    atomic_min_pos_double((unsigned long long*)&dt_patch[one_slot ? 0 : patch], dtl);
}

__global__ void k_fv_ghosts(int P, int g, int D, long npatches, double* luh) {
  const int S = P + 2 * g;
  const long nghost = (long)S * S - (long)P * P;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nghost * npatches) return;
  const long patch = gid / nghost;
  long r = gid % nghost;
  // enumerate ghost cells: rows [0,g) and [g+P,S) fully, then side columns
  int j, k;
  const long top = (long)g * S;
  if (r < top) { j = (int)(r / S); k = (int)(r % S); }
  else if (r < 2 * top) { r -= top; j = g + P + (int)(r / S); k = (int)(r % S); }
  else {
    r -= 2 * top;
    j = g + (int)(r / (2 * g));
    const int c = (int)(r % (2 * g));
    k = c < g ? c : P + c;
  }
  const int sj = g + ((j - g) % P + P) % P, sk = g + ((k - g) % P + P) % P;
  double* base = luh + patch * (long)S * S * D;
  for (int m = 0; m < D; m++) base[((long)j * S + k) * D + m] = base[((long)sj * S + sk) * D + m];
}

static exa_status_t check_fv(const exa_fv_desc_t* d, int want_ghost) {
  if (!d) return set_error(EXA_EINVAL, "NULL descriptor");
  if (d->dim != 2 && d->dim != 3) return set_error(EXA_EINVAL, "dim must be 2 or 3");
  if (d->dim == 3 && d->pde != EXA_PDE_EULER) return set_error(EXA_EINVAL, "3D FV: pde must be EXA_PDE_EULER");
  if (d->nvar != kV || d->npar < 0 || d->npar > 8) return set_error(EXA_EINVAL, "nvar must be 5");
  if (d->patch < 1) return set_error(EXA_EINVAL, "patch must be >= 1");
  if (want_ghost && d->ghost < want_ghost) return set_error(EXA_EINVAL, "ghost layer too thin");
  if (d->pde != EXA_PDE_EULER && d->pde != EXA_PDE_EULER_PLANAR) return set_error(EXA_EINVAL, "pde");
  return ensure_tables();
}

static FVArgs fv_args(const exa_fv_desc_t* d) {
  FVArgs a{};
  a.npx = a.npy = 1;
  a.P = d->patch;
  a.g = d->ghost;
  a.S = d->patch + 2 * d->ghost;
  a.npar = d->npar;
  a.hx = d->dx[0] / d->patch;
  a.hy = d->dx[1] / d->patch;
  return a;
}

exa_status_t upload_tables_fv() { return EXA_OK; }

// Scalars of a device-resident periodic patch (3 x 64 bit):
// [0] dt of the current step, [1] simulated time, [2] next dt (atomic min).
__global__ void k_fv_slots_init(unsigned long long* s) {
  s[0] = 0x7FF0000000000000ULL;
  s[2] = 0x7FF0000000000000ULL;
}

__global__ void k_fv_commit(unsigned long long* s) {
  double* time = (double*)(s + 1);
  *time += __longlong_as_double((long long)s[0]);
  s[0] = s[2];
  s[2] = 0x7FF0000000000000ULL;
}

// ----------------------------------------------------- serving batch
// All live periodic patches of one scheme advanced by one launch: CTA t
// takes global tile t, finds its patch by binary search over the patches'
// first tiles, and runs the same tile body as the single-patch kernels.
__device__ __forceinline__ int fv_serve_find(const FVServePatch* pt, int np, int tile) {
  int lo = 0, hi = np - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pt[mid].tile0 <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ FVArgs fv_serve_args(const FVServePatch& p) {
  FVArgs a{};
  a.npx = a.npy = 1;
  a.P = p.P;
  a.g = p.g;
  a.S = p.P + 2 * p.g;
  a.npar = 0;
  a.hx = p.hx;
  a.hy = p.hy;
  const int par = (int)(p.slots[3] & 1ULL);
  a.luh = p.buf[par];
  a.out = p.buf[par ^ 1];
  a.dt_dev = (const double*)p.slots;
  a.next_dt = p.slots + 2;
  return a;
}

template <bool PLANAR>
__global__ void __launch_bounds__(FVP_NT, 3) k_fv_muscl_serve(const FVServePatch* __restrict__ pt, int np) {
  extern __shared__ double sm[];
  const FVServePatch& p = pt[fv_serve_find(pt, np, blockIdx.x)];
  const FVArgs a = fv_serve_args(p);
  const int t = blockIdx.x - p.tile0;
  fv_muscl_periodic_tile<PLANAR, false>(a, t % p.tiles_x, t / p.tiles_x, sm);
}

template <bool PLANAR>
__global__ void __launch_bounds__(FV_NT, 5) k_fv_godunov_serve(const FVServePatch* __restrict__ pt, int np) {
  const FVServePatch& p = pt[fv_serve_find(pt, np, blockIdx.x)];
  const FVArgs a = fv_serve_args(p);
  const int t = blockIdx.x - p.tile0;
  fv_godunov_tile<PLANAR, true>(a, t % p.tiles_x, t / p.tiles_x, 0);
}

// per patch: time += dt, dt = next dt, next dt = +inf, state buffer flipped
__global__ void k_fv_serve_commit(const FVServePatch* __restrict__ pt, int np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  unsigned long long* s = pt[i].slots;
  double* time = (double*)(s + 1);
  *time += __longlong_as_double((long long)s[0]);
  s[0] = s[2];
  s[2] = 0x7FF0000000000000ULL;
  s[3] ^= 1ULL;
}

int fv_serve_tiles(int scheme, int patch, int* tiles_x) {
  const int tx = scheme == 0 ? FV_TX : FVP_TX, ty = scheme == 0 ? FV_TY : FVP_TY;
  const int nx = (patch + tx - 1) / tx, ny = (patch + ty - 1) / ty;
  if (tiles_x) *tiles_x = nx;
  return nx * ny;
}

exa_status_t fv_serve_step_async(int scheme, bool planar, const FVServePatch* table, int np, int ntiles,
                                 cudaStream_t st) {
  if (np <= 0) return EXA_OK;
  if (scheme == 0) {
    static bool gattr[2] = {false, false};
    if (!gattr[planar]) {
      cudaError_t e = cudaFuncSetAttribute(planar ? k_fv_godunov_serve<true> : k_fv_godunov_serve<false>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return cuda_status(e, "godunov serve attribute");
      gattr[planar] = true;
    }
    if (planar) k_fv_godunov_serve<true><<<ntiles, FV_NT, 0, st>>>(table, np);
    else k_fv_godunov_serve<false><<<ntiles, FV_NT, 0, st>>>(table, np);
  } else {
    static bool attr[2] = {false, false};
    if (!attr[planar]) {
      auto kern = planar ? k_fv_muscl_serve<true> : k_fv_muscl_serve<false>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMusclPeriodicSmem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return cuda_status(e, "muscl serve attribute");
      attr[planar] = true;
    }
    if (planar) k_fv_muscl_serve<true><<<ntiles, FVP_NT, kMusclPeriodicSmem, st>>>(table, np);
    else k_fv_muscl_serve<false><<<ntiles, FVP_NT, kMusclPeriodicSmem, st>>>(table, np);
  }
  k_fv_serve_commit<<<(np + 127) / 128, 128, 0, st>>>(table, np);
  count_launch(2);
  return cuda_status(cudaGetLastError(), "fv serve step");
}

__device__ __forceinline__ double fv_noise_u01(unsigned long long seed, unsigned long long idx) {
  unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (idx + 1ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// cell-centred density sine wave rho = 1 + amp sin(2 pi (x + y)), u = v = 1,
// p = 1, with seeded relative density noise; ghosts are filled by the step
__global__ void k_fv_ic(int P, int g, int D, double hx, double hy, double amp, unsigned long long seed,
                        double noise, double* luh) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int S = P + 2 * g;
  if (i >= (long)S * S) return;
  const int j = (int)(i / S), k = (int)(i % S);
  const double x = (k - g + 0.5) * hx, y = (j - g + 0.5) * hy;
  const double pi = 3.14159265358979323846;
  double rho = 1.0 + amp * sin(2 * pi * (x + y));
  if (noise != 0.0) rho *= 1.0 + noise * (2.0 * fv_noise_u01(seed, (unsigned long long)i) - 1.0);
  double* q = luh + i * D;
  q[0] = rho;
  q[1] = rho;
  q[2] = rho;
  q[3] = 0.0;
  q[4] = 1.0 / (kGamma - 1) + rho;  // p/(g-1) + rho (u^2+v^2)/2 with u = v = 1
  for (int m = kV; m < D; m++) q[m] = 0.0;
}

exa_status_t launch_fv_ic(const exa_fv_desc_t& d, double* luh, double amp, uint64_t seed, double noise,
                          cudaStream_t st) {
  const int S = d.patch + 2 * d.ghost;
  const long n = (long)S * S;
  k_fv_ic<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d.patch, d.ghost, d.nvar + d.npar, d.dx[0] / d.patch,
                                                       d.dx[1] / d.patch, amp, seed, noise, luh);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv_ic");
}

// Device-resident stepping of a single periodic patch.  prime: the CFL dt
// (commons::stableTimeStepSize rule) of the current state into slot [0].
// step: one fused update (periodic tile loads, luh_new = luh + fluxes, next
// dt of the new state into slot [2]), then commit (time += dt, dt <- next).
// No host synchronisation; two launches per step.
exa_status_t fv_patch_prime_async(const exa_fv_desc_t& d, const double* luh, unsigned long long* slots,
                                  cudaStream_t st) {
  FVArgs a = fv_args(&d);
  a.luh = luh;
  k_fv_slots_init<<<1, 1, 0, st>>>(slots);
  const long cells = (long)d.patch * d.patch;
  unsigned bx = (unsigned)((cells + 255) / 256);
  if (bx > 1024) bx = 1024;
  if (d.pde == EXA_PDE_EULER_PLANAR) k_fv_stable_dt<true><<<dim3(bx, 1), 256, 0, st>>>(a, (double*)slots, 0);
  else k_fv_stable_dt<false><<<dim3(bx, 1), 256, 0, st>>>(a, (double*)slots, 0);
  count_launch(2);
  return cuda_status(cudaGetLastError(), "fv prime");
}

exa_status_t fv_patch_step_async(int scheme, const exa_fv_desc_t& d, const double* luh, double* luh_new,
                                 unsigned long long* slots, cudaStream_t st) {
  FVArgs a = fv_args(&d);
  a.luh = luh;
  a.out = luh_new;
  a.dt_dev = (const double*)slots;
  a.next_dt = slots + 2;
  a.max_dt = nullptr;
  const bool planar = d.pde == EXA_PDE_EULER_PLANAR;
  dim3 grid((d.patch + FVP_TX - 1) / FVP_TX, (d.patch + FVP_TY - 1) / FVP_TY, 1);
  if (scheme == 0) {
    // shared face fluxes per tile (k_fv_godunov<..., FUSED>): measured faster
    // for first order than per-cell face fluxes (k_fv_godunov_periodic),
    // whose doubled Riemann work is not paid back by the saved barrier
    dim3 gt((d.patch + FV_TX - 1) / FV_TX, (d.patch + FV_TY - 1) / FV_TY, 1);
    static bool gattr[2] = {false, false};
    if (!gattr[planar]) {
      cudaError_t e = cudaFuncSetAttribute(planar ? k_fv_godunov<true, true> : k_fv_godunov<false, true>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return cuda_status(e, "godunov attribute");
      gattr[planar] = true;
    }
    if (tune_get(kTuneFvGodunov, 0) != 1) {
      const dim3 gs((unsigned)((d.patch + FVS_WARPS * FVS_W - 1) / (FVS_WARPS * FVS_W)),
                    (unsigned)((d.patch + FVS_H - 1) / FVS_H), 1);
      if (planar) k_fv_godunov_sweep<true, false><<<gs, 32 * FVS_WARPS, 0, st>>>(a);
      else k_fv_godunov_sweep<false, false><<<gs, 32 * FVS_WARPS, 0, st>>>(a);
    } else if (planar) {
      k_fv_godunov<true, true><<<gt, FV_NT, 0, st>>>(a);
    } else {
      k_fv_godunov<false, true><<<gt, FV_NT, 0, st>>>(a);
    }
  } else {
    static bool attr[2] = {false, false};
    if (!attr[planar]) {
      auto kern = planar ? k_fv_muscl_periodic<true, false> : k_fv_muscl_periodic<false, false>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMusclPeriodicSmem);
      // three CTAs of ~72 KB per SM need the largest shared-memory carveout
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return cuda_status(e, "muscl attribute");
      attr[planar] = true;
    }
    if (planar) k_fv_muscl_periodic<true, false><<<grid, FVP_NT, kMusclPeriodicSmem, st>>>(a);
    else k_fv_muscl_periodic<false, false><<<grid, FVP_NT, kMusclPeriodicSmem, st>>>(a);
  }
  k_fv_commit<<<1, 1, 0, st>>>(slots);
  count_launch(2);
  return cuda_status(cudaGetLastError(), "fv patch step");
}

template <bool PLANAR>
__global__ void k_rusanov_one(int d, const double* qL, const double* qR, double* out) {
  // out = [f (5 values), s_max]; the 2D/3D flux only differs in the
  // direction index, so the 3D case evaluates the flux with DIM = 3
  double f[kV];
  const double s = rusanov<PLANAR>(qL, qR, d > 1 ? 0 : d, f);
  if (d > 1) {
    const double sm = fmax(euler_max_eig<PLANAR>(qL, d), euler_max_eig<PLANAR>(qR, d));
    double FL[3][kV], FR[3][kV];
    euler_flux<3, PLANAR>(qL, FL);
    euler_flux<3, PLANAR>(qR, FR);
    for (int i = 0; i < kV; i++) {
      double v = 0.5 * sm * (qL[i] - qR[i]);
      v += 0.5 * (FL[d][i] + FR[d][i]);
      out[i] = v;
    }
    out[kV] = sm;
    return;
  }
  for (int i = 0; i < kV; i++) out[i] = f[i];
  out[kV] = s;
}

exa_status_t launch_rusanov_one(int pde, int d, const double* qL, const double* qR, double* out) {
  if (pde == EXA_PDE_EULER_PLANAR) k_rusanov_one<true><<<1, 1>>>(d, qL, qR, out);
  else k_rusanov_one<false><<<1, 1>>>(d, qL, qR, out);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_rusanov_one");
}

}  // namespace exa

using namespace exa;

extern "C" {

static exa_status_t fv_update(int scheme, const exa_fv_desc_t* desc, long npatches, double* luh_new,
                              const double* luh, double dt, double* max_dt, void* stream) {
  if (exa_status_t s = check_fv(desc, scheme == 0 ? 1 : 2)) return s;
  if (npatches < 0 || !luh_new || !luh) return set_error(EXA_EINVAL, "bad argument");
  if (npatches == 0) return EXA_OK;
  if (npatches > 65535) return set_error(EXA_EINVAL, "at most 65535 patches per call");
  cudaStream_t st = as_stream(stream);
  if (desc->dim == 3) {
    if (max_dt) {
      std::vector<unsigned long long> inf(npatches, 0x7FF0000000000000ULL);
      cudaError_t e = cudaMemcpyAsync(max_dt, inf.data(), 8 * npatches, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return cuda_status(e, "max_dt init");
    }
    const double h[3] = {desc->dx[0] / desc->patch, desc->dx[1] / desc->patch, desc->dx[2] / desc->patch};
    return fv3_update(scheme, desc->patch, desc->ghost, desc->nvar + desc->npar, h, npatches, luh_new, luh, dt,
                      nullptr, max_dt, nullptr, nullptr, st);
  }
  FVArgs a = fv_args(desc);
  a.dt = dt;
  a.luh = luh;
  a.out = luh_new;
  a.max_dt = (unsigned long long*)max_dt;
  if (max_dt) {
    // +inf bit pattern 0x7FF0000000000000 = bytes 00..00 F0 7F
    std::vector<unsigned long long> inf(npatches, 0x7FF0000000000000ULL);
    cudaError_t e = cudaMemcpyAsync(max_dt, inf.data(), 8 * npatches, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "max_dt init");
  }
  dim3 grid((desc->patch + FV_TX - 1) / FV_TX, (desc->patch + FV_TY - 1) / FV_TY, (unsigned)npatches);
  const bool planar = desc->pde == EXA_PDE_EULER_PLANAR;
  if (scheme == 0) {
    if (planar) k_fv_godunov<true, false><<<grid, FV_NT, 0, st>>>(a);
    else k_fv_godunov<false, false><<<grid, FV_NT, 0, st>>>(a);
  } else {
    static bool attr[2] = {false, false};
    if (!attr[planar]) {
      cudaError_t e = planar ? cudaFuncSetAttribute(k_fv_muscl<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMusclSmem)
                             : cudaFuncSetAttribute(k_fv_muscl<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMusclSmem);
      if (e != cudaSuccess) return cuda_status(e, "muscl attribute");
      attr[planar] = true;
    }
    if (planar) k_fv_muscl<true, false><<<grid, FV_NT, kMusclSmem, st>>>(a);
    else k_fv_muscl<false, false><<<grid, FV_NT, kMusclSmem, st>>>(a);
  }
  count_launch();
  return cuda_status(cudaGetLastError(), scheme == 0 ? "k_fv_godunov" : "k_fv_muscl");
}

exa_status_t exa_fv_godunov_update(const exa_fv_desc_t* desc, long npatches, double* luh_new,
                                   const double* luh, double dt, double* max_dt, void* stream) {
  return fv_update(0, desc, npatches, luh_new, luh, dt, max_dt, stream);
}

exa_status_t exa_fv_musclhancock_update(const exa_fv_desc_t* desc, long npatches, double* luh_new,
                                        const double* luh, double dt, double* max_dt, void* stream) {
  return fv_update(1, desc, npatches, luh_new, luh, dt, max_dt, stream);
}

exa_status_t exa_fv_stable_dt(const exa_fv_desc_t* desc, long npatches, const double* luh,
                              double* dt_patch, void* stream) {
  if (exa_status_t s = check_fv(desc, 0)) return s;
  if (npatches < 0 || !luh || !dt_patch) return set_error(EXA_EINVAL, "bad argument");
  if (npatches == 0) return EXA_OK;
  cudaStream_t st = as_stream(stream);
  std::vector<unsigned long long> inf(npatches, 0x7FF0000000000000ULL);
  cudaError_t e = cudaMemcpyAsync(dt_patch, inf.data(), 8 * npatches, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "dt init");
  if (desc->dim == 3) {
    const double h[3] = {desc->dx[0] / desc->patch, desc->dx[1] / desc->patch, desc->dx[2] / desc->patch};
    return fv3_stable_dt(desc->patch, desc->ghost, desc->nvar + desc->npar, h, npatches, luh, dt_patch, st);
  }
  FVArgs a = fv_args(desc);
  a.luh = luh;
  const long cells = (long)desc->patch * desc->patch;
  unsigned bx = (unsigned)((cells + 255) / 256);
  if (bx > 1024) bx = 1024;
  dim3 grid(bx, (unsigned)npatches);
  if (desc->pde == EXA_PDE_EULER_PLANAR) k_fv_stable_dt<true><<<grid, 256, 0, st>>>(a, dt_patch, 0);
  else k_fv_stable_dt<false><<<grid, 256, 0, st>>>(a, dt_patch, 0);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv_stable_dt");
}

exa_status_t exa_fv_periodic_ghosts(const exa_fv_desc_t* desc, long npatches, double* luh, void* stream) {
  if (exa_status_t s = check_fv(desc, 0)) return s;
  if (npatches < 0 || !luh) return set_error(EXA_EINVAL, "bad argument");
  if (desc->dim == 3) {
    if (npatches == 0) return EXA_OK;
    return fv3_periodic_ghosts(desc->patch, desc->ghost, desc->nvar + desc->npar, npatches, luh, as_stream(stream));
  }
  const int S = desc->patch + 2 * desc->ghost;
  const long work = ((long)S * S - (long)desc->patch * desc->patch) * npatches;
  if (work == 0) return EXA_OK;
  k_fv_ghosts<<<(unsigned)((work + 255) / 256), 256, 0, as_stream(stream)>>>(
      desc->patch, desc->ghost, desc->nvar + desc->npar, npatches, luh);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv_ghosts");
}

// ------------------------------------------------ device-resident FV domain
}  // extern "C"

struct exa_fv_grid {
  int scheme = 0;
  exa_fv_desc_t desc{};
  cudaStream_t st = nullptr;
  double* luh = nullptr;
  double* luh_new = nullptr;
  unsigned long long* slots = nullptr;  // [0] dt, [1] time, [2] next dt, [3] steps
  size_t count = 0;                     // doubles per state copy
  bool primed = false;
};

extern "C" {

exa_status_t exa_fv_grid_create(int scheme, int patch, double length, int pde, exa_fv_grid** out) {
  if (!out) return set_error(EXA_EINVAL, "NULL argument");
  if (scheme != 0 && scheme != 1) return set_error(EXA_EINVAL, "scheme must be 0 (Godunov) or 1 (MUSCL-Hancock)");
  if (!(length > 0)) return set_error(EXA_EINVAL, "length must be > 0");
  exa_fv_desc_t d{2, patch, scheme == 0 ? 1 : 2, kV, 0, pde, {length, length, 1.0}};
  if (exa_status_t s = check_fv(&d, d.ghost)) return s;
  exa_fv_grid* g = new (std::nothrow) exa_fv_grid;
  if (!g) return set_error(EXA_ENOMEM, "host allocation");
  g->scheme = scheme;
  g->desc = d;
  const size_t S = (size_t)patch + 2 * d.ghost;
  g->count = S * S * kV;
  cudaError_t e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->luh, g->count * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&g->luh_new, g->count * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&g->slots, 4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(g->luh, 0, g->count * sizeof(double), g->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->luh_new, 0, g->count * sizeof(double), g->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->slots, 0, 4 * sizeof(unsigned long long), g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) {
    exa_fv_grid_destroy(g);
    return cuda_status(e, "fv grid allocation");
  }
  *out = g;
  return EXA_OK;
}

exa_status_t exa_fv_grid_destroy(exa_fv_grid* g) {
  if (!g) return EXA_OK;
  if (g->st) cudaStreamSynchronize(g->st);
  cudaFree(g->luh);
  cudaFree(g->luh_new);
  cudaFree(g->slots);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
  return EXA_OK;
}

size_t exa_fv_grid_state_size(const exa_fv_grid* g) { return g ? g->count : 0; }

exa_status_t exa_fv_grid_init(exa_fv_grid* g, double amp, uint64_t seed, double noise) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  if (exa_status_t s = launch_fv_ic(g->desc, g->luh, amp, seed, noise, g->st)) return s;
  g->primed = false;
  // both buffers hold the state: the steps write interiors only, so the
  // ghost cells of a stepped state are the initial ones in either buffer
  cudaError_t e = cudaMemcpyAsync(g->luh_new, g->luh, g->count * sizeof(double), cudaMemcpyDeviceToDevice, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "fv grid init");
}

exa_status_t exa_fv_grid_set_state(exa_fv_grid* g, const double* host) {
  if (!g || !host) return set_error(EXA_EINVAL, "NULL argument");
  cudaError_t e = cudaMemcpyAsync(g->luh, host, g->count * sizeof(double), cudaMemcpyHostToDevice, g->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->luh_new, g->luh, g->count * sizeof(double), cudaMemcpyDeviceToDevice, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  g->primed = false;
  return cuda_status(e, "fv grid set_state");
}

exa_status_t exa_fv_grid_get_state(exa_fv_grid* g, double* host) {
  if (!g || !host) return set_error(EXA_EINVAL, "NULL argument");
  cudaError_t e = cudaMemcpyAsync(host, g->luh, g->count * sizeof(double), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "fv grid get_state");
}

exa_status_t exa_fv_grid_step(exa_fv_grid* g, int nsteps) {
  if (!g || nsteps < 0) return set_error(EXA_EINVAL, "bad argument");
  if (!g->primed) {
    if (exa_status_t s = fv_patch_prime_async(g->desc, g->luh, g->slots, g->st)) return s;
    g->primed = true;
  }
  for (int i = 0; i < nsteps; i++) {
    if (exa_status_t s = fv_patch_step_async(g->scheme, g->desc, g->luh, g->luh_new, g->slots, g->st))
      return s;
    std::swap(g->luh, g->luh_new);
  }
  return EXA_OK;
}

exa_status_t exa_fv_grid_status(exa_fv_grid* g, double* time, double* dt_next) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  unsigned long long h[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(h, g->slots, 16, cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) return cuda_status(e, "fv grid status");
  double t, dt;
  memcpy(&dt, &h[0], 8);
  memcpy(&t, &h[1], 8);
  if (time) *time = t;
  if (dt_next) *dt_next = g->primed ? dt : 0.0;
  return EXA_OK;
}

exa_status_t exa_fv_grid_stream(exa_fv_grid* g, void** stream) {
  if (!g || !stream) return set_error(EXA_EINVAL, "NULL argument");
  *stream = g->st;
  return EXA_OK;
}

exa_status_t exa_fv_grid_device_state(exa_fv_grid* g, double** luh_dev) {
  if (!g || !luh_dev) return set_error(EXA_EINVAL, "NULL argument");
  *luh_dev = g->luh;
  return EXA_OK;
}

}  // extern "C"

// ----------------------------------------------- grid of periodic patches
// The reference's finite-volume layout: a uniform grid of cells, each with
// its own patch of patch^2 subcells and g ghost layers; per step the ghost
// layers facing a neighbour are copied from the neighbour's boundary layers
// (ghostLayerFilling, kernels/finitevolumes/commons/c/commons.cpph:337-405,
// called per face by FiniteVolumesSolver::mergeNeighbours,
// FiniteVolumesSolver.cpp:659-686; corner ghosts are not filled there and
// the stencils never read them), then every patch takes the same
// Godunov / MUSCL-Hancock step with the global minimum dt.  Here the patch
// grid is periodic, npx x npy patches stored back to back (patch-major,
// x fastest), which is the batched FV entry points' layout.
namespace exa {

// one thread per face-ghost cell of every patch; at a domain-boundary face
// (bcx / bcy != 0) the ghosts mirror the patch's own boundary layers, ghost k
// <- interior g - 1 - k counted from the face (FiniteVolumesSolver::
// mergeWithBoundaryData, commons.cpph:99-340), the normal momentum negated
// for a reflecting wall
__global__ void k_fv_patch_exchange(int P, int g, int D, int npx, int npy, int bcx, int bcy, double* luh) {
  const int S = P + 2 * g;
  const long per = 4L * g * P;  // face ghosts per patch: left, right, bottom, top
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= per * npx * npy) return;
  const long patch = gid / per;
  const int r = (int)(gid % per);
  const int side = r / (g * P), i = (r / g) % P, k = r % g;  // i along the face, k across
  const int px = (int)(patch % npx), py = (int)(patch / npx);
  // destination (j, x) and source (nj, nx) in patch (qx, qy)
  int j, x, nj, nx, qx = px, qy = py, flip = -1;
  if (side == 0) {        // left ghosts <- left neighbour's right boundary layer
    j = g + i; x = k; nj = j;
    if (bcx && px == 0) { nx = 2 * g - 1 - k; flip = bcx == EXA_BC_REFLECT ? 1 : -1; }
    else { qx = (px + npx - 1) % npx; nx = P + k; }
  } else if (side == 1) { // right ghosts <- right neighbour's left boundary layer
    j = g + i; x = g + P + k; nj = j;
    if (bcx && px == npx - 1) { nx = g + P - 1 - k; flip = bcx == EXA_BC_REFLECT ? 1 : -1; }
    else { qx = (px + 1) % npx; nx = g + k; }
  } else if (side == 2) { // bottom ghosts <- lower neighbour's top boundary layer
    j = k; x = g + i; nx = x;
    if (bcy && py == 0) { nj = 2 * g - 1 - k; flip = bcy == EXA_BC_REFLECT ? 2 : -1; }
    else { qy = (py + npy - 1) % npy; nj = P + k; }
  } else {                // top ghosts <- upper neighbour's bottom boundary layer
    j = g + P + k; x = g + i; nx = x;
    if (bcy && py == npy - 1) { nj = g + P - 1 - k; flip = bcy == EXA_BC_REFLECT ? 2 : -1; }
    else { qy = (py + 1) % npy; nj = g + k; }
  }
  const long src_patch = (long)qy * npx + qx;
  double* dst = luh + (patch * S * S + (long)j * S + x) * D;
  const double* src = luh + (src_patch * S * S + (long)nj * S + nx) * D;
  for (int m = 0; m < D; m++) dst[m] = m == flip ? -src[m] : src[m];
}

// density sine wave of the whole domain on every patch (global coordinates
// and noise index), ghosts included
__global__ void k_fv_patch_ic(int P, int g, int D, int npx, int npy, double hx, double hy, double amp,
                              unsigned long long seed, double noise, double* luh) {
  const int S = P + 2 * g;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)S * S * npx * npy) return;
  const long patch = gid / ((long)S * S);
  const int c = (int)(gid % ((long)S * S));
  const int j = c / S, k = c % S;
  const int px = (int)(patch % npx), py = (int)(patch / npx);
  const double x = (px * P + k - g + 0.5) * hx, y = (py * P + j - g + 0.5) * hy;
  const double pi = 3.14159265358979323846;
  double rho = 1.0 + amp * sin(2 * pi * (x + y));
  if (noise != 0.0) rho *= 1.0 + noise * (2.0 * fv_noise_u01(seed, (unsigned long long)gid) - 1.0);
  double* q = luh + gid * D;
  q[0] = rho;
  q[1] = rho;
  q[2] = rho;
  q[3] = 0.0;
  q[4] = 1.0 / (kGamma - 1) + rho;
  for (int m = kV; m < D; m++) q[m] = 0.0;
}

}  // namespace exa

namespace exa {
// Small patches (patch <= 16, the subcell patches of the limiting ADER-DG
// grid, stepped for a list of troubled cells): one CTA of 128 threads per
// patch.  The whole patch with its ghosts (contiguous in
// memory) is staged in shared memory, MUSCL-Hancock's ring cells compute
// their evolved face extrapolations, and every interior cell evaluates its
// own four face fluxes, applies them in the reference's order and writes
// only the interior of the output; the new state's CFL dt is reduced in the
// same pass.  Same arithmetic per cell as the tile kernels.
constexpr int FVS_NT = 128;
constexpr int kFvSmallMax = 16;

template <bool PLANAR, int SCHEME>
__global__ void __launch_bounds__(FVS_NT) k_fv_patch_small(FVArgs a) {
  constexpr int V = kV;
  extern __shared__ double sm[];
  const int P = a.P, g = a.g, S = a.S, D = V + a.npar, pb = g, pe = g + P;
  const int R = P + 2;  // ring side (MUSCL)
  constexpr int C = kV + 1;
  double* su = sm;       // [S][S][V]
  double* wLx = su + S * S * V;
  double* wRx = wLx + R * R * V;
  double* wLy = wRx + R * R * V;
  double* wRy = wLy + R * R * V;
  // Godunov: per-cell [F_d, lambda_d] (x: rows pb..pe-1, columns pb-1..pe;
  // y: rows pb-1..pe, columns pb..pe-1); MUSCL-Hancock: one Rusanov flux
  // per face (x: [P][P+1], y: [P+1][P])
  double* scx = su + S * S * V;
  double* scy = scx + P * R * C;
  double* sfx = wRy + R * R * V;
  double* sfy = sfx + P * (P + 1) * V;
  // one patch per iteration: patch blockIdx.x, or with a selection the
  // entries blockIdx.x, blockIdx.x + gridDim.x, ... of the list
  const long npatch = a.count ? (long)*a.count : (long)gridDim.x;
  for (long e = blockIdx.x; e < npatch; e += gridDim.x) {
    const long patch = a.list ? (long)a.list[e] : e;
    const double* luh = a.luh + patch * (long)S * S * D;
    double* out = a.out + patch * (long)S * S * D;
    const int tid = threadIdx.x;
    const double hx = a.hx, hy = a.hy, dt = *a.dt_dev;
    // reciprocal cell sizes: multiplications instead of the reference's
    // divisions (an FP64 division is a long dependent chain)
    const double ihx = 1.0 / hx, ihy = 1.0 / hy;
    for (int i = tid; i < S * S * V; i += FVS_NT) su[i] = luh[i];  // D == V: no parameters here
    __syncthreads();
    if (SCHEME == 1) {
      for (int i = tid; i < R * R; i += FVS_NT) {
        const int j = pb - 1 + i / R, k = pb - 1 + i % R;
        const double* U = &su[(j * S + k) * V];
        const bool has_x = j >= pb && j < pe;
        const bool has_y = k >= pb && k < pe;
        const bool interior = has_x && has_y;
        double lx[V], rx[V], ly[V], ry[V];
  #pragma unroll
        for (int m = 0; m < V; m++) { lx[m] = rx[m] = ly[m] = ry[m] = 0.0; }
        if (has_x) {
  #pragma unroll
          for (int m = 0; m < V; m++) {
            const double sl = minmod(U[V + m] - U[m], U[m] - U[-V + m]) * ihx;
            lx[m] = U[m] - 0.5 * hx * sl;
            rx[m] = U[m] + 0.5 * hx * sl;
          }
        }
        if (has_y) {
  #pragma unroll
          for (int m = 0; m < V; m++) {
            const double sl = minmod(U[S * V + m] - U[m], U[m] - U[-S * V + m]) * ihy;
            ly[m] = U[m] - 0.5 * hy * sl;
            ry[m] = U[m] + 0.5 * hy * sl;
          }
        }
        if (interior) {
          double Qt[V];
          double F[2][V];
  #pragma unroll
          for (int m = 0; m < V; m++) Qt[m] = 0.0;
          euler_flux<2, PLANAR>(lx, F);
  #pragma unroll
          for (int m = 0; m < V; m++) Qt[m] += F[0][m] * ihx;
          euler_flux<2, PLANAR>(rx, F);
  #pragma unroll
          for (int m = 0; m < V; m++) Qt[m] -= F[0][m] * ihx;
          euler_flux<2, PLANAR>(ly, F);
  #pragma unroll
          for (int m = 0; m < V; m++) Qt[m] += F[1][m] * ihy;
          euler_flux<2, PLANAR>(ry, F);
  #pragma unroll
          for (int m = 0; m < V; m++) Qt[m] -= F[1][m] * ihy;
  #pragma unroll
          for (int m = 0; m < V; m++) {
            lx[m] += 0.5 * dt * Qt[m];
            rx[m] += 0.5 * dt * Qt[m];
            ly[m] += 0.5 * dt * Qt[m];
            ry[m] += 0.5 * dt * Qt[m];
          }
        }
  #pragma unroll
        for (int m = 0; m < V; m++) {
          wLx[i * V + m] = lx[m];
          wRx[i * V + m] = rx[m];
          wLy[i * V + m] = ly[m];
          wRy[i * V + m] = ry[m];
        }
      }
      __syncthreads();
      // each face's Rusanov flux once (the reference solves every face once)
      for (int i = tid; i < 2 * P * (P + 1); i += FVS_NT) {
        if (i < P * (P + 1)) {
          const int r = i / (P + 1), c = i % (P + 1);  // face left of column pb + c, row pb + r
          const int ic = (r + 1) * R + c + 1;
          rusanov<PLANAR>(&wRx[(ic - 1) * V], &wLx[ic * V], 0, &sfx[i * V]);
        } else {
          const int i2 = i - P * (P + 1);
          const int r = i2 / P, c = i2 % P;  // face below row pb + r, column pb + c
          const int ic = (r + 1) * R + c + 1;
          rusanov<PLANAR>(&wRy[(ic - R) * V], &wLy[ic * V], 1, &sfy[i2 * V]);
        }
      }
      __syncthreads();
    } else {
      // per-cell flux and eigenvalue bound, once per cell and direction
      for (int i = tid; i < 2 * P * R; i += FVS_NT) {
        if (i < P * R) {
          const int j = pb + i / R, k = pb - 1 + i % R;
          fv_cell_flux<PLANAR>(&su[(j * S + k) * V], 0, &scx[i * C]);
        } else {
          const int i2 = i - P * R;
          const int j = pb - 1 + i2 / P, k = pb + i2 % P;
          fv_cell_flux<PLANAR>(&su[(j * S + k) * V], 1, &scy[i2 * C]);
        }
      }
      __syncthreads();
    }
    const double cx = dt / hx, cy = dt / hy;
    double dtn = DBL_MAX;
    for (int i = tid; i < P * P; i += FVS_NT) {
      const int j = pb + i / P, k = pb + i % P;
      const int r = i / P, c = i % P;
      const double* U = &su[(j * S + k) * V];
      double fxl[V], fxr[V], fyb[V], fyt[V];
      if (SCHEME == 0) {
        const double* xl = &scx[(r * R + c) * C];  // cells k-1, k, k+1 of row j
        fv_face_flux(U - V, U, xl, xl + C, fxl);
        fv_face_flux(U, U + V, xl + C, xl + 2 * C, fxr);
        const double* yb = &scy[(r * P + c) * C];  // cells j-1, j, j+1 of column k
        fv_face_flux(U - S * V, U, yb, yb + P * C, fyb);
        fv_face_flux(U, U + S * V, yb + P * C, yb + 2 * P * C, fyt);
      } else {
#pragma unroll
        for (int m = 0; m < V; m++) {
          fxl[m] = sfx[(r * (P + 1) + c) * V + m];
          fxr[m] = sfx[(r * (P + 1) + c + 1) * V + m];
          fyb[m] = sfy[(r * P + c) * V + m];
          fyt[m] = sfy[((r + 1) * P + c) * V + m];
        }
      }
      fv_update_store_dt<PLANAR>(a, out + ((long)j * S + k) * D, U, fxl, fxr, fyb, fyt, cx, cy, dtn);
    }
    for (int o = 16; o > 0; o >>= 1) dtn = fmin(dtn, __shfl_xor_sync(0xffffffffu, dtn, o));
    if ((tid & 31) == 0 && a.next_dt) atomic_min_pos_double(a.next_dt, dtn);
    __syncthreads();
  }
}

inline size_t fv_small_smem(int P, int g, int scheme) {
  const size_t S = P + 2 * g, R = P + 2;
  return sizeof(double) * (S * S * kV + (scheme == 1 ? 4 * R * R * kV + 2 * P * (P + 1) * kV
                                                     : 2 * P * R * (kV + 1)));
}

// Subcell patches of the limiting ADER-DG grid: patch `cell` of a periodic
// npx x npy grid of cells.  Face ghosts of the listed patches from the face
// neighbours' boundary layers (grid-stride over list entries x ghosts).
// at a domain-boundary face (bcx / bcy != 0) the ghosts mirror the patch's
// own boundary layers, ghost k <- interior g - 1 - k counted from the face
// (FiniteVolumesSolver::mergeWithBoundaryData with commons.cpph:175-340),
// the normal momentum negated for a reflecting wall
__global__ void k_fv_subcell_exchange(int P, int g, int npx, int npy, int bcx, int bcy, double* lim,
                                      const int* list, const int* count) {
  const int S = P + 2 * g;
  const long per = 4L * g * P;
  const long total = (long)*count * per;
  for (long gid = (long)blockIdx.x * blockDim.x + threadIdx.x; gid < total; gid += (long)gridDim.x * blockDim.x) {
    const long patch = list[gid / per];
    const int r = (int)(gid % per);
    const int side = r / (g * P), i = (r / g) % P, k = r % g;
    const int px = (int)(patch % npx), py = (int)(patch / npx);
    int j, x, nj, nx, qx = px, qy = py, flip = -1;
    if (side == 0) {
      j = g + i; x = k; nj = j;
      if (bcx && px == 0) { nx = 2 * g - 1 - k; flip = bcx == EXA_BC_REFLECT ? 1 : -1; }
      else { qx = (px + npx - 1) % npx; nx = P + k; }
    } else if (side == 1) {
      j = g + i; x = g + P + k; nj = j;
      if (bcx && px == npx - 1) { nx = g + P - 1 - k; flip = bcx == EXA_BC_REFLECT ? 1 : -1; }
      else { qx = (px + 1) % npx; nx = g + k; }
    } else if (side == 2) {
      j = k; x = g + i; nx = x;
      if (bcy && py == 0) { nj = 2 * g - 1 - k; flip = bcy == EXA_BC_REFLECT ? 2 : -1; }
      else { qy = (py + npy - 1) % npy; nj = P + k; }
    } else {
      j = g + P + k; x = g + i; nx = x;
      if (bcy && py == npy - 1) { nj = g + P - 1 - k; flip = bcy == EXA_BC_REFLECT ? 2 : -1; }
      else { qy = (py + 1) % npy; nj = g + k; }
    }
    const long src_patch = (long)qy * npx + qx;
    double* dst = lim + (patch * S * S + (long)j * S + x) * kV;
    const double* src = lim + (src_patch * S * S + (long)nj * S + nx) * kV;
#pragma unroll
    for (int m = 0; m < kV; m++) dst[m] = m == flip ? -src[m] : src[m];
  }
}

exa_status_t fv_subcell_step(int scheme, int planar, int P, int g, int npx, int npy, double hx, double hy,
                             double* lim, const int* list, const int* count, long maxcells, const double* dt_dev,
                             cudaStream_t st, const int* bc) {
  if (P > kFvSmallMax || (scheme == 0 && g < 1) || (scheme == 1 && g < 2))
    return set_error(EXA_EINVAL, "subcell FV: patch too large or ghost layer too thin");
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  k_fv_subcell_exchange<<<(unsigned)(8 * sms), 256, 0, st>>>(P, g, npx, npy, bc ? bc[0] : 0, bc ? bc[1] : 0, lim,
                                                              list, count);
  count_launch();
  if (exa_status_t s = cuda_status(cudaGetLastError(), "k_fv_subcell_exchange")) return s;
  FVArgs a{};
  a.P = P;
  a.g = g;
  a.S = P + 2 * g;
  a.hx = hx;
  a.hy = hy;
  a.dt_dev = dt_dev;
  a.luh = lim;
  a.out = lim;  // in place: each CTA stages its patch before it writes the interior
  a.list = list;
  a.count = count;
  const size_t smem = fv_small_smem(P, g, scheme);
  auto kern = scheme == 0 ? (planar ? k_fv_patch_small<true, 0> : k_fv_patch_small<false, 0>)
                          : (planar ? k_fv_patch_small<true, 1> : k_fv_patch_small<false, 1>);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e, "subcell FV attribute");
  const long grid = maxcells < 16L * sms ? maxcells : 16L * sms;  // CTAs loop over the listed patches
  kern<<<(unsigned)grid, FVS_NT, smem, st>>>(a);
  count_launch();
  return cuda_status(cudaGetLastError(), "k_fv_patch_small (subcells)");
}
}  // namespace exa

struct exa_fv_patchgrid {
  int scheme = 0, npx = 0, npy = 0;
  exa_fv_desc_t desc{};
  cudaStream_t st = nullptr;
  double* luh = nullptr;
  double* luh_new = nullptr;
  unsigned long long* slots = nullptr;  // [0] dt, [1] time, [2] next dt, [3] last dt
  size_t count = 0;
  long npatches = 0;
  bool primed = false;  // slot [0] holds the CFL dt of the current state
  int bc[2] = {0, 0};   // EXA_BC_* per dimension
};

namespace exa {
// fused patch-grid steps: time += dt, last <- dt, dt <- next, next <- +inf
__global__ void k_fv_patch_commit(unsigned long long* s) {
  double* time = (double*)(s + 1);
  *time += __longlong_as_double((long long)s[0]);
  s[3] = s[0];
  s[0] = s[2];
  s[2] = 0x7FF0000000000000ULL;
}
}  // namespace exa

// One step of the patch grid: one fused tile launch over the global cell
// view (a ghost cell is read as the neighbour cell it would hold after the
// exchange, so no exchange pass), the next dt reduced in the same pass, and
// the commit rotating the dt slots.  The CFL dt of a state that was set or
// initialised is reduced once first.
static exa_status_t fv_patchgrid_step_one(exa_fv_patchgrid* g) {
  using namespace exa;
  const exa_fv_desc_t& d = g->desc;
  const bool planar = d.pde == EXA_PDE_EULER_PLANAR;
  const int S = d.patch + 2 * d.ghost;
  FVArgs a = fv_args(&d);
  a.npx = g->npx;
  a.npy = g->npy;
  a.bcx = g->bc[0];
  a.bcy = g->bc[1];
  if (!g->primed) {
    k_fv_slots_init<<<1, 1, 0, g->st>>>(g->slots);
    count_launch();
    const long per0 = (long)S * S * kV;
    const long cells = (long)d.patch * d.patch;
    unsigned bx = (unsigned)((cells + 255) / 256);
    if (bx > 64) bx = 64;
    for (long p0 = 0; p0 < g->npatches; p0 += 65535) {
      const unsigned np = (unsigned)(g->npatches - p0 < 65535 ? g->npatches - p0 : 65535);
      a.luh = g->luh + p0 * per0;
      if (planar) k_fv_stable_dt<true><<<dim3(bx, np), 256, 0, g->st>>>(a, (double*)g->slots, 1);
      else k_fv_stable_dt<false><<<dim3(bx, np), 256, 0, g->st>>>(a, (double*)g->slots, 1);
      count_launch();
    }
    if (exa_status_t s = cuda_status(cudaGetLastError(), "fv patch grid dt")) return s;
    g->primed = true;
  }
  a.luh = g->luh;
  a.out = g->luh_new;
  a.dt_dev = (const double*)g->slots;
  a.next_dt = g->slots + 2;
  a.max_dt = nullptr;
  const long NX = (long)d.patch * g->npx, NY = (long)d.patch * g->npy;
  if (g->scheme == 0) {
    static bool gattr[2] = {false, false};
    if (!gattr[planar]) {
      cudaError_t e = cudaFuncSetAttribute(planar ? k_fv_godunov<true, true, true> : k_fv_godunov<false, true, true>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return cuda_status(e, "godunov attribute");
      gattr[planar] = true;
    }
    if (tune_get(kTuneFvGodunov, 0) != 1) {
      const dim3 gs((unsigned)((NX + FVS_WARPS * FVS_W - 1) / (FVS_WARPS * FVS_W)),
                    (unsigned)((NY + FVS_H - 1) / FVS_H), 1);
      if (planar) k_fv_godunov_sweep<true, true><<<gs, 32 * FVS_WARPS, 0, g->st>>>(a);
      else k_fv_godunov_sweep<false, true><<<gs, 32 * FVS_WARPS, 0, g->st>>>(a);
    } else {
      const dim3 grid((unsigned)((NX + FV_TX - 1) / FV_TX), (unsigned)((NY + FV_TY - 1) / FV_TY), 1);
      if (planar) k_fv_godunov<true, true, true><<<grid, FV_NT, 0, g->st>>>(a);
      else k_fv_godunov<false, true, true><<<grid, FV_NT, 0, g->st>>>(a);
    }
  } else {
    static bool attr[2] = {false, false};
    if (!attr[planar]) {
      auto kern = planar ? k_fv_muscl_periodic<true, true> : k_fv_muscl_periodic<false, true>;
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMusclGridSmem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return cuda_status(e, "muscl attribute");
      attr[planar] = true;
    }
    const dim3 grid((unsigned)((NX + FVP_TX - 1) / FVP_TX), (unsigned)((NY + FVP_TY - 1) / FVP_TY), 1);
    if (planar) k_fv_muscl_periodic<true, true><<<grid, FVP_NT, kMusclGridSmem, g->st>>>(a);
    else k_fv_muscl_periodic<false, true><<<grid, FVP_NT, kMusclGridSmem, g->st>>>(a);
  }
  k_fv_patch_commit<<<1, 1, 0, g->st>>>(g->slots);
  count_launch(2);
  std::swap(g->luh, g->luh_new);
  return cuda_status(cudaGetLastError(), "fv patch grid step");
}

extern "C" {

exa_status_t exa_fv_patchgrid_create(int scheme, int patch, int npx, int npy, double length, int pde,
                                     exa_fv_patchgrid** out) {
  if (!out) return set_error(EXA_EINVAL, "NULL argument");
  if (scheme != 0 && scheme != 1) return set_error(EXA_EINVAL, "scheme must be 0 (Godunov) or 1 (MUSCL-Hancock)");
  if (npx < 1 || npy < 1 || !(length > 0)) return set_error(EXA_EINVAL, "bad patch grid");
  // desc.dx is the patch (cell) extent: length / number of patches
  exa_fv_desc_t d{2, patch, scheme == 0 ? 1 : 2, kV, 0, pde, {length / npx, length / npy, 1.0}};
  if (exa_status_t s = check_fv(&d, d.ghost)) return s;
  if (patch < d.ghost) return set_error(EXA_EINVAL, "patch smaller than its ghost width");
  exa_fv_patchgrid* g = new (std::nothrow) exa_fv_patchgrid;
  if (!g) return set_error(EXA_ENOMEM, "host allocation");
  g->scheme = scheme;
  g->npx = npx;
  g->npy = npy;
  g->desc = d;
  g->npatches = (long)npx * npy;
  const size_t S = (size_t)patch + 2 * d.ghost;
  g->count = S * S * kV * g->npatches;
  cudaError_t e = cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&g->luh, g->count * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&g->luh_new, g->count * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&g->slots, 4 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(g->slots, 0, 4 * sizeof(unsigned long long), g->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->luh, 0, g->count * sizeof(double), g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) {
    exa_fv_patchgrid_destroy(g);
    return cuda_status(e, "fv patch grid allocation");
  }
  *out = g;
  return EXA_OK;
}

exa_status_t exa_fv_patchgrid_destroy(exa_fv_patchgrid* g) {
  if (!g) return EXA_OK;
  if (g->st) cudaStreamSynchronize(g->st);
  cudaFree(g->luh);
  cudaFree(g->luh_new);
  cudaFree(g->slots);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
  return EXA_OK;
}

size_t exa_fv_patchgrid_state_size(const exa_fv_patchgrid* g) { return g ? g->count : 0; }

exa_status_t exa_fv_patchgrid_init(exa_fv_patchgrid* g, double amp, uint64_t seed, double noise) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  const exa_fv_desc_t& d = g->desc;
  const long n = (long)(d.patch + 2 * d.ghost) * (d.patch + 2 * d.ghost) * g->npatches;
  k_fv_patch_ic<<<(unsigned)((n + 255) / 256), 256, 0, g->st>>>(d.patch, d.ghost, kV, g->npx, g->npy,
                                                               d.dx[0] / d.patch, d.dx[1] / d.patch, amp,
                                                               seed, noise, g->luh);
  count_launch();
  g->primed = false;
  cudaError_t e = cudaMemsetAsync(g->slots, 0, 4 * sizeof(unsigned long long), g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "fv patch grid init");
}

exa_status_t exa_fv_patchgrid_set_state(exa_fv_patchgrid* g, const double* host) {
  if (!g || !host) return set_error(EXA_EINVAL, "NULL argument");
  cudaError_t e = cudaMemcpyAsync(g->luh, host, g->count * sizeof(double), cudaMemcpyHostToDevice, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  g->primed = false;
  return cuda_status(e, "fv patch grid set_state");
}

exa_status_t exa_fv_patchgrid_get_state(exa_fv_patchgrid* g, double* host) {
  if (!g || !host) return set_error(EXA_EINVAL, "NULL argument");
  // the steps read no ghost cell and write none: fill the face ghosts here
  // so the returned state is the one the reference holds after its
  // neighbour merge (corner ghosts are not filled, as there)
  const exa_fv_desc_t& d = g->desc;
  const long nex = 4L * d.ghost * d.patch * g->npatches;
  k_fv_patch_exchange<<<(unsigned)((nex + 255) / 256), 256, 0, g->st>>>(d.patch, d.ghost, kV, g->npx, g->npy,
                                                                       g->bc[0], g->bc[1], g->luh);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host, g->luh, g->count * sizeof(double), cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  return cuda_status(e, "fv patch grid get_state");
}

exa_status_t exa_fv_patchgrid_step(exa_fv_patchgrid* g, int nsteps) {
  if (!g || nsteps < 0) return set_error(EXA_EINVAL, "bad argument");
  for (int i = 0; i < nsteps; i++)
    if (exa_status_t s = fv_patchgrid_step_one(g)) return s;
  return EXA_OK;
}

exa_status_t exa_fv_patchgrid_status(exa_fv_patchgrid* g, double* time, double* last_dt) {
  if (!g) return set_error(EXA_EINVAL, "NULL grid");
  unsigned long long h[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpyAsync(h, g->slots, 32, cudaMemcpyDeviceToHost, g->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->st);
  if (e != cudaSuccess) return cuda_status(e, "fv patch grid status");
  double t, dt;
  memcpy(&dt, &h[3], 8);
  memcpy(&t, &h[1], 8);
  if (time) *time = t;
  if (last_dt) *last_dt = dt;
  return EXA_OK;
}

exa_status_t exa_fv_patchgrid_set_boundary(exa_fv_patchgrid* g, const int* bc) {
  if (!g || !bc) return set_error(EXA_EINVAL, "NULL argument");
  for (int i = 0; i < 2; i++)
    if (bc[i] < EXA_BC_PERIODIC || bc[i] > EXA_BC_REFLECT) return set_error(EXA_EINVAL, "unknown boundary rule");
  g->bc[0] = bc[0];
  g->bc[1] = bc[1];
  return EXA_OK;
}

exa_status_t exa_fv_patchgrid_stream(exa_fv_patchgrid* g, void** stream) {
  if (!g || !stream) return set_error(EXA_EINVAL, "NULL argument");
  *stream = g->st;
  return EXA_OK;
}

}  // extern "C"
