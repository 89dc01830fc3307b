// A-posteriori subcell limiter kernels for batches of cells resident on the
// GPU: the reference's kernels/limiter/generic/c/Limiter.cpp
//   projectOnFVLimiterSpace      (:23-64)   DG nodes -> subcell means
//   projectOnDGSpace             (:67-110)  subcell means -> DG nodes
//   findCellLocalMinAndMax       (:212-251) with the Gauss-Lobatto (:258-306)
//                                           and subcell (:312-368) checks
//   findCellLocalLimiterMinAndMax (:170-207)
//   discreteMaximumPrincipleAndMinAndMaxSearch (:113-167)
// plus the copy of the new extrema to every face block that
// LimitingADERDGSolver::determineSolverMinAndMax / determineLimiterMinAndMax
// (exahype/solvers/LimitingADERDGSolver.cpp:1080-1150) do after the search.
//
// The reference evaluates every projection as a direct B^dim-term sum per
// output point.  The operators are tensor products of one 1D table, so here
// they are applied as dim one-dimensional passes (sum factorisation) in
// shared memory: a pass reads each line of its input once into registers
// and writes all outputs of the line, with the table entries as
// compile-time constant-bank operands (order is a template parameter).
// Several cells share a CTA so that every pass has enough lines for the
// 256 threads; threads take (cell, line, variable) items with the variable
// fastest, so the final pass's global stores are contiguous runs.
//
// Layouts (the reference's, KernelUtils.h idx4): luh [z][y][x][nvar] with B
// points per direction; lim [z][y][x][nvar] with S + 2g points per
// direction (S = 2N+1 subcells, g ghost layers); only the interior of lim is
// read or written.  Min/max blocks are [2 dim][nobs] per cell.  The
// observables are the first nobs variables (the generated solvers' default
// mapDiscreteMaximumPrincipleObservables,
// AbstractGenericADERDGSolverHeader.template:159-163).
#include <cfloat>

#include "exa_device.cuh"

#define EXA_TABLE_QUAL static const
#include "dg_tables.h"

namespace exa {

constexpr int kLimMaxOrder = 6;  // B <= 7, S <= 13
constexpr int kLimNT = 256;
constexpr int kLimMaxSmem = 200 * 1024;

struct LimConst {
  double uh2lim[7][13];  // [k][i]: mean of phi_k over subcell i
  double uh2lob[7][7];   // [k][i]: phi_k at Gauss-Lobatto node i
  double lim2uh[13][7];  // [i][k]: conservative least-squares inverse
};
static __constant__ LimConst c_lim[kLimMaxOrder + 1];

enum { kTabUh2Lim = 0, kTabUh2Lob = 1, kTabLim2Uh = 2 };

template <int TAB, int B>
__device__ __forceinline__ double lim_coef(int p, int m) {
  if (TAB == kTabUh2Lim) return c_lim[B - 1].uh2lim[p][m];
  if (TAB == kTabUh2Lob) return c_lim[B - 1].uh2lob[p][m];
  return c_lim[B - 1].lim2uh[p][m];
}

// std::min / std::max semantics: (b < a) ? b : a and (a < b) ? b : a
__device__ __forceinline__ double lim_min(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double lim_max(double a, double b) { return a < b ? b : a; }

// One 1D pass: applies table TAB (NI inputs -> NO outputs, T[p][m]) along
// direction D of a point array of extents EX x EY x EZ (x fastest), for
// `ncell` cells and variables v < nv.  Input point p of cell c starts at
// in + c * cs_in + p * ps_in.  Each thread takes (cell, line, variable)
// items, the variable fastest, starting with item (threadIdx.x - t0) mod NT
// (t0 lets a pass continue where the previous pass of the same phase left
// the threads); it hands the inputs and the NO outputs of its line to
// out.line<D>(c, x, y, z, v, inputs, outputs, item) with the D coordinate
// of (x, y, z) 0.  Strides and counts are plain ints: with the variable
// count a compile-time constant in the caller they fold into immediate
// offsets.
template <int TAB, int B, int EX, int EY, int EZ, int D, int NO, class Out>
__device__ __forceinline__ void lim_pass(const double* in, int ps_in, int cs_in, int ncell, int nv, Out& out,
                                         int t0 = 0) {
  constexpr int NI = D == 0 ? EX : (D == 1 ? EY : EZ);
  constexpr int LINES = EX * EY * EZ / NI;
  constexpr int SD = D == 0 ? 1 : (D == 1 ? EX : EX * EY);
  const int items = ncell * LINES * nv;
  for (int it = (threadIdx.x + kLimNT - t0 % kLimNT) % kLimNT; it < items; it += kLimNT) {
    const int v = it % nv;
    const int line = (it / nv) % LINES;
    const int c = it / (nv * LINES);
    int x = 0, y = 0, z = 0;
    if (D == 0) {
      y = line % EY;
      z = line / EY;
    } else if (D == 1) {
      x = line % EX;
      z = line / EX;
    } else {
      x = line % EX;
      y = line / EX;
    }
    const double* src = in + c * cs_in + ((z * EY + y) * EX + x) * ps_in + v;
    double a[NI];
#pragma unroll
    for (int p = 0; p < NI; p++) a[p] = src[p * SD * ps_in];
    double o[NO];
#pragma unroll
    for (int m = 0; m < NO; m++) {
      double acc = 0.0;
#pragma unroll
      for (int p = 0; p < NI; p++) acc = fma(lim_coef<TAB, B>(p, m), a[p], acc);
      o[m] = acc;
    }
    out.template line<D, NI, NO>(c, x, y, z, v, a, o, it);
  }
}

// writes a pass's outputs to a shared-memory array of extents ox x oy x .
struct SmemOut {
  double* base;
  int ps, cs, ox, oy;
  template <int D, int NI, int NO>
  __device__ __forceinline__ void line(int c, int x, int y, int z, int v, const double (&)[NI],
                                       const double (&o)[NO], int) {
    double* p = base + c * cs + ((z * oy + y) * ox + x) * ps + v;
    const int st = D == 0 ? ps : (D == 1 ? ox * ps : ox * oy * ps);
#pragma unroll
    for (int m = 0; m < NO; m++) p[m * st] = o[m];
  }
};

// writes to the interior of ghosted global patches (or plain luh arrays:
// off = 0, ext = B)
template <int DIM>
struct GlobalOut {
  double* base;  // cell 0 of the array
  long cs;       // doubles per cell
  int nvar, ext, off;
  long c0;       // first cell (selection index) of the CTA
  const int* list;
  template <int D, int NI, int NO>
  __device__ __forceinline__ void line(int c, int x, int y, int z, int v, const double (&)[NI],
                                       const double (&o)[NO], int) {
    const long pt = DIM == 3 ? ((long)(z + off) * ext + (y + off)) * ext + (x + off) : (long)(y + off) * ext + (x + off);
    const long cell = list ? (long)list[c0 + c] : c0 + c;
    double* p = base + cell * cs + pt * nvar + v;
    const long st = (D == 0 ? 1L : (D == 1 ? (long)ext : (long)ext * ext)) * nvar;
#pragma unroll
    for (int m = 0; m < NO; m++) p[m * st] = o[m];
  }
};

// extrema of the outputs of a line, stored per item
struct MinMaxOut {
  double* pmn;
  double* pmx;
  template <int D, int NI, int NO>
  __device__ __forceinline__ void line(int, int, int, int, int, const double (&)[NI], const double (&o)[NO],
                                       int it) {
    double mn = o[0], mx = o[0];
#pragma unroll
    for (int m = 1; m < NO; m++) {
      mn = lim_min(mn, o[m]);
      mx = lim_max(mx, o[m]);
    }
    pmn[it] = mn;
    pmx[it] = mx;
  }
};

// a shared-memory store plus the extrema of the pass's INPUT line (the
// nodes themselves, seen by the first pass over luh)
struct SmemOutInputMinMax {
  SmemOut s;
  double* pmn;
  double* pmx;
  template <int D, int NI, int NO>
  __device__ __forceinline__ void line(int c, int x, int y, int z, int v, const double (&a)[NI],
                                       const double (&o)[NO], int it) {
    s.line<D, NI, NO>(c, x, y, z, v, a, o, it);
    double mn = a[0], mx = a[0];
#pragma unroll
    for (int p = 1; p < NI; p++) {
      mn = lim_min(mn, a[p]);
      mx = lim_max(mx, a[p]);
    }
    pmn[it] = mn;
    pmx[it] = mx;
  }
};

// cooperative copy of `n` doubles (global -> shared)
__device__ __forceinline__ void lim_copy_in(double* dst, const double* src, long n) {
  for (long i = threadIdx.x; i < n; i += kLimNT) dst[i] = src[i];
}

template <int B>
struct LimOcc {
  // resident CTAs per SM the kernels are compiled for (register budget of
  // 64 / 85 / 255 per thread: the least that compiles without spills)
  static constexpr int value = B <= 4 ? 4 : (B == 5 ? 3 : 1);
};

// Optional cell selection: the kernels run on cells list[0 .. *count) (at
// most ncells) instead of cells 0 .. ncells; a device-resident count lets a
// fixed launch sequence serve a selection that changes from step to step.
struct LimSel {
  const int* list = nullptr;
  const int* count = nullptr;
  __device__ __forceinline__ long cells(long ncells) const {
    return count ? min(ncells, (long)*count) : ncells;
  }
  __device__ __forceinline__ long cell(long k) const { return list ? (long)list[k] : k; }
};

// copies the selected cells' input arrays (n doubles each) to shared memory
__device__ __forceinline__ void lim_copy_cells(double* dst, const double* src, int n, long c0, int nc,
                                               const LimSel& sel) {
  if (!sel.list) {
    lim_copy_in(dst, src + c0 * n, (long)nc * n);
    return;
  }
  for (int i = threadIdx.x; i < nc * n; i += kLimNT) {
    const int c = i / n;
    dst[i] = src[sel.cell(c0 + c) * n + (i - c * n)];
  }
}

// ------------------------------------------------------------ DG -> FV
// shared memory per cell (doubles per variable): luh, pass-x and pass-y
// results (3D)
template <int DIM, int B>
__host__ __device__ constexpr int lim_to_fv_cell_doubles_per_var() {
  return DIM == 3 ? B * B * B + B * B * (2 * B - 1) + B * (2 * B - 1) * (2 * B - 1) : B * B + B * (2 * B - 1);
}

// NVT: the variable count when known at compile time (0 = runtime nvar)
template <int DIM, int B, int NVT>
__global__ void __launch_bounds__(kLimNT, LimOcc<B>::value)
    k_lim_to_fv(int nvar_rt, int ghost, long ncells, int cpb, const double* luh, double* lim, LimSel sel) {
  constexpr int S = 2 * B - 1;
  constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  const int nvar = NVT ? NVT : nvar_rt;
  extern __shared__ double sm[];
  const long nce = sel.cells(ncells);
  // one cell block per iteration (a single one unless a selection launched
  // fewer CTAs than blocks)
  for (long c0 = (long)blockIdx.x * cpb; c0 < nce; c0 += (long)gridDim.x * cpb) {
    const int nc = (int)min((long)cpb, nce - c0);
    const int SG = S + 2 * ghost;
    const long lim_cell = (long)nvar * (DIM == 3 ? SG * SG * SG : SG * SG);
    double* A = sm;
    double* T1 = A + cpb * NPC * nvar;
    lim_copy_cells(A, luh, NPC * nvar, c0, nc, sel);
    __syncthreads();
    GlobalOut<DIM> go{lim, lim_cell, nvar, SG, ghost, c0, sel.list};
    if (DIM == 2) {
      SmemOut o1{T1, nvar, S * B * nvar, S, B};
      lim_pass<kTabUh2Lim, B, B, B, 1, 0, S>(A, nvar, NPC * nvar, nc, nvar, o1);
      __syncthreads();
      lim_pass<kTabUh2Lim, B, S, B, 1, 1, S>(T1, nvar, S * B * nvar, nc, nvar, go);
    } else {
      double* T2 = T1 + cpb * B * B * S * nvar;
      SmemOut o1{T1, nvar, B * B * S * nvar, S, B};
      lim_pass<kTabUh2Lim, B, B, B, B, 0, S>(A, nvar, NPC * nvar, nc, nvar, o1);
      __syncthreads();
      SmemOut o2{T2, nvar, B * S * S * nvar, S, S};
      lim_pass<kTabUh2Lim, B, S, B, B, 1, S>(T1, nvar, B * B * S * nvar, nc, nvar, o2);
      __syncthreads();
      lim_pass<kTabUh2Lim, B, S, S, B, 2, S>(T2, nvar, B * S * S * nvar, nc, nvar, go);
    }
    __syncthreads();
  }
}

// interior subcells of nc ghosted patches -> shared [c][z][y][x][nvar]
// (rows of S * nvar contiguous doubles); each thread keeps four loads in
// flight before it stores them
template <int DIM, int S>
__device__ __forceinline__ void lim_stage_interior(double* A, const double* __restrict__ lim, long lim_cell, int nvar,
                                                   int ghost, long c0, int nc, const LimSel& sel) {
  const int SG = S + 2 * ghost;
  const int rowlen = S * nvar;
  constexpr int rows = DIM == 3 ? S * S : S;
  constexpr int U = 4;
  const int total = nc * rows * rowlen;
  for (int i0 = threadIdx.x; i0 < total; i0 += U * kLimNT) {
    double r[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int i = i0 + u * kLimNT;
      if (i < total) {
        const int k = i % rowlen;
        const int q = i / rowlen;
        const int row = q % rows;
        const int c = q / rows;
        const int yy = row % S, zz = row / S;
        const long p = DIM == 3 ? ((long)(zz + ghost) * SG + (yy + ghost)) * SG + ghost : (long)(yy + ghost) * SG + ghost;
        r[u] = __ldg(lim + sel.cell(c0 + c) * lim_cell + p * nvar + k);
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++)
      if (i0 + u * kLimNT < total) A[i0 + u * kLimNT] = r[u];
  }
}

// ------------------------------------------------------------ FV -> DG
// shared memory per cell (doubles per variable): the staged subcells (later
// reused for the pass-y result) and the pass-x result
template <int DIM, int B>
__host__ __device__ constexpr int lim_to_dg_cell_doubles_per_var() {
  return DIM == 3 ? (2 * B - 1) * (2 * B - 1) * (2 * B - 1) + (2 * B - 1) * (2 * B - 1) * B
                  : (2 * B - 1) * (2 * B - 1) + (2 * B - 1) * B;
}

template <int DIM, int B, int NVT>
__global__ void __launch_bounds__(kLimNT, LimOcc<B>::value)
    k_lim_to_dg(int nvar_rt, int ghost, long ncells, int cpb, const double* lim, double* luh, LimSel sel) {
  constexpr int S = 2 * B - 1;
  constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  constexpr int NS = DIM == 3 ? S * S * S : S * S;
  const int nvar = NVT ? NVT : nvar_rt;
  extern __shared__ double sm[];
  const long nce = sel.cells(ncells);
  // one cell block per iteration (a single one unless a selection launched
  // fewer CTAs than blocks)
  for (long c0 = (long)blockIdx.x * cpb; c0 < nce; c0 += (long)gridDim.x * cpb) {
    const int nc = (int)min((long)cpb, nce - c0);
    const int SG = S + 2 * ghost;
    const long lim_cell = (long)nvar * (DIM == 3 ? SG * SG * SG : SG * SG);
    double* A = sm;  // interior subcells [c][z][y][x][v]
    double* T1 = A + cpb * NS * nvar;
    lim_stage_interior<DIM, S>(A, lim, lim_cell, nvar, ghost, c0, nc, sel);
    __syncthreads();
    GlobalOut<DIM> go{luh, (long)NPC * nvar, nvar, B, 0, c0, sel.list};
    if (DIM == 2) {
      SmemOut o1{T1, nvar, S * B * nvar, B, S};
      lim_pass<kTabLim2Uh, B, S, S, 1, 0, B>(A, nvar, NS * nvar, nc, nvar, o1);
      __syncthreads();
      lim_pass<kTabLim2Uh, B, B, S, 1, 1, B>(T1, nvar, S * B * nvar, nc, nvar, go);
    } else {
      double* T2 = A;  // the staged subcells are dead after pass x
      SmemOut o1{T1, nvar, S * S * B * nvar, B, S};
      lim_pass<kTabLim2Uh, B, S, S, S, 0, B>(A, nvar, NS * nvar, nc, nvar, o1);
      __syncthreads();
      SmemOut o2{T2, nvar, S * B * B * nvar, B, B};
      lim_pass<kTabLim2Uh, B, B, S, S, 1, B>(T1, nvar, S * S * B * nvar, nc, nvar, o2);
      __syncthreads();
      lim_pass<kTabLim2Uh, B, B, B, S, 2, B>(T2, nvar, S * B * B * nvar, nc, nvar, go);
    }
    __syncthreads();
  }
}

// ------------------------------------------------ min/max and the DMP
// The Gauss-Lobatto (B -> B) and subcell (B -> S) evaluations run side by
// side, pass by pass; the first pass also takes the extrema of the nodes
// (its input lines).  Per cell and observable, shared memory holds: the
// pass-x results of both (B^3 + B^2 S), the pass-y result of the subcells
// (B S^2) and of the Lobatto points (B^3, in the luh staging area, dead after
// pass x), and the per-line extrema of nodes, Lobatto points and subcells.
template <int DIM, int B>
struct LimMM {
  static constexpr int S = 2 * B - 1;
  static constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  static constexpr int XL = DIM == 3 ? B * B * B : B * B;  // Lobatto pass-x result
  static constexpr int XS = DIM == 3 ? B * B * S : B * S;  // subcell pass-x result
  static constexpr int YS = DIM == 3 ? B * S * S : 0;      // subcell pass-y result
  static constexpr int NODE_LINES = DIM == 3 ? B * B : B;  // pass-x lines
  static constexpr int LOB_LINES = DIM == 3 ? B * B : B;   // final Lobatto lines
  static constexpr int SUB_LINES = DIM == 3 ? S * S : S;   // final subcell lines
  static constexpr int LINES = NODE_LINES + LOB_LINES + SUB_LINES;
  // doubles per cell
  __host__ __device__ static constexpr int doubles(int nvar, int nobs) {
    return NPC * nvar + (XL + XS + YS + 2 * LINES) * nobs;
  }
};

// mode 0: findCellLocalMinAndMax, result copied to all faces;
// mode 1: discreteMaximumPrincipleAndMinAndMaxSearch (obs_min/max in/out,
//         dmp_ok[cell] = 1 if the DMP holds).
template <int DIM, int B, int NVT>
__global__ void __launch_bounds__(kLimNT, LimOcc<B>::value)
    k_lim_min_max(int mode, int nvar_rt, int nobs_rt, long ncells, int cpb, const double* luh, double relaxation,
                  double scaling, double* obs_min, double* obs_max, int* dmp_ok) {
  using M = LimMM<DIM, B>;
  constexpr int S = M::S, NPC = M::NPC, NF = 2 * DIM;
  const int nvar = NVT ? NVT : nvar_rt;
  const int nobs = NVT ? NVT : nobs_rt;
  extern __shared__ double sm[];
  const long c0 = (long)blockIdx.x * cpb;
  const int nc = (int)min((long)cpb, ncells - c0);
  double* A = sm;                         // luh, later the Lobatto pass-y result
  double* XL = A + cpb * NPC * nvar;      // [c][z][y][x][obs]
  double* XS = XL + cpb * M::XL * nobs;
  double* YS = XS + cpb * M::XS * nobs;
  double* pmn = YS + cpb * M::YS * nobs;  // [node | lob | sub lines]
  double* pmx = pmn + cpb * M::LINES * nobs;
  double* pn_mn = pmn;                    // node lines   [c][line][obs]
  double* pl_mn = pmn + cpb * M::NODE_LINES * nobs;
  double* ps_mn = pl_mn + cpb * M::LOB_LINES * nobs;
  double* pn_mx = pmx;
  double* pl_mx = pmx + cpb * M::NODE_LINES * nobs;
  double* ps_mx = pl_mx + cpb * M::LOB_LINES * nobs;
  if (mode == 1)
    for (int c = threadIdx.x; c < nc; c += kLimNT) dmp_ok[c0 + c] = 1;
  lim_copy_in(A, luh + c0 * NPC * nvar, (long)nc * NPC * nvar);
  __syncthreads();
  const int ix = nc * M::NODE_LINES * nobs;  // items of one pass-x
  if (DIM == 2) {
    SmemOutInputMinMax ol{{XL, nobs, B * B * nobs, B, B}, pn_mn, pn_mx};
    lim_pass<kTabUh2Lob, B, B, B, 1, 0, B>(A, nvar, NPC * nvar, nc, nobs, ol);
    SmemOut os{XS, nobs, S * B * nobs, S, B};
    lim_pass<kTabUh2Lim, B, B, B, 1, 0, S>(A, nvar, NPC * nvar, nc, nobs, os, ix);
    __syncthreads();
    MinMaxOut ml{pl_mn, pl_mx}, ms{ps_mn, ps_mx};
    lim_pass<kTabUh2Lob, B, B, B, 1, 1, B>(XL, nobs, B * B * nobs, nc, nobs, ml);
    lim_pass<kTabUh2Lim, B, S, B, 1, 1, S>(XS, nobs, S * B * nobs, nc, nobs, ms, nc * B * nobs);
  } else {
    SmemOutInputMinMax ol{{XL, nobs, B * B * B * nobs, B, B}, pn_mn, pn_mx};
    lim_pass<kTabUh2Lob, B, B, B, B, 0, B>(A, nvar, NPC * nvar, nc, nobs, ol);
    SmemOut os{XS, nobs, B * B * S * nobs, S, B};
    lim_pass<kTabUh2Lim, B, B, B, B, 0, S>(A, nvar, NPC * nvar, nc, nobs, os, ix);
    __syncthreads();
    double* YL = A;  // luh is dead after pass x
    SmemOut yl{YL, nobs, B * B * B * nobs, B, B};
    lim_pass<kTabUh2Lob, B, B, B, B, 1, B>(XL, nobs, B * B * B * nobs, nc, nobs, yl);
    SmemOut ys{YS, nobs, B * S * S * nobs, S, S};
    lim_pass<kTabUh2Lim, B, S, B, B, 1, S>(XS, nobs, B * B * S * nobs, nc, nobs, ys, nc * B * B * nobs);
    __syncthreads();
    MinMaxOut ml{pl_mn, pl_mx}, ms{ps_mn, ps_mx};
    lim_pass<kTabUh2Lob, B, B, B, B, 2, B>(YL, nobs, B * B * B * nobs, nc, nobs, ml);
    lim_pass<kTabUh2Lim, B, S, S, B, 2, S>(YS, nobs, B * S * S * nobs, nc, nobs, ms, nc * B * B * nobs);
  }
  __syncthreads();
  // per (cell, observable): the new extrema -> face blocks, and the DMP
  auto finish = [&](int pair, double mn, double mx) {
    const int c = pair / nobs, v = pair % nobs;
    double* bmn = obs_min + (c0 + c) * NF * nobs;
    double* bmx = obs_max + (c0 + c) * NF * nobs;
    if (mode == 0) {
      for (int f = 0; f < NF; f++) {
        bmn[f * nobs + v] = mn;
        bmx[f * nobs + v] = mx;
      }
    } else {
      double lo = bmn[v], hi = bmx[v];
      for (int f = 1; f < NF; f++) {
        lo = lim_min(lo, bmn[f * nobs + v]);
        hi = lim_max(hi, bmx[f * nobs + v]);
      }
      const double sd = lim_max((hi - lo) * scaling, relaxation);
      if (mn < lo - sd || mx > hi + sd) atomicAnd(dmp_ok + c0 + c, 0);
      bmn[v] = mn;
      bmx[v] = mx;
      bmn[v + nobs] = lo;
      bmx[v + nobs] = hi;
    }
  };
  auto line_index = [&](int c, int v, int l) {
    if (l < M::NODE_LINES) return (c * M::NODE_LINES + l) * nobs + v;
    if (l < M::NODE_LINES + M::LOB_LINES)
      return cpb * M::NODE_LINES * nobs + (c * M::LOB_LINES + l - M::NODE_LINES) * nobs + v;
    return cpb * (M::NODE_LINES + M::LOB_LINES) * nobs + (c * M::SUB_LINES + l - M::NODE_LINES - M::LOB_LINES) * nobs +
           v;
  };
  // reduction over the line extrema: a thread per pair when the pairs have
  // few lines (2D), a warp per pair otherwise
  if (M::LINES <= 32) {
    for (int pair = threadIdx.x; pair < nc * nobs; pair += kLimNT) {
      const int c = pair / nobs, v = pair % nobs;
      double mn = DBL_MAX, mx = -DBL_MAX;
#pragma unroll
      for (int l = 0; l < M::LINES; l++) {
        const int k = line_index(c, v, l);
        mn = lim_min(mn, pmn[k]);
        mx = lim_max(mx, pmx[k]);
      }
      finish(pair, mn, mx);
    }
  } else {
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int pair = warp; pair < nc * nobs; pair += kLimNT / 32) {
      const int c = pair / nobs, v = pair % nobs;
      double mn = DBL_MAX, mx = -DBL_MAX;
      for (int l = lane; l < M::LINES; l += 32) {
        const int k = line_index(c, v, l);
        mn = lim_min(mn, pmn[k]);
        mx = lim_max(mx, pmx[k]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        mn = lim_min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = lim_max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      }
      if (lane == 0) finish(pair, mn, mx);
    }
  }
}

// findCellLocalLimiterMinAndMax: extrema over the staged interior subcells,
// one warp per (cell, observable), written to every face block
template <int DIM, int B>
__global__ void __launch_bounds__(kLimNT) k_lim_fv_min_max(int nvar, int nobs, int ghost, long ncells, int cpb,
                                                           const double* lim, double* obs_min, double* obs_max,
                                                           LimSel sel) {
  constexpr int S = 2 * B - 1;
  constexpr int NS = DIM == 3 ? S * S * S : S * S;
  extern __shared__ double sm[];
  const long nce = sel.cells(ncells);
  // one cell block per iteration (a single one unless a selection launched
  // fewer CTAs than blocks)
  for (long c0 = (long)blockIdx.x * cpb; c0 < nce; c0 += (long)gridDim.x * cpb) {
    const int nc = (int)min((long)cpb, nce - c0);
    const int SG = S + 2 * ghost;
    const long lim_cell = (long)nvar * (DIM == 3 ? SG * SG * SG : SG * SG);
    lim_stage_interior<DIM, S>(sm, lim, lim_cell, nvar, ghost, c0, nc, sel);
    __syncthreads();
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int pair = warp; pair < nc * nobs; pair += kLimNT / 32) {
      const int c = pair / nobs, v = pair % nobs;
      double mn = DBL_MAX, mx = -DBL_MAX;
      for (int p = lane; p < NS; p += 32) {
        const double q = sm[((long)c * NS + p) * nvar + v];
        mn = lim_min(mn, q);
        mx = lim_max(mx, q);
      }
  #pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        mn = lim_min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = lim_max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      }
      if (lane == 0)
        for (int f = 0; f < 2 * DIM; f++) {
          obs_min[(sel.cell(c0 + c) * 2 * DIM + f) * nobs + v] = mn;
          obs_max[(sel.cell(c0 + c) * 2 * DIM + f) * nobs + v] = mx;
        }
    }
    __syncthreads();
  }
}

// cells per CTA: enough items for two rounds of the final pass, within a
// shared-memory budget that leaves room for `occ` resident CTAs per SM
static int lim_cpb(long items_per_cell, long smem_per_cell, long ncells, int occ) {
  long cpb = (2 * kLimNT + items_per_cell - 1) / items_per_cell;
  if (cpb > 64) cpb = 64;
  long cap = (220L * 1024 / occ) / smem_per_cell;
  if (cap < 1) cap = 1;
  if (cpb > cap) cpb = cap;
  if (cpb > ncells) cpb = ncells;
  return (int)(cpb < 1 ? 1 : cpb);
}

template <class K>
static cudaError_t lim_prepare(K kern, size_t smem) {
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

template <int DIM, int B, int NVT>
static exa_status_t lim_run(int op, int nvar, int nobs, int ghost, long ncells, const double* in, double* out,
                            double* mn, double* mx, int* ok, double relax, double scaling, cudaStream_t st,
                            LimSel sel) {
  constexpr int S = 2 * B - 1;
  long per_cell, items;
  if (op == kLimToFv) {
    per_cell = (long)lim_to_fv_cell_doubles_per_var<DIM, B>() * nvar;
    items = (long)(DIM == 3 ? S * S : S) * nvar;
  } else if (op == kLimToDg) {
    per_cell = (long)lim_to_dg_cell_doubles_per_var<DIM, B>() * nvar;
    items = (long)(DIM == 3 ? B * B : B) * nvar;
  } else if (op == kLimFvMinMax) {
    per_cell = (long)(DIM == 3 ? S * S * S : S * S) * nvar;
    items = 32L * nobs;
  } else {
    per_cell = LimMM<DIM, B>::doubles(nvar, nobs);
    items = (long)LimMM<DIM, B>::SUB_LINES * nobs;
  }
  per_cell *= (long)sizeof(double);
  if (per_cell > kLimMaxSmem) return set_error(EXA_EINVAL, "limiter: cell too large for shared memory");
  int cpb = lim_cpb(items, per_cell, ncells, LimOcc<B>::value);
  const int cpb_set = tune_get(kTuneLimiterCellsPerCta, 0);
  if (cpb_set > 0 && (long)cpb_set * per_cell <= kLimMaxSmem) cpb = cpb_set;
  const size_t smem = (size_t)cpb * per_cell;
  long nblk = (ncells + cpb - 1) / cpb;
  if (sel.count) {
    // a selection usually holds a few cells: CTAs loop over the blocks
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    nblk = nblk < 4L * sms ? nblk : 4L * sms;
  }
  if (nblk > 0x7fffffffL) return set_error(EXA_EINVAL, "limiter: too many cells");
  cudaError_t e = cudaSuccess;
  if (op == kLimToFv) {
    e = lim_prepare(k_lim_to_fv<DIM, B, NVT>, smem);
    if (e == cudaSuccess)
      k_lim_to_fv<DIM, B, NVT><<<(unsigned)nblk, kLimNT, smem, st>>>(nvar, ghost, ncells, cpb, in, out, sel);
  } else if (op == kLimToDg) {
    e = lim_prepare(k_lim_to_dg<DIM, B, NVT>, smem);
    if (e == cudaSuccess)
      k_lim_to_dg<DIM, B, NVT><<<(unsigned)nblk, kLimNT, smem, st>>>(nvar, ghost, ncells, cpb, in, out, sel);
  } else if (op == kLimFvMinMax) {
    e = lim_prepare(k_lim_fv_min_max<DIM, B>, smem);
    if (e == cudaSuccess)
      k_lim_fv_min_max<DIM, B><<<(unsigned)nblk, kLimNT, smem, st>>>(nvar, nobs, ghost, ncells, cpb, in, mn, mx,
                                                                       sel);
  } else {
    auto kern = k_lim_min_max<DIM, B, NVT>;
    e = lim_prepare(kern, smem);
    if (e == cudaSuccess)
      kern<<<(unsigned)nblk, kLimNT, smem, st>>>(op == kLimDmp ? 1 : 0, nvar, nobs, ncells, cpb, in, relax, scaling, mn,
                                                  mx, ok);
  }
  if (e != cudaSuccess) return cuda_status(e, "limiter: shared-memory attribute");
  count_launch();
  return cuda_status(cudaGetLastError(), "limiter kernel");
}

// the Euler case (5 variables, 5 observables) runs kernels specialised for
// it; any other count the generic ones
template <int DIM, int B>
static exa_status_t lim_run_nv(int op, int nvar, int nobs, int ghost, long ncells, const double* in, double* out,
                               double* mn, double* mx, int* ok, double relax, double scaling, cudaStream_t st,
                               LimSel sel) {
  const bool five = nvar == 5 && (op < kLimMinMax || op == kLimFvMinMax || nobs == 5);
  if (five) return lim_run<DIM, B, 5>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
  return lim_run<DIM, B, 0>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
}

template <int DIM>
static exa_status_t lim_dispatch(int op, int order, int nvar, int nobs, int ghost, long ncells, const double* in,
                                 double* out, double* mn, double* mx, int* ok, double relax, double scaling,
                                 cudaStream_t st, LimSel sel) {
  switch (order) {
    case 1: return lim_run_nv<DIM, 2>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
    case 2: return lim_run_nv<DIM, 3>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
    case 3: return lim_run_nv<DIM, 4>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
    case 4: return lim_run_nv<DIM, 5>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
    case 5: return lim_run_nv<DIM, 6>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
    case 6: return lim_run_nv<DIM, 7>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
  }
  return set_error(EXA_EINVAL, "limiter: order must be in 1..6");
}

static exa_status_t lim_entry(int op, int dim, int order, int nvar, int nobs, int ghost, long ncells,
                              const double* in, double* out, double* mn, double* mx, int* ok, double relax,
                              double scaling, void* stream, LimSel sel = LimSel()) {
  if (exa_status_t s = ensure_tables()) return s;
  if (dim != 2 && dim != 3) return set_error(EXA_EINVAL, "limiter: dim must be 2 or 3");
  if (nvar < 1 || nvar > 64) return set_error(EXA_EINVAL, "limiter: nvar must be in 1..64");
  if (ghost < 0 || ghost > 8) return set_error(EXA_EINVAL, "limiter: ghost layer width must be in 0..8");
  if (ncells < 0) return set_error(EXA_EINVAL, "limiter: negative cell count");
  if (op >= kLimMinMax) {
    if (nobs < 0 || nobs > nvar) return set_error(EXA_EINVAL, "limiter: nobs must be in 0..nvar");
    if (!in || (nobs > 0 && (!mn || !mx)) || (op == kLimDmp && !ok))
      return set_error(EXA_EINVAL, "limiter: NULL pointer");
    // without observables the solver layer skips the search altogether
    // (LimitingADERDGSolver.cpp:993-1026); the DMP entry needs one
    if (nobs == 0) return op == kLimDmp ? set_error(EXA_EINVAL, "limiter: DMP needs nobs >= 1") : EXA_OK;
  } else if (!in || !out) {
    return set_error(EXA_EINVAL, "limiter: NULL pointer");
  }
  if (ncells == 0) return EXA_OK;
  cudaStream_t st = as_stream(stream);
  return dim == 2 ? lim_dispatch<2>(op, order, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel)
                  : lim_dispatch<3>(op, order, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st, sel);
}

exa_status_t limiter_launch(int op, int dim, int order, int nvar, int nobs, int ghost, long ncells, const double* in,
                            double* out, double* mn, double* mx, int* ok, double relax, double scaling,
                            cudaStream_t st, const int* list, const int* count) {
  LimSel sel;
  sel.list = list;
  sel.count = count;
  return lim_entry(op, dim, order, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling,
                   reinterpret_cast<void*>(st), sel);
}

exa_status_t upload_tables_limiter() {
  static LimConst h[kLimMaxOrder + 1];
  for (int n = 0; n <= kLimMaxOrder; n++) {
    const int B = n + 1, S = 2 * n + 1;
    for (int k = 0; k < 7; k++) {
      for (int i = 0; i < 13; i++) h[n].uh2lim[k][i] = (k < B && i < S) ? exa_uh2lim[n][k][i] : 0.0;
      for (int i = 0; i < 7; i++) h[n].uh2lob[k][i] = (k < B && i < B) ? exa_uh2lob[n][k][i] : 0.0;
    }
    for (int i = 0; i < 13; i++)
      for (int k = 0; k < 7; k++) h[n].lim2uh[i][k] = (i < S && k < B) ? exa_lim2uh[n][i][k] : 0.0;
  }
  return cuda_status(cudaMemcpyToSymbol(c_lim, h, sizeof(h)), "upload tables (limiter)");
}

}  // namespace exa

using namespace exa;

extern "C" {

exa_status_t exa_limiter_project_on_fv(int dim, int order, int nvar, int ghost_layer_width, long ncells,
                                       const double* luh, double* lim, void* stream) {
  return lim_entry(kLimToFv, dim, order, nvar, 0, ghost_layer_width, ncells, luh, lim, nullptr, nullptr, nullptr,
                   0.0, 0.0, stream);
}

exa_status_t exa_limiter_project_on_dg(int dim, int order, int nvar, int ghost_layer_width, long ncells,
                                       const double* lim, double* luh, void* stream) {
  return lim_entry(kLimToDg, dim, order, nvar, 0, ghost_layer_width, ncells, lim, luh, nullptr, nullptr, nullptr,
                   0.0, 0.0, stream);
}

exa_status_t exa_limiter_local_min_max(int dim, int order, int nvar, int nobs, long ncells, const double* luh,
                                       double* obs_min, double* obs_max, void* stream) {
  return lim_entry(kLimMinMax, dim, order, nvar, nobs, 0, ncells, luh, nullptr, obs_min, obs_max, nullptr, 0.0, 0.0,
                   stream);
}

exa_status_t exa_limiter_fv_min_max(int dim, int order, int nvar, int nobs, int ghost_layer_width, long ncells,
                                    const double* lim, double* obs_min, double* obs_max, void* stream) {
  return lim_entry(kLimFvMinMax, dim, order, nvar, nobs, ghost_layer_width, ncells, lim, nullptr, obs_min, obs_max,
                   nullptr, 0.0, 0.0, stream);
}

exa_status_t exa_limiter_dmp(int dim, int order, int nvar, int nobs, long ncells, const double* luh,
                             double relaxation, double difference_scaling, double* obs_min, double* obs_max,
                             int* dmp_ok, void* stream) {
  return lim_entry(kLimDmp, dim, order, nvar, nobs, 0, ncells, luh, nullptr, obs_min, obs_max, dmp_ok, relaxation,
                   difference_scaling, stream);
}

}  // extern "C"
