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

// One 1D pass: applies table TAB (NI inputs -> NO outputs, T[p][m]) along
// direction D of a point array of extents EX x EY x EZ (x fastest), for
// `ncell` cells and variables v < nv.  Input point p of cell c starts at
// in + c * cs_in + p * ps_in.  out.put(c, x, y, z, v, value) receives every
// output (with the D coordinate replaced by the output index);
// out.line_done(item) closes each line.
template <int TAB, int B, int EX, int EY, int EZ, int D, int NO, class Out>
__device__ __forceinline__ void lim_pass(const double* in, int ps_in, int cs_in, int ncell, int nv, Out& out) {
  constexpr int NI = D == 0 ? EX : (D == 1 ? EY : EZ);
  constexpr int LINES = EX * EY * EZ / NI;
  constexpr int SD = D == 0 ? 1 : (D == 1 ? EX : EX * EY);
  const int items = ncell * LINES * nv;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
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
#pragma unroll
    for (int m = 0; m < NO; m++) {
      double acc = 0.0;
#pragma unroll
      for (int p = 0; p < NI; p++) acc = fma(lim_coef<TAB, B>(p, m), a[p], acc);
      if (D == 0) out.put(c, m, y, z, v, acc);
      else if (D == 1) out.put(c, x, m, z, v, acc);
      else out.put(c, x, y, m, v, acc);
    }
    out.line_done(it);
  }
}

// writes a pass's outputs to a shared-memory array of extents OX x OY x OZ
struct SmemOut {
  double* base;
  int ps, cs, ox, oy;
  __device__ __forceinline__ void put(int c, int x, int y, int z, int v, double val) {
    base[c * cs + ((z * oy + y) * ox + x) * ps + v] = val;
  }
  __device__ __forceinline__ void line_done(int) {}
};

// writes to the interior of ghosted global patches (or plain luh arrays)
struct GlobalOut {
  double* base;  // first cell of the CTA
  long cs;       // doubles per cell
  int nvar, ext, off, dim;
  __device__ __forceinline__ void put(int c, int x, int y, int z, int v, double val) {
    const long p = dim == 3 ? ((long)(z + off) * ext + (y + off)) * ext + (x + off)
                            : (long)(y + off) * ext + (x + off);
    base[c * cs + p * nvar + v] = val;
  }
  __device__ __forceinline__ void line_done(int) {}
};

// running min/max of the outputs of a line, stored per item at its end
struct MinMaxOut {
  double* pmn;
  double* pmx;
  double mn = DBL_MAX, mx = -DBL_MAX;
  __device__ __forceinline__ void put(int, int, int, int, int, double val) {
    mn = fmin(mn, val);
    mx = fmax(mx, val);
  }
  __device__ __forceinline__ void line_done(int it) {
    pmn[it] = mn;
    pmx[it] = mx;
    mn = DBL_MAX;
    mx = -DBL_MAX;
  }
};

// cooperative copy of `n` doubles (global -> shared)
__device__ __forceinline__ void lim_copy_in(double* dst, const double* src, long n) {
  for (long i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

// ------------------------------------------------------------ DG -> FV
// shared memory per cell (doubles): luh, pass-x result, pass-y result (3D)
template <int DIM, int B>
__host__ __device__ constexpr int lim_to_fv_cell_doubles_per_var() {
  return DIM == 3 ? B * B * B + B * B * (2 * B - 1) + B * (2 * B - 1) * (2 * B - 1)
                  : B * B + B * (2 * B - 1);
}

template <int DIM, int B>
__global__ void __launch_bounds__(kLimNT) k_lim_to_fv(int nvar, int ghost, long ncells, int cpb, const double* luh,
                                                      double* lim) {
  constexpr int S = 2 * B - 1;
  extern __shared__ double sm[];
  const long c0 = (long)blockIdx.x * cpb;
  const int nc = (int)min((long)cpb, ncells - c0);
  constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  const int SG = S + 2 * ghost;
  const long lim_cell = (long)nvar * (DIM == 3 ? SG * SG * SG : SG * SG);
  double* A = sm;
  double* T1 = A + cpb * NPC * nvar;
  lim_copy_in(A, luh + c0 * NPC * nvar, (long)nc * NPC * nvar);
  __syncthreads();
  GlobalOut go{lim + c0 * lim_cell, lim_cell, nvar, SG, ghost, DIM};
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
}

// interior subcells of nc ghosted patches -> shared [c][z][y][x][nvar]
// (rows of S * nvar contiguous doubles)
template <int DIM, int S>
__device__ __forceinline__ void lim_stage_interior(double* A, const double* lim, long lim_cell, int nvar, int ghost,
                                                   int nc) {
  const int SG = S + 2 * ghost;
  const int rowlen = S * nvar;
  constexpr int rows = DIM == 3 ? S * S : S;
  const long total = (long)nc * rows * rowlen;
  for (long i = threadIdx.x; i < total; i += blockDim.x) {
    const int k = (int)(i % rowlen);
    const long r = i / rowlen;
    const int row = (int)(r % rows);
    const long c = r / rows;
    const int yy = row % S, zz = row / S;
    const long p = DIM == 3 ? ((long)(zz + ghost) * SG + (yy + ghost)) * SG + ghost : (long)(yy + ghost) * SG + ghost;
    A[(c * rows + row) * rowlen + k] = lim[c * lim_cell + p * nvar + k];
  }
}

// ------------------------------------------------------------ FV -> DG
template <int DIM, int B>
__host__ __device__ constexpr int lim_to_dg_cell_doubles_per_var() {
  return DIM == 3 ? (2 * B - 1) * (2 * B - 1) * (2 * B - 1) + (2 * B - 1) * (2 * B - 1) * B +
                        (2 * B - 1) * B * B
                  : (2 * B - 1) * (2 * B - 1) + (2 * B - 1) * B;
}

template <int DIM, int B>
__global__ void __launch_bounds__(kLimNT) k_lim_to_dg(int nvar, int ghost, long ncells, int cpb, const double* lim,
                                                      double* luh) {
  constexpr int S = 2 * B - 1;
  extern __shared__ double sm[];
  const long c0 = (long)blockIdx.x * cpb;
  const int nc = (int)min((long)cpb, ncells - c0);
  constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  constexpr int NS = DIM == 3 ? S * S * S : S * S;
  const int SG = S + 2 * ghost;
  const long lim_cell = (long)nvar * (DIM == 3 ? SG * SG * SG : SG * SG);
  double* A = sm;  // interior subcells [c][z][y][x][v]
  double* T1 = A + cpb * NS * nvar;
  lim_stage_interior<DIM, S>(A, lim + c0 * lim_cell, lim_cell, nvar, ghost, nc);
  __syncthreads();
  GlobalOut go{luh + c0 * NPC * nvar, (long)NPC * nvar, nvar, B, 0, DIM};
  if (DIM == 2) {
    SmemOut o1{T1, nvar, S * B * nvar, B, S};
    lim_pass<kTabLim2Uh, B, S, S, 1, 0, B>(A, nvar, NS * nvar, nc, nvar, o1);
    __syncthreads();
    lim_pass<kTabLim2Uh, B, B, S, 1, 1, B>(T1, nvar, S * B * nvar, nc, nvar, go);
  } else {
    double* T2 = T1 + cpb * S * S * B * nvar;
    SmemOut o1{T1, nvar, S * S * B * nvar, B, S};
    lim_pass<kTabLim2Uh, B, S, S, S, 0, B>(A, nvar, NS * nvar, nc, nvar, o1);
    __syncthreads();
    SmemOut o2{T2, nvar, S * B * B * nvar, B, B};
    lim_pass<kTabLim2Uh, B, B, S, S, 1, B>(T1, nvar, S * S * B * nvar, nc, nvar, o2);
    __syncthreads();
    lim_pass<kTabLim2Uh, B, B, B, S, 2, B>(T2, nvar, S * B * B * nvar, nc, nvar, go);
  }
}

// ------------------------------------------------ min/max and the DMP
// Per cell: luh (nvar per point) + two scratch arrays for the observables +
// per-line partial extrema of the two final passes.
template <int DIM, int B>
__host__ __device__ constexpr int lim_mm_scratch_per_obs() {
  // pass-x and pass-y results of the subcell projection (the larger one)
  return DIM == 3 ? B * B * (2 * B - 1) + B * (2 * B - 1) * (2 * B - 1) : B * (2 * B - 1);
}
template <int DIM, int B>
__host__ __device__ constexpr int lim_mm_lines() {
  // final-pass lines: Gauss-Lobatto (B^(dim-1)) + subcells (S^(dim-1))
  return DIM == 3 ? B * B + (2 * B - 1) * (2 * B - 1) : B + (2 * B - 1);
}

// Projects the observables of the staged cells with table TAB (B -> NO per
// direction); the extrema of every final-pass line land in pmn/pmx[item].
template <int DIM, int B, int TAB, int NO>
__device__ __forceinline__ void lim_mm_project(const double* A, int nvar, int nobs, int nc, double* T1, double* T2,
                                               double* pmn, double* pmx) {
  constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  MinMaxOut mm{pmn, pmx};
  if (DIM == 2) {
    SmemOut o1{T1, nobs, NO * B * nobs, NO, B};
    lim_pass<TAB, B, B, B, 1, 0, NO>(A, nvar, NPC * nvar, nc, nobs, o1);
    __syncthreads();
    lim_pass<TAB, B, NO, B, 1, 1, NO>(T1, nobs, NO * B * nobs, nc, nobs, mm);
  } else {
    SmemOut o1{T1, nobs, B * B * NO * nobs, NO, B};
    lim_pass<TAB, B, B, B, B, 0, NO>(A, nvar, NPC * nvar, nc, nobs, o1);
    __syncthreads();
    SmemOut o2{T2, nobs, B * NO * NO * nobs, NO, NO};
    lim_pass<TAB, B, NO, B, B, 1, NO>(T1, nobs, B * B * NO * nobs, nc, nobs, o2);
    __syncthreads();
    lim_pass<TAB, B, NO, NO, B, 2, NO>(T2, nobs, B * NO * NO * nobs, nc, nobs, mm);
  }
  __syncthreads();
}

// mode 0: findCellLocalMinAndMax, result copied to all faces;
// mode 1: discreteMaximumPrincipleAndMinAndMaxSearch (obs_min/max in/out,
//         dmp_ok[cell] = 1 if the DMP holds).
template <int DIM, int B>
__global__ void __launch_bounds__(kLimNT) k_lim_min_max(int mode, int nvar, int nobs, long ncells, int cpb,
                                                        const double* luh, double relaxation, double scaling,
                                                        double* obs_min, double* obs_max, int* dmp_ok) {
  constexpr int S = 2 * B - 1;
  constexpr int NPC = DIM == 3 ? B * B * B : B * B;
  constexpr int LOB_LINES = DIM == 3 ? B * B : B;
  constexpr int SUB_LINES = DIM == 3 ? S * S : S;
  constexpr int LINES = LOB_LINES + SUB_LINES;
  constexpr int NF = 2 * DIM;
  extern __shared__ double sm[];
  const long c0 = (long)blockIdx.x * cpb;
  const int nc = (int)min((long)cpb, ncells - c0);
  double* A = sm;
  double* T1 = A + cpb * NPC * nvar;
  double* T2 = T1 + cpb * (DIM == 3 ? B * B * S : B * S) * nobs;
  double* pmn = T1 + cpb * lim_mm_scratch_per_obs<DIM, B>() * nobs;  // [c][LINES][nobs]
  double* pmx = pmn + cpb * LINES * nobs;
  if (mode == 1)
    for (int c = threadIdx.x; c < nc; c += blockDim.x) dmp_ok[c0 + c] = 1;
  lim_copy_in(A, luh + c0 * NPC * nvar, (long)nc * NPC * nvar);
  __syncthreads();
  // line extrema: Gauss-Lobatto lines in [0, cpb LOB_LINES nobs), subcell
  // lines after them (items numbered (cell, line, observable))
  lim_mm_project<DIM, B, kTabUh2Lob, B>(A, nvar, nobs, nc, T1, T2, pmn, pmx);
  lim_mm_project<DIM, B, kTabUh2Lim, S>(A, nvar, nobs, nc, T1, T2, pmn + cpb * LOB_LINES * nobs,
                                         pmx + cpb * LOB_LINES * nobs);
  // reduction: one warp per (cell, observable)
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  for (int pair = warp; pair < nc * nobs; pair += blockDim.x / 32) {
    const int c = pair / nobs, v = pair % nobs;
    double mn = DBL_MAX, mx = -DBL_MAX;
    for (int p = lane; p < NPC; p += 32) {
      const double q = A[(c * NPC + p) * nvar + v];
      mn = fmin(mn, q);
      mx = fmax(mx, q);
    }
    for (int l = lane; l < LOB_LINES; l += 32) {
      const int k = (c * LOB_LINES + l) * nobs + v;
      mn = fmin(mn, pmn[k]);
      mx = fmax(mx, pmx[k]);
    }
    for (int l = lane; l < SUB_LINES; l += 32) {
      const int k = cpb * LOB_LINES * nobs + (c * SUB_LINES + l) * nobs + v;
      mn = fmin(mn, pmn[k]);
      mx = fmax(mx, pmx[k]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane != 0) continue;
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
        lo = fmin(lo, bmn[f * nobs + v]);
        hi = fmax(hi, bmx[f * nobs + v]);
      }
      const double sd = fmax((hi - lo) * scaling, relaxation);
      if (mn < lo - sd || mx > hi + sd) atomicAnd(dmp_ok + c0 + c, 0);
      bmn[v] = mn;
      bmx[v] = mx;
      bmn[v + nobs] = lo;
      bmx[v + nobs] = hi;
    }
  }
}

// findCellLocalLimiterMinAndMax: extrema over the staged interior subcells,
// one warp per (cell, observable), written to every face block
template <int DIM, int B>
__global__ void __launch_bounds__(kLimNT) k_lim_fv_min_max(int nvar, int nobs, int ghost, long ncells, int cpb,
                                                           const double* lim, double* obs_min, double* obs_max) {
  constexpr int S = 2 * B - 1;
  constexpr int NS = DIM == 3 ? S * S * S : S * S;
  extern __shared__ double sm[];
  const long c0 = (long)blockIdx.x * cpb;
  const int nc = (int)min((long)cpb, ncells - c0);
  const int SG = S + 2 * ghost;
  const long lim_cell = (long)nvar * (DIM == 3 ? SG * SG * SG : SG * SG);
  lim_stage_interior<DIM, S>(sm, lim + c0 * lim_cell, lim_cell, nvar, ghost, nc);
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  for (int pair = warp; pair < nc * nobs; pair += blockDim.x / 32) {
    const int c = pair / nobs, v = pair % nobs;
    double mn = DBL_MAX, mx = -DBL_MAX;
    for (int p = lane; p < NS; p += 32) {
      const double q = sm[((long)c * NS + p) * nvar + v];
      mn = fmin(mn, q);
      mx = fmax(mx, q);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if (lane == 0)
      for (int f = 0; f < 2 * DIM; f++) {
        obs_min[((c0 + c) * 2 * DIM + f) * nobs + v] = mn;
        obs_max[((c0 + c) * 2 * DIM + f) * nobs + v] = mx;
      }
  }
}

template <int DIM, int B>
__host__ __device__ constexpr int lim_mm_doubles(int nvar, int nobs) {
  return (DIM == 3 ? B * B * B : B * B) * nvar + (lim_mm_scratch_per_obs<DIM, B>() + 2 * lim_mm_lines<DIM, B>()) * nobs;
}

// cells per CTA: enough final-pass items for two rounds of the CTA's
// threads, within the shared-memory budget
static int lim_cpb(long items_per_cell, long smem_per_cell, long ncells) {
  long cpb = (2 * kLimNT + items_per_cell - 1) / items_per_cell;
  if (cpb > 64) cpb = 64;
  const long cap = kLimMaxSmem / smem_per_cell;
  if (cpb > cap) cpb = cap;
  if (cpb > ncells) cpb = ncells;
  return (int)(cpb < 1 ? 1 : cpb);
}

enum LimOp { kLimToFv = 0, kLimToDg = 1, kLimMinMax = 2, kLimDmp = 3, kLimFvMinMax = 4 };

template <int DIM, int B>
static exa_status_t lim_run(int op, int nvar, int nobs, int ghost, long ncells, const double* in, double* out,
                            double* mn, double* mx, int* ok, double relax, double scaling, cudaStream_t st) {
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
    per_cell = lim_mm_doubles<DIM, B>(nvar, nobs);
    items = (long)lim_mm_lines<DIM, B>() * nobs;
  }
  per_cell *= (long)sizeof(double);
  if (per_cell > kLimMaxSmem) return set_error(EXA_EINVAL, "limiter: cell too large for shared memory");
  const int cpb = lim_cpb(items, per_cell, ncells);
  const size_t smem = (size_t)cpb * per_cell;
  const long nblk = (ncells + cpb - 1) / cpb;
  if (nblk > 0x7fffffffL) return set_error(EXA_EINVAL, "limiter: too many cells");
  cudaError_t e = cudaSuccess;
  if (op == kLimToFv) {
    e = cudaFuncSetAttribute(k_lim_to_fv<DIM, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_lim_to_fv<DIM, B><<<(unsigned)nblk, kLimNT, smem, st>>>(nvar, ghost, ncells, cpb, in, out);
  } else if (op == kLimToDg) {
    e = cudaFuncSetAttribute(k_lim_to_dg<DIM, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_lim_to_dg<DIM, B><<<(unsigned)nblk, kLimNT, smem, st>>>(nvar, ghost, ncells, cpb, in, out);
  } else if (op == kLimFvMinMax) {
    e = cudaFuncSetAttribute(k_lim_fv_min_max<DIM, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      k_lim_fv_min_max<DIM, B><<<(unsigned)nblk, kLimNT, smem, st>>>(nvar, nobs, ghost, ncells, cpb, in, mn, mx);
  } else {
    e = cudaFuncSetAttribute(k_lim_min_max<DIM, B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
      k_lim_min_max<DIM, B><<<(unsigned)nblk, kLimNT, smem, st>>>(op == kLimDmp ? 1 : 0, nvar, nobs, ncells, cpb, in,
                                                                   relax, scaling, mn, mx, ok);
  }
  if (e != cudaSuccess) return cuda_status(e, "limiter: shared-memory attribute");
  count_launch();
  return cuda_status(cudaGetLastError(), "limiter kernel");
}

template <int DIM>
static exa_status_t lim_dispatch(int op, int order, int nvar, int nobs, int ghost, long ncells, const double* in,
                                 double* out, double* mn, double* mx, int* ok, double relax, double scaling,
                                 cudaStream_t st) {
  switch (order) {
    case 1: return lim_run<DIM, 2>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
    case 2: return lim_run<DIM, 3>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
    case 3: return lim_run<DIM, 4>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
    case 4: return lim_run<DIM, 5>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
    case 5: return lim_run<DIM, 6>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
    case 6: return lim_run<DIM, 7>(op, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
  }
  return set_error(EXA_EINVAL, "limiter: order must be in 1..6");
}

static exa_status_t lim_entry(int op, int dim, int order, int nvar, int nobs, int ghost, long ncells,
                              const double* in, double* out, double* mn, double* mx, int* ok, double relax,
                              double scaling, void* stream) {
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
  return dim == 2 ? lim_dispatch<2>(op, order, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st)
                  : lim_dispatch<3>(op, order, nvar, nobs, ghost, ncells, in, out, mn, mx, ok, relax, scaling, st);
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
