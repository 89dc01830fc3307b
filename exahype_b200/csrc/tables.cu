// Host-side derivation of the per-order operator tables uploaded to
// constant memory (exa::DGConst), from the generated dg_tables.h.
#include <mutex>
#include <vector>

#include "exa_device.cuh"

#define EXA_TABLE_QUAL static const
#include "dg_tables.h"

namespace exa {

static DGConst g_tables[kMaxOrder + 1];
static DGConstF g_tables_f[kMaxOrder + 1];
static std::once_flag g_once;

static void build() {
  for (int N = 0; N <= kMaxOrder; N++) {
    DGConst& T = g_tables[N];
    const int B = N + 1;
    for (int i = 0; i < 10; i++) {
      T.w[i] = exa_gl_weights[N][i];
      T.nodes[i] = exa_gl_nodes[N][i];
      T.fl[i] = exa_flcoeff[N][i];
      T.fr[i] = exa_frcoeff[N][i];
      T.c0[i] = 0.0;
      for (int j = 0; j < 10; j++) {
        T.kxi[i][j] = exa_kxi[N][i][j];
        T.deriv[i][j] = 0.0;
        T.tA[i][j] = 0.0;
      }
    }
    for (int l = 0; l < B; l++)
      for (int p = 0; p < B; p++) T.deriv[l][p] = exa_kxi[N][p][l] / exa_gl_weights[N][l];
    for (int t = 0; t < B; t++) {
      double c = 0.0;
      for (int n = 0; n < B; n++) {
        T.tA[t][n] = exa_ik1[N][t][n] * exa_gl_weights[N][n];
        c += exa_ik1[N][t][n] * exa_f0[N][n];
      }
      T.c0[t] = c;
    }
    T.pnpm = exa_pnpm[N];
    DGConstF& F = g_tables_f[N];
    for (int i = 0; i < 10; i++) {
      F.w[i] = (float)T.w[i];
      for (int j = 0; j < 10; j++) {
        F.deriv[i][j] = (float)T.deriv[i][j];
        F.derivT[j][i] = (float)T.deriv[i][j];
        F.tA[i][j] = (float)T.tA[i][j];
      }
    }
  }
}

const void* host_dg_tables(size_t* bytes) {
  std::call_once(g_once, build);
  if (bytes) *bytes = sizeof(g_tables);
  return g_tables;
}

const void* host_dg_tables_f(size_t* bytes) {
  std::call_once(g_once, build);
  if (bytes) *bytes = sizeof(g_tables_f);
  return g_tables_f;
}

double host_pnpm(int order) { return exa_pnpm[order]; }

}  // namespace exa
