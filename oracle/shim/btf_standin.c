/*
 * btf_order for the reference build under oracle/_ref.  It runs the oracle's
 * own block triangular form (oracle/btf_oracle.c: Hopcroft-Karp maximum
 * transversal + Tarjan components), so the reference build links no engine
 * code.  A parity test can instead inject a given ordering
 * (btf_standin_inject) so that the reference's merge, UBTF split, DAG and
 * block factors are compared with the engine's from the same permutation:
 * SuiteSparse's own traversal order is not available here.  maxwork is
 * ignored and work reports 0.  Test infrastructure only.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "suitesparse/btf.h"

extern int32_t or_btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q, int32_t* R,
                            int32_t* nmatch);

static int32_t g_inj_n = -1, g_inj_nblocks = 0, g_inj_nmatch = 0;
static int32_t *g_inj_P = NULL, *g_inj_Q = NULL, *g_inj_R = NULL;

/* Injects P, Q (SuiteSparse conventions), R[nblocks+1] and nmatch for the
 * next btf_order calls of order n; n < 0 clears the injection. */
void btf_standin_inject(int32_t n, const int32_t* P, const int32_t* Q, const int32_t* R, int32_t nblocks,
                        int32_t nmatch) {
  free(g_inj_P);
  free(g_inj_Q);
  free(g_inj_R);
  g_inj_P = g_inj_Q = g_inj_R = NULL;
  g_inj_n = -1;
  if (n < 0) return;
  g_inj_P = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  g_inj_Q = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  g_inj_R = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nblocks + 1));
  if (!g_inj_P || !g_inj_Q || !g_inj_R) return;
  memcpy(g_inj_P, P, sizeof(int32_t) * (size_t)n);
  memcpy(g_inj_Q, Q, sizeof(int32_t) * (size_t)n);
  memcpy(g_inj_R, R, sizeof(int32_t) * (size_t)(nblocks + 1));
  g_inj_nblocks = nblocks;
  g_inj_nmatch = nmatch;
  g_inj_n = n;
}

int32_t btf_order(int32_t n, int32_t* Ap, int32_t* Ai, double maxwork, double* work, int32_t* P, int32_t* Q,
                  int32_t* R, int32_t* nmatch, int32_t* Work) {
  (void)maxwork;
  (void)Work;
  if (work) *work = 0.0;
  if (g_inj_n == n && g_inj_P) {
    memcpy(P, g_inj_P, sizeof(int32_t) * (size_t)n);
    memcpy(Q, g_inj_Q, sizeof(int32_t) * (size_t)n);
    memcpy(R, g_inj_R, sizeof(int32_t) * (size_t)(g_inj_nblocks + 1));
    if (nmatch) *nmatch = g_inj_nmatch;
    return g_inj_nblocks;
  }
  return or_btf_order(n, Ap, Ai, P, Q, R, nmatch);
}
