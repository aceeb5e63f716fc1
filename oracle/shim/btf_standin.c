/*
 * btf_order for the reference build under oracle/_ref: forwards to the
 * engine's btf_order (libbdlu.so, same calling convention), so the reference's
 * merge, UBTF split, DAG and block factors can be compared with the engine's
 * starting from the same permutation.  SuiteSparse's own traversal order is
 * not available here; the block partition (strongly connected components) is
 * checked independently against scipy in tests/test_analysis.py.  maxwork is
 * ignored and work reports 0.  Test infrastructure only.
 */
#include <stdint.h>

#include "suitesparse/btf.h"

extern int32_t bdlu_btf_order(int32_t n, const int32_t* Ap, const int32_t* Ai, int32_t* P, int32_t* Q, int32_t* R,
                              int32_t* nmatch);

int32_t btf_order(int32_t n, int32_t* Ap, int32_t* Ai, double maxwork, double* work, int32_t* P, int32_t* Q,
                  int32_t* R, int32_t* nmatch, int32_t* Work) {
  (void)maxwork;
  (void)Work;
  if (work) *work = 0.0;
  return bdlu_btf_order(n, Ap, Ai, P, Q, R, nmatch);
}
