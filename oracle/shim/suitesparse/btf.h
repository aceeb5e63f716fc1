/*
 * Stand-in declaration of SuiteSparse btf_order (blockdaglu/src/btf_dynamic.h:
 * 19-28 calling convention) for compiling the reference's sources as an
 * oracle.  btf_standin.c runs the oracle's own block triangular form
 * (oracle/btf_oracle.c), or an ordering a parity test injected so both sides
 * start from the same permutation (SuiteSparse's own traversal order is not
 * available here).
 */
#ifndef BDLU_SHIM_BTF_H_
#define BDLU_SHIM_BTF_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BTF_FLIP(j) (-(j) - 2)
#define BTF_ISFLIPPED(j) ((j) < -1)
#define BTF_UNFLIP(j) ((BTF_ISFLIPPED(j)) ? BTF_FLIP(j) : (j))

int32_t btf_order(int32_t n, int32_t* Ap, int32_t* Ai, double maxwork, double* work, int32_t* P, int32_t* Q,
                  int32_t* R, int32_t* nmatch, int32_t* Work);

#ifdef __cplusplus
}
#endif

#endif
