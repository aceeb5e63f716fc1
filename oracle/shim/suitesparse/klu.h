/*
 * Stand-in declarations for the SuiteSparse KLU interface, used only to
 * compile the reference's own sources as an oracle here (SuiteSparse is not
 * installed).  Only the fields and functions the reference touches are
 * declared (blockdaglu/src/klu_dynamic.h:20-43; fields used in solver.cpp and
 * ubtf_block_solver.cpp).  The implementation in klu_standin.c is a dense
 * partial-pivoting LU, not KLU; results of the reference's KLU route built on
 * it are labelled "KLU unavailable on this box".
 */
#ifndef BDLU_SHIM_KLU_H_
#define BDLU_SHIM_KLU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KLU_OK 0
#define KLU_SINGULAR 1
#define KLU_OUT_OF_MEMORY (-2)
#define KLU_INVALID (-3)
#define KLU_TOO_LARGE (-4)

typedef struct klu_common_struct {
  double tol;            /* pivot tolerance: keep the diagonal if |a_kk| >= tol * max */
  int btf;
  int ordering;
  int scale;             /* 0/-1 none, 1 sum, 2 max row scaling */
  int halt_if_singular;
  int status;
  int numerical_rank;
  double rcond;          /* min |u_kk| / max |u_kk| */
} klu_common;

typedef struct klu_symbolic_struct {
  int32_t n;
  int32_t nblocks;
  int32_t* P;
  int32_t* Q;
  int32_t* R;
} klu_symbolic;

typedef struct klu_numeric_struct {
  int32_t n;
  int32_t lnz;
  int32_t unz;
  int32_t nzoff;
  double* lu;      /* column-major n*n */
  int32_t* perm;   /* factor row k = original row perm[k] */
  double* rs;      /* row scale by original row, 1 if unscaled */
} klu_numeric;

int klu_defaults(klu_common* common);
klu_symbolic* klu_analyze(int32_t n, int32_t* Ap, int32_t* Ai, klu_common* common);
klu_symbolic* klu_analyze_given(int32_t n, int32_t* Ap, int32_t* Ai, int32_t* P, int32_t* Q, klu_common* common);
klu_numeric* klu_factor(int32_t* Ap, int32_t* Ai, double* Ax, klu_symbolic* symbolic, klu_common* common);
int klu_solve(klu_symbolic* symbolic, klu_numeric* numeric, int32_t ldim, int32_t nrhs, double* B, klu_common* common);
int klu_extract(klu_numeric* numeric, klu_symbolic* symbolic, int32_t* Lp, int32_t* Li, double* Lx, int32_t* Up,
                int32_t* Ui, double* Ux, int32_t* Fp, int32_t* Fi, double* Fx, int32_t* P, int32_t* Q, double* Rs,
                int32_t* R, klu_common* common);
int klu_free_symbolic(klu_symbolic** symbolic, klu_common* common);
int klu_free_numeric(klu_numeric** numeric, klu_common* common);

#ifdef __cplusplus
}
#endif

#endif
