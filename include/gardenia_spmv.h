/*
 * gardenia_spmv.h -- C++ drop-in for the reference's SpMV driver surface
 * (src/spmv/spmv.h:29-30): y <- y + A*x over a CSR matrix, host arrays,
 * y updated in place; stdout "\truntime [gpr_b200] = X ms."; failures print
 * to stderr and exit, as the reference does.
 */
#ifndef GARDENIA_SPMV_H_
#define GARDENIA_SPMV_H_

typedef float ValueType; /* include/common.h:16, src/spmv/spmv.h:28 */

void SpmvSolver(int m, int nnz, int *Ap, int *Aj, ValueType *Ax, ValueType *x,
                ValueType *y);
/* src/spmv/verifier.cc:24-62: serial recompute from (x, y), maximum relative
 * error against test_y, "Correct" if <= 5*sqrt(FLT_EPSILON). */
void SpmvVerifier(int m, int nnz, int *Ap, int *Aj, ValueType *Ax, ValueType *x,
                  ValueType *y, ValueType *test_y);

#endif
