/*
 * gardenia_symgs.h -- C++ drop-in for the reference's SymGS driver surface
 * (src/symgs/symgs.h:28-29): one multicolour symmetric Gauss-Seidel sweep
 * (colours forward, then backward) over a CSR matrix, host arrays, x updated
 * in place; `indices` lists the rows colour by colour and color_offsets
 * holds the colour boundaries (size = colours + 1).  stdout as the
 * reference's solvers; failures print to stderr and exit.  The colouring
 * must be valid (no entry joins two rows of one colour).
 */
#ifndef GARDENIA_SYMGS_H_
#define GARDENIA_SYMGS_H_

#include <vector>

typedef float ValueType; /* include/common.h:16 */

void SymGSSolver(int m, int nnz, int *Ap, int *Aj, int *indices, ValueType *Ax, ValueType *x,
                 ValueType *b, std::vector<int> color_offsets);
/* src/symgs/verifier.cc:64-88: serial sweep from x_host, maximum relative
 * error against test_x, "Correct" when every entry agrees within 1e-4
 * absolute + 1e-4 relative, else "POSSIBLE FAILURE". */
void SymGSVerifier(int num_rows, int *Ap, int *Aj, int *indices, ValueType *Ax,
                   ValueType *test_x, ValueType *x_host, ValueType *b,
                   std::vector<int> color_offsets);

#endif
