/*
 * extern "C" entry points over the reference's own CUDA solvers, recompiled
 * for sm_100a from the reference tree into oracle/_ref (a second baseline on
 * the GPU).  TEST INFRASTRUCTURE ONLY: loaded by the tests, never by the
 * product library.  One shared library per solver file, since every variant
 * defines the same C++ symbol:
 *   REF_GPU_PR    PRSolver    src/pr/pr.h:23, defined in src/pr/gather.cu or gather_warp.cu
 *   REF_GPU_SPMV  SpmvSolver  src/spmv/spmv.h:29, defined in src/spmv/base.cu
 */
#include <stdio.h>

double gpr_ref_epsilon = 0.001;  // src/pr/pr.h:4
int gpr_ref_max_iter = 30;       // src/pr/pr.h:5

extern "C" void ref_set_constants(double epsilon, int max_iter) {
  gpr_ref_epsilon = epsilon;
  gpr_ref_max_iter = max_iter;
}

#ifdef REF_GPU_PR
void PRSolver(int m, int nnz, int *in_row_offsets, int *in_column_indices,
              int *out_row_offsets, int *out_column_indices, int *degree, float *scores);
extern "C" void ref_gpu_pr_solver(int m, int nnz, int *in_rowptr, int *in_col, int *degree,
                                  float *scores) {
  PRSolver(m, nnz, in_rowptr, in_col, in_rowptr, in_col, degree, scores);
  fflush(stdout);
}
#endif

#ifdef REF_GPU_SPMV
void SpmvSolver(int m, int nnz, int *Ap, int *Aj, float *Ax, float *x, float *y);
extern "C" void ref_gpu_spmv_solver(int m, int nnz, int *Ap, int *Aj, float *Ax, float *x,
                                    float *y) {
  SpmvSolver(m, nnz, Ap, Aj, Ax, x, y);
  fflush(stdout);
}
#endif
