/*
 * extern "C" entry points over the reference's own OpenMP solvers, verifiers
 * and graph loader (compiled from the reference tree into oracle/_ref).
 * TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: loaded by the tests and by bench.py's
 * CPU-baseline and reference legs, never by the product library.
 *
 * Bound symbols (C++ linkage in the reference):
 *   PRSolver      src/pr/pr.h:23,      defined in src/pr/omp_base.cc:9
 *   PRVerifier    src/pr/pr.h:24,      defined in src/pr/verifier.cc:10
 *   SpmvSolver    src/spmv/spmv.h:29,  defined in src/spmv/omp_base.cc:8
 *   SpmvVerifier  src/spmv/spmv.h:30,  defined in src/spmv/verifier.cc:24
 *   SymGSSolver   src/symgs/symgs.h:28, defined in src/symgs/omp_base.cc:28
 *   read_graph    include/graph_io.h:280
 */
#include "common.h"
#include "graph_io.h"

#include <vector>

double gpr_ref_epsilon = 0.001;  // src/pr/pr.h:4
int gpr_ref_max_iter = 30;       // src/pr/pr.h:5

void PRSolver(int m, int nnz, int *in_row_offsets, int *in_column_indices,
              int *out_row_offsets, int *out_column_indices, int *degree,
              ScoreT *scores);
void PRVerifier(int m, int *in_row_offsets, int *in_column_indices,
                int *out_row_offsets, int *out_column_indices, int *degree,
                float *scores, double target_error);
void SpmvSolver(int m, int nnz, int *Ap, int *Aj, float *Ax, float *x, float *y);
void SpmvVerifier(int m, int nnz, int *Ap, int *Aj, float *Ax, float *x,
                  float *y, float *test_y);
void SymGSSolver(int m, int nnz, int *Ap, int *Aj, int *indices, ValueType *Ax, ValueType *x,
                 ValueType *b, std::vector<int> color_offsets);

extern "C" {

void ref_set_constants(double epsilon, int max_iter) {
  gpr_ref_epsilon = epsilon;
  gpr_ref_max_iter = max_iter;
}

void ref_pr_solver(int m, int nnz, int *in_rowptr, int *in_col, int *out_rowptr,
                   int *out_col, int *degree, float *scores) {
  PRSolver(m, nnz, in_rowptr, in_col, out_rowptr, out_col, degree, scores);
  fflush(stdout);
}

void ref_pr_verifier(int m, int *in_rowptr, int *in_col, int *out_rowptr,
                     int *out_col, int *degree, float *scores, double target) {
  PRVerifier(m, in_rowptr, in_col, out_rowptr, out_col, degree, scores, target);
  fflush(stdout);
}

void ref_spmv_solver(int m, int nnz, int *Ap, int *Aj, float *Ax, float *x, float *y) {
  SpmvSolver(m, nnz, Ap, Aj, Ax, x, y);
  fflush(stdout);
}

void ref_spmv_verifier(int m, int nnz, int *Ap, int *Aj, float *Ax, float *x,
                       float *y, float *test_y) {
  SpmvVerifier(m, nnz, Ap, Aj, Ax, x, y, test_y);
  fflush(stdout);
}

/* SymGSSolver (src/symgs/symgs.h:28, omp_base.cc:28-45) with the colour
 * boundaries passed as an array of n_offsets ints. */
void ref_symgs_solver(int m, int nnz, int *Ap, int *Aj, int *indices, float *Ax, float *x,
                      float *b, int *color_offsets, int n_offsets) {
  std::vector<int> co(color_offsets, color_offsets + n_offsets);
  SymGSSolver(m, nnz, Ap, Aj, indices, Ax, x, b, co);
  fflush(stdout);
}

/* read_graph with explicit flags; arrays are malloc'd by the reference
 * loader and released with ref_free. */
int ref_read_graph(const char *path, int symmetrize, int transpose, int sorted,
                   int remove_selfloops, int remove_redundents, int *m_out,
                   int *nnz_out, int **rowptr, int **col, int **degree,
                   float **weight) {
  char *argv[2];
  argv[0] = (char *)"ref";
  argv[1] = (char *)path;
  int m = 0, n = 0, nnz = 0;
  read_graph(2, argv, m, n, nnz, *rowptr, *col, *degree, *weight,
             symmetrize != 0, transpose != 0, sorted != 0,
             remove_selfloops != 0, remove_redundents != 0);
  *m_out = m;
  *nnz_out = nnz;
  fflush(stdout);
  return 0;
}

void ref_free(void *p) { free(p); }

}  // extern "C"
