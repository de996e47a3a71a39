// C++ drop-ins with the reference's symbols (src/pr/pr.h:23-24,
// src/spmv/spmv.h:29-30, src/symgs/symgs.h:28-29) over the C ABI of gpr.h.  Output lines and the
// print-and-exit error convention follow the reference drivers.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "gardenia_pr.h"
#include "gardenia_spmv.h"
#include "gardenia_symgs.h"
#include "gardenia_timer.h"
#include "gpr.h"

namespace {

[[noreturn]] void die(const char *where) {
  fprintf(stderr, "%s: %s\n", where, gpr_last_error());
  exit(EXIT_FAILURE);
}

// EPSILON / MAX_ITER of src/pr/pr.h:4-5, overridable at run time.
void pr_constants(double *tol, int *max_iter) {
  *tol = 0.001;
  *max_iter = 30;
  if (const char *e = getenv("GPR_TOL")) *tol = atof(e);
  if (const char *e = getenv("GPR_MAX_ITER")) *max_iter = atoi(e);
}

void pr_run(int m, int nnz, int *rowptr, int *col, int *degree, ScoreT *scores) {
  gpr_pr_opts o;
  gpr_pr_opts_default(&o);
  pr_constants(&o.tol, &o.max_iter);
  o.damping = kDamp;
  printf("Launching B200 PR solver (gpr, sm_100a) ...\n");
  gpr_graph *g = nullptr;
  if (gpr_graph_create(m, nnz, rowptr, col, degree, &g) != GPR_OK) die("PRSolver");
  gpr_pr_stats st;
  if (gpr_pagerank(g, scores, &o, &st) != GPR_OK) die("PRSolver");
  std::vector<double> hist(st.iterations > 0 ? st.iterations : 1);
  if (gpr_graph_residuals(g, hist.data(), st.iterations) != GPR_OK) die("PRSolver");
  for (int i = 0; i < st.iterations; ++i) printf(" %2d    %lf\n", i + 1, hist[i]);
  printf("\titerations = %d.\n", st.iterations);
  printf("\truntime [%s] = %f ms.\n", "gpr_b200", st.solve_ms);
  gpr_graph_destroy(g);
}

}  // namespace

void PRSolver(int m, int nnz, int *in_row_offsets, int *in_column_indices,
              int *out_row_offsets, int *out_column_indices, int *degree, ScoreT *scores) {
  (void)out_row_offsets;  // the pull solver reads the in-CSR only (src/pr/gather.cu:41)
  (void)out_column_indices;
  pr_run(m, nnz, in_row_offsets, in_column_indices, degree, scores);
}

void PageRank(int m, int nnz, int *row_offsets, int *column_indices, int *degree,
              ScoreT *scores) {
  pr_run(m, nnz, row_offsets, column_indices, degree, scores);
}

// src/pr/verifier.cc:10-69: a serial pull run (timed, printed, not compared),
// then one serial PUSH sweep from the scores under test over the out-CSR;
// "Correct" when its L1 distance to those scores is below target_error.
void PRVerifier(int m, int *in_row_offsets, int *in_column_indices, int *out_row_offsets,
                int *out_column_indices, int *degree, ScoreT *scores_to_test,
                double target_error) {
  printf("Verifying...\n");
  double tol;
  int max_iter;
  pr_constants(&tol, &max_iter);
  const ScoreT base = (1.0f - kDamp) / m;
  std::vector<ScoreT> s(m, 1.0f / m), contrib(m);
  Timer t;
  t.Start();
  int it = 0;
  for (; it < max_iter; ++it) {
    double error = 0;
    for (int n = 0; n < m; ++n) contrib[n] = s[n] / degree[n];
    for (int v = 0; v < m; ++v) {
      ScoreT total = 0;
      for (int e = in_row_offsets[v]; e < in_row_offsets[v + 1]; ++e)
        total += contrib[in_column_indices[e]];
      const ScoreT old = s[v];
      s[v] = base + kDamp * total;
      error += fabsf(s[v] - old);
    }
    printf(" %2d    %lf\n", it + 1, error);
    if (error < tol) break;
  }
  t.Stop();
  printf("\titerations = %d.\n", it + 1);
  printf("\truntime [serial] = %f ms.\n", t.Millisecs());
  std::vector<float> sums(m, 0.0f);
  for (int u = 0; u < m; ++u) {
    const float c = scores_to_test[u] / degree[u];
    for (int e = out_row_offsets[u]; e < out_row_offsets[u + 1]; ++e)
      sums[out_column_indices[e]] += c;
  }
  double error = 0;
  for (int v = 0; v < m; ++v) error += fabsf(base + kDamp * sums[v] - scores_to_test[v]);
  if (error < target_error) printf("Correct\n");
  else printf("Total Error: %f\n", error);
}

void SpmvSolver(int m, int nnz, int *Ap, int *Aj, ValueType *Ax, ValueType *x, ValueType *y) {
  printf("Launching B200 SpMV solver (gpr, sm_100a) ...\n");
  gpr_matrix *A = nullptr;
  if (gpr_matrix_create(m, nnz, Ap, Aj, Ax, &A) != GPR_OK) die("SpmvSolver");
  float *dx = nullptr, *dy = nullptr;
  cudaEvent_t e0, e1;
  if (cudaMalloc(&dx, sizeof(float) * (m ? m : 1)) != cudaSuccess ||
      cudaMalloc(&dy, sizeof(float) * (m ? m : 1)) != cudaSuccess ||
      cudaMemcpy(dx, x, sizeof(float) * m, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dy, y, sizeof(float) * m, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    fprintf(stderr, "SpmvSolver: CUDA setup failed\n");
    exit(EXIT_FAILURE);
  }
  cudaEventRecord(e0, 0);
  if (gpr_spmv(A, dx, dy, nullptr) != GPR_OK) die("SpmvSolver");
  cudaEventRecord(e1, 0);
  if (cudaMemcpy(y, dy, sizeof(float) * m, cudaMemcpyDeviceToHost) != cudaSuccess) {
    fprintf(stderr, "SpmvSolver: copy back failed\n");
    exit(EXIT_FAILURE);
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  printf("\truntime [%s] = %f ms.\n", "gpr_b200", ms);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dx);
  cudaFree(dy);
  gpr_matrix_destroy(A);
}

// src/spmv/verifier.cc:9-62.
void SpmvVerifier(int m, int nnz, int *Ap, int *Aj, ValueType *Ax, ValueType *x, ValueType *y,
                  ValueType *test_y) {
  (void)nnz;
  printf("Verifying...\n");
  std::vector<ValueType> ref(y, y + m);
  Timer t;
  t.Start();
  for (int i = 0; i < m; ++i) {
    ValueType sum = ref[i];
    for (int jj = Ap[i]; jj < Ap[i + 1]; ++jj) sum += x[Aj[jj]] * Ax[jj];
    ref[i] = sum;
  }
  t.Stop();
  printf("\truntime [serial] = %f ms.\n", t.Millisecs());
  const float eps = sqrtf(FLT_EPSILON);
  float max_error = 0.0f;
  for (int i = 0; i < m; ++i) {
    const float err = fabsf(test_y[i] - ref[i]);
    if (err != 0.0f) {
      const float r = err / (fabsf(test_y[i]) + fabsf(ref[i]) + eps);
      if (r > max_error) max_error = r;
    }
  }
  printf("\t[max error %9f]\n", max_error);
  if (max_error > 5 * sqrtf(FLT_EPSILON)) printf("POSSIBLE FAILURE\n");
  else printf("Correct\n");
}

// ---- SymGS ---------------------------------------------------------------

void SymGSSolver(int m, int nnz, int *Ap, int *Aj, int *indices, ValueType *Ax, ValueType *x,
                 ValueType *b, std::vector<int> color_offsets) {
  printf("Launching B200 SymGS solver (gpr, sm_100a, %d colours) ...\n",
         (int)color_offsets.size() - 1);
  gpr_symgs *h = nullptr;
  if (gpr_symgs_create(m, nnz, Ap, Aj, Ax, indices, color_offsets.data(),
                       (int)color_offsets.size() - 1, &h) != GPR_OK)
    die("SymGSSolver");
  double ms = 0.0;
  if (gpr_symgs_apply(h, x, b, 1, &ms) != GPR_OK) die("SymGSSolver");
  gpr_symgs_destroy(h);
  printf("\truntime [%s] = %f ms.\n", "gpr_b200", ms);
}

namespace {

// One row sweep of src/symgs/verifier.cc:56-70 (gs_serial).
void gs_rows(const int *Ap, const int *Aj, const int *indices, const ValueType *Ax, ValueType *x,
             const ValueType *b, int begin, int end) {
  for (int i = begin; i != end; ++i) {
    const int r = indices[i];
    ValueType rsum = 0, diag = 0;
    for (int jj = Ap[r]; jj < Ap[r + 1]; ++jj) {
      const int j = Aj[jj];
      if (j == r) diag = Ax[jj];
      else rsum += x[j] * Ax[jj];
    }
    if (diag != 0) x[r] = (b[r] - rsum) / diag;
  }
}

}  // namespace

void SymGSVerifier(int num_rows, int *Ap, int *Aj, int *indices, ValueType *Ax,
                   ValueType *test_x, ValueType *x_host, ValueType *b,
                   std::vector<int> color_offsets) {
  printf("Verifying...\n");
  std::vector<ValueType> x(x_host, x_host + num_rows);
  Timer t;
  t.Start();
  const int nc = (int)color_offsets.size() - 1;
  for (int c = 0; c < nc; ++c)
    gs_rows(Ap, Aj, indices, Ax, x.data(), b, color_offsets[c], color_offsets[c + 1]);
  for (int c = nc; c > 0; --c)
    gs_rows(Ap, Aj, indices, Ax, x.data(), b, color_offsets[c - 1], color_offsets[c]);
  t.Stop();
  printf("\truntime [verify] = %f ms.\n", t.Millisecs());
  const ValueType eps = sqrtf(FLT_EPSILON);
  ValueType max_error = 0;
  bool ok = true;
  for (int i = 0; i < num_rows; ++i) {
    const ValueType a = test_x[i], r = x[i];
    const ValueType err = fabsf(a - r);
    if (err != 0) max_error = fmaxf(max_error, err / (fabsf(a) + fabsf(r) + eps));
    if (ok && fabs((double)(a - r)) > 1e-4 * (fabs((double)a) + fabs((double)r)) + 1e-4) {
      ok = false;
      printf("x_test[%d] (%f) != x[%d] (%f)\n", i, a, i, r);
    }
  }
  printf("\t[max error %9f]\n", max_error);
  printf(ok ? "Correct\n" : "POSSIBLE FAILURE\n");
}
