/*
 * gardenia_pr.h -- C++ drop-in for the reference's PageRank driver surface.
 *
 * Same names, parameter types and C++ linkage as src/pr/pr.h:23-24, so a
 * driver written against the reference (src/pr/main.cc) links against
 * libgpr.so instead of one of the reference's solver objects
 * (src/pr/Makefile:17-47).  Semantics follow the reference's pull solvers:
 *   - scores holds the initial scores on entry and the result on return;
 *   - EPSILON / MAX_ITER default to the reference's 0.001 / 30
 *     (src/pr/pr.h:4-5); the environment variables GPR_TOL and GPR_MAX_ITER
 *     override them at run time (the reference needs a recompile);
 *   - stdout carries the reference's lines: one " %2d    %lf" residual line
 *     per sweep, "\titerations = N." and "\truntime [gpr_b200] = X ms.";
 *   - on any failure the message goes to stderr and the process exits with
 *     EXIT_FAILURE, as CUDA_SAFE_CALL does (include/cutil_subset.h:4-12).
 * The C ABI in gpr.h offers the same solvers with status codes instead.
 */
#ifndef GARDENIA_PR_H_
#define GARDENIA_PR_H_

typedef float ScoreT;          /* include/common.h:13 */
static const float kDamp = 0.85f; /* include/common.h:18 */

/* src/pr/pr.h:23 -- the out-CSR is accepted and ignored (pull solver). */
void PRSolver(int m, int nnz, int *in_row_offsets, int *in_column_indices,
              int *out_row_offsets, int *out_column_indices, int *degree,
              ScoreT *scores);
/* src/pr/pr.h:24 -- serial pull reference run plus the one-sweep push check
 * of src/pr/verifier.cc:10-69; prints "Correct" or "Total Error: X". */
void PRVerifier(int m, int *in_row_offsets, int *in_column_indices,
                int *out_row_offsets, int *out_column_indices, int *degree,
                ScoreT *scores, double target_error);
/* Pull PageRank over the in-CSR and out-degree (the 6-argument entry point
 * of this path; same behaviour as PRSolver). */
void PageRank(int m, int nnz, int *row_offsets, int *column_indices,
              int *degree, ScoreT *scores);

#endif
