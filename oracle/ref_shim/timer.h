/*
 * Build shim for the reference's OpenMP sources (oracle/_ref only).
 *
 * src/pr/pr.h:4-5 hard-codes `#define EPSILON 0.001` and `#define MAX_ITER 30`
 * without include guards, so -D cannot change them.  src/pr/omp_base.cc and
 * src/pr/verifier.cc include "timer.h" right after "pr.h"; this file is found
 * first through -iquote, re-points both names at run-time globals, and then
 * pulls in the reference's own include/timer.h with #include_next.  The
 * reference sources themselves are compiled unmodified where they lie.
 */
#undef EPSILON
#undef MAX_ITER
extern double gpr_ref_epsilon;
extern int gpr_ref_max_iter;
#define EPSILON gpr_ref_epsilon
#define MAX_ITER gpr_ref_max_iter
#include_next "timer.h"
