/*
 * oracle.c -- CPU restatement of the reference's PageRank / SpMV hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by the
 * tests, by __graft_entry__.smoke() and by the CPU-baseline / reference legs
 * of bench.py.  The product library (gardenia_ocl_b200/) never links, loads
 * or calls it, and there is no CPU fallback built on it.
 *
 * Pinning: orc_pr_plain_f32 and orc_spmv_f32 are checked bit-for-bit against
 * the reference's own OpenMP code compiled from its sources (oracle/_ref,
 * built by oracle/Makefile) on the reference's datasets and on seeded
 * synthetic graphs; tests/golden/ holds the fixtures that carry that pin to
 * machines without the reference tree.
 *
 * Everything here is plain C99 + OpenMP, single precision where the
 * reference is single precision, so results are bit-comparable.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Plain pull PageRank, FP32 values, FP64 L1 residual.                       */
/* Follows src/pr/omp_base.cc:9-49 (PRSolver):                               */
/*   base = (1.0f - kDamp) / m                       (omp_base.cc:16)        */
/*   contrib[n] = scores[n] / degree[n]              (omp_base.cc:25-27)     */
/*   s = base + kDamp * sum_{in-edges} contrib       (omp_base.cc:30-39)     */
/*   error += fabs(s_new - s_old) in double          (omp_base.cc:24,40)     */
/*   stop after the sweep whose error < EPSILON, or after MAX_ITER sweeps    */
/*   (omp_base.cc:23,43).                                                    */
/* kDamp is the float constant 0.85f (include/common.h:18).                  */
/* The per-vertex sum runs in CSR order, one float add per edge, exactly as  */
/* the reference's inner loop (omp_base.cc:34-37).  The `volatile`-free      */
/* expression forms below compile to separate mul/add (no contraction:       */
/* -ffp-contract=off in oracle/Makefile).                                    */
/* Returns the number of sweeps executed; err_hist (may be NULL) receives    */
/* the residual of each sweep.                                               */
/* ------------------------------------------------------------------------ */
int orc_pr_plain_f32(int m, const int *rowptr, const int *col,
                     const int *outdeg, float *scores, float damping,
                     double tol, int max_iter, double *err_hist)
{
    const float base = (1.0f - damping) / (float)m;
    float *contrib = (float *)malloc(sizeof(float) * (size_t)(m > 0 ? m : 1));
    int iter, sweeps = 0;
    for (iter = 0; iter < max_iter; iter++) {
        double error = 0.0;
        int n;
#pragma omp parallel for schedule(static)
        for (n = 0; n < m; n++) contrib[n] = scores[n] / (float)outdeg[n];
#pragma omp parallel for reduction(+ : error) schedule(dynamic, 64)
        for (n = 0; n < m; n++) {
            float total = 0.0f;
            int e;
            for (e = rowptr[n]; e < rowptr[n + 1]; e++) total += contrib[col[e]];
            float old = scores[n];
            float prod = damping * total;
            float s = base + prod;
            scores[n] = s;
            error += (double)fabsf(s - old);
        }
        sweeps = iter + 1;
        if (err_hist) err_hist[iter] = error;
        if (error < tol) break;
    }
    free(contrib);
    return sweeps;
}

/* ------------------------------------------------------------------------ */
/* FP64 fixed point of the same recurrence (the "FP64 host oracle").        */
/* d = (double)damping (so 0.85f -> 0.85000002384185791), base = (1-d)/m,    */
/* no dangling-mass redistribution (omp_base.cc:39 has none).               */
/* Iterates until the L1 change is below tol or max_iter sweeps.            */
/* Returns sweeps executed.                                                  */
/* ------------------------------------------------------------------------ */
int orc_pr_f64(int m, const int *rowptr, const int *col, const int *outdeg,
               double *scores, float damping, double tol, int max_iter,
               double *final_err)
{
    const double d = (double)damping;
    const double base = (1.0 - d) / (double)m;
    double *contrib = (double *)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    int iter, sweeps = 0;
    double error = 0.0;
    for (iter = 0; iter < max_iter; iter++) {
        int n;
        error = 0.0;
#pragma omp parallel for schedule(static)
        for (n = 0; n < m; n++) contrib[n] = scores[n] / (double)outdeg[n];
#pragma omp parallel for reduction(+ : error) schedule(dynamic, 64)
        for (n = 0; n < m; n++) {
            double total = 0.0;
            int e;
            for (e = rowptr[n]; e < rowptr[n + 1]; e++) total += contrib[col[e]];
            double s = base + d * total;
            error += fabs(s - scores[n]);
            scores[n] = s;
        }
        sweeps = iter + 1;
        if (error < tol) break;
    }
    if (final_err) *final_err = error;
    free(contrib);
    return sweeps;
}

/* FP64 residual of a candidate FP32 score vector: r = base + d*M*s - s.
 * Returns ||r||_1; since every column of the pull operator sums to at most
 * d, ||s - s*||_1 <= ||r||_1 / (1 - d). */
double orc_pr_residual_f64(int m, const int *rowptr, const int *col,
                           const int *outdeg, const float *scores, float damping)
{
    const double d = (double)damping;
    const double base = (1.0 - d) / (double)m;
    double r1 = 0.0;
    int n;
#pragma omp parallel for reduction(+ : r1) schedule(dynamic, 64)
    for (n = 0; n < m; n++) {
        double total = 0.0;
        int e;
        for (e = rowptr[n]; e < rowptr[n + 1]; e++) {
            int u = col[e];
            total += (double)scores[u] / (double)outdeg[u];
        }
        r1 += fabs(base + d * total - (double)scores[n]);
    }
    return r1;
}

/* Max / L1 error of an FP32 vector against an FP64 vector. */
void orc_err_vs_f64(int n, const float *a, const double *ref, double *max_err,
                    double *l1_err)
{
    double mx = 0.0, l1 = 0.0;
    int i;
    for (i = 0; i < n; i++) {
        double e = fabs((double)a[i] - ref[i]);
        if (e > mx) mx = e;
        l1 += e;
    }
    *max_err = mx;
    *l1_err = l1;
}

/* ------------------------------------------------------------------------ */
/* The reference verifier's acceptance check (src/pr/verifier.cc:50-68):   */
/* one serial PUSH sweep over the out-CSR from the scores under test, then  */
/* the L1 distance between that sweep and the scores under test.            */
/* ------------------------------------------------------------------------ */
double orc_pr_push_check(int m, const int *out_rowptr, const int *out_col,
                         const int *outdeg, const float *scores, float damping)
{
    const float base = (1.0f - damping) / (float)m;
    float *sums = (float *)calloc((size_t)(m > 0 ? m : 1), sizeof(float));
    double error = 0.0;
    int src, i;
    for (src = 0; src < m; src++) {
        float c = scores[src] / (float)outdeg[src];
        int e;
        for (e = out_rowptr[src]; e < out_rowptr[src + 1]; e++) sums[out_col[e]] += c;
    }
    for (i = 0; i < m; i++) {
        float prod = damping * sums[i];
        float s = base + prod;
        error += (double)fabsf(s - scores[i]);
    }
    free(sums);
    return error;
}

/* ------------------------------------------------------------------------ */
/* CSR SpMV y <- y + A x, FP32, sequential in-row order.                    */
/* Follows src/spmv/omp_base.cc:8-32 (SpmvSolver): sum starts at y[i] and   */
/* adds x[j] * Ax[jj] for jj in row order (omp_base.cc:18-28).              */
/* ------------------------------------------------------------------------ */
void orc_spmv_f32(int m, const int *Ap, const int *Aj, const float *Ax,
                  const float *x, float *y)
{
    int i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < m; i++) {
        float sum = y[i];
        int jj;
        for (jj = Ap[i]; jj < Ap[i + 1]; jj++) {
            float prod = x[Aj[jj]] * Ax[jj];
            sum += prod;
        }
        y[i] = sum;
    }
}

/* maximum_relative_error, src/spmv/verifier.cc:9-22: max over i of
 * |a-b| / (|a| + |b| + sqrt(FLT_EPSILON)), skipping exact matches. */
float orc_max_rel_err_f32(const float *a, const float *b, long long n)
{
    const float eps = sqrtf(1.1920928955078125e-07f);
    float mx = 0.0f;
    long long i;
    for (i = 0; i < n; i++) {
        float err = fabsf(a[i] - b[i]);
        if (err != 0.0f) {
            float r = err / (fabsf(a[i]) + fabsf(b[i]) + eps);
            if (r > mx) mx = r;
        }
    }
    return mx;
}

/* ------------------------------------------------------------------------ */
/* Batched personalized PageRank (no reference file: the reference computes
 * one global PageRank). */
/* For each vector q with seed s_q:                                          */
/*   x_new[v] = d * sum_{u in in(v)} x[u]/outdeg[u]                          */
/*            + [v == s_q] * ((1 - d) + d * dangling_q)                      */
/*   dangling_q = sum over outdeg==0 vertices u of x[u]    (FP64)            */
/* x starts at e_{s_q}.  Vector q stops updating after the first sweep whose */
/* L1 change is below tol.  x is row-major [m][k].  FP64 throughout.         */
/* iters[q] receives the sweeps vector q executed.                           */
/* ------------------------------------------------------------------------ */
void orc_ppr_f64(int m, const int *rowptr, const int *col, const int *outdeg,
                 int k, const int *seeds, float damping, double tol,
                 int max_iter, double *x, int *iters)
{
    const double d = (double)damping;
    double *c = (double *)malloc(sizeof(double) * (size_t)m * (size_t)k);
    double *xn = (double *)malloc(sizeof(double) * (size_t)m * (size_t)k);
    double *dang = (double *)malloc(sizeof(double) * (size_t)k);
    double *err = (double *)malloc(sizeof(double) * (size_t)k);
    int *active = (int *)malloc(sizeof(int) * (size_t)k);
    int q, it, v;
    for (v = 0; v < m; v++)
        for (q = 0; q < k; q++) x[(size_t)v * k + q] = 0.0;
    for (q = 0; q < k; q++) {
        x[(size_t)seeds[q] * k + q] = 1.0;
        active[q] = 1;
        iters[q] = 0;
    }
    for (it = 0; it < max_iter; it++) {
        int any = 0;
        for (q = 0; q < k; q++) { dang[q] = 0.0; err[q] = 0.0; any |= active[q]; }
        if (!any) break;
        for (v = 0; v < m; v++) {
            for (q = 0; q < k; q++) {
                double xv = x[(size_t)v * k + q];
                if (outdeg[v] == 0) { dang[q] += xv; c[(size_t)v * k + q] = 0.0; }
                else c[(size_t)v * k + q] = xv / (double)outdeg[v];
            }
        }
#pragma omp parallel for schedule(dynamic, 64)
        for (v = 0; v < m; v++) {
            int e, qq;
            for (qq = 0; qq < k; qq++) xn[(size_t)v * k + qq] = 0.0;
            for (e = rowptr[v]; e < rowptr[v + 1]; e++) {
                const double *cu = c + (size_t)col[e] * k;
                for (qq = 0; qq < k; qq++) xn[(size_t)v * k + qq] += cu[qq];
            }
            for (qq = 0; qq < k; qq++) xn[(size_t)v * k + qq] *= d;
        }
        for (q = 0; q < k; q++) xn[(size_t)seeds[q] * k + q] += (1.0 - d) + d * dang[q];
        for (v = 0; v < m; v++)
            for (q = 0; q < k; q++)
                if (active[q]) err[q] += fabs(xn[(size_t)v * k + q] - x[(size_t)v * k + q]);
        for (v = 0; v < m; v++)
            for (q = 0; q < k; q++)
                if (active[q]) x[(size_t)v * k + q] = xn[(size_t)v * k + q];
        for (q = 0; q < k; q++) {
            if (!active[q]) continue;
            iters[q] = it + 1;
            if (err[q] < tol) active[q] = 0;
        }
    }
    free(c); free(xn); free(dang); free(err); free(active);
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic graph generators (the reference has none; its inputs    */
/* are external files).  A counter-based hash makes every draw a pure       */
/* function of (seed, index), so the GPU generators in the product library  */
/* produce bit-identical graphs; the tests compare the two.                 */
/* Mixer: the SplitMix64 finaliser (Steele, Lea, Flood 2014).               */
/* ------------------------------------------------------------------------ */
static inline uint64_t orc_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
static inline uint64_t orc_hash3(uint64_t seed, uint64_t a, uint64_t b)
{
    return orc_mix64(seed ^ orc_mix64(a * 0x9E3779B97F4A7C15ULL + b));
}

/* Bijective scramble of [0, 2^scale): two multiply / xorshift rounds. */
static inline uint32_t orc_scramble(uint32_t v, int scale, uint64_t seed)
{
    const uint64_t mask = (scale >= 32) ? 0xffffffffULL : ((1ULL << scale) - 1ULL);
    const uint64_t k1 = (orc_mix64(seed ^ 0x1234567ULL) | 1ULL) & mask;
    const uint64_t k2 = (orc_mix64(seed ^ 0x89abcdefULL) | 1ULL) & mask;
    const uint64_t k3 = orc_mix64(seed ^ 0x5555ULL) & mask;
    const int sh = scale / 2 + 1;
    uint64_t x = v;
    x = (x * k1) & mask;
    x ^= x >> sh;
    x = (x * k2) & mask;
    x ^= x >> sh;
    x = (x + k3) & mask;
    return (uint32_t)x;
}

/* Probability thresholds of one RMAT level as 32-bit integers. */
void orc_rmat_thresholds(double a, double b, double c, uint32_t th[3])
{
    double t0 = a, t1 = a + b, t2 = a + b + c;
    th[0] = (uint32_t)(t0 * 4294967296.0);
    th[1] = (uint32_t)(t1 * 4294967296.0);
    th[2] = (uint32_t)(t2 * 4294967296.0);
}

/* Edge e of an RMAT graph: per level one 32-bit draw picks a quadrant
 * (a: src0/dst0, b: src0/dst1, c: src1/dst0, d: src1/dst1), MSB first. */
static inline void orc_rmat_edge(uint64_t e, int scale, const uint32_t th[3],
                                 uint64_t seed, int scramble, uint32_t *src,
                                 uint32_t *dst)
{
    uint32_t s = 0, t = 0;
    uint64_t h = 0;
    int l;
    for (l = 0; l < scale; l++) {
        if ((l & 1) == 0) h = orc_hash3(seed, e, (uint64_t)(l >> 1));
        uint32_t r = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
        uint32_t sb = 0, tb = 0;
        if (r < th[0]) { sb = 0; tb = 0; }
        else if (r < th[1]) { sb = 0; tb = 1; }
        else if (r < th[2]) { sb = 1; tb = 0; }
        else { sb = 1; tb = 1; }
        s = (s << 1) | sb;
        t = (t << 1) | tb;
    }
    if (scramble) {
        s = orc_scramble(s, scale, seed);
        t = orc_scramble(t, scale, seed);
    }
    *src = s;
    *dst = t;
}

void orc_rmat_edges(int scale, long long nedges, double a, double b, double c,
                    unsigned long long seed, int scramble, int *src, int *dst)
{
    uint32_t th[3];
    long long e;
    orc_rmat_thresholds(a, b, c, th);
#pragma omp parallel for schedule(static)
    for (e = 0; e < nedges; e++) {
        uint32_t s, t;
        orc_rmat_edge((uint64_t)e, scale, th, seed, scramble, &s, &t);
        src[e] = (int)s;
        dst[e] = (int)t;
    }
}

static int orc_cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* Build the pull (in-)CSR of an edge list: row = dst, columns = distinct
 * sources in ascending order, self-loops dropped, duplicates dropped.
 * Also the out-degree of every vertex in the deduplicated graph.
 * Two passes: count, scatter; then per-row sort + unique + compaction.
 * rowptr has m+1 entries; col must hold nedges entries (upper bound);
 * returns the final nnz. */
long long orc_build_in_csr(int m, long long nedges, const int *src,
                           const int *dst, int *rowptr, int *col, int *outdeg)
{
    long long *cnt = (long long *)calloc((size_t)m + 1, sizeof(long long));
    long long *cur = (long long *)malloc(sizeof(long long) * ((size_t)m + 1));
    int *uniq = (int *)malloc(sizeof(int) * ((size_t)m + 1));
    long long e, nnz = 0;
    int v;
    for (e = 0; e < nedges; e++)
        if (src[e] != dst[e]) cnt[dst[e] + 1]++;
    for (v = 0; v < m; v++) cnt[v + 1] += cnt[v];
    memcpy(cur, cnt, sizeof(long long) * ((size_t)m + 1));
    for (e = 0; e < nedges; e++)
        if (src[e] != dst[e]) col[cur[dst[e]]++] = src[e];
#pragma omp parallel for schedule(dynamic, 256)
    for (v = 0; v < m; v++) {
        long long b = cnt[v], n = cnt[v + 1] - cnt[v], i, w = 0;
        if (n > 1) qsort(col + b, (size_t)n, sizeof(int), orc_cmp_int);
        for (i = 0; i < n; i++)
            if (i == 0 || col[b + i] != col[b + i - 1]) col[b + w++] = col[b + i];
        uniq[v] = (int)w;
    }
    rowptr[0] = 0;
    for (v = 0; v < m; v++) {
        long long b = cnt[v], i;
        for (i = 0; i < uniq[v]; i++) col[nnz + i] = col[b + i];
        nnz += uniq[v];
        rowptr[v + 1] = (int)nnz;
    }
    memset(outdeg, 0, sizeof(int) * (size_t)m);
    for (e = 0; e < nnz; e++) outdeg[col[e]]++;
    free(cnt); free(cur); free(uniq);
    return nnz;
}

/* 27-point 3-D Laplacian on an n^3 grid, natural ordering
 * (row = (z*n + y)*n + x), columns ascending, 26 on the diagonal and -1
 * off it.  Ap has n^3+1 entries; Aj/Ax need (3n-2)^3 entries. */
long long orc_stencil27(int n, int *Ap, int *Aj, float *Ax)
{
    long long nnz = 0;
    int x, y, z, dz, dy, dx;
    long long row = 0;
    for (z = 0; z < n; z++)
        for (y = 0; y < n; y++)
            for (x = 0; x < n; x++, row++) {
                Ap[row] = (int)nnz;
                for (dz = -1; dz <= 1; dz++)
                    for (dy = -1; dy <= 1; dy++)
                        for (dx = -1; dx <= 1; dx++) {
                            int zz = z + dz, yy = y + dy, xx = x + dx;
                            if (zz < 0 || zz >= n || yy < 0 || yy >= n || xx < 0 || xx >= n) continue;
                            Aj[nnz] = (zz * n + yy) * n + xx;
                            Ax[nnz] = (dz == 0 && dy == 0 && dx == 0) ? 26.0f : -1.0f;
                            nnz++;
                        }
            }
    Ap[row] = (int)nnz;
    return nnz;
}

/* Seeded uniform [0,1) floats with 24 random bits (exact in FP32). */
void orc_uniform_f32(long long n, unsigned long long seed, float *out)
{
    long long i;
#pragma omp parallel for schedule(static)
    for (i = 0; i < n; i++)
        out[i] = (float)(orc_hash3(seed, (uint64_t)i, 0x7u) >> 40) * (1.0f / 16777216.0f);
}

/* Seeded uniform integers in [0, hi). */
void orc_uniform_int(long long n, unsigned long long seed, int hi, int *out)
{
    long long i;
    for (i = 0; i < n; i++)
        out[i] = (int)(orc_hash3(seed, (uint64_t)i, 0x9u) % (uint64_t)hi);
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Uneven multi-graph batch (a batch of independent graphs solved together; */
/* the reference has no counterpart -- each of its runs reads one file).    */
/*                                                                          */
/* Graph g of a batch with seed S:                                          */
/*   size   m_g = floor(exp(ln m_min + u (ln m_max - ln m_min))), clamped,  */
/*          u = top 53 bits of hash3(S, g, 0x6d67) / 2^53 (log-uniform)     */
/*   type   g odd: Chung-Lu power law, g even: Erdos-Renyi                  */
/*   edges  m_g * deg raw draws e = 0.. with h = hash3(G_g, e, 0),          */
/*          G_g = hash3(S, g, 0x9e37):                                      */
/*     Erdos-Renyi: src = (h >> 32) * m_g >> 32, dst = (h & 0xffffffff) *   */
/*                  m_g >> 32 (both uniform in [0, m_g))                    */
/*     Chung-Lu:    src = first i with P[i] > x * P[m_g - 1], x = top 53    */
/*                  bits of h / 2^53; dst the same with hash3(G_g, e, 1);   */
/*                  P[i] = sum_{j <= i} (j + 1)^(-1 / (gamma - 1)), summed  */
/*                  in double in index order (weights of a power-law degree */
/*                  sequence with exponent gamma, Chung & Lu 2002)          */
/*   then self-loops and duplicate edges are dropped (orc_build_in_csr).    */
/* The batch is one block-diagonal graph: graph g owns vertices             */
/* [voff[g], voff[g+1]), in the order g = 0, 1, ...                         */
/* ------------------------------------------------------------------------ */
int orc_multigraph_size(int g, int m_min, int m_max, unsigned long long seed)
{
    const uint64_t h = orc_hash3(seed, (uint64_t)g, 0x6d67u);
    const double u = (double)(h >> 11) * 0x1.0p-53;
    const double lo = log((double)m_min), hi = log((double)m_max);
    const double t = u * (hi - lo);
    int m = (int)floor(exp(lo + t));
    if (m < m_min) m = m_min;
    if (m > m_max) m = m_max;
    return m;
}

void orc_chung_lu_prefix(int n, double gamma, double *P)
{
    const double alpha = -1.0 / (gamma - 1.0);
    double acc = 0.0;
    int i;
    for (i = 0; i < n; i++) {
        acc += pow((double)(i + 1), alpha);
        P[i] = acc;
    }
}

static inline int orc_cl_draw(uint64_t h, const double *P, int m)
{
    const double x = (double)(h >> 11) * 0x1.0p-53;
    const double y = x * P[m - 1];
    int lo = 0, hi = m;  /* first i in [0, m) with P[i] > y */
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if (P[mid] > y) hi = mid;
        else lo = mid + 1;
    }
    return lo < m ? lo : m - 1;
}

/* Raw edge draws of graph g (local vertex ids), m_g * deg of them. */
void orc_multigraph_edges(int g, int m_g, int deg, unsigned long long seed,
                          const double *P, int *src, int *dst)
{
    const uint64_t gs = orc_hash3(seed, (uint64_t)g, 0x9e37u);
    const long long ne = (long long)m_g * deg;
    long long e;
#pragma omp parallel for schedule(static)
    for (e = 0; e < ne; e++) {
        const uint64_t h = orc_hash3(gs, (uint64_t)e, 0);
        if (g & 1) {
            src[e] = orc_cl_draw(h, P, m_g);
            dst[e] = orc_cl_draw(orc_hash3(gs, (uint64_t)e, 1), P, m_g);
        } else {
            src[e] = (int)(((h >> 32) * (uint64_t)m_g) >> 32);
            dst[e] = (int)(((h & 0xffffffffULL) * (uint64_t)m_g) >> 32);
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Symmetric Gauss-Seidel smoother, multicolour order (src/symgs/verifier.cc */
/* :56-79 gs_serial and SymGSVerifier; src/symgs/omp_base.cc:8-45): colours  */
/* 0..n-1 forward, then n-1..0 backward, rows of a colour in `indices`       */
/* order; each row sums x[j]*Ax[jj] over its off-diagonal entries in CSR     */
/* order (one rounded multiply and one rounded add per entry), takes the     */
/* last diagonal entry as diag, and if diag != 0 sets                        */
/* x[row] = (b[row] - rsum) / diag.                                          */
/* ------------------------------------------------------------------------ */
static void orc_gs_rows(const int *Ap, const int *Aj, const float *Ax, const int *indices,
                        int begin, int end, float *x, const float *b)
{
    int i;
    for (i = begin; i < end; i++) {
        const int r = indices[i];
        float rsum = 0.0f, diag = 0.0f;
        int jj;
        for (jj = Ap[r]; jj < Ap[r + 1]; jj++) {
            const int j = Aj[jj];
            if (j == r) diag = Ax[jj];
            else {
                const float p = x[j] * Ax[jj];
                rsum = rsum + p;
            }
        }
        if (diag != 0.0f) x[r] = (b[r] - rsum) / diag;
    }
}

void orc_symgs_f32(int m, const int *Ap, const int *Aj, const float *Ax, const int *indices,
                   const int *color_offsets, int ncolors, float *x, const float *b)
{
    int c;
    (void)m;
    for (c = 0; c < ncolors; c++)
        orc_gs_rows(Ap, Aj, Ax, indices, color_offsets[c], color_offsets[c + 1], x, b);
    for (c = ncolors; c > 0; c--)
        orc_gs_rows(Ap, Aj, Ax, indices, color_offsets[c - 1], color_offsets[c], x, b);
}

/* First-fit greedy colouring in vertex order over the off-diagonal entries
 * (a valid colouring of a structurally symmetric matrix's graph; the
 * reference takes its colouring from its vertex-colouring kernel, src/vc).
 * Returns the number of colours. */
int orc_greedy_coloring(int m, const int *Ap, const int *Aj, int *colors)
{
    int v, nc = 0;
    int *mark = (int *)malloc(sizeof(int) * ((size_t)m + 1));
    for (v = 0; v < m; v++) colors[v] = -1;
    for (v = 0; v <= m; v++) mark[v] = -1;
    for (v = 0; v < m; v++) {
        int jj, c = 0;
        for (jj = Ap[v]; jj < Ap[v + 1]; jj++) {
            const int u = Aj[jj];
            if (u != v && colors[u] >= 0) mark[colors[u]] = v;
        }
        while (mark[c] == v) c++;
        colors[v] = c;
        if (c + 1 > nc) nc = c + 1;
    }
    free(mark);
    return nc;
}
