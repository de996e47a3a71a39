/*
 * gpr.h -- C ABI of the B200 pull-PageRank / CSR-SpMV library (libgpr.so).
 *
 * Plain pointers and sizes only; every entry point returns a gpr_status and
 * never exits the process.  gpr_last_error() gives a message for the last
 * failure on the calling thread.
 *
 * The reference (Gardenia, src/pr and src/spmv) has no C ABI: its boundary is
 * the link-time C++ symbol PRSolver / SpmvSolver chosen by the Makefile
 * (src/pr/Makefile:17-47, src/spmv/Makefile:16-50).  The C++ drop-ins with
 * those exact signatures are declared in gardenia_pr.h / gardenia_spmv.h and
 * are thin wrappers over the functions below.  Each function here cites the
 * reference interface it replaces.
 *
 * Pointers named h_* are host memory; d_* are device memory on the current
 * CUDA device; "any" pointers may be either (the library checks with
 * cudaPointerGetAttributes and copies when needed).  Streams are passed as
 * void* (a cudaStream_t; NULL = the legacy default stream).
 *
 * A handle (graph, matrix, multi-graph batch, SymGS) is used by one host
 * thread at a time: it caches per-handle tables and CUDA graphs.  Different
 * handles may be used from different threads.
 */
#ifndef GPR_H_
#define GPR_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GPR_OK = 0,
  GPR_EINVAL = 1,     /* bad argument or malformed CSR */
  GPR_ENOMEM = 2,     /* device or host allocation failed */
  GPR_ECUDA = 3,      /* a CUDA runtime call failed */
  GPR_ETIMEOUT = 4,   /* a bounded device-side wait ran out */
  GPR_ENODEV = 5,     /* no usable CUDA device */
  GPR_EUNSUPPORTED = 6
} gpr_status;

/* Precision of the stored / gathered contributions. */
typedef enum {
  GPR_PREC_FP32 = 0,  /* plain form: FP32 everywhere, FP64 residual */
  GPR_PREC_BF16 = 1,  /* BF16 contributions, FP32 accumulation, FP32 refinement */
  GPR_PREC_FP16 = 2   /* reserved: every solver returns GPR_EUNSUPPORTED (the gather is
                         bound by its request count, not its bytes, so a 2-byte form
                         gains nothing; BF16 covers the mixed form) */
} gpr_precision;

/* How the iteration loop is driven. */
typedef enum {
  GPR_LOOP_AUTO = 0,        /* pick from the graph size */
  GPR_LOOP_PERSISTENT = 1,  /* one cooperative launch, bounded grid barrier per sweep */
  GPR_LOOP_GRAPH = 2        /* one launch per sweep, captured into a CUDA graph */
} gpr_loop;

typedef struct {
  float damping;        /* kDamp, include/common.h:18 (0.85f) */
  double tol;           /* EPSILON, src/pr/pr.h:4 (1e-3); stop when the sweep's L1 change < tol */
  int max_iter;         /* MAX_ITER, src/pr/pr.h:5 (30) */
  int precision;        /* gpr_precision */
  int loop;             /* gpr_loop */
  double timeout_s;     /* bound on every device-side wait (grid barrier); default 5 s */
  int refine_max;       /* mixed precision: max FP32 refinement sweeps (default 64) */
  int variant;          /* sweep-kernel variant, 0..7 (0 = default; the autotuner's choices) */
  int reserved[1];      /* reserved[0] > 0: the grid barrier also waits for that many CTAs
                           that do not exist, so its bounded wait runs out (tests of the
                           GPR_ETIMEOUT path); keep 0 otherwise */
  int form;             /* gpr_form: which sweep sums the rows (FP32 solves of gpr_pagerank) */
  int ppr_repack;       /* gpr_ppr, FP32 sweeps: once at most half of the vectors are still
                           updating, continue with those packed into the next narrower
                           layout (1, the default) or keep the layout (0) */
  int pad[4];           /* keep 0 */
} gpr_pr_opts;

/* Sweep forms of gpr_pagerank (FP32).  Both compute the reference's
 * recurrence (src/pr/omp_base.cc:23-44) and meet its parity bar (1e-6 per
 * vertex, sweep count within one); they differ in the order of each row's sum.
 *   EXACT    rows of <= 64 in-edges add their contributions one by one in CSR
 *            order with rounded float adds, as the reference does: such rows
 *            are bit-identical to the reference's.
 *   BLOCKED  rows (all but the hubs, gpr_layout_opts.blocked_long) are summed
 *            block by block from source-ordered edges (far fewer memory
 *            requests on large graphs), in 64-bit fixed point: the exact sum
 *            of the FP32 contributions rounded once to 2^-S (S >= 31, chosen
 *            per solve from the edge count and the largest score), then to
 *            FP32.  Deterministic.  Needs a graph created with
 *            GPR_LAYOUT_BLOCKED and the persistent loop.
 *   AUTO     BLOCKED when the graph has its layout, at least 50,331,648 edges
 *            (below that EXACT measured faster: RMAT scale 21 3.6 vs 3.9 ms,
 *            scale 22 7.6 vs 6.8 ms) and the persistent loop runs, else EXACT. */
typedef enum {
  GPR_FORM_AUTO = 0,
  GPR_FORM_EXACT = 1,
  GPR_FORM_BLOCKED = 2
} gpr_form;

typedef struct {
  int iterations;       /* sweeps executed (the reference prints the same number, gather.cu:83);
                           m = 0: the empty sweeps the reference's loop counts, 1 when
                           tol > 0 and max_iter when tol = 0 (omp_base.cc:23-43) */
  int refine_iterations;/* FP32 sweeps spent in the refinement tail (mixed precision) */
  double residual;      /* L1 change of the last sweep (FP64) */
  double solve_ms;      /* device time of the solve (CUDA events), excluding copies */
  double loop_ms;       /* device time of the sweep loop alone (persistent kernel or step launches) */
  int gpu_launches;     /* kernels launched by this solve */
  int reserved[5];
} gpr_pr_stats;

typedef struct gpr_graph gpr_graph;    /* device-resident pull graph (PR) */
typedef struct gpr_matrix gpr_matrix;  /* device-resident CSR matrix (SpMV) */

/* ---- library ---------------------------------------------------------- */
const char *gpr_last_error(void);
const char *gpr_version(void);
int gpr_pr_opts_default(gpr_pr_opts *opts);

/* ---- PageRank graph ------------------------------------------------------
 * Pull graph from the in-CSR (row v lists the sources u of edges u->v) and
 * the out-degree of every vertex: the arguments the reference's pull solver
 * reads (src/pr/omp_base.cc:9, row_offsets / column_indices / degree).
 * The library keeps its own relabelled device copy; the caller's arrays are
 * not retained. */
int gpr_graph_create(int m, long long nnz, const int *any_rowptr,
                     const int *any_col, const int *any_outdeg,
                     gpr_graph **out);
/* Layout knobs (the autotuner's search space); zero fields take defaults. */
enum {
  GPR_LAYOUT_BATCHED = 1, /* also keep a relabelled CSR: needed by gpr_ppr */
  GPR_LAYOUT_PUSH = 2,    /* also keep it for gpr_pagerank_push */
  GPR_LAYOUT_BLOCKED = 4  /* also build the blocked form's layout (one radix sort of the
                             edges at creation; ~4 bytes per edge more on the device) */
};
typedef struct {
  int sell_max;   /* max edges per lane in a SELL slice: rows of in-degree <= sell_max get
                     one lane, wider rows 2..32 lanes (default 64) */
  int chunk;      /* edges per long-row chunk, multiple of 128 (default 4096) */
  int chunk_min;  /* rows with more in-edges than this are cut into chunks (default 4096) */
  int hot_entries;/* contributions of the highest in-degree vertices kept in shared memory
                     by the persistent kernel, multiple of 4, <= 56832 (default 32768) */
  int flags;      /* GPR_LAYOUT_* bits */
  int block_rows; /* blocked form: rows per block, <= 12288 (default: about rows / (2 SMs),
                     256 .. 12288) */
  int tile_words; /* blocked form: most entry words per tile, >= 512 (default 1048576;
                     the tiles that would end a sweep late are halved further) */
  int blocked_long; /* blocked form: rows with more in-edges than this are summed in chunks,
                       the others in blocks; values below chunk_min act as chunk_min.
                       0 (default): a row is chunked when it holds more than 1/8 of the
                       in-edges of the block_rows rows that start at it (a hub whose
                       additions would queue on one shared-memory word) */
} gpr_layout_opts;
int gpr_graph_create_ex(int m, long long nnz, const int *any_rowptr,
                        const int *any_col, const int *any_outdeg,
                        const gpr_layout_opts *lopts, gpr_graph **out);
int gpr_graph_destroy(gpr_graph *g);
int gpr_graph_info(const gpr_graph *g, int *m, long long *nnz,
                   long long *device_bytes);
/* Bin sizes of the relabelled layout (rows > sell_max in-edges, rows with
 * any in-edge, long-row chunks, SELL slices, stored edge slots). */
int gpr_graph_layout(const gpr_graph *g, int *n_long, int *n_nz, int *n_chunks,
                     int *n_slices, long long *long_elems, long long *sell_elems);
/* Run later solves on `stream` (a cudaStream_t owned by the caller) instead
 * of the graph's own stream. */
int gpr_graph_set_stream(gpr_graph *g, void *stream);
/* Per-sweep L1 residuals of the last solve (the numbers the reference prints
 * each iteration, src/pr/omp_base.cc:42).  Copies min(n, sweeps) values. */
int gpr_graph_residuals(const gpr_graph *g, double *h_out, int n);

/* Solve.  scores (host or device, m floats) holds the initial scores on
 * entry and the result on return, like the reference's scores argument
 * (src/pr/omp_base.cc:9, src/pr/main.cc:26-29).  Synchronous. */
int gpr_pagerank(gpr_graph *g, float *any_scores, const gpr_pr_opts *opts,
                 gpr_pr_stats *stats);

/* FP64 L1 residual || base + d*M*s - s ||_1 of a score vector on the GPU;
 * ||s - s*||_1 <= residual / (1 - d) bounds the distance to the fixed point. */
int gpr_pr_residual_f64(gpr_graph *g, const float *any_scores, float damping,
                        double *residual);

/* ---- reference-shaped one-shot calls (host arrays in, results in place) -- */
/* PRSolver, src/pr/pr.h:23.  The out-CSR is accepted and ignored, as in the
 * pull variants (src/pr/omp_base.cc:9, src/pr/gather.cu:41). */
int gpr_pr_solver(int m, int nnz, const int *in_row_offsets,
                  const int *in_column_indices, const int *out_row_offsets,
                  const int *out_column_indices, const int *degree,
                  float *scores, const gpr_pr_opts *opts, gpr_pr_stats *stats);
/* PageRank(m, nnz, row_offsets, column_indices, degree, scores): the pull
 * entry point named for this path (in-CSR + out-degree), same contract. */
int gpr_page_rank(int m, int nnz, const int *row_offsets,
                  const int *column_indices, const int *degree, float *scores,
                  const gpr_pr_opts *opts, gpr_pr_stats *stats);

/* ---- Batched personalized PageRank (no counterpart in the reference) ------
 * k <= 128 seed vectors in one persistent launch: for vector q with seed
 * h_seeds[q], x_q = d * M x_q + ((1-d) + d * dangling_q) e_{seed_q}, from
 * x_q = e_{seed_q}; vector q stops after the first sweep whose FP64 L1 change
 * is below opts->tol.  opts->precision: GPR_PREC_FP32 or GPR_PREC_BF16
 * (contributions stored in BF16 until the change is below max(tol, 1e-3),
 * FP32 accumulation, then FP32 sweeps until it is below tol (1-d)/d, so that
 * the BF16 start costs no accuracy).  any_x receives x as an
 * m x k row-major array (vertex-major, host or device); h_iters (k ints, may
 * be NULL) the sweeps of each vector.  opts->loop: GPR_LOOP_AUTO /
 * GPR_LOOP_PERSISTENT run all sweeps in one cooperative launch (grid barrier
 * bounded by opts->timeout_s); GPR_LOOP_GRAPH runs one launch per sweep in a
 * CUDA-graph while loop (also used when the grid cannot be co-resident);
 * both give bit-identical results.  The graph must be created with
 * GPR_LAYOUT_BATCHED. */
int gpr_ppr(gpr_graph *g, int k, const int *h_seeds, float *any_x,
            const gpr_pr_opts *opts, int *h_iters, gpr_pr_stats *stats);

/* ---- push-style PageRank --------------------------------------------------
 * The reference's push variants (src/pr/scatter.cu:16-41, lb.cu:20-82)
 * scatter each source's contribution to its out-neighbours with atomic adds.
 * Same recurrence and stop rule as gpr_pagerank (so the two directions solve
 * the same problem); edges sorted by source, hot destinations accumulated in
 * shared memory, one persistent launch.  Atomic adds make the last bits of
 * the result vary from run to run.  The graph must be created with
 * GPR_LAYOUT_PUSH (or GPR_LAYOUT_BATCHED); FP32 only. */
int gpr_pagerank_push(gpr_graph *g, float *any_scores, const gpr_pr_opts *opts,
                      gpr_pr_stats *stats);

/* ---- uneven multi-graph batch ------------------------------------------------
 * No counterpart in the reference (each reference run solves one graph read
 * from one file, src/pr/main.cc:14-34).  A batch of independent graphs stored
 * as one block-diagonal pull graph: graph g owns vertices
 * [h_voff[g], h_voff[g+1]) (h_voff: n_graphs + 1 host ints, h_voff[0] = 0),
 * and every in-edge of its rows comes from that range (global vertex ids;
 * GPR_EINVAL otherwise).  rowptr / col / outdeg are the usual in-CSR and
 * out-degrees over all h_voff[n_graphs] vertices.  h_lopts (n_graphs entries,
 * or NULL for the defaults) gives each graph its own bins: sell_max, chunk,
 * chunk_min as in gpr_graph_create_ex (hot_entries is ignored).  When any
 * graph's flags hold GPR_LAYOUT_BLOCKED the batch also builds the blocked
 * form's layout: every graph's rows with in-edges in blocks of block_rows
 * rows that never span two graphs, tiles of up to tile_words words (the
 * first such graph's values; 0: defaults as in gpr_graph_create_ex).
 * opts->form then works as for gpr_pagerank: BLOCKED sums every graph's rows
 * in 64-bit fixed point (one exponent S for the batch, from its edge count
 * and the largest m_g x |initial score|), FP32 and the persistent loop only;
 * AUTO picks it from 50,331,648 edges in the batch, else the units form.
 *
 * gpr_multigraph_pagerank solves every graph as gpr_pagerank would solve it
 * alone -- base (1 - kDamp) / m_g, its own L1 residual, stop after its first
 * sweep with residual < tol or after max_iter sweeps -- all graphs in one
 * persistent launch (opts->loop GPR_LOOP_GRAPH, or a device that cannot
 * co-schedule it: one launch per sweep in a CUDA-graph while loop, same
 * results).  any_scores: all vertices, initialised by the caller
 * (the reference uses 1/m_g, src/pr/main.cc:27-28), updated in place.
 * h_iters / h_residuals (n_graphs entries each, may be NULL) receive each
 * graph's sweeps and last residual (a graph with no vertices: the empty
 * sweeps the reference's loop counts, residual 0).  precision GPR_PREC_FP32, or
 * GPR_PREC_BF16 (BF16 contributions to max(tol, 1e-3), then FP32 sweeps to
 * tol); stats->iterations is the launch's sweep count (the largest graph
 * count per phase). */
typedef struct gpr_multigraph gpr_multigraph;
int gpr_multigraph_create(int n_graphs, const int *h_voff, long long nnz,
                          const int *any_rowptr, const int *any_col,
                          const int *any_outdeg, const gpr_layout_opts *h_lopts,
                          gpr_multigraph **out);
int gpr_multigraph_destroy(gpr_multigraph *mg);
int gpr_multigraph_info(const gpr_multigraph *mg, int *n_graphs, int *m,
                        long long *nnz, int *n_units, long long *edge_slots);
int gpr_multigraph_set_stream(gpr_multigraph *mg, void *stream);
int gpr_multigraph_pagerank(gpr_multigraph *mg, float *any_scores,
                            const gpr_pr_opts *opts, int *h_iters,
                            double *h_residuals, gpr_pr_stats *stats);

/* ---- autotuner -------------------------------------------------------------
 * No counterpart in the reference (its launch shape is fixed at compile time,
 * include/common.h:30, src/pr/Makefile:17-47).  Picks the form (exact order,
 * or GPR_LAYOUT_BLOCKED with its block_rows / tile_words / blocked_long), the
 * layout bins (sell_max = lanes-per-row bound of the SELL width classes,
 * chunk_min / chunk = chunked-row threshold and chunk size), the
 * shared-memory hot prefix and the sweep-kernel variant for a graph's
 * in-degree distribution by timing candidates on the graph (coordinate
 * descent from the defaults, each candidate the best of 3 solves of exactly
 * `sweeps` sweeps after a warm-up solve, kept only when 3% faster than the
 * current pick), and caches the pick per distribution signature in the text
 * file cache_path (NULL: no cache).  A cached signature returns at once
 * (from_cache = 1). */
typedef struct {
  gpr_layout_opts layout;       /* pass to gpr_graph_create_ex */
  int variant;                  /* pass as gpr_pr_opts.variant */
  int from_cache;               /* 1: read from the cache, nothing timed */
  int candidates;               /* configurations timed */
  double ms_per_sweep;          /* the pick, measured (or as cached) */
  double default_ms_per_sweep;  /* the defaults, measured (0 when cached) */
  char signature[48];           /* distribution signature (cache key) */
} gpr_tune_result;
int gpr_tune_graph(int m, long long nnz, const int *any_rowptr,
                   const int *any_col, const int *any_outdeg,
                   const char *cache_path, int sweeps, gpr_tune_result *out);
/* Batch: first the blocked form for the whole batch (carried by the group
 * with the largest edge share, with its block_rows / tile_words); else graphs
 * grouped by signature, one group's bins tuned at a time on the whole batch.
 * h_lopts_out (n_graphs entries) receives each graph's options for
 * gpr_multigraph_create; out (may be NULL) describes the largest group. */
int gpr_tune_multigraph(int n_graphs, const int *h_voff, long long nnz,
                        const int *any_rowptr, const int *any_col,
                        const int *any_outdeg, const char *cache_path,
                        int sweeps, gpr_layout_opts *h_lopts_out,
                        gpr_tune_result *out);
/* The signature of a host CSR (batch != 0: the per-graph key of the batch
 * tuner), and a cache lookup; both host-only. */
int gpr_tune_signature(int m, long long nnz, const int *h_rowptr, int batch,
                       char *buf, int len);
int gpr_tune_cache_lookup(const char *cache_path, const char *signature,
                          gpr_tune_result *out);

/* ---- PageRank without any allocation ----------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory (their allocator owns the device heap, or the call
 * may not take the synchronisation cudaMalloc / cudaFree can cause): solves
 * directly on the caller's device CSR (d_rowptr / d_col = in-CSR, d_outdeg =
 * out-degrees, d_scores in/out, all device memory) on `stream`, with its
 * scratch in a fixed device array inside the library (about 8 MiB, held by
 * every GPU that loads the library until exit).  Limits: m <= 1,048,576
 * vertices (gpr_pagerank_noalloc_max_vertices) and max_iter <= 1000, else
 * GPR_EINVAL.  The CSR is validated on the device on every call with m > 0
 * (row offsets monotone from 0 to nnz, columns in range, out-degrees >= 0),
 * also when max_iter is 0; m == 0 with nnz != 0 is rejected.  The first call
 * on a device looks up the array's device address and should come before any
 * stream capture.  Calls share the array, so calls that overlap on the GPU
 * race; run them one at a time.  Synchronous: the call waits for `stream`
 * (and only that stream) before it returns.  Scores follow the reference's
 * float arithmetic row by row; opts->loop / variant / precision are ignored. */
int gpr_pagerank_noalloc(int m, int nnz, const int *d_rowptr, const int *d_col,
                         const int *d_outdeg, float *d_scores,
                         const gpr_pr_opts *opts, gpr_pr_stats *stats,
                         void *stream);
long long gpr_pagerank_noalloc_max_vertices(void);

/* ---- SpMV ------------------------------------------------------------------
 * y <- y + A*x over a CSR matrix (src/spmv/spmv.h:29, omp_base.cc:8-32). */
int gpr_matrix_create(int m, long long nnz, const int *any_Ap,
                      const int *any_Aj, const float *any_Ax, gpr_matrix **out);
int gpr_matrix_destroy(gpr_matrix *A);
int gpr_matrix_layout(const gpr_matrix *A, int *n_long, int *n_chunks,
                      int *n_slices, long long *sell_elems);
/* x, y on the device; asynchronous on `stream`. */
int gpr_spmv(gpr_matrix *A, const float *d_x, float *d_y, void *stream);
/* SpmvSolver, src/spmv/spmv.h:29: host arrays, y updated in place. */
int gpr_spmv_solver(int m, int nnz, const int *Ap, const int *Aj,
                    const float *Ax, const float *x, float *y);

/* ---- symmetric Gauss-Seidel (multicolour) ----------------------------------
 * src/symgs: one sweep = the colours of a vertex colouring forward, then
 * backward; rows of one colour are updated together; each row sums
 * x[j]*Ax[jj] over its off-diagonal entries in CSR order and, when its last
 * diagonal entry d != 0, sets x = (b - sum) / d (src/symgs/omp_base.cc:8-45).
 * indices: the rows colour by colour; color_offsets: n_colors + 1 boundaries.
 * Results are bit-identical to the reference's.  The colouring must be valid
 * (no entry joins two rows of one colour; GPR_EINVAL otherwise).  Matrix
 * arrays may be host or device memory; the layout is built on the host. */
typedef struct gpr_symgs gpr_symgs;
int gpr_symgs_create(int m, long long nnz, const int *any_Ap, const int *any_Aj,
                     const float *any_Ax, const int *any_indices,
                     const int *any_color_offsets, int n_colors, gpr_symgs **out);
int gpr_symgs_destroy(gpr_symgs *h);
/* `sweeps` sweeps in one persistent launch; x (in/out) and b host or device;
 * loop_ms (may be NULL) receives the device time of the launch. */
int gpr_symgs_apply(gpr_symgs *h, float *any_x, const float *any_b, int sweeps,
                    double *loop_ms);
/* SymGSSolver, src/symgs/symgs.h:28: one sweep, x updated in place. */
int gpr_symgs_solver(int m, int nnz, const int *Ap, const int *Aj,
                     const int *indices, const float *Ax, float *x,
                     const float *b, const int *color_offsets, int n_colors);

/* ---- graph construction on the GPU (inputs for the solvers) ------------- */
/* Seeded RMAT pull graph (self-loops and duplicates removed, columns
 * ascending): fills device arrays allocated by the library; release with
 * gpr_free.  a,b,c are the quadrant probabilities (d = 1-a-b-c). */
int gpr_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                 unsigned long long seed, int scramble, int **d_rowptr,
                 int **d_col, int **d_outdeg, long long *nnz);
/* Seeded uneven batch of n_graphs graphs as one block-diagonal pull graph:
 * graph g owns vertices [h_voff[g], h_voff[g+1]) (h_voff: n_graphs + 1 ints,
 * filled by the call), with m_g log-uniform in [m_min, m_max]; odd g are
 * Chung-Lu power-law graphs (cl_deg edge draws per vertex, degree exponent
 * gamma), even g Erdos-Renyi graphs (er_deg draws per vertex); self-loops and
 * duplicate edges dropped, global vertex ids, columns ascending.  The draws
 * are a pure function of (seed, g, edge index), restated in the oracle. */
int gpr_gen_multigraph(int n_graphs, int m_min, int m_max, int er_deg,
                       int cl_deg, double gamma, unsigned long long seed,
                       int *h_voff, int **d_rowptr, int **d_col,
                       int **d_outdeg, long long *nnz);
/* 27-point Laplacian on an n^3 grid (26 / -1), natural ordering. */
int gpr_gen_stencil27(int n, int **d_Ap, int **d_Aj, float **d_Ax,
                      long long *nnz);
/* Seeded uniform [0,1) floats (24 random bits). */
int gpr_gen_uniform(long long n, unsigned long long seed, float *d_out);
int gpr_free(void *d_ptr);
/* The library keeps device blocks of 1 MiB and more after they are freed
 * (at most 24 GiB, reused by later requests that fit them within 1/8), so
 * one-shot calls do not map and unmap gigabytes each time.  Freeing a block
 * synchronises the device first, as cudaFree does.  gpr_release_cached returns
 * every cached block to the CUDA driver (released_bytes may be NULL);
 * gpr_cached_bytes reports how much is held. */
int gpr_release_cached(long long *released_bytes);
int gpr_cached_bytes(long long *bytes);
/* Device allocation / copy helpers for callers without a CUDA runtime of
 * their own (copies use cudaMemcpyDefault: any direction). */
int gpr_malloc(void **d_ptr, size_t bytes);
int gpr_memcpy(void *dst, const void *src, size_t bytes);
int gpr_synchronize(void);
/* Make `device` current for the calling thread's later gpr calls (handles
 * remember the device they were created on). */
int gpr_set_device(int device);

/* ---- graph_io (host) ------------------------------------------------------
 * read_graph of include/graph_io.h:280 for foreign callers: same parsers and
 * flags as the C++ read_graph in gardenia_graph_io.h; arrays are malloc'd and
 * released with gpr_read_graph_free.  Where the C++ read_graph prints a
 * message and exits (as the reference does), this returns GPR_EINVAL (a file
 * that cannot be opened, of no known format, or malformed: missing lines,
 * a negative vertex count, an index out of range) or GPR_ENOMEM, with the
 * reason in gpr_last_error() and nothing left allocated. */
int gpr_read_graph(const char *path, int symmetrize, int transpose, int sorted,
                   int remove_selfloops, int remove_redundents, int *m, int *nnz,
                   int **row_offsets, int **column_indices, int **degree,
                   float **weight);
void gpr_read_graph_free(void *p);

/* The file's edges in the order the reference pushes them into its
 * per-vertex lists (graph_io.h:133-261): entry k appends (col[k], wt[k]) to
 * the list of vertex row[k]; symmetrize / transpose as in read_graph.
 * Parsed by `threads` threads (<= 0: all cores, GPR_IO_THREADS overrides);
 * arrays malloc'd, released with gpr_read_graph_free.  Returns GPR_OK,
 * GPR_EINVAL when the file cannot be read or is malformed, or GPR_ENOMEM;
 * the reason is in gpr_last_error() and nothing is left allocated. */
int gpr_parse_edges(const char *path, int symmetrize, int transpose, int threads,
                    int *m, int *nnz_header, long long *n_push, int **row,
                    int **col, float **wt);
/* fill_data (graph_io.h:21-130) on the GPU over such a push list: lists in
 * push order (stable), optionally sorted by column, self-loops dropped, then
 * an entry equal to the previous kept one dropped.  Rows and columns match
 * the reference for every flag; with `sorted` the weights of duplicate
 * columns may come in another order (std::sort leaves it unspecified).
 * Outputs are device arrays allocated here (gpr_free); d_wt may be NULL. */
int gpr_csr_from_edges(int m, long long n, const int *any_row, const int *any_col,
                       const float *any_wt, int sorted, int remove_selfloops,
                       int remove_redundents, int **d_rowptr, int **d_col,
                       float **d_wt, long long *nnz);
/* read_graph with the parse above and the CSR built on the GPU (device
 * outputs; d_wt may be NULL). */
int gpr_read_graph_gpu(const char *path, int symmetrize, int transpose, int sorted,
                       int remove_selfloops, int remove_redundents, int *m,
                       long long *nnz, int **d_rowptr, int **d_col, int **d_degree,
                       float **d_wt);
/* The PR driver's two reads (src/pr/main.cc:23-24: out-CSR, then the
 * transposed in-CSR, both unsorted with self-loops and repeats removed) from
 * one parse: the in-CSR is built from the same pushes with row and column
 * swapped.  Identical to the reference's two read_graph calls. */
int gpr_read_graph_pr(const char *path, int symmetrize, int *m,
                      long long *nnz_out_csr, long long *nnz_in_csr,
                      int **d_out_rowptr, int **d_out_col, int **d_out_degree,
                      int **d_in_rowptr, int **d_in_col);

#ifdef __cplusplus
}
#endif
#endif /* GPR_H_ */
