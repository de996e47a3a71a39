// Internal helpers and device layouts shared by the libgpr translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <vector>

#include "gpr.h"

namespace gpr {

// Thread-local message of the last failure (gpr_last_error).
void set_error(const char *fmt, ...);

// Device allocation that records ENOMEM / ECUDA in the error slot.
int dmalloc(void **p, size_t bytes, const char *what);
template <typename T>
int dalloc(T **p, size_t count, const char *what) {
  return dmalloc(reinterpret_cast<void **>(p), (count ? count : 1) * sizeof(T), what);
}
void dfree(void *p);

// While an instance lives, dfree on this thread only records the pointers;
// the destructor frees them.  A free synchronises the device (cudaFree, or
// the block cache's wait before reuse), so code that overlaps a copy on one
// stream with work on another holds one until both streams are done.
class DeferFrees {
 public:
  DeferFrees();
  ~DeferFrees();
  DeferFrees(const DeferFrees &) = delete;
  DeferFrees &operator=(const DeferFrees &) = delete;

 private:
  std::vector<void *> list_;
  std::vector<void *> *prev_;
};

// True if `p` is device (or managed) memory of the current context.
bool is_device_ptr(const void *p);

// Copies `bytes` from a host-or-device pointer into a fresh device buffer,
// or returns the pointer itself (owned = false) when it is already on the
// device.
int to_device(const void *any, size_t bytes, void **dev, bool *owned,
              cudaStream_t st, const char *what);

// ---------------------------------------------------------------------------
// Pull-graph layout after relabelling vertices by descending in-degree.
//
//   new row i  <->  old vertex perm[i]
//   rows [0, n_long)      in-degree > chunk_min: CSR whose row starts are
//                         16-byte aligned, each row cut into chunks of
//                         `chunk` edges (one warp per chunk)
//   rows [n_long, n_nz)   1 <= in-degree <= chunk_min: SELL-32 slices in
//                         width classes.  A class gives every row w lanes
//                         (w = 32, 16, 8, 4, 2, 1, widest first), w being the
//                         smallest power of two with ceil(deg / w) <= lane_max;
//                         a slice holds 32/w consecutive rows, column-major:
//                         element (j, lane) = edge j*w + (lane % w) of row
//                         lane / w.  With w = 1 a lane sums its row in the
//                         original CSR order.
//   rows [n_nz, m)        in-degree 0
//
// Every padding entry of either edge array holds the sentinel index m, whose
// contribution slot is kept at 0.
// ---------------------------------------------------------------------------
constexpr int kMaxCls = 6;

struct PrClasses {
  int n_cls = 0;
  int lw[kMaxCls] = {0};          // log2(lanes per row) of each class
  int row[kMaxCls + 1] = {0};     // first row of each class; row[n_cls] = n_nz
  int slice[kMaxCls + 1] = {0};   // first slice of each class; slice[n_cls] = n_slices
};

struct PrLayout {
  int m = 0;
  long long nnz = 0;
  int n_long = 0, n_nz = 0;
  int lane_max = 0, chunk_min = 0, chunk = 0;
  int n_chunks = 0, n_slices = 0, n_zblk = 0;
  int max_row_chunks = 0;         // chunks of the longest row
  PrClasses cls;
  int *perm = nullptr;            // [m] new -> old
  int *outdeg = nullptr;          // [m] out-degree in new order
  long long *long_ptr = nullptr;  // [n_long+1] padded offsets into long_col
  int *long_col = nullptr;        // relabelled sources of the long rows
  int *row_cbeg = nullptr;        // [n_long+1] first chunk of each long row
  int *chunk_row = nullptr;       // [n_chunks] row of each chunk
  long long *slice_ptr = nullptr; // [n_slices+1] offsets into sell_col
  int *sell_col = nullptr;        // relabelled sources, SELL-32 column-major
  int *csr_ptr = nullptr;         // [m+1] relabelled CSR (batched solvers only)
  int *csr_col = nullptr;         // [nnz]
  long long long_elems = 0, sell_elems = 0;
  long long device_bytes = 0;
};

// Class of slice s (classes are few; the scan is warp-uniform).
__host__ __device__ inline int slice_class(const PrClasses &c, int s) {
  int k = 0;
  while (k + 1 < c.n_cls && s >= c.slice[k + 1]) ++k;
  return k;
}

// Work packets: cuts units 0..n_units-1 (device costs `cost`, which the scan
// leaves unchanged) into runs of consecutive units of about equal total cost,
// about `want` of them; a unit costlier than the target is a packet alone.
// *pk_out (device, npk + 1 entries) receives the first unit of each packet and
// n_units last.  Synchronizes `st`.
int make_packets(long long *cost, int n_units, long long want, int **pk_out, int *npk_out,
                 cudaStream_t st);

// Relabelled layout of a pull graph.  When col_ready is given, d_col may
// still be arriving (a copy recorded on another stream): the build does all
// that needs only the row offsets and out-degrees first, then waits for the
// event and checks the column range before reading columns.
int build_pr_layout(int m, long long nnz, const int *d_rowptr, const int *d_col,
                    const int *d_outdeg, int lane_max, int chunk_min, int chunk,
                    bool keep_csr, PrLayout *L, cudaStream_t st, cudaEvent_t col_ready = nullptr);
void free_pr_layout(PrLayout *L);

// Destination-blocked, source-ordered layout of the rows [n_long, n_nz) of a
// PrLayout (gpr_blocked.cu describes the storage).
constexpr int kRunWords = 512;        // most entry words of one run (a warp's unit)
constexpr int kTileRuns = 1 << 16;    // most runs in one tile
constexpr int kBlockedRows = 12288;   // rows per block (accumulators in shared memory)
constexpr int kBlockedMaxRows = 12288;
constexpr int kTileWordsDefault = 1 << 20;
// GPR_FORM_AUTO picks the blocked form from this many edges up
constexpr long long kBlockedAutoMinEdges = 3LL << 24;

struct BlockedLayout {
  int R = 0, tile_slots = 0;
  int run_words = 0;  // most entry words per run: 128 x the kernel's index loads per lane
  int row0 = 0;      // first blocked row; rows [0, row0) are summed in chunks
  int n_chunks = 0;  // chunks of rows [0, row0): a prefix of the exact-order chunks
  int n_blocks = 0, n_tiles = 0;
  long long n_runs = 0, slots = 0, edges = 0;
  unsigned *entry = nullptr;             // [slots]
  uint2 *runs = nullptr;                 // [n_runs] {first word, segment << 16 | words}
  int4 *tiles = nullptr;                 // [n_tiles] {block, run0, run1, residual slot}
  int4 *blocks = nullptr;                // [n_blocks] {row0, nrows, tiles, row range}
  std::vector<int> range_tiles;          // [ranges + 1] residual slots of each row range
  unsigned long long *gacc = nullptr;    // [gacc_rows] sums of multi-tile blocks, rows row0 on
  long long gacc_rows = 0;
  int *bcnt = nullptr;                   // [n_blocks] tiles done in the current sweep
  long long device_bytes = 0;
};

// Rows of the blocked form that stay chunked: the first *row0 rows of the
// exact-order layout's chunked rows [0, L.n_long), either those with more than
// long_min in-edges or, when long_min is 0, those holding more than 1/8 of the
// in-edges of the R rows that start at them; and their *n_chunks chunks.
// Synchronizes st.
int blocked_split(const PrLayout &L, const int *d_rowptr, int long_min, int R, int *row0,
                  int *n_chunks, cudaStream_t st);
int build_blocked_layout(int m, long long nnz, const int *d_rowptr, const int *d_col,
                         const PrLayout &L, int row0, int n_chunks, int R, int tile_slots,
                         int run_words, int workers, BlockedLayout *B, cudaStream_t st);
// The same for several row ranges of the relabelled order (perm: new -> old),
// ascending and disjoint (one per graph of a batch): blocks never span two
// ranges; blocks[b].w is the block's range, tiles[t].w the tile's residual
// slot, numbered range by range (B->range_tiles).
int build_blocked_ranges(int m, long long nnz, const int *d_rowptr, const int *d_col,
                         const int *d_perm, const std::vector<int> &rb,
                         const std::vector<int> &re, int R, int tile_slots, int run_words,
                         int workers, BlockedLayout *B, cudaStream_t st);
// CTAs per SM of the blocked kernel for blocks of R rows: two 512-thread CTAs
// when both fit beside an L1 of about half the SM's 256 KB, else one of 1024.
inline int blocked_ctas_per_sm(int R) { return R <= 8192 ? 2 : 1; }
void free_blocked_layout(BlockedLayout *B);

// Validates a device CSR (rowptr[0] = 0, monotone, rowptr[m] = nnz, every
// column in [0, ncols) when d_col is given) and, when d_outdeg is given,
// out-degrees >= 0.  validate_cols checks the columns alone.
int validate_csr(int m, long long nnz, int ncols, const int *d_rowptr,
                 const int *d_col, const int *d_outdeg, cudaStream_t st);
int validate_cols(long long nnz, int ncols, const int *d_col, cudaStream_t st);

// ---------------------------------------------------------------------------
// SpMV layout: natural row order.  Rows with more than sell_max entries are
// long rows handled in chunks (listed in long_rows); every other row sits in
// a SELL-32 slice with its own length (sell_len, 255 marks a long row whose
// lane is idle in the slice).
// ---------------------------------------------------------------------------
struct SpmvLayout {
  int m = 0;
  long long nnz = 0;
  int sell_max = 0, chunk = 0;
  int n_long = 0, n_chunks = 0, n_slices = 0;
  int *long_rows = nullptr;        // [n_long] row ids, ascending
  long long *long_ptr = nullptr;   // [n_long+1] padded offsets
  int *long_col = nullptr;
  float *long_val = nullptr;
  int *row_cbeg = nullptr;         // [n_long+1]
  int *chunk_row = nullptr;        // [n_chunks] index into long_rows
  long long *slice_ptr = nullptr;  // [n_slices+1]
  int *sell_col = nullptr;
  float *sell_val = nullptr;
  unsigned char *sell_len = nullptr;  // [m]
  long long long_elems = 0, sell_elems = 0;
  long long device_bytes = 0;
};

int build_spmv_layout(int m, long long nnz, const int *d_Ap, const int *d_Aj,
                      const float *d_Ax, int sell_max, int chunk, SpmvLayout *L,
                      cudaStream_t st);
void free_spmv_layout(SpmvLayout *L);

}  // namespace gpr

#define GPR_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      gpr::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call,             \
                     cudaGetErrorString(e_));                                 \
      return GPR_ECUDA;                                                       \
    }                                                                         \
  } while (0)

namespace gpr {
// Status of one CUDA call, for code that must release buffers before it
// returns (GPR_CUDA returns at once): GPR_OK, or GPR_ECUDA with the error set.
inline int cuda_status(cudaError_t e, const char *file, int line, const char *what) {
  if (e == cudaSuccess) return GPR_OK;
  set_error("%s:%d: %s: %s", file, line, what, cudaGetErrorString(e));
  return GPR_ECUDA;
}
}  // namespace gpr
#define GPR_CUDA_RC(call) gpr::cuda_status((call), __FILE__, __LINE__, #call)

#define GPR_TRY(call)                                                         \
  do {                                                                        \
    int s_ = (call);                                                          \
    if (s_ != GPR_OK) return s_;                                              \
  } while (0)

// Device-resident pull graph behind the opaque gpr_graph handle.
struct gpr_graph {
  int device = 0;
  gpr::PrLayout L;
  float *s = nullptr;        // [m] scores, new order
  float *c0 = nullptr;       // [m+1] contributions (sweep parity 0 input)
  float *c1 = nullptr;       // [m+1]
  float *partial = nullptr;  // [n_chunks] partial sums of long-row chunks
  int *cnt = nullptr;        // [n_long] arrival counters of multi-chunk rows
  double *cta_err = nullptr; // [2 * max grid] per-CTA residual partials
  double *err_hist = nullptr;// [err_cap] residual of every sweep
  unsigned *bar = nullptr;   // [4] grid barrier: arrivals, generation
  int *status = nullptr;     // [4] error flags, sweeps done, done flag
  float *scores_tmp = nullptr; // [m] device copy of host scores
  double *res_tmp = nullptr;   // [m+1+n_long] FP64 residual scratch
  int err_cap = 0;
  int last_sweeps = 0;
  int hot = 0;                 // FP32 contributions staged in shared memory per sweep
  int hot_bytes = 0;           // shared-memory budget of the hot prefix
  int grid_hot[12] = {0};      // cooperative grid of each persistent sweep kernel
  void *h0 = nullptr, *h1 = nullptr;  // BF16 contributions of the mixed form (on first use)
  int *wq = nullptr;           // [2] work-queue heads of the hot kernel
  bool hot_ok = false;         // every hot-kernel variant is co-resident at grid_hot
  int grid_step = 0, max_grid = 0;
  bool coop = false;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
  // Chunk table of the batched solver (rows above b_dmax in-edges cut into
  // b_chunk-edge chunks), built on first use for a given (b_dmax, b_chunk).
  int *b_cbeg = nullptr, *b_crow = nullptr;
  int b_nlong = -1, b_nchunks = 0, b_dmax = 0, b_chunk = 0;
  // Chunk descriptors (int4 per chunk) and the packet table (first unit of
  // each of b_npk packets), rebuilt with the chunk table or for another
  // packet count b_pk_want.
  void *b_cdesc = nullptr;
  int *b_pk = nullptr;
  int b_npk = -1;
  long long b_pk_want = 0;
  // Packet tables of the narrower layouts a batched solve packs its
  // still-updating vectors into, by log2 of the rows per row group.
  int *b_pkr[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int b_npkr[6] = {-1, -1, -1, -1, -1, -1};
  long long b_pkwr[6] = {0, 0, 0, 0, 0, 0};
  // Push solver: edges sorted by source and the per-vertex accumulators,
  // built on first use.
  int *push_src = nullptr, *push_dst = nullptr;
  float *push_sum = nullptr;
  // Graph mode: the instantiated sweep-loop graph and the kernel and
  // arguments it was built for.
  cudaGraph_t loop_graph = nullptr;
  cudaGraphExec_t loop_exec = nullptr;
  int loop_ki = -1;
  // Blocked form (GPR_LAYOUT_BLOCKED): its layout, the persistent kernel's
  // grid and co-residency, the tile-queue heads and the largest |score|.
  gpr::BlockedLayout B;
  bool has_blocked = false, blocked_ok = false;
  int grid_blocked = 0, blocked_ctas = 1;  // blocked-form CTAs: total, per SM
  int *tq = nullptr;
  unsigned *fx_max = nullptr;
  alignas(8) unsigned char loop_args[512] = {0};
};

namespace gpr {
constexpr int kZeroRowsPerUnit = 128;  // rows per zero-in-degree work unit
constexpr int kSellMaxDefault = 64;    // SpMV: row length bound of the SELL bin;
                                       // PR: max edges per lane in a SELL slice
constexpr int kChunkMinDefault = 4096; // PR: rows with more in-edges are chunked
constexpr int kChunkDefault = 4096;    // edges per long-row chunk (multiple of 128)
constexpr int kBlock = 256;            // threads per CTA of the per-sweep kernels
constexpr int kHotDefault = 32768;     // contributions staged in shared memory (128 KB)
constexpr int kHotMax = 56832;         // 222 KB: the most one CTA may take

__host__ __device__ inline long long ceil_div(long long a, long long b) {
  return (a + b - 1) / b;
}

// Sweeps the reference's loop counts on a graph with no vertices
// (src/pr/omp_base.cc:23-43): every sweep's residual is 0, so the loop stops
// after the first sweep when 0 < tol and runs to max_iter otherwise.
inline int empty_graph_sweeps(double tol, int max_iter) {
  return max_iter <= 0 ? 0 : (0.0 < tol ? 1 : max_iter);
}
}  // namespace gpr
