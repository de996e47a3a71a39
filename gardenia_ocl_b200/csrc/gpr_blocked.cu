// Destination-blocked, source-ordered layout of the pull graph (the blocked
// form of the sweep).
//
// A pull sweep gathers contrib[u] for every edge u -> v.  In CSR order the
// sources of consecutive gathers are unrelated, so on a large power-law graph
// nearly every gather outside the shared-memory hot prefix is its own L2
// request (one request per edge is the bound of the exact-order kernel).
// Here the rows with at most long_min in-edges (long_min >= chunk_min: every
// row the exact-order kernel puts in SELL slices, and the chunked rows up to
// long_min) are cut into blocks of R consecutive rows of the relabelled order, and the edges of each block are sorted by SOURCE: a
// warp's 32 gathers then fall on one or two 128-byte lines, and a block's
// edges fetch each contribution line about once (RMAT scale 24, R = 12288:
// ~0.16 sectors per edge instead of ~0.64 requests).  The sums are formed in
// shared memory by the CTA that owns the block (gpr_pagerank.cu, k_pr_blocked).
//
// Storage, per block b (rows [row0, row0 + nrows)):
//   entries  one 32-bit word per edge: (source & 0xFFFF) << 16 | (row - row0),
//            grouped by the 65536-source segment (source >> 16) and, inside a
//            group, by source; every group starts on a multiple of 4 words
//            (padding words are 0xFFFFFFFF and read nothing)
//   runs     {first word, segment << 16 | words}: at most run_words words (128
//            per index load of a lane; 512) of one group (one warp's unit of work)
//   tiles    {block, first run, end run, residual slot}: consecutive runs of one block,
//            at most tile_slots words and kTileRuns runs (one CTA's unit), in
//            descending size (the CTA queue hands out the heaviest first)
//   blocks   {row0, nrows, tiles, row range}
// Rows of heavier in-degree (the first row0 rows, chunked) and rows without
// in-edges keep the exact-order layout's work units: the chunks of rows
// [0, row0) are the first row_cbeg[row0] chunks of the exact-order layout.
//
// Construction: every in-edge of a blocked row gets the key (block << 32 |
// source) and the value (row - row0); one radix sort orders them; the group
// starts are selected on the device and the run / tile tables (a few hundred
// thousand entries) are cut on the host.
//
// Tail of the sweep: CTAs take tiles heaviest first, each as it frees, so the
// sweep ends when the last CTA finishes its last tile.  With tiles of nearly
// one size, tiles / CTAs just above an integer leaves most CTAs idle for a
// whole tile (RMAT scale 22: 890 tiles of 73K words on 296 CTAs, a quarter of
// the sweep at the grid barrier).  The builder plays the queue on the host
// (tile time = words + 2 per block row + 1024, for opening and closing it)
// and halves, at a run boundary, every tile that would end after 1.02 x the
// balanced time, until none does (or none can be halved).  A tile's real time
// also grows with the sparsity of its block (RMAT scale 24: ~0.7 ns per word
// in blocks of < 20 edges per row, ~0.19 in the densest), but ordering and
// splitting by that estimate measured slower than by words: each extra split
// adds a cross-tile flush of the block's rows.
#include <cub/cub.cuh>

#include <algorithm>
#include <functional>
#include <queue>
#include <type_traits>
#include <vector>

#include "gpr_internal.cuh"

namespace gpr {

namespace {

// In-degrees of the rows [0, n) of the relabelled order.
__global__ void k_new_degrees(int n, const int *__restrict__ perm, const int *__restrict__ rowptr,
                              int *deg) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) {
    const int o = perm[r];
    deg[r] = rowptr[o + 1] - rowptr[o];
  }
}

__global__ void k_inverse(int m, const int *__restrict__ perm, int *inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) inv[perm[i]] = i;
}

// Sort keys of the blocked edges.  Wide: key = block << 32 | source (64
// bits), value = row in block.  Compact (when the bits fit 31): key = block
// << sb | source >> 3, the 8-source sector in sb >= 13 bits (32 bits: fewer
// passes and two thirds of the bytes of the sort), value = (source & 7) << 16
// | row in block.  Both order a block's edges by segment (source >> 16), then by
// sector: a warp's gathers share lines either way (within a sector the
// compact sort keeps the edges in input order; the sums do not depend on it).
// Excluded edges get the key ~0 (sorted last).
template <bool C>
struct BlockKey {
  using T = typename std::conditional<C, unsigned, unsigned long long>::type;
  static constexpr T none = ~(T)0;
  __device__ static T make(unsigned long long blk, unsigned src, int sb) {
    return C ? (T)((blk << sb) | (src >> 3)) : (T)((blk << 32) | src);
  }
  __device__ static unsigned value(unsigned src, unsigned dl) {
    return C ? ((src & 7u) << 16) | dl : dl;
  }
  __device__ static unsigned long long group(T k) { return C ? (k >> 13) : (k >> 16); }
  __device__ static int block(T k, int sb) { return C ? (int)(k >> sb) : (int)(k >> 32); }
  __device__ static int segment(T k, int sb) {
    return C ? (int)((k & ((1u << sb) - 1u)) >> 13) : (int)((k & 0xFFFFFFFFull) >> 16);
  }
  // the entry word: (source & 0xFFFF) << 16 | row in block
  __device__ static unsigned entry(T k, unsigned v) {
    const unsigned lo = C ? ((unsigned)(k & 0x1FFFu) << 3) | ((v >> 16) & 7u)
                          : (unsigned)(k & 0xFFFFull);
    return (lo << 16) | (v & 0xFFFFu);
  }
};

// One warp per original row: the keys and values of its in-edges when its
// new label falls in a blocked range [rb[i], re[i]) (ranges ascending and
// disjoint, range i's blocks numbered from bb[i]); other edges get the key ~0.
template <bool C>
__global__ void k_block_keys(int m, const int *__restrict__ rowptr, const int *__restrict__ col,
                             const int *__restrict__ inv, int n_ranges, const int *__restrict__ rb,
                             const int *__restrict__ re, const int *__restrict__ bb, int R, int sb,
                             typename BlockKey<C>::T *key, unsigned *val) {
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= m) return;
  const int o = (int)w;
  const int r = inv[o];
  int lo = 0, hi = n_ranges - 1;  // the last range starting at or before r
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (rb[mid] <= r) lo = mid;
    else hi = mid - 1;
  }
  const bool in = r >= rb[lo] && r < re[lo];
  const unsigned long long blk = in ? (unsigned long long)(bb[lo] + (r - rb[lo]) / R) : 0ull;
  const unsigned dl = in ? (unsigned)((r - rb[lo]) % R) : 0u;
  for (int e = rowptr[o] + lane; e < rowptr[o + 1]; e += 32) {
    const unsigned src = (unsigned)inv[col[e]];
    key[e] = in ? BlockKey<C>::make(blk, src, sb) : BlockKey<C>::none;
    val[e] = BlockKey<C>::value(src, dl);
  }
}

// First index whose key is ~0 (the blocked edges precede it): one thread.
template <bool C>
__global__ void k_count_blocked(long long n, const typename BlockKey<C>::T *__restrict__ key,
                                long long *out) {
  long long lo = 0, hi = n;
  while (lo < hi) {
    const long long mid = (lo + hi) / 2;
    if (key[mid] == BlockKey<C>::none) hi = mid;
    else lo = mid + 1;
  }
  *out = lo;
}

// 1 where a (block, segment) group starts
template <bool C>
__global__ void k_group_flags(long long n, const typename BlockKey<C>::T *__restrict__ key,
                              int *flag) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n)
    flag[i] = (i == 0 || BlockKey<C>::group(key[i]) != BlockKey<C>::group(key[i - 1])) ? 1 : 0;
}

template <bool C>
__global__ void k_group_keys(int ng, const int *__restrict__ gstart,
                             const typename BlockKey<C>::T *__restrict__ key, int sb, int *gblk,
                             int *gseg) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < ng) {
    const typename BlockKey<C>::T k = key[gstart[g]];
    gblk[g] = BlockKey<C>::block(k, sb);
    gseg[g] = BlockKey<C>::segment(k, sb);
  }
}

// Entry i of the sorted edges goes to word gpos[gid] + (i - gstart[gid]),
// gid = (inclusive count of group starts up to i) - 1.
template <bool C>
__global__ void k_place(long long n, const typename BlockKey<C>::T *__restrict__ key,
                        const unsigned *__restrict__ val, const int *__restrict__ gid1,
                        const int *__restrict__ gstart, const long long *__restrict__ gpos,
                        unsigned *entry) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = gid1[i] - 1;
  entry[gpos[g] + (i - gstart[g])] = BlockKey<C>::entry(key[i], val[i]);
}

unsigned grid_of(long long n, int block = 256) {
  const long long g = (n + block - 1) / block;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

void free_blocked_layout(BlockedLayout *B) {
  dfree(B->entry);
  dfree(B->runs);
  dfree(B->tiles);
  dfree(B->blocks);
  dfree(B->gacc);
  dfree(B->bcnt);
  *B = BlockedLayout();
}

int blocked_split(const PrLayout &L, const int *d_rowptr, int long_min, int R, int *row0,
                  int *n_chunks, cudaStream_t st) {
  *row0 = 0;
  *n_chunks = 0;
  if (L.n_long == 0) return GPR_OK;
  // in-degrees of the chunkable rows and of the R rows after them
  const int n = (int)std::min<long long>(L.n_nz, (long long)L.n_long + R);
  int *d_deg = nullptr;
  int rc = dalloc(&d_deg, (size_t)n, "blocked: heavy rows");
  if (rc != GPR_OK) return rc;
  std::vector<int> deg((size_t)n);
  k_new_degrees<<<grid_of(n), 256, 0, st>>>(n, L.perm, d_rowptr, d_deg);
  rc = GPR_CUDA_RC(cudaGetLastError());
  if (rc == GPR_OK)
    rc = GPR_CUDA_RC(cudaMemcpyAsync(deg.data(), d_deg, sizeof(int) * (size_t)n,
                                     cudaMemcpyDeviceToHost, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaStreamSynchronize(st));
  dfree(d_deg);
  if (rc != GPR_OK) return rc;
  // The chunked rows are a prefix (the order is by descending in-degree).
  // With long_min > 0: the rows above long_min in-edges.  Otherwise the rows
  // that would hold more than 1/8 of the edges of a block starting at them:
  // their additions would queue on one shared-memory word (a star's hub),
  // which chunks sum without contention.
  int cnt = 0;
  if (long_min > 0) {
    while (cnt < L.n_long && deg[cnt] > long_min) ++cnt;
  } else {
    long long win = 0;  // in-edges of rows [cnt, cnt + R)
    for (int j = 0; j < std::min(n, R); ++j) win += deg[j];
    while (cnt < L.n_long && 8LL * deg[cnt] > win) {
      win -= deg[cnt];
      if (cnt + R < n) win += deg[cnt + R];
      ++cnt;
    }
  }
  int cb = 0;
  rc = GPR_CUDA_RC(cudaMemcpyAsync(&cb, L.row_cbeg + cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaStreamSynchronize(st));
  if (rc != GPR_OK) return rc;
  *row0 = cnt;
  *n_chunks = cb;
  return GPR_OK;
}

int build_blocked_layout(int m, long long nnz, const int *d_rowptr, const int *d_col,
                         const PrLayout &L, int row0, int n_chunks, int R, int tile_slots,
                         int run_words, int workers, BlockedLayout *B, cudaStream_t st) {
  if (row0 < 0 || row0 > L.n_long) {
    set_error("blocked layout: first blocked row %d outside [0, %d]", row0, L.n_long);
    return GPR_EINVAL;
  }
  const std::vector<int> rb{row0}, re{L.n_nz};
  const int rc = build_blocked_ranges(m, nnz, d_rowptr, d_col, L.perm, rb, re, R, tile_slots,
                                      run_words, workers, B, st);
  B->n_chunks = n_chunks;
  return rc;
}

int build_blocked_ranges(int m, long long nnz, const int *d_rowptr, const int *d_col,
                         const int *d_perm, const std::vector<int> &rb,
                         const std::vector<int> &re, int R, int tile_slots, int run_words,
                         int workers, BlockedLayout *B, cudaStream_t st) {
  *B = BlockedLayout();
  B->R = R;
  B->run_words = run_words;
  B->tile_slots = tile_slots;
  const int n_ranges = (int)rb.size();
  bool ranges_ok = n_ranges >= 1 && re.size() == rb.size();
  for (int i = 0; ranges_ok && i < n_ranges; ++i)
    ranges_ok = rb[i] >= 0 && re[i] >= rb[i] && re[i] <= m && (i == 0 || rb[i] >= re[i - 1]);
  if (R < 1 || R > kBlockedMaxRows || tile_slots < kRunWords || !ranges_ok || run_words < 128 ||
      run_words > 512 || run_words % 128 != 0) {
    set_error("blocked layout: block rows %d must be in [1, %d], tile words %d >= %d, row "
              "ranges ascending and disjoint", R, kBlockedMaxRows, tile_slots, kRunWords);
    return GPR_EINVAL;
  }
  // Blocks: each range cut into blocks of R rows; accumulators of the rows
  // [row0, row end of the last range).
  std::vector<int> bb(n_ranges + 1, 0);
  for (int i = 0; i < n_ranges; ++i) bb[i + 1] = bb[i] + (int)ceil_div(re[i] - rb[i], R);
  B->n_blocks = bb[n_ranges];
  B->row0 = rb[0];
  B->range_tiles.assign(n_ranges + 1, 0);
  const int n_rows = re[n_ranges - 1] - rb[0];
  if (B->n_blocks == 0 || nnz == 0) {
    B->n_blocks = 0;
    return GPR_OK;
  }
  // Keys and values of every edge; blocked ones first after the sort.
  int *inv = nullptr, *d_rng = nullptr;
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  unsigned *v0 = nullptr, *v1 = nullptr;
  void *tmp = nullptr;
  int rc = GPR_OK;
  auto fail = [&](int code) {
    dfree(inv); dfree(d_rng); dfree(k0); dfree(k1); dfree(v0); dfree(v1); dfree(tmp);
    free_blocked_layout(B);
    return code;
  };
  if ((rc = dalloc(&inv, (size_t)m + 2, "blocked: inverse")) != GPR_OK ||
      (rc = dalloc(&d_rng, 3 * (size_t)n_ranges, "blocked: row ranges")) != GPR_OK ||
      (rc = dalloc(&k0, (size_t)nnz, "blocked: keys")) != GPR_OK ||
      (rc = dalloc(&k1, (size_t)nnz, "blocked: keys")) != GPR_OK ||
      (rc = dalloc(&v0, (size_t)nnz, "blocked: rows")) != GPR_OK ||
      (rc = dalloc(&v1, (size_t)nnz, "blocked: rows")) != GPR_OK)
    return fail(rc);
  if ((rc = GPR_CUDA_RC(cudaMemcpyAsync(d_rng, rb.data(), sizeof(int) * n_ranges,
                                        cudaMemcpyHostToDevice, st))) != GPR_OK ||
      (rc = GPR_CUDA_RC(cudaMemcpyAsync(d_rng + n_ranges, re.data(), sizeof(int) * n_ranges,
                                        cudaMemcpyHostToDevice, st))) != GPR_OK ||
      (rc = GPR_CUDA_RC(cudaMemcpyAsync(d_rng + 2 * n_ranges, bb.data(), sizeof(int) * n_ranges,
                                        cudaMemcpyHostToDevice, st))) != GPR_OK)
    return fail(rc);
  // Sort on (block, source or sector): the bits of the sources, then of the
  // blocks (the ~0 keys of the excluded edges have every bit set and sort
  // last).  Compact keys when block and sector fit 31 bits.
  int blk_bits = 1, src_bits = 3;
  while ((1LL << blk_bits) <= B->n_blocks) ++blk_bits;
  while ((1LL << src_bits) < m) ++src_bits;
  const int sb = std::max(src_bits - 3, 13);  // sector bits: key >> 13 is (block, segment)
  const bool compact = sb + blk_bits <= 31;
  const int end_bit = compact ? sb + blk_bits : 32 + blk_bits;
  unsigned *c0 = reinterpret_cast<unsigned *>(k0), *c1 = reinterpret_cast<unsigned *>(k1);
  k_inverse<<<grid_of(m), 256, 0, st>>>(m, d_perm, inv);
  if (compact)
    k_block_keys<true><<<grid_of((long long)m * 32), 256, 0, st>>>(
        m, d_rowptr, d_col, inv, n_ranges, d_rng, d_rng + n_ranges, d_rng + 2 * n_ranges, R, sb,
        c0, v0);
  else
    k_block_keys<false><<<grid_of((long long)m * 32), 256, 0, st>>>(
        m, d_rowptr, d_col, inv, n_ranges, d_rng, d_rng + n_ranges, d_rng + 2 * n_ranges, R, sb,
        k0, v0);
  if ((rc = GPR_CUDA_RC(cudaGetLastError())) != GPR_OK) return fail(rc);
  auto sort = [&](auto *ka, auto *kb_) -> int {
    using KT = typename std::remove_pointer<decltype(ka)>::type;
    size_t tb = 0;
    cub::DoubleBuffer<KT> kb(ka, kb_);
    cub::DoubleBuffer<unsigned> vb(v0, v1);
    int r = GPR_CUDA_RC(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, (int)nnz, 0, end_bit, st));
    if (r == GPR_OK) r = dmalloc(&tmp, tb, "blocked: sort scratch");
    if (r == GPR_OK)
      r = GPR_CUDA_RC(cub::DeviceRadixSort::SortPairs(tmp, tb, kb, vb, (int)nnz, 0, end_bit, st));
    dfree(tmp);
    tmp = nullptr;
    if (r == GPR_OK && kb.Current() != ka) {
      std::swap(k0, k1);
      std::swap(c0, c1);
    }
    if (r == GPR_OK && vb.Current() != v0) std::swap(v0, v1);
    return r;
  };
  if ((rc = compact ? sort(c0, c1) : sort(k0, k1)) != GPR_OK) return fail(rc);
  // Number of blocked edges: the keys before the first ~0.
  long long n_edges = 0;
  {
    long long *d_n = reinterpret_cast<long long *>(inv);  // inv is no longer needed
    if (compact) k_count_blocked<true><<<1, 1, 0, st>>>(nnz, c0, d_n);
    else k_count_blocked<false><<<1, 1, 0, st>>>(nnz, k0, d_n);
    if ((rc = GPR_CUDA_RC(cudaGetLastError())) != GPR_OK ||
        (rc = GPR_CUDA_RC(cudaMemcpyAsync(&n_edges, d_n, sizeof(n_edges), cudaMemcpyDeviceToHost,
                                          st))) != GPR_OK ||
        (rc = GPR_CUDA_RC(cudaStreamSynchronize(st))) != GPR_OK)
      return fail(rc);
  }
  B->edges = n_edges;
  if (n_edges == 0) {
    dfree(inv); dfree(d_rng); dfree(k0); dfree(k1); dfree(v0); dfree(v1);
    B->n_blocks = 0;
    return GPR_OK;
  }
  // Group starts (block, segment) and their keys.
  int *flag = reinterpret_cast<int *>(k1);  // k1 is free now
  int *gid1 = reinterpret_cast<int *>(v1);                       // so is v1
  if (compact) k_group_flags<true><<<grid_of(n_edges), 256, 0, st>>>(n_edges, c0, flag);
  else k_group_flags<false><<<grid_of(n_edges), 256, 0, st>>>(n_edges, k0, flag);
  int *gstart = nullptr, *nsel = nullptr;
  if ((rc = dalloc(&gstart, (size_t)n_edges, "blocked: groups")) != GPR_OK ||
      (rc = dalloc(&nsel, 1, "blocked: group count")) != GPR_OK) {
    dfree(gstart);
    return fail(rc);
  }
  int ng = 0;
  {
    size_t tb = 0;
    cub::CountingInputIterator<int> it(0);
    rc = GPR_CUDA_RC(cub::DeviceSelect::Flagged(nullptr, tb, it, flag, gstart, nsel, (int)n_edges, st));
    if (rc == GPR_OK) rc = dmalloc(&tmp, tb, "blocked: select scratch");
    if (rc == GPR_OK)
      rc = GPR_CUDA_RC(cub::DeviceSelect::Flagged(tmp, tb, it, flag, gstart, nsel, (int)n_edges, st));
    dfree(tmp);
    tmp = nullptr;
    // inclusive count of group starts: the group of every entry
    tb = 0;
    if (rc == GPR_OK)
      rc = GPR_CUDA_RC(cub::DeviceScan::InclusiveSum(nullptr, tb, flag, gid1, (int)n_edges, st));
    if (rc == GPR_OK) rc = dmalloc(&tmp, tb, "blocked: scan scratch");
    if (rc == GPR_OK)
      rc = GPR_CUDA_RC(cub::DeviceScan::InclusiveSum(tmp, tb, flag, gid1, (int)n_edges, st));
    dfree(tmp);
    tmp = nullptr;
    if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(&ng, nsel, sizeof(int),
                                                       cudaMemcpyDeviceToHost, st));
    if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaStreamSynchronize(st));
  }
  dfree(nsel);
  if (rc != GPR_OK) {
    dfree(gstart);
    return fail(rc);
  }
  std::vector<int> h_gstart(ng), h_gblk(ng), h_gseg(ng);
  {
    int *gblk = nullptr, *gseg = nullptr;
    rc = dalloc(&gblk, (size_t)ng, "blocked: group blocks");
    if (rc == GPR_OK) rc = dalloc(&gseg, (size_t)ng, "blocked: group segments");
    if (rc == GPR_OK) {
      if (compact) k_group_keys<true><<<grid_of(ng), 256, 0, st>>>(ng, gstart, c0, sb, gblk, gseg);
      else k_group_keys<false><<<grid_of(ng), 256, 0, st>>>(ng, gstart, k0, sb, gblk, gseg);
      rc = GPR_CUDA_RC(cudaGetLastError());
    }
    if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(h_gstart.data(), gstart, sizeof(int) * ng,
                                                       cudaMemcpyDeviceToHost, st));
    if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(h_gblk.data(), gblk, sizeof(int) * ng,
                                                       cudaMemcpyDeviceToHost, st));
    if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(h_gseg.data(), gseg, sizeof(int) * ng,
                                                       cudaMemcpyDeviceToHost, st));
    if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaStreamSynchronize(st));
    dfree(gblk);
    dfree(gseg);
  }
  if (rc != GPR_OK) {
    dfree(gstart);
    return fail(rc);
  }
  // Host: padded group offsets, runs, tiles, blocks.
  std::vector<long long> gpos(ng + 1);
  std::vector<uint2> runs;
  std::vector<int4> tiles;
  std::vector<int4> blocks(B->n_blocks);
  for (int i = 0; i < n_ranges; ++i)
    for (int b = bb[i]; b < bb[i + 1]; ++b) {
      const int r0 = rb[i] + (b - bb[i]) * R;
      blocks[b] = make_int4(r0, std::min(R, re[i] - r0), 0, i);
    }
  runs.reserve((size_t)(n_edges / run_words) + ng + 1);
  long long pos = 0;
  int g = 0;
  while (g < ng) {
    const int b = h_gblk[g];
    // the groups of block b
    int g1 = g;
    while (g1 < ng && h_gblk[g1] == b) ++g1;
    int tile_run0 = (int)runs.size(), tile_runs = 0;
    long long tile_words = 0;
    auto close_tile = [&]() {
      if (tile_runs > 0) {
        tiles.push_back(make_int4(b, tile_run0, (int)runs.size(), (int)tile_words));
        blocks[b].z += 1;
      }
      tile_run0 = (int)runs.size();
      tile_runs = 0;
      tile_words = 0;
    };
    for (int q = g; q < g1; ++q) {
      const long long size = (q + 1 < ng ? (long long)h_gstart[q + 1] : n_edges) - h_gstart[q];
      const long long padded = (size + 3) / 4 * 4;
      gpos[q] = pos;
      for (long long off = 0; off < padded; off += run_words) {
        const int len = (int)std::min<long long>(run_words, padded - off);
        if (tile_runs > 0 && (tile_words + len > tile_slots || tile_runs == kTileRuns)) close_tile();
        runs.push_back(make_uint2((unsigned)(pos + off), ((unsigned)h_gseg[q] << 16) | (unsigned)len));
        ++tile_runs;
        tile_words += len;
      }
      pos += padded;
    }
    close_tile();
    g = g1;
  }
  gpos[ng] = pos;
  if (pos > 0xFFFFFFF0LL) {
    set_error("blocked layout: %lld entry words exceed 32-bit offsets", pos);
    dfree(gstart);
    return fail(GPR_EINVAL);
  }
  const double open_close = 2.0 * R + 1024.0;
  auto cost = [&](const int4 &t) { return t.w + open_close; };
  // Queue order: heaviest first; with several row ranges (a batch of graphs,
  // largest first), range by range, so the CTAs work on few graphs at a
  // time and those graphs' contributions stay in L2 (512-graph batch, 187 MB
  // of contributions: 48.7 -> 44.9 ms per solve).
  auto by_cost = [&](const int4 &x, const int4 &y) {
    if (blocks[x.x].w != blocks[y.x].w) return blocks[x.x].w < blocks[y.x].w;
    return x.w > y.w;
  };
  for (int round = 0; round < 24 && workers > 0; ++round) {
    std::stable_sort(tiles.begin(), tiles.end(), by_cost);
    std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
    for (int i = 0; i < workers; ++i) free_at.push(0.0);
    std::vector<double> end(tiles.size());
    double total = 0.0;
    for (size_t i = 0; i < tiles.size(); ++i) {
      end[i] = free_at.top() + cost(tiles[i]);
      free_at.pop();
      free_at.push(end[i]);
      total += cost(tiles[i]);
    }
    const double share = total / workers;
    std::vector<int4> next;
    next.reserve(tiles.size() + workers);
    bool split = false;
    for (size_t i = 0; i < tiles.size(); ++i) {
      const int4 t = tiles[i];
      if (end[i] <= 1.02 * share || t.z - t.y < 2) {
        next.push_back(t);
        continue;
      }
      int mid = t.y, left = 0;
      while (mid < t.z - 1 && left + (int)(runs[mid].y & 0xFFFFu) <= t.w / 2)
        left += (int)(runs[mid++].y & 0xFFFFu);
      if (mid == t.y) left += (int)(runs[mid++].y & 0xFFFFu);
      next.push_back(make_int4(t.x, t.y, mid, left));
      next.push_back(make_int4(t.x, mid, t.z, t.w - left));
      blocks[t.x].z += 1;
      split = true;
    }
    tiles.swap(next);
    if (!split) break;
  }
  std::stable_sort(tiles.begin(), tiles.end(), by_cost);
  // Each tile's residual slot (its .w on the device; the words are host-only):
  // tiles numbered range by range, so a range's slots are contiguous.
  for (const int4 &t : tiles) B->range_tiles[blocks[t.x].w + 1] += 1;
  for (int i = 0; i < n_ranges; ++i) B->range_tiles[i + 1] += B->range_tiles[i];
  {
    std::vector<int> next_slot(B->range_tiles.begin(), B->range_tiles.end() - 1);
    for (int4 &t : tiles) t.w = next_slot[blocks[t.x].w]++;
  }
  B->slots = pos;
  B->n_runs = (long long)runs.size();
  B->n_tiles = (int)tiles.size();
  // Device tables and the entries.
  long long *d_gpos = nullptr;
  rc = dalloc(&d_gpos, (size_t)ng, "blocked: group offsets");
  if (rc == GPR_OK) rc = dalloc(&B->entry, (size_t)pos, "blocked: entries");
  if (rc == GPR_OK) rc = dalloc(&B->runs, (size_t)B->n_runs, "blocked: runs");
  if (rc == GPR_OK) rc = dalloc(&B->tiles, (size_t)B->n_tiles, "blocked: tiles");
  if (rc == GPR_OK) rc = dalloc(&B->blocks, (size_t)B->n_blocks, "blocked: blocks");
  if (rc == GPR_OK) rc = dalloc(&B->gacc, (size_t)n_rows, "blocked: cross-tile sums");
  B->gacc_rows = n_rows;
  if (rc == GPR_OK) rc = dalloc(&B->bcnt, (size_t)B->n_blocks, "blocked: tile counters");
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(d_gpos, gpos.data(), sizeof(long long) * ng,
                                                     cudaMemcpyHostToDevice, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(B->runs, runs.data(), sizeof(uint2) * runs.size(),
                                                     cudaMemcpyHostToDevice, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(B->tiles, tiles.data(), sizeof(int4) * tiles.size(),
                                                     cudaMemcpyHostToDevice, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemcpyAsync(B->blocks, blocks.data(), sizeof(int4) * blocks.size(),
                                                     cudaMemcpyHostToDevice, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemsetAsync(B->entry, 0xFF, sizeof(unsigned) * (size_t)pos, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemsetAsync(B->gacc, 0, sizeof(unsigned long long) * n_rows, st));
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemsetAsync(B->bcnt, 0, sizeof(int) * B->n_blocks, st));
  if (rc == GPR_OK) {
    if (compact)
      k_place<true><<<grid_of(n_edges), 256, 0, st>>>(n_edges, c0, v0, gid1, gstart, d_gpos, B->entry);
    else
      k_place<false><<<grid_of(n_edges), 256, 0, st>>>(n_edges, k0, v0, gid1, gstart, d_gpos, B->entry);
    rc = GPR_CUDA_RC(cudaGetLastError());
  }
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaStreamSynchronize(st));
  dfree(d_gpos);
  dfree(gstart);
  if (rc != GPR_OK) return fail(rc);
  dfree(inv); dfree(d_rng); dfree(k0); dfree(k1); dfree(v0); dfree(v1);
  B->device_bytes = 4 * pos + 8 * B->n_runs + 16LL * B->n_tiles + 16LL * B->n_blocks +
                    8LL * n_rows + 4LL * B->n_blocks;
  return GPR_OK;
}

}  // namespace gpr
