// Pull PageRank on B200: sweep kernels, graph handle and solve driver.
//
// One sweep is one pass of the reference's iteration body
// (src/pr/omp_base.cc:23-44): every vertex pulls the contributions of its
// in-neighbours, updates its score, and adds |s_new - s_old| to an FP64 L1
// residual.  The contribution of the NEXT sweep (score / out-degree,
// omp_base.cc:25-27) is produced in the same pass from the freshly written
// score, so a sweep reads each per-vertex array once.  Contributions are
// double-buffered (c0/c1 by sweep parity).
//
// Work units, one warp each, over the relabelled layout (gpr_internal.cuh):
//   chunk  -- up to `chunk` edges of a long row; 128-bit index loads;
//             partial sums of multi-chunk rows are combined by the last
//             arriving warp in a fixed order (deterministic)
//   slice  -- 32 consecutive short rows, one lane per row, summing its row
//             in CSR order with one rounded float add per edge exactly like
//             the reference's inner loop (omp_base.cc:34-37)
//   zero   -- 128 rows without in-edges
//
// The score update uses explicitly rounded multiply and add
// (base + kDamp*sum, omp_base.cc:39) so no FMA contraction changes results,
// and the contribution uses IEEE division (omp_base.cc:26).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include <cuda_bf16.h>

#include "gpr_device.cuh"
#include "gpr_internal.cuh"
#include "gpr_blocked.cuh"
#include "gpr_guard.h"

using gpr::PrLayout;
using gpr::kBlockedMaxRows;
using gpr::kTileRuns;

namespace {

struct PrArgs {
  int m, n_long, n_nz, n_chunks, n_slices, n_zblk, chunk;
  gpr::PrClasses cls;
  const long long *long_ptr;
  const int *long_col;
  const int *row_cbeg;
  const int *chunk_row;
  const long long *slice_ptr;
  const int *sell_col;
  const int *outdeg;
  float *s;
  void *c0, *c1;   // contributions by sweep parity: float or __nv_bfloat16
  float *partial;
  int *cnt;
  double *cta_err, *err_hist;
  unsigned *bar;
  int *status;
  float base, damp;
  double tol;
  int max_iter;
  int bar_expect;
  long long timeout_ns;
  int hot;                // contributions [0, hot) are staged in shared memory
  int *wq;                // [2] work-queue heads of the hot kernel, by sweep parity
  int batch;              // units per work-queue grab
  unsigned long long cond;  // graph mode: while-node condition handle (0: none)
  // blocked form (gpr_blocked.cu): tiles of source-ordered entries per block
  int n_tiles, acc_rows;  // acc_rows: high words of the shared accumulators start here
  int blk_row0;           // first blocked row (rows before it are chunked)
  const int4 *tiles;
  const int4 *blocks;
  const uint2 *runs;
  const unsigned *entry;
  unsigned long long *gacc;
  int *bcnt;
  int *tq;                // [2] tile-queue heads by sweep parity
  float fx_scale;         // 2^S: contributions as 64-bit fixed point
  double fx_inv;          // 2^-S
};

using namespace gpr::dev;

// Score update of row r from its pulled sum and its prefetched old score and
// out-degree; returns |s_new - s_old|.
template <typename T>
__device__ __forceinline__ double row_update(const PrArgs &a, int r, float sum, float so, int od,
                                             T *cout, const Policies &pol) {
  const float sn = __fadd_rn(a.base, __fmul_rn(a.damp, sum));
  st_f32(a.s + r, sn, pol.stream);
  st_c(cout + r, __fdiv_rn(sn, __int2float_rn(od)), pol.keep);
  return (double)fabsf(__fsub_rn(sn, so));
}

// One chunk of a long row: U4 16-byte index loads per lane in flight, then
// 4*U4 independent gathers.
template <int U4, typename Gather, typename T>
__device__ __forceinline__ double do_chunk(const PrArgs &a, const Gather &gat, T *cout, int c,
                                           int lane, const Policies &pol) {
  const int r = a.chunk_row[c];
  const int cb = a.row_cbeg[r];
  const int nc = a.row_cbeg[r + 1] - cb;
  float so = 0.f;
  int od = 1;
  if (lane == 0) {
    so = ld_f32_stream(a.s + r, pol.stream);
    od = ld_s32_stream(a.outdeg + r, pol.stream);
  }
  const long long b = a.long_ptr[r] + (long long)(c - cb) * a.chunk;
  const long long e = min(b + (long long)a.chunk, a.long_ptr[r + 1]);
  float acc = 0.f;
  for (long long k0 = b + 4 * lane; k0 < e; k0 += 128 * U4) {
    int4 q[U4];
#pragma unroll
    for (int i = 0; i < U4; ++i)
      q[i] = (k0 + 128 * i < e) ? ld_idx4(a.long_col + k0 + 128 * i, pol.stream)
                                : make_int4(a.m, a.m, a.m, a.m);
    float v[4 * U4];
#pragma unroll
    for (int i = 0; i < U4; ++i) {
      v[4 * i + 0] = gat(q[i].x);
      v[4 * i + 1] = gat(q[i].y);
      v[4 * i + 2] = gat(q[i].z);
      v[4 * i + 3] = gat(q[i].w);
    }
#pragma unroll
    for (int i = 0; i < 4 * U4; ++i) acc += v[i];
  }
  acc = warp_sum(acc);
  if (nc == 1) return lane == 0 ? row_update(a, r, acc, so, od, cout, pol) : 0.0;
  int last = 0;
  if (lane == 0) {
    a.partial[c] = acc;
    __threadfence();
    last = atomicAdd(a.cnt + r, 1) == nc - 1;
  }
  last = __shfl_sync(kFull, last, 0);
  if (!last) return 0.0;
  __threadfence();
  float t = 0.f;
  for (int q = lane; q < nc; q += 32) t += __ldcg(a.partial + cb + q);
  t = warp_sum(t);
  if (lane != 0) return 0.0;
  atomicExch(a.cnt + r, 0);
  return row_update(a, r, t, so, od, cout, pol);
}

// One SELL slice: 32 >> lw rows, w = 1 << lw lanes per row.  Each lane runs
// batches of U independent index loads followed by U independent gathers;
// entries past the slice length read the sentinel slot (an exact +0).
template <int U, typename Gather, typename T>
__device__ __forceinline__ double do_slice(const PrArgs &a, const Gather &gat, T *cout,
                                           int sidx, int lane, const Policies &pol) {
  const int c = gpr::slice_class(a.cls, sidx);
  const int lw = a.cls.lw[c];
  const int row0 = a.cls.row[c] + ((sidx - a.cls.slice[c]) << (5 - lw));
  const int r = row0 + (lane >> lw);
  const bool lead = (lane & ((1 << lw) - 1)) == 0;
  const bool valid = r < a.cls.row[c + 1];
  float so = 0.f;
  int od = 1;
  if (valid && lead) {
    so = ld_f32_stream(a.s + r, pol.stream);
    od = ld_s32_stream(a.outdeg + r, pol.stream);
  }
  const long long b = a.slice_ptr[sidx];
  const int len = (int)((a.slice_ptr[sidx + 1] - b) >> 5);
  const int *p = a.sell_col + b + lane;
  float acc = 0.f;
  for (int j0 = 0; j0 < len; j0 += U) {
    int ci[U];
#pragma unroll
    for (int q = 0; q < U; ++q) ci[q] = (j0 + q < len) ? ld_idx(p + 32 * (j0 + q), pol.stream) : a.m;
    float v[U];
#pragma unroll
    for (int q = 0; q < U; ++q) v[q] = gat(ci[q]);
#pragma unroll
    for (int q = 0; q < U; ++q) acc = __fadd_rn(acc, v[q]);
  }
  for (int o = (1 << lw) >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  return (valid && lead) ? row_update(a, r, acc, so, od, cout, pol) : 0.0;
}

// Rows without in-edges: s = base from the first sweep on, so they are
// updated in sweep 0 and only their contribution is copied into the other
// buffer in sweep 1; later sweeps skip them (their residual term is 0).
template <typename T>
__device__ __forceinline__ double do_zero(const PrArgs &a, T *cout, int z, int lane, int it,
                                          const Policies &pol) {
  double err = 0.0;
  const int r0 = a.n_nz + z * gpr::kZeroRowsPerUnit;
#pragma unroll
  for (int q = 0; q < gpr::kZeroRowsPerUnit / 32; ++q) {
    const int r = r0 + 32 * q + lane;
    if (r < a.m) {
      const int od = ld_s32_stream(a.outdeg + r, pol.stream);
      if (it == 0) {
        err += row_update(a, r, 0.f, ld_f32_stream(a.s + r, pol.stream), od, cout, pol);
      } else {
        const float sn = __fadd_rn(a.base, __fmul_rn(a.damp, 0.f));
        st_c(cout + r, __fdiv_rn(sn, __int2float_rn(od)), pol.keep);
      }
    }
  }
  return err;
}

template <int U, int U4, typename T>
__device__ __forceinline__ double sweep(const PrArgs &a, const T *cin, T *cout,
                                        long long gw, long long nw, int lane, int it,
                                        const Policies &pol) {
  const long long u1 = a.n_chunks, u2 = u1 + a.n_slices;
  const long long u3 = u2 + (it < 2 ? a.n_zblk : 0);
  double err = 0.0;
  const GlobalGather<T> gat{cin, pol.keep};
  for (long long u = gw; u < u3; u += nw) {
    if (u < u1) err += do_chunk<U4>(a, gat, cout, (int)u, lane, pol);
    else if (u < u2) err += do_slice<U>(a, gat, cout, (int)(u - u1), lane, pol);
    else err += do_zero(a, cout, (int)(u - u2), lane, it, pol);
  }
  return err;
}

// Sum over the CTA; the result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

// Grid barrier that also reduces the per-CTA residuals of sweep `it` into
// err_hist[it].  The CTA that arrives last sums the partials in CTA order
// (deterministic) and opens the next generation.  Every wait is bounded by
// timeout_ns of %globaltimer; on expiry the CTA raises status[0] bit 0 and
// the caller returns.  Requires co-resident CTAs (cooperative launch).
__device__ bool barrier_reduce(const PrArgs &a, int it, double cta_total) {
  __shared__ int s_state;
  __shared__ unsigned s_gen;
  const unsigned G = gridDim.x;
  if (threadIdx.x == 0) {
    a.cta_err[(size_t)(it & 1) * G + blockIdx.x] = cta_total;
    s_gen = ld_acquire(a.bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(a.bar, 1u);
    s_state = (arrived == (unsigned)a.bar_expect - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (s_state == 1) {
    if (threadIdx.x < 32) {
      __threadfence();
      const double *src = a.cta_err + (size_t)(it & 1) * G;
      double t = 0.0;
      for (unsigned i = threadIdx.x; i < G; i += 32) t += __ldcg(src + i);
      t = warp_sum(t);
      if (threadIdx.x == 0) {
        a.err_hist[it] = t;
        if (a.wq) atomicExch(a.wq + (it & 1), 0);  // reused by sweep it + 2
        if (a.tq) atomicExch(a.tq + (it & 1), 0);
        atomicExch(a.bar, 0u);
        __threadfence();
        atomicAdd(a.bar + 1, 1u);
      }
    }
  } else if (threadIdx.x == 0) {
    const long long t0 = global_ns();
    unsigned spins = 0;
    while (ld_acquire(a.bar + 1) == s_gen) {
      if ((++spins & 31u) == 0 && global_ns() - t0 > a.timeout_ns) {
        atomicOr(a.status, 1);
        s_state = 2;
        break;
      }
      __nanosleep(100);
    }
    __threadfence();
  }
  __syncthreads();
  return s_state != 2;
}

// All sweeps in one cooperative launch, one 1024-thread CTA per SM.
// Each sweep first stages contributions [0, hot) -- the vertices of highest
// in-degree, which a power-law graph gathers most -- into shared memory, so
// those gathers never reach the L1->L2 request path.  Warps take batches of
// kQueueBatch chunk/slice units from a global work queue (one head per sweep
// parity, reset by the barrier); the batch size is chosen so each warp makes
// about four grabs per sweep, which keeps the single queue head cold while
// the light units at the end of the queue still balance the tail.
// Zero-in-degree rows are spread over all warps in the two sweeps that need
// them.

template <int U, int U4, bool GENERIC, int MINB, typename T>
__global__ void __launch_bounds__(1024, MINB) k_pr_hot(PrArgs a) {
  extern __shared__ float4 s_hot4[];
  T *s_hot = reinterpret_cast<T *>(s_hot4);
  const int lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const long long gw = (long long)blockIdx.x * nwarps + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * nwarps;
  const Policies pol = make_policies();
  const int n_heavy = a.n_chunks + a.n_slices;
  int it = 0;
  while (it < a.max_iter) {
    const T *cin = static_cast<const T *>((it & 1) ? a.c1 : a.c0);
    T *cout = static_cast<T *>((it & 1) ? a.c0 : a.c1);
    const float4 *src = reinterpret_cast<const float4 *>(cin);
    const int n16 = (int)((size_t)a.hot * sizeof(T) / 16);
    for (int i = threadIdx.x; i < n16; i += blockDim.x) s_hot4[i] = ld_contrib4(src + i, pol.keep);
    __syncthreads();
    using Gat = typename std::conditional<GENERIC, HotGatherGeneric<T>, HotGather<T>>::type;
    const Gat gat{cin, s_hot, a.hot, pol.keep};
    double err = 0.0;
    for (;;) {
      int u0 = 0;
      if (lane == 0) u0 = atomicAdd(a.wq + (it & 1), a.batch);
      u0 = __shfl_sync(kFull, u0, 0);
      if (u0 >= n_heavy) break;
      const int u1 = min(u0 + a.batch, n_heavy);
      for (int u = u0; u < u1; ++u) {
        if (u < a.n_chunks) err += do_chunk<U4>(a, gat, cout, u, lane, pol);
        else err += do_slice<U>(a, gat, cout, u - a.n_chunks, lane, pol);
      }
    }
    if (it < 2)
      for (long long z = gw; z < a.n_zblk; z += nw) err += do_zero(a, cout, (int)z, lane, it, pol);
    const double tot = block_sum(err);
    if (!barrier_reduce(a, it, tot)) return;
    const double total = __ldcg(a.err_hist + it);
    ++it;
    if (total < a.tol) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.status[1] = it;
    a.status[2] = 1;
  }
}

// ---- blocked form (device code: gpr_blocked.cuh) ---------------------------

// All sweeps of the blocked form in one cooperative launch, MINB CTAs of NT
// threads per SM (one of 1024, or two of 512: then one CTA's warps keep
// gathering while the other's wait at the barrier that closes a tile or
// finalize its block).  Per sweep: CTAs take tiles from a queue (heaviest first; the
// next tile is claimed while the current one closes), then warps take the
// chunks of the rows above chunk_min in-edges, with the first contributions
// staged in the shared memory the accumulators used, then the zero-in-degree
// rows (sweeps 0 and 1), then the bounded grid barrier with the residual.
template <int PV, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_pr_blocked(PrArgs a) {
  extern __shared__ unsigned s_acc[];  // [2 * acc_rows]: low / high words
  __shared__ int s_tile, s_next_tile, s_last, s_next;
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * (NT / 32) + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * (NT / 32);
  const Policies pol = make_policies();
  int it = 0;
  while (it < a.max_iter) {
    const float *cin = static_cast<const float *>((it & 1) ? a.c1 : a.c0);
    float *cout = static_cast<float *>((it & 1) ? a.c0 : a.c1);
    double err = 0.0;
    if (threadIdx.x == 0) s_next_tile = atomicAdd(a.tq + (it & 1), 1);
    for (;;) {
      __syncthreads();
      if (threadIdx.x == 0) s_tile = s_next_tile;
      __syncthreads();
      const int t = s_tile;
      if (t >= a.n_tiles) break;
      err += gpr::blk::blocked_tile<PV, NT>(a, cin, cout, t, s_acc, &s_next, &s_last,
                                            &s_next_tile, a.tq + (it & 1), a.base, pol);
    }
    // chunks of the heaviest rows, the hottest contributions from shared
    // memory (none staged when the chunks are few)
    if (a.n_chunks > 0) {
      float *s_hot = reinterpret_cast<float *>(s_acc);
      const int n16 = a.hot / 4;
      const float4 *src = reinterpret_cast<const float4 *>(cin);
      for (int i = threadIdx.x; i < n16; i += blockDim.x)
        reinterpret_cast<float4 *>(s_hot)[i] = ld_contrib4(src + i, pol.keep);
      __syncthreads();
      const HotGatherGeneric<float> gat{cin, s_hot, a.hot, pol.keep};
      for (;;) {
        int u0 = 0;
        if (lane == 0) u0 = atomicAdd(a.wq + (it & 1), a.batch);
        u0 = __shfl_sync(kFull, u0, 0);
        if (u0 >= a.n_chunks) break;
        const int u1 = min(u0 + a.batch, a.n_chunks);
        for (int u = u0; u < u1; ++u) err += do_chunk<4>(a, gat, cout, u, lane, pol);
      }
    }
    if (it < 2)
      for (long long z = gw; z < a.n_zblk; z += nw) err += do_zero(a, cout, (int)z, lane, it, pol);
    const double tot = block_sum(err);
    if (!barrier_reduce(a, it, tot)) return;
    const double total = __ldcg(a.err_hist + it);
    ++it;
    if (total < a.tol) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.status[1] = it;
    a.status[2] = 1;
  }
}

// Largest |score| (bits of a non-negative float order like the float; a NaN
// sorts above every finite value and infinity).
__global__ void k_max_abs(int m, const float *__restrict__ s, unsigned *out) {
  unsigned mx = 0u;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x)
    mx = max(mx, __float_as_uint(s[i]) & 0x7FFFFFFFu);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// The blocked-form kernel with `ctas` CTAs per SM (1: 1024 threads, 2: 512).
const void *blocked_kernel(int ctas) {
  return ctas == 2 ? (const void *)k_pr_blocked<4, 512, 2> : (const void *)k_pr_blocked<4, 1024, 1>;
}

// One sweep per launch (graph mode).  The sweep index and the done flag live
// in device memory, so a captured sequence of launches needs no host input;
// launches after convergence return at once.
// In graph mode the launch is the body of a CUDA-graph while node whose
// condition starts at 1 and is only ever cleared: by the CTA that closes the
// sweep when the solve is done, by a launch that finds the solve done, and by
// CTA 0 of the max_iter-th launch (status[3] counts launches), so the loop
// ends within max_iter launches whatever the sweeps compute.
template <int U, int U4, typename T>
__global__ void __launch_bounds__(gpr::kBlock) k_pr_step(PrArgs a) {
  __shared__ int s_it, s_last;
  if (threadIdx.x == 0) {
    const int done = *(volatile int *)(a.status + 2);
    s_it = done ? -1 : *(volatile int *)(a.status + 1);
    if (a.cond && blockIdx.x == 0) {
      const int n = atomicAdd(a.status + 3, 1) + 1;
      if (done || n >= a.max_iter) cudaGraphSetConditional(a.cond, 0u);
    }
  }
  __syncthreads();
  const int it = s_it;
  if (it < 0) return;
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const Policies pol = make_policies();
  const T *cin = static_cast<const T *>((it & 1) ? a.c1 : a.c0);
  T *cout = static_cast<T *>((it & 1) ? a.c0 : a.c1);
  const double err = sweep<U, U4, T>(a, cin, cout, gw, nw, lane, it, pol);
  const double tot = block_sum(err);
  if (threadIdx.x == 0) {
    a.cta_err[blockIdx.x] = tot;
    __threadfence();
    s_last = atomicAdd(a.bar, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x < 32) {
    __threadfence();
    double t = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += 32) t += __ldcg(a.cta_err + i);
    t = warp_sum(t);
    if (threadIdx.x == 0) {
      a.err_hist[it] = t;
      atomicExch(a.bar, 0u);
      a.status[1] = it + 1;
      const bool done = t < a.tol || it + 1 >= a.max_iter;
      if (done) a.status[2] = 1;
      __threadfence();
      if (a.cond && done) cudaGraphSetConditional(a.cond, 0u);
    }
  }
}

// Scores into the relabelled order and the first sweep's contributions.
template <typename T>
__global__ void k_pr_prologue(int m, const int *__restrict__ perm, const int *__restrict__ outdeg,
                              const float *__restrict__ scores_in, float *s, T *c0, T *c1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    const float v = scores_in[perm[i]];
    s[i] = v;
    c0[i] = (T)__fdiv_rn(v, __int2float_rn(outdeg[i]));
  } else if (i == m) {
    c0[m] = (T)0.f;  // sentinel slots of the padding entries
    c1[m] = (T)0.f;
  }
}

__global__ void k_pr_scatter(int m, const int *__restrict__ perm, const float *__restrict__ s,
                             float *scores_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) scores_out[perm[i]] = s[i];
}

// ---- FP64 residual (a-posteriori bound) ------------------------------------
__global__ void k_res_prologue(int m, const int *__restrict__ perm, const int *__restrict__ outdeg,
                               const float *__restrict__ scores, double *cd, double *sd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    const double v = (double)scores[perm[i]];
    sd[i] = v;
    cd[i] = v / (double)outdeg[i];
  } else if (i == m) {
    cd[m] = 0.0;
  }
}

__global__ void k_res_sweep(PrArgs a, const double *__restrict__ cd, const double *__restrict__ sd,
                            double d, double base, double *long_acc, double *out) {
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long u1 = a.n_chunks, u2 = u1 + a.n_slices, u3 = u2 + a.n_zblk;
  double err = 0.0;
  for (long long u = gw; u < u3; u += nw) {
    if (u < u1) {
      const int c = (int)u, r = a.chunk_row[c];
      const int cb = a.row_cbeg[r];
      const long long b = a.long_ptr[r] + (long long)(c - cb) * a.chunk;
      const long long e = min(b + (long long)a.chunk, a.long_ptr[r + 1]);
      double acc = 0.0;
      for (long long k = b + lane; k < e; k += 32) acc += cd[a.long_col[k]];
      acc = warp_sum(acc);
      if (lane == 0) atomicAdd(long_acc + r, acc);
    } else if (u < u2) {
      const int sidx = (int)(u - u1);
      const int c = gpr::slice_class(a.cls, sidx);
      const int lw = a.cls.lw[c];
      const int r = a.cls.row[c] + ((sidx - a.cls.slice[c]) << (5 - lw)) + (lane >> lw);
      const long long b = a.slice_ptr[sidx];
      const int len = (int)((a.slice_ptr[sidx + 1] - b) >> 5);
      double acc = 0.0;
      for (int j = 0; j < len; ++j) acc += cd[a.sell_col[b + 32LL * j + lane]];
      for (int o = (1 << lw) >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
      if (r < a.cls.row[c + 1] && (lane & ((1 << lw) - 1)) == 0) err += fabs(base + d * acc - sd[r]);
    } else {
      const int r0 = a.n_nz + (int)(u - u2) * gpr::kZeroRowsPerUnit;
      for (int q = 0; q < gpr::kZeroRowsPerUnit / 32; ++q) {
        const int r = r0 + 32 * q + lane;
        if (r < a.m) err += fabs(base - sd[r]);
      }
    }
  }
  err = warp_sum(err);
  if (lane == 0) atomicAdd(out, err);
}

__global__ void k_res_long(int n_long, const double *__restrict__ long_acc,
                           const double *__restrict__ sd, double d, double base, double *out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (r < n_long) e = fabs(base + d * long_acc[r] - sd[r]);
  e = warp_sum(e);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, e);
}

inline unsigned grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  return (unsigned)(g < 1 ? 1 : g);
}

// Variants of the sweep kernels: (slice batch U, int4 loads per lane U4,
// one generic load per gather or shared + predicated global, CTAs per SM).
// Variant 0 is the default; the others are the autotuner's choices.
struct SweepKernels {
  const void *persistent;
  void (*step)(PrArgs);
  int ctas_per_sm;  // persistent kernel: co-resident 1024-thread CTAs per SM
  int hot_bytes;    // most shared memory one CTA stages
  int elem;         // bytes per contribution: 4 (FP32) or 2 (BF16)
};
using bf16 = __nv_bfloat16;
// Indices 0..7: the FP32 variants a caller selects with opts.variant;
// index kBf16Kernel: the BF16-contribution kernel of the mixed form.
const SweepKernels kKernels[] = {
    {(const void *)k_pr_hot<16, 4, true, 1, float>, k_pr_step<16, 4, float>, 1, 227328, 4},
    {(const void *)k_pr_hot<8, 2, false, 1, float>, k_pr_step<8, 2, float>, 1, 227328, 4},
    {(const void *)k_pr_hot<4, 2, false, 1, float>, k_pr_step<4, 2, float>, 1, 227328, 4},
    {(const void *)k_pr_hot<32, 8, false, 1, float>, k_pr_step<32, 8, float>, 1, 227328, 4},
    {(const void *)k_pr_hot<16, 4, false, 1, float>, k_pr_step<16, 4, float>, 1, 227328, 4},
    {(const void *)k_pr_hot<8, 2, true, 1, float>, k_pr_step<8, 2, float>, 1, 227328, 4},
    {(const void *)k_pr_hot<8, 2, false, 2, float>, k_pr_step<8, 2, float>, 2, 98304, 4},
    {(const void *)k_pr_hot<8, 2, true, 2, float>, k_pr_step<8, 2, float>, 2, 98304, 4},
    {(const void *)k_pr_hot<16, 4, true, 1, bf16>, k_pr_step<16, 4, bf16>, 1, 227328, 2},
};
constexpr int kHotBlock = 1024;
constexpr int kNumVariants = 8;
constexpr int kBf16Kernel = 8;
constexpr int kNumKernels = sizeof(kKernels) / sizeof(kKernels[0]);
// The BF16 phase of the mixed form stops once the L1 change is below this
// (or the caller's tol if larger): about where BF16 rounding of the
// contributions stops the residual from falling further.
constexpr double kBf16Tol = 1e-3;

// Contributions kernel ki stages in shared memory: the caller's hot budget in
// bytes, covering the sentinel slot m when the whole array fits, a multiple
// of 16 bytes.
int hot_entries(const gpr_graph *g, int ki) {
  const int elem = kKernels[ki].elem, per16 = 16 / elem;
  long long n = std::min<long long>((long long)g->hot_bytes, kKernels[ki].hot_bytes) / elem;
  const long long all = ((long long)g->L.m + 1 + per16 - 1) / per16 * per16;
  n = std::min(n, all);
  return (int)(n / per16 * per16);
}

PrArgs make_args(gpr_graph *g, const gpr_pr_opts &o, int ki) {
  const PrLayout &L = g->L;
  PrArgs a;
  memset(&a, 0, sizeof(a));  // padding too: cached graphs compare the bytes
  a.m = L.m;
  a.n_long = L.n_long;
  a.n_nz = L.n_nz;
  a.n_chunks = L.n_chunks;
  a.n_slices = L.n_slices;
  a.n_zblk = L.n_zblk;
  a.chunk = L.chunk;
  a.cls = L.cls;
  a.long_ptr = L.long_ptr;
  a.long_col = L.long_col;
  a.row_cbeg = L.row_cbeg;
  a.chunk_row = L.chunk_row;
  a.slice_ptr = L.slice_ptr;
  a.sell_col = L.sell_col;
  a.outdeg = L.outdeg;
  a.s = g->s;
  a.c0 = kKernels[ki].elem == 2 ? (void *)g->h0 : (void *)g->c0;
  a.c1 = kKernels[ki].elem == 2 ? (void *)g->h1 : (void *)g->c1;
  a.partial = g->partial;
  a.cnt = g->cnt;
  a.cta_err = g->cta_err;
  a.err_hist = g->err_hist;
  a.bar = g->bar;
  a.status = g->status;
  a.damp = o.damping;
  a.base = (1.0f - o.damping) / (float)L.m;  // src/pr/omp_base.cc:16
  a.tol = o.tol;
  a.max_iter = o.max_iter;
  a.bar_expect = g->grid_hot[ki];
  a.hot = hot_entries(g, ki);
  a.wq = g->wq;
  {
    const long long heavy = (long long)L.n_chunks + L.n_slices;
    const long long warps = (long long)g->grid_hot[ki] * (kHotBlock / 32);
    a.batch = (int)std::max<long long>(1, heavy / (warps * 4));
  }
  a.timeout_ns = (long long)(o.timeout_s * 1e9);
  return a;
}

void drop_loop_graph(gpr_graph *g);

void destroy(gpr_graph *g) {
  if (!g) return;
  drop_loop_graph(g);
  gpr::free_pr_layout(&g->L);
  gpr::dfree(g->s);
  gpr::dfree(g->c0);
  gpr::dfree(g->c1);
  gpr::dfree(g->h0);
  gpr::dfree(g->h1);
  gpr::dfree(g->partial);
  gpr::dfree(g->cnt);
  gpr::dfree(g->cta_err);
  gpr::dfree(g->err_hist);
  gpr::dfree(g->bar);
  gpr::dfree(g->status);
  gpr::dfree(g->scores_tmp);
  gpr::dfree(g->res_tmp);
  gpr::dfree(g->wq);
  gpr::dfree(g->b_cbeg);
  gpr::dfree(g->b_crow);
  gpr::dfree(g->b_cdesc);
  gpr::dfree(g->b_pk);
  for (int i = 0; i < 6; ++i) gpr::dfree(g->b_pkr[i]);
  gpr::dfree(g->push_src);
  gpr::dfree(g->push_dst);
  gpr::dfree(g->push_sum);
  gpr::free_blocked_layout(&g->B);
  gpr::dfree(g->tq);
  gpr::dfree(g->fx_max);
  if (g->e0) cudaEventDestroy(g->e0);
  if (g->e1) cudaEventDestroy(g->e1);
  if (g->e2) cudaEventDestroy(g->e2);
  if (g->e3) cudaEventDestroy(g->e3);
  if (g->own_stream && g->st) cudaStreamDestroy(g->st);
  delete g;
}

int create_impl(int m, long long nnz, const int *any_rowptr, const int *any_col,
                const int *any_outdeg, int lane_max, int chunk_min, int chunk, int hot_max,
                bool keep_csr, bool blocked, int block_rows, int tile_words, int blocked_long,
                gpr_graph *g) {
  GPR_CUDA(cudaGetDevice(&g->device));
  GPR_CUDA(cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking));
  g->own_stream = true;
  GPR_CUDA(cudaEventCreate(&g->e0));
  GPR_CUDA(cudaEventCreate(&g->e1));
  GPR_CUDA(cudaEventCreate(&g->e2));
  GPR_CUDA(cudaEventCreate(&g->e3));
  cudaStream_t st = g->st;
  void *rp = nullptr, *cp = nullptr, *dp = nullptr;
  bool orp = false, ocp = false, odp = false;
  int rc = GPR_OK;
  {
    // No device-wide synchronisation (a free) while the column copy runs.
    gpr::DeferFrees defer;
    rc = gpr::to_device(any_rowptr, sizeof(int) * ((size_t)m + 1), &rp, &orp, st, "rowptr");
    if (rc == GPR_OK)
      rc = gpr::to_device(any_outdeg, sizeof(int) * (size_t)m, &dp, &odp, st, "outdeg");
    // Column indices in host memory (the largest copy) go on a second stream
    // after the row offsets and out-degrees, so that the layout's degree work
    // runs while they arrive; the build waits for them before reading columns.
    const bool host_col = nnz > 0 && any_col && !gpr::is_device_ptr(any_col);
    cudaStream_t cs = nullptr;
    cudaEvent_t ev_rows = nullptr, ev_col = nullptr;
    if (rc == GPR_OK && host_col) {
      const size_t bytes = sizeof(int) * (size_t)nnz;
      rc = gpr::dmalloc(&cp, bytes, "col");
      ocp = rc == GPR_OK;
      if (rc == GPR_OK) {
        cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_rows, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_col, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev_rows, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ev_rows, 0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(cp, any_col, bytes, cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) e = cudaEventRecord(ev_col, cs);
        if (e != cudaSuccess) {
          gpr::set_error("copy of col to the device: %s", cudaGetErrorString(e));
          rc = GPR_ECUDA;
        }
      }
    } else if (rc == GPR_OK) {
      rc = gpr::to_device(any_col, sizeof(int) * (size_t)nnz, &cp, &ocp, st, "col");
    }
    if (rc == GPR_OK)
      rc = gpr::validate_csr(m, nnz, m, (const int *)rp, host_col ? nullptr : (const int *)cp,
                             (const int *)dp, st);
    if (rc == GPR_OK)
      rc = gpr::build_pr_layout(m, nnz, (const int *)rp, (const int *)cp, (const int *)dp,
                                lane_max, chunk_min, chunk, keep_csr, &g->L, st,
                                host_col ? ev_col : nullptr);
    cudaStreamSynchronize(st);
    if (cs) {
      cudaStreamSynchronize(cs);  // the column copy is done before its buffer is freed
      cudaStreamDestroy(cs);
    }
    if (ev_rows) cudaEventDestroy(ev_rows);
    if (ev_col) cudaEventDestroy(ev_col);
  }
  if (rc == GPR_OK && blocked) {
    // Default rows per block: about two blocks per SM.  Default tile size:
    // whole blocks up to 1M words (a multi-tile block adds one 8-byte atomic
    // per row and tile); the builder halves the tiles that would end the
    // sweep late.
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, g->device);
    if (block_rows == 0)
      block_rows = (int)std::min<long long>(
          gpr::kBlockedRows,
          std::max<long long>(256, gpr::ceil_div((long long)g->L.n_nz, 2LL * nsm)));
    int row0 = 0, n_chunks = 0;
    rc = gpr::blocked_split(g->L, (const int *)rp,
                            blocked_long > 0 ? std::max(blocked_long, chunk_min) : 0, block_rows,
                            &row0, &n_chunks, st);
    if (tile_words == 0) tile_words = gpr::kTileWordsDefault;
    if (rc == GPR_OK)
      rc = gpr::build_blocked_layout(m, nnz, (const int *)rp, (const int *)cp, g->L, row0,
                                     n_chunks, block_rows, tile_words, gpr::kRunWords,
                                     nsm * gpr::blocked_ctas_per_sm(block_rows), &g->B, st);
    g->has_blocked = rc == GPR_OK;
  }
  if (orp) gpr::dfree(rp);
  if (ocp) gpr::dfree(cp);
  if (odp) gpr::dfree(dp);
  GPR_TRY(rc);
  const PrLayout &L = g->L;
  GPR_TRY(gpr::dalloc(&g->s, (size_t)m, "scores"));
  // Hot prefix budget in bytes (FP32: hot_max entries).  Contribution
  // buffers are padded so the staging loads stay in bounds; padding stays 0.
  g->hot_bytes = 4 * hot_max;
  g->hot = hot_entries(g, 0);
  const size_t cn = (size_t)std::max<long long>((long long)m + 1, g->hot) + 4;
  GPR_TRY(gpr::dalloc(&g->c0, cn, "contrib0"));
  GPR_TRY(gpr::dalloc(&g->c1, cn, "contrib1"));
  GPR_CUDA(cudaMemsetAsync(g->c0, 0, sizeof(float) * cn, st));
  GPR_CUDA(cudaMemsetAsync(g->c1, 0, sizeof(float) * cn, st));
  GPR_TRY(gpr::dalloc(&g->partial, (size_t)L.n_chunks, "chunk partials"));
  GPR_TRY(gpr::dalloc(&g->cnt, (size_t)L.n_long, "chunk counters"));
  GPR_TRY(gpr::dalloc(&g->bar, 4, "barrier"));
  GPR_TRY(gpr::dalloc(&g->status, 4, "status"));
  GPR_TRY(gpr::dalloc(&g->scores_tmp, (size_t)m, "score staging"));
  GPR_CUDA(cudaMemsetAsync(g->cnt, 0, sizeof(int) * (L.n_long ? L.n_long : 1), st));

  int sms = 0, coop = 0;
  GPR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  GPR_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device));
  const long long units = (long long)L.n_chunks + L.n_slices + L.n_zblk;
  const long long warps_per_cta = gpr::kBlock / 32;
  const long long need = gpr::ceil_div(units, warps_per_cta);
  g->coop = coop != 0;
  g->hot_ok = g->coop;
  const long long heavy = (long long)L.n_chunks + L.n_slices;
  for (int v = 0; v < kNumKernels; ++v) {
    int per_sm = 0;
    const size_t smem = (size_t)hot_entries(g, v) * kKernels[v].elem;
    GPR_CUDA(cudaFuncSetAttribute(kKernels[v].persistent,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    GPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kKernels[v].persistent,
                                                           kHotBlock, smem));
    if (per_sm < kKernels[v].ctas_per_sm) g->hot_ok = false;
    g->grid_hot[v] = (int)std::max<long long>(
        1, std::min<long long>((long long)sms * kKernels[v].ctas_per_sm, gpr::ceil_div(heavy, 32)));
  }
  GPR_TRY(gpr::dalloc(&g->wq, 2, "work queue"));
  long long step = need < 1 ? 1 : need;
  if (step > (long long)sms * 32) step = (long long)sms * 32;
  g->grid_step = (int)step;
  g->max_grid = g->grid_step;
  for (int v = 0; v < kNumKernels; ++v) g->max_grid = std::max(g->max_grid, g->grid_hot[v]);
  if (g->has_blocked) {
    int smem_sm = 0;
    GPR_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                    g->device));
    // Two 512-thread CTAs per SM (one gathers while the other closes a tile)
    // when both fit beside an L1 of about half the SM's 256 KB, else one
    // 1024-thread CTA: the gathers' L1 line hits are worth more than the
    // overlap (RMAT scale 24 with 12288-row blocks: 2x slower sweeps with
    // two CTAs and a 28 KB L1).
    g->blocked_ctas = gpr::blocked_ctas_per_sm(g->B.R);
    int per_sm = 0;
    for (;;) {
      // the smallest shared-memory carveout that holds the CTAs: the rest of
      // the SM's 256 KB stays L1
      const void *k = blocked_kernel(g->blocked_ctas);
      const int smem = 8 * g->B.R;
      cudaFuncAttributes fa;
      GPR_CUDA(cudaFuncGetAttributes(&fa, k));
      const long long need = (long long)g->blocked_ctas * (smem + (long long)fa.sharedSizeBytes + 1024);
      const int carve = (int)std::min<long long>(100, gpr::ceil_div(100 * need, smem_sm));
      GPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      GPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
      GPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, k, 1024 / g->blocked_ctas, smem));
      if (per_sm >= g->blocked_ctas || g->blocked_ctas == 1) break;
      g->blocked_ctas = 1;
    }
    g->blocked_ok = g->coop && per_sm >= g->blocked_ctas;
    g->grid_blocked = sms * g->blocked_ctas;
    g->max_grid = std::max(g->max_grid, g->grid_blocked);
    GPR_TRY(gpr::dalloc(&g->tq, 2, "tile queue"));
    GPR_TRY(gpr::dalloc(&g->fx_max, 1, "largest score"));
  }
  GPR_TRY(gpr::dalloc(&g->cta_err, 2 * (size_t)g->max_grid, "cta residuals"));
  g->err_cap = 128;
  GPR_TRY(gpr::dalloc(&g->err_hist, (size_t)g->err_cap, "residual history"));
  GPR_CUDA(cudaStreamSynchronize(st));
  return GPR_OK;
}

// Graph mode: the sweep loop as one CUDA graph -- a while node whose body is
// one k_pr_step launch; the kernel clears the condition when the solve is
// done.  The instantiated graph is kept and reused while the kernel and its
// arguments are unchanged.
void drop_loop_graph(gpr_graph *g) {
  if (g->loop_exec) cudaGraphExecDestroy(g->loop_exec);
  if (g->loop_graph) cudaGraphDestroy(g->loop_graph);
  g->loop_exec = nullptr;
  g->loop_graph = nullptr;
  g->loop_ki = -1;
}

int graph_loop(gpr_graph *g, const PrArgs &a, int ki, cudaStream_t st) {
  static_assert(sizeof(PrArgs) <= sizeof(g->loop_args), "loop_args too small");
  if (!g->loop_exec || g->loop_ki != ki || memcmp(g->loop_args, &a, sizeof(PrArgs)) != 0) {
    drop_loop_graph(g);
    cudaGraph_t graph = nullptr;
    GPR_CUDA(cudaGraphCreate(&graph, 0));
    g->loop_graph = graph;
    cudaGraphConditionalHandle h;
    GPR_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cn;
    GPR_CUDA(cudaGraphAddNode(&cn, graph, nullptr, 0, &cp));
    PrArgs ac = a;
    ac.cond = h;
    void *kargs[] = {&ac};
    cudaKernelNodeParams kp;
    memset(&kp, 0, sizeof(kp));
    kp.func = (void *)kKernels[ki].step;
    kp.gridDim = dim3(g->grid_step);
    kp.blockDim = dim3(gpr::kBlock);
    kp.kernelParams = kargs;
    cudaGraphNode_t kn;
    GPR_CUDA(cudaGraphAddKernelNode(&kn, cp.conditional.phGraph_out[0], nullptr, 0, &kp));
    GPR_CUDA(cudaGraphInstantiate(&g->loop_exec, graph, 0));
    g->loop_ki = ki;
    memcpy(g->loop_args, &a, sizeof(PrArgs));
  }
  GPR_CUDA(cudaGraphLaunch(g->loop_exec, st));
  return GPR_OK;
}

// solve_impl status: the blocked form cannot represent these scores (a
// non-finite score); the caller solves with the exact-order form instead.
constexpr int kBlockedFallback = 100;

// Fixed-point exponent S of the blocked form for a solve from scores whose
// largest magnitude is mx.  Every sweep's total |score| is at most
// B0 = max(1, m * mx) (a sweep maps total mass M to at most (1-d) + d*M), and
// a row's sum is at most that, so |sum| * 2^S < 2^63 needs S <= 62 - log2(B0).
// Within that, S puts a typical contribution (about B0 / nnz) near 2^28, so
// most fit the low 32-bit word of the accumulator; S >= 31 unless B0 > 2^31.
int blocked_shift(int m, long long nnz, float mx) {
  const double b0 = std::max(1.0, (double)m * (double)mx);
  const int cap = 62 - (int)ceil(log2(b0));
  const int pref = (int)floor(log2(std::max(1.0, (double)nnz) / b0)) + 28;
  return std::min(cap, std::max(31, pref));
}

// One solve with sweep kernel ki (or, when `blocked`, the blocked form) from
// the scores in d_scores (device, vertex order); the result is written back
// to d_scores.
int solve_impl(gpr_graph *g, float *d_scores, const gpr_pr_opts &o, int ki, gpr_pr_stats *out,
               bool blocked = false) {
  const int m = g->L.m;
  cudaStream_t st = g->st;
  if (kKernels[ki].elem == 2 && !g->h0) {
    const size_t cnh = (size_t)std::max<long long>((long long)m + 1, hot_entries(g, ki)) + 8;
    GPR_TRY(gpr::dalloc(reinterpret_cast<bf16 **>(&g->h0), cnh, "bf16 contrib0"));
    GPR_TRY(gpr::dalloc(reinterpret_cast<bf16 **>(&g->h1), cnh, "bf16 contrib1"));
    GPR_CUDA(cudaMemsetAsync(g->h0, 0, 2 * cnh, st));
    GPR_CUDA(cudaMemsetAsync(g->h1, 0, 2 * cnh, st));
  }
  GPR_CUDA(cudaMemsetAsync(g->bar, 0, 4 * sizeof(unsigned), st));
  GPR_CUDA(cudaMemsetAsync(g->status, 0, 4 * sizeof(int), st));
  GPR_CUDA(cudaMemsetAsync(g->wq, 0, 2 * sizeof(int), st));
  if (g->L.n_long) GPR_CUDA(cudaMemsetAsync(g->cnt, 0, sizeof(int) * g->L.n_long, st));
  const gpr::BlockedLayout &B = g->B;
  if (blocked) {
    GPR_CUDA(cudaMemsetAsync(g->tq, 0, 2 * sizeof(int), st));
    GPR_CUDA(cudaMemsetAsync(g->fx_max, 0, sizeof(unsigned), st));
    if (B.n_blocks) {
      // clean after an abandoned solve; a completed sweep leaves them clean
      GPR_CUDA(cudaMemsetAsync(B.bcnt, 0, sizeof(int) * B.n_blocks, st));
      GPR_CUDA(cudaMemsetAsync(B.gacc, 0, 8 * (size_t)B.gacc_rows, st));
    }
  }
  PrArgs a = make_args(g, o, ki);
  if (blocked) {
    a.n_tiles = B.n_tiles;
    a.tiles = B.tiles;
    a.blocks = B.blocks;
    a.runs = B.runs;
    a.entry = B.entry;
    a.gacc = B.gacc;
    a.bcnt = B.bcnt;
    a.tq = g->tq;
    a.bar_expect = g->grid_blocked;
    a.acc_rows = B.R;
    a.blk_row0 = B.row0;
    a.n_chunks = B.n_chunks;
    // stage the hottest contributions only when every warp has chunks to take
    const long long warps = (long long)g->grid_blocked * (32 / g->blocked_ctas);
    a.hot = B.n_chunks >= 4 * warps ? std::min(hot_entries(g, 0), 2 * B.R) / 4 * 4 : 0;
    a.batch = (int)std::max<long long>(1, (long long)B.n_chunks / (warps * 4));
  }
  if (o.reserved[0] > 0) a.bar_expect += o.reserved[0];  // test hook: a barrier nobody completes
  int launches = 0;
  bool graph_mode = false;
  GPR_CUDA(cudaEventRecord(g->e0, st));
  if (kKernels[ki].elem == 2)
    k_pr_prologue<bf16><<<grid_for((long long)m + 1), 256, 0, st>>>(
        m, g->L.perm, g->L.outdeg, d_scores, g->s, static_cast<bf16 *>(g->h0),
        static_cast<bf16 *>(g->h1));
  else
    k_pr_prologue<float><<<grid_for((long long)m + 1), 256, 0, st>>>(
        m, g->L.perm, g->L.outdeg, d_scores, g->s, g->c0, g->c1);
  ++launches;
  if (blocked) {
    k_max_abs<<<std::min<unsigned>(grid_for(m), 148 * 8), 256, 0, st>>>(m, g->s, g->fx_max);
    ++launches;
    GPR_CUDA(cudaGetLastError());
    unsigned bits = 0;
    GPR_CUDA(cudaMemcpyAsync(&bits, g->fx_max, sizeof(bits), cudaMemcpyDeviceToHost, st));
    GPR_CUDA(cudaStreamSynchronize(st));
    float mx;
    memcpy(&mx, &bits, sizeof(mx));
    if (!isfinite(mx)) return kBlockedFallback;
    const int S = blocked_shift(m, g->L.nnz, mx);
    a.fx_scale = ldexpf(1.f, S);
    a.fx_inv = ldexp(1.0, -S);
  }
  int loop = o.loop;
  if (loop == GPR_LOOP_AUTO) loop = GPR_LOOP_PERSISTENT;
  if (loop == GPR_LOOP_PERSISTENT && !g->hot_ok) loop = GPR_LOOP_GRAPH;
  GPR_CUDA(cudaEventRecord(g->e2, st));
  if (o.max_iter > 0 && blocked) {
    void *args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel(blocked_kernel(g->blocked_ctas),
                                                dim3(g->grid_blocked),
                                                dim3(1024 / g->blocked_ctas), args,
                                                8 * (size_t)B.R, st);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
      cudaGetLastError();
      return kBlockedFallback;
    }
    if (e != cudaSuccess) {
      gpr::set_error("cooperative launch: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
    ++launches;
  } else if (o.max_iter > 0) {
    if (loop == GPR_LOOP_PERSISTENT) {
      void *args[] = {&a};
      cudaError_t e = cudaLaunchCooperativeKernel(kKernels[ki].persistent, dim3(g->grid_hot[ki]),
                                                  dim3(kHotBlock), args,
                                                  (size_t)a.hot * kKernels[ki].elem, st);
      if (e == cudaErrorCooperativeLaunchTooLarge) {
        cudaGetLastError();
        loop = GPR_LOOP_GRAPH;
      } else if (e != cudaSuccess) {
        gpr::set_error("cooperative launch: %s", cudaGetErrorString(e));
        return GPR_ECUDA;
      } else {
        ++launches;
      }
    }
    if (loop == GPR_LOOP_GRAPH) {
      GPR_TRY(graph_loop(g, a, ki, st));
      graph_mode = true;
    }
  }
  GPR_CUDA(cudaEventRecord(g->e3, st));
  k_pr_scatter<<<grid_for(m), 256, 0, st>>>(m, g->L.perm, g->s, d_scores);
  ++launches;
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaEventRecord(g->e1, st));
  int hs[4];
  GPR_CUDA(cudaMemcpyAsync(hs, g->status, sizeof(hs), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f, lms = 0.f;
  GPR_CUDA(cudaEventElapsedTime(&ms, g->e0, g->e1));
  GPR_CUDA(cudaEventElapsedTime(&lms, g->e2, g->e3));
  memset(out, 0, sizeof(*out));
  out->loop_ms = lms;
  out->iterations = hs[1];
  g->last_sweeps = hs[1];
  out->solve_ms = ms;
  out->gpu_launches = launches + (graph_mode ? hs[1] : 0);
  if (hs[1] > 0)
    GPR_CUDA(cudaMemcpy(&out->residual, g->err_hist + hs[1] - 1, sizeof(double),
                        cudaMemcpyDeviceToHost));
  if (hs[0] & 1) {
    gpr::set_error("grid barrier wait exceeded %.3f s (sweep loop abandoned)", o.timeout_s);
    return GPR_ETIMEOUT;
  }
  return GPR_OK;
}

int pagerank_impl(gpr_graph *g, float *any_scores, const gpr_pr_opts *opts_in,
                  gpr_pr_stats *stats) {
  gpr_pr_opts o;
  if (opts_in) o = *opts_in;
  else gpr_pr_opts_default(&o);
  if (!(o.damping >= 0.f && o.damping <= 1.f) || o.max_iter < 0 || !(o.tol >= 0.0) ||
      !(o.timeout_s > 0.0) || o.variant < 0 || o.variant >= kNumVariants ||
      o.form < GPR_FORM_AUTO || o.form > GPR_FORM_BLOCKED) {
    gpr::set_error("gpr_pagerank: invalid options (damping %g, tol %g, max_iter %d, timeout %g, "
                   "variant %d, form %d)", (double)o.damping, o.tol, o.max_iter, o.timeout_s,
                   o.variant, o.form);
    return GPR_EINVAL;
  }
  if (o.form == GPR_FORM_BLOCKED) {
    if (!g->has_blocked) {
      gpr::set_error("gpr_pagerank: GPR_FORM_BLOCKED on a graph created without "
                     "GPR_LAYOUT_BLOCKED");
      return GPR_EINVAL;
    }
    if (o.precision != GPR_PREC_FP32 || o.loop == GPR_LOOP_GRAPH || !g->blocked_ok) {
      gpr::set_error("gpr_pagerank: GPR_FORM_BLOCKED needs GPR_PREC_FP32 and the persistent "
                     "loop (cooperative launch of one CTA per SM)");
      return GPR_EUNSUPPORTED;
    }
  }
  if (o.precision != GPR_PREC_FP32 && o.precision != GPR_PREC_BF16) {
    gpr::set_error("gpr_pagerank: precision %d not supported (GPR_PREC_FP32 or GPR_PREC_BF16)",
                   o.precision);
    return GPR_EUNSUPPORTED;
  }
  const int m = g->L.m;
  gpr_pr_stats st_local;
  memset(&st_local, 0, sizeof(st_local));
  if (m == 0 || any_scores == nullptr) {
    if (m != 0) {
      if (stats) *stats = st_local;
      gpr::set_error("gpr_pagerank: NULL scores");
      return GPR_EINVAL;
    }
    // no vertices: the sweeps are empty and their residuals 0
    st_local.iterations = gpr::empty_graph_sweeps(o.tol, o.max_iter);
    g->last_sweeps = st_local.iterations;
    if (stats) *stats = st_local;
    return GPR_OK;
  }
  cudaStream_t st = g->st;
  if (o.max_iter > g->err_cap) {
    gpr::dfree(g->err_hist);
    g->err_hist = nullptr;
    g->err_cap = o.max_iter;
    GPR_TRY(gpr::dalloc(&g->err_hist, (size_t)g->err_cap, "residual history"));
  }
  float *d_scores = any_scores;
  const bool host = !gpr::is_device_ptr(any_scores);
  if (host) {
    d_scores = g->scores_tmp;
    GPR_CUDA(cudaMemcpyAsync(d_scores, any_scores, sizeof(float) * (size_t)m,
                             cudaMemcpyHostToDevice, st));
  }
  int rc = GPR_OK;
  const bool use_blocked =
      o.precision == GPR_PREC_FP32 && g->has_blocked && g->blocked_ok &&
      o.loop != GPR_LOOP_GRAPH && o.form != GPR_FORM_EXACT &&
      (o.form == GPR_FORM_BLOCKED || g->L.nnz >= gpr::kBlockedAutoMinEdges);
  if (use_blocked) {
    rc = solve_impl(g, d_scores, o, 0, &st_local, true);
    if (rc == kBlockedFallback) {
      if (o.form == GPR_FORM_BLOCKED) {
        gpr::set_error("gpr_pagerank: GPR_FORM_BLOCKED needs finite scores and a "
                       "co-resident grid");
        rc = GPR_EINVAL;
      } else {
        rc = solve_impl(g, d_scores, o, o.variant, &st_local);
      }
    }
  } else if (o.precision == GPR_PREC_FP32) {
    rc = solve_impl(g, d_scores, o, o.variant, &st_local);
  } else {
    // Mixed form: BF16 contributions (twice the entries in the shared-memory
    // cache, half the bytes per gather) until the change is below
    // max(tol, kBf16Tol), then plain FP32 sweeps from those scores to tol.
    gpr_pr_opts o1 = o;
    o1.tol = std::max(o.tol, kBf16Tol);
    gpr_pr_stats s1, s2;
    rc = solve_impl(g, d_scores, o1, kBf16Kernel, &s1);
    if (rc == GPR_OK) {
      gpr_pr_opts o2 = o;
      o2.max_iter = std::max(0, o.max_iter - s1.iterations);
      rc = solve_impl(g, d_scores, o2, o.variant, &s2);
      st_local = s2;
      st_local.iterations = s1.iterations + s2.iterations;
      st_local.refine_iterations = s2.iterations;
      st_local.solve_ms = s1.solve_ms + s2.solve_ms;
      st_local.loop_ms = s1.loop_ms + s2.loop_ms;
      st_local.gpu_launches = s1.gpu_launches + s2.gpu_launches;
      if (s2.iterations == 0) st_local.residual = s1.residual;
    }
  }
  if (host && rc == GPR_OK)
    GPR_CUDA(cudaMemcpy(any_scores, d_scores, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost));
  if (stats) *stats = st_local;
  return rc;
}

}  // namespace

extern "C" {

int gpr_graph_create(int m, long long nnz, const int *any_rowptr, const int *any_col,
                     const int *any_outdeg, gpr_graph **out) {
  return gpr_graph_create_ex(m, nnz, any_rowptr, any_col, any_outdeg, nullptr, out);
}

int gpr_graph_create_ex(int m, long long nnz, const int *any_rowptr, const int *any_col,
                        const int *any_outdeg, const gpr_layout_opts *lopts, gpr_graph **out) {
  GPR_ENTRY_BEGIN
  int lane_max = gpr::kSellMaxDefault, chunk = gpr::kChunkDefault,
      chunk_min = gpr::kChunkMinDefault, hot_max = gpr::kHotDefault;
  if (lopts && lopts->sell_max) lane_max = lopts->sell_max;
  if (lopts && lopts->chunk) chunk = lopts->chunk;
  if (lopts && lopts->chunk_min) chunk_min = lopts->chunk_min;
  if (lopts && lopts->hot_entries) hot_max = lopts->hot_entries;
  int block_rows = 0, tile_words = 0;  // 0: sized to the graph at creation
  int blocked_long = 0;  // 0: rows that would crowd a block are chunked
  if (lopts) block_rows = lopts->block_rows;
  if (lopts) tile_words = lopts->tile_words;
  if (lopts && lopts->blocked_long) blocked_long = lopts->blocked_long;
  if (lane_max < 1 || lane_max > 1024 || chunk < 128 || chunk % 128 != 0 || chunk_min < 1 ||
      hot_max < 4 || hot_max > gpr::kHotMax || hot_max % 4 != 0 || block_rows < 0 ||
      block_rows > gpr::kBlockedMaxRows || tile_words < 0 ||
      (tile_words > 0 && tile_words < gpr::kRunWords) || blocked_long < 0) {
    gpr::set_error("gpr_graph_create_ex: invalid layout options (lane_max %d, chunk %d, "
                   "chunk_min %d, hot_entries %d, block_rows %d, tile_words %d, blocked_long %d)",
                   lane_max, chunk, chunk_min, hot_max, block_rows, tile_words, blocked_long);
    return GPR_EINVAL;
  }
  if (!out) {
    gpr::set_error("gpr_graph_create: NULL out");
    return GPR_EINVAL;
  }
  *out = nullptr;
  if (m < 0 || nnz < 0 || nnz > 0x7fffffffLL || (m > 0 && (!any_rowptr || !any_outdeg)) ||
      (nnz > 0 && !any_col)) {
    gpr::set_error("gpr_graph_create: invalid arguments (m=%d nnz=%lld)", m, nnz);
    return GPR_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    gpr::set_error("gpr_graph_create: no CUDA device");
    return GPR_ENODEV;
  }
  gpr_graph *g = new gpr_graph();
  const bool keep_csr = lopts && (lopts->flags & (GPR_LAYOUT_BATCHED | GPR_LAYOUT_PUSH));
  const bool blocked = lopts && (lopts->flags & GPR_LAYOUT_BLOCKED);
  int rc = create_impl(m, nnz, any_rowptr, any_col, any_outdeg, lane_max, chunk_min, chunk,
                       hot_max, keep_csr, blocked, block_rows, tile_words, blocked_long, g);
  if (rc != GPR_OK) {
    destroy(g);
    return rc;
  }
  *out = g;
  return GPR_OK;
  GPR_ENTRY_END("gpr_graph_create_ex")
}

int gpr_graph_destroy(gpr_graph *g) {
  destroy(g);
  return GPR_OK;
}

int gpr_graph_info(const gpr_graph *g, int *m, long long *nnz, long long *device_bytes) {
  if (!g) {
    gpr::set_error("gpr_graph_info: NULL graph");
    return GPR_EINVAL;
  }
  if (m) *m = g->L.m;
  if (nnz) *nnz = g->L.nnz;
  if (device_bytes) *device_bytes = g->L.device_bytes + 12LL * g->L.m;
  return GPR_OK;
}

int gpr_graph_set_stream(gpr_graph *g, void *stream) {
  if (!g) {
    gpr::set_error("gpr_graph_set_stream: NULL graph");
    return GPR_EINVAL;
  }
  if (g->own_stream && g->st) cudaStreamDestroy(g->st);
  g->own_stream = false;
  g->st = (cudaStream_t)stream;
  return GPR_OK;
}

int gpr_graph_layout(const gpr_graph *g, int *n_long, int *n_nz, int *n_chunks, int *n_slices,
                     long long *long_elems, long long *sell_elems) {
  if (!g) {
    gpr::set_error("gpr_graph_layout: NULL graph");
    return GPR_EINVAL;
  }
  if (n_long) *n_long = g->L.n_long;
  if (n_nz) *n_nz = g->L.n_nz;
  if (n_chunks) *n_chunks = g->L.n_chunks;
  if (n_slices) *n_slices = g->L.n_slices;
  if (long_elems) *long_elems = g->L.long_elems;
  if (sell_elems) *sell_elems = g->L.sell_elems;
  return GPR_OK;
}

int gpr_graph_residuals(const gpr_graph *g, double *h_out, int n) {
  if (!g || (n > 0 && !h_out)) {
    gpr::set_error("gpr_graph_residuals: NULL argument");
    return GPR_EINVAL;
  }
  const int k = n < g->last_sweeps ? n : g->last_sweeps;
  if (k > 0 && g->L.m == 0) {
    for (int i = 0; i < k; ++i) h_out[i] = 0.0;  // empty sweeps (nothing on the device)
  } else if (k > 0) {
    GPR_CUDA(cudaMemcpy(h_out, g->err_hist, sizeof(double) * (size_t)k, cudaMemcpyDeviceToHost));
  }
  return GPR_OK;
}

int gpr_pagerank(gpr_graph *g, float *any_scores, const gpr_pr_opts *opts, gpr_pr_stats *stats) {
  GPR_ENTRY_BEGIN
  if (!g) {
    gpr::set_error("gpr_pagerank: NULL graph");
    return GPR_EINVAL;
  }
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != g->device) GPR_CUDA(cudaSetDevice(g->device));
  int rc = pagerank_impl(g, any_scores, opts, stats);
  if (cur != g->device && cur >= 0) cudaSetDevice(cur);
  return rc;
  GPR_ENTRY_END("gpr_pagerank")
}

int gpr_pr_residual_f64(gpr_graph *g, const float *any_scores, float damping, double *residual) {
  GPR_ENTRY_BEGIN
  if (!g || !any_scores || !residual) {
    gpr::set_error("gpr_pr_residual_f64: NULL argument");
    return GPR_EINVAL;
  }
  const PrLayout &L = g->L;
  const int m = L.m;
  cudaStream_t st = g->st;
  void *dv = nullptr;
  bool owned = false;
  GPR_TRY(gpr::to_device(any_scores, sizeof(float) * (size_t)m, &dv, &owned, st, "scores"));
  if (!g->res_tmp) {
    int rc = gpr::dalloc(&g->res_tmp, 2 * (size_t)m + 2 + L.n_long, "residual scratch");
    if (rc != GPR_OK) {
      if (owned) gpr::dfree(dv);
      return rc;
    }
  }
  double *cd = g->res_tmp, *sd = g->res_tmp + m + 1, *acc = sd + m, *out = acc + L.n_long;
  gpr_pr_opts o;
  gpr_pr_opts_default(&o);
  o.damping = damping;
  PrArgs a = make_args(g, o, 0);
  const double d = (double)damping, base = (1.0 - d) / (double)m;
  cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(double) * ((size_t)L.n_long + 1), st);
  if (e == cudaSuccess) {
    k_res_prologue<<<grid_for((long long)m + 1), 256, 0, st>>>(m, L.perm, L.outdeg,
                                                               (const float *)dv, cd, sd);
    const long long units = (long long)L.n_chunks + L.n_slices + L.n_zblk;
    k_res_sweep<<<grid_for(units * 32), 256, 0, st>>>(a, cd, sd, d, base, acc, out);
    if (L.n_long)
      k_res_long<<<grid_for(L.n_long), 256, 0, st>>>(L.n_long, acc, sd, d, base, out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(residual, out, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (owned) gpr::dfree(dv);
  if (e != cudaSuccess) {
    gpr::set_error("gpr_pr_residual_f64: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  return GPR_OK;
  GPR_ENTRY_END("gpr_pr_residual_f64")
}

int gpr_page_rank(int m, int nnz, const int *row_offsets, const int *column_indices,
                  const int *degree, float *scores, const gpr_pr_opts *opts,
                  gpr_pr_stats *stats) {
  GPR_ENTRY_BEGIN
  gpr_graph *g = nullptr;
  GPR_TRY(gpr_graph_create(m, nnz, row_offsets, column_indices, degree, &g));
  int rc = gpr_pagerank(g, scores, opts, stats);
  gpr_graph_destroy(g);
  return rc;
  GPR_ENTRY_END("gpr_page_rank")
}

int gpr_pr_solver(int m, int nnz, const int *in_row_offsets, const int *in_column_indices,
                  const int *out_row_offsets, const int *out_column_indices, const int *degree,
                  float *scores, const gpr_pr_opts *opts, gpr_pr_stats *stats) {
  GPR_ENTRY_BEGIN
  (void)out_row_offsets;  // pull variants ignore the out-CSR (src/pr/gather.cu:41)
  (void)out_column_indices;
  return gpr_page_rank(m, nnz, in_row_offsets, in_column_indices, degree, scores, opts, stats);
  GPR_ENTRY_END("gpr_pr_solver")
}

}  // extern "C"
