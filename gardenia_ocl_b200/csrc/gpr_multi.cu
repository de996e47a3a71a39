// Uneven multi-graph batch: many independent pull graphs solved together in
// one persistent cooperative launch.
//
// No reference file: every reference run reads and solves one graph
// (src/pr/main.cc:14-34).  Each graph of a batch is solved exactly as
// gpr_pagerank solves it alone -- the iteration body of src/pr/omp_base.cc
// with its own base (1 - kDamp) / m_g (omp_base.cc:16), its own FP64 L1
// residual and its own stop rule (omp_base.cc:23,43) -- so a graph's scores
// and sweep count do not depend on the batch around it.
//
// Input: one block-diagonal pull graph.  Graph g owns vertices
// [voff[g], voff[g+1]) and the in-edges of its rows come from that range
// (global vertex ids).
//
// Layout (device, built once): graphs are reordered by descending edge count
// (largest first, so the work queue ends with small units) and inside each
// graph vertices are relabelled by descending in-degree, as in the
// single-graph layout.  Each graph is cut into work units with its own bins
// (lane_max, chunk_min, chunk -- the per-graph layout options an autotuner
// chooses): chunks of long rows, SELL-32 slices of width class w, and blocks
// of 128 in-degree-0 rows.  A unit's descriptor names its graph, kind, rows
// and class; its edges are one contiguous, 16-byte-aligned range of a single
// edge array in unit order.
//
// Per sweep, warps take batches of units from a global queue.  Units of a
// frozen graph are skipped.  Each unit stores its FP64 residual; the warp
// that completes the last unit of a graph in a sweep sums that graph's unit
// residuals in unit order (deterministic), and freezes the graph when the sum
// is below tol or its sweep cap is reached.  One bounded grid barrier per
// sweep; the launch ends when no graph is left updating.
#include <cub/cub.cuh>
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "gpr_blocked.cuh"
#include "gpr_device.cuh"
#include "gpr_internal.cuh"
#include "gpr_guard.h"

using namespace gpr::dev;

namespace {

enum { kUnitChunk = 0, kUnitSlice = 1, kUnitZero = 2 };
constexpr int kMultiBlock = 1024;
constexpr double kBf16Tol = 1e-3;  // BF16 phase of the mixed form (as the single-graph solver)
using bf16 = __nv_bfloat16;

// Unit descriptor (int4):
//   x  first row (relabelled, global)
//   y  chunk: unit index of the row's first chunk
//   z  chunk: chunks of the row; slice / zero: rows in the unit
//   w  internal graph << 8 | kind << 4 | log2(lanes per row) (slices)
struct MultiArgs {
  int M, G, n_heavy, n_zero;
  const int4 *meta;
  const long long *uoff;  // [units + 1] edge offsets (multiples of 4)
  const int *ecol;        // relabelled sources; padding holds the sentinel M
  const int *outdeg;      // [M] relabelled
  const int *gm;          // [G] vertices of each graph (internal order)
  const int *hb, *zb;     // [G+1] heavy / zero unit ranges of each graph
  const int *cap;         // [G] sweep cap of each graph
  int *stop;              // [G] the graph updates in sweeps < stop[g]
  int *gdone;             // [G] units of the graph finished in the current sweep
  double *gres;           // [G] L1 change of the graph's last sweep
  const int *lazy;        // graphs with vertices but no heavy units
  int n_lazy;
  float *s;
  void *c0, *c1;          // contributions by sweep parity (float or bf16), [M + 1]
  float *partial;         // [n_heavy] chunk partial sums, by unit
  int *cnt;               // [n_heavy] arrivals at multi-chunk rows, by first unit
  double *uerr;           // [units] L1 change of each unit
  int *n_next;            // [2] graphs still updating in the next sweep, by parity
  unsigned *bar;          // [2] arrivals, generation
  int *status;            // [0] error flags, [1] sweeps of the launch, [2] done
  int *wq;                // [2] work-queue heads by parity
  const int *pk;          // [n_pk + 1] first unit of each work packet
  int n_hpk, n_pk;        // packets of heavy units; all packets (zero units last)
  float damp;
  double tol;
  int max_iter, bar_expect;
  long long timeout_ns;
  unsigned long long cond;  // graph mode: while-node condition handle (0: none)
  // blocked form (gpr_blocked.cuh): each graph's rows with in-edges in
  // blocks, tiles of source-ordered entries; null tb: the units form
  const int *tb;          // [G+1] residual slots (tiles) of each graph
  double *terr;           // [tiles] residual of each tile, by slot
  int n_tiles, acc_rows, blk_row0;
  const int4 *tiles;
  const int4 *blocks;     // .w: the block's graph
  const uint2 *runs;
  const unsigned *entry;
  unsigned long long *gacc;
  int *bcnt;
  int *tq;                // [2] tile-queue heads by parity
  float fx_scale;         // 2^S: contributions as 64-bit fixed point
  double fx_inv;          // 2^-S
};

template <typename T>
__device__ __forceinline__ double mrow_update(const MultiArgs &a, float base, int r, float sum,
                                              float so, int od, T *cout, const Policies &pol) {
  const float sn = __fadd_rn(base, __fmul_rn(a.damp, sum));
  st_f32(a.s + r, sn, pol.stream);
  st_c(cout + r, __fdiv_rn(sn, __int2float_rn(od)), pol.keep);
  return (double)fabsf(__fsub_rn(sn, so));
}

// One chunk of a long row (same per-lane order and combine as the
// single-graph kernel, so per-graph results match it bit for bit).
template <int U4, typename T>
__device__ __forceinline__ double m_chunk(const MultiArgs &a, const GlobalGather<T> &gat, T *cout,
                                          int u, int4 md, long long b, long long e, float base,
                                          int lane, const Policies &pol) {
  const int r = md.x, cb = md.y, nc = md.z;
  float so = 0.f;
  int od = 1;
  if (lane == 0) {
    so = ld_f32_stream(a.s + r, pol.stream);
    od = ld_s32_stream(a.outdeg + r, pol.stream);
  }
  float acc = 0.f;
  for (long long k0 = b + 4 * lane; k0 < e; k0 += 128 * U4) {
    int4 q[U4];
#pragma unroll
    for (int i = 0; i < U4; ++i)
      q[i] = (k0 + 128 * i < e) ? ld_idx4(a.ecol + k0 + 128 * i, pol.stream)
                                : make_int4(a.M, a.M, a.M, a.M);
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
  if (nc == 1) return lane == 0 ? mrow_update(a, base, r, acc, so, od, cout, pol) : 0.0;
  int last = 0;
  if (lane == 0) {
    a.partial[u] = acc;
    __threadfence();
    last = atomicAdd(a.cnt + cb, 1) == nc - 1;
  }
  last = __shfl_sync(kFull, last, 0);
  if (!last) return 0.0;
  __threadfence();
  float t = 0.f;
  for (int q = lane; q < nc; q += 32) t += __ldcg(a.partial + cb + q);
  t = warp_sum(t);
  if (lane != 0) return 0.0;
  atomicExch(a.cnt + cb, 0);
  return mrow_update(a, base, r, t, so, od, cout, pol);
}

// One SELL-32 slice of 32 >> lw rows, w = 1 << lw lanes per row.
template <int U, typename T>
__device__ __forceinline__ double m_slice(const MultiArgs &a, const GlobalGather<T> &gat, T *cout,
                                          int u, int4 md, long long b, long long e, float base,
                                          int lane, const Policies &pol) {
  const int lw = md.w & 15;
  const int r = md.x + (lane >> lw);
  const bool lead = (lane & ((1 << lw) - 1)) == 0;
  const bool valid = (lane >> lw) < md.z;
  float so = 0.f;
  int od = 1;
  if (valid && lead) {
    so = ld_f32_stream(a.s + r, pol.stream);
    od = ld_s32_stream(a.outdeg + r, pol.stream);
  }
  const int len = (int)((e - b) >> 5);
  const int *p = a.ecol + b + lane;
  float acc = 0.f;
  for (int j0 = 0; j0 < len; j0 += U) {
    int ci[U];
#pragma unroll
    for (int q = 0; q < U; ++q) ci[q] = (j0 + q < len) ? ld_idx(p + 32 * (j0 + q), pol.stream) : a.M;
    float v[U];
#pragma unroll
    for (int q = 0; q < U; ++q) v[q] = gat(ci[q]);
#pragma unroll
    for (int q = 0; q < U; ++q) acc = __fadd_rn(acc, v[q]);
  }
  for (int o = (1 << lw) >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  return (valid && lead) ? mrow_update(a, base, r, acc, so, od, cout, pol) : 0.0;
}

// Rows without in-edges: updated in sweep 0, contribution copied in sweep 1.
template <typename T>
__device__ __forceinline__ double m_zero(const MultiArgs &a, T *cout, int4 md, float base,
                                         int lane, int it, const Policies &pol) {
  double err = 0.0;
#pragma unroll
  for (int q = 0; q < gpr::kZeroRowsPerUnit / 32; ++q) {
    const int i = 32 * q + lane;
    if (i < md.z) {
      const int r = md.x + i;
      const int od = ld_s32_stream(a.outdeg + r, pol.stream);
      if (it == 0) {
        err += mrow_update(a, base, r, 0.f, ld_f32_stream(a.s + r, pol.stream), od, cout, pol);
      } else {
        const float sn = __fadd_rn(base, __fmul_rn(a.damp, 0.f));
        st_c(cout + r, __fdiv_rn(sn, __int2float_rn(od)), pol.keep);
      }
    }
  }
  return err;
}

// Lane's share of sum(v[b..e)): elements b + lane + 32 j, eight independent
// accumulators so eight loads are in flight, combined in a fixed order
// (deterministic for a given range).
__device__ __forceinline__ double range_sum(const double *v, int b, int e, int lane) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int u = b + lane;
  for (; u + 32 * 7 < e; u += 32 * 8) {
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] += __ldcg(v + u + 32 * q);
  }
#pragma unroll
  for (int q = 0; q < 8; ++q)
    if (u + 32 * q < e) acc[q] += __ldcg(v + u + 32 * q);
  return ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
}

// `done` units of graph g finished by this warp in sweep it (in the blocked
// form a tile counts as one unit).  The warp that completes the graph's last
// unit sums the graph's unit (or tile) residuals in slot order and decides
// whether the graph keeps updating.
__device__ __forceinline__ void finish_units(const MultiArgs &a, int g, int done, int it,
                                             int lane) {
  int last = 0;
  if (lane == 0) {
    const int heavy = a.tb ? a.tb[g + 1] - a.tb[g] : a.hb[g + 1] - a.hb[g];
    const int expect = heavy + (it < 2 ? a.zb[g + 1] - a.zb[g] : 0);
    __threadfence();
    last = atomicAdd(a.gdone + g, done) + done == expect;
  }
  last = __shfl_sync(kFull, last, 0);
  if (!last) return;
  __threadfence();
  double t = a.tb ? range_sum(a.terr, a.tb[g], a.tb[g + 1], lane)
                  : range_sum(a.uerr, a.hb[g], a.hb[g + 1], lane);
  if (it < 2) t += range_sum(a.uerr, a.zb[g], a.zb[g + 1], lane);
  t = warp_sum(t);
  if (lane == 0) {
    a.gres[g] = t;
    atomicExch(a.gdone + g, 0);
    if (t < a.tol || it + 1 >= a.cap[g]) atomicExch(a.stop + g, it + 1);
    else atomicAdd(a.n_next + ((it + 1) & 1), 1);
  }
}

// Grid barrier closing sweep it.  The last CTA to arrive settles the graphs
// that have no heavy units (their residual is 0 from sweep 2 on), resets the
// queue head and graph counter that sweep it + 2 reuses, and opens the next
// generation.  Waits are bounded by timeout_ns; on expiry status[0] bit 0 is
// raised and the caller returns.
// Closing of sweep it, by one thread of the last CTA to finish it (every
// CTA's work of the sweep visible): settles the graphs that have no heavy
// units (their residual is 0 from sweep 2 on) and resets the queue head and
// graph counter that sweep it + 2 reuses.
__device__ void multi_close(const MultiArgs &a, int it) {
  if (it >= 2)
    for (int i = 0; i < a.n_lazy; ++i) {
      const int g = a.lazy[i];
      if (it < __ldcg(a.stop + g)) {
        a.gres[g] = 0.0;
        if (0.0 < a.tol || it + 1 >= a.cap[g]) atomicExch(a.stop + g, it + 1);
        else atomicAdd(a.n_next + ((it + 1) & 1), 1);
      }
    }
  atomicExch(a.wq + (it & 1), 0);
  if (a.tq) atomicExch(a.tq + (it & 1), 0);
  atomicExch(a.n_next + (it & 1), 0);
}

__device__ bool multi_barrier(const MultiArgs &a, int it) {
  __shared__ int s_state;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned gen = ld_acquire(a.bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(a.bar, 1u);
    s_state = 0;
    if (arrived == (unsigned)a.bar_expect - 1u) {
      __threadfence();
      multi_close(a, it);
      atomicExch(a.bar, 0u);
      __threadfence();
      atomicAdd(a.bar + 1, 1u);
    } else {
      const long long t0 = global_ns();
      unsigned spins = 0;
      while (ld_acquire(a.bar + 1) == gen) {
        if ((++spins & 31u) == 0 && global_ns() - t0 > a.timeout_ns) {
          atomicOr(a.status, 1);
          s_state = 2;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return s_state != 2;
}

// The units of sweep it: warps take packets from the queue, skip the units
// of frozen graphs, and close the graphs whose last unit they finish.
template <int U, int U4, typename T>
__device__ __forceinline__ void multi_sweep(const MultiArgs &a, int it, int lane,
                                            const Policies &pol) {
  const T *cin = static_cast<const T *>((it & 1) ? a.c1 : a.c0);
  T *cout = static_cast<T *>((it & 1) ? a.c0 : a.c1);
  const GlobalGather<T> gat{cin, pol.keep};
  const int n_pk = it < 2 ? a.n_pk : a.n_hpk;
  for (;;) {
    int p = 0;
    if (lane == 0) p = atomicAdd(a.wq + (it & 1), 1);
    p = __shfl_sync(kFull, p, 0);
    if (p >= n_pk) break;
    const int u0 = __ldg(a.pk + p), u1 = __ldg(a.pk + p + 1);
    int cur = -1, done = 0;
    bool act = false;
    float base = 0.f;
    int4 md_n = make_int4(0, 0, 0, 0);
    long long b_n = 0, e_n = 0;
    if (u0 < u1) {
      md_n = __ldg(a.meta + u0);
      b_n = __ldg(a.uoff + u0);
      e_n = __ldg(a.uoff + u0 + 1);
    }
    for (int u = u0; u < u1; ++u) {
      const int4 md = md_n;
      const long long ub = b_n, ue = e_n;
      if (u + 1 < u1) {  // the next unit's descriptor and end offset are in flight meanwhile
        md_n = __ldg(a.meta + u + 1);
        b_n = ue;
        e_n = __ldg(a.uoff + u + 2);
      }
      const int g = md.w >> 8;
      if (g != cur) {
        if (done) finish_units(a, cur, done, it, lane);
        cur = g;
        done = 0;
        act = it < __ldcg(a.stop + g);
        base = __fdiv_rn(__fsub_rn(1.0f, a.damp), __int2float_rn(__ldg(a.gm + g)));
      }
      if (!act) continue;
      const int kind = (md.w >> 4) & 15;
      double err;
      if (kind == kUnitChunk) err = m_chunk<U4>(a, gat, cout, u, md, ub, ue, base, lane, pol);
      else if (kind == kUnitSlice) err = m_slice<U>(a, gat, cout, u, md, ub, ue, base, lane, pol);
      else err = m_zero(a, cout, md, base, lane, it, pol);
      err = warp_sum(err);
      if (lane == 0) a.uerr[u] = err;
      ++done;
    }
    if (done) finish_units(a, cur, done, it, lane);
  }
}

// All sweeps in one cooperative launch, a bounded grid barrier between them.
template <int U, int U4, typename T>
__global__ void __launch_bounds__(kMultiBlock, 1) k_multi(MultiArgs a) {
  const int lane = threadIdx.x & 31;
  const Policies pol = make_policies();
  int it = 0;
  while (it < a.max_iter) {
    multi_sweep<U, U4, T>(a, it, lane, pol);
    if (!multi_barrier(a, it)) return;
    const int n = __ldcg(a.n_next + ((it + 1) & 1));
    ++it;
    if (n == 0) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.status[1] = it;
    a.status[2] = 1;
  }
}

// All sweeps of the blocked form in one cooperative launch (FP32), MINB CTAs
// of NT threads per SM.  Per sweep: CTAs take tiles from a queue (heaviest
// first), skipping the tiles of graphs that no longer update; a tile's
// residual goes to its graph's slot and the CTA that finishes a graph's last
// unit closes the graph (as the units form does).  Then, in sweeps 0 and 1,
// warps take the packets of zero-in-degree rows.  One bounded grid barrier
// per sweep.
template <int PV, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_multi_blocked(MultiArgs a) {
  extern __shared__ unsigned s_acc[];  // [2 * acc_rows]: low / high words
  __shared__ int s_tile, s_next_tile, s_last, s_next;
  __shared__ double s_red[NT / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Policies pol = make_policies();
  int it = 0;
  while (it < a.max_iter) {
    const float *cin = static_cast<const float *>((it & 1) ? a.c1 : a.c0);
    float *cout = static_cast<float *>((it & 1) ? a.c0 : a.c1);
    int *tq = a.tq + (it & 1);
    if (threadIdx.x == 0) s_next_tile = atomicAdd(tq, 1);
    for (;;) {
      __syncthreads();
      if (threadIdx.x == 0) s_tile = s_next_tile;
      __syncthreads();
      const int t = s_tile;
      if (t >= a.n_tiles) break;
      const int4 td = __ldg(a.tiles + t);
      const int g = __ldg(&a.blocks[td.x].w);
      if (it >= __ldcg(a.stop + g)) {  // the graph no longer updates
        if (threadIdx.x == 0) s_next_tile = atomicAdd(tq, 1);
        continue;
      }
      const float base = __fdiv_rn(__fsub_rn(1.0f, a.damp), __int2float_rn(__ldg(a.gm + g)));
      double err = gpr::blk::blocked_tile<PV, NT>(a, cin, cout, t, s_acc, &s_next, &s_last,
                                                  &s_next_tile, tq, base, pol);
      err = warp_sum(err);
      if (lane == 0) s_red[warp] = err;
      __syncthreads();
      if (warp == 0) {
        double e = lane < NT / 32 ? s_red[lane] : 0.0;
        e = warp_sum(e);
        if (lane == 0) a.terr[td.w] = e;
        finish_units(a, g, 1, it, lane);
      }
    }
    if (it < 2) {  // zero-in-degree rows: the zero packets of the units form
      for (;;) {
        int p = 0;
        if (lane == 0) p = atomicAdd(a.wq + (it & 1), 1);
        p = a.n_hpk + __shfl_sync(kFull, p, 0);
        if (p >= a.n_pk) break;
        const int u0 = __ldg(a.pk + p), u1 = __ldg(a.pk + p + 1);
        int cur = -1, done = 0;
        bool act = false;
        float base = 0.f;
        for (int u = u0; u < u1; ++u) {
          const int4 md = __ldg(a.meta + u);
          const int g = md.w >> 8;
          if (g != cur) {
            if (done) finish_units(a, cur, done, it, lane);
            cur = g;
            done = 0;
            act = it < __ldcg(a.stop + g);
            base = __fdiv_rn(__fsub_rn(1.0f, a.damp), __int2float_rn(__ldg(a.gm + g)));
          }
          if (!act) continue;
          double err = m_zero(a, cout, md, base, lane, it, pol);
          err = warp_sum(err);
          if (lane == 0) a.uerr[u] = err;
          ++done;
        }
        if (done) finish_units(a, cur, done, it, lane);
      }
    }
    if (!multi_barrier(a, it)) return;
    const int n = __ldcg(a.n_next + ((it + 1) & 1));
    ++it;
    if (n == 0) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.status[1] = it;
    a.status[2] = 1;
  }
}

// Largest |score| (bits of a non-negative float order like the float; a NaN
// sorts above every finite value and infinity).
__global__ void k_multi_max_abs(int m, const float *__restrict__ s, unsigned *out) {
  unsigned mx = 0u;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
       i += (long long)gridDim.x * blockDim.x)
    mx = max(mx, __float_as_uint(s[i]) & 0x7FFFFFFFu);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// One sweep per launch (graph mode): the body of a CUDA-graph while node.
// status[1] holds the sweeps done and status[2] the done flag, so the
// captured launch needs no host input; the last CTA to finish a sweep closes
// it (no CTA waits for another, so the grid need not be co-resident).  The
// node's condition starts at 1 and is only cleared: by the CTA that closes
// the last sweep, by a launch that finds the solve done, and by CTA 0 of the
// max_iter-th launch (status[3] counts launches).
template <int U, int U4, typename T>
__global__ void __launch_bounds__(kMultiBlock, 1) k_multi_step(MultiArgs a) {
  __shared__ int s_it, s_last;
  if (threadIdx.x == 0) {
    const int n_done = *(volatile int *)(a.status + 1);
    const bool fin = *(volatile int *)(a.status + 2) != 0;
    s_it = !fin && n_done < a.max_iter ? n_done : -1;
    if (a.cond && blockIdx.x == 0) {
      const int n = atomicAdd(a.status + 3, 1) + 1;
      if (s_it < 0 || n >= a.max_iter) cudaGraphSetConditional(a.cond, 0u);
    }
  }
  __syncthreads();
  const int it = s_it;
  if (it < 0) return;
  const Policies pol = make_policies();
  multi_sweep<U, U4, T>(a, it, threadIdx.x & 31, pol);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(a.bar, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  multi_close(a, it);
  atomicExch(a.bar, 0u);
  const int n = __ldcg(a.n_next + ((it + 1) & 1));
  const bool done = n == 0 || it + 1 >= a.max_iter;
  a.status[1] = it + 1;
  if (done) a.status[2] = 1;
  __threadfence();
  if (a.cond && done) cudaGraphSetConditional(a.cond, 0u);
}

template <typename T>
__global__ void k_multi_prologue(int M, const int *__restrict__ perm,
                                 const int *__restrict__ outdeg, const float *__restrict__ in,
                                 float *s, T *c0, T *c1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) {
    const float v = in[perm[i]];
    s[i] = v;
    c0[i] = (T)__fdiv_rn(v, __int2float_rn(outdeg[i]));
  } else if (i == M) {
    c0[M] = (T)0.f;
    c1[M] = (T)0.f;
  }
}

__global__ void k_multi_scatter(int M, const int *__restrict__ perm, const float *__restrict__ s,
                                float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) out[perm[i]] = s[i];
}

// ---- layout construction ----------------------------------------------------

__device__ __forceinline__ int find_graph(const int *__restrict__ off, int G, long long x) {
  int lo = 0, hi = G;  // last g with off[g] <= x (off non-decreasing)
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Every edge of a row of graph g must come from graph g's vertex range.
__global__ void k_check_blocks(long long nnz, int G, const int *__restrict__ eoff,
                               const int *__restrict__ voff, const int *__restrict__ col,
                               int *flag) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    const int lo = find_graph(eoff, G, e);  // the graph whose edge range holds e
    const int c = col[e];
    if (c < voff[lo] || c >= voff[lo + 1]) atomicOr(flag, 32);
  }
}

__global__ void k_gather_eoff(int G, const int *__restrict__ voff, const int *__restrict__ rowptr,
                              int *eoff) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g <= G) eoff[g] = rowptr[voff[g]];
}

// Sort key of vertex v: (internal graph, descending in-degree); value v.
__global__ void k_vertex_keys(int M, int G, const int *__restrict__ voff,
                              const int *__restrict__ rank, const int *__restrict__ rowptr,
                              unsigned long long *key, int *iota) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < M) {
    const int g = find_graph(voff, G, v);
    const unsigned d = (unsigned)(rowptr[v + 1] - rowptr[v]);
    key[v] = ((unsigned long long)rank[g] << 32) | (unsigned long long)(0x7fffffffu - d);
    iota[v] = v;
  }
}

__global__ void k_multi_relabel(int M, const int *__restrict__ perm,
                                const int *__restrict__ outdeg, const int *__restrict__ rowptr,
                                int *outdeg_new, int *sdeg, int *inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) {
    const int o = perm[i];
    outdeg_new[i] = outdeg[o];
    sdeg[i] = rowptr[o + 1] - rowptr[o];
    inv[o] = i;
  }
}

// bounds[r * 8 + k] = rows of internal graph r with in-degree > th[r * 8 + k]
// (in-degrees descend inside each graph's row range).
__global__ void k_multi_bounds(int G, const int *__restrict__ ivoff, const int *__restrict__ sdeg,
                               const int *__restrict__ th, int nth, int *bounds) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= G * nth) return;
  const int r = t / nth, k = t % nth;
  const int b = ivoff[r], e = ivoff[r + 1], x = th[r * 8 + k];
  int lo = b, hi = e;  // first row with degree <= x
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (sdeg[mid] > x) lo = mid + 1;
    else hi = mid;
  }
  bounds[r * 8 + k] = lo - b;
}

__global__ void k_unit_lens(int n_units, const int4 *__restrict__ meta,
                            const int *__restrict__ sdeg, const int *__restrict__ gchunk,
                            long long *len) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n_units) {
    const int4 md = meta[u];
    const int kind = (md.w >> 4) & 15;
    long long l = 0;
    if (kind == kUnitChunk) {
      const long long p = ((long long)sdeg[md.x] + 3) & ~3LL;
      const long long ch = gchunk[md.w >> 8];
      const long long k = u - md.y;
      l = min(ch, p - k * ch);
    } else if (kind == kUnitSlice) {
      const int lw = md.w & 15;
      l = 32LL * (((long long)sdeg[md.x] + (1 << lw) - 1) >> lw);
    }
    len[u] = l;
  } else if (u == n_units) {
    len[u] = 0;
  }
}

// One warp per unit: relabelled sources, sentinel M in padding.
__global__ void k_fill_units(int n_units, int M, const int4 *__restrict__ meta,
                             const long long *__restrict__ uoff, const int *__restrict__ gchunk,
                             const int *__restrict__ perm, const int *__restrict__ inv,
                             const int *__restrict__ sdeg, const int *__restrict__ rowptr,
                             const int *__restrict__ col, int *ecol) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long u = w0; u < n_units; u += nw) {
    const int4 md = meta[u];
    const int kind = (md.w >> 4) & 15;
    const long long b = uoff[u], len = uoff[u + 1] - b;
    if (kind == kUnitChunk) {
      const long long ch = gchunk[md.w >> 8];
      const long long k = u - md.y;
      const long long sb = rowptr[perm[md.x]] + k * ch;
      const long long deg = sdeg[md.x] - k * ch;
      for (long long j = lane; j < len; j += 32) ecol[b + j] = j < deg ? inv[col[sb + j]] : M;
    } else if (kind == kUnitSlice) {
      const int lw = md.w & 15;
      const bool valid = (lane >> lw) < md.z;
      const int r = md.x + (lane >> lw), l = lane & ((1 << lw) - 1);
      const int deg = valid ? sdeg[r] : 0;
      const long long sb = valid ? rowptr[perm[r]] : 0;
      for (long long j = 0; j < (len >> 5); ++j) {
        const long long e = (j << lw) + l;
        ecol[b + 32 * j + lane] = e < deg ? inv[col[sb + e]] : M;
      }
    }
  }
}

inline unsigned grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 0x7fffffffLL) g = 0x7fffffffLL;
  return (unsigned)g;
}

inline unsigned capped(long long n) { return std::min<unsigned>(grid_for(n), 148u * 64u); }

}  // namespace

struct gpr_multigraph {
  int device = 0;
  int G = 0, M = 0;
  long long nnz = 0;
  int n_heavy = 0, n_zero = 0;
  long long edge_slots = 0;
  std::vector<int> rank;        // user graph -> internal graph
  std::vector<int> order;       // internal graph -> user graph
  std::vector<int> ivoff;       // [G+1] internal vertex offsets
  std::vector<int> lazy_h;
  int *perm = nullptr, *outdeg = nullptr, *ecol = nullptr;
  int4 *meta = nullptr;
  long long *uoff = nullptr;
  int *gm = nullptr, *hb = nullptr, *zb = nullptr, *cap = nullptr, *stop = nullptr;
  int *gdone = nullptr, *lazy = nullptr;
  double *gres = nullptr;
  float *s = nullptr, *c0 = nullptr, *c1 = nullptr;
  bf16 *h0 = nullptr, *h1 = nullptr;
  float *partial = nullptr;
  int *cnt = nullptr;
  double *uerr = nullptr;
  int *n_next = nullptr;
  unsigned *bar = nullptr;
  int *status = nullptr, *wq = nullptr;
  int *pk = nullptr;             // work packets: first unit of each
  int n_hpk = 0, n_pk = 0;
  float *scores_tmp = nullptr;
  int grid = 0;
  bool coop_ok = false;
  cudaStream_t st = nullptr;
  bool own_stream = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
  long long device_bytes = 0;
  // blocked form: each graph's rows with in-edges in blocks
  gpr::BlockedLayout B;
  bool has_blocked = false, blocked_ok = false;
  int grid_blocked = 0, blocked_ctas = 1, max_gm = 0;
  int *tq = nullptr, *tb = nullptr, *lazy_b = nullptr;
  std::vector<int> lazy_bh;     // graphs with vertices but no tiles
  double *terr = nullptr;
  unsigned *fx_max = nullptr;
};

namespace {

const void *multi_kernel(bool bf) {
  return bf ? (const void *)k_multi<16, 4, bf16> : (const void *)k_multi<16, 4, float>;
}

const void *multi_step_kernel(bool bf) {
  return bf ? (const void *)k_multi_step<16, 4, bf16> : (const void *)k_multi_step<16, 4, float>;
}

// The blocked batch kernel with `ctas` CTAs per SM (1: 1024 threads, 2: 512).
const void *multi_blocked_kernel(int ctas) {
  return ctas == 2 ? (const void *)k_multi_blocked<4, 512, 2>
                   : (const void *)k_multi_blocked<4, 1024, 1>;
}

// solve_phase status: the blocked form cannot represent these scores
constexpr int kMultiBlockedFallback = 100;

void destroy_multi(gpr_multigraph *g) {
  if (!g) return;
  void *ptrs[] = {g->perm,  g->outdeg, g->ecol,    g->meta,    g->uoff,   g->gm,
                  g->hb,    g->zb,     g->cap,     g->stop,    g->gdone,  g->lazy,
                  g->gres,  g->s,      g->c0,      g->c1,      g->h0,     g->h1,
                  g->partial, g->cnt,  g->uerr,    g->n_next,  g->bar,    g->status,
                  g->wq,    g->scores_tmp, g->pk, g->tq, g->tb, g->lazy_b, g->terr, g->fx_max};
  for (void *p : ptrs) gpr::dfree(p);
  gpr::free_blocked_layout(&g->B);
  if (g->e0) cudaEventDestroy(g->e0);
  if (g->e1) cudaEventDestroy(g->e1);
  if (g->e2) cudaEventDestroy(g->e2);
  if (g->e3) cudaEventDestroy(g->e3);
  if (g->own_stream && g->st) cudaStreamDestroy(g->st);
  delete g;
}

struct Tmp {
  std::vector<void *> p;
  template <typename X>
  int get(X **out, size_t n, const char *what) {
    int rc = gpr::dalloc(out, n, what);
    if (rc == GPR_OK) p.push_back(*out);
    return rc;
  }
  ~Tmp() {
    for (void *q : p) gpr::dfree(q);
  }
};

int build_multi(gpr_multigraph *g, const int *h_voff, const int *d_rowptr, const int *d_col,
                const int *d_outdeg, const gpr_layout_opts *lopts) {
  const gpr_layout_opts *blo = nullptr;  // the first graph's options that ask for blocks
  for (int ug = 0; lopts && ug < g->G && !blo; ++ug)
    if (lopts[ug].flags & GPR_LAYOUT_BLOCKED) blo = lopts + ug;
  const int G = g->G, M = g->M;
  cudaStream_t st = g->st;
  Tmp T;
  int *dvoff = nullptr, *deoff = nullptr, *flag = nullptr;
  GPR_TRY(T.get(&dvoff, (size_t)G + 1, "vertex offsets"));
  GPR_TRY(T.get(&deoff, (size_t)G + 1, "edge offsets"));
  GPR_TRY(T.get(&flag, 1, "validation flag"));
  GPR_CUDA(cudaMemcpyAsync(dvoff, h_voff, sizeof(int) * ((size_t)G + 1), cudaMemcpyHostToDevice, st));
  k_gather_eoff<<<grid_for((long long)G + 1), 256, 0, st>>>(G, dvoff, d_rowptr, deoff);
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
  if (g->nnz > 0) {
    k_check_blocks<<<capped(g->nnz), 256, 0, st>>>(g->nnz, G, deoff, dvoff, d_col, flag);
    GPR_CUDA(cudaGetLastError());
  }
  std::vector<int> eoff(G + 1);
  int hflag = 0;
  GPR_CUDA(cudaMemcpyAsync(eoff.data(), deoff, sizeof(int) * eoff.size(), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  if (hflag) {
    gpr::set_error("gpr_multigraph_create: an edge of graph g comes from outside graph g's "
                   "vertex range (the batch must be block-diagonal)");
    return GPR_EINVAL;
  }
  // Internal order: descending edge count, ties by user index.
  g->order.resize(G);
  std::iota(g->order.begin(), g->order.end(), 0);
  std::stable_sort(g->order.begin(), g->order.end(), [&](int x, int y) {
    return eoff[x + 1] - eoff[x] > eoff[y + 1] - eoff[y];
  });
  g->rank.assign(G, 0);
  g->ivoff.assign(G + 1, 0);
  for (int r = 0; r < G; ++r) {
    const int ug = g->order[r];
    g->rank[ug] = r;
    g->ivoff[r + 1] = g->ivoff[r] + (h_voff[ug + 1] - h_voff[ug]);
  }
  // Relabel: sort vertices by (internal graph, descending in-degree), stable.
  int *drank = nullptr, *iota = nullptr, *sdeg = nullptr, *inv = nullptr;
  unsigned long long *key = nullptr, *key2 = nullptr;
  GPR_TRY(T.get(&drank, (size_t)G, "graph ranks"));
  GPR_TRY(T.get(&iota, (size_t)M, "iota"));
  GPR_TRY(T.get(&sdeg, (size_t)M, "sorted degree"));
  GPR_TRY(T.get(&inv, (size_t)M, "inverse permutation"));
  GPR_TRY(T.get(&key, (size_t)M, "vertex keys"));
  GPR_TRY(T.get(&key2, (size_t)M, "vertex keys (sorted)"));
  GPR_TRY(gpr::dalloc(&g->perm, (size_t)M, "permutation"));
  GPR_TRY(gpr::dalloc(&g->outdeg, (size_t)M, "out-degree"));
  GPR_CUDA(cudaMemcpyAsync(drank, g->rank.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
  k_vertex_keys<<<grid_for(M), 256, 0, st>>>(M, G, dvoff, drank, d_rowptr, key, iota);
  GPR_CUDA(cudaGetLastError());
  {
    int gbits = 1;
    while ((1LL << gbits) < G) ++gbits;
    size_t tb = 0;
    GPR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, iota, g->perm, M, 0,
                                             32 + gbits, st));
    void *tmp = nullptr;
    GPR_TRY(gpr::dmalloc(&tmp, tb, "sort scratch"));
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, iota, g->perm, M, 0,
                                                    32 + gbits, st);
    gpr::dfree(tmp);
    if (e != cudaSuccess) {
      gpr::set_error("vertex sort: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  }
  k_multi_relabel<<<grid_for(M), 256, 0, st>>>(M, g->perm, d_outdeg, d_rowptr, g->outdeg, sdeg,
                                               inv);
  GPR_CUDA(cudaGetLastError());
  // Per-graph bins (thresholds as in the single-graph layout).
  std::vector<int> lane_max(G), chunk_min(G), chunk(G), th(8 * (size_t)G, 0);
  const int nth = 7;
  for (int r = 0; r < G; ++r) {
    const int ug = g->order[r];
    const gpr_layout_opts *lo = lopts ? lopts + ug : nullptr;
    lane_max[r] = lo && lo->sell_max ? lo->sell_max : gpr::kSellMaxDefault;
    chunk_min[r] = lo && lo->chunk_min ? lo->chunk_min : gpr::kChunkMinDefault;
    chunk[r] = lo && lo->chunk ? lo->chunk : gpr::kChunkDefault;
    int *t = th.data() + 8 * (size_t)r;
    t[0] = chunk_min[r];
    for (int lw = 4; lw >= 0; --lw) t[5 - lw] = (int)std::min<long long>((long long)lane_max[r] << lw, chunk_min[r]);
    t[6] = 0;
  }
  int *dth = nullptr, *dbounds = nullptr, *divoff = nullptr;
  GPR_TRY(T.get(&dth, th.size(), "thresholds"));
  GPR_TRY(T.get(&dbounds, th.size(), "class bounds"));
  GPR_TRY(T.get(&divoff, (size_t)G + 1, "internal offsets"));
  GPR_CUDA(cudaMemcpyAsync(dth, th.data(), sizeof(int) * th.size(), cudaMemcpyHostToDevice, st));
  GPR_CUDA(cudaMemcpyAsync(divoff, g->ivoff.data(), sizeof(int) * ((size_t)G + 1),
                           cudaMemcpyHostToDevice, st));
  k_multi_bounds<<<grid_for((long long)G * nth), 256, 0, st>>>(G, divoff, sdeg, dth, nth, dbounds);
  GPR_CUDA(cudaGetLastError());
  std::vector<int> bounds(8 * (size_t)G);
  GPR_CUDA(cudaMemcpyAsync(bounds.data(), dbounds, sizeof(int) * bounds.size(),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  // Long-row in-degrees (chunk counts) to the host.
  std::vector<std::vector<int>> longdeg(G);
  for (int r = 0; r < G; ++r) {
    const int nl = bounds[8 * (size_t)r];
    if (nl > 0) {
      longdeg[r].resize(nl);
      GPR_CUDA(cudaMemcpyAsync(longdeg[r].data(), sdeg + g->ivoff[r], sizeof(int) * nl,
                               cudaMemcpyDeviceToHost, st));
    }
  }
  GPR_CUDA(cudaStreamSynchronize(st));
  // Unit descriptors: heavy units graph by graph, then the zero units.
  std::vector<int4> meta, zmeta;
  std::vector<int> hb(G + 1, 0), zb(G + 1, 0), gm(G);
  g->lazy_h.clear();
  for (int r = 0; r < G; ++r) {
    const int v0 = g->ivoff[r], mg = g->ivoff[r + 1] - v0;
    const int *b = bounds.data() + 8 * (size_t)r;
    gm[r] = mg;
    hb[r] = (int)meta.size();
    for (int i = 0; i < b[0]; ++i) {
      const long long p = ((long long)longdeg[r][i] + 3) & ~3LL;
      const int nc = (int)gpr::ceil_div(p, chunk[r]);
      const int cb = (int)meta.size();
      for (int k = 0; k < nc; ++k) meta.push_back(make_int4(v0 + i, cb, nc, r << 8 | kUnitChunk << 4));
    }
    for (int lw = 5; lw >= 0; --lw) {
      const int r0 = v0 + b[5 - lw], r1 = v0 + b[6 - lw];
      for (int x = r0; x < r1; x += 32 >> lw)
        meta.push_back(make_int4(x, 0, std::min(32 >> lw, r1 - x), r << 8 | kUnitSlice << 4 | lw));
    }
    hb[r + 1] = (int)meta.size();
    zb[r] = (int)zmeta.size();
    for (int x = v0 + b[6]; x < v0 + mg; x += gpr::kZeroRowsPerUnit)
      zmeta.push_back(make_int4(x, 0, std::min(gpr::kZeroRowsPerUnit, v0 + mg - x), r << 8 | kUnitZero << 4));
    zb[r + 1] = (int)zmeta.size();
    if (mg > 0 && hb[r + 1] == hb[r]) g->lazy_h.push_back(r);
  }
  if ((long long)meta.size() + (long long)zmeta.size() > 0x7fffffffLL) {
    gpr::set_error("gpr_multigraph_create: too many work units");
    return GPR_EINVAL;
  }
  g->n_heavy = (int)meta.size();
  g->n_zero = (int)zmeta.size();
  for (int &z : zb) z += g->n_heavy;
  meta.insert(meta.end(), zmeta.begin(), zmeta.end());
  const int U = (int)meta.size();
  GPR_TRY(gpr::dalloc(&g->meta, (size_t)U, "unit descriptors"));
  GPR_TRY(gpr::dalloc(&g->uoff, (size_t)U + 1, "unit offsets"));
  int *dchunk = nullptr;
  GPR_TRY(T.get(&dchunk, (size_t)G, "chunk sizes"));
  GPR_CUDA(cudaMemcpyAsync(g->meta, meta.data(), sizeof(int4) * (size_t)U, cudaMemcpyHostToDevice, st));
  GPR_CUDA(cudaMemcpyAsync(dchunk, chunk.data(), sizeof(int) * (size_t)G, cudaMemcpyHostToDevice, st));
  k_unit_lens<<<grid_for((long long)U + 1), 256, 0, st>>>(U, g->meta, sdeg, dchunk, g->uoff);
  GPR_CUDA(cudaGetLastError());
  {
    size_t tb = 0;
    GPR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, g->uoff, g->uoff, U + 1, st));
    void *tmp = nullptr;
    GPR_TRY(gpr::dmalloc(&tmp, tb, "scan scratch"));
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tb, g->uoff, g->uoff, U + 1, st);
    gpr::dfree(tmp);
    if (e != cudaSuccess) {
      gpr::set_error("unit offsets: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  }
  GPR_CUDA(cudaMemcpyAsync(&g->edge_slots, g->uoff + U, sizeof(long long), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  GPR_TRY(gpr::dalloc(&g->ecol, (size_t)g->edge_slots, "unit edges"));
  // Work packets: consecutive units of about equal cost (edge slots plus a
  // per-unit overhead; zero units by rows), about 32 grabs per warp per
  // sweep (measured on the 512-graph batch: 4 / 8 / 16 / 32 per warp ->
  // 256 / 282 / 292 / 294 GTEPS); heavy and zero units never share a packet.
  {
    std::vector<long long> uo((size_t)U + 1);
    GPR_CUDA(cudaMemcpyAsync(uo.data(), g->uoff, sizeof(long long) * uo.size(),
                             cudaMemcpyDeviceToHost, st));
    GPR_CUDA(cudaStreamSynchronize(st));
    auto cost = [&](int u) -> long long {
      const int kind = (meta[u].w >> 4) & 15;
      return kind == kUnitZero ? 4LL * meta[u].z : (uo[u + 1] - uo[u]) + 64;
    };
    long long total = 0;
    for (int u = 0; u < g->n_heavy; ++u) total += cost(u);
    int sms = 0;
    GPR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    const long long target = std::max<long long>(256, total / ((long long)sms * (kMultiBlock / 32) * 32));
    std::vector<int> pk;
    auto cut = [&](int b, int e) {
      long long c = 0;
      for (int u = b; u < e; ++u) {
        if (c == 0) pk.push_back(u);
        c += cost(u);
        if (c >= target) c = 0;
      }
    };
    cut(0, g->n_heavy);
    g->n_hpk = (int)pk.size();
    cut(g->n_heavy, U);
    g->n_pk = (int)pk.size();
    pk.push_back(U);
    GPR_TRY(gpr::dalloc(&g->pk, pk.size(), "work packets"));
    GPR_CUDA(cudaMemcpyAsync(g->pk, pk.data(), sizeof(int) * pk.size(), cudaMemcpyHostToDevice, st));
    GPR_CUDA(cudaStreamSynchronize(st));
  }
  if (U > 0) {
    k_fill_units<<<capped(32LL * U), 256, 0, st>>>(U, M, g->meta, g->uoff, dchunk, g->perm, inv,
                                                   sdeg, d_rowptr, d_col, g->ecol);
    GPR_CUDA(cudaGetLastError());
  }
  // Per-graph state.
  GPR_TRY(gpr::dalloc(&g->gm, (size_t)G, "graph sizes"));
  GPR_TRY(gpr::dalloc(&g->hb, (size_t)G + 1, "heavy ranges"));
  GPR_TRY(gpr::dalloc(&g->zb, (size_t)G + 1, "zero ranges"));
  GPR_TRY(gpr::dalloc(&g->cap, (size_t)G, "sweep caps"));
  GPR_TRY(gpr::dalloc(&g->stop, (size_t)G, "stop sweeps"));
  GPR_TRY(gpr::dalloc(&g->gdone, (size_t)G, "graph counters"));
  GPR_TRY(gpr::dalloc(&g->gres, (size_t)G, "graph residuals"));
  GPR_TRY(gpr::dalloc(&g->lazy, g->lazy_h.size(), "graphs without heavy units"));
  GPR_CUDA(cudaMemcpyAsync(g->gm, gm.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
  GPR_CUDA(cudaMemcpyAsync(g->hb, hb.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
  GPR_CUDA(cudaMemcpyAsync(g->zb, zb.data(), sizeof(int) * (G + 1), cudaMemcpyHostToDevice, st));
  if (!g->lazy_h.empty())
    GPR_CUDA(cudaMemcpyAsync(g->lazy, g->lazy_h.data(), sizeof(int) * g->lazy_h.size(),
                             cudaMemcpyHostToDevice, st));
  // Per-vertex and per-unit state.
  GPR_TRY(gpr::dalloc(&g->s, (size_t)M, "scores"));
  GPR_TRY(gpr::dalloc(&g->c0, (size_t)M + 4, "contrib0"));
  GPR_TRY(gpr::dalloc(&g->c1, (size_t)M + 4, "contrib1"));
  GPR_TRY(gpr::dalloc(&g->partial, (size_t)g->n_heavy, "chunk partials"));
  GPR_TRY(gpr::dalloc(&g->cnt, (size_t)g->n_heavy, "chunk counters"));
  GPR_TRY(gpr::dalloc(&g->uerr, (size_t)U, "unit residuals"));
  GPR_TRY(gpr::dalloc(&g->n_next, 2, "graph count"));
  GPR_TRY(gpr::dalloc(&g->bar, 2, "barrier"));
  GPR_TRY(gpr::dalloc(&g->status, 4, "status"));
  GPR_TRY(gpr::dalloc(&g->wq, 2, "work queue"));
  GPR_TRY(gpr::dalloc(&g->scores_tmp, (size_t)M, "score staging"));
  GPR_CUDA(cudaMemsetAsync(g->c0, 0, sizeof(float) * ((size_t)M + 4), st));
  GPR_CUDA(cudaMemsetAsync(g->c1, 0, sizeof(float) * ((size_t)M + 4), st));
  GPR_CUDA(cudaMemsetAsync(g->cnt, 0, sizeof(int) * (size_t)std::max(g->n_heavy, 1), st));
  g->device_bytes = 4LL * g->edge_slots + 16LL * U + 8LL * (U + 1) + 8LL * U + 8LL * g->n_heavy +
                    20LL * M;
  int sms = 0, coop = 0, per_sm = 0;
  GPR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  GPR_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device));
  g->coop_ok = coop != 0;
  for (int bf = 0; bf < 2; ++bf) {
    GPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, multi_kernel(bf), kMultiBlock, 0));
    if (per_sm < 1) g->coop_ok = false;
  }
  g->grid = (int)std::max<long long>(1, std::min<long long>(sms, gpr::ceil_div(U, 32)));
  GPR_CUDA(cudaStreamSynchronize(st));
  for (int r = 0; r < G; ++r) g->max_gm = std::max(g->max_gm, gm[r]);
  if (blo) {
    // Blocked form: the rows with in-edges of each graph (the first rows of
    // its range) in blocks of R rows, never spanning two graphs.
    std::vector<int> rb(G), re(G);
    long long rows = 0;
    for (int r = 0; r < G; ++r) {
      rb[r] = g->ivoff[r];
      re[r] = g->ivoff[r] + bounds[8 * (size_t)r + 6];
      rows += re[r] - rb[r];
    }
    const int R = blo->block_rows
                      ? blo->block_rows
                      : (int)std::min<long long>(gpr::kBlockedRows,
                                                 std::max<long long>(256, gpr::ceil_div(rows, 2LL * sms)));
    const int tile_words = blo->tile_words ? blo->tile_words : gpr::kTileWordsDefault;
    GPR_TRY(gpr::build_blocked_ranges(M, g->nnz, d_rowptr, d_col, g->perm, rb, re, R, tile_words,
                                      gpr::kRunWords, sms * gpr::blocked_ctas_per_sm(R), &g->B,
                                      st));
    const gpr::BlockedLayout &B = g->B;
    g->lazy_bh.clear();
    for (int r = 0; r < G; ++r)
      if (g->ivoff[r + 1] > g->ivoff[r] && B.range_tiles[r + 1] == B.range_tiles[r])
        g->lazy_bh.push_back(r);
    GPR_TRY(gpr::dalloc(&g->tb, (size_t)G + 1, "graph tile slots"));
    GPR_TRY(gpr::dalloc(&g->terr, (size_t)std::max(B.n_tiles, 1), "tile residuals"));
    GPR_TRY(gpr::dalloc(&g->lazy_b, std::max<size_t>(g->lazy_bh.size(), 1), "graphs without tiles"));
    GPR_TRY(gpr::dalloc(&g->tq, 2, "tile queue"));
    GPR_TRY(gpr::dalloc(&g->fx_max, 1, "largest score"));
    GPR_CUDA(cudaMemcpyAsync(g->tb, B.range_tiles.data(), sizeof(int) * ((size_t)G + 1),
                             cudaMemcpyHostToDevice, st));
    if (!g->lazy_bh.empty())
      GPR_CUDA(cudaMemcpyAsync(g->lazy_b, g->lazy_bh.data(), sizeof(int) * g->lazy_bh.size(),
                               cudaMemcpyHostToDevice, st));
    // CTAs per SM and the smallest carveout that holds them (as the
    // single-graph blocked kernel)
    int smem_sm = 0, per_bsm = 0;
    GPR_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, g->device));
    g->blocked_ctas = gpr::blocked_ctas_per_sm(B.R > 0 ? B.R : R);
    const int smem = 8 * std::max(B.R, 1);
    for (;;) {
      const void *k = multi_blocked_kernel(g->blocked_ctas);
      cudaFuncAttributes fa;
      GPR_CUDA(cudaFuncGetAttributes(&fa, k));
      const long long need = (long long)g->blocked_ctas * (smem + (long long)fa.sharedSizeBytes + 1024);
      const int carve = (int)std::min<long long>(100, gpr::ceil_div(100 * need, smem_sm));
      GPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      GPR_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
      GPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_bsm, k, 1024 / g->blocked_ctas, smem));
      if (per_bsm >= g->blocked_ctas || g->blocked_ctas == 1) break;
      g->blocked_ctas = 1;
    }
    g->grid_blocked = sms * g->blocked_ctas;
    g->blocked_ok = g->coop_ok && per_bsm >= g->blocked_ctas;
    g->has_blocked = true;
    g->device_bytes += B.device_bytes + 8LL * std::max(B.n_tiles, 1) + 4LL * (G + 1);
    GPR_CUDA(cudaStreamSynchronize(st));
  }
  return GPR_OK;
}

// One phase over all graphs with kernel precision bf; caps[r] per internal
// graph.  Reads back the sweeps (stop) and last residual of every graph.
int solve_phase(gpr_multigraph *g, float *d_scores, const gpr_pr_opts &o, bool bf,
                const std::vector<int> &caps, std::vector<int> *iters, std::vector<double> *res,
                gpr_pr_stats *out, bool blocked = false) {
  const int G = g->G, M = g->M;
  cudaStream_t st = g->st;
  if (bf && !g->h0) {
    GPR_TRY(gpr::dalloc(&g->h0, (size_t)M + 8, "bf16 contrib0"));
    GPR_TRY(gpr::dalloc(&g->h1, (size_t)M + 8, "bf16 contrib1"));
    GPR_CUDA(cudaMemsetAsync(g->h0, 0, 2 * ((size_t)M + 8), st));
    GPR_CUDA(cudaMemsetAsync(g->h1, 0, 2 * ((size_t)M + 8), st));
  }
  int max_cap = 0;
  for (int c : caps) max_cap = std::max(max_cap, c);
  GPR_CUDA(cudaMemsetAsync(g->bar, 0, 2 * sizeof(unsigned), st));
  GPR_CUDA(cudaMemsetAsync(g->status, 0, 4 * sizeof(int), st));
  GPR_CUDA(cudaMemsetAsync(g->wq, 0, 2 * sizeof(int), st));
  GPR_CUDA(cudaMemsetAsync(g->n_next, 0, 2 * sizeof(int), st));
  GPR_CUDA(cudaMemsetAsync(g->gdone, 0, sizeof(int) * G, st));
  GPR_CUDA(cudaMemsetAsync(g->gres, 0, sizeof(double) * G, st));
  GPR_CUDA(cudaMemsetAsync(g->cnt, 0, sizeof(int) * (size_t)std::max(g->n_heavy, 1), st));
  GPR_CUDA(cudaMemcpyAsync(g->cap, caps.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
  GPR_CUDA(cudaMemcpyAsync(g->stop, caps.data(), sizeof(int) * G, cudaMemcpyHostToDevice, st));
  MultiArgs a;
  memset(&a, 0, sizeof(a));
  a.M = M;
  a.G = G;
  a.n_heavy = g->n_heavy;
  a.n_zero = g->n_zero;
  a.meta = g->meta;
  a.uoff = g->uoff;
  a.ecol = g->ecol;
  a.outdeg = g->outdeg;
  a.gm = g->gm;
  a.hb = g->hb;
  a.zb = g->zb;
  a.cap = g->cap;
  a.stop = g->stop;
  a.gdone = g->gdone;
  a.gres = g->gres;
  a.lazy = g->lazy;
  a.n_lazy = (int)g->lazy_h.size();
  a.s = g->s;
  a.c0 = bf ? (void *)g->h0 : (void *)g->c0;
  a.c1 = bf ? (void *)g->h1 : (void *)g->c1;
  a.partial = g->partial;
  a.cnt = g->cnt;
  a.uerr = g->uerr;
  a.n_next = g->n_next;
  a.bar = g->bar;
  a.status = g->status;
  a.wq = g->wq;
  a.damp = o.damping;
  a.tol = o.tol;
  a.max_iter = max_cap;
  a.bar_expect = g->grid + (o.reserved[0] > 0 ? o.reserved[0] : 0);
  a.pk = g->pk;
  a.n_hpk = g->n_hpk;
  a.n_pk = g->n_pk;
  a.timeout_ns = (long long)(o.timeout_s * 1e9);
  a.cond = 0;
  if (blocked) {
    const gpr::BlockedLayout &B = g->B;
    GPR_CUDA(cudaMemsetAsync(g->tq, 0, 2 * sizeof(int), st));
    GPR_CUDA(cudaMemsetAsync(g->fx_max, 0, sizeof(unsigned), st));
    if (B.n_blocks) {
      // clean after an abandoned solve; a completed sweep leaves them clean
      GPR_CUDA(cudaMemsetAsync(B.bcnt, 0, sizeof(int) * B.n_blocks, st));
      GPR_CUDA(cudaMemsetAsync(B.gacc, 0, 8 * (size_t)B.gacc_rows, st));
    }
    // Fixed-point exponent from the largest initial score: every graph's
    // total |score| stays at most max(1, m_g max|s0|) <= B0 (as gpr_pagerank).
    k_multi_max_abs<<<std::min<long long>(grid_for(M), 148 * 8), 256, 0, st>>>(M, d_scores, g->fx_max);
    GPR_CUDA(cudaGetLastError());
    unsigned bits = 0;
    GPR_CUDA(cudaMemcpyAsync(&bits, g->fx_max, sizeof(bits), cudaMemcpyDeviceToHost, st));
    GPR_CUDA(cudaStreamSynchronize(st));
    float mx;
    memcpy(&mx, &bits, sizeof(mx));
    if (!isfinite(mx)) return kMultiBlockedFallback;
    const double b0 = std::max(1.0, (double)g->max_gm * (double)mx);
    const int cap = 62 - (int)ceil(log2(b0));
    const int pref = (int)floor(log2(std::max(1.0, (double)g->nnz) / b0)) + 28;
    const int S = std::min(cap, std::max(31, pref));
    a.fx_scale = ldexpf(1.f, S);
    a.fx_inv = ldexp(1.0, -S);
    a.tb = g->tb;
    a.terr = g->terr;
    a.n_tiles = B.n_tiles;
    a.acc_rows = B.R;
    a.blk_row0 = B.row0;
    a.tiles = B.tiles;
    a.blocks = B.blocks;
    a.runs = B.runs;
    a.entry = B.entry;
    a.gacc = B.gacc;
    a.bcnt = B.bcnt;
    a.tq = g->tq;
    a.lazy = g->lazy_b;
    a.n_lazy = (int)g->lazy_bh.size();
    a.bar_expect = g->grid_blocked + (o.reserved[0] > 0 ? o.reserved[0] : 0);
  }
  // Graph mode when asked for, or when the persistent kernel cannot be
  // co-resident: the sweep loop as a CUDA-graph while node whose body is one
  // k_multi_step launch, built here and released after the phase.
  const bool graph_mode = !blocked && (o.loop == GPR_LOOP_GRAPH || !g->coop_ok);
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  if (max_cap > 0 && graph_mode) {
    cudaGraphConditionalHandle h = 0;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t cn = nullptr, kn = nullptr;
    cudaError_t e = cudaGraphCreate(&graph, 0);
    if (e == cudaSuccess)
      e = cudaGraphConditionalHandleCreate(&h, graph, 1u, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&cn, graph, nullptr, 0, &cp);
    }
    MultiArgs ac = a;
    ac.cond = h;
    void *kargs[] = {&ac};
    cudaKernelNodeParams kp;
    memset(&kp, 0, sizeof(kp));
    kp.func = const_cast<void *>(multi_step_kernel(bf));
    kp.gridDim = dim3(g->grid);
    kp.blockDim = dim3(kMultiBlock);
    kp.kernelParams = kargs;
    if (e == cudaSuccess) e = cudaGraphAddKernelNode(&kn, cp.conditional.phGraph_out[0], nullptr, 0, &kp);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
      if (exec) cudaGraphExecDestroy(exec);
      if (graph) cudaGraphDestroy(graph);
      gpr::set_error("multi-graph loop graph: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  }
  int launches = 0;
  GPR_CUDA(cudaEventRecord(g->e0, st));
  if (bf)
    k_multi_prologue<bf16><<<grid_for((long long)M + 1), 256, 0, st>>>(M, g->perm, g->outdeg,
                                                                       d_scores, g->s, g->h0, g->h1);
  else
    k_multi_prologue<float><<<grid_for((long long)M + 1), 256, 0, st>>>(M, g->perm, g->outdeg,
                                                                        d_scores, g->s, g->c0, g->c1);
  ++launches;
  GPR_CUDA(cudaEventRecord(g->e2, st));
  if (max_cap > 0 && graph_mode) {
    cudaError_t e = cudaGraphLaunch(exec, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      gpr::set_error("multi-graph loop graph: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  } else if (max_cap > 0 && blocked) {
    void *args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel(
        multi_blocked_kernel(g->blocked_ctas), dim3(g->grid_blocked),
        dim3(1024 / g->blocked_ctas), args, 8 * (size_t)g->B.R, st);
    if (e == cudaErrorCooperativeLaunchTooLarge) {
      cudaGetLastError();
      return kMultiBlockedFallback;
    }
    if (e != cudaSuccess) {
      gpr::set_error("multi-graph cooperative launch: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
    ++launches;
  } else if (max_cap > 0) {
    void *args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel(multi_kernel(bf), dim3(g->grid), dim3(kMultiBlock),
                                                args, 0, st);
    if (e != cudaSuccess) {
      gpr::set_error("multi-graph cooperative launch: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
    ++launches;
  }
  GPR_CUDA(cudaEventRecord(g->e3, st));
  k_multi_scatter<<<grid_for(M), 256, 0, st>>>(M, g->perm, g->s, d_scores);
  ++launches;
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaEventRecord(g->e1, st));
  int hs[4];
  iters->assign(G, 0);
  res->assign(G, 0.0);
  GPR_CUDA(cudaMemcpyAsync(hs, g->status, sizeof(hs), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaMemcpyAsync(iters->data(), g->stop, sizeof(int) * G, cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaMemcpyAsync(res->data(), g->gres, sizeof(double) * G, cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f, lms = 0.f;
  GPR_CUDA(cudaEventElapsedTime(&ms, g->e0, g->e1));
  GPR_CUDA(cudaEventElapsedTime(&lms, g->e2, g->e3));
  memset(out, 0, sizeof(*out));
  out->iterations = max_cap > 0 ? hs[1] : 0;
  out->solve_ms = ms;
  out->loop_ms = lms;
  out->gpu_launches = launches + (max_cap > 0 && graph_mode ? hs[3] : 0) + (blocked ? 1 : 0);
  double rmax = 0.0;
  for (double r : *res) rmax = std::max(rmax, r);
  out->residual = rmax;
  if (hs[0] & 1) {
    gpr::set_error("grid barrier wait exceeded %.3f s (sweep loop abandoned)", o.timeout_s);
    return GPR_ETIMEOUT;
  }
  return GPR_OK;
}

int multi_pagerank_impl(gpr_multigraph *g, float *any_scores, const gpr_pr_opts *opts_in,
                        int *h_iters, double *h_res, gpr_pr_stats *stats) {
  gpr_pr_opts o;
  if (opts_in) o = *opts_in;
  else gpr_pr_opts_default(&o);
  if (!(o.damping >= 0.f && o.damping <= 1.f) || o.max_iter < 0 || !(o.tol >= 0.0) ||
      !(o.timeout_s > 0.0)) {
    gpr::set_error("gpr_multigraph_pagerank: invalid options");
    return GPR_EINVAL;
  }
  if (o.precision != GPR_PREC_FP32 && o.precision != GPR_PREC_BF16) {
    gpr::set_error("gpr_multigraph_pagerank: precision %d not supported", o.precision);
    return GPR_EUNSUPPORTED;
  }
  if (o.form != GPR_FORM_AUTO && o.form != GPR_FORM_EXACT && o.form != GPR_FORM_BLOCKED) {
    gpr::set_error("gpr_multigraph_pagerank: unknown form %d", o.form);
    return GPR_EINVAL;
  }
  if (o.form == GPR_FORM_BLOCKED) {
    if (!g->has_blocked) {
      gpr::set_error("gpr_multigraph_pagerank: GPR_FORM_BLOCKED needs a batch created with "
                     "GPR_LAYOUT_BLOCKED");
      return GPR_EINVAL;
    }
    if (o.precision != GPR_PREC_FP32 || o.loop == GPR_LOOP_GRAPH || !g->blocked_ok) {
      gpr::set_error("gpr_multigraph_pagerank: GPR_FORM_BLOCKED runs FP32 in the persistent "
                     "loop only");
      return GPR_EUNSUPPORTED;
    }
  }
  const bool use_blocked = o.precision == GPR_PREC_FP32 && g->has_blocked && g->blocked_ok &&
                           o.loop != GPR_LOOP_GRAPH && o.form != GPR_FORM_EXACT &&
                           (o.form == GPR_FORM_BLOCKED || g->nnz >= gpr::kBlockedAutoMinEdges);
  gpr_pr_stats sl;
  memset(&sl, 0, sizeof(sl));
  const int G = g->G, M = g->M;
  // a graph with no vertices runs empty sweeps with residual 0
  const int empty_sweeps = gpr::empty_graph_sweeps(o.tol, o.max_iter);
  if (M == 0) {
    if (stats) *stats = sl;
    if (h_iters) for (int ug = 0; ug < G; ++ug) h_iters[ug] = empty_sweeps;
    if (h_res) memset(h_res, 0, sizeof(double) * G);
    return GPR_OK;
  }
  if (!any_scores) {
    gpr::set_error("gpr_multigraph_pagerank: NULL scores");
    return GPR_EINVAL;
  }
  cudaStream_t st = g->st;
  float *d_scores = any_scores;
  const bool host = !gpr::is_device_ptr(any_scores);
  if (host) {
    d_scores = g->scores_tmp;
    GPR_CUDA(cudaMemcpyAsync(d_scores, any_scores, sizeof(float) * (size_t)M,
                             cudaMemcpyHostToDevice, st));
  }
  std::vector<int> caps(G), it1, it2;
  std::vector<double> r1, r2;
  for (int r = 0; r < G; ++r) caps[r] = g->ivoff[r + 1] > g->ivoff[r] ? o.max_iter : 0;
  int rc;
  std::vector<int> refine(G, 0);
  if (o.precision == GPR_PREC_FP32) {
    rc = use_blocked ? solve_phase(g, d_scores, o, false, caps, &it1, &r1, &sl, true)
                     : kMultiBlockedFallback;
    if (rc == kMultiBlockedFallback) {
      if (o.form == GPR_FORM_BLOCKED) {
        gpr::set_error("gpr_multigraph_pagerank: GPR_FORM_BLOCKED needs finite scores and a "
                       "co-resident grid");
        rc = GPR_EINVAL;
      } else {
        rc = solve_phase(g, d_scores, o, false, caps, &it1, &r1, &sl);
      }
    }
  } else {
    gpr_pr_opts o1 = o;
    o1.tol = std::max(o.tol, kBf16Tol);
    gpr_pr_stats s1, s2;
    rc = solve_phase(g, d_scores, o1, true, caps, &it1, &r1, &s1);
    if (rc == GPR_OK) {
      std::vector<int> caps2(G);
      for (int r = 0; r < G; ++r) caps2[r] = caps[r] > 0 ? std::max(0, o.max_iter - it1[r]) : 0;
      rc = solve_phase(g, d_scores, o, false, caps2, &it2, &r2, &s2);
      if (rc == GPR_OK) {
        for (int r = 0; r < G; ++r) {
          refine[r] = it2[r];
          if (it2[r] == 0) r2[r] = r1[r];
          it1[r] += it2[r];
        }
        r1 = r2;
        sl = s2;
        sl.iterations = s1.iterations + s2.iterations;
        sl.refine_iterations = s2.iterations;
        sl.solve_ms = s1.solve_ms + s2.solve_ms;
        sl.loop_ms = s1.loop_ms + s2.loop_ms;
        sl.gpu_launches = s1.gpu_launches + s2.gpu_launches;
      }
    }
  }
  if (rc == GPR_OK && host)
    GPR_CUDA(cudaMemcpy(any_scores, d_scores, sizeof(float) * (size_t)M, cudaMemcpyDeviceToHost));
  if (rc == GPR_OK) {
    for (int ug = 0; ug < G; ++ug) {
      const int r = g->rank[ug];
      if (h_iters) h_iters[ug] = g->ivoff[r + 1] > g->ivoff[r] ? it1[r] : empty_sweeps;
      if (h_res) h_res[ug] = r1[r];
    }
  }
  if (stats) *stats = sl;
  return rc;
}

}  // namespace

extern "C" {

int gpr_multigraph_create(int n_graphs, const int *h_voff, long long nnz, const int *any_rowptr,
                          const int *any_col, const int *any_outdeg,
                          const gpr_layout_opts *h_lopts, gpr_multigraph **out) {
  GPR_ENTRY_BEGIN
  if (!out) {
    gpr::set_error("gpr_multigraph_create: NULL out");
    return GPR_EINVAL;
  }
  *out = nullptr;
  if (n_graphs < 1 || !h_voff || h_voff[0] != 0 || nnz < 0 || nnz > 0x7fffffffLL) {
    gpr::set_error("gpr_multigraph_create: invalid arguments (n_graphs=%d, nnz=%lld)", n_graphs, nnz);
    return GPR_EINVAL;
  }
  for (int g = 0; g < n_graphs; ++g)
    if (h_voff[g + 1] < h_voff[g]) {
      gpr::set_error("gpr_multigraph_create: vertex offsets decrease at graph %d", g);
      return GPR_EINVAL;
    }
  if (h_lopts)
    for (int g = 0; g < n_graphs; ++g) {
      const gpr_layout_opts &l = h_lopts[g];
      if (l.sell_max < 0 || l.sell_max > 1024 || l.chunk < 0 || l.chunk % 128 != 0 ||
          l.chunk_min < 0) {
        gpr::set_error("gpr_multigraph_create: invalid layout options of graph %d", g);
        return GPR_EINVAL;
      }
    }
  const int M = h_voff[n_graphs];
  if ((M > 0 && (!any_rowptr || !any_outdeg)) || (nnz > 0 && !any_col)) {
    gpr::set_error("gpr_multigraph_create: NULL arrays");
    return GPR_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    gpr::set_error("gpr_multigraph_create: no CUDA device");
    return GPR_ENODEV;
  }
  gpr_multigraph *g = new gpr_multigraph();
  g->G = n_graphs;
  g->M = M;
  g->nnz = nnz;
  int rc = GPR_OK;
  void *rp = nullptr, *cp = nullptr, *dp = nullptr;
  bool orp = false, ocp = false, odp = false;
  do {
    if (cudaGetDevice(&g->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&g->e0) != cudaSuccess || cudaEventCreate(&g->e1) != cudaSuccess ||
        cudaEventCreate(&g->e2) != cudaSuccess || cudaEventCreate(&g->e3) != cudaSuccess) {
      gpr::set_error("gpr_multigraph_create: stream / event creation failed");
      rc = GPR_ECUDA;
      break;
    }
    g->own_stream = true;
    rc = gpr::to_device(any_rowptr, sizeof(int) * ((size_t)M + 1), &rp, &orp, g->st, "rowptr");
    if (rc == GPR_OK) rc = gpr::to_device(any_col, sizeof(int) * (size_t)nnz, &cp, &ocp, g->st, "col");
    if (rc == GPR_OK)
      rc = gpr::to_device(any_outdeg, sizeof(int) * (size_t)M, &dp, &odp, g->st, "outdeg");
    if (rc == GPR_OK)
      rc = gpr::validate_csr(M, nnz, M, (const int *)rp, (const int *)cp, (const int *)dp, g->st);
    if (rc == GPR_OK && M > 0)
      rc = build_multi(g, h_voff, (const int *)rp, (const int *)cp, (const int *)dp, h_lopts);
    const cudaError_t se = cudaStreamSynchronize(g->st);
    if (rc == GPR_OK && se != cudaSuccess) {
      gpr::set_error("gpr_multigraph_create: %s", cudaGetErrorString(se));
      rc = GPR_ECUDA;
    }
  } while (0);
  if (orp) gpr::dfree(rp);
  if (ocp) gpr::dfree(cp);
  if (odp) gpr::dfree(dp);
  if (rc != GPR_OK) {
    destroy_multi(g);
    return rc;
  }
  *out = g;
  return GPR_OK;
  GPR_ENTRY_END("gpr_multigraph_create")
}

int gpr_multigraph_destroy(gpr_multigraph *g) {
  destroy_multi(g);
  return GPR_OK;
}

int gpr_multigraph_info(const gpr_multigraph *g, int *n_graphs, int *m, long long *nnz,
                        int *n_units, long long *edge_slots) {
  if (!g) {
    gpr::set_error("gpr_multigraph_info: NULL handle");
    return GPR_EINVAL;
  }
  if (n_graphs) *n_graphs = g->G;
  if (m) *m = g->M;
  if (nnz) *nnz = g->nnz;
  if (n_units) *n_units = g->n_heavy + g->n_zero;
  if (edge_slots) *edge_slots = g->edge_slots;
  return GPR_OK;
}

int gpr_multigraph_set_stream(gpr_multigraph *g, void *stream) {
  if (!g) {
    gpr::set_error("gpr_multigraph_set_stream: NULL handle");
    return GPR_EINVAL;
  }
  if (g->own_stream && g->st) cudaStreamDestroy(g->st);
  g->own_stream = false;
  g->st = (cudaStream_t)stream;
  return GPR_OK;
}

int gpr_multigraph_pagerank(gpr_multigraph *g, float *any_scores, const gpr_pr_opts *opts,
                            int *h_iters, double *h_residuals, gpr_pr_stats *stats) {
  GPR_ENTRY_BEGIN
  if (!g) {
    gpr::set_error("gpr_multigraph_pagerank: NULL handle");
    return GPR_EINVAL;
  }
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != g->device) GPR_CUDA(cudaSetDevice(g->device));
  int rc = multi_pagerank_impl(g, any_scores, opts, h_iters, h_residuals, stats);
  if (cur != g->device && cur >= 0) cudaSetDevice(cur);
  return rc;
  GPR_ENTRY_END("gpr_multigraph_pagerank")
}

}  // extern "C"
