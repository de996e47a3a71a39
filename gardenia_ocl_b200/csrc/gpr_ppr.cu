// Batched personalized PageRank: k seed vectors solved together as a fused
// pull-SpMM, all sweeps in one persistent cooperative launch or (loop
// GPR_LOOP_GRAPH) one launch per sweep inside a CUDA-graph while loop.
//
// No reference file: the reference computes one global PageRank
// (src/pr/omp_base.cc).  For each vector q with seed s_q:
//   x_new[v][q] = d * sum_{u in in(v)} x[u][q] / outdeg[u]
//               + [v == s_q] * ((1 - d) + d * dangling_q)
//   dangling_q  = sum over out-degree-0 vertices u of x[u][q]   (FP64)
// x starts at e_{s_q}; vector q stops updating after the first sweep whose
// FP64 L1 change is below tol (oracle/oracle.c orc_ppr_f64 restates this).
//
// Layout: the graph's relabelled CSR (descending in-degree), x[m][K] FP32,
// contributions c[m+1][K] in FP32 or BF16 (double-buffered by sweep parity,
// row m is a zero sentinel), K = the vector count rounded up to 8..128.  One
// gather of an in-neighbour's row serves all K vectors, so the 4-byte index
// stream and the per-request cost are shared by K edge-vector pairs.
//   lanes per row L = K / 4, rows per warp R = 32 / L, components per lane
//   C = 4 (contiguous, one vector load per gather), so one warp-wide load
//   instruction serves R rows and 8 gathers per lane are in flight.
// Rows with in-degree 0 hold x = 0 except at seeds, so only rows with
// in-edges and the k seed rows are updated.  Rows longer than 8 sub-group
// rounds are cut into chunks of 8192 / L edges whose K-wide partial sums the
// last arriving warp adds in a fixed order; the other rows go in groups of R.
// Warps take packets (runs of these units of about equal cost) from one
// queue.  Residual and dangling sums are reduced per CTA and then over CTAs
// in CTA order by the last CTA to finish the sweep (deterministic); every
// barrier wait is bounded.
#include <cub/cub.cuh>
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpr_device.cuh"
#include "gpr_internal.cuh"
#include "gpr_guard.h"

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kPprBlock = 256;

struct PprArgs {
  int m, n_long, n_nz, n_chunks, k, n_pk;
  const int *csr_ptr, *csr_col, *row_cbeg, *outdeg;
  const int4 *cdesc;     // [n_chunks] {row, first edge, end edge, first chunk of the row or -1}
  const int *pk;         // [n_pk + 1] first unit of each packet
  float *x;              // [m][K]
  void *c0, *c1;         // [m+1][K] of T
  float *partial;        // [n_chunks][K]
  int *cnt;              // [n_long]
  const int *seed;       // [K] relabelled seed vertex (-1: padding vector)
  double *cta_red;       // [2][G][K]: residual, dangling
  double *seed_red;      // [2][K]: residual, dangling of in-degree-0 seed rows
  double *res_hist;      // [max_iter][K]
  double *dang;          // [2][K] dangling mass of the current iterate, by parity
  unsigned *active;      // [2][4] bit q: vector q still updating, by parity
  int *iters;            // [K]
  unsigned *bar;         // [2] arrivals, generation
  int *status;           // [0] error flags, [1] sweeps, [2] 1: vectors still updating,
                         // 2: stopped for packing (at most repack_below still updating)
  int *wq;               // [2] packet-queue heads by sweep parity
  float damp;
  double tol;
  int max_iter, bar_expect;
  int repack_below;      // > 0: stop once at most this many vectors are still updating
  long long timeout_ns;
  unsigned long long cond;  // graph mode: while-node condition handle (0: none)
};

// Lanes per row L = K / 4, rows per warp R = 32 / L, components per lane
// C = 4 (one 16-byte FP32 or 8-byte BF16 load per gather): K=8 -> 2x16,
// 16 -> 4x8, 32 -> 8x4, 64 -> 16x2, 128 -> 32x1.  Each lane loads P column
// indices per round, so a sub-group covers E = L * P >= 8 edges per round and
// every lane has 8 gathers in flight: P = 4, 2, 1, 1, 1.
template <int K>
struct Shape {
  static constexpr int L = K / 4;
  static constexpr int R = 32 / L;
  static constexpr int C = 4;
  static constexpr int P = L >= 8 ? 1 : 8 / L;
  static constexpr int E = L * P;
  // Early fetch: each row's scores and out-degree (and the next row group's
  // offsets) are loaded before its gathers.  It pays where a warp updates
  // several rows at once (K <= 32: 4-16 rows per warp; measured on RMAT s22
  // +15% at K = 8, +8% at K = 32); at K >= 64 the extra registers cost more
  // occupancy than the overlap gains (-28% at K = 128).
  static constexpr bool early = K <= 32;
  // Co-resident 256-thread CTAs per SM the register budget is held to:
  // K <= 16 trades a few spills for 24 warps instead of 16 (+8% at K = 8,
  // 4 CTAs lost 3%); K = 32 and 64 fit 2 without spills (3 gained nothing);
  // K = 128 fits 4.
  static constexpr int min_ctas = K <= 16 ? 3 : K <= 64 ? 2 : 4;
};

using gpr::dev::global_ns;
using gpr::dev::ld_acquire;

__device__ __forceinline__ int ld_idx(const int *p) {
  int v;
  asm("ld.global.nc.L1::no_allocate.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// C consecutive components of one contribution row, widened to float.
template <int C>
__device__ __forceinline__ void load_row(const float *p, float (&v)[C]) {
  if constexpr (C == 1) {
    asm volatile("ld.global.f32 %0, [%1];" : "=f"(v[0]) : "l"(p));
  } else if constexpr (C == 2) {
    asm volatile("ld.global.v2.f32 {%0,%1}, [%2];" : "=f"(v[0]), "=f"(v[1]) : "l"(p));
  } else {
    asm volatile("ld.global.v4.f32 {%0,%1,%2,%3}, [%4];"
                 : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]) : "l"(p));
  }
}

template <int C>
__device__ __forceinline__ void load_row(const __nv_bfloat16 *p, float (&v)[C]) {
  if constexpr (C == 1) {
    unsigned short h;
    asm volatile("ld.global.u16 %0, [%1];" : "=h"(h) : "l"(p));
    v[0] = __uint_as_float((unsigned)h << 16);
  } else if constexpr (C == 2) {
    unsigned w;
    asm volatile("ld.global.u32 %0, [%1];" : "=r"(w) : "l"(p));
    v[0] = __uint_as_float(w << 16);
    v[1] = __uint_as_float(w & 0xffff0000u);
  } else {
    unsigned w0, w1;
    asm volatile("ld.global.v2.u32 {%0,%1}, [%2];" : "=r"(w0), "=r"(w1) : "l"(p));
    v[0] = __uint_as_float(w0 << 16);
    v[1] = __uint_as_float(w0 & 0xffff0000u);
    v[2] = __uint_as_float(w1 << 16);
    v[3] = __uint_as_float(w1 & 0xffff0000u);
  }
}

__device__ __forceinline__ void store_c(float *p, float v) { *p = v; }
__device__ __forceinline__ void store_c(__nv_bfloat16 *p, float v) { *p = __float2bfloat16_rn(v); }

__device__ __forceinline__ bool is_active(const unsigned (&act)[4], int q) {
  return (act[q >> 5] >> (q & 31)) & 1u;
}

// Sums in-neighbour rows over `niter` rounds; niter is warp-uniform.  In
// round j this lane's sub-group covers edges [first + j*stride, +E) clipped
// to `end`: lane lq holds the indices of edges lq + p*L (p < P), the
// sub-group broadcasts them, and every lane gathers its C components of each
// row.  Edges past the sub-group's end (or lanes with no live component)
// gather the zero sentinel row, so every shuffle runs on the full warp.
template <int K, typename T>
__device__ __forceinline__ void gather_edges(const PprArgs &a, const T *cin, long long first,
                                             long long end, long long stride, int niter, int lq,
                                             bool live, float (&acc)[Shape<K>::C]) {
  constexpr int L = Shape<K>::L, C = Shape<K>::C, P = Shape<K>::P, E = Shape<K>::E;
  constexpr int UB = 8;  // gathers in flight per lane
  int nxt[P];
#pragma unroll
  for (int p = 0; p < P; ++p)
    nxt[p] = (niter > 0 && first + lq + p * L < end) ? ld_idx(a.csr_col + first + lq + p * L) : a.m;
  for (int j = 0; j < niter; ++j) {
    const long long eb = first + (long long)j * stride;
    int my[P];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      my[p] = nxt[p];
      // next round's indices are in flight while this round gathers
      const long long en = eb + stride + lq + p * L;
      nxt[p] = (j + 1 < niter && en < end) ? ld_idx(a.csr_col + en) : a.m;
    }
    const int ng = (int)max(0LL, min((long long)E, end - eb));
    const int nmax = (int)__reduce_max_sync(kFull, (unsigned)ng);
    if constexpr (P == 1) {
      for (int t0 = 0; t0 < nmax; t0 += UB) {
        float v[UB][C];
#pragma unroll
        for (int t = 0; t < UB; ++t) {
          const int u = __shfl_sync(kFull, my[0], (t0 + t) & (L - 1), L);
          const int uu = (t0 + t < ng && live) ? u : a.m;
          load_row<C>(cin + (size_t)uu * K + lq * C, v[t]);
        }
#pragma unroll
        for (int t = 0; t < UB; ++t)
#pragma unroll
          for (int c = 0; c < C; ++c) acc[c] += v[t][c];
      }
    } else {
      static_assert(E == UB, "one block of gathers per round");
      float v[UB][C];
#pragma unroll
      for (int t = 0; t < UB; ++t) {
        const int u = __shfl_sync(kFull, my[t / L], t % L, L);
        const int uu = (t < ng && live) ? u : a.m;
        if (t < nmax) {
          load_row<C>(cin + (size_t)uu * K + lq * C, v[t]);
        } else {
#pragma unroll
          for (int c = 0; c < C; ++c) v[t][c] = 0.f;
        }
      }
#pragma unroll
      for (int t = 0; t < UB; ++t)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] += v[t][c];
    }
  }
}

// Out-degree and current scores (this lane's C components) of row v, issued
// before the row's gathers so that they are in flight together.
template <int K>
__device__ __forceinline__ void row_fetch(const PprArgs &a, int v, int lq, int &od,
                                          float (&xo)[Shape<K>::C]) {
  static_assert(Shape<K>::C == 4, "one 16-byte load of x");
  asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(od) : "l"(a.outdeg + v));
  asm volatile("ld.global.v4.f32 {%0,%1,%2,%3}, [%4];"
               : "=f"(xo[0]), "=f"(xo[1]), "=f"(xo[2]), "=f"(xo[3])
               : "l"(a.x + (size_t)v * K + lq * 4));
}

// Update of row v from its pulled sums (acc) for this lane's components;
// od and xo from row_fetch, sd the lane's seed vertices.
template <int K, typename T>
__device__ __forceinline__ void row_update(const PprArgs &a, T *cout, int v, int lq,
                                           const unsigned (&act)[4], const double *dang_cur,
                                           const int (&sd)[Shape<K>::C],
                                           const float (&acc)[Shape<K>::C], int od,
                                           const float (&xo)[Shape<K>::C],
                                           double (&err)[Shape<K>::C], double (&dng)[Shape<K>::C]) {
  constexpr int C = Shape<K>::C;
  const float inv = od > 0 ? 1.0f / (float)od : 0.f;
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const int q = lq * C + c;
    if (!is_active(act, q)) continue;
    float xn = a.damp * acc[c];
    if (sd[c] == v) xn += (float)((1.0 - (double)a.damp) + (double)a.damp * dang_cur[q]);
    const size_t o = (size_t)v * K + q;
    a.x[o] = xn;
    err[c] += fabs((double)xn - (double)xo[c]);
    store_c(cout + o, od > 0 ? xn * inv : 0.f);
    if (od == 0) dng[c] += (double)xn;
  }
}

// One sweep of this CTA's share: packets of units, the seed rows without
// in-edges, and the CTA's residual and dangling sums (per vector, warps in
// order) into cta_red.  Ends with the CTA synchronised.
template <int K, typename T>
__device__ __forceinline__ void ppr_sweep(const PprArgs &a, int it, const int (&sd)[Shape<K>::C],
                                          double *s_red) {
  constexpr int L = Shape<K>::L, R = Shape<K>::R, C = Shape<K>::C, E = Shape<K>::E;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int g = lane / L, lq = lane % L;
  const int G = gridDim.x;
  const T *cin = reinterpret_cast<const T *>((it & 1) ? a.c1 : a.c0);
  T *cout = reinterpret_cast<T *>((it & 1) ? a.c0 : a.c1);
  const double *dang_cur = a.dang + (it & 1) * K;
  unsigned act[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) act[i] = __ldcg(a.active + (it & 1) * 4 + i);
  bool live = false;
#pragma unroll
  for (int c = 0; c < C; ++c) live |= is_active(act, lq * C + c);
  double err[C], dng[C];
#pragma unroll
  for (int c = 0; c < C; ++c) err[c] = dng[c] = 0.0;
  // Warps take packets (runs of units of about equal cost) from one queue;
  // units [0, n_chunks) are chunks of long rows, the rest groups of R rows.
  for (;;) {
    int p = 0;
    if (lane == 0) p = atomicAdd(a.wq + (it & 1), 1);
    p = __shfl_sync(kFull, p, 0);
    if (p >= a.n_pk) break;
    const int u1 = __ldg(a.pk + p + 1);
    int u = __ldg(a.pk + p);
    for (; u < u1 && u < a.n_chunks; ++u) {
      float acc[C], xo[C];
      int od = 0;
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = 0.f;
      const int4 d = __ldg(a.cdesc + u);
      const int r = d.x, cb = d.w;
      const long long b = d.y, e = d.z;
      if (Shape<K>::early && cb < 0) row_fetch<K>(a, r, lq, od, xo);  // the row's only chunk
      const int niter = (int)gpr::ceil_div(e - b, (long long)R * E);
      gather_edges<K, T>(a, cin, b + (long long)g * E, e, (long long)R * E, niter, lq, live,
                         acc);
#pragma unroll
      for (int o = L; o < 32; o <<= 1)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] += __shfl_xor_sync(kFull, acc[c], o);
      if (cb < 0) {
        if (!Shape<K>::early) row_fetch<K>(a, r, lq, od, xo);
        if (g == 0) row_update<K, T>(a, cout, r, lq, act, dang_cur, sd, acc, od, xo, err, dng);
        continue;
      }
      if (g == 0)
#pragma unroll
        for (int c = 0; c < C; ++c) a.partial[(size_t)u * K + lq * C + c] = acc[c];
      __threadfence();
      __syncwarp();
      const int nc = __ldg(a.row_cbeg + r + 1) - cb;
      int last = 0;
      if (lane == 0) last = atomicAdd(a.cnt + r, 1) == nc - 1;
      last = __shfl_sync(kFull, last, 0);
      if (!last) continue;
      __threadfence();
      // Sum the row's chunk partials in chunk order (sub-group 0).
      row_fetch<K>(a, r, lq, od, xo);
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = 0.f;
      for (int q = 0; q < nc; ++q)
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] += __ldcg(a.partial + (size_t)(cb + q) * K + lq * C + c);
      if (lane == 0) atomicExch(a.cnt + r, 0);
      if (g == 0) row_update<K, T>(a, cout, r, lq, act, dang_cur, sd, acc, od, xo, err, dng);
    }
    if (u >= u1) continue;
    // Row groups; with the early fetch, the next group's row offsets are
    // in flight while this group gathers.
    int v = a.n_long + (u - a.n_chunks) * R + g;
    int p0 = 0, p1 = 0;
    if (Shape<K>::early && v < a.n_nz) {
      p0 = a.csr_ptr[v];
      p1 = a.csr_ptr[v + 1];
    }
    for (; u < u1; ++u, v += R) {
      const bool has = v < a.n_nz;
      if (!Shape<K>::early) {
        p0 = has ? a.csr_ptr[v] : 0;
        p1 = has ? a.csr_ptr[v + 1] : 0;
      }
      const long long e0 = p0, e1 = p1;
      if (Shape<K>::early) {
        if (u + 1 < u1 && v + R < a.n_nz) {
          asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(p0) : "l"(a.csr_ptr + v + R));
          asm volatile("ld.global.nc.s32 %0, [%1];" : "=r"(p1) : "l"(a.csr_ptr + v + R + 1));
        } else {
          p0 = p1 = 0;
        }
      }
      float acc[C], xo[C];
      int od = 0;
#pragma unroll
      for (int c = 0; c < C; ++c) acc[c] = 0.f;
      if (Shape<K>::early && has) row_fetch<K>(a, v, lq, od, xo);
      // Rows of one warp have nearly equal degrees (degree order); the
      // sub-groups loop to the warp's longest row.
      long long span = e1 - e0;
#pragma unroll
      for (int o = L; o < 32; o <<= 1) span = max(span, __shfl_xor_sync(kFull, span, o));
      gather_edges<K, T>(a, cin, e0, e1, (long long)E, (int)gpr::ceil_div(span, E), lq,
                         live && has, acc);
      // edges past this row's end gathered the sentinel row (zeros)
      if (!Shape<K>::early && has) row_fetch<K>(a, v, lq, od, xo);
      if (has) row_update<K, T>(a, cout, v, lq, act, dang_cur, sd, acc, od, xo, err, dng);
    }
  }
  // Seed rows without in-edges: only their teleport term changes.
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt < a.k) {
    const int q = gt, v = a.seed[q];
    double se = 0.0, sd = 0.0;
    if (v >= a.n_nz && is_active(act, q)) {
      const float xn = (float)((1.0 - (double)a.damp) + (double)a.damp * dang_cur[q]);
      const size_t o = (size_t)v * K + q;
      const float xo = a.x[o];
      const int od = a.outdeg[v];
      a.x[o] = xn;
      store_c(cout + o, od > 0 ? xn * (1.0f / (float)od) : 0.f);
      se = fabs((double)xn - (double)xo);
      if (od == 0) sd = (double)xn;
    }
    a.seed_red[q] = se;
    a.seed_red[K + q] = sd;
  }
  // CTA reduction: sub-groups, then warps in order.
#pragma unroll
  for (int o = L; o < 32; o <<= 1)
#pragma unroll
    for (int c = 0; c < C; ++c) {
      err[c] += __shfl_xor_sync(kFull, err[c], o);
      dng[c] += __shfl_xor_sync(kFull, dng[c], o);
    }
  if (g == 0)
#pragma unroll
    for (int c = 0; c < C; ++c) {
      s_red[(size_t)wid * K + lq * C + c] = err[c];
      s_red[(size_t)(nwarps + wid) * K + lq * C + c] = dng[c];
    }
  __syncthreads();
  for (int q = threadIdx.x; q < K; q += blockDim.x) {
    double te = 0.0, td = 0.0;
    for (int w = 0; w < nwarps; ++w) {
      te += s_red[(size_t)w * K + q];
      td += s_red[(size_t)(nwarps + w) * K + q];
    }
    a.cta_red[(size_t)blockIdx.x * K + q] = te;
    a.cta_red[(size_t)(G + blockIdx.x) * K + q] = td;
  }
  __syncthreads();
}

// Closes sweep it; run by all threads of the last CTA to finish the sweep,
// after every CTA's cta_red and seed_red are visible.  Sums each vector's
// residual and dangling mass over CTAs in CTA order (deterministic), records
// the residual and sweep count of the vectors that updated, freezes those
// below tol, publishes the next sweep's masks and dangling mass, sets
// status[2] to whether any vector keeps updating and resets the queue head
// that sweep it + 2 reuses.
template <int K>
__device__ __forceinline__ void ppr_close(const PprArgs &a, int it, unsigned *s_act) {
  const int G = gridDim.x;
  const double *dang_cur = a.dang + (it & 1) * K;
  unsigned act[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) act[i] = __ldcg(a.active + (it & 1) * 4 + i);
  if (threadIdx.x < 4) s_act[threadIdx.x] = act[threadIdx.x];
  __syncthreads();
  for (int q = threadIdx.x; q < K; q += blockDim.x) {
    double te = __ldcg(a.seed_red + q), td = __ldcg(a.seed_red + K + q);
    for (int c = 0; c < G; ++c) {
      te += __ldcg(a.cta_red + (size_t)c * K + q);
      td += __ldcg(a.cta_red + (size_t)(G + c) * K + q);
    }
    a.res_hist[(size_t)it * K + q] = te;
    const bool was = is_active(act, q);
    a.dang[((it + 1) & 1) * K + q] = was ? td : dang_cur[q];
    if (was) {
      a.iters[q] = it + 1;
      if (te < a.tol) atomicAnd(&s_act[q >> 5], ~(1u << (q & 31)));
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned any = 0;
    int n = 0;
    for (int i = 0; i < 4; ++i) {
      a.active[((it + 1) & 1) * 4 + i] = s_act[i];
      any |= s_act[i];
      n += __popc(s_act[i]);
    }
    a.status[2] = any == 0 ? 0 : (n <= a.repack_below ? 2 : 1);
    atomicExch(a.wq + (it & 1), 0);
  }
  __syncthreads();
}

// The close as a call: for K <= 16, where the sweep runs at the register
// limit, keeping it out of the sweep kernel's body leaves the sweep fewer
// spills (+4% at K = 8); for wider vectors inlining is faster (-18% at
// K = 128 as a call).
template <int K>
__device__ __noinline__ void ppr_close_call(const PprArgs &a, int it, unsigned *s_act) {
  ppr_close<K>(a, it, s_act);
}

template <int K>
__device__ __forceinline__ void close_sweep(const PprArgs &a, int it, unsigned *s_act) {
  if constexpr (K <= 16) ppr_close_call<K>(a, it, s_act);
  else ppr_close<K>(a, it, s_act);
}

// All sweeps in one cooperative launch, a bounded grid barrier between them.
template <int K, typename T>
__global__ void __launch_bounds__(kPprBlock, Shape<K>::min_ctas) k_ppr(PprArgs a) {
  constexpr int L = Shape<K>::L, C = Shape<K>::C;
  extern __shared__ double s_red[];  // [2][warps][K]
  __shared__ unsigned s_act[4];
  __shared__ int s_state;
  __shared__ unsigned s_gen;
  const int lq = (threadIdx.x & 31) % L;
  int sd[C];  // seed vertices of this lane's components (-1: padding)
#pragma unroll
  for (int c = 0; c < C; ++c) sd[c] = a.seed[lq * C + c];
  int it = 0;
  while (it < a.max_iter) {
    ppr_sweep<K, T>(a, it, sd, s_red);
    // Grid barrier; the last CTA closes the sweep.
    if (threadIdx.x == 0) {
      s_gen = ld_acquire(a.bar + 1);
      __threadfence();
      const unsigned arrived = atomicAdd(a.bar, 1u);
      s_state = (arrived == (unsigned)a.bar_expect - 1u) ? 1 : 0;
    }
    __syncthreads();
    if (s_state == 1) {
      __threadfence();
      close_sweep<K>(a, it, s_act);
      if (threadIdx.x == 0) {
        atomicExch(a.bar, 0u);
        __threadfence();
        atomicAdd(a.bar + 1, 1u);
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
    if (s_state == 2) return;
    ++it;
    if (__ldcg(a.status + 2) != 1) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.status[1] = it;
}

// One sweep per launch (graph mode): the body of a CUDA-graph while node.
// The sweep index (status[1]) and the any-vector-active flag (status[2]) live
// in device memory, so the captured launch needs no host input.  The last
// CTA to finish a sweep closes it; no CTA waits for another, so the grid need
// not be co-resident.  The node's condition starts at 1 and is only cleared:
// by the CTA that closes the last sweep, by a launch that finds the solve
// done, and by CTA 0 of the max_iter-th launch (status[3] counts launches).
template <int K, typename T>
__global__ void __launch_bounds__(kPprBlock, Shape<K>::min_ctas) k_ppr_step(PprArgs a) {
  constexpr int L = Shape<K>::L, C = Shape<K>::C;
  extern __shared__ double s_red[];  // [2][warps][K]
  __shared__ unsigned s_act[4];
  __shared__ int s_it, s_last;
  if (threadIdx.x == 0) {
    const int n_done = *(volatile int *)(a.status + 1);
    const bool live = n_done == 0 || *(volatile int *)(a.status + 2) == 1;
    s_it = live && n_done < a.max_iter ? n_done : -1;
    if (a.cond && blockIdx.x == 0) {
      const int n = atomicAdd(a.status + 3, 1) + 1;
      if (s_it < 0 || n >= a.max_iter) cudaGraphSetConditional(a.cond, 0u);
    }
  }
  __syncthreads();
  const int it = s_it;
  if (it < 0) return;
  const int lq = (threadIdx.x & 31) % L;
  int sd[C];
#pragma unroll
  for (int c = 0; c < C; ++c) sd[c] = a.seed[lq * C + c];
  ppr_sweep<K, T>(a, it, sd, s_red);
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(a.bar, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  close_sweep<K>(a, it, s_act);
  if (threadIdx.x == 0) {
    atomicExch(a.bar, 0u);
    a.status[1] = it + 1;
    __threadfence();
    if (a.cond && (a.status[2] != 1 || it + 1 >= a.max_iter)) cudaGraphSetConditional(a.cond, 0u);
  }
}

// x = e_seed, contributions of the seeds, initial dangling mass and masks.
template <int K, typename T>
__global__ void k_ppr_init(PprArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < K) {
    const int v = q < a.k ? a.seed[q] : -1;
    if (v >= 0) {
      const int od = a.outdeg[v];
      a.x[(size_t)v * K + q] = 1.0f;
      store_c(reinterpret_cast<T *>(a.c0) + (size_t)v * K + q, od > 0 ? 1.0f / (float)od : 0.f);
      a.dang[q] = od == 0 ? 1.0 : 0.0;
    } else {
      a.dang[q] = 0.0;
    }
    a.iters[q] = 0;
  }
  if (q < 4) {
    unsigned w = 0;
    for (int b = 0; b < 32; ++b)
      if (q * 32 + b < a.k) w |= 1u << b;
    a.active[q] = w;
    a.active[4 + q] = w;
  }
}

// Start of the FP32 refinement after the BF16 phase: FP32 contributions of
// the current iterate, its dangling mass, every vector active again.
template <int K>
__global__ void k_ppr_refine_init(PprArgs a, const double *__restrict__ dang_src) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < (long long)a.m * K) {
    const int v = (int)(t / K), q = (int)(t % K);
    const int od = a.outdeg[v];
    reinterpret_cast<float *>(a.c0)[t] = (q < a.k && od > 0) ? a.x[t] / (float)od : 0.f;
  }
  if (t < K) {
    a.dang[t] = dang_src[t];
    a.iters[t] = 0;
  }
  if (t < 4) {
    unsigned w = 0;
    for (int b = 0; b < 32; ++b)
      if ((int)t * 32 + b < a.k) w |= 1u << b;
    a.active[t] = w;
    a.active[4 + t] = w;
  }
}

template <int K>
__global__ void k_ppr_scatter(int m, int k, const int *__restrict__ perm,
                              const float *__restrict__ x, float *out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)m * k) return;
  const int v = (int)(t / k), q = (int)(t % k);
  out[(size_t)perm[v] * k + q] = x[(size_t)v * K + q];
}

// Packing of the still-updating vectors into a narrower layout of Kn slots:
// slot j of the new layout takes slot sel[j] of the old one (x, the
// contributions the next sweep reads, including the zero sentinel row m, the
// dangling mass of the current iterate and the seed); slots past n_sel are
// padding (seed -1, zeros).
__global__ void k_ppr_pack(int m, int K, int Kn, int n_sel, const int *__restrict__ sel,
                           const float *__restrict__ x, const float *__restrict__ c,
                           const double *__restrict__ dang, const int *__restrict__ seed,
                           float *xn, float *cn, double *dangn, int *seedn) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < ((long long)m + 1) * Kn) {
    const long long v = t / Kn;
    const int j = (int)(t % Kn);
    const bool in = j < n_sel;
    const int q = in ? sel[j] : 0;
    if (v < m) xn[t] = in ? x[v * K + q] : 0.f;
    cn[t] = in ? c[v * K + q] : 0.f;
  }
  if (t < Kn) {
    const bool in = t < n_sel;
    dangn[t] = in ? dang[sel[t]] : 0.0;
    dangn[Kn + t] = 0.0;
    seedn[t] = in ? seed[sel[t]] : -1;
  }
}

// Results of a packed layout back into the layout of K slots: slot j of the
// packed layout is slot slot_of[j] there (-1: padding).
__global__ void k_ppr_unpack(int m, int K, int Kn, const int *__restrict__ slot_of,
                             const float *__restrict__ xn, float *x) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)m * Kn) return;
  const long long v = t / Kn;
  const int j = (int)(t % Kn);
  const int q = slot_of[j];
  if (q >= 0) x[v * K + q] = xn[t];
}

// Masks of a fresh packed layout of Kn slots: the first n vectors updating,
// sweep counts 0.
__global__ void k_ppr_masks(int n, int Kn, int *iters, unsigned *active) {
  const int t = threadIdx.x;
  if (t < Kn) iters[t] = 0;
  if (t < 4) {
    unsigned w = 0;
    for (int b = 0; b < 32; ++b)
      if (t * 32 + b < n) w |= 1u << b;
    active[t] = w;
    active[4 + t] = w;
  }
}

__global__ void k_invert_for_seeds(int m, const int *__restrict__ perm, int k,
                                   const int *__restrict__ seeds_old, int *seed_new) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m) return;
  const int o = perm[v];
  for (int q = 0; q < k; ++q)
    if (seeds_old[q] == o) seed_new[q] = v;
}

// ---- batched-solver chunk table --------------------------------------------
__global__ void k_b_count(int n_nz, const int *__restrict__ ptr, int dmax, int *out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_nz) return;
  const int d = ptr[r + 1] - ptr[r];
  const int dn = r + 1 < n_nz ? ptr[r + 2] - ptr[r + 1] : -1;
  if (d > dmax && dn <= dmax) *out = r + 1;  // rows are in descending degree order
}

__global__ void k_b_lens(int n, const int *__restrict__ ptr, int chunk, int *nch) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < n) nch[r] = (ptr[r + 1] - ptr[r] + chunk - 1) / chunk;
  else if (r == n) nch[r] = 0;
}

__global__ void k_b_fill(int n, const int *__restrict__ cbeg, int *crow) {
  const int lane = threadIdx.x & 31;
  const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = w; r < n; r += nw)
    for (int c = cbeg[r] + lane; c < cbeg[r + 1]; c += 32) crow[c] = (int)r;
}

// Chunk descriptors {row, first edge, end edge, first chunk of the row, or
// -1 when the row has one chunk}.
__global__ void k_b_desc(int nch, int chunk, const int *__restrict__ ptr,
                         const int *__restrict__ cbeg, const int *__restrict__ crow, int4 *desc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nch) return;
  const int r = crow[c], cb = cbeg[r], nc = cbeg[r + 1] - cb;
  const int b = ptr[r] + (c - cb) * chunk;
  desc[c] = make_int4(r, b, min(b + chunk, ptr[r + 1]), nc == 1 ? -1 : cb);
}

int build_chunk_table(gpr_graph *g, int dmax, int chunk, cudaStream_t st) {
  if (g->b_nlong >= 0 && g->b_dmax == dmax && g->b_chunk == chunk) return GPR_OK;
  gpr::dfree(g->b_cbeg);
  gpr::dfree(g->b_crow);
  gpr::dfree(g->b_cdesc);
  gpr::dfree(g->b_pk);
  g->b_cbeg = g->b_crow = g->b_pk = nullptr;
  g->b_cdesc = nullptr;
  g->b_nlong = -1;
  g->b_npk = -1;
  for (int i = 0; i < 6; ++i) {
    gpr::dfree(g->b_pkr[i]);
    g->b_pkr[i] = nullptr;
    g->b_npkr[i] = -1;
  }
  const gpr::PrLayout &L = g->L;
  int *cnt = nullptr;
  GPR_TRY(gpr::dalloc(&cnt, 1, "chunk count"));
  int nlong = 0;
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    if (L.n_nz > 0)
      k_b_count<<<(unsigned)gpr::ceil_div(L.n_nz, 256), 256, 0, st>>>(L.n_nz, L.csr_ptr, dmax,
                                                                       cnt);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&nlong, cnt, sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  gpr::dfree(cnt);
  if (e != cudaSuccess) {
    gpr::set_error("gpr_ppr chunk table: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  GPR_TRY(gpr::dalloc(&g->b_cbeg, (size_t)nlong + 1, "batched chunk offsets"));
  k_b_lens<<<(unsigned)gpr::ceil_div((long long)nlong + 1, 256), 256, 0, st>>>(nlong, L.csr_ptr,
                                                                              chunk, g->b_cbeg);
  size_t tb = 0;
  GPR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, g->b_cbeg, g->b_cbeg, nlong + 1, st));
  void *tmp = nullptr;
  GPR_TRY(gpr::dmalloc(&tmp, tb, "scan scratch"));
  e = cub::DeviceScan::ExclusiveSum(tmp, tb, g->b_cbeg, g->b_cbeg, nlong + 1, st);
  int nch = 0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&nch, g->b_cbeg + nlong, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  gpr::dfree(tmp);
  if (e != cudaSuccess) {
    gpr::set_error("gpr_ppr chunk table: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  GPR_TRY(gpr::dalloc(&g->b_crow, (size_t)nch, "batched chunk rows"));
  if (nlong > 0) {
    unsigned gr = (unsigned)gpr::ceil_div(32LL * nlong, 256);
    if (gr > 148u * 32u) gr = 148u * 32u;
    k_b_fill<<<gr, 256, 0, st>>>(nlong, g->b_cbeg, g->b_crow);
  }
  GPR_TRY(gpr::dalloc(reinterpret_cast<int **>(&g->b_cdesc), (size_t)std::max(1, nch) * 4,
                      "batched chunk descriptors"));
  if (nch > 0)
    k_b_desc<<<(unsigned)gpr::ceil_div(nch, 256), 256, 0, st>>>(
        nch, chunk, L.csr_ptr, g->b_cbeg, g->b_crow, reinterpret_cast<int4 *>(g->b_cdesc));
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaStreamSynchronize(st));
  g->b_nlong = nlong;
  g->b_nchunks = nch;
  g->b_dmax = dmax;
  g->b_chunk = chunk;
  return GPR_OK;
}

// ---- packets: runs of consecutive units of about equal cost -----------------
// Cost of a unit in edge slots: a chunk's edges, or R times the first (widest)
// row of a row group, plus kUnitCost for the per-unit latency (descriptor,
// row offsets, score update).
constexpr long long kUnitCost = 64;

__global__ void k_pk_cost(int n_chunks, int n_units, int R, int n_long, int n_nz,
                          const int4 *__restrict__ desc, const int *__restrict__ ptr,
                          long long *cost) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n_units) return;
  long long c;
  if (u < n_chunks) {
    const int4 d = desc[u];
    c = d.z - d.y;
  } else {
    const int v = n_long + (u - n_chunks) * R;
    c = (long long)R * (ptr[v + 1] - ptr[v]);
  }
  cost[u] = c + kUnitCost;
}

// Cuts the units (chunks, then row groups of R rows) into about `want`
// packets of equal cost; a unit above the target cost is a packet alone.
// Cached per chunk table and `want`.
int build_packets(gpr_graph *g, int R, long long want, cudaStream_t st) {
  if (g->b_npk >= 0 && g->b_pk_want == want) return GPR_OK;
  gpr::dfree(g->b_pk);
  g->b_pk = nullptr;
  g->b_npk = -1;
  const gpr::PrLayout &L = g->L;
  const int n_units = g->b_nchunks + (int)gpr::ceil_div((long long)L.n_nz - g->b_nlong, R);
  long long *cost = nullptr;
  GPR_TRY(gpr::dalloc(&cost, (size_t)std::max(1, n_units), "packet costs"));
  int rc = GPR_OK;
  if (n_units > 0) {
    k_pk_cost<<<(unsigned)gpr::ceil_div(n_units, 256), 256, 0, st>>>(
        g->b_nchunks, n_units, R, g->b_nlong, L.n_nz, reinterpret_cast<const int4 *>(g->b_cdesc),
        L.csr_ptr, cost);
    rc = GPR_CUDA_RC(cudaGetLastError());
  }
  int npk = 0;
  if (rc == GPR_OK) rc = gpr::make_packets(cost, n_units, want, &g->b_pk, &npk, st);
  gpr::dfree(cost);
  GPR_TRY(rc);
  g->b_npk = npk;
  g->b_pk_want = want;
  return GPR_OK;
}

// Packets for row groups of R rows over the current chunk table, cached per
// R (the layouts of a solve's packed levels); the packet array stays owned by
// the graph.
int packets_for(gpr_graph *g, int R, long long want, cudaStream_t st, int **pk, int *npk) {
  int slot = 0;
  while ((1 << slot) < R) ++slot;
  if (g->b_npkr[slot] < 0 || g->b_pkwr[slot] != want) {
    gpr::dfree(g->b_pkr[slot]);
    g->b_pkr[slot] = nullptr;
    g->b_npkr[slot] = -1;
    const gpr::PrLayout &L = g->L;
    const int n_units = g->b_nchunks + (int)gpr::ceil_div((long long)L.n_nz - g->b_nlong, R);
    long long *cost = nullptr;
    GPR_TRY(gpr::dalloc(&cost, (size_t)std::max(1, n_units), "packet costs"));
    int rc = GPR_OK;
    if (n_units > 0) {
      k_pk_cost<<<(unsigned)gpr::ceil_div(n_units, 256), 256, 0, st>>>(
          g->b_nchunks, n_units, R, g->b_nlong, L.n_nz,
          reinterpret_cast<const int4 *>(g->b_cdesc), L.csr_ptr, cost);
      rc = GPR_CUDA_RC(cudaGetLastError());
    }
    int n = 0;
    if (rc == GPR_OK) rc = gpr::make_packets(cost, n_units, want, &g->b_pkr[slot], &n, st);
    gpr::dfree(cost);
    GPR_TRY(rc);
    g->b_npkr[slot] = n;
    g->b_pkwr[slot] = want;
  }
  *pk = g->b_pkr[slot];
  *npk = g->b_npkr[slot];
  return GPR_OK;
}

struct PprKernels {
  const void *solve;  // persistent: all sweeps in one cooperative launch
  const void *step;   // one sweep per launch (graph mode)
  void (*init)(PprArgs);
  void (*scatter)(int, int, const int *, const float *, float *);
  void (*refine_init)(PprArgs, const double *);
};

template <int K, typename T>
PprKernels kernels_for() {
  return {(const void *)k_ppr<K, T>, (const void *)k_ppr_step<K, T>, k_ppr_init<K, T>,
          k_ppr_scatter<K>, k_ppr_refine_init<K>};
}

int pick_k(int k) {
  for (int K : {8, 16, 32, 64, 128})
    if (k <= K) return K;
  return -1;
}

PprKernels select(int K, bool bf16) {
  switch (K) {
    case 8: return bf16 ? kernels_for<8, __nv_bfloat16>() : kernels_for<8, float>();
    case 16: return bf16 ? kernels_for<16, __nv_bfloat16>() : kernels_for<16, float>();
    case 32: return bf16 ? kernels_for<32, __nv_bfloat16>() : kernels_for<32, float>();
    case 64: return bf16 ? kernels_for<64, __nv_bfloat16>() : kernels_for<64, float>();
    default: return bf16 ? kernels_for<128, __nv_bfloat16>() : kernels_for<128, float>();
  }
}

struct Bufs {
  void *p[64] = {nullptr};
  int n = 0;
  template <typename X>
  int get(X **out, size_t count, const char *what) {
    if (n >= 64) {
      gpr::set_error("gpr_ppr: too many scratch buffers");
      return GPR_ENOMEM;
    }
    int rc = gpr::dalloc(out, count, what);
    if (rc == GPR_OK) p[n++] = *out;
    return rc;
  }
  ~Bufs() {
    for (int i = 0; i < n; ++i) gpr::dfree(p[i]);
  }
};

}  // namespace

extern "C" int gpr_ppr(gpr_graph *g, int k, const int *h_seeds, float *any_x,
                       const gpr_pr_opts *opts_in, int *h_iters, gpr_pr_stats *stats) {
  GPR_ENTRY_BEGIN
  gpr_pr_opts o;
  if (opts_in) o = *opts_in;
  else gpr_pr_opts_default(&o);
  if (!g || k < 1 || !h_seeds || !any_x) {
    gpr::set_error("gpr_ppr: invalid arguments");
    return GPR_EINVAL;
  }
  const int K = pick_k(k);
  if (K < 0) {
    gpr::set_error("gpr_ppr: k=%d vectors exceeds 128 per call", k);
    return GPR_EINVAL;
  }
  const gpr::PrLayout &L = g->L;
  const int m = L.m;
  if (!L.csr_ptr) {
    gpr::set_error("gpr_ppr: the graph was created without GPR_LAYOUT_BATCHED");
    return GPR_EINVAL;
  }
  if (o.precision != GPR_PREC_FP32 && o.precision != GPR_PREC_BF16) {
    gpr::set_error("gpr_ppr: precision %d not supported (FP32 or BF16)", o.precision);
    return GPR_EUNSUPPORTED;
  }
  if (o.max_iter < 0 || !(o.tol >= 0.0) || !(o.timeout_s > 0.0)) {
    gpr::set_error("gpr_ppr: invalid options");
    return GPR_EINVAL;
  }
  for (int q = 0; q < k; ++q)
    if (h_seeds[q] < 0 || h_seeds[q] >= m) {
      gpr::set_error("gpr_ppr: seed %d of vector %d out of range", h_seeds[q], q);
      return GPR_EINVAL;
    }
  // BF16 form: BF16 contributions down to tol_lo, above the BF16 rounding
  // floor, then FP32 refinement sweeps from that iterate down to tol_fix.
  // The BF16 start leaves its error in the slowest modes, which shrink by d
  // per sweep, so a refinement that stopped at a change below tol could
  // still be d/(1-d) * tol from the fixed point (5.7 tol at d = 0.85); it
  // stops at tol * (1-d)/d instead, which bounds that tail by tol and puts
  // the result as close to the FP64 fixed point as the plain FP32 solve
  // (measured on RMAT s12-s22).
  const bool bf16 = o.precision == GPR_PREC_BF16;
  const double tol_lo = std::max(o.tol, 1e-3);
  const double d_fix = std::min(std::max((double)o.damping, 1e-6), 1.0 - 1e-6);
  const double tol_fix = o.tol * (1.0 - d_fix) / d_fix;
  const PprKernels k32 = select(K, false), k16 = select(K, true);
  cudaStream_t st = g->st;
  int sms = 0;
  GPR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  const size_t smem = sizeof(double) * 2 * (kPprBlock / 32) * K;
  // The kernel's shape for this K (Shape<K>): L lanes per row, R rows per
  // warp, E edges per sub-group round.
  const int Lb = K / 4, R = 32 / Lb, Eb = Lb >= 8 ? Lb : 8;
  // Rows above 8 rounds of one sub-group are cut into chunks that the whole
  // warp works on, 8192 / L edges each (4096 for K = 8, 256 for K = 128), so
  // a chunk costs every lane about 256 gathers for every K.
  const int b_dmax = 8 * Eb, b_chunk = 8192 / Lb;
  GPR_TRY(build_chunk_table(g, b_dmax, b_chunk, st));
  const long long units =
      (long long)g->b_nchunks + gpr::ceil_div((long long)L.n_nz - g->b_nlong, R);
  auto grid_of = [&](const PprKernels &kk, int Kx, long long units_x, int *grid) -> int {
    const size_t smem_x = sizeof(double) * 2 * (kPprBlock / 32) * Kx;
    int per_sm = 0;
    GPR_CUDA(cudaFuncSetAttribute(kk.solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_x));
    GPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kk.solve, kPprBlock, smem_x));
    if (per_sm < 1) {
      gpr::set_error("gpr_ppr: kernel cannot be resident");
      return GPR_ECUDA;
    }
    *grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * per_sm,
                                                          gpr::ceil_div(units_x, kPprBlock / 32)));
    return GPR_OK;
  };
  int G32 = 0, G16 = 0;
  GPR_TRY(grid_of(k32, K, units, &G32));
  if (bf16) GPR_TRY(grid_of(k16, K, units, &G16));
  const int Gmax = std::max(G32, G16);
  // About 32 packets per warp of the larger grid: fine enough that the end
  // of a sweep is not held by one warp's last packet (measured on RMAT s22:
  // 4 per warp loses 20-30% against 16-32; 64 and more cost queue traffic).
  GPR_TRY(build_packets(g, R, (long long)Gmax * (kPprBlock / 32) * 32, st));
  Bufs B;
  float *x = nullptr, *partial = nullptr, *xout = nullptr;
  void *c0 = nullptr, *c1 = nullptr, *h0 = nullptr, *h1 = nullptr;
  int *cnt = nullptr, *seed = nullptr, *seeds_old = nullptr, *iters = nullptr, *status = nullptr,
      *wq = nullptr;
  double *cta_red = nullptr, *seed_red = nullptr, *res_hist = nullptr, *dang = nullptr;
  unsigned *active = nullptr, *bar = nullptr;
  const int max_iter = o.max_iter;
  GPR_TRY(B.get(&x, (size_t)m * K, "ppr x"));
  GPR_TRY(B.get((float **)&c0, ((size_t)m + 1) * K, "ppr contrib0"));
  GPR_TRY(B.get((float **)&c1, ((size_t)m + 1) * K, "ppr contrib1"));
  if (bf16) {
    GPR_TRY(B.get((__nv_bfloat16 **)&h0, ((size_t)m + 1) * K, "ppr bf16 contrib0"));
    GPR_TRY(B.get((__nv_bfloat16 **)&h1, ((size_t)m + 1) * K, "ppr bf16 contrib1"));
    GPR_CUDA(cudaMemsetAsync(h0, 0, ((size_t)m + 1) * K * 2, st));
    GPR_CUDA(cudaMemsetAsync(h1, 0, ((size_t)m + 1) * K * 2, st));
  }
  GPR_TRY(B.get(&partial, (size_t)std::max(1, g->b_nchunks) * K, "ppr partials"));
  GPR_TRY(B.get(&cnt, (size_t)std::max(1, g->b_nlong), "ppr counters"));
  GPR_TRY(B.get(&seed, (size_t)K, "ppr seeds"));
  GPR_TRY(B.get(&seeds_old, (size_t)k, "ppr seeds (input)"));
  GPR_TRY(B.get(&iters, (size_t)K, "ppr iterations"));
  GPR_TRY(B.get(&status, 4, "ppr status"));
  GPR_TRY(B.get(&wq, 4, "ppr queues"));
  // per-CTA sums of the widest layout; a packed layout (K/2 or narrower) runs
  // at most 4 CTAs per SM and fits
  GPR_TRY(B.get(&cta_red, (size_t)2 * std::max(Gmax, 4 * sms) * K, "ppr cta sums"));
  GPR_TRY(B.get(&seed_red, (size_t)2 * K, "ppr seed sums"));
  GPR_TRY(B.get(&res_hist, (size_t)std::max(1, max_iter) * K, "ppr residuals"));
  GPR_TRY(B.get(&dang, (size_t)2 * K, "ppr dangling"));
  GPR_TRY(B.get(&active, 8, "ppr masks"));
  GPR_TRY(B.get(&bar, 2, "ppr barrier"));
  GPR_CUDA(cudaMemsetAsync(x, 0, sizeof(float) * (size_t)m * K, st));
  GPR_CUDA(cudaMemsetAsync(c0, 0, ((size_t)m + 1) * K * 4, st));
  GPR_CUDA(cudaMemsetAsync(c1, 0, ((size_t)m + 1) * K * 4, st));
  GPR_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * std::max(1, g->b_nlong), st));
  GPR_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned) * 2, st));
  GPR_CUDA(cudaMemsetAsync(seed, 0xff, sizeof(int) * K, st));
  GPR_CUDA(cudaMemsetAsync(seed_red, 0, sizeof(double) * 2 * K, st));
  GPR_CUDA(cudaMemcpyAsync(seeds_old, h_seeds, sizeof(int) * k, cudaMemcpyHostToDevice, st));
  k_invert_for_seeds<<<(unsigned)gpr::ceil_div(m, 256), 256, 0, st>>>(m, L.perm, k, seeds_old,
                                                                       seed);
  PprArgs a;
  memset(&a, 0, sizeof(a));
  a.m = m;
  a.n_long = g->b_nlong;
  a.n_nz = L.n_nz;
  a.n_chunks = g->b_nchunks;
  a.k = k;
  a.csr_ptr = L.csr_ptr;
  a.csr_col = L.csr_col;
  a.row_cbeg = g->b_cbeg;
  a.cdesc = reinterpret_cast<const int4 *>(g->b_cdesc);
  a.pk = g->b_pk;
  a.n_pk = g->b_npk;
  a.outdeg = L.outdeg;
  a.x = x;
  a.partial = partial;
  a.cnt = cnt;
  a.seed = seed;
  a.cta_red = cta_red;
  a.seed_red = seed_red;
  a.res_hist = res_hist;
  a.dang = dang;
  a.active = active;
  a.iters = iters;
  a.bar = bar;
  a.status = status;
  a.wq = wq;
  a.damp = o.damping;
  a.max_iter = max_iter;
  a.timeout_ns = (long long)(o.timeout_s * 1e9);
  int launches = 0;
  // Graph mode: the sweep loop as one CUDA graph, a while node whose body is
  // one k_ppr_step launch (the kernel clears the condition when the phase is
  // done).  Built, run and released per phase; `mark` records the loop's
  // start event after the graph is built, right before its launch.
  auto step_loop = [&](const PprKernels &kk, int G, size_t smem, bool mark) -> int {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
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
    PprArgs ac = a;
    ac.cond = h;
    void *kargs[] = {&ac};
    cudaKernelNodeParams kp;
    memset(&kp, 0, sizeof(kp));
    kp.func = const_cast<void *>(kk.step);
    kp.gridDim = dim3(G);
    kp.blockDim = dim3(kPprBlock);
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = kargs;
    if (e == cudaSuccess) e = cudaGraphAddKernelNode(&kn, cp.conditional.phGraph_out[0], nullptr, 0, &kp);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e == cudaSuccess && mark) e = cudaEventRecord(g->e2, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      gpr::set_error("gpr_ppr graph loop: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
    return GPR_OK;
  };
  // One phase: sweeps until every vector's change is below `tol`, in one
  // cooperative launch, or (GPR_LOOP_GRAPH, or when the grid cannot be
  // co-resident) in the graph loop.  The first phase (`mark`) records the
  // start event of the sweep loop right before its launch.
  auto phase = [&](const PprKernels &kk, int G, int Kx, double tol, bool mark, int *sweeps,
                   std::vector<int> *it_out, int *stop) -> int {
    const size_t smem = sizeof(double) * 2 * (kPprBlock / 32) * Kx;
    a.tol = tol;
    a.bar_expect = G + (o.reserved[0] > 0 ? o.reserved[0] : 0);
    GPR_CUDA(cudaMemsetAsync(status, 0, sizeof(int) * 4, st));
    GPR_CUDA(cudaMemsetAsync(wq, 0, sizeof(int) * 4, st));
    bool graph_mode = o.loop == GPR_LOOP_GRAPH;
    if (mark && (max_iter <= 0 || !graph_mode)) GPR_CUDA(cudaEventRecord(g->e2, st));
    if (max_iter > 0 && !graph_mode) {
      void *args[] = {&a};
      cudaError_t e = cudaLaunchCooperativeKernel(kk.solve, dim3(G), dim3(kPprBlock), args, smem, st);
      if (e == cudaErrorCooperativeLaunchTooLarge) {
        cudaGetLastError();
        graph_mode = true;
      } else if (e != cudaSuccess) {
        gpr::set_error("gpr_ppr: %s", cudaGetErrorString(e));
        return GPR_ECUDA;
      } else {
        ++launches;
      }
    }
    if (max_iter > 0 && graph_mode) GPR_TRY(step_loop(kk, G, smem, mark && o.loop == GPR_LOOP_GRAPH));
    int hs[4];
    GPR_CUDA(cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st));
    it_out->assign(Kx, 0);
    GPR_CUDA(cudaMemcpyAsync(it_out->data(), iters, sizeof(int) * Kx, cudaMemcpyDeviceToHost, st));
    GPR_CUDA(cudaStreamSynchronize(st));
    *sweeps = hs[1];
    *stop = hs[2];
    if (max_iter > 0 && graph_mode) launches += hs[3];
    if (hs[0] & 1) {
      gpr::set_error("gpr_ppr: grid barrier wait exceeded %.3f s", o.timeout_s);
      return GPR_ETIMEOUT;
    }
    return GPR_OK;
  };
  // FP32 sweeps to `tol` with packing: the widest layout first; whenever at
  // most half of its vectors are still updating (and it is wider than 8), the
  // kernel stops, those vectors' x, next contributions, dangling mass and
  // seeds are packed into the next narrower layout, and the sweeps go on
  // there with the remaining sweep budget.  Vectors that stopped keep their
  // final x in the widest layout (the master), where every packed layout is
  // written back.  sweeps: launches' sweeps in total; it_total: per vector.
  int last_sw = 0, last_K = K;  // sweeps and width of the last layout (its residuals)
  auto fp32_phase = [&](double tol, bool mark, int *sweeps, std::vector<int> *it_total) -> int {
    it_total->assign(K, 0);
    *sweeps = 0;
    int Kc = K, Gc = G32;
    PprKernels kc = k32;
    float *xc = x;
    void *cc0 = c0, *cc1 = c1;
    double *dc = dang;
    int *sc = seed;
    std::vector<int> slot_of(K);  // master slot of each slot of the current layout
    for (int q = 0; q < K; ++q) slot_of[q] = q < k ? q : -1;
    int *d_slot_of = nullptr;
    bool first = true;
    for (;;) {
      a.repack_below = (o.ppr_repack && Kc > 8) ? Kc / 2 : 0;
      a.max_iter = max_iter - *sweeps;
      int sw = 0, stop = 0;
      std::vector<int> itc;
      GPR_TRY(phase(kc, Gc, Kc, tol, mark && first, &sw, &itc, &stop));
      first = false;
      *sweeps += sw;
      last_sw = sw;
      last_K = Kc;
      for (int q = 0; q < Kc; ++q)
        if (slot_of[q] >= 0) (*it_total)[slot_of[q]] += itc[q];
      const bool packed = Kc != K;
      if (stop != 2 || *sweeps >= max_iter) {
        if (packed) {  // the packed layout's results back into the master
          k_ppr_unpack<<<(unsigned)gpr::ceil_div((long long)m * Kc, 256), 256, 0, st>>>(
              m, K, Kc, d_slot_of, xc, x);
          ++launches;
          GPR_CUDA(cudaGetLastError());
        }
        break;
      }
      // the slots still updating after the last sweep
      unsigned act[4];
      GPR_CUDA(cudaMemcpyAsync(act, active + (sw & 1) * 4, sizeof(act), cudaMemcpyDeviceToHost,
                               st));
      GPR_CUDA(cudaStreamSynchronize(st));
      std::vector<int> sel;
      for (int q = 0; q < Kc; ++q)
        if ((act[q >> 5] >> (q & 31)) & 1u) sel.push_back(q);
      const int Kn = pick_k((int)sel.size());
      if (packed) {
        k_ppr_unpack<<<(unsigned)gpr::ceil_div((long long)m * Kc, 256), 256, 0, st>>>(
            m, K, Kc, d_slot_of, xc, x);
        ++launches;
      }
      float *xn = nullptr, *cn0 = nullptr, *cn1 = nullptr;
      double *dn = nullptr;
      int *sn = nullptr, *d_sel = nullptr, *d_so = nullptr;
      GPR_TRY(B.get(&xn, (size_t)m * Kn, "ppr packed x"));
      GPR_TRY(B.get(&cn0, ((size_t)m + 1) * Kn, "ppr packed contrib0"));
      GPR_TRY(B.get(&cn1, ((size_t)m + 1) * Kn, "ppr packed contrib1"));
      GPR_TRY(B.get(&dn, (size_t)2 * Kn, "ppr packed dangling"));
      GPR_TRY(B.get(&sn, (size_t)Kn, "ppr packed seeds"));
      GPR_TRY(B.get(&d_sel, sel.size(), "ppr packed selection"));
      GPR_TRY(B.get(&d_so, (size_t)Kn, "ppr packed slots"));
      std::vector<int> so(Kn, -1);
      for (size_t j = 0; j < sel.size(); ++j) so[j] = slot_of[sel[j]];
      GPR_CUDA(cudaMemcpyAsync(d_sel, sel.data(), sizeof(int) * sel.size(), cudaMemcpyHostToDevice,
                               st));
      GPR_CUDA(cudaMemcpyAsync(d_so, so.data(), sizeof(int) * Kn, cudaMemcpyHostToDevice, st));
      GPR_CUDA(cudaMemsetAsync(cn1, 0, sizeof(float) * ((size_t)m + 1) * Kn, st));
      const float *ccur = static_cast<const float *>((sw & 1) ? cc1 : cc0);
      k_ppr_pack<<<(unsigned)gpr::ceil_div(((long long)m + 1) * Kn, 256), 256, 0, st>>>(
          m, Kc, Kn, (int)sel.size(), d_sel, xc, ccur, dc + (sw & 1) * Kc, sc, xn, cn0, dn, sn);
      k_ppr_masks<<<1, 128, 0, st>>>((int)sel.size(), Kn, iters, active);
      launches += 2;
      GPR_CUDA(cudaGetLastError());
      // the narrower layout's kernels, grid and packets
      Kc = Kn;
      kc = select(Kc, false);
      const int Rn = 32 / (Kc / 4);
      const long long units_n =
          (long long)g->b_nchunks + gpr::ceil_div((long long)L.n_nz - g->b_nlong, Rn);
      GPR_TRY(grid_of(kc, Kc, units_n, &Gc));
      int *pk = nullptr, npk = 0;
      GPR_TRY(packets_for(g, Rn, (long long)Gc * (kPprBlock / 32) * 32, st, &pk, &npk));
      a.pk = pk;
      a.n_pk = npk;
      a.k = (int)sel.size();
      a.x = xn;
      a.c0 = cn0;
      a.c1 = cn1;
      a.dang = dn;
      a.seed = sn;
      xc = xn;
      cc0 = cn0;
      cc1 = cn1;
      dc = dn;
      sc = sn;
      d_slot_of = d_so;
      slot_of = so;
    }
    return GPR_OK;
  };
  GPR_CUDA(cudaEventRecord(g->e0, st));
  int s1 = 0, s2 = 0, stop1 = 0;
  std::vector<int> it1(K, 0), it2(K, 0);
  if (bf16) {
    a.c0 = h0;
    a.c1 = h1;
    k16.init<<<1, 128, 0, st>>>(a);
    ++launches;
    a.repack_below = 0;
    GPR_TRY(phase(k16, G16, K, tol_lo, true, &s1, &it1, &stop1));
    a.c0 = c0;
    a.c1 = c1;
    k32.refine_init<<<(unsigned)gpr::ceil_div((long long)m * K, 256), 256, 0, st>>>(
        a, dang + (s1 & 1) * K);
    ++launches;
  } else {
    a.c0 = c0;
    a.c1 = c1;
    k32.init<<<1, 128, 0, st>>>(a);
    ++launches;
  }
  GPR_TRY(fp32_phase(bf16 ? tol_fix : o.tol, !bf16, &s2, &it2));
  GPR_CUDA(cudaEventRecord(g->e3, st));
  const bool host_out = !gpr::is_device_ptr(any_x);
  float *dout = any_x;
  if (host_out) {
    GPR_TRY(B.get(&xout, (size_t)m * k, "ppr output staging"));
    dout = xout;
  }
  k32.scatter<<<(unsigned)gpr::ceil_div((long long)m * k, 256), 256, 0, st>>>(m, k, L.perm, x,
                                                                              dout);
  ++launches;
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaEventRecord(g->e1, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  if (host_out)
    GPR_CUDA(cudaMemcpy(any_x, xout, sizeof(float) * (size_t)m * k, cudaMemcpyDeviceToHost));
  float ms = 0.f, lms = 0.f;
  GPR_CUDA(cudaEventElapsedTime(&ms, g->e0, g->e1));
  GPR_CUDA(cudaEventElapsedTime(&lms, g->e2, g->e3));
  if (h_iters)
    for (int q = 0; q < k; ++q) h_iters[q] = it1[q] + it2[q];
  if (stats) {
    memset(stats, 0, sizeof(*stats));
    stats->iterations = s1 + s2;
    stats->refine_iterations = bf16 ? s2 : 0;
    stats->solve_ms = ms;
    stats->loop_ms = lms;
    stats->gpu_launches = launches;
    if (last_sw > 0) {
      // the last sweep of the last layout: the vectors that updated longest
      std::vector<double> last(last_K);
      GPR_CUDA(cudaMemcpy(last.data(), res_hist + (size_t)(last_sw - 1) * last_K,
                          sizeof(double) * last_K, cudaMemcpyDeviceToHost));
      double mx = 0;
      for (int q = 0; q < std::min(k, last_K); ++q) mx = std::max(mx, last[q]);
      stats->residual = mx;
    }
  }
  return GPR_OK;
  GPR_ENTRY_END("gpr_ppr")
}
