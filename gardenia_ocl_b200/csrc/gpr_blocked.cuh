// Device code of the blocked form of the pull sweep (layout: gpr_blocked.cu),
// shared by the single-graph kernel (gpr_pagerank.cu) and the multi-graph
// batch (gpr_multi.cu).  Templated on the kernel's argument struct, which
// provides: entry, runs, tiles, blocks (the layout), acc_rows, gacc, bcnt,
// blk_row0 (cross-tile accumulators of rows blk_row0 on), fx_scale, fx_inv,
// s, outdeg, damp.  The base of the update is given per tile (one graph's
// (1 - d) / m_g).
#pragma once

#include "gpr_device.cuh"

namespace gpr {
namespace blk {

using namespace gpr::dev;

// The blocked rows are summed block by block (gpr_blocked.cu): the CTA that
// takes a tile zeroes one accumulator per row of the tile's block in shared
// memory, its warps take the tile's runs (source-ordered entries, so a warp's
// gathers share lines) and add each contribution to its row's accumulator.
// The accumulators are 64-bit fixed point, value * 2^S, held as two 32-bit
// words: the low word is added with an atomic that returns the old word, so
// its carry is exact, and the high word gets the contribution's high bits
// plus the carry (most contributions fit the low word).  Integer addition is
// associative, so every row's sum is the same whatever the order in which
// warps and tiles add: results do not change from run to run, and each sum is
// the exact sum of the FP32 contributions rounded once to 2^-S.  The sum is
// rounded to FP32 and the update uses the reference's float operations
// (src/pr/omp_base.cc:39, 26).  A block cut into several tiles adds its
// tiles' sums into a 64-bit global accumulator per row; the CTA that
// completes the block's last tile finalizes it and clears the accumulators.
__device__ __forceinline__ void use_u32(unsigned x) { asm volatile("" ::"r"(x)); }
__device__ __forceinline__ void use_f32(float x) { asm volatile("" ::"f"(x)); }

// Four entries of a run; lanes past the run's end read padding words.
__device__ __forceinline__ uint4 ld_entry4(const unsigned *p, bool pred, uint64_t pol) {
  uint4 v = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu);
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " @p ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%5], %6;\n}"
      : "+r"(v.x), "+r"(v.y), "+r"(v.z), "+r"(v.w)
      : "r"((int)pred), "l"(p), "l"(pol));
  return v;
}

// Contribution of an entry's source (segment base | low 16 bits); padding
// entries read nothing and give 0.
__device__ __forceinline__ float gather_entry(const float *cin, unsigned segbase, unsigned w,
                                              uint64_t pol) {
  float v = 0.f;
  const float *p = cin + (segbase | (w >> 16));
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.u32 p, %1, 0xFFFFFFFF;\n"
      " @p ld.global.L2::cache_hint.f32 %0, [%2], %3;\n}"
      : "+f"(v)
      : "r"(w), "l"(p), "l"(pol));
  return v;
}

// Rows row0 + i, i < nrows, from their fixed-point sums (shared accumulators
// or, when `global`, the cross-tile accumulators, which are cleared); eight
// rows per thread are loaded before any is updated.  NT threads per CTA.
template <int NT, typename Args>
__device__ __forceinline__ double blocked_finalize(const Args &a, float *cout, int row0,
                                                   int nrows, const unsigned *acc, bool global,
                                                   float base, const Policies &pol) {
  double err = 0.0;
  for (int i0 = threadIdx.x; i0 < nrows; i0 += 8 * NT) {
    long long x[8];
    float so[8];
    int od[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = i0 + NT * k;
      x[k] = 0;
      so[k] = 0.f;
      od[k] = 1;
      if (i < nrows) {
        const int r = row0 + i;
        x[k] = global ? (long long)__ldcg(a.gacc + (r - a.blk_row0))
                      : (long long)(((unsigned long long)acc[a.acc_rows + i] << 32) | acc[i]);
        so[k] = ld_f32_stream(a.s + r, pol.stream);
        od[k] = ld_s32_stream(a.outdeg + r, pol.stream);
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = i0 + NT * k;
      if (i < nrows) {
        const int r = row0 + i;
        if (global) a.gacc[r - a.blk_row0] = 0ull;
        const float sum = (float)((double)x[k] * a.fx_inv);
        const float sn = __fadd_rn(base, __fmul_rn(a.damp, sum));
        st_f32(a.s + r, sn, pol.stream);
        st_c(cout + r, __fdiv_rn(sn, __int2float_rn(od[k])), pol.keep);
        err += (double)fabsf(__fsub_rn(sn, so[k]));
      }
    }
  }
  return err;
}

// Index words of a run (lanes past its end get padding words).
template <int PV, typename Args>
__device__ __forceinline__ void load_run(const Args &a, uint2 rd, int lane, uint4 *q,
                                         const Policies &pol) {
  const int len = (int)(rd.y & 0xFFFFu);
#pragma unroll
  for (int i = 0; i < PV; ++i)
    q[i] = ld_entry4(a.entry + rd.x + 128 * i + 4 * lane, 128 * i + 4 * lane < len, pol.stream);
}

// The run's contributions: wait for its index words, issue every gather, wait
// for them, then add them to the rows' fixed-point accumulators (PV even:
// the additions go eight at a time).
template <int PV, typename Args>
__device__ __forceinline__ void add_run(const Args &a, const float *cin, unsigned *acc,
                                        uint2 rd, const uint4 *q, const Policies &pol) {
  static_assert(PV % 2 == 0, "eight contributions per addition batch");
  const unsigned segbase = (rd.y >> 16) << 16;
#pragma unroll
  for (int i = 0; i < PV; ++i) {
    use_u32(q[i].x); use_u32(q[i].y); use_u32(q[i].z); use_u32(q[i].w);
  }
  float v[4 * PV];
#pragma unroll
  for (int i = 0; i < PV; ++i) {
    v[4 * i + 0] = gather_entry(cin, segbase, q[i].x, pol.keep);
    v[4 * i + 1] = gather_entry(cin, segbase, q[i].y, pol.keep);
    v[4 * i + 2] = gather_entry(cin, segbase, q[i].z, pol.keep);
    v[4 * i + 3] = gather_entry(cin, segbase, q[i].w, pol.keep);
  }
#pragma unroll
  for (int i = 0; i < 4 * PV; ++i) use_f32(v[i]);
  unsigned wv[4 * PV];
#pragma unroll
  for (int i = 0; i < PV; ++i) {
    wv[4 * i + 0] = q[i].x; wv[4 * i + 1] = q[i].y; wv[4 * i + 2] = q[i].z; wv[4 * i + 3] = q[i].w;
  }
#pragma unroll
  for (int h = 0; h < 4 * PV; h += 8) {
    unsigned lo[8], hw[8], old[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const long long x = __float2ll_rn(v[h + i] * a.fx_scale);
      lo[i] = (unsigned)x;
      hw[i] = (unsigned)((unsigned long long)x >> 32);
      old[i] = 0u;
      if (wv[h + i] != 0xFFFFFFFFu) old[i] = atomicAdd(acc + (wv[h + i] & 0xFFFFu), lo[i]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const unsigned hc = hw[i] + (old[i] + lo[i] < old[i] ? 1u : 0u);
      if (wv[h + i] != 0xFFFFFFFFu && hc) atomicAdd(acc + a.acc_rows + (wv[h + i] & 0xFFFFu), hc);
    }
  }
}

// One tile: zero the block's accumulators, add the tile's runs, then finalize
// the block (single tile) or add into the cross-tile accumulators.  Warps
// take runs from a shared counter; the CTA claims its next tile from the
// queue `tq` once its runs are done (the claim's latency hides behind the
// close of this tile, and the tile goes to a CTA that is about to be free).
template <int PV, int NT, typename Args>
__device__ __forceinline__ double blocked_tile(const Args &a, const float *cin, float *cout,
                                               int t, unsigned *acc, int *s_next, int *s_last,
                                               int *s_next_tile, int *tq, float base,
                                               const Policies &pol) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int4 td = a.tiles[t];
  const int4 bd = a.blocks[td.x];
  const int nr = td.z - td.y;
  const uint2 *runs = a.runs + td.y;
  for (int i = threadIdx.x; i < bd.y; i += NT) {
    acc[i] = 0u;
    acc[a.acc_rows + i] = 0u;
  }
  if (threadIdx.x == 0) *s_next = NT / 32;
  __syncthreads();
  int r = warp;
  uint2 rd = make_uint2(0u, 0u);
  if (r < nr) rd = __ldg(runs + r);
  while (r < nr) {
    int rn = 0;
    if (lane == 0) rn = atomicAdd(s_next, 1);
    uint4 q[PV];
    load_run<PV>(a, rd, lane, q, pol);
    // the next run's descriptor is fetched while this run's loads are in flight
    rn = __shfl_sync(kFull, rn, 0);
    uint2 nd = make_uint2(0u, 0u);
    if (rn < nr) nd = __ldg(runs + rn);
    add_run<PV>(a, cin, acc, rd, q, pol);
    r = rn;
    rd = nd;
  }
  if (threadIdx.x == 0) *s_next_tile = atomicAdd(tq, 1);
  __syncthreads();
  double err = 0.0;
  if (bd.z == 1) {
    err = blocked_finalize<NT>(a, cout, bd.x, bd.y, acc, false, base, pol);
  } else {
    for (int i = threadIdx.x; i < bd.y; i += NT) {
      const unsigned long long x = ((unsigned long long)acc[a.acc_rows + i] << 32) | acc[i];
      if (x) atomicAdd(a.gacc + (bd.x - a.blk_row0) + i, x);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      *s_last = atomicAdd(a.bcnt + td.x, 1) == bd.z - 1;
    }
    __syncthreads();
    if (*s_last) {
      __threadfence();
      err = blocked_finalize<NT>(a, cout, bd.x, bd.y, acc, true, base, pol);
      if (threadIdx.x == 0) a.bcnt[td.x] = 0;
    }
  }
  return err;
}

}  // namespace blk
}  // namespace gpr
