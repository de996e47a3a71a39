// Push-style PageRank: every source adds its contribution to its
// out-neighbours' accumulators with atomic adds.
//
// The reference's push variants (src/pr/scatter.cu:16-41, lb.cu:20-82) launch
// a thread per source that atomically adds kDamp*score/degree to each
// destination, then a second kernel per sweep that swaps the buffers and sums
// the L1 change.  Here the recurrence is the pull solver's (contribution =
// score / out-degree, score = base + kDamp * sum, FP64 L1 residual, stop after
// the sweep whose residual is below tol: src/pr/omp_base.cc:23-44), so the two
// directions solve the same problem and can be compared on the same graph.
//
// Layout: the in-CSR's edges as a list sorted by source (relabelled ids,
// built on first use), so each warp reads 32 consecutive edges -- equal work
// for every warp, and the contribution loads of one warp fall on a few
// neighbouring sources.  One persistent cooperative launch for all sweeps:
//   scatter  warps take tiles of 32 x U edges; destinations below `hot` (the
//            highest in-degree vertices, which receive most adds) accumulate
//            in shared memory with shared atomics and are flushed once per
//            sweep, the rest go to global accumulators as fire-and-forget L2
//            reductions;
//   barrier  (bounded);
//   update   every vertex: score, contribution, |change|, accumulator reset;
//   barrier  with the per-CTA residuals summed in CTA order.
// Atomic adds make the sum order, and so the last bits of a result, vary
// from run to run; the sweep count and the 1e-6 agreement with the reference
// do not.
#include <cub/cub.cuh>
#include <math.h>
#include <string.h>

#include <algorithm>

#include "gpr_device.cuh"
#include "gpr_internal.cuh"
#include "gpr_guard.h"

using namespace gpr::dev;

namespace {

constexpr int kPushBlock = 1024;
constexpr int kPushU = 8;  // edges per lane in flight

struct PushArgs {
  int m;
  long long nnz;
  const int *src, *dst;  // edges sorted by source
  const int *outdeg;
  float *s, *c, *sum;
  int hot;
  unsigned *bar;
  double *cta_part, *err_hist;
  int *status;
  float base, damp;
  double tol;
  int max_iter;
  unsigned bar_expect;
  long long timeout_ns;
};

__global__ void __launch_bounds__(kPushBlock, 1) k_pr_push(PushArgs a) {
  extern __shared__ float s_acc[];
  const int lane = threadIdx.x & 31;
  const long long gw = (long long)blockIdx.x * (kPushBlock / 32) + (threadIdx.x >> 5);
  const long long nw = (long long)gridDim.x * (kPushBlock / 32);
  const long long gt = (long long)blockIdx.x * kPushBlock + threadIdx.x;
  const long long nt = (long long)gridDim.x * kPushBlock;
  const Policies pol = make_policies();
  const long long tiles = (a.nnz + 32LL * kPushU - 1) / (32LL * kPushU);
  int it = 0;
  while (it < a.max_iter) {
    for (int i = threadIdx.x; i < a.hot; i += kPushBlock) s_acc[i] = 0.f;
    __syncthreads();
    for (long long t = gw; t < tiles; t += nw) {
      const long long e0 = t * 32 * kPushU + lane;
      int u[kPushU], v[kPushU];
#pragma unroll
      for (int q = 0; q < kPushU; ++q) {
        const long long e = e0 + 32 * q;
        u[q] = e < a.nnz ? ld_s32_stream(a.src + e, pol.stream) : -1;
        v[q] = e < a.nnz ? ld_s32_stream(a.dst + e, pol.stream) : 0;
      }
      float x[kPushU];
#pragma unroll
      for (int q = 0; q < kPushU; ++q) x[q] = u[q] >= 0 ? ld_contrib(a.c + u[q], pol.keep) : 0.f;
#pragma unroll
      for (int q = 0; q < kPushU; ++q) {
        if (u[q] < 0) continue;
        if (v[q] < a.hot) atomicAdd(s_acc + v[q], x[q]);
        else atomicAdd(a.sum + v[q], x[q]);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < a.hot; i += kPushBlock) {
      const float y = s_acc[i];
      if (y != 0.f) atomicAdd(a.sum + i, y);
    }
    if (!grid_barrier(a.bar, a.bar_expect, nullptr, 0.0, nullptr, a.status, a.timeout_ns)) return;
    double err = 0.0;
    for (long long v = gt; v < a.m; v += nt) {
      const float sn = __fadd_rn(a.base, __fmul_rn(a.damp, __ldcg(a.sum + v)));
      err += (double)fabsf(__fsub_rn(sn, a.s[v]));
      a.s[v] = sn;
      a.c[v] = __fdiv_rn(sn, __int2float_rn(a.outdeg[v]));
      a.sum[v] = 0.f;
    }
    const double tot = block_sum_double(err);
    if (!grid_barrier(a.bar, a.bar_expect, a.cta_part, tot, a.err_hist + it, a.status,
                      a.timeout_ns))
      return;
    const double total = __ldcg(a.err_hist + it);
    ++it;
    if (total < a.tol) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) a.status[1] = it;
}

__global__ void k_push_prologue(int m, const int *__restrict__ perm,
                                const int *__restrict__ outdeg, const float *__restrict__ in,
                                float *s, float *c, float *sum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    const float v = in[perm[i]];
    s[i] = v;
    c[i] = __fdiv_rn(v, __int2float_rn(outdeg[i]));
    sum[i] = 0.f;
  }
}

__global__ void k_push_scatter(int m, const int *__restrict__ perm, const float *__restrict__ s,
                               float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[perm[i]] = s[i];
}

// dst[e] = row of edge e in the relabelled in-CSR (one warp per row).
__global__ void k_edge_rows(int m, const int *__restrict__ ptr, int *row) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = w0; r < m; r += nw)
    for (int e = ptr[r] + lane; e < ptr[r + 1]; e += 32) row[e] = (int)r;
}

inline unsigned grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  return (unsigned)std::max<long long>(1, std::min<long long>(g, 0x7fffffffLL));
}

// Edges of the relabelled in-CSR sorted by source (stable: destinations of
// one source ascending).
int build_push_edges(gpr_graph *g) {
  const gpr::PrLayout &L = g->L;
  if (!L.csr_ptr) {
    gpr::set_error("gpr_pagerank_push: create the graph with GPR_LAYOUT_PUSH (keeps the CSR)");
    return GPR_EUNSUPPORTED;
  }
  cudaStream_t st = g->st;
  const long long n = L.nnz;
  int *rows = nullptr, *src = nullptr, *dst = nullptr;
  int rc = gpr::dalloc(&rows, (size_t)n, "edge rows");
  if (rc == GPR_OK) rc = gpr::dalloc(&src, (size_t)n, "push sources");
  if (rc == GPR_OK) rc = gpr::dalloc(&dst, (size_t)n, "push destinations");
  if (rc == GPR_OK && n > 0) {
    k_edge_rows<<<std::min<unsigned>(grid_for(32LL * L.m), 148u * 64u), 256, 0, st>>>(
        L.m, L.csr_ptr, rows);
    int bits = 1;
    while ((1LL << bits) < L.m) ++bits;
    size_t tb = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cub::DeviceRadixSort::SortPairs(nullptr, tb, L.csr_col, src, rows, dst, (int)n, 0, bits,
                                          st);
    void *tmp = nullptr;
    if (e == cudaSuccess) rc = gpr::dmalloc(&tmp, tb, "sort scratch");
    if (e == cudaSuccess && rc == GPR_OK)
      e = cub::DeviceRadixSort::SortPairs(tmp, tb, L.csr_col, src, rows, dst, (int)n, 0, bits, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    gpr::dfree(tmp);
    if (e != cudaSuccess) {
      gpr::set_error("push edge sort: %s", cudaGetErrorString(e));
      rc = GPR_ECUDA;
    }
  }
  gpr::dfree(rows);
  if (rc == GPR_OK) rc = gpr::dalloc(&g->push_sum, (size_t)L.m + 1, "push accumulators");
  if (rc != GPR_OK) {
    gpr::dfree(src);
    gpr::dfree(dst);
    return rc;
  }
  g->push_src = src;
  g->push_dst = dst;
  return GPR_OK;
}

int push_impl(gpr_graph *g, float *any_scores, const gpr_pr_opts &o, gpr_pr_stats *out) {
  const gpr::PrLayout &L = g->L;
  const int m = L.m;
  memset(out, 0, sizeof(*out));
  if (m == 0) {  // no vertices: the sweeps are empty and their residuals 0
    out->iterations = gpr::empty_graph_sweeps(o.tol, o.max_iter);
    g->last_sweeps = out->iterations;
    return GPR_OK;
  }
  if (!g->push_src) GPR_TRY(build_push_edges(g));
  cudaStream_t st = g->st;
  float *d_scores = any_scores;
  const bool host = !gpr::is_device_ptr(any_scores);
  if (host) {
    d_scores = g->scores_tmp;
    GPR_CUDA(cudaMemcpyAsync(d_scores, any_scores, sizeof(float) * (size_t)m,
                             cudaMemcpyHostToDevice, st));
  }
  if (o.max_iter > g->err_cap) {
    gpr::dfree(g->err_hist);
    g->err_hist = nullptr;
    g->err_cap = o.max_iter;
    GPR_TRY(gpr::dalloc(&g->err_hist, (size_t)g->err_cap, "residual history"));
  }
  int sms = 0, per_sm = 0, coop = 0;
  GPR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
  GPR_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, g->device));
  const int hot = std::min(gpr::kHotDefault, m);
  const size_t smem = sizeof(float) * (size_t)hot;
  GPR_CUDA(cudaFuncSetAttribute((const void *)k_pr_push,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  GPR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_pr_push,
                                                         kPushBlock, smem));
  if (!coop || per_sm < 1) {
    gpr::set_error("gpr_pagerank_push: the device cannot co-schedule the persistent kernel");
    return GPR_EUNSUPPORTED;
  }
  // cta_err holds 2 * max_grid partials
  const int grid = std::max(1, std::min(sms, 2 * g->max_grid));
  PushArgs a;
  memset(&a, 0, sizeof(a));
  a.m = m;
  a.nnz = L.nnz;
  a.src = g->push_src;
  a.dst = g->push_dst;
  a.outdeg = L.outdeg;
  a.s = g->s;
  a.c = g->c0;
  a.sum = g->push_sum;
  a.hot = hot;
  a.bar = g->bar;
  a.cta_part = g->cta_err;
  a.err_hist = g->err_hist;
  a.status = g->status;
  a.base = (1.0f - o.damping) / (float)m;  // src/pr/omp_base.cc:16
  a.damp = o.damping;
  a.tol = o.tol;
  a.max_iter = o.max_iter;
  a.bar_expect = (unsigned)grid + (o.reserved[0] > 0 ? (unsigned)o.reserved[0] : 0u);
  a.timeout_ns = (long long)(o.timeout_s * 1e9);
  GPR_CUDA(cudaMemsetAsync(g->bar, 0, 4 * sizeof(unsigned), st));
  GPR_CUDA(cudaMemsetAsync(g->status, 0, 4 * sizeof(int), st));
  GPR_CUDA(cudaEventRecord(g->e0, st));
  k_push_prologue<<<grid_for(m), 256, 0, st>>>(m, L.perm, L.outdeg, d_scores, g->s, g->c0,
                                              g->push_sum);
  GPR_CUDA(cudaEventRecord(g->e2, st));
  int launches = 1;
  if (o.max_iter > 0) {
    void *args[] = {&a};
    GPR_CUDA(cudaLaunchCooperativeKernel((const void *)k_pr_push, dim3(grid), dim3(kPushBlock),
                                         args, smem, st));
    ++launches;
  }
  GPR_CUDA(cudaEventRecord(g->e3, st));
  k_push_scatter<<<grid_for(m), 256, 0, st>>>(m, L.perm, g->s, d_scores);
  ++launches;
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaEventRecord(g->e1, st));
  int hs[4];
  GPR_CUDA(cudaMemcpyAsync(hs, g->status, sizeof(hs), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  float ms = 0.f, lms = 0.f;
  GPR_CUDA(cudaEventElapsedTime(&ms, g->e0, g->e1));
  GPR_CUDA(cudaEventElapsedTime(&lms, g->e2, g->e3));
  out->iterations = o.max_iter > 0 ? hs[1] : 0;
  out->solve_ms = ms;
  out->loop_ms = lms;
  out->gpu_launches = launches;
  g->last_sweeps = out->iterations;
  if (out->iterations > 0)
    GPR_CUDA(cudaMemcpy(&out->residual, g->err_hist + out->iterations - 1, sizeof(double),
                        cudaMemcpyDeviceToHost));
  if (hs[0] & 1) {
    gpr::set_error("grid barrier wait exceeded %.3f s (sweep loop abandoned)", o.timeout_s);
    return GPR_ETIMEOUT;
  }
  if (host)
    GPR_CUDA(cudaMemcpy(any_scores, d_scores, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost));
  return GPR_OK;
}

}  // namespace

extern "C" int gpr_pagerank_push(gpr_graph *g, float *any_scores, const gpr_pr_opts *opts,
                                 gpr_pr_stats *stats) {
  GPR_ENTRY_BEGIN
  if (!g) {
    gpr::set_error("gpr_pagerank_push: NULL graph");
    return GPR_EINVAL;
  }
  gpr_pr_opts o;
  if (opts) o = *opts;
  else gpr_pr_opts_default(&o);
  if (!(o.damping >= 0.f && o.damping <= 1.f) || o.max_iter < 0 || !(o.tol >= 0.0) ||
      !(o.timeout_s > 0.0) || (g->L.m > 0 && !any_scores)) {
    gpr::set_error("gpr_pagerank_push: invalid arguments");
    return GPR_EINVAL;
  }
  if (o.precision != GPR_PREC_FP32) {
    gpr::set_error("gpr_pagerank_push: only GPR_PREC_FP32");
    return GPR_EUNSUPPORTED;
  }
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != g->device) GPR_CUDA(cudaSetDevice(g->device));
  gpr_pr_stats st;
  int rc = push_impl(g, any_scores, o, &st);
  if (stats) *stats = st;
  if (cur != g->device && cur >= 0) cudaSetDevice(cur);
  return rc;
  GPR_ENTRY_END("gpr_pagerank_push")
}
