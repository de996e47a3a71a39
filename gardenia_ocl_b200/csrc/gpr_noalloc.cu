// PageRank entry point that allocates no memory.
//
// Some callers cannot let a library call cudaMalloc: a host framework that
// reserves the device heap for its own allocator up front, or a latency-
// critical caller that may not take the device-wide synchronisation that
// cudaMalloc / cudaFree can cause.  gpr_pagerank_noalloc serves them: it
// solves directly on the caller's device CSR, and the only memory it needs
// beyond the caller's inputs and outputs -- two contribution buffers, the
// per-CTA residual partials, the per-sweep residual history and a few status
// words -- lives in one file-scope device array, g_noalloc_scratch, of fixed
// size (kNoAllocBytes, about 8 MiB).  Every GPU that loads the library holds
// that array until the process exits.
//
// Host code only ever sees a host-side stand-in for the array's name, so the
// device address is looked up once per device with cudaGetSymbolAddress, with
// that device current, on the first call made on it; that first call should
// therefore come before any stream capture.  All calls share the array and it
// keeps the previous call's contents: the words that must start at zero are
// cleared at the start of every call, and calls that overlap on the GPU (on
// different streams, or from different host threads) race on it.
//
// The sweep is one thread per row, summing the row in CSR order with the
// reference's float operations (src/pr/omp_base.cc:34-39), so its scores are
// identical to the reference's; the residual is reduced in FP64 per CTA and
// combined by the last CTA of each sweep.
#include <math.h>
#include <string.h>

#include <chrono>
#include <mutex>

#include "gpr_internal.cuh"
#include "gpr_guard.h"

namespace {

constexpr int kNoAllocMaxVertices = 1 << 20;  // largest m accepted
constexpr int kNoAllocMaxIter = 1000;         // largest max_iter accepted
constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocMaxCtas = (kNoAllocMaxVertices + kNoAllocBlock - 1) / kNoAllocBlock;

// Byte layout of the scratch array (all offsets 256-byte aligned).
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffContrib0 = 0;
constexpr size_t kOffContrib1 = align256(kOffContrib0 + sizeof(float) * (kNoAllocMaxVertices + 1));
constexpr size_t kOffCtaErr = align256(kOffContrib1 + sizeof(float) * (kNoAllocMaxVertices + 1));
constexpr size_t kOffHist = align256(kOffCtaErr + sizeof(double) * kNoAllocMaxCtas);
constexpr size_t kOffWords = align256(kOffHist + sizeof(double) * kNoAllocMaxIter);
constexpr size_t kNoAllocBytes = align256(kOffWords + sizeof(int) * 8);

// words[0] arrival count, [1] sweeps done, [2] done flag, [3] CSR error flags
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

struct NoAllocArgs {
  int m;
  const int *rowptr, *col, *outdeg;
  float *s;
  float *c0, *c1;
  double *cta_err, *hist;
  int *words;
  float base, damp;
  double tol;
  int max_iter;
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void k_na_validate(int m, long long nnz, const int *__restrict__ rowptr,
                              const int *__restrict__ col, const int *__restrict__ outdeg,
                              int *words) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i <= m; i += stride) {
    if (i == 0 && rowptr[0] != 0) atomicOr(words + 3, 1);
    if (i == m && (long long)rowptr[m] != nnz) atomicOr(words + 3, 2);
    if (i < m && (rowptr[i] > rowptr[i + 1] || outdeg[i] < 0)) atomicOr(words + 3, 4);
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    const int c = col[e];
    if (c < 0 || c >= m) atomicOr(words + 3, 8);
  }
}

__global__ void k_na_prologue(NoAllocArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < a.m) a.c0[i] = __fdiv_rn(a.s[i], __int2float_rn(a.outdeg[i]));
}

// One sweep; sweep index and done flag live in the scratch words, so launches
// after convergence return at once.
__global__ void __launch_bounds__(kNoAllocBlock) k_na_sweep(NoAllocArgs a) {
  __shared__ int s_it, s_last;
  __shared__ double red[kNoAllocBlock / 32];
  if (threadIdx.x == 0) {
    const int done = *(volatile int *)(a.words + 2);
    s_it = done ? -1 : *(volatile int *)(a.words + 1);
  }
  __syncthreads();
  const int it = s_it;
  if (it < 0) return;
  const float *cin = (it & 1) ? a.c1 : a.c0;
  float *cout = (it & 1) ? a.c0 : a.c1;
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  double err = 0.0;
  if (v < a.m) {
    float total = 0.f;
    for (int e = a.rowptr[v]; e < a.rowptr[v + 1]; ++e) total = __fadd_rn(total, cin[a.col[e]]);
    const float so = a.s[v];
    const float sn = __fadd_rn(a.base, __fmul_rn(a.damp, total));
    a.s[v] = sn;
    cout[v] = __fdiv_rn(sn, __int2float_rn(a.outdeg[v]));
    err = (double)fabsf(__fsub_rn(sn, so));
  }
  err = warp_sum_d(err);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = err;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kNoAllocBlock / 32; ++w) t += red[w];
    a.cta_err[blockIdx.x] = t;
    __threadfence();
    s_last = atomicAdd(a.words, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && threadIdx.x < 32) {
    __threadfence();
    double t = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += 32) t += __ldcg(a.cta_err + i);
    t = warp_sum_d(t);
    if (threadIdx.x == 0) {
      a.hist[it] = t;
      atomicExch(a.words, 0);
      a.words[1] = it + 1;
      if (t < a.tol || it + 1 >= a.max_iter) a.words[2] = 1;
      __threadfence();
    }
  }
}

std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[64] = {nullptr};

// Device address of the scratch array on the current device, looked up once.
int scratch_for_current_device(unsigned char **out) {
  int dev = 0;
  GPR_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    gpr::set_error("gpr_pagerank_noalloc: device index %d out of range", dev);
    return GPR_EINVAL;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      gpr::set_error("gpr_pagerank_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
    g_scratch_ptr[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch_ptr[dev];
  return GPR_OK;
}

}  // namespace

extern "C" {

long long gpr_pagerank_noalloc_max_vertices(void) { return kNoAllocMaxVertices; }

int gpr_pagerank_noalloc(int m, int nnz, const int *d_rowptr, const int *d_col,
                         const int *d_outdeg, float *d_scores, const gpr_pr_opts *opts,
                         gpr_pr_stats *stats, void *stream) {
  GPR_ENTRY_BEGIN
  gpr_pr_opts o;
  if (opts) o = *opts;
  else gpr_pr_opts_default(&o);
  if (m < 0 || nnz < 0 || (m == 0 && nnz != 0) ||
      (m > 0 && (!d_rowptr || !d_outdeg || !d_scores)) || (nnz > 0 && !d_col)) {
    gpr::set_error("gpr_pagerank_noalloc: invalid arguments (m=%d nnz=%d)", m, nnz);
    return GPR_EINVAL;
  }
  if (m > kNoAllocMaxVertices) {
    gpr::set_error("gpr_pagerank_noalloc: m=%d exceeds the fixed scratch limit of %d vertices",
                   m, kNoAllocMaxVertices);
    return GPR_EINVAL;
  }
  if (o.max_iter < 0 || o.max_iter > kNoAllocMaxIter || !(o.tol >= 0.0) ||
      !(o.damping >= 0.f && o.damping <= 1.f)) {
    gpr::set_error("gpr_pagerank_noalloc: invalid options (max_iter %d must be in [0, %d])",
                   o.max_iter, kNoAllocMaxIter);
    return GPR_EINVAL;
  }
  gpr_pr_stats st;
  memset(&st, 0, sizeof(st));
  if (m == 0) {
    // no vertices: the sweeps are empty and their residuals 0
    st.iterations = gpr::empty_graph_sweeps(o.tol, o.max_iter);
    if (stats) *stats = st;
    return GPR_OK;
  }
  const auto t0 = std::chrono::steady_clock::now();
  unsigned char *base = nullptr;
  GPR_TRY(scratch_for_current_device(&base));
  cudaStream_t s = (cudaStream_t)stream;
  NoAllocArgs a;
  a.m = m;
  a.rowptr = d_rowptr;
  a.col = d_col;
  a.outdeg = d_outdeg;
  a.s = d_scores;
  a.c0 = reinterpret_cast<float *>(base + kOffContrib0);
  a.c1 = reinterpret_cast<float *>(base + kOffContrib1);
  a.cta_err = reinterpret_cast<double *>(base + kOffCtaErr);
  a.hist = reinterpret_cast<double *>(base + kOffHist);
  a.words = reinterpret_cast<int *>(base + kOffWords);
  a.damp = o.damping;
  a.base = (1.0f - o.damping) / (float)m;  // src/pr/omp_base.cc:16
  a.tol = o.tol;
  a.max_iter = o.max_iter;
  const unsigned grid = (unsigned)((m + kNoAllocBlock - 1) / kNoAllocBlock);
  GPR_CUDA(cudaMemsetAsync(a.words, 0, sizeof(int) * 8, s));
  k_na_validate<<<148 * 8, 256, 0, s>>>(m, nnz, d_rowptr, d_col, d_outdeg, a.words);
  GPR_CUDA(cudaGetLastError());
  int words[4];
  GPR_CUDA(cudaMemcpyAsync(words, a.words, sizeof(words), cudaMemcpyDeviceToHost, s));
  GPR_CUDA(cudaStreamSynchronize(s));
  if (words[3]) {
    gpr::set_error("gpr_pagerank_noalloc: malformed CSR (flags 0x%x)", words[3]);
    return GPR_EINVAL;
  }
  if (o.max_iter == 0) {
    if (stats) *stats = st;
    return GPR_OK;
  }
  k_na_prologue<<<grid, kNoAllocBlock, 0, s>>>(a);
  GPR_CUDA(cudaGetLastError());
  int launches = 2, issued = 0, done = 0;
  while (!done && issued < o.max_iter) {
    for (int q = 0; q < 8 && issued < o.max_iter; ++q, ++issued) {
      k_na_sweep<<<grid, kNoAllocBlock, 0, s>>>(a);
      ++launches;
    }
    GPR_CUDA(cudaGetLastError());
    GPR_CUDA(cudaMemcpyAsync(words, a.words, sizeof(words), cudaMemcpyDeviceToHost, s));
    GPR_CUDA(cudaStreamSynchronize(s));
    done = words[2];
  }
  st.iterations = words[1];
  if (st.iterations > 0) {
    // on the caller's stream: no device-wide synchronisation
    GPR_CUDA(cudaMemcpyAsync(&st.residual, a.hist + st.iterations - 1, sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    GPR_CUDA(cudaStreamSynchronize(s));
  }
  st.gpu_launches = launches;
  st.solve_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  st.loop_ms = st.solve_ms;
  if (stats) *stats = st;
  return GPR_OK;
  GPR_ENTRY_END("gpr_pagerank_noalloc")
}

}  // extern "C"
