// CSR SpMV y <- y + A*x on B200 (src/spmv/omp_base.cc:8-32 semantics).
//
// Rows keep their natural order (x locality of stencil-like matrices is the
// main asset).  Rows with at most sell_max entries live in SELL-32 slices,
// one lane per row: the lane starts from y[r] and adds x[j]*Ax[jj] in CSR
// order with explicitly rounded multiply and add, i.e. the same float
// operations in the same order as the reference's loop, so those rows are
// bit-identical to it.  Longer rows are split into chunks of `chunk` entries
// (one warp per chunk, 128-bit loads) whose partial sums the last arriving
// warp combines in a fixed order.
#include <string.h>

#include "gpr_internal.cuh"
#include "gpr_guard.h"

using gpr::SpmvLayout;

struct gpr_matrix {
  int device = 0;
  SpmvLayout L;
  float *partial = nullptr;  // [n_chunks]
  int *cnt = nullptr;        // [n_long]
  int grid = 0;
};

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Entries per lane per round of a SELL row: each round loads kSpmvU column
// indices and values, then gathers their x.  On the 27-point 128^3 stencil
// 4 / 8 / 16 per round ran at 85% / 99% / 90% of the measured copy bandwidth.
constexpr int kSpmvU = 8;

struct SpArgs {
  int m, n_long, n_chunks, n_slices, chunk;
  const int *long_rows;
  const long long *long_ptr;
  const int *long_col;
  const float *long_val;
  const int *row_cbeg;
  const int *chunk_row;
  const long long *slice_ptr;
  const int *sell_col;
  const float *sell_val;
  const unsigned char *sell_len;
  const float *x;
  float *y;
  float *partial;
  int *cnt;
};

__device__ __forceinline__ uint64_t evict_first_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ int ld_s32(const int *p, uint64_t pol) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_f32(const float *p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int4 ld_s32x4(const int *p, uint64_t pol) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float4 ld_f32x4(const float *p, uint64_t pol) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ void do_slice(const SpArgs &a, int s, int lane, uint64_t pol) {
  const long long b = a.slice_ptr[s];
  const int slen = (int)((a.slice_ptr[s + 1] - b) >> 5);
  const int r = s * 32 + lane;
  if (r >= a.m) return;
  const int d = a.sell_len[r];
  if (d == 255) return;  // long row: handled by its chunks
  const int *pc = a.sell_col + b + lane;
  const float *pv = a.sell_val + b + lane;
  float acc = a.y[r];
  int j = 0;
  for (; j + kSpmvU <= d; j += kSpmvU) {
    int c[kSpmvU];
    float v[kSpmvU], xv[kSpmvU];
#pragma unroll
    for (int q = 0; q < kSpmvU; ++q) {
      c[q] = ld_s32(pc + 32 * (j + q), pol);
      v[q] = ld_f32(pv + 32 * (j + q), pol);
    }
#pragma unroll
    for (int q = 0; q < kSpmvU; ++q) xv[q] = __ldg(a.x + c[q]);
#pragma unroll
    for (int q = 0; q < kSpmvU; ++q) acc = __fadd_rn(acc, __fmul_rn(xv[q], v[q]));
  }
  for (; j < d; ++j) {
    const int c = ld_s32(pc + 32 * j, pol);
    const float v = ld_f32(pv + 32 * j, pol);
    acc = __fadd_rn(acc, __fmul_rn(__ldg(a.x + c), v));
  }
  (void)slen;
  a.y[r] = acc;
}

__device__ __forceinline__ void do_chunk(const SpArgs &a, int c, int lane, uint64_t pol) {
  const int li = a.chunk_row[c];
  const int cb = a.row_cbeg[li];
  const int nc = a.row_cbeg[li + 1] - cb;
  const long long b = a.long_ptr[li] + (long long)(c - cb) * a.chunk;
  const long long e = min(b + (long long)a.chunk, a.long_ptr[li + 1]);
  float acc = 0.f;
  for (long long k = b + 4 * lane; k < e; k += 128) {
    const int4 q = ld_s32x4(a.long_col + k, pol);
    const float4 v = ld_f32x4(a.long_val + k, pol);
    acc += (__ldg(a.x + q.x) * v.x + __ldg(a.x + q.y) * v.y) +
           (__ldg(a.x + q.z) * v.z + __ldg(a.x + q.w) * v.w);
  }
  acc = warp_sum(acc);
  const int r = a.long_rows[li];
  if (nc == 1) {
    if (lane == 0) a.y[r] = a.y[r] + acc;
    return;
  }
  int last = 0;
  if (lane == 0) {
    a.partial[c] = acc;
    __threadfence();
    last = atomicAdd(a.cnt + li, 1) == nc - 1;
  }
  last = __shfl_sync(kFull, last, 0);
  if (!last) return;
  __threadfence();
  float t = 0.f;
  for (int q = lane; q < nc; q += 32) t += __ldcg(a.partial + cb + q);
  t = warp_sum(t);
  if (lane == 0) {
    atomicExch(a.cnt + li, 0);
    a.y[r] = a.y[r] + t;
  }
}

__global__ void __launch_bounds__(gpr::kBlock) k_spmv(SpArgs a) {
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const uint64_t pol = evict_first_policy();
  const long long u1 = a.n_chunks, u2 = u1 + a.n_slices;
  for (long long u = gw; u < u2; u += nw) {
    if (u < u1) do_chunk(a, (int)u, lane, pol);
    else do_slice(a, (int)(u - u1), lane, pol);
  }
}

void destroy(gpr_matrix *A) {
  if (!A) return;
  gpr::free_spmv_layout(&A->L);
  gpr::dfree(A->partial);
  gpr::dfree(A->cnt);
  delete A;
}

int create_impl(int m, long long nnz, const int *any_Ap, const int *any_Aj, const float *any_Ax,
                gpr_matrix *A) {
  GPR_CUDA(cudaGetDevice(&A->device));
  cudaStream_t st = 0;
  void *ap = nullptr, *aj = nullptr, *ax = nullptr;
  bool oap = false, oaj = false, oax = false;
  int rc = gpr::to_device(any_Ap, sizeof(int) * ((size_t)m + 1), &ap, &oap, st, "Ap");
  if (rc == GPR_OK) rc = gpr::to_device(any_Aj, sizeof(int) * (size_t)nnz, &aj, &oaj, st, "Aj");
  if (rc == GPR_OK) rc = gpr::to_device(any_Ax, sizeof(float) * (size_t)nnz, &ax, &oax, st, "Ax");
  if (rc == GPR_OK)
    rc = gpr::validate_csr(m, nnz, m, (const int *)ap, (const int *)aj, nullptr, st);
  if (rc == GPR_OK)
    rc = gpr::build_spmv_layout(m, nnz, (const int *)ap, (const int *)aj, (const float *)ax,
                                gpr::kSellMaxDefault, gpr::kChunkDefault, &A->L, st);
  cudaStreamSynchronize(st);
  if (oap) gpr::dfree(ap);
  if (oaj) gpr::dfree(aj);
  if (oax) gpr::dfree(ax);
  GPR_TRY(rc);
  GPR_TRY(gpr::dalloc(&A->partial, (size_t)A->L.n_chunks, "spmv partials"));
  GPR_TRY(gpr::dalloc(&A->cnt, (size_t)A->L.n_long, "spmv counters"));
  GPR_CUDA(cudaMemset(A->cnt, 0, sizeof(int) * (A->L.n_long ? A->L.n_long : 1)));
  const long long units = (long long)A->L.n_chunks + A->L.n_slices;
  long long g = gpr::ceil_div(units, gpr::kBlock / 32);
  A->grid = (int)(g < 1 ? 1 : (g > 0x7fffffff ? 0x7fffffff : g));
  return GPR_OK;
}

}  // namespace

extern "C" {

int gpr_matrix_create(int m, long long nnz, const int *any_Ap, const int *any_Aj,
                      const float *any_Ax, gpr_matrix **out) {
  GPR_ENTRY_BEGIN
  if (!out) {
    gpr::set_error("gpr_matrix_create: NULL out");
    return GPR_EINVAL;
  }
  *out = nullptr;
  if (m < 0 || nnz < 0 || nnz > 0x7fffffffLL || (m > 0 && !any_Ap) ||
      (nnz > 0 && (!any_Aj || !any_Ax))) {
    gpr::set_error("gpr_matrix_create: invalid arguments (m=%d nnz=%lld)", m, nnz);
    return GPR_EINVAL;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    gpr::set_error("gpr_matrix_create: no CUDA device");
    return GPR_ENODEV;
  }
  gpr_matrix *A = new gpr_matrix();
  int rc = create_impl(m, nnz, any_Ap, any_Aj, any_Ax, A);
  if (rc != GPR_OK) {
    destroy(A);
    return rc;
  }
  *out = A;
  return GPR_OK;
  GPR_ENTRY_END("gpr_matrix_create")
}

int gpr_matrix_destroy(gpr_matrix *A) {
  destroy(A);
  return GPR_OK;
}

int gpr_spmv(gpr_matrix *A, const float *d_x, float *d_y, void *stream) {
  if (!A || (A->L.m > 0 && (!d_x || !d_y))) {
    gpr::set_error("gpr_spmv: NULL argument");
    return GPR_EINVAL;
  }
  if (A->L.m == 0) return GPR_OK;
  const SpmvLayout &L = A->L;
  SpArgs a;
  a.m = L.m;
  a.n_long = L.n_long;
  a.n_chunks = L.n_chunks;
  a.n_slices = L.n_slices;
  a.chunk = L.chunk;
  a.long_rows = L.long_rows;
  a.long_ptr = L.long_ptr;
  a.long_col = L.long_col;
  a.long_val = L.long_val;
  a.row_cbeg = L.row_cbeg;
  a.chunk_row = L.chunk_row;
  a.slice_ptr = L.slice_ptr;
  a.sell_col = L.sell_col;
  a.sell_val = L.sell_val;
  a.sell_len = L.sell_len;
  a.x = d_x;
  a.y = d_y;
  a.partial = A->partial;
  a.cnt = A->cnt;
  k_spmv<<<A->grid, gpr::kBlock, 0, (cudaStream_t)stream>>>(a);
  GPR_CUDA(cudaGetLastError());
  return GPR_OK;
}

int gpr_matrix_layout(const gpr_matrix *A, int *n_long, int *n_chunks, int *n_slices,
                      long long *sell_elems) {
  if (!A) {
    gpr::set_error("gpr_matrix_layout: NULL matrix");
    return GPR_EINVAL;
  }
  if (n_long) *n_long = A->L.n_long;
  if (n_chunks) *n_chunks = A->L.n_chunks;
  if (n_slices) *n_slices = A->L.n_slices;
  if (sell_elems) *sell_elems = A->L.sell_elems;
  return GPR_OK;
}

int gpr_spmv_solver(int m, int nnz, const int *Ap, const int *Aj, const float *Ax, const float *x,
                    float *y) {
  GPR_ENTRY_BEGIN
  if (m < 0 || (m > 0 && (!x || !y))) {
    gpr::set_error("gpr_spmv_solver: invalid arguments");
    return GPR_EINVAL;
  }
  gpr_matrix *A = nullptr;
  GPR_TRY(gpr_matrix_create(m, nnz, Ap, Aj, Ax, &A));
  void *dx = nullptr, *dy = nullptr;
  bool ox = false, oy = false;
  int rc = gpr::to_device(x, sizeof(float) * (size_t)m, &dx, &ox, 0, "x");
  if (rc == GPR_OK) rc = gpr::to_device(y, sizeof(float) * (size_t)m, &dy, &oy, 0, "y");
  if (rc == GPR_OK) rc = gpr_spmv(A, (const float *)dx, (float *)dy, 0);
  if (rc == GPR_OK && oy) {
    cudaError_t e = cudaMemcpy(y, dy, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      gpr::set_error("gpr_spmv_solver: copy back: %s", cudaGetErrorString(e));
      rc = GPR_ECUDA;
    }
  } else if (rc == GPR_OK) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      gpr::set_error("gpr_spmv_solver: %s", cudaGetErrorString(e));
      rc = GPR_ECUDA;
    }
  }
  if (ox) gpr::dfree(dx);
  if (oy) gpr::dfree(dy);
  gpr_matrix_destroy(A);
  return rc;
  GPR_ENTRY_END("gpr_spmv_solver")
}

}  // extern "C"
