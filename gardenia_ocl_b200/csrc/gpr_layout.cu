// Device-side construction of the PR and SpMV layouts from a CSR.
//
// PR: vertices are relabelled by descending in-degree (stable), which turns
// the degree bins into contiguous row ranges (no row lists to read per sweep)
// and packs the most-gathered contributions of a power-law graph into a
// small, cache-friendly prefix.  Edge order inside each row is preserved.
#include <cub/cub.cuh>

#include "gpr_internal.cuh"

namespace gpr {

namespace {

__global__ void k_validate_rows(int m, long long nnz, const int *__restrict__ rowptr,
                                const int *__restrict__ outdeg, int *flag) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i > m) return;
  if (i == 0 && rowptr[0] != 0) atomicOr(flag, 1);
  if (i == m && (long long)rowptr[m] != nnz) atomicOr(flag, 2);
  if (i < m) {
    if (rowptr[i] > rowptr[i + 1]) atomicOr(flag, 4);
    if (outdeg && outdeg[i] < 0) atomicOr(flag, 16);
  }
}

__global__ void k_validate_cols(long long nnz, int ncols, const int *__restrict__ col,
                                int *flag) {
  long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    int c = col[e];
    if (c < 0 || c >= ncols) atomicOr(flag, 8);
  }
}

__global__ void k_indeg_iota(int m, const int *__restrict__ rowptr, int *indeg, int *iota) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    indeg[i] = rowptr[i + 1] - rowptr[i];
    iota[i] = i;
  }
}

// Sorted (descending) degrees -> out[k] = number of rows with degree > th[k].
__global__ void k_bounds(int m, const int *__restrict__ sdeg, const int *__restrict__ th, int nth,
                         int *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  int d = sdeg[i];
  int dn = (i + 1 < m) ? sdeg[i + 1] : -1;
  for (int k = 0; k < nth; ++k)
    if (d > th[k] && dn <= th[k]) out[k] = i + 1;
}

__global__ void k_relabel(int m, const int *__restrict__ perm, const int *__restrict__ outdeg,
                          int *outdeg_new, int *inv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    int o = perm[i];
    outdeg_new[i] = outdeg[o];
    inv[o] = i;
  }
}

__global__ void k_long_lens(int n_long, const int *__restrict__ sdeg, int chunk,
                            long long *plen, int *nch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_long) {
    long long p = ((long long)sdeg[i] + 3) & ~3LL;
    plen[i] = p;
    nch[i] = (int)((p + chunk - 1) / chunk);
  } else if (i == n_long) {
    plen[i] = 0;
    nch[i] = 0;
  }
}

__global__ void k_fill_chunk_row(int n_long, const int *__restrict__ cbeg, int *chunk_row) {
  int lane = threadIdx.x & 31;
  long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = w; r < n_long; r += nw)
    for (int c = cbeg[r] + lane; c < cbeg[r + 1]; c += 32) chunk_row[c] = (int)r;
}

// One warp per long row: relabelled sources, padded with the sentinel m.
__global__ void k_fill_long(int n_long, int m, const int *__restrict__ perm,
                            const int *__restrict__ inv, const int *__restrict__ rowptr,
                            const int *__restrict__ col, const long long *__restrict__ lptr,
                            int *long_col) {
  int lane = threadIdx.x & 31;
  long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = w; r < n_long; r += nw) {
    int o = perm[r];
    long long sb = rowptr[o];
    long long deg = rowptr[o + 1] - sb;
    long long db = lptr[r], plen = lptr[r + 1] - db;
    for (long long k = lane; k < plen; k += 32)
      long_col[db + k] = (k < deg) ? inv[col[sb + k]] : m;
  }
}

// Slice s of class c: 32 >> lw rows starting at row0; its length is the
// per-lane edge count of its first (longest) row.
__global__ void k_slice_lens(int n_slices, PrClasses cls, const int *__restrict__ sdeg,
                             long long *slen) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n_slices) {
    const int c = slice_class(cls, s);
    const int lw = cls.lw[c];
    const int row0 = cls.row[c] + ((s - cls.slice[c]) << (5 - lw));
    slen[s] = 32LL * (((long long)sdeg[row0] + (1 << lw) - 1) >> lw);
  } else if (s == n_slices) {
    slen[s] = 0;
  }
}

// One thread per (slice, lane): lane holds edges l, l+w, l+2w, ... of its row.
__global__ void k_fill_sell(int n_slices, int m, PrClasses cls, const int *__restrict__ perm,
                            const int *__restrict__ inv, const int *__restrict__ rowptr,
                            const int *__restrict__ col, const int *__restrict__ sdeg,
                            const long long *__restrict__ sptr, int *sell_col) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 32LL * n_slices) return;
  const int s = (int)(t >> 5), lane = (int)(t & 31);
  const int c = slice_class(cls, s);
  const int lw = cls.lw[c];
  const int row0 = cls.row[c] + ((s - cls.slice[c]) << (5 - lw));
  const int r = row0 + (lane >> lw), l = lane & ((1 << lw) - 1);
  const long long base = sptr[s];
  const int len = (int)((sptr[s + 1] - base) >> 5);
  int deg = 0;
  long long sb = 0;
  if (r < cls.row[c + 1]) {
    deg = sdeg[r];
    sb = rowptr[perm[r]];
  }
  for (int j = 0; j < len; ++j) {
    const long long e = ((long long)j << lw) + l;
    sell_col[base + 32LL * j + lane] = (e < deg) ? inv[col[sb + e]] : m;
  }
}

__global__ void k_csr_lens(int m, const int *__restrict__ sdeg, int *len) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) len[i] = sdeg[i];
  else if (i == m) len[i] = 0;
}

// One warp per row: relabelled CSR in new row order, edge order preserved.
__global__ void k_fill_csr(int m, const int *__restrict__ perm, const int *__restrict__ inv,
                           const int *__restrict__ rowptr, const int *__restrict__ col,
                           const int *__restrict__ nptr, int *ncol) {
  int lane = threadIdx.x & 31;
  long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = w; r < m; r += nw) {
    const long long sb = rowptr[perm[r]];
    const long long db = nptr[r], deg = nptr[r + 1] - db;
    for (long long k = lane; k < deg; k += 32) ncol[db + k] = inv[col[sb + k]];
  }
}

template <typename T>
int exclusive_scan(T *d, long long n, cudaStream_t st) {
  size_t tmp_bytes = 0;
  GPR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d, d, (int)n, st));
  void *tmp = nullptr;
  GPR_TRY(dmalloc(&tmp, tmp_bytes, "scan scratch"));
  cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, d, d, (int)n, st);
  gpr::dfree(tmp);
  if (e != cudaSuccess) {
    set_error("DeviceScan::ExclusiveSum: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  return GPR_OK;
}

inline unsigned grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 0x7fffffffLL) g = 0x7fffffffLL;
  return (unsigned)g;
}

struct Scratch {
  void *p[8] = {nullptr};
  ~Scratch() {
    for (void *q : p) dfree(q);
  }
};

}  // namespace

int validate_csr(int m, long long nnz, int ncols, const int *d_rowptr, const int *d_col,
                 const int *d_outdeg, cudaStream_t st) {
  if (m < 0 || nnz < 0 || nnz > 0x7fffffffLL) {
    set_error("invalid sizes m=%d nnz=%lld", m, nnz);
    return GPR_EINVAL;
  }
  int *flag = nullptr;
  GPR_TRY(dalloc(&flag, 1, "validation flag"));
  int h = 0;
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    k_validate_rows<<<grid_for((long long)m + 1), 256, 0, st>>>(m, nnz, d_rowptr, d_outdeg, flag);
    if (nnz > 0 && d_col) {
      long long g = grid_for(nnz);
      if (g > 148 * 64) g = 148 * 64;
      k_validate_cols<<<(unsigned)g, 256, 0, st>>>(nnz, ncols, d_col, flag);
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  gpr::dfree(flag);
  if (e != cudaSuccess) {
    set_error("CSR validation: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  if (h) {
    set_error("malformed CSR (flags 0x%x: 1 rowptr[0]!=0, 2 rowptr[m]!=nnz, 4 rowptr not "
              "monotone, 8 column out of range, 16 negative degree)", h);
    return GPR_EINVAL;
  }
  return GPR_OK;
}

int validate_cols(long long nnz, int ncols, const int *d_col, cudaStream_t st) {
  if (nnz <= 0) return GPR_OK;
  int *flag = nullptr;
  GPR_TRY(dalloc(&flag, 1, "validation flag"));
  int h = 0;
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    long long g = grid_for(nnz);
    if (g > 148 * 64) g = 148 * 64;
    k_validate_cols<<<(unsigned)g, 256, 0, st>>>(nnz, ncols, d_col, flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  gpr::dfree(flag);
  if (e != cudaSuccess) {
    set_error("CSR validation: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  if (h) {
    set_error("malformed CSR (flags 0x%x: 1 rowptr[0]!=0, 2 rowptr[m]!=nnz, 4 rowptr not "
              "monotone, 8 column out of range, 16 negative degree)", h);
    return GPR_EINVAL;
  }
  return GPR_OK;
}

int build_pr_layout(int m, long long nnz, const int *d_rowptr, const int *d_col,
                    const int *d_outdeg, int lane_max, int chunk_min, int chunk, bool keep_csr,
                    PrLayout *L, cudaStream_t st, cudaEvent_t col_ready) {
  *L = PrLayout();
  L->m = m;
  L->nnz = nnz;
  L->lane_max = lane_max;
  L->chunk_min = chunk_min;
  L->chunk = chunk;
  if (m <= 0) return GPR_OK;
  Scratch S;
  int *indeg = nullptr, *iota = nullptr, *sdeg = nullptr, *inv = nullptr, *bounds = nullptr;
  GPR_TRY(dalloc(&indeg, m, "in-degree"));
  S.p[0] = indeg;
  GPR_TRY(dalloc(&iota, m, "iota"));
  S.p[1] = iota;
  GPR_TRY(dalloc(&sdeg, m, "sorted degree"));
  S.p[2] = sdeg;
  GPR_TRY(dalloc(&inv, m, "inverse permutation"));
  S.p[3] = inv;
  GPR_TRY(dalloc(&bounds, 16, "bounds"));
  S.p[4] = bounds;
  GPR_TRY(dalloc(&L->perm, m, "permutation"));
  GPR_TRY(dalloc(&L->outdeg, m, "out-degree"));

  k_indeg_iota<<<grid_for(m), 256, 0, st>>>(m, d_rowptr, indeg, iota);
  {
    size_t tb = 0;
    GPR_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, indeg, sdeg, iota, L->perm,
                                                       m, 0, 32, st));
    void *tmp = nullptr;
    GPR_TRY(dmalloc(&tmp, tb, "sort scratch"));
    cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(tmp, tb, indeg, sdeg, iota,
                                                              L->perm, m, 0, 32, st);
    gpr::dfree(tmp);
    if (e != cudaSuccess) {
      set_error("degree sort: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  }
  // Degree thresholds, descending: chunked rows, then width classes
  // w = 32 .. 1 (class w holds lane_max*w/2 < deg <= lane_max*w), then 0.
  int th[8], nth = 0;
  th[nth++] = chunk_min;
  for (int lw = 4; lw >= 0; --lw) {
    long long t = (long long)lane_max << lw;
    th[nth++] = (int)(t < chunk_min ? t : chunk_min);
  }
  th[nth++] = 0;
  GPR_CUDA(cudaMemsetAsync(bounds, 0, 16 * sizeof(int), st));
  GPR_CUDA(cudaMemcpyAsync(bounds + 8, th, nth * sizeof(int), cudaMemcpyHostToDevice, st));
  k_bounds<<<grid_for(m), 256, 0, st>>>(m, sdeg, bounds + 8, nth, bounds);
  k_relabel<<<grid_for(m), 256, 0, st>>>(m, L->perm, d_outdeg, L->outdeg, inv);
  int hb[8];
  GPR_CUDA(cudaMemcpyAsync(hb, bounds, nth * sizeof(int), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  L->n_long = hb[0];
  L->n_nz = hb[nth - 1];
  // Classes: widest first; class with lw spans rows [hb[4-lw], hb[5-lw]).
  PrClasses &C = L->cls;
  int slices = 0;
  for (int lw = 5; lw >= 0; --lw) {
    const int r0 = hb[5 - lw], r1 = hb[6 - lw];
    if (r1 <= r0) continue;
    C.lw[C.n_cls] = lw;
    C.row[C.n_cls] = r0;
    C.slice[C.n_cls] = slices;
    slices += (int)ceil_div(r1 - r0, 32 >> lw);
    ++C.n_cls;
  }
  C.row[C.n_cls] = L->n_nz;
  C.slice[C.n_cls] = slices;
  L->n_slices = slices;

  // Long rows: padded CSR + chunk table.
  GPR_TRY(dalloc(&L->long_ptr, (size_t)L->n_long + 1, "long row offsets"));
  GPR_TRY(dalloc(&L->row_cbeg, (size_t)L->n_long + 1, "long row chunk offsets"));
  k_long_lens<<<grid_for((long long)L->n_long + 1), 256, 0, st>>>(L->n_long, sdeg, chunk,
                                                                   L->long_ptr, L->row_cbeg);
  GPR_TRY(exclusive_scan(L->long_ptr, (long long)L->n_long + 1, st));
  GPR_TRY(exclusive_scan(L->row_cbeg, (long long)L->n_long + 1, st));
  GPR_CUDA(cudaMemcpyAsync(&L->long_elems, L->long_ptr + L->n_long, sizeof(long long),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaMemcpyAsync(&L->n_chunks, L->row_cbeg + L->n_long, sizeof(int),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  if (L->n_long > 0) {
    int top = 0;
    GPR_CUDA(cudaMemcpy(&top, sdeg, sizeof(int), cudaMemcpyDeviceToHost));
    L->max_row_chunks = (int)ceil_div(((long long)top + 3) & ~3LL, chunk);
  }
  GPR_TRY(dalloc(&L->long_col, (size_t)L->long_elems, "long rows"));
  GPR_TRY(dalloc(&L->chunk_row, (size_t)L->n_chunks, "chunk rows"));
  const unsigned g_long = std::min(grid_for(32LL * L->n_long), 148u * 32u);
  if (L->n_long > 0) k_fill_chunk_row<<<g_long, 256, 0, st>>>(L->n_long, L->row_cbeg, L->chunk_row);

  // SELL-32 slices over rows [n_long, n_nz).
  GPR_TRY(dalloc(&L->slice_ptr, (size_t)L->n_slices + 1, "slice offsets"));
  k_slice_lens<<<grid_for((long long)L->n_slices + 1), 256, 0, st>>>(L->n_slices, C, sdeg,
                                                                      L->slice_ptr);
  GPR_TRY(exclusive_scan(L->slice_ptr, (long long)L->n_slices + 1, st));
  GPR_CUDA(cudaMemcpyAsync(&L->sell_elems, L->slice_ptr + L->n_slices, sizeof(long long),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  GPR_TRY(dalloc(&L->sell_col, (size_t)L->sell_elems, "sell slices"));

  // Everything above needs only the row offsets and out-degrees; the column
  // indices are read from here on.  When they are still being copied in
  // (col_ready), wait for them and check their range first.
  if (col_ready) {
    GPR_CUDA(cudaStreamWaitEvent(st, col_ready, 0));
    GPR_TRY(validate_cols(nnz, m, d_col, st));
  }
  if (L->n_long > 0)
    k_fill_long<<<g_long, 256, 0, st>>>(L->n_long, m, L->perm, inv, d_rowptr, d_col, L->long_ptr,
                                        L->long_col);
  if (L->n_slices > 0)
    k_fill_sell<<<grid_for(32LL * L->n_slices), 256, 0, st>>>(
        L->n_slices, m, C, L->perm, inv, d_rowptr, d_col, sdeg, L->slice_ptr, L->sell_col);
  L->n_zblk = (int)ceil_div((long long)m - L->n_nz, kZeroRowsPerUnit);
  if (keep_csr) {
    GPR_TRY(dalloc(&L->csr_ptr, (size_t)m + 1, "relabelled row offsets"));
    GPR_TRY(dalloc(&L->csr_col, (size_t)nnz, "relabelled columns"));
    k_csr_lens<<<grid_for((long long)m + 1), 256, 0, st>>>(m, sdeg, L->csr_ptr);
    GPR_TRY(exclusive_scan(L->csr_ptr, (long long)m + 1, st));
    unsigned g = grid_for(32LL * m);
    if (g > 148u * 64u) g = 148u * 64u;
    k_fill_csr<<<g, 256, 0, st>>>(m, L->perm, inv, d_rowptr, d_col, L->csr_ptr, L->csr_col);
  }
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaStreamSynchronize(st));
  L->device_bytes = 4LL * (2LL * m) + 8LL * (L->n_long + 1) + 4LL * L->long_elems +
                    4LL * (L->n_long + 1) + 4LL * L->n_chunks + 8LL * (L->n_slices + 1) +
                    4LL * L->sell_elems + (keep_csr ? 4LL * (m + 1) + 4LL * nnz : 0);
  return GPR_OK;
}

void free_pr_layout(PrLayout *L) {
  dfree(L->perm);
  dfree(L->outdeg);
  dfree(L->long_ptr);
  dfree(L->long_col);
  dfree(L->row_cbeg);
  dfree(L->chunk_row);
  dfree(L->slice_ptr);
  dfree(L->sell_col);
  dfree(L->csr_ptr);
  dfree(L->csr_col);
  *L = PrLayout();
}

// ---------------------------------------------------------------------------
// SpMV layout (natural row order)
// ---------------------------------------------------------------------------
namespace {

__global__ void k_spmv_flags(int m, const int *__restrict__ Ap, int sell_max, int *is_long,
                             unsigned char *sell_len) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    int d = Ap[i + 1] - Ap[i];
    int lg = d > sell_max;
    is_long[i] = lg;
    sell_len[i] = lg ? (unsigned char)255 : (unsigned char)d;
  }
}

__global__ void k_spmv_long_lens(int n_long, const int *__restrict__ rows,
                                 const int *__restrict__ Ap, int chunk, long long *plen,
                                 int *nch) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_long) {
    int r = rows[i];
    long long p = ((long long)(Ap[r + 1] - Ap[r]) + 3) & ~3LL;
    plen[i] = p;
    nch[i] = (int)((p + chunk - 1) / chunk);
  } else if (i == n_long) {
    plen[i] = 0;
    nch[i] = 0;
  }
}

__global__ void k_spmv_fill_long(int n_long, const int *__restrict__ rows,
                                 const int *__restrict__ Ap, const int *__restrict__ Aj,
                                 const float *__restrict__ Ax,
                                 const long long *__restrict__ lptr, int *lcol, float *lval) {
  int lane = threadIdx.x & 31;
  long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long i = w; i < n_long; i += nw) {
    int r = rows[i];
    long long sb = Ap[r], deg = Ap[r + 1] - sb;
    long long db = lptr[i], plen = lptr[i + 1] - db;
    for (long long k = lane; k < plen; k += 32) {
      bool v = k < deg;
      lcol[db + k] = v ? Aj[sb + k] : 0;
      lval[db + k] = v ? Ax[sb + k] : 0.0f;
    }
  }
}

__global__ void k_spmv_slice_lens(int m, int n_slices, const unsigned char *__restrict__ len,
                                  long long *slen) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n_slices) {
    int mx = 0;
    for (int l = 0; l < 32; ++l) {
      long long r = 32LL * s + l;
      if (r < m && len[r] != 255 && len[r] > mx) mx = len[r];
    }
    slen[s] = 32LL * mx;
  } else if (s == n_slices) {
    slen[s] = 0;
  }
}

__global__ void k_spmv_fill_sell(int m, int n_slices, const int *__restrict__ Ap,
                                 const int *__restrict__ Aj, const float *__restrict__ Ax,
                                 const unsigned char *__restrict__ len,
                                 const long long *__restrict__ sptr, int *scol, float *sval) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 32LL * n_slices) return;
  int s = (int)(t >> 5), lane = (int)(t & 31);
  long long base = sptr[s];
  int slen = (int)((sptr[s + 1] - base) >> 5);
  long long r = 32LL * s + lane;
  int d = 0;
  long long sb = 0;
  if (r < m && len[r] != 255) {
    d = len[r];
    sb = Ap[r];
  }
  for (int j = 0; j < slen; ++j) {
    bool v = j < d;
    scol[base + 32LL * j + lane] = v ? Aj[sb + j] : 0;
    sval[base + 32LL * j + lane] = v ? Ax[sb + j] : 0.0f;
  }
}

}  // namespace

int build_spmv_layout(int m, long long nnz, const int *d_Ap, const int *d_Aj,
                      const float *d_Ax, int sell_max, int chunk, SpmvLayout *L,
                      cudaStream_t st) {
  *L = SpmvLayout();
  L->m = m;
  L->nnz = nnz;
  L->sell_max = sell_max > 254 ? 254 : sell_max;
  L->chunk = chunk;
  if (m <= 0) return GPR_OK;
  Scratch S;
  int *is_long = nullptr, *iota = nullptr, *nsel = nullptr;
  GPR_TRY(dalloc(&is_long, m, "long flags"));
  S.p[0] = is_long;
  GPR_TRY(dalloc(&iota, m, "iota"));
  S.p[1] = iota;
  GPR_TRY(dalloc(&nsel, 1, "selected count"));
  S.p[2] = nsel;
  GPR_TRY(dalloc(&L->sell_len, m, "row lengths"));
  GPR_TRY(dalloc(&L->long_rows, m, "long rows"));
  k_spmv_flags<<<grid_for(m), 256, 0, st>>>(m, d_Ap, L->sell_max, is_long, L->sell_len);
  {
    cub::CountingInputIterator<int> it(0);
    size_t tb = 0;
    GPR_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, is_long, L->long_rows, nsel, m, st));
    void *tmp = nullptr;
    GPR_TRY(dmalloc(&tmp, tb, "select scratch"));
    cudaError_t e = cub::DeviceSelect::Flagged(tmp, tb, it, is_long, L->long_rows, nsel, m, st);
    gpr::dfree(tmp);
    if (e != cudaSuccess) {
      set_error("long-row select: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  }
  GPR_CUDA(cudaMemcpyAsync(&L->n_long, nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  GPR_TRY(dalloc(&L->long_ptr, (size_t)L->n_long + 1, "long offsets"));
  GPR_TRY(dalloc(&L->row_cbeg, (size_t)L->n_long + 1, "long chunk offsets"));
  k_spmv_long_lens<<<grid_for((long long)L->n_long + 1), 256, 0, st>>>(
      L->n_long, L->long_rows, d_Ap, chunk, L->long_ptr, L->row_cbeg);
  GPR_TRY(exclusive_scan(L->long_ptr, (long long)L->n_long + 1, st));
  GPR_TRY(exclusive_scan(L->row_cbeg, (long long)L->n_long + 1, st));
  GPR_CUDA(cudaMemcpyAsync(&L->long_elems, L->long_ptr + L->n_long, sizeof(long long),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaMemcpyAsync(&L->n_chunks, L->row_cbeg + L->n_long, sizeof(int),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  GPR_TRY(dalloc(&L->long_col, (size_t)L->long_elems, "long cols"));
  GPR_TRY(dalloc(&L->long_val, (size_t)L->long_elems, "long vals"));
  GPR_TRY(dalloc(&L->chunk_row, (size_t)L->n_chunks, "chunk rows"));
  if (L->n_long > 0) {
    unsigned g = grid_for(32LL * L->n_long);
    if (g > 148u * 32u) g = 148u * 32u;
    k_fill_chunk_row<<<g, 256, 0, st>>>(L->n_long, L->row_cbeg, L->chunk_row);
    k_spmv_fill_long<<<g, 256, 0, st>>>(L->n_long, L->long_rows, d_Ap, d_Aj, d_Ax,
                                        L->long_ptr, L->long_col, L->long_val);
  }
  L->n_slices = (int)ceil_div(m, 32);
  GPR_TRY(dalloc(&L->slice_ptr, (size_t)L->n_slices + 1, "slice offsets"));
  k_spmv_slice_lens<<<grid_for((long long)L->n_slices + 1), 256, 0, st>>>(
      m, L->n_slices, L->sell_len, L->slice_ptr);
  GPR_TRY(exclusive_scan(L->slice_ptr, (long long)L->n_slices + 1, st));
  GPR_CUDA(cudaMemcpyAsync(&L->sell_elems, L->slice_ptr + L->n_slices, sizeof(long long),
                           cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  GPR_TRY(dalloc(&L->sell_col, (size_t)L->sell_elems, "sell cols"));
  GPR_TRY(dalloc(&L->sell_val, (size_t)L->sell_elems, "sell vals"));
  k_spmv_fill_sell<<<grid_for(32LL * L->n_slices), 256, 0, st>>>(
      m, L->n_slices, d_Ap, d_Aj, d_Ax, L->sell_len, L->slice_ptr, L->sell_col, L->sell_val);
  GPR_CUDA(cudaGetLastError());
  GPR_CUDA(cudaStreamSynchronize(st));
  L->device_bytes = (long long)m * 5 + 8LL * (L->n_long + 1) * 2 + 8LL * L->long_elems +
                    4LL * L->n_chunks + 8LL * (L->n_slices + 1) + 8LL * L->sell_elems;
  return GPR_OK;
}

void free_spmv_layout(SpmvLayout *L) {
  dfree(L->long_rows);
  dfree(L->long_ptr);
  dfree(L->long_col);
  dfree(L->long_val);
  dfree(L->row_cbeg);
  dfree(L->chunk_row);
  dfree(L->slice_ptr);
  dfree(L->sell_col);
  dfree(L->sell_val);
  dfree(L->sell_len);
  *L = SpmvLayout();
}

}  // namespace gpr
