// CSR construction on the GPU from the reference's push list.
//
// The reference turns a file into per-vertex lists (vector<vector<Edge>>,
// include/graph_io.h:133-261) and then into a CSR with fill_data
// (graph_io.h:21-130): optional sort of each list by column, removal of
// self-loops (order kept), removal of an entry equal to the previous kept
// one, row offsets by list length.  Its PR driver reads each file twice, once
// as the out-CSR and once transposed as the in-CSR (src/pr/main.cc:23-24).
//
// Here the file is parsed once, in parallel, into pushes in file order
// (gpr_parse_edges); a stable radix sort of the pushes by row rebuilds every
// list in push order, and the same fill_data steps run as flag kernels and
// compactions.  The in-CSR of the PR driver is the same pushes with row and
// column swapped, so one parse gives both.  With `sorted` the rows are sorted
// by (row, column) stably, where the reference's std::sort leaves the order
// of equal columns unspecified: rows and columns are identical, and the
// weights of duplicate columns may come in another order.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "gpr_internal.cuh"
#include "gpr_guard.h"

extern "C" int gpr_parse_edges(const char *path, int symmetrize, int transpose, int threads,
                               int *m_out, int *nnz_header, long long *n_push, int **row,
                               int **col, float **wt);
extern "C" void gpr_read_graph_free(void *p);

namespace {

inline unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148LL * 64) g = 148LL * 64;
  return (unsigned)g;
}

__global__ void k_push_keys(long long n, const int *__restrict__ row, const int *__restrict__ col,
                            int sorted, unsigned long long *key, int *idx) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long r = (unsigned)row[i];
    key[i] = sorted ? (r << 32) | (unsigned)col[i] : r;
    idx[i] = (int)i;
  }
}

// keep[i]: entry i (sorted order) is not a self-loop (when asked).
__global__ void k_flag_selfloops(long long n, const int *__restrict__ idx,
                                 const int *__restrict__ row, const int *__restrict__ col,
                                 int on, unsigned char *keep) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const int k = idx[i];
    keep[i] = !(on && row[k] == col[k]);
  }
}

// keep[i]: entry i is not equal to entry i-1 of the same row (when asked).
__global__ void k_flag_repeats(long long n, const int *__restrict__ idx,
                               const int *__restrict__ row, const int *__restrict__ col, int on,
                               unsigned char *keep) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    bool k = true;
    if (on && i > 0) {
      const int a = idx[i], b = idx[i - 1];
      k = !(row[a] == row[b] && col[a] == col[b]);
    }
    keep[i] = k;
  }
}

__global__ void k_emit(long long n, const int *__restrict__ idx, const int *__restrict__ row,
                       const int *__restrict__ col, const float *__restrict__ wt, int *rowcnt,
                       int *out_col, float *out_wt) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const int k = idx[i];
    out_col[i] = col[k];
    if (out_wt) out_wt[i] = wt ? wt[k] : 1.0f;
    atomicAdd(rowcnt + row[k], 1);
  }
}

__global__ void k_row_lengths(int m, const int *__restrict__ rowptr, int *deg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) deg[i] = rowptr[i + 1] - rowptr[i];
}

__global__ void k_check_range(long long n, int m, const int *__restrict__ row,
                              const int *__restrict__ col, int *flag) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    if (row[i] < 0 || row[i] >= m || col[i] < 0 || col[i] >= m) atomicOr(flag, 1);
}

// Every row id and column must name a vertex in [0, m).
int check_range(int m, long long n, const int *d_row, const int *d_col, cudaStream_t st) {
  int *flag = nullptr;
  GPR_TRY(gpr::dalloc(&flag, 1, "range flag"));
  int h = 0;
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    k_check_range<<<grid_for(n), 256, 0, st>>>(n, m, d_row, d_col, flag);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    e = cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  gpr::dfree(flag);
  if (e != cudaSuccess) {
    gpr::set_error("edge range check: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  if (h) {
    gpr::set_error("gpr_csr_from_edges: a row or column is outside [0, m)");
    return GPR_EINVAL;
  }
  return GPR_OK;
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

// Keeps the entries of idx[0, n) whose flag is set; returns the new count.
int compact(int *&idx, int *&spare, const unsigned char *keep, long long n, int *nsel,
            long long *n_out, cudaStream_t st) {
  size_t tb = 0;
  GPR_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, idx, keep, spare, nsel, n, st));
  void *tmp = nullptr;
  GPR_TRY(gpr::dmalloc(&tmp, tb, "select scratch"));
  cudaError_t e = cub::DeviceSelect::Flagged(tmp, tb, idx, keep, spare, nsel, n, st);
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, nsel, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  gpr::dfree(tmp);
  if (e != cudaSuccess) {
    gpr::set_error("compaction: %s", cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  std::swap(idx, spare);
  *n_out = h;
  return GPR_OK;
}

int build_csr(int m, long long n, const int *d_row, const int *d_col, const float *d_wt,
              bool sorted, bool rm_self, bool rm_dup, int **out_rowptr, int **out_col,
              float **out_wt, long long *nnz_out, cudaStream_t st) {
  Tmp T;
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  int *i0 = nullptr, *i1 = nullptr, *nsel = nullptr;
  unsigned char *keep = nullptr;
  GPR_TRY(T.get(&k0, (size_t)n, "push keys"));
  GPR_TRY(T.get(&k1, (size_t)n, "push keys (sorted)"));
  GPR_TRY(T.get(&i0, (size_t)n, "push order"));
  GPR_TRY(T.get(&i1, (size_t)n, "push order (sorted)"));
  GPR_TRY(T.get(&keep, (size_t)n, "keep flags"));
  GPR_TRY(T.get(&nsel, 1, "selected count"));
  int rbits = 1;
  while ((1LL << rbits) < m) ++rbits;
  if (n > 0) {
    k_push_keys<<<grid_for(n), 256, 0, st>>>(n, d_row, d_col, sorted ? 1 : 0, k0, i0);
    const int end_bit = sorted ? 32 + rbits : rbits;
    size_t tb = 0;
    GPR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0, k1, i0, i1, (int)n, 0, end_bit, st));
    void *tmp = nullptr;
    GPR_TRY(gpr::dmalloc(&tmp, tb, "sort scratch"));
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tb, k0, k1, i0, i1, (int)n, 0, end_bit, st);
    gpr::dfree(tmp);
    if (e != cudaSuccess) {
      gpr::set_error("push sort: %s", cudaGetErrorString(e));
      return GPR_ECUDA;
    }
  }
  long long cur = n;
  int *idx = i1, *spare = i0;
  if (rm_self && cur > 0) {
    k_flag_selfloops<<<grid_for(cur), 256, 0, st>>>(cur, idx, d_row, d_col, 1, keep);
    GPR_TRY(compact(idx, spare, keep, cur, nsel, &cur, st));
  }
  if (rm_dup && cur > 0) {
    k_flag_repeats<<<grid_for(cur), 256, 0, st>>>(cur, idx, d_row, d_col, 1, keep);
    GPR_TRY(compact(idx, spare, keep, cur, nsel, &cur, st));
  }
  int *rowptr = nullptr, *col = nullptr;
  float *wt = nullptr;
  int rc = gpr::dalloc(&rowptr, (size_t)m + 1, "rowptr");
  if (rc == GPR_OK) rc = gpr::dalloc(&col, (size_t)cur, "col");
  if (rc == GPR_OK && out_wt) rc = gpr::dalloc(&wt, (size_t)cur, "weight");
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaMemsetAsync(rowptr, 0, sizeof(int) * ((size_t)m + 1), st));
  if (rc == GPR_OK) {
    if (cur > 0)
      k_emit<<<grid_for(cur), 256, 0, st>>>(cur, idx, d_row, d_col, d_wt, rowptr + 1, col, wt);
    size_t tb = 0;
    cub::DeviceScan::InclusiveSum(nullptr, tb, rowptr, rowptr, m + 1, st);
    void *tmp = nullptr;
    rc = gpr::dmalloc(&tmp, tb, "scan scratch");
    if (rc == GPR_OK) {
      cudaError_t e = cub::DeviceScan::InclusiveSum(tmp, tb, rowptr, rowptr, m + 1, st);
      if (e == cudaSuccess) e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      gpr::dfree(tmp);
      if (e != cudaSuccess) {
        gpr::set_error("row offsets: %s", cudaGetErrorString(e));
        rc = GPR_ECUDA;
      }
    }
  }
  if (rc != GPR_OK) {
    gpr::dfree(rowptr);
    gpr::dfree(col);
    gpr::dfree(wt);
    return rc;
  }
  *out_rowptr = rowptr;
  *out_col = col;
  if (out_wt) *out_wt = wt;
  *nnz_out = cur;
  return GPR_OK;
}

struct HostPushes {
  int m = 0, nnz = 0;
  long long n = 0;
  int *row = nullptr, *col = nullptr;
  float *wt = nullptr;
  ~HostPushes() {
    gpr_read_graph_free(row);
    gpr_read_graph_free(col);
    gpr_read_graph_free(wt);
  }
};

int parse(const char *path, bool symmetrize, HostPushes *H) {
  if (gpr_parse_edges(path, symmetrize ? 1 : 0, 0, 0, &H->m, &H->nnz, &H->n, &H->row, &H->col,
                      &H->wt) != 0) {
    gpr::set_error("cannot read %s", path);
    return GPR_EINVAL;
  }
  return GPR_OK;
}

// Row lengths of a device CSR into a new device array: the out-degree the
// reference's read fills (include/graph_io.h:289-294).
int row_lengths(int m, const int *d_rowptr, int **out) {
  int *deg = nullptr;
  GPR_TRY(gpr::dalloc(&deg, (size_t)m, "degree"));
  int rc = GPR_OK;
  if (m > 0) {
    k_row_lengths<<<(m + 255) / 256, 256>>>(m, d_rowptr, deg);
    rc = GPR_CUDA_RC(cudaGetLastError());
  }
  if (rc == GPR_OK) rc = GPR_CUDA_RC(cudaDeviceSynchronize());
  if (rc != GPR_OK) {
    gpr::dfree(deg);
    return rc;
  }
  *out = deg;
  return GPR_OK;
}

// Releases a device CSR handed out by gpr_csr_from_edges (NULL-safe).
void free_csr(int **rowptr, int **col, float **wt) {
  gpr::dfree(*rowptr);
  gpr::dfree(*col);
  *rowptr = *col = nullptr;
  if (wt) {
    gpr::dfree(*wt);
    *wt = nullptr;
  }
}

}  // namespace

extern "C" {

int gpr_csr_from_edges(int m, long long n, const int *any_row, const int *any_col,
                       const float *any_wt, int sorted, int remove_selfloops,
                       int remove_redundents, int **d_rowptr, int **d_col, float **d_wt,
                       long long *nnz_out) {
  GPR_ENTRY_BEGIN
  if (m < 0 || n < 0 || n > 0x7fffffffLL || (n > 0 && (!any_row || !any_col)) || !d_rowptr ||
      !d_col || !nnz_out) {
    gpr::set_error("gpr_csr_from_edges: invalid arguments");
    return GPR_EINVAL;
  }
  cudaStream_t st = 0;
  void *r = nullptr, *c = nullptr, *w = nullptr;
  bool orow = false, ocol = false, owt = false;
  int rc = gpr::to_device(any_row, sizeof(int) * (size_t)n, &r, &orow, st, "rows");
  if (rc == GPR_OK) rc = gpr::to_device(any_col, sizeof(int) * (size_t)n, &c, &ocol, st, "cols");
  if (rc == GPR_OK && any_wt)
    rc = gpr::to_device(any_wt, sizeof(float) * (size_t)n, &w, &owt, st, "weights");
  if (rc == GPR_OK && n > 0) rc = check_range(m, n, (const int *)r, (const int *)c, st);
  if (rc == GPR_OK)
    rc = build_csr(m, n, (const int *)r, (const int *)c, (const float *)w, sorted != 0,
                   remove_selfloops != 0, remove_redundents != 0, d_rowptr, d_col, d_wt, nnz_out,
                   st);
  if (orow) gpr::dfree(r);
  if (ocol) gpr::dfree(c);
  if (owt) gpr::dfree(w);
  return rc;
  GPR_ENTRY_END("gpr_csr_from_edges")
}

int gpr_read_graph_gpu(const char *path, int symmetrize, int transpose, int sorted,
                       int remove_selfloops, int remove_redundents, int *m_out,
                       long long *nnz_out, int **d_rowptr, int **d_col, int **d_degree,
                       float **d_wt) {
  GPR_ENTRY_BEGIN
  if (!path || !m_out || !nnz_out || !d_rowptr || !d_col || !d_degree) {
    gpr::set_error("gpr_read_graph_gpu: NULL argument");
    return GPR_EINVAL;
  }
  HostPushes H;
  if (gpr_parse_edges(path, symmetrize, transpose, 0, &H.m, &H.nnz, &H.n, &H.row, &H.col,
                      &H.wt) != 0) {
    gpr::set_error("gpr_read_graph_gpu: cannot read %s", path);
    return GPR_EINVAL;
  }
  GPR_TRY(gpr_csr_from_edges(H.m, H.n, H.row, H.col, H.wt, sorted, remove_selfloops,
                             remove_redundents, d_rowptr, d_col, d_wt, nnz_out));
  const int rc = row_lengths(H.m, *d_rowptr, d_degree);
  if (rc != GPR_OK) {
    free_csr(d_rowptr, d_col, d_wt);
    return rc;
  }
  *m_out = H.m;
  return GPR_OK;
  GPR_ENTRY_END("gpr_read_graph_gpu")
}

int gpr_read_graph_pr(const char *path, int symmetrize, int *m_out, long long *nnz_out_csr,
                      long long *nnz_in_csr, int **d_out_rowptr, int **d_out_col,
                      int **d_out_degree, int **d_in_rowptr, int **d_in_col) {
  GPR_ENTRY_BEGIN
  if (!path || !m_out || !nnz_out_csr || !nnz_in_csr || !d_out_rowptr || !d_out_col ||
      !d_out_degree || !d_in_rowptr || !d_in_col) {
    gpr::set_error("gpr_read_graph_pr: NULL argument");
    return GPR_EINVAL;
  }
  HostPushes H;
  GPR_TRY(parse(path, symmetrize != 0, &H));
  // src/pr/main.cc:23-24: sorted = false, self-loops and repeats removed.
  GPR_TRY(gpr_csr_from_edges(H.m, H.n, H.row, H.col, nullptr, 0, 1, 1, d_out_rowptr, d_out_col,
                             nullptr, nnz_out_csr));
  // Transposed read: the same pushes with row and column swapped (with
  // symmetrize the reference ignores the transpose flag: the same lists).
  const int *in_row = symmetrize ? H.row : H.col, *in_col = symmetrize ? H.col : H.row;
  *d_in_rowptr = *d_in_col = nullptr;
  int rc = gpr_csr_from_edges(H.m, H.n, in_row, in_col, nullptr, 0, 1, 1, d_in_rowptr, d_in_col,
                              nullptr, nnz_in_csr);
  if (rc == GPR_OK) rc = row_lengths(H.m, *d_out_rowptr, d_out_degree);
  if (rc != GPR_OK) {
    free_csr(d_out_rowptr, d_out_col, nullptr);
    free_csr(d_in_rowptr, d_in_col, nullptr);
    return rc;
  }
  *m_out = H.m;
  return GPR_OK;
  GPR_ENTRY_END("gpr_read_graph_pr")
}

}  // extern "C"
