// Symmetric Gauss-Seidel smoother (multicolour) on B200.
//
// The reference (src/symgs) sweeps the colours of a vertex colouring forward
// and then backward; within a colour no two rows are neighbours, so they are
// updated in parallel (src/symgs/omp_base.cc:8-45, base.cu: a kernel per
// colour).  Each row sums x[j] * Ax[jj] over its off-diagonal entries in CSR
// order, takes the last diagonal entry, and sets x = (b - rsum) / diag when
// diag != 0.
//
// Here: the matrix is re-laid out once per colour as SELL-32 slices of 32
// rows (rows of a colour ordered by descending off-diagonal count, so a
// slice's rows have similar lengths), column-major (column, value) pairs of
// the off-diagonal entries in CSR order, with each row's diagonal and length
// beside them.  One lane per row sums in CSR order with explicitly rounded
// multiplies and adds, so every row is bit-identical to the reference (rows
// of a colour are independent, so their order does not matter).  One
// persistent cooperative launch runs all colour passes of all sweeps with a
// bounded grid barrier between passes.  The colouring is checked at create:
// a colouring with neighbours of one colour would make the result depend on
// thread timing and is rejected.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "gpr_device.cuh"
#include "gpr_internal.cuh"
#include "gpr_guard.h"

using namespace gpr::dev;

namespace {

constexpr int kSymgsBlock = 1024;
// Two 1024-thread CTAs per SM (32 registers) and 4 entries per lane in
// flight.  A pass is a chain of dependent loads per slice (row data, entries,
// the gathered x) ended by a grid barrier; with twice the warps a colour's
// 8,192 slices of the 128^3 stencil take one slice per warp instead of two.
// Measured per sweep on that stencil (same box): one CTA per SM with 24
// entries in flight 0.264 ms; two CTAs with 2 / 3 / 4 / 6 / 8 entries 0.218 /
// 0.212 / 0.212 / 0.220 / 0.245 ms (8: spills).
constexpr int kSymgsU = 4;
constexpr int kSymgsCtasPerSm = 2;

struct SymgsArgs {
  int nc;
  const int *cslice;      // [nc + 1] first slice of each colour
  const long long *sptr;  // [n_slices + 1] entry offsets (multiples of 32)
  const int *scol;
  const float *sval;
  const int *srow;        // [n_slices * 32] row of each lane (-1: none)
  const int *slen;        // [n_slices * 32] off-diagonal entries of each lane's row
  const float *sdiag;     // [n_slices * 32] diagonal of each lane's row (0: none)
  float *x;
  const float *b;
  int sweeps;
  unsigned *bar;
  int *status;
  unsigned bar_expect;
  long long timeout_ns;
};

__global__ void __launch_bounds__(kSymgsBlock, kSymgsCtasPerSm) k_symgs(SymgsArgs a) {
  const int lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (kSymgsBlock / 32) + (threadIdx.x >> 5);
  const int nw = gridDim.x * (kSymgsBlock / 32);
  const Policies pol = make_policies();
  // A pass sets each row of its colour from the x of other colours only (no
  // row has a neighbour of its own colour, the diagonal is not in the sum),
  // so a pass that repeats the colour of the pass before it -- the turn from
  // forward to backward, and colour 0 from one sweep to the next -- would
  // write the same values again: it is skipped, with its barrier.
  int prev = -1;
  unsigned episode = 0;  // barriers passed in this launch
  for (int sw = 0; sw < a.sweeps; ++sw) {
    for (int p = 0; p < 2 * a.nc; ++p) {
      const int c = p < a.nc ? p : 2 * a.nc - 1 - p;
      if (c == prev) continue;
      prev = c;
      for (int s = a.cslice[c] + gw; s < a.cslice[c + 1]; s += nw) {
        const int k = s * 32 + lane;
        const int r = a.srow[k], len = a.slen[k];
        const long long b0 = a.sptr[s];
        const int width = (int)((a.sptr[s + 1] - b0) >> 5);
        float rsum = 0.f;
        for (int j0 = 0; j0 < width; j0 += kSymgsU) {
          int cj[kSymgsU];
          float vj[kSymgsU];
#pragma unroll
          for (int q = 0; q < kSymgsU; ++q) {
            const bool in = j0 + q < len;
            cj[q] = in ? ld_s32_stream(a.scol + b0 + 32LL * (j0 + q) + lane, pol.stream) : -1;
            vj[q] = in ? ld_f32_stream(a.sval + b0 + 32LL * (j0 + q) + lane, pol.stream) : 0.f;
          }
          float xv[kSymgsU];
#pragma unroll
          for (int q = 0; q < kSymgsU; ++q) xv[q] = cj[q] >= 0 ? ld_contrib(a.x + cj[q], pol.keep) : 0.f;
#pragma unroll
          for (int q = 0; q < kSymgsU; ++q)
            if (cj[q] >= 0) rsum = __fadd_rn(rsum, __fmul_rn(xv[q], vj[q]));
        }
        if (r >= 0) {
          const float d = a.sdiag[k];
          if (d != 0.f) a.x[r] = __fdiv_rn(__fsub_rn(a.b[r], rsum), d);
        }
      }
      if (!grid_barrier_count(a.bar, a.bar_expect * ++episode, a.status, a.timeout_ns)) return;
    }
  }
}

}  // namespace

struct gpr_symgs {
  int device = 0, m = 0, nc = 0;
  long long nnz = 0;
  int n_slices = 0;
  long long slots = 0;
  int *cslice = nullptr;
  long long *sptr = nullptr;
  int *scol = nullptr, *srow = nullptr, *slen = nullptr;
  float *sval = nullptr, *sdiag = nullptr;
  float *x_tmp = nullptr, *b_tmp = nullptr;
  unsigned *bar = nullptr;
  int *status = nullptr;
  int grid = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

namespace {

void destroy_symgs(gpr_symgs *h) {
  if (!h) return;
  void *p[] = {h->cslice, h->sptr, h->scol, h->srow, h->slen, h->sval,
               h->sdiag,  h->x_tmp, h->b_tmp, h->bar, h->status};
  for (void *q : p) gpr::dfree(q);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

template <typename T>
int upload(T **d, const std::vector<T> &v, const char *what, cudaStream_t st) {
  GPR_TRY(gpr::dalloc(d, v.size(), what));
  if (!v.empty())
    GPR_CUDA(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st));
  return GPR_OK;
}

// Host copy of an array given as host or device memory.
template <typename T>
int to_host(const T *any, size_t n, std::vector<T> *h) {
  h->resize(n);
  if (n) GPR_CUDA(cudaMemcpy(h->data(), any, sizeof(T) * n, cudaMemcpyDefault));
  return GPR_OK;
}

int build_symgs(gpr_symgs *h, const int *Ap, const int *Aj, const float *Ax, const int *idx,
                const int *co) {
  const int m = h->m, nc = h->nc;
  // Validation: row offsets, columns, the permutation, colour boundaries,
  // and that no off-diagonal entry joins two rows of one colour.
  if (Ap[0] != 0 || (long long)Ap[m] != h->nnz) {
    gpr::set_error("gpr_symgs_create: malformed row offsets");
    return GPR_EINVAL;
  }
  if (co[0] != 0 || co[nc] != m) {
    gpr::set_error("gpr_symgs_create: colour offsets must run from 0 to m");
    return GPR_EINVAL;
  }
  std::vector<int> color(m, -1);
  for (int c = 0; c < nc; ++c) {
    if (co[c + 1] < co[c]) {
      gpr::set_error("gpr_symgs_create: colour offsets decrease");
      return GPR_EINVAL;
    }
    for (int i = co[c]; i < co[c + 1]; ++i) {
      const int r = idx[i];
      if (r < 0 || r >= m || color[r] >= 0) {
        gpr::set_error("gpr_symgs_create: indices are not a permutation of the rows");
        return GPR_EINVAL;
      }
      color[r] = c;
    }
  }
  std::vector<int> offd(m, 0);
  std::vector<float> diag(m, 0.f);
  for (int r = 0; r < m; ++r) {
    if (Ap[r + 1] < Ap[r]) {
      gpr::set_error("gpr_symgs_create: malformed row offsets");
      return GPR_EINVAL;
    }
    for (int e = Ap[r]; e < Ap[r + 1]; ++e) {
      const int j = Aj[e];
      if (j < 0 || j >= m) {
        gpr::set_error("gpr_symgs_create: column out of range");
        return GPR_EINVAL;
      }
      if (j == r) {
        diag[r] = Ax[e];  // the last diagonal entry counts
      } else {
        if (color[j] == color[r]) {
          gpr::set_error("gpr_symgs_create: rows %d and %d share colour %d but are joined by "
                         "an entry (not a valid colouring)", r, j, color[r]);
          return GPR_EINVAL;
        }
        ++offd[r];
      }
    }
  }
  // Slices: per colour, rows by descending off-diagonal count (stable).
  std::vector<int> cslice(nc + 1, 0), srow, slen;
  std::vector<float> sdiag;
  std::vector<long long> sptr(1, 0);
  for (int c = 0; c < nc; ++c) {
    std::vector<int> rows(idx + co[c], idx + co[c + 1]);
    std::stable_sort(rows.begin(), rows.end(), [&](int a, int b) { return offd[a] > offd[b]; });
    for (size_t i = 0; i < rows.size(); i += 32) {
      int width = 0;
      for (int l = 0; l < 32; ++l) {
        const bool in = i + l < rows.size();
        const int r = in ? rows[i + l] : -1;
        srow.push_back(r);
        slen.push_back(in ? offd[r] : 0);
        sdiag.push_back(in ? diag[r] : 0.f);
        if (in) width = std::max(width, offd[r]);
      }
      sptr.push_back(sptr.back() + 32LL * width);
    }
    cslice[c + 1] = (int)srow.size() / 32;
  }
  h->n_slices = (int)srow.size() / 32;
  h->slots = sptr.back();
  std::vector<int> scol((size_t)h->slots, -1);
  std::vector<float> sval((size_t)h->slots, 0.f);
  for (int s = 0; s < h->n_slices; ++s)
    for (int l = 0; l < 32; ++l) {
      const int r = srow[(size_t)s * 32 + l];
      if (r < 0) continue;
      long long j = 0;
      for (int e = Ap[r]; e < Ap[r + 1]; ++e) {
        if (Aj[e] == r) continue;
        scol[(size_t)(sptr[s] + 32 * j + l)] = Aj[e];
        sval[(size_t)(sptr[s] + 32 * j + l)] = Ax[e];
        ++j;
      }
    }
  cudaStream_t st = h->st;
  GPR_TRY(upload(&h->cslice, cslice, "colour slices", st));
  GPR_TRY(upload(&h->sptr, sptr, "slice offsets", st));
  GPR_TRY(upload(&h->scol, scol, "slice columns", st));
  GPR_TRY(upload(&h->sval, sval, "slice values", st));
  GPR_TRY(upload(&h->srow, srow, "slice rows", st));
  GPR_TRY(upload(&h->slen, slen, "slice lengths", st));
  GPR_TRY(upload(&h->sdiag, sdiag, "slice diagonals", st));
  GPR_CUDA(cudaStreamSynchronize(st));
  return GPR_OK;
}

}  // namespace

extern "C" {

int gpr_symgs_create(int m, long long nnz, const int *any_Ap, const int *any_Aj,
                     const float *any_Ax, const int *any_indices, const int *any_color_offsets,
                     int n_colors, gpr_symgs **out) {
  GPR_ENTRY_BEGIN
  if (!out) {
    gpr::set_error("gpr_symgs_create: NULL out");
    return GPR_EINVAL;
  }
  *out = nullptr;
  if (m < 1 || nnz < 0 || nnz > 0x7fffffffLL || n_colors < 1 || !any_Ap || !any_indices ||
      !any_color_offsets || (nnz > 0 && (!any_Aj || !any_Ax))) {
    gpr::set_error("gpr_symgs_create: invalid arguments");
    return GPR_EINVAL;
  }
  std::vector<int> Ap, Aj, idx, co;
  std::vector<float> Ax;
  GPR_TRY(to_host(any_Ap, (size_t)m + 1, &Ap));
  GPR_TRY(to_host(any_Aj, (size_t)nnz, &Aj));
  GPR_TRY(to_host(any_Ax, (size_t)nnz, &Ax));
  GPR_TRY(to_host(any_indices, (size_t)m, &idx));
  GPR_TRY(to_host(any_color_offsets, (size_t)n_colors + 1, &co));
  gpr_symgs *h = new gpr_symgs();
  h->m = m;
  h->nnz = nnz;
  h->nc = n_colors;
  int rc = GPR_OK;
  if (cudaGetDevice(&h->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->e0) != cudaSuccess || cudaEventCreate(&h->e1) != cudaSuccess) {
    gpr::set_error("gpr_symgs_create: stream / event creation failed");
    rc = GPR_ECUDA;
  }
  if (rc == GPR_OK) rc = build_symgs(h, Ap.data(), Aj.data(), Ax.data(), idx.data(), co.data());
  if (rc == GPR_OK) rc = gpr::dalloc(&h->x_tmp, (size_t)m, "x staging");
  if (rc == GPR_OK) rc = gpr::dalloc(&h->b_tmp, (size_t)m, "b staging");
  if (rc == GPR_OK) rc = gpr::dalloc(&h->bar, 2, "barrier");
  if (rc == GPR_OK) rc = gpr::dalloc(&h->status, 4, "status");
  if (rc == GPR_OK) {
    int sms = 0, per_sm = 0, coop = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)k_symgs, kSymgsBlock, 0);
    if (!coop || per_sm < 1) {
      gpr::set_error("gpr_symgs_create: the device cannot co-schedule the persistent kernel");
      rc = GPR_EUNSUPPORTED;
    }
    int most = 0;  // slices of the largest colour
    for (int c = 0; c < n_colors; ++c) most = std::max(most, co[c + 1] - co[c]);
    h->grid = std::max(1, std::min(sms * per_sm, (int)gpr::ceil_div(gpr::ceil_div(most, 32), 32)));
  }
  if (rc != GPR_OK) {
    destroy_symgs(h);
    return rc;
  }
  *out = h;
  return GPR_OK;
  GPR_ENTRY_END("gpr_symgs_create")
}

int gpr_symgs_destroy(gpr_symgs *h) {
  destroy_symgs(h);
  return GPR_OK;
}

int gpr_symgs_apply(gpr_symgs *h, float *any_x, const float *any_b, int sweeps, double *loop_ms) {
  GPR_ENTRY_BEGIN
  if (!h || !any_x || !any_b || sweeps < 0) {
    gpr::set_error("gpr_symgs_apply: invalid arguments");
    return GPR_EINVAL;
  }
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != h->device) GPR_CUDA(cudaSetDevice(h->device));
  cudaStream_t st = h->st;
  const size_t bytes = sizeof(float) * (size_t)h->m;
  const bool hx = !gpr::is_device_ptr(any_x), hb = !gpr::is_device_ptr(any_b);
  float *dx = hx ? h->x_tmp : any_x;
  const float *db = hb ? h->b_tmp : any_b;
  if (hx) GPR_CUDA(cudaMemcpyAsync(dx, any_x, bytes, cudaMemcpyHostToDevice, st));
  if (hb) GPR_CUDA(cudaMemcpyAsync(h->b_tmp, any_b, bytes, cudaMemcpyHostToDevice, st));
  SymgsArgs a;
  memset(&a, 0, sizeof(a));
  a.nc = h->nc;
  a.cslice = h->cslice;
  a.sptr = h->sptr;
  a.scol = h->scol;
  a.sval = h->sval;
  a.srow = h->srow;
  a.slen = h->slen;
  a.sdiag = h->sdiag;
  a.x = dx;
  a.b = db;
  a.sweeps = sweeps;
  a.bar = h->bar;
  a.status = h->status;
  a.bar_expect = (unsigned)h->grid;
  a.timeout_ns = 5000000000LL;
  GPR_CUDA(cudaMemsetAsync(h->bar, 0, 2 * sizeof(unsigned), st));
  GPR_CUDA(cudaMemsetAsync(h->status, 0, 4 * sizeof(int), st));
  GPR_CUDA(cudaEventRecord(h->e0, st));
  if (sweeps > 0) {
    void *args[] = {&a};
    GPR_CUDA(cudaLaunchCooperativeKernel((const void *)k_symgs, dim3(h->grid), dim3(kSymgsBlock),
                                         args, 0, st));
  }
  GPR_CUDA(cudaEventRecord(h->e1, st));
  int hs = 0;
  GPR_CUDA(cudaMemcpyAsync(&hs, h->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  if (hx) GPR_CUDA(cudaMemcpyAsync(any_x, dx, bytes, cudaMemcpyDeviceToHost, st));
  GPR_CUDA(cudaStreamSynchronize(st));
  if (loop_ms) {
    float ms = 0.f;
    GPR_CUDA(cudaEventElapsedTime(&ms, h->e0, h->e1));
    *loop_ms = ms;
  }
  if (cur != h->device && cur >= 0) cudaSetDevice(cur);
  if (hs & 1) {
    gpr::set_error("gpr_symgs_apply: grid barrier wait exceeded 5 s");
    return GPR_ETIMEOUT;
  }
  return GPR_OK;
  GPR_ENTRY_END("gpr_symgs_apply")
}

int gpr_symgs_solver(int m, int nnz, const int *Ap, const int *Aj, const int *indices,
                     const float *Ax, float *x, const float *b, const int *color_offsets,
                     int n_colors) {
  GPR_ENTRY_BEGIN
  gpr_symgs *h = nullptr;
  GPR_TRY(gpr_symgs_create(m, nnz, Ap, Aj, Ax, indices, color_offsets, n_colors, &h));
  const int rc = gpr_symgs_apply(h, x, b, 1, nullptr);
  gpr_symgs_destroy(h);
  return rc;
  GPR_ENTRY_END("gpr_symgs_solver")
}

}  // extern "C"
