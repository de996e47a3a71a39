// Seeded synthetic inputs generated on the GPU.
//
// The reference ships no generator (its inputs are external .gr/.mtx files,
// include/graph_io.h:133-261).  These produce the benchmark inputs directly
// in device memory.  Every draw is a pure function of (seed, index) through
// the SplitMix64 finaliser (Steele, Lea, Flood 2014), so the same graph can
// be rebuilt anywhere from its parameters.
#include <cub/cub.cuh>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gpr_internal.cuh"
#include "gpr_guard.h"

namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
  return mix64(seed ^ mix64(a * 0x9E3779B97F4A7C15ULL + b));
}

struct Scramble {
  uint64_t mask, k1, k2, k3;
  int sh;
};

Scramble make_scramble(int scale, uint64_t seed) {
  Scramble s;
  s.mask = (scale >= 32) ? 0xffffffffULL : ((1ULL << scale) - 1ULL);
  s.k1 = (mix64(seed ^ 0x1234567ULL) | 1ULL) & s.mask;
  s.k2 = (mix64(seed ^ 0x89abcdefULL) | 1ULL) & s.mask;
  s.k3 = mix64(seed ^ 0x5555ULL) & s.mask;
  s.sh = scale / 2 + 1;
  return s;
}

// Bijection of [0, 2^scale): multiply by an odd constant / xorshift, twice.
__device__ __forceinline__ uint32_t scramble(uint32_t v, const Scramble &s) {
  uint64_t x = v;
  x = (x * s.k1) & s.mask;
  x ^= x >> s.sh;
  x = (x * s.k2) & s.mask;
  x ^= x >> s.sh;
  x = (x + s.k3) & s.mask;
  return (uint32_t)x;
}

constexpr uint64_t kDropKey = ~0ULL;

// Edge e -> key (dst << 32 | src); self-loops map to kDropKey.
__global__ void k_rmat_keys(long long ne, int scale, uint32_t t0, uint32_t t1, uint32_t t2,
                            uint64_t seed, int do_scramble, Scramble sc, uint64_t *keys) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += stride) {
    uint32_t s = 0, t = 0;
    uint64_t h = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 1) == 0) h = hash3(seed, (uint64_t)e, (uint64_t)(l >> 1));
      const uint32_t r = (l & 1) ? (uint32_t)(h >> 32) : (uint32_t)h;
      uint32_t sb, tb;
      if (r < t0) { sb = 0; tb = 0; }
      else if (r < t1) { sb = 0; tb = 1; }
      else if (r < t2) { sb = 1; tb = 0; }
      else { sb = 1; tb = 1; }
      s = (s << 1) | sb;
      t = (t << 1) | tb;
    }
    if (do_scramble) {
      s = scramble(s, sc);
      t = scramble(t, sc);
    }
    keys[e] = (s == t) ? kDropKey : (((uint64_t)t << 32) | s);
  }
}

__global__ void k_split_keys(long long n, const uint64_t *__restrict__ keys, int *col,
                             int *indeg, int *outdeg) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t k = keys[i];
    const int src = (int)(uint32_t)k, dst = (int)(k >> 32);
    col[i] = src;
    atomicAdd(indeg + dst, 1);
    atomicAdd(outdeg + src, 1);
  }
}

__global__ void k_stencil_counts(int n, int *cnt) {
  const long long m = (long long)n * n * n;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < m) {
    const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((long long)n * n));
    const int cx = 1 + (x > 0) + (x < n - 1), cy = 1 + (y > 0) + (y < n - 1),
              cz = 1 + (z > 0) + (z < n - 1);
    cnt[i] = cx * cy * cz;
  } else if (i == m) {
    cnt[i] = 0;
  }
}

__global__ void k_stencil_fill(int n, const int *__restrict__ Ap, int *Aj, float *Ax) {
  const long long m = (long long)n * n * n;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((long long)n * n));
  long long p = Ap[i];
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int zz = z + dz, yy = y + dy, xx = x + dx;
        if (zz < 0 || zz >= n || yy < 0 || yy >= n || xx < 0 || xx >= n) continue;
        Aj[p] = (zz * n + yy) * n + xx;
        Ax[p] = (dz == 0 && dy == 0 && dx == 0) ? 26.0f : -1.0f;
        ++p;
      }
}

__global__ void k_uniform(long long n, uint64_t seed, float *out) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = (float)(hash3(seed, (uint64_t)i, 0x7u) >> 40) * (1.0f / 16777216.0f);
}

unsigned capped_grid(long long n) {
  long long g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148LL * 64) g = 148LL * 64;
  return (unsigned)g;
}

// Keys (dst << 32 | src, kDropKey for dropped draws) -> in-CSR with ascending
// distinct sources per row, and out-degrees.  k0 holds the keys; k1 is
// scratch of the same size.  Allocates the three outputs.
int csr_from_keys(long long ne, int m, uint64_t *k0, uint64_t *k1, int **d_rowptr, int **d_col,
                  int **d_outdeg, long long *nnz_out) {
  cudaStream_t st = 0;
  int *nsel = nullptr;
  void *tmp = nullptr;
  int rc = GPR_OK;
  long long nnz = 0;
  int *rowptr = nullptr, *col = nullptr, *outdeg = nullptr;
  do {
    if ((rc = gpr::dalloc(&nsel, 1, "unique count")) != GPR_OK) break;
    cub::DoubleBuffer<uint64_t> db(k0, k1);
    size_t tb = 0, tb2 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, tb, db, (int)ne, 0, 64, st);
    cub::DeviceSelect::Unique(nullptr, tb2, k0, k1, nsel, (int)ne, st);
    if (tb2 > tb) tb = tb2;
    if ((rc = gpr::dmalloc(&tmp, tb, "sort scratch")) != GPR_OK) break;
    cudaError_t e = cub::DeviceRadixSort::SortKeys(tmp, tb, db, (int)ne, 0, 64, st);
    uint64_t *sorted = db.Current(), *uniq = db.Alternate();
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(tmp, tb, sorted, uniq, nsel, (int)ne, st);
    int nu = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nu, nsel, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    uint64_t lastkey = 0;
    if (e == cudaSuccess && nu > 0)
      e = cudaMemcpy(&lastkey, uniq + nu - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      gpr::set_error("edge sort: %s", cudaGetErrorString(e));
      rc = GPR_ECUDA;
      break;
    }
    nnz = (nu > 0 && lastkey == kDropKey) ? nu - 1 : nu;
    if ((rc = gpr::dalloc(&rowptr, (size_t)m + 1, "rowptr")) != GPR_OK) break;
    if ((rc = gpr::dalloc(&col, (size_t)nnz, "col")) != GPR_OK) break;
    if ((rc = gpr::dalloc(&outdeg, (size_t)m, "outdeg")) != GPR_OK) break;
    if ((rc = GPR_CUDA_RC(cudaMemsetAsync(rowptr, 0, sizeof(int) * ((size_t)m + 1), st))) != GPR_OK)
      break;
    if ((rc = GPR_CUDA_RC(cudaMemsetAsync(outdeg, 0, sizeof(int) * (size_t)m, st))) != GPR_OK) break;
    k_split_keys<<<capped_grid(nnz), 256, 0, st>>>(nnz, uniq, col, rowptr, outdeg);
    gpr::dfree(tmp);
    tmp = nullptr;
    size_t ts = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, ts, rowptr, rowptr, m + 1, st);
    if ((rc = gpr::dmalloc(&tmp, ts, "scan scratch")) != GPR_OK) break;
    e = cub::DeviceScan::ExclusiveSum(tmp, ts, rowptr, rowptr, m + 1, st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      gpr::set_error("CSR from edges: %s", cudaGetErrorString(e));
      rc = GPR_ECUDA;
      break;
    }
  } while (0);
  gpr::dfree(nsel);
  gpr::dfree(tmp);
  if (rc != GPR_OK) {
    gpr::dfree(rowptr);
    gpr::dfree(col);
    gpr::dfree(outdeg);
    return rc;
  }
  *d_rowptr = rowptr;
  *d_col = col;
  *d_outdeg = outdeg;
  *nnz_out = nnz;
  return GPR_OK;
}

// Size of graph g of a multi-graph batch: log-uniform in [m_min, m_max].
int multigraph_size(int g, int m_min, int m_max, uint64_t seed) {
  const uint64_t h = hash3(seed, (uint64_t)g, 0x6d67u);
  const double u = (double)(h >> 11) * 0x1.0p-53;
  const double lo = log((double)m_min), hi = log((double)m_max);
  const double t = u * (hi - lo);
  int m = (int)floor(exp(lo + t));
  return std::min(std::max(m, m_min), m_max);
}

// Draw of a Chung-Lu endpoint: first i in [0, m) with P[i] > x * P[m - 1].
__device__ __forceinline__ int cl_draw(uint64_t h, const double *__restrict__ P, int m) {
  const double x = (double)(h >> 11) * 0x1.0p-53;
  const double y = __dmul_rn(x, P[m - 1]);
  int lo = 0, hi = m;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (P[mid] > y) hi = mid;
    else lo = mid + 1;
  }
  return lo < m ? lo : m - 1;
}

// Draw e of the batch (graph found by binary search over the draw offsets)
// -> global key (dst << 32 | src), self-loops -> kDropKey.  Odd graphs are
// Chung-Lu, even graphs Erdos-Renyi.
__global__ void k_multi_keys(long long ne, int G, const long long *__restrict__ eoff,
                             const int *__restrict__ voff, const unsigned long long *__restrict__ gs,
                             const double *__restrict__ P, uint64_t *keys) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < ne; e += stride) {
    int lo = 0, hi = G;  // last g with eoff[g] <= e
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (eoff[mid] <= e) lo = mid;
      else hi = mid;
    }
    const int g = lo, v0 = voff[g], mg = voff[g + 1] - v0;
    const uint64_t le = (uint64_t)(e - eoff[g]);
    const uint64_t h = hash3(gs[g], le, 0);
    uint32_t s, t;
    if (g & 1) {
      s = (uint32_t)cl_draw(h, P, mg);
      t = (uint32_t)cl_draw(hash3(gs[g], le, 1), P, mg);
    } else {
      s = (uint32_t)(((h >> 32) * (uint64_t)mg) >> 32);
      t = (uint32_t)(((h & 0xffffffffULL) * (uint64_t)mg) >> 32);
    }
    keys[e] = (s == t) ? kDropKey : (((uint64_t)(v0 + t) << 32) | (uint64_t)(v0 + s));
  }
}

}  // namespace

extern "C" {

int gpr_gen_rmat(int scale, int edge_factor, double a, double b, double c,
                 unsigned long long seed, int do_scramble, int **d_rowptr, int **d_col,
                 int **d_outdeg, long long *nnz_out) {
  GPR_ENTRY_BEGIN
  if (scale < 1 || scale > 30 || edge_factor < 1 || !d_rowptr || !d_col || !d_outdeg ||
      !nnz_out || !(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) {
    gpr::set_error("gpr_gen_rmat: invalid arguments");
    return GPR_EINVAL;
  }
  const int m = 1 << scale;
  const long long ne = (long long)m * edge_factor;
  if (ne > 0x7fffffffLL) {
    gpr::set_error("gpr_gen_rmat: %lld edges exceed int32 CSR", ne);
    return GPR_EINVAL;
  }
  *d_rowptr = nullptr;
  *d_col = nullptr;
  *d_outdeg = nullptr;
  const uint32_t t0 = (uint32_t)(a * 4294967296.0);
  const uint32_t t1 = (uint32_t)((a + b) * 4294967296.0);
  const uint32_t t2 = (uint32_t)((a + b + c) * 4294967296.0);
  uint64_t *k0 = nullptr, *k1 = nullptr;
  int rc = gpr::dalloc(&k0, (size_t)ne, "rmat keys");
  if (rc == GPR_OK) rc = gpr::dalloc(&k1, (size_t)ne, "rmat keys (alt)");
  if (rc == GPR_OK) {
    k_rmat_keys<<<capped_grid(ne), 256>>>(ne, scale, t0, t1, t2, seed, do_scramble,
                                           make_scramble(scale, seed), k0);
    rc = GPR_CUDA_RC(cudaGetLastError());
  }
  if (rc == GPR_OK) {
    rc = csr_from_keys(ne, m, k0, k1, d_rowptr, d_col, d_outdeg, nnz_out);
  }
  gpr::dfree(k0);
  gpr::dfree(k1);
  return rc;
  GPR_ENTRY_END("gpr_gen_rmat")
}

int gpr_gen_multigraph(int n_graphs, int m_min, int m_max, int er_deg, int cl_deg, double gamma,
                       unsigned long long seed, int *h_voff, int **d_rowptr, int **d_col,
                       int **d_outdeg, long long *nnz_out) {
  GPR_ENTRY_BEGIN
  if (n_graphs < 1 || m_min < 1 || m_max < m_min || er_deg < 1 || cl_deg < 1 ||
      !(gamma > 1.0) || !h_voff || !d_rowptr || !d_col || !d_outdeg || !nnz_out) {
    gpr::set_error("gpr_gen_multigraph: invalid arguments");
    return GPR_EINVAL;
  }
  *d_rowptr = nullptr;
  *d_col = nullptr;
  *d_outdeg = nullptr;
  std::vector<int> voff(n_graphs + 1, 0);
  std::vector<long long> eoff(n_graphs + 1, 0);
  std::vector<unsigned long long> gs(n_graphs);
  int m_big = 1;
  for (int g = 0; g < n_graphs; ++g) {
    const int mg = multigraph_size(g, m_min, m_max, seed);
    m_big = std::max(m_big, mg);
    if ((long long)voff[g] + mg > 0x7fffffffLL) {
      gpr::set_error("gpr_gen_multigraph: more than 2^31-1 vertices");
      return GPR_EINVAL;
    }
    voff[g + 1] = voff[g] + mg;
    eoff[g + 1] = eoff[g] + (long long)mg * ((g & 1) ? cl_deg : er_deg);
    gs[g] = hash3(seed, (uint64_t)g, 0x9e37u);
  }
  const long long ne = eoff[n_graphs];
  if (ne > 0x7fffffffLL) {
    gpr::set_error("gpr_gen_multigraph: %lld edge draws exceed int32 CSR", ne);
    return GPR_EINVAL;
  }
  // Chung-Lu weights (j + 1)^(-1/(gamma - 1)), prefix-summed in index order.
  std::vector<double> P(m_big);
  {
    const double alpha = -1.0 / (gamma - 1.0);
    double acc = 0.0;
    for (int i = 0; i < m_big; ++i) {
      acc += pow((double)(i + 1), alpha);
      P[i] = acc;
    }
  }
  uint64_t *k0 = nullptr, *k1 = nullptr;
  int *dvoff = nullptr;
  long long *deoff = nullptr;
  unsigned long long *dgs = nullptr;
  double *dP = nullptr;
  int rc = gpr::dalloc(&k0, (size_t)ne, "multigraph keys");
  if (rc == GPR_OK) rc = gpr::dalloc(&k1, (size_t)ne, "multigraph keys (alt)");
  if (rc == GPR_OK) rc = gpr::dalloc(&dvoff, (size_t)n_graphs + 1, "vertex offsets");
  if (rc == GPR_OK) rc = gpr::dalloc(&deoff, (size_t)n_graphs + 1, "draw offsets");
  if (rc == GPR_OK) rc = gpr::dalloc(&dgs, (size_t)n_graphs, "graph seeds");
  if (rc == GPR_OK) rc = gpr::dalloc(&dP, (size_t)m_big, "Chung-Lu prefix");
  if (rc == GPR_OK)
    rc = GPR_CUDA_RC(cudaMemcpy(dvoff, voff.data(), sizeof(int) * voff.size(), cudaMemcpyHostToDevice));
  if (rc == GPR_OK)
    rc = GPR_CUDA_RC(
        cudaMemcpy(deoff, eoff.data(), sizeof(long long) * eoff.size(), cudaMemcpyHostToDevice));
  if (rc == GPR_OK)
    rc = GPR_CUDA_RC(
        cudaMemcpy(dgs, gs.data(), sizeof(unsigned long long) * gs.size(), cudaMemcpyHostToDevice));
  if (rc == GPR_OK)
    rc = GPR_CUDA_RC(cudaMemcpy(dP, P.data(), sizeof(double) * P.size(), cudaMemcpyHostToDevice));
  if (rc == GPR_OK) {
    k_multi_keys<<<capped_grid(ne), 256>>>(ne, n_graphs, deoff, dvoff, dgs, dP, k0);
    rc = GPR_CUDA_RC(cudaGetLastError());
  }
  if (rc == GPR_OK) {
    rc = csr_from_keys(ne, voff[n_graphs], k0, k1, d_rowptr, d_col, d_outdeg, nnz_out);
  }
  gpr::dfree(k0);
  gpr::dfree(k1);
  gpr::dfree(dvoff);
  gpr::dfree(deoff);
  gpr::dfree(dgs);
  gpr::dfree(dP);
  if (rc == GPR_OK) memcpy(h_voff, voff.data(), sizeof(int) * voff.size());
  return rc;
  GPR_ENTRY_END("gpr_gen_multigraph")
}

int gpr_gen_stencil27(int n, int **d_Ap, int **d_Aj, float **d_Ax, long long *nnz_out) {
  GPR_ENTRY_BEGIN
  if (n < 1 || n > 1290 || !d_Ap || !d_Aj || !d_Ax || !nnz_out) {
    gpr::set_error("gpr_gen_stencil27: invalid arguments");
    return GPR_EINVAL;
  }
  const long long m = (long long)n * n * n;
  const long long nnz = (long long)(3 * n - 2) * (3 * n - 2) * (3 * n - 2);
  if (nnz > 0x7fffffffLL) {
    gpr::set_error("gpr_gen_stencil27: %lld nonzeros exceed int32 CSR", nnz);
    return GPR_EINVAL;
  }
  int *Ap = nullptr, *Aj = nullptr;
  float *Ax = nullptr;
  void *tmp = nullptr;
  int rc = GPR_OK;
  do {
    if ((rc = gpr::dalloc(&Ap, (size_t)m + 1, "Ap")) != GPR_OK) break;
    if ((rc = gpr::dalloc(&Aj, (size_t)nnz, "Aj")) != GPR_OK) break;
    if ((rc = gpr::dalloc(&Ax, (size_t)nnz, "Ax")) != GPR_OK) break;
    const unsigned g = (unsigned)((m + 1 + 255) / 256);
    k_stencil_counts<<<g, 256>>>(n, Ap);
    size_t ts = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, ts, Ap, Ap, (int)(m + 1));
    if ((rc = gpr::dmalloc(&tmp, ts, "scan scratch")) != GPR_OK) break;
    cub::DeviceScan::ExclusiveSum(tmp, ts, Ap, Ap, (int)(m + 1));
    k_stencil_fill<<<g, 256>>>(n, Ap, Aj, Ax);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      gpr::set_error("gpr_gen_stencil27: %s", cudaGetErrorString(e));
      rc = GPR_ECUDA;
    }
  } while (0);
  gpr::dfree(tmp);
  if (rc != GPR_OK) {
    gpr::dfree(Ap);
    gpr::dfree(Aj);
    gpr::dfree(Ax);
    return rc;
  }
  *d_Ap = Ap;
  *d_Aj = Aj;
  *d_Ax = Ax;
  *nnz_out = nnz;
  return GPR_OK;
  GPR_ENTRY_END("gpr_gen_stencil27")
}

int gpr_gen_uniform(long long n, unsigned long long seed, float *d_out) {
  if (n < 0 || (n > 0 && !d_out)) {
    gpr::set_error("gpr_gen_uniform: invalid arguments");
    return GPR_EINVAL;
  }
  if (n == 0) return GPR_OK;
  k_uniform<<<capped_grid(n), 256>>>(n, seed, d_out);
  GPR_CUDA(cudaGetLastError());
  return GPR_OK;
}

}  // extern "C"
