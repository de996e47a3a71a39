// Throughput of random 4-byte gathers from global memory (working sets from
// 64 KB to 256 MB: L1-, L2- and DRAM-resident), from local shared memory, and
// from distributed shared memory across thread-block clusters of 2..16 CTAs.
// These are the per-SM service rates that bound the PageRank gather (see the
// roofline notes of the sweep kernels).  Built as gardenia_ocl_b200/lib/
// gpr_probe_gather by `make -C gardenia_ocl_b200/csrc probe`; prints one line
// per case.
#include <cooperative_groups.h>
#include <cstdio>
#include <cstdint>
namespace cg = cooperative_groups;

__device__ __forceinline__ unsigned xs(unsigned x) { x ^= x << 13; x ^= x >> 17; x ^= x << 5; return x; }

__global__ void k_gmem(const float* __restrict__ a, unsigned mask, int iters, float* out) {
  unsigned x = 0x9e3779b9u * (blockIdx.x * blockDim.x + threadIdx.x + 1);
  float acc = 0.f;
  for (int i = 0; i < iters; ++i) {
    unsigned id[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { x = xs(x); id[q] = x & mask; }
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = a[id[q]];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += v[q];
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void k_smem(int n_log2, int iters, float* out) {
  extern __shared__ float s[];
  const int n = 1 << n_log2;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = (float)i;
  __syncthreads();
  unsigned x = 0x9e3779b9u * (blockIdx.x * blockDim.x + threadIdx.x + 1);
  float acc = 0.f;
  for (int i = 0; i < iters; ++i) {
    unsigned id[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { x = xs(x); id[q] = x & (n - 1); }
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = s[id[q]];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += v[q];
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <int CS>
__global__ void k_dsmem(int n_log2, int iters, float* out) {
  extern __shared__ float s[];
  cg::cluster_group cl = cg::this_cluster();
  const int n = 1 << n_log2;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s[i] = (float)i;
  cl.sync();
  unsigned x = 0x9e3779b9u * (blockIdx.x * blockDim.x + threadIdx.x + 1);
  float acc = 0.f;
  float* base[CS];
#pragma unroll
  for (int r = 0; r < CS; ++r) base[r] = cl.map_shared_rank(s, r);
  for (int i = 0; i < iters; ++i) {
    unsigned id[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) { x = xs(x); id[q] = x & (n * CS - 1); }
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const unsigned r = id[q] >> n_log2;
      const float* p = cl.map_shared_rank(s, (int)r);
      v[q] = p[id[q] & (n - 1)];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += v[q];
  }
  cl.sync();
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

int main() {
  int sms; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  float *a, *out;
  size_t maxn = 1ull << 26;  // 256 MB
  cudaMalloc(&a, maxn * 4); cudaMemset(a, 0, maxn * 4);
  cudaMalloc(&out, 148 * 2048 * 4 * 4);
  cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
  const int iters = 256;
  auto report = [&](const char* what, long long gathers, float ms) {
    printf("%-40s %8.3f ms  %8.1f Ggather/s  %6.2f gathers/clk/SM(@1.9GHz)\n", what, ms,
           gathers / ms / 1e6, gathers / (ms * 1e-3) / sms / 1.9e9);
  };
  for (int lg = 14; lg <= 26; lg += 2) {
    for (int t : {1024}) {
      int blocks = sms * (2048 / t);
      k_gmem<<<blocks, t>>>(a, (1u << lg) - 1, iters, out);
      cudaEventRecord(e0);
      k_gmem<<<blocks, t>>>(a, (1u << lg) - 1, iters, out);
      cudaEventRecord(e1); cudaEventSynchronize(e1);
      float ms; cudaEventElapsedTime(&ms, e0, e1);
      char b[64]; snprintf(b, 64, "global %6d KB", (4 << lg) >> 10);
      report(b, (long long)blocks * t * iters * 8, ms);
    }
  }
  cudaFuncSetAttribute(k_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  for (int lg : {12, 14, 15}) {
    size_t sm = (size_t)4 << lg;
    int blocks = sms;
    k_smem<<<blocks, 1024, sm>>>(lg, iters, out);
    cudaEventRecord(e0);
    k_smem<<<blocks, 1024, sm>>>(lg, iters, out);
    cudaEventRecord(e1); cudaEventSynchronize(e1);
    float ms; cudaEventElapsedTime(&ms, e0, e1);
    char b[64]; snprintf(b, 64, "smem %6zu KB (1 CTA x1024/SM)", sm >> 10);
    report(b, (long long)blocks * 1024 * iters * 8, ms);
  }
  auto run_ds = [&](auto kern, int cs, int lg) {
    size_t sm = (size_t)4 << lg;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (cs > 8) cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
    cfg.attrs = at; cfg.numAttrs = 1;
    cfg.blockDim = dim3(1024); cfg.dynamicSmemBytes = sm;
    int ncl = 0;
    cfg.gridDim = dim3(cs);
    cudaOccupancyMaxActiveClusters(&ncl, (void*)kern, &cfg);
    if (ncl <= 0) { printf("cluster %d: not launchable (%s)\n", cs, cudaGetErrorString(cudaGetLastError())); return; }
    cfg.gridDim = dim3(ncl * cs);
    cudaLaunchKernelEx(&cfg, kern, lg, iters, out);
    cudaEventRecord(e0);
    cudaLaunchKernelEx(&cfg, kern, lg, iters, out);
    cudaEventRecord(e1); cudaEventSynchronize(e1);
    cudaError_t e = cudaGetLastError();
    float ms; cudaEventElapsedTime(&ms, e0, e1);
    char b[96]; snprintf(b, 96, "dsmem cl=%2d x %4zu KB (%d clusters) %s", cs, sm >> 10, ncl, e ? cudaGetErrorString(e) : "");
    report(b, (long long)ncl * cs * 1024 * iters * 8, ms * (float)sms / (ncl * cs));
  };
  run_ds(k_dsmem<2>, 2, 15);
  run_ds(k_dsmem<4>, 4, 15);
  run_ds(k_dsmem<8>, 8, 15);
  run_ds(k_dsmem<16>, 16, 15);
  run_ds(k_dsmem<8>, 8, 12);
  printf("done: %s\n", cudaGetErrorString(cudaDeviceSynchronize()));
  return 0;
}
