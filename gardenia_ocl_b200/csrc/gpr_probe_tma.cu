// Throughput of random row fetches with the tensor memory accelerator's
// 4-row gather (cp.async.bulk.tensor.2d ... tile::gather4) against plain
// random 4-byte loads, over a float array viewed as rows of 4 (16 bytes).
// A measurement tool, not part of libgpr: built as gardenia_ocl_b200/lib/
// gpr_probe_tma by `make -C gardenia_ocl_b200/csrc probe`; prints one line
// per case.
//
// Every thread owns an mbarrier and B destination slots of 128 bytes in
// shared memory; per round it arms the mbarrier for B * 64 bytes, issues B
// gather4 copies of 4 random rows each, and waits (bounded) for completion.
// Rows are always inside the tensor and the x coordinate is 0.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

__device__ __forceinline__ unsigned xs(unsigned x) {
  x ^= x << 13;
  x ^= x >> 17;
  x ^= x << 5;
  return x;
}

__device__ __forceinline__ unsigned saddr(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ long long now_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for phase `phase` of the mbarrier, at most limit_ns; false on expiry.
__device__ __forceinline__ bool wait_bounded(uint64_t *mbar, unsigned phase, long long limit_ns) {
  const long long t0 = now_ns();
  for (unsigned spin = 0;; ++spin) {
    unsigned done = 0;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
        "selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(saddr(mbar)), "r"(phase)
        : "memory");
    if (done) return true;
    if ((spin & 63u) == 63u && now_ns() - t0 > limit_ns) return false;
  }
}

template <int B>
__global__ void k_tma(const __grid_constant__ CUtensorMap tmap, unsigned rmask, int iters,
                      float *out, int *err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  if (saddr(smem) & 127u) {  // destinations must be 128-byte aligned: do not issue
    if (threadIdx.x == 0) atomicOr(err, 2);
    return;
  }
  float *slot = reinterpret_cast<float *>(smem) + (size_t)threadIdx.x * B * 32;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + (size_t)blockDim.x * B * 128) + threadIdx.x;
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(mbar)));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  unsigned x = 0x9e3779b9u * (blockIdx.x * blockDim.x + threadIdx.x + 1);
  unsigned phase = 0;
  float acc = 0.f;
  bool ok = true;
  for (int i = 0; i < iters && ok; ++i) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(mbar)),
                 "r"(B * 64)
                 : "memory");
#pragma unroll
    for (int b = 0; b < B; ++b) {
      int r[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        x = xs(x);
        r[q] = (int)(x & rmask);
      }
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::"
          "bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(saddr(slot + b * 32)),
          "l"(&tmap), "r"(0), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(saddr(mbar))
          : "memory");
    }
    if (!wait_bounded(mbar, phase, 2000000000LL)) {
      atomicOr(err, 1);
      wait_bounded(mbar, phase, 1000000000LL);  // let copies in flight land
      ok = false;
      break;
    }
    phase ^= 1u;
#pragma unroll
    for (int b = 0; b < B; ++b) acc += slot[b * 32] + slot[b * 32 + 4] + slot[b * 32 + 8] + slot[b * 32 + 12];
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void k_lsu(const float *__restrict__ a, unsigned mask, int iters, float *out) {
  unsigned x = 0x9e3779b9u * (blockIdx.x * blockDim.x + threadIdx.x + 1);
  float acc = 0.f;
  for (int i = 0; i < iters; ++i) {
    unsigned id[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      x = xs(x);
      id[q] = (x & mask) * 4;
    }
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = a[id[q]];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc += v[q];
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

int main() {
  int sms = 0, clk_khz = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, 0);
  const double ghz = clk_khz / 1e6;
  const size_t max_rows = size_t(1) << 24;  // 16M rows x 16 B = 256 MB
  float *a = nullptr, *out = nullptr;
  int *err = nullptr;
  if (cudaMalloc(&a, max_rows * 16) != cudaSuccess || cudaMalloc(&out, 148 * 2048 * 4 * 4) ||
      cudaMalloc(&err, 4)) {
    printf("alloc failed\n");
    return 1;
  }
  cudaMemset(a, 0, max_rows * 16);
  cudaMemset(err, 0, 4);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto report = [&](const char *what, double rows, float ms) {
    printf("%-44s %8.3f ms  %8.1f G rows/s  %6.2f rows/clk/SM\n", what, ms, rows / ms / 1e6,
           rows / (ms * 1e-3) / sms / (ghz * 1e9));
  };
  constexpr int B = 4, T = 256, ITERS = 256;
  const size_t smem = (size_t)T * B * 128 + T * 8;
  cudaFuncSetAttribute(k_tma<B>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tma<B>, T, smem);
  for (int lg = 16; lg <= 24; lg += 2) {
    const size_t rows = size_t(1) << lg;
    CUtensorMap tm;
    cuuint64_t dims[2] = {4, rows};
    cuuint64_t strides[1] = {16};
    cuuint32_t box[2] = {4, 1};
    cuuint32_t estr[2] = {1, 1};
    CUresult rc = cuTensorMapEncodeTiled(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, a, dims, strides,
                                         box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                         CU_TENSOR_MAP_SWIZZLE_NONE,
                                         CU_TENSOR_MAP_L2_PROMOTION_NONE,
                                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (rc != CUDA_SUCCESS) {
      printf("cuTensorMapEncodeTiled failed: %d\n", (int)rc);
      return 1;
    }
    const int blocks = sms * per_sm;
    k_tma<B><<<blocks, T, smem>>>(tm, (unsigned)(rows - 1), ITERS, out, err);
    cudaEventRecord(e0);
    k_tma<B><<<blocks, T, smem>>>(tm, (unsigned)(rows - 1), ITERS, out, err);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    int herr = 0;
    cudaMemcpy(&herr, err, 4, cudaMemcpyDeviceToHost);
    char b[96];
    snprintf(b, sizeof(b), "tma gather4 %6zu KB (%d CTA x %d/SM)%s", (rows * 16) >> 10, per_sm, T,
             herr & 2 ? " UNALIGNED (skipped)" : herr ? " WAIT LIMIT" : "");
    report(b, (double)blocks * T * ITERS * B * 4, ms);
    const int lb = sms * 2;
    k_lsu<<<lb, 1024>>>(a, (unsigned)(rows - 1), ITERS, out);
    cudaEventRecord(e0);
    k_lsu<<<lb, 1024>>>(a, (unsigned)(rows - 1), ITERS, out);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    snprintf(b, sizeof(b), "lsu 4-byte loads %6zu KB", (rows * 16) >> 10);
    report(b, (double)lb * 1024 * ITERS * 8, ms);
  }
  printf("done: %s\n", cudaGetErrorString(cudaDeviceSynchronize()));
  return 0;
}
