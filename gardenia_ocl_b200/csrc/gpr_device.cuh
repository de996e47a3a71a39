// Device-side helpers shared by the sweep kernels: cache-policy loads and
// stores, contribution element access (FP32 / BF16), gather sources, warp
// reductions and the timer used by bounded waits.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include <type_traits>

namespace gpr {
namespace dev {

constexpr unsigned kFull = 0xffffffffu;

struct Policies {
  uint64_t stream;  // evict-first: data read or written once per sweep
  uint64_t keep;    // evict-last: contributions, gathered many times
};

__device__ __forceinline__ Policies make_policies() {
  Policies p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p.stream));
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p.keep));
  return p;
}

// Edge indices are read exactly once per sweep: no L1 allocation, evict-first
// in L2 so they do not push the contributions out.
__device__ __forceinline__ int ld_idx(const int *p, uint64_t pol) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
      : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ int4 ld_idx4(const int *p, uint64_t pol) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p), "l"(pol));
  return v;
}

// Contribution gather.  A plain (coherent, L1-cached) load: the persistent
// kernel rewrites these buffers between sweeps, so the non-coherent path
// must not be used; the grid barrier's fences order the accesses.
__device__ __forceinline__ float ld_contrib(const float *p, uint64_t pol) {
  float v;
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ float4 ld_contrib4(const float4 *p, uint64_t pol) {
  float4 v;
  asm volatile("ld.global.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p), "l"(pol));
  return v;
}

// Contribution elements are FP32 (plain form) or BF16 (mixed form); the sum
// is always FP32.
__device__ __forceinline__ float ld_c(const float *p, uint64_t pol) { return ld_contrib(p, pol); }
__device__ __forceinline__ float ld_c(const __nv_bfloat16 *p, uint64_t pol) {
  unsigned short h;
  asm volatile("ld.global.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(h) : "l"(p), "l"(pol));
  return __uint_as_float((unsigned)h << 16);
}
__device__ __forceinline__ float ld_c_generic(const float *p) {
  float v;
  asm volatile("ld.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_c_generic(const __nv_bfloat16 *p) {
  unsigned short h;
  asm volatile("ld.b16 %0, [%1];" : "=h"(h) : "l"(p));
  return __uint_as_float((unsigned)h << 16);
}
__device__ __forceinline__ float from_c(float v) { return v; }
__device__ __forceinline__ float from_c(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ void st_c(float *p, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" :: "l"(p), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_c(__nv_bfloat16 *p, float v, uint64_t pol) {
  const unsigned short h = __bfloat16_as_ushort(__float2bfloat16_rn(v));
  asm volatile("st.global.L2::cache_hint.b16 [%0], %1, %2;" :: "l"(p), "h"(h), "l"(pol) : "memory");
}

// Contribution sources.  GlobalGather reads the contribution array;
// HotGather serves indices below `hot` from the copy of the array's prefix
// in shared memory (the highest in-degree vertices, which a power-law graph
// gathers most) and the rest with a predicated global load, branch-free.
template <typename T>
struct GlobalGather {
  const T *cin;
  uint64_t pol;
  __device__ __forceinline__ float operator()(int idx) const { return ld_c(cin + idx, pol); }
};

template <typename T>
struct HotGather {
  const T *cin;
  const T *hot;
  int n_hot;
  uint64_t pol;
  __device__ __forceinline__ float operator()(int idx) const {
    const float h = from_c(hot[min(idx, n_hot - 1)]);
    const float g = idx >= n_hot ? ld_c(cin + idx, pol) : 0.f;
    return idx < n_hot ? h : g;
  }
};

template <>
struct HotGather<float> {
  const float *cin;
  const float *hot;
  int n_hot;
  uint64_t pol;
  __device__ __forceinline__ float operator()(int idx) const {
    const float h = hot[min(idx, n_hot - 1)];
    float g = 0.f;
    asm volatile(
        "{\n .reg .pred p;\n setp.ge.s32 p, %1, %2;\n"
        " @p ld.global.L2::cache_hint.f32 %0, [%3], %4;\n}"
        : "+f"(g) : "r"(idx), "r"(n_hot), "l"(cin + idx), "l"(pol));
    return idx < n_hot ? h : g;
  }
};

// Same sources through one generic-address load: a lane's pointer falls in
// shared memory for hot indices and in global memory otherwise, so a gather
// costs one load instruction instead of two.
template <typename T>
struct HotGatherGeneric {
  const T *cin;
  const T *hot;
  int n_hot;
  uint64_t pol;
  __device__ __forceinline__ float operator()(int idx) const {
    return ld_c_generic(idx < n_hot ? hot + idx : cin + idx);
  }
};

__device__ __forceinline__ float ld_f32_stream(const float *p, uint64_t pol) {
  float v;
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ int ld_s32_stream(const int *p, uint64_t pol) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
      : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

__device__ __forceinline__ void st_f32(float *p, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" :: "l"(p), "f"(v), "l"(pol) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ long long global_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ double block_sum_double(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

// Bounded grid barrier of a cooperative launch.  bar[0] counts arrivals,
// bar[1] is the generation.  When cta_part is given, every CTA first stores
// its value in cta_part[blockIdx.x] and the last CTA to arrive sums them in
// CTA order (deterministic) into *sum_out before it opens the next
// generation.  Waits are bounded by timeout_ns of %globaltimer; on expiry
// status[0] bit 0 is raised and false is returned.  Call from every thread.
// Grid barrier without a reduction: `count` (zeroed before the launch) only
// grows; episode e of a launch (1, 2, ...) is complete when it reaches
// expect * e, so no CTA has to publish anything after the last arrival and a
// waiter sees the release on its next poll.  The comparison is wrap-safe.
// The wait is bounded by timeout_ns: on expiry status[0] bit 0 is raised and
// false is returned.
__device__ __forceinline__ bool grid_barrier_count(unsigned *count, unsigned target, int *status,
                                                   long long timeout_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1u);
    s_ok = 1;
    const long long t0 = global_ns();
    unsigned spins = 0;
    while ((int)(ld_acquire(count) - target) < 0) {
      if ((++spins & 63u) == 0 && global_ns() - t0 > timeout_ns) {
        atomicOr(status, 1);
        s_ok = 0;
        break;
      }
      __nanosleep(50);
    }
    __threadfence();
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned expect, double *cta_part,
                                             double cta_value, double *sum_out, int *status,
                                             long long timeout_ns) {
  __shared__ int s_state;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (cta_part) cta_part[blockIdx.x] = cta_value;
    const unsigned gen = ld_acquire(bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    s_state = 0;
    if (arrived == expect - 1u) {
      __threadfence();
      if (cta_part) {
        double t = 0.0;
        for (unsigned i = 0; i < gridDim.x; ++i) t += __ldcg(cta_part + i);
        *sum_out = t;
      }
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long t0 = global_ns();
      unsigned spins = 0;
      while (ld_acquire(bar + 1) == gen) {
        if ((++spins & 31u) == 0 && global_ns() - t0 > timeout_ns) {
          atomicOr(status, 1);
          s_state = 2;
          break;
        }
        __nanosleep(100);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return s_state != 2;
}

}  // namespace dev
}  // namespace gpr
