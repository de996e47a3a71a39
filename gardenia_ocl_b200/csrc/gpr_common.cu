// Error slot, allocation helpers and small C-ABI entry points.
#include <cub/cub.cuh>
#include <stdarg.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "gpr_internal.cuh"

namespace gpr {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

// Block cache of large device allocations.  One-shot solver calls (the
// reference's PRSolver shape: copy in, build, solve, free) allocate and free
// gigabytes per call; mapping and unmapping that much memory makes cudaMalloc
// / cudaFree slow and erratic.  Blocks of at least kCacheMin bytes are kept
// after dfree (which first synchronises the device, as cudaFree does, so no
// kernel still uses the block) and handed out again to requests that fit
// them within 1/8.  At most kCacheCap bytes stay cached; an allocation that
// fails releases the cache and retries; gpr_release_cached() empties it.
namespace {

constexpr size_t kCacheMin = size_t(1) << 20;
constexpr size_t kCacheCap = size_t(24) << 30;

struct Block {
  void *p;
  size_t bytes;
  int device;
};

std::mutex g_mu;
std::unordered_map<void *, Block> g_live;  // cached-class blocks handed out
std::vector<Block> g_free;                // cached, unused
size_t g_free_bytes = 0;

void release_free_locked(int device) {
  for (size_t i = 0; i < g_free.size();) {
    if (device < 0 || g_free[i].device == device) {
      int cur = -1;
      cudaGetDevice(&cur);
      if (cur != g_free[i].device) cudaSetDevice(g_free[i].device);
      cudaFree(g_free[i].p);
      if (cur >= 0 && cur != g_free[i].device) cudaSetDevice(cur);
      g_free_bytes -= g_free[i].bytes;
      g_free[i] = g_free.back();
      g_free.pop_back();
    } else {
      ++i;
    }
  }
}

}  // namespace

int dmalloc(void **p, size_t bytes, const char *what) {
  *p = nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  if (bytes >= kCacheMin) {
    std::lock_guard<std::mutex> lk(g_mu);
    int best = -1;
    for (size_t i = 0; i < g_free.size(); ++i) {
      const Block &b = g_free[i];
      if (b.device == dev && b.bytes >= bytes && b.bytes - bytes <= bytes / 8 &&
          (best < 0 || b.bytes < g_free[best].bytes))
        best = (int)i;
    }
    if (best >= 0) {
      Block b = g_free[best];
      g_free[best] = g_free.back();
      g_free.pop_back();
      g_free_bytes -= b.bytes;
      g_live[b.p] = b;
      *p = b.p;
      return GPR_OK;
    }
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(g_mu);
      release_free_locked(dev);
    }
    e = cudaMalloc(p, bytes);
  }
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    *p = nullptr;
    set_error("cudaMalloc(%zu bytes) for %s: out of device memory", bytes, what);
    return GPR_ENOMEM;
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error("cudaMalloc(%zu bytes) for %s: %s", bytes, what, cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  if (bytes >= kCacheMin) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_live[*p] = Block{*p, bytes, dev};
  }
  return GPR_OK;
}

namespace {
thread_local std::vector<void *> *t_deferred = nullptr;
}  // namespace

DeferFrees::DeferFrees() : prev_(t_deferred) { t_deferred = &list_; }

DeferFrees::~DeferFrees() {
  t_deferred = prev_;
  for (void *p : list_) dfree(p);
}

void dfree(void *p) {
  if (!p) return;
  if (t_deferred) {
    t_deferred->push_back(p);
    return;
  }
  std::unique_lock<std::mutex> lk(g_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) {
    lk.unlock();
    cudaFree(p);
    return;
  }
  Block b = it->second;
  g_live.erase(it);
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != b.device) cudaSetDevice(b.device);
  cudaDeviceSynchronize();  // what cudaFree would wait for
  if (cur >= 0 && cur != b.device) cudaSetDevice(cur);
  g_free.push_back(b);
  g_free_bytes += b.bytes;
  while (g_free_bytes > kCacheCap && !g_free.empty()) {
    size_t big = 0;
    for (size_t i = 1; i < g_free.size(); ++i)
      if (g_free[i].bytes > g_free[big].bytes) big = i;
    Block v = g_free[big];
    g_free[big] = g_free.back();
    g_free.pop_back();
    g_free_bytes -= v.bytes;
    if (cur != v.device) cudaSetDevice(v.device);
    cudaFree(v.p);
    if (cur >= 0 && cur != v.device) cudaSetDevice(cur);
  }
}

size_t cached_bytes() {
  std::lock_guard<std::mutex> lk(g_mu);
  return g_free_bytes;
}

namespace {
__global__ void k_pk_flag(int n, const long long *__restrict__ excl, long long target, int *flag) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n) flag[u] = (u == 0 || excl[u] / target != excl[u - 1] / target) ? 1 : 0;
}

__global__ void k_pk_emit(int n, const int *__restrict__ flag, const int *__restrict__ pos,
                          int *pk) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < n && flag[u]) pk[pos[u]] = u;
  if (u == n - 1) pk[pos[u] + flag[u]] = n;
}
}  // namespace

int make_packets(long long *cost, int n_units, long long want, int **pk_out, int *npk_out,
                 cudaStream_t st) {
  *pk_out = nullptr;
  *npk_out = 0;
  if (n_units <= 0) {
    GPR_TRY(dalloc(pk_out, 1, "packets"));
    GPR_CUDA(cudaMemsetAsync(*pk_out, 0, sizeof(int), st));
    return GPR_OK;
  }
  long long *excl = nullptr;
  int *flag = nullptr, *pos = nullptr;
  void *tmp = nullptr;
  size_t tb1 = 0, tb2 = 0;
  int rc = GPR_OK;
  long long tail[2] = {0, 0};
  int ftail[2] = {0, 0};
  const unsigned nb = (unsigned)ceil_div(n_units, 256);
  cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, tb1, cost, excl, n_units, st);
  if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, flag, pos, n_units, st);
  if (e != cudaSuccess) goto cuda_fail;
  if ((rc = dalloc(&excl, n_units, "packet prefix")) != GPR_OK ||
      (rc = dalloc(&flag, n_units, "packet flags")) != GPR_OK ||
      (rc = dalloc(&pos, n_units, "packet positions")) != GPR_OK ||
      (rc = dmalloc(&tmp, std::max(tb1, tb2), "scan scratch")) != GPR_OK)
    goto done;
  e = cub::DeviceScan::ExclusiveSum(tmp, tb1, cost, excl, n_units, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&tail[0], excl + n_units - 1, sizeof(long long), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&tail[1], cost + n_units - 1, sizeof(long long), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) goto cuda_fail;
  {
    const long long target = std::max(1LL, ceil_div(tail[0] + tail[1], std::max(1LL, want)));
    k_pk_flag<<<nb, 256, 0, st>>>(n_units, excl, target, flag);
    e = cub::DeviceScan::ExclusiveSum(tmp, tb2, flag, pos, n_units, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&ftail[0], pos + n_units - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&ftail[1], flag + n_units - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) goto cuda_fail;
    const int npk = ftail[0] + ftail[1];
    if ((rc = dalloc(pk_out, (size_t)npk + 1, "packets")) != GPR_OK) goto done;
    k_pk_emit<<<nb, 256, 0, st>>>(n_units, flag, pos, *pk_out);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) goto cuda_fail;
    *npk_out = npk;
  }
  goto done;
cuda_fail:
  set_error("packet table: %s", cudaGetErrorString(e));
  rc = GPR_ECUDA;
done:
  if (rc != GPR_OK) {
    dfree(*pk_out);
    *pk_out = nullptr;
  }
  dfree(excl);
  dfree(flag);
  dfree(pos);
  dfree(tmp);
  return rc;
}

bool is_device_ptr(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

int to_device(const void *any, size_t bytes, void **dev, bool *owned,
              cudaStream_t st, const char *what) {
  if (any == nullptr || is_device_ptr(any)) {
    *dev = const_cast<void *>(any);
    *owned = false;
    return GPR_OK;
  }
  GPR_TRY(dmalloc(dev, bytes ? bytes : 1, what));
  *owned = true;
  if (bytes) {
    cudaError_t e = cudaMemcpyAsync(*dev, any, bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      set_error("copy of %s to the device: %s", what, cudaGetErrorString(e));
      dfree(*dev);
      *dev = nullptr;
      *owned = false;
      return GPR_ECUDA;
    }
  }
  return GPR_OK;
}

}  // namespace gpr

extern "C" {

const char *gpr_last_error(void) { return gpr::g_err; }

const char *gpr_version(void) { return "gpr 0.1 (sm_100a)"; }

int gpr_pr_opts_default(gpr_pr_opts *o) {
  if (!o) {
    gpr::set_error("gpr_pr_opts_default: NULL opts");
    return GPR_EINVAL;
  }
  memset(o, 0, sizeof(*o));
  o->damping = 0.85f;   // include/common.h:18
  o->tol = 0.001;       // src/pr/pr.h:4
  o->max_iter = 30;     // src/pr/pr.h:5
  o->precision = GPR_PREC_FP32;
  o->loop = GPR_LOOP_AUTO;
  o->timeout_s = 5.0;
  o->refine_max = 64;
  o->ppr_repack = 1;
  return GPR_OK;
}

int gpr_free(void *d_ptr) {
  gpr::dfree(d_ptr);
  GPR_CUDA(cudaGetLastError());
  return GPR_OK;
}

int gpr_release_cached(long long *released_bytes) {
  {
    std::lock_guard<std::mutex> lk(gpr::g_mu);
    if (released_bytes) *released_bytes = (long long)gpr::g_free_bytes;
    gpr::release_free_locked(-1);
  }
  GPR_CUDA(cudaGetLastError());
  return GPR_OK;
}

int gpr_cached_bytes(long long *bytes) {
  if (!bytes) {
    gpr::set_error("gpr_cached_bytes: NULL out");
    return GPR_EINVAL;
  }
  *bytes = (long long)gpr::cached_bytes();
  return GPR_OK;
}

int gpr_malloc(void **d_ptr, size_t bytes) {
  if (!d_ptr) {
    gpr::set_error("gpr_malloc: NULL out");
    return GPR_EINVAL;
  }
  return gpr::dmalloc(d_ptr, bytes ? bytes : 1, "gpr_malloc");
}

int gpr_memcpy(void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return GPR_OK;
  if (!dst || !src) {
    gpr::set_error("gpr_memcpy: NULL pointer");
    return GPR_EINVAL;
  }
  GPR_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
  return GPR_OK;
}

int gpr_set_device(int device) {
  GPR_CUDA(cudaSetDevice(device));
  return GPR_OK;
}

int gpr_synchronize(void) {
  GPR_CUDA(cudaDeviceSynchronize());
  return GPR_OK;
}

}  // extern "C"
