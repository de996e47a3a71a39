// Error slot, allocation helpers and small C-ABI entry points.
#include <stdarg.h>
#include <string.h>

#include "gpr_internal.cuh"

namespace gpr {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int dmalloc(void **p, size_t bytes, const char *what) {
  *p = nullptr;
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    set_error("cudaMalloc(%zu bytes) for %s: out of device memory", bytes, what);
    return GPR_ENOMEM;
  }
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes) for %s: %s", bytes, what, cudaGetErrorString(e));
    return GPR_ECUDA;
  }
  return GPR_OK;
}

void dfree(void *p) {
  if (p) cudaFree(p);
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
      cudaFree(*dev);
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
  return GPR_OK;
}

int gpr_free(void *d_ptr) {
  if (d_ptr) GPR_CUDA(cudaFree(d_ptr));
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
