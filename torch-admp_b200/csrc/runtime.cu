// Status strings, last-error messages and the device error word.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include "runtime.h"

namespace admp {

static __device__ DevError g_dev_error;

static thread_local char g_msg[512] = "";
static bool g_sync = true;
static DevError* g_err_ptr[64] = {nullptr};

bool sync_checks() { return g_sync; }

void set_last_message(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
}

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return code;
}

void set_last_cuda_error(cudaError_t e, const char* expr, const char* file, int line) {
  set_last_message("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), expr, file, line);
}

DevError* scratch_error(cudaStream_t) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!g_err_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dev_error);
    if (e != cudaSuccess) {
      set_last_cuda_error(e, "cudaGetSymbolAddress(g_dev_error)", __FILE__, __LINE__);
      return nullptr;
    }
    g_err_ptr[dev] = (DevError*)p;
  }
  return g_err_ptr[dev];
}

static const char* where_name(int w) {
  switch (w) {
    case 1: return "pair energy";
    case 2: return "pair distances";
    case 3: return "pair distances backward";
    case 4: return "neighbour list";
    case 5: return "QEq pair coefficients";
    case 6: return "PME positions";
    default: return "kernel";
  }
}

int check_error(DevError* err, cudaStream_t st) {
  if (!g_sync) return ADMP_OK;
  DevError h;
  cudaError_t e = cudaMemcpyAsync(&h, err, sizeof(DevError), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "error-word readback", __FILE__, __LINE__);
    return ADMP_ERR_CUDA;
  }
  if (h.code != 0) {
    cudaMemsetAsync(err, 0, sizeof(DevError), st);
    cudaStreamSynchronize(st);
    if (h.code == ADMP_ERR_BAD_INDEX)
      set_last_message("%s: index out of range at element %lld", where_name(h.where), h.detail);
    else if (h.code == ADMP_ERR_NONFINITE)
      set_last_message("%s: non-finite value at element %lld", where_name(h.where), h.detail);
    else
      set_last_message("%s: device error %d (detail %lld)", where_name(h.where), h.code, h.detail);
    return h.code;
  }
  return ADMP_OK;
}

}  // namespace admp

using namespace admp;

extern "C" int admp_abi_version(void) { return ADMP_ABI_VERSION; }

extern "C" const char* admp_status_string(int s) {
  switch (s) {
    case ADMP_OK: return "ok";
    case ADMP_ERR_BAD_ARG: return "bad argument";
    case ADMP_ERR_CUTOFF_TOO_LARGE: return "cutoff larger than half the minimum box height";
    case ADMP_ERR_NOT_CONVERGED: return "not converged";
    case ADMP_ERR_WORKSPACE: return "workspace too small";
    case ADMP_ERR_CUDA: return "CUDA error";
    case ADMP_ERR_BAD_INDEX: return "index out of range";
    case ADMP_ERR_CAPACITY: return "output capacity too small";
    case ADMP_ERR_NONFINITE: return "non-finite input";
    case ADMP_ERR_MESH: return "unsupported mesh size";
    default: return "unknown status";
  }
}

extern "C" const char* admp_last_error_message(void) { return g_msg; }

extern "C" void admp_set_sync_checks(int on) { g_sync = on != 0; }

extern "C" int admp_check_errors(void* stream) {
  bool saved = g_sync;
  g_sync = true;
  DevError* e = scratch_error((cudaStream_t)stream);
  int r = e ? check_error(e, (cudaStream_t)stream) : ADMP_ERR_CUDA;
  g_sync = saved;
  return r;
}
