// Status strings, last-error messages and the device error word.
#include <map>
#include <mutex>
#include <utility>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "runtime.h"

namespace admp {

static __device__ DevError g_dev_error;

static thread_local char g_msg[512] = "";
static bool g_sync = true;
static DevError* g_err_ptr[64] = {nullptr};

bool sync_checks() { return g_sync; }

// (kernel, device) -> largest dynamic shared memory limit already set
static std::mutex g_smem_mu;
static std::map<std::pair<const void*, int>, size_t> g_smem_set;

bool smem_already(const void* fn, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_smem_mu);
  size_t& v = g_smem_set[std::make_pair(fn, dev)];
  if (v >= bytes) return true;
  v = bytes;
  return false;
}

static long long g_launches = 0;
void count_launches(int n) { g_launches += n; }

struct ProfRec {
  cudaEvent_t a, b;
  int kernel;
  double bytes;
};
static bool g_prof = false;
static ProfRec* g_prof_recs = nullptr;
static int g_prof_cap = 0, g_prof_n = 0;

bool prof_on() { return g_prof; }

int prof_begin(cudaStream_t st) {
  if (!g_prof || g_prof_n >= g_prof_cap) return -1;
  ProfRec& r = g_prof_recs[g_prof_n];
  if (cudaEventRecord(r.a, st) != cudaSuccess) return -1;
  return g_prof_n++;
}

void prof_end(int slot, int kernel, double bytes, cudaStream_t st) {
  if (slot < 0) return;
  ProfRec& r = g_prof_recs[slot];
  r.kernel = kernel;
  r.bytes = bytes;
  cudaEventRecord(r.b, st);
}

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

extern "C" long long admp_launch_count(void) { return g_launches; }

extern "C" int admp_profile_enable(int capacity) {
  if (g_prof_recs) {
    for (int k = 0; k < g_prof_cap; ++k) {
      cudaEventDestroy(g_prof_recs[k].a);
      cudaEventDestroy(g_prof_recs[k].b);
    }
    free(g_prof_recs);
    g_prof_recs = nullptr;
  }
  g_prof = capacity > 0;
  g_prof_cap = 0;
  g_prof_n = 0;
  if (!g_prof) return ADMP_OK;
  g_prof_recs = (ProfRec*)calloc((size_t)capacity, sizeof(ProfRec));
  if (!g_prof_recs) return fail(ADMP_ERR_BAD_ARG, "profile: out of host memory");
  for (int k = 0; k < capacity; ++k) {
    if (cudaEventCreate(&g_prof_recs[k].a) != cudaSuccess || cudaEventCreate(&g_prof_recs[k].b) != cudaSuccess)
      return fail(ADMP_ERR_CUDA, "profile: cudaEventCreate failed");
    g_prof_cap = k + 1;
  }
  return ADMP_OK;
}

// Per-kernel totals since the last enable: ms[k], launches[k], bytes[k]
// (arrays of PK_COUNT).  Synchronises on the recorded events.
extern "C" int admp_profile_read(double* ms, long long* launches, double* bytes, int n) {
  for (int k = 0; k < n; ++k) {
    ms[k] = 0.0;
    launches[k] = 0;
    bytes[k] = 0.0;
  }
  for (int i = 0; i < g_prof_n; ++i) {
    ProfRec& r = g_prof_recs[i];
    if (cudaEventSynchronize(r.b) != cudaSuccess) return fail(ADMP_ERR_CUDA, "profile: event sync failed");
    float t = 0.f;
    if (cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess) continue;
    if (r.kernel >= 0 && r.kernel < n) {
      ms[r.kernel] += t;
      launches[r.kernel] += 1;
      bytes[r.kernel] += r.bytes;
    }
  }
  return ADMP_OK;
}

extern "C" int admp_check_errors(void* stream) {
  bool saved = g_sync;
  g_sync = true;
  DevError* e = scratch_error((cudaStream_t)stream);
  int r = e ? check_error(e, (cudaStream_t)stream) : ADMP_ERR_CUDA;
  g_sync = saved;
  return r;
}
