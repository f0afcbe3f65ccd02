// Host-side runtime helpers shared by the entry points.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "admp_common.cuh"

namespace admp {

// Device error word of the current device (a file-scope __device__ variable,
// so no allocation).  Kernels record the first bad condition there.
DevError* scratch_error(cudaStream_t st);
// When synchronous checks are on (default), synchronise `st`, read and clear
// the error word and turn it into a status.  Otherwise return ADMP_OK and
// leave the error sticky for admp_check_errors().
int check_error(DevError* err, cudaStream_t st);
// Record a message and return `code`.
int fail(int code, const char* fmt, ...);
bool sync_checks();

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Kernel launch counter (all launches made by this library) and an optional
// CUDA-event profiler for the hot kernels.  Profiling is off by default; when
// on, each instrumented launch is bracketed by events on its own stream and
// tagged with the algorithmic bytes it moves.
enum ProfKernel {
  PK_SPREAD = 0, PK_FFT_Z_FWD, PK_FFT_Y_FWD, PK_FFT_X_GREEN, PK_FFT_Y_INV, PK_FFT_Z_INV, PK_GATHER,
  PK_PAIR_EF, PK_CSR_SPMV, PK_NEIGHBORS, PK_CG_VECTOR,
  // the CG matvec's mesh passes on the tensor cores
  PK_TC_Z_FWD, PK_TC_Y_FWD, PK_TC_X, PK_TC_Y_INV, PK_TC_Z_INV, PK_COUNT
};
void count_launches(int n);
bool prof_on();
int prof_begin(cudaStream_t st);                       // returns a slot (or -1)
void prof_end(int slot, int kernel, double bytes, cudaStream_t st);

// Carves typed sub-buffers out of a caller workspace.
struct Carver {
  char* base;
  size_t cap;
  size_t off;
  Carver(void* b, size_t c) : base((char*)b), cap(c), off(0) {}
  template <typename X>
  X* take(size_t n) {
    off = align_up(off, 256);
    X* p = base ? (X*)(base + off) : nullptr;
    off += n * sizeof(X);
    return p;
  }
  bool ok() const { return off <= cap; }
};

// Raises a kernel's dynamic shared-memory limit to `bytes` (static shared
// memory counts against the default 48 KB too, so the limit is always set);
// remembers the largest value set per kernel and device.
bool smem_already(const void* fn, size_t bytes);
template <typename K>
inline cudaError_t ensure_smem(K kernel, size_t bytes) {
  if (bytes == 0 || smem_already((const void*)kernel, bytes)) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace admp
