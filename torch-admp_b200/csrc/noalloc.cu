// admp_pme_recip_noalloc: the reciprocal-space PME entry point for callers
// that cannot allocate device memory when they call us.
//
// admp_pme_recip needs a scratch workspace (charge mesh, half spectrum and
// per-frame accumulators) that its caller allocates.  Some callers cannot do
// that at call time: a plugin running inside a molecular-dynamics engine that
// owns all device memory through its own pool and gives plugins none, or a
// time-step loop that must not call cudaMalloc because cudaMalloc can
// synchronise the whole device and stall the engine's other streams.  This
// variant takes the same inputs and outputs but keeps its scratch in one
// fixed-size array in the library's own device memory, so it allocates
// nothing.
//
// The array is a file-scope __device__ variable: every GPU that loads the
// library holds kNoAllocScratchBytes (16 MiB) of it until the process exits.
// Under CUDA's lazy module loading the module, and with it the array, is
// created on a device by the first call there (its cudaGetSymbolAddress), so
// that first call does allocate: callers make it before their no-allocation
// region.  The address cached per device is not valid after cudaDeviceReset.
// Requests whose scratch does not fit are rejected with ADMP_ERR_WORKSPACE.
// All calls share the array and it keeps the previous call's contents; the
// code clears what must start at zero (mesh and accumulators) on every call.
// Calls that overlap on the GPU (two streams, or two host threads) race on
// the array and must not be issued concurrently.
#include <mutex>

#include "runtime.h"

namespace admp {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static void* g_noalloc_addr[64] = {nullptr};
static std::mutex g_noalloc_mu;

// Device address of the scratch array on the current device.  In host code
// `g_noalloc_scratch` only names a host-side stand-in, so the address has to
// come from cudaGetSymbolAddress, once per device, with that device current.
static int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
    return ADMP_ERR_CUDA;
  }
  if (dev < 0 || dev >= 64) return fail(ADMP_ERR_BAD_ARG, "admp_pme_recip_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_last_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      return ADMP_ERR_CUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return ADMP_OK;
}

}  // namespace admp

using namespace admp;

extern "C" size_t admp_pme_recip_noalloc_max_scratch(void) { return kNoAllocScratchBytes; }

extern "C" int admp_pme_recip_noalloc(int dtype, int nframes, int natoms, const int* kmesh, const void* pos,
                                      const void* box, const void* q, double kappa, double ke, double* energy,
                                      void* dE_dpos, void* dE_dq, void* dE_dbox, void* stream) {
  if (nframes == 0) return ADMP_OK;
  if (nframes < 0 || natoms < 0 || !kmesh) return fail(ADMP_ERR_BAD_ARG, "admp_pme_recip_noalloc: args");
  if (dtype != ADMP_F64 && dtype != ADMP_F32) return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  const size_t need = admp_pme_recip_workspace_size(dtype, nframes, kmesh);
  if (need == 0) return fail(ADMP_ERR_MESH, "admp_pme_recip_noalloc: unsupported mesh sizes");
  if (need > kNoAllocScratchBytes)
    return fail(ADMP_ERR_WORKSPACE,
                "admp_pme_recip_noalloc: these %d frame(s) need %zu bytes of scratch, more than its fixed "
                "%zu-byte buffer; use admp_pme_recip with a caller workspace or fewer/smaller meshes",
                nframes, need, kNoAllocScratchBytes);
  void* scratch = nullptr;
  int s = noalloc_scratch(&scratch);
  if (s) return s;
  return admp_pme_recip(dtype, nframes, natoms, kmesh, pos, box, q, kappa, ke, energy, dE_dpos, dE_dq, dE_dbox,
                        scratch, kNoAllocScratchBytes, stream);
}
