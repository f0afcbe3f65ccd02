// admp_pme_recip: reciprocal-space PME energy and gradients for nframes
// systems (CoulombForceModule._forward_pbc_reciprocal, pme.py:351-446, and
// the autograd backward through spread_charges / setup_kpts, recip.py).
#include "pme_host.h"

namespace admp {

template <typename T>
static int recip_chunk_plan(int c0, int nsys, int N, const int* kmesh, double kappa, RecipPlan<T>& p) {
  SysSpec sys[kMaxBatch];
  for (int s = 0; s < nsys; ++s) {
    sys[s].natoms = N;
    sys[s].atom_off = s * N;
    for (int d = 0; d < 3; ++d) sys[s].K[d] = kmesh[3 * (c0 + s) + d];
    sys[s].kappa = kappa;
    sys[s].box_idx = s;
  }
  return build_recip_plan<T>(sys, nsys, p);
}

template <typename T>
static size_t recip_ws_bytes(const RecipPlan<T>& p) {
  Carver c(nullptr, 0);
  c.take<unsigned char>(sys_table_bytes());
  c.take<T>(p.mesh_elems);
  c.take<Cplx<T>>(p.spec_elems);
  c.take<double>((size_t)p.b.nsys * kAccStride);
  return c.off;
}

template <typename T>
static int recip_ws_size(int nf, const int* kmesh, size_t* out) {
  size_t best = 0;
  for (int c0 = 0; c0 < nf; c0 += kMaxBatch) {
    const int ns = nf - c0 < kMaxBatch ? nf - c0 : kMaxBatch;
    RecipPlan<T> p;
    int s = recip_chunk_plan<T>(c0, ns, 1, kmesh, 1.0, p);
    if (s) return s;
    size_t b = recip_ws_bytes(p);
    best = b > best ? b : best;
  }
  *out = best;
  return ADMP_OK;
}

template <typename T>
static int pme_recip_impl(int nf, int N, const int* kmesh, const T* pos, const T* box, const T* q, double kappa,
                          double ke, double* energy, T* dpos, T* dq, T* dbox, void* ws, size_t bytes,
                          cudaStream_t st) {
  for (int c0 = 0; c0 < nf; c0 += kMaxBatch) {
    const int ns = nf - c0 < kMaxBatch ? nf - c0 : kMaxBatch;
    RecipPlan<T> p;
    int s = recip_chunk_plan<T>(c0, ns, N, kmesh, kappa, p);
    if (s) return s;
    Carver c(ws, bytes);
    SysDesc* table = reinterpret_cast<SysDesc*>(c.take<unsigned char>(sys_table_bytes()));
    T* mesh = c.take<T>(p.mesh_elems);
    Cplx<T>* spec = c.take<Cplx<T>>(p.spec_elems);
    double* acc = c.take<double>((size_t)ns * kAccStride);
    if (!c.ok() || !ws) return fail(ADMP_ERR_WORKSPACE, "pme_recip workspace: need %zu bytes, got %zu", c.off, bytes);
    s = bind_plan<T>(p, table, st);
    if (s) return s;
    ADMP_CUDA_TRY(cudaMemsetAsync(acc, 0, sizeof(double) * ns * kAccStride, st));
    const size_t ao = (size_t)c0 * N;
    s = launch_recip<T>(p, pos + ao * 3, box + (size_t)c0 * 9, q + ao, mesh, spec, acc, ke, dq ? dq + ao : nullptr,
                        dpos ? dpos + ao * 3 : nullptr, st);
    if (s) return s;
    recip_finalize_kernel<T><<<(ns + 127) / 128, 128, 0, st>>>(p.b, box + (size_t)c0 * 9, acc,
                                                               energy ? energy + c0 : nullptr,
                                                               dbox ? dbox + (size_t)c0 * 9 : nullptr);
    ADMP_CUDA_TRY(cudaGetLastError());
  }
  return ADMP_OK;
}

}  // namespace admp

using namespace admp;

extern "C" size_t admp_pme_recip_workspace_size(int dtype, int nframes, const int* kmesh) {
  if (nframes <= 0 || !kmesh) return 0;
  size_t out = 0;
  int s = dtype == ADMP_F32 ? recip_ws_size<float>(nframes, kmesh, &out) : recip_ws_size<double>(nframes, kmesh, &out);
  return s ? 0 : out;
}

extern "C" int admp_pme_recip(int dtype, int nframes, int natoms, const int* kmesh, const void* pos, const void* box,
                              const void* q, double kappa, double ke, double* energy, void* dE_dpos, void* dE_dq,
                              void* dE_dbox, void* workspace, size_t workspace_bytes, void* stream) {
  if (nframes == 0) return ADMP_OK;
  if (nframes < 0 || natoms < 0 || !kmesh || !box || !(kappa > 0)) return fail(ADMP_ERR_BAD_ARG, "admp_pme_recip: args");
  if (natoms > 0 && (!pos || !q)) return fail(ADMP_ERR_BAD_ARG, "admp_pme_recip: null pos/q");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return pme_recip_impl<double>(nframes, natoms, kmesh, (const double*)pos, (const double*)box, (const double*)q,
                                  kappa, ke, energy, (double*)dE_dpos, (double*)dE_dq, (double*)dE_dbox, workspace,
                                  workspace_bytes, st);
  if (dtype == ADMP_F32)
    return pme_recip_impl<float>(nframes, natoms, kmesh, (const float*)pos, (const float*)box, (const float*)q, kappa,
                                 ke, energy, (float*)dE_dpos, (float*)dE_dq, (float*)dE_dbox, workspace,
                                 workspace_bytes, st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}
