// Host-side batch building and launch sequence for the reciprocal PME kernels.
#pragma once

#include <vector>

#include "dft_tc.cuh"
#include "pme_kernels.cuh"
#include "runtime.h"

namespace admp {

struct SysSpec {
  int natoms;
  int atom_off;
  int K[3];
  double kappa;
  int box_idx;
  long long green_off = -1;  // cached Green's function offset; -1: same as the spectrum offset
};

// Launch geometry of a batch.  hs is the host copy of the per-system table;
// bind_plan uploads it and points b.s at the device copy.
template <typename T>
struct RecipPlan {
  Batch b;
  SysDesc hs[kMaxBatch];
  size_t mesh_elems = 0;  // real mesh elements (all systems)
  size_t spec_elems = 0;  // complex spectrum elements
  size_t smem_z = 0, smem_y = 0, smem_x = 0;
  // fused slab passes: a block per run of x planes (blk_slab offsets), when a plane fits
  bool slab = false;
  int buf_elems = 0;
  size_t smem_slab = 0;
  // FP32 CG matvecs: x pass on the tensor cores (every K0 <= kTcMaxK), and the y and z passes too
  // (every K1, K2 <= kTcMaxK)
  bool tc_x = false;
  bool tc_y = false;
};

// The per-system table as one by-value parameter: the only launch of a call
// that carries it.
struct SysTable {
  SysDesc s[kMaxBatch];
};

static __global__ void sys_table_kernel(SysTable t, int n, SysDesc* __restrict__ dst) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = t.s[i];
}

// Upload the plan's system table to `dev` (kMaxBatch entries of device
// memory owned by the caller's workspace or pools) on stream `st`; the
// launches that follow on the same stream read it through b.s.
template <typename T>
inline int bind_plan(RecipPlan<T>& p, SysDesc* dev, cudaStream_t st) {
  if (!dev) return fail(ADMP_ERR_WORKSPACE, "no device memory for the system table");
  SysTable t;
  for (int s = 0; s < p.b.nsys; ++s) t.s[s] = p.hs[s];
  sys_table_kernel<<<1, 128, 0, st>>>(t, p.b.nsys, dev);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  p.b.s = dev;
  return ADMP_OK;
}

// The plan's launch descriptor with the first-block column of family F
// (F_ATOM is the plan's own; the FFT passes take theirs at their launches).
template <typename T>
inline Batch family_batch(const RecipPlan<T>& p, int F) {
  Batch b = p.b;
  b.fam = F;
  for (int s = 0; s < b.nsys; ++s) {
    const SysDesc& d = p.hs[s];
    b.blk[s] = F == F_ATOM ? d.blk_atom
               : F == F_Z  ? d.blk_z
               : F == F_Y  ? d.blk_y
               : F == F_X  ? d.blk_x
               : F == F_XT ? d.blk_xt
               : F == F_YT ? d.blk_yt
               : F == F_ZT ? d.blk_zt
                           : d.blk_slab;
  }
  return b;
}

// device bytes of a system table (kept 256-byte aligned for what follows it)
inline size_t sys_table_bytes() { return align_up(sizeof(SysDesc) * kMaxBatch, 256); }

template <typename T>
inline int build_recip_plan(const SysSpec* sys, int nsys, RecipPlan<T>& p) {
  if (nsys <= 0 || nsys > kMaxBatch) return fail(ADMP_ERR_BAD_ARG, "batch of %d systems (max %d)", nsys, kMaxBatch);
  Batch& b = p.b;
  b.nsys = nsys;
  b.apb = 256;
  b.done = nullptr;
  b.done_stride = 0;
  b.status_off = 0;
  b.s = nullptr;
  int maxK[3] = {1, 1, 1};
  for (int s = 0; s < nsys; ++s)
    for (int d = 0; d < 3; ++d) {
      if (sys[s].K[d] <= 0 || sys[s].K[d] > 4096)
        return fail(ADMP_ERR_MESH, "mesh size %d out of range [1, 4096]", sys[s].K[d]);
      maxK[d] = maxK[d] > sys[s].K[d] ? maxK[d] : sys[s].K[d];
    }
  b.maxK0 = maxK[0];
  b.maxK1 = maxK[1];
  b.maxK2 = maxK[2];
  const size_t cs = sizeof(Cplx<T>);
  const size_t budget = 150 * 1024;
  // z passes: lp line pairs of length K2 per block, two buffers
  int lp = (int)((sizeof(T) == 4 ? 4096 : 2048) / maxK[2]);
  lp = lp < 1 ? 1 : (lp > 64 ? 64 : lp);
  while (lp > 1 && (2 * (size_t)lp + 1) * maxK[2] * cs > budget) --lp;
  b.lp = lp;
  int zb = sizeof(T) == 4 ? 32 : 16;
  const int mk01 = maxK[0] > maxK[1] ? maxK[0] : maxK[1];
  while (zb > 1 && (2 * (size_t)zb + 1) * mk01 * cs + (mk01 + 2 * zb) * 8 + zb * 16 > budget) zb >>= 1;
  b.zb = zb;
  p.smem_z = (2 * (size_t)lp + 1) * maxK[2] * cs;
  p.smem_y = (2 * (size_t)zb + 1) * maxK[1] * cs;
  p.smem_x = (2 * (size_t)zb + 1) * maxK[0] * cs + ((size_t)maxK[0] + 2 * zb) * 8 + (size_t)zb * 16;
  if (p.smem_z > 227 * 1024 || p.smem_y > 227 * 1024 || p.smem_x > 227 * 1024)
    return fail(ADMP_ERR_MESH, "mesh %dx%dx%d too large for the shared-memory FFT", maxK[0], maxK[1], maxK[2]);
  int ba = 0, bz = 0, by = 0, bx = 0, bxt = 0, byt = 0, bzt = 0;
  size_t mo = 0, so = 0;
  for (int s = 0; s < nsys; ++s) {
    SysDesc& d = p.hs[s];
    d.atom_off = sys[s].atom_off;
    d.natoms = sys[s].natoms;
    d.K0 = sys[s].K[0];
    d.K1 = sys[s].K[1];
    d.K2 = sys[s].K[2];
    d.K2h = d.K2 / 2 + 1;
    d.kappa = sys[s].kappa;
    d.box_idx = sys[s].box_idx;
    d.flags = 0;
    d.blk_atom = ba;
    d.blk_z = bz;
    d.blk_y = by;
    d.blk_x = bx;
    d.blk_xt = bxt;
    d.blk_yt = byt;
    d.blk_zt = bzt;
    d.mesh_off = (int64_t)mo;
    d.spec_off = (int64_t)so;
    d.green_off = sys[s].green_off >= 0 ? (int64_t)sys[s].green_off : (int64_t)so;
    const int ncb = (d.K2h + zb - 1) / zb;
    ba += (d.natoms + b.apb - 1) / b.apb;
    bz += ((d.K0 * d.K1 + 1) / 2 + lp - 1) / lp;
    by += d.K0 * ncb;
    bx += (d.K1 * d.K2h + zb - 1) / zb;  // x passes: runs of zb flattened (y, kz) columns
    bxt += (d.K1 * d.K2h + kTcRows - 1) / kTcRows;
    byt += (d.K0 * d.K2h + kTcRows - 1) / kTcRows;
    bzt += (d.K0 * d.K1 + kTcRows - 1) / kTcRows;
    mo += align_up((size_t)d.K0 * d.K1 * d.K2, 64);
    so += align_up((size_t)d.K0 * d.K1 * d.K2h, 32);
  }
  b.nblk_atom = ba;
  b.nblk_xt = bxt;
  b.nblk_yt = byt;
  b.nblk_zt = bzt;
  p.tc_x = sizeof(T) == 4 && maxK[0] <= kTcMaxK;
  p.tc_y = p.tc_x && maxK[1] <= kTcMaxK && maxK[2] <= kTcMaxK;
  b.nblk_z = bz;
  b.nblk_y = by;
  b.nblk_x = bx;
  p.mesh_elems = mo;
  p.spec_elems = so;
  // fused slab passes: two buffers of at least one plane (max(ceil(K1/2) K2, K1 (K2/2+1)) complex) and at
  // least kSlabTarget complex values, so that small meshes take several planes per block; plus twiddles
  const int kSlabTarget = sizeof(T) == 4 ? 3072 : 1536;
  int be = kSlabTarget;
  for (int s = 0; s < nsys; ++s) {
    const int a = slab_plane_elems(sys[s].K[1], sys[s].K[2]);
    be = be > a ? be : a;
  }
  p.buf_elems = be;
  p.smem_slab = (2 * (size_t)be + maxK[1] + maxK[2]) * cs;
  p.slab = p.smem_slab <= 200 * 1024;
  b.nblk_slab = 0;
  for (int s = 0; s < nsys; ++s) {
    p.hs[s].blk_slab = b.nblk_slab;
    const int ppb = slab_ppb(be, slab_plane_elems(sys[s].K[1], sys[s].K[2]), sys[s].K[0]);
    b.nblk_slab += (sys[s].K[0] + ppb - 1) / ppb;
  }
  b.fam = F_ATOM;
  for (int s = 0; s < nsys; ++s) b.blk[s] = p.hs[s].blk_atom;
  return ADMP_OK;
}

// Mesh -> potential: the five FFT passes with the Green's function.
// 2 G_s for every half-spectrum point of the batch, at each system's green_off
template <typename T>
inline int launch_green_build(const RecipPlan<T>& p, const T* box, T* green, double ke, cudaStream_t st) {
  if (p.b.nblk_x) green_build_kernel<T><<<p.b.nblk_x, 256, 0, st>>>(family_batch(p, F_X), box, green, ke);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

template <typename T>
inline int launch_fft_green(const RecipPlan<T>& p, T* mesh, Cplx<T>* spec, const T* box, double* acc, double ke,
                            cudaStream_t st, const T* green = nullptr) {
  const Batch& b = p.b;
  const Batch bsl = family_batch(p, F_SLAB), bz = family_batch(p, F_Z), by = family_batch(p, F_Y),
              bx = family_batch(p, F_X);
  ADMP_CUDA_TRY(ensure_smem(fft_z_fwd_kernel<T>, p.smem_z));
  ADMP_CUDA_TRY(ensure_smem(fft_z_inv_kernel<T>, p.smem_z));
  ADMP_CUDA_TRY(ensure_smem(fft_y_kernel<T, false>, p.smem_y));
  ADMP_CUDA_TRY(ensure_smem(fft_y_kernel<T, true>, p.smem_y));
  ADMP_CUDA_TRY(ensure_smem(fft_x_green_kernel<T>, p.smem_x));
  ADMP_CUDA_TRY(ensure_smem(fft_x_apply_kernel<T>, p.smem_x));
  // algorithmic bytes: z passes read/write M reals + Mh complex, y/x passes Mh complex in and out
  const double rb = (double)p.mesh_elems * sizeof(T), cb = (double)p.spec_elems * sizeof(Cplx<T>);
  int h;
  // FP32 CG matvecs on the tensor cores: every pass a matrix product
  const uint32_t* tct = (green && p.tc_x) ? tc_tables(st) : nullptr;
  if (tct) ADMP_CUDA_TRY(ensure_smem(tc_x_apply_kernel, (size_t)kTcSmem));
  if (tct && p.tc_y) {
    ADMP_CUDA_TRY(ensure_smem(tc_y_kernel<false>, (size_t)kTcSmem));
    ADMP_CUDA_TRY(ensure_smem(tc_y_kernel<true>, (size_t)kTcSmem));
    ADMP_CUDA_TRY(ensure_smem(tc_zf_kernel, (size_t)kTcSmem));
    ADMP_CUDA_TRY(ensure_smem(tc_zi_kernel, (size_t)kTcSmem));
    const Batch bzt = family_batch(p, F_ZT);
    Cplx<float>* sp = (Cplx<float>*)spec;
    const Batch byt = family_batch(p, F_YT);
    h = prof_begin(st);
    if (b.nblk_zt) tc_zf_kernel<<<b.nblk_zt, 256, kTcSmem, st>>>(bzt, (const float*)mesh, sp, tct);
    prof_end(h, PK_TC_Z_FWD, rb + cb, st);
    h = prof_begin(st);
    if (b.nblk_yt) tc_y_kernel<false><<<b.nblk_yt, 256, kTcSmem, st>>>(byt, sp, tct);
    prof_end(h, PK_TC_Y_FWD, 2 * cb, st);
    h = prof_begin(st);
    if (b.nblk_xt)
      tc_x_apply_kernel<<<b.nblk_xt, 256, kTcSmem, st>>>(family_batch(p, F_XT), sp, (const float*)green, tct);
    prof_end(h, PK_TC_X, 2 * cb + (double)p.spec_elems * sizeof(T), st);
    h = prof_begin(st);
    if (b.nblk_yt) tc_y_kernel<true><<<b.nblk_yt, 256, kTcSmem, st>>>(byt, sp, tct);
    prof_end(h, PK_TC_Y_INV, 2 * cb, st);
    h = prof_begin(st);
    if (b.nblk_zt) tc_zi_kernel<<<b.nblk_zt, 256, kTcSmem, st>>>(bzt, sp, (float*)mesh, tct);
    prof_end(h, PK_TC_Z_INV, rb + cb, st);
    count_launches(5);
    ADMP_CUDA_TRY(cudaGetLastError());
    return ADMP_OK;
  }
  if (p.slab) {
    ADMP_CUDA_TRY(ensure_smem(fft_slab_fwd_kernel<T>, p.smem_slab));
    ADMP_CUDA_TRY(ensure_smem(fft_slab_inv_kernel<T>, p.smem_slab));
    h = prof_begin(st);
    if (b.nblk_slab) fft_slab_fwd_kernel<T><<<b.nblk_slab, 256, p.smem_slab, st>>>(bsl, mesh, spec, p.buf_elems);
    prof_end(h, PK_FFT_Z_FWD, rb + cb, st);
  } else {
    h = prof_begin(st);
    if (b.nblk_z) fft_z_fwd_kernel<T><<<b.nblk_z, 256, p.smem_z, st>>>(bz, mesh, spec);
    prof_end(h, PK_FFT_Z_FWD, rb + cb, st);
    h = prof_begin(st);
    if (b.nblk_y) fft_y_kernel<T, false><<<b.nblk_y, 256, p.smem_y, st>>>(by, spec);
    prof_end(h, PK_FFT_Y_FWD, 2 * cb, st);
  }
  h = prof_begin(st);
  if (b.nblk_x) {
    if (tct)
      tc_x_apply_kernel<<<b.nblk_xt, 256, kTcSmem, st>>>(family_batch(p, F_XT), (Cplx<float>*)spec,
                                                          (const float*)green, tct);
    else if (green)
      fft_x_apply_kernel<T><<<b.nblk_x, 256, p.smem_x, st>>>(bx, spec, green);
    else
      fft_x_green_kernel<T><<<b.nblk_x, 256, p.smem_x, st>>>(bx, spec, box, acc, ke);
  }
  // spectrum in and out, plus the cached Green's function (one real per entry) when it is read
  prof_end(h, PK_FFT_X_GREEN, 2 * cb + (green ? (double)p.spec_elems * sizeof(T) : 0.0), st);
  if (p.slab) {
    h = prof_begin(st);
    if (b.nblk_slab) fft_slab_inv_kernel<T><<<b.nblk_slab, 256, p.smem_slab, st>>>(bsl, spec, mesh, p.buf_elems);
    prof_end(h, PK_FFT_Z_INV, rb + cb, st);
    count_launches(3);
  } else {
    h = prof_begin(st);
    if (b.nblk_y) fft_y_kernel<T, true><<<b.nblk_y, 256, p.smem_y, st>>>(by, spec);
    prof_end(h, PK_FFT_Y_INV, 2 * cb, st);
    h = prof_begin(st);
    if (b.nblk_z) fft_z_inv_kernel<T><<<b.nblk_z, 256, p.smem_z, st>>>(bz, spec, mesh);
    prof_end(h, PK_FFT_Z_INV, rb + cb, st);
    count_launches(5);
  }
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

// Full reciprocal evaluation: spread q, FFT/Green, gather.
// `dE_dq` receives the potential (dE/dq), `dE_dpos` the gradient; both accumulate.
template <typename T>
inline size_t spread_smem() {
  return 8 * WarpStencil<T, false>::bytes();
}
template <typename T, bool F>
inline size_t gather_smem() {
  return 8 * WarpStencil<T, F>::bytes();
}

template <typename T>
inline double plan_atoms(const RecipPlan<T>& p) {
  double n = 0;
  for (int s = 0; s < p.b.nsys; ++s) n += p.hs[s].natoms;
  return n;
}

template <typename T>
inline int launch_spread(const Batch& b, const T* pos, const T* box, const T* q, T* mesh, const int* order,
                         cudaStream_t st) {
  if (!b.nblk_atom) return ADMP_OK;
  ADMP_CUDA_TRY(ensure_smem(spread_kernel<T>, spread_smem<T>()));
  spread_kernel<T><<<b.nblk_atom, 256, spread_smem<T>(), st>>>(b, pos, box, q, mesh, order);
  return ADMP_OK;
}

template <typename T, bool F>
inline int launch_gather(const Batch& b, const T* pos, const T* box, const T* q, const T* phi, T* dE_dq,
                         T* dE_dpos, double* acc, const int* order, cudaStream_t st) {
  if (!b.nblk_atom) return ADMP_OK;
  ADMP_CUDA_TRY(ensure_smem(gather_kernel<T, F>, gather_smem<T, F>()));
  gather_kernel<T, F><<<b.nblk_atom, 256, gather_smem<T, F>(), st>>>(b, pos, box, q, phi, dE_dq, dE_dpos, acc, T(1),
                                                                     order);
  return ADMP_OK;
}

template <typename T>
inline int launch_recip(const RecipPlan<T>& p, const T* pos, const T* box, const T* q, T* mesh, Cplx<T>* spec,
                        double* acc, double ke, T* dE_dq, T* dE_dpos, cudaStream_t st,
                        const int* order = nullptr) {
  const Batch& b = p.b;
  const double na = plan_atoms(p), mb = (double)p.mesh_elems * sizeof(T);
  ADMP_CUDA_TRY(cudaMemsetAsync(mesh, 0, p.mesh_elems * sizeof(T), st));
  int h = prof_begin(st);
  int s = launch_spread<T>(b, pos, box, q, mesh, order, st);
  if (s) return s;
  prof_end(h, PK_SPREAD, na * 4 * sizeof(T) + mb, st);
  count_launches(1);
  s = launch_fft_green<T>(p, mesh, spec, box, acc, ke, st);
  if (s) return s;
  h = prof_begin(st);
  s = launch_gather<T, true>(b, pos, box, q, mesh, dE_dq, dE_dpos, acc, order, st);
  if (s) return s;
  prof_end(h, PK_GATHER, mb + na * 4 * sizeof(T) + na * 3 * sizeof(T), st);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

// Potential only (for the CG matvec): phi_i = dE/dq_i of the charges v.
template <typename T>
inline int launch_recip_potential(const RecipPlan<T>& p, const T* pos, const T* box, const T* v, T* mesh,
                                  Cplx<T>* spec, double* acc, double ke, T* pot, cudaStream_t st,
                                  const int* order = nullptr, const T* green = nullptr) {
  const Batch& b = p.b;
  const double na = plan_atoms(p), mb = (double)p.mesh_elems * sizeof(T);
  ADMP_CUDA_TRY(cudaMemsetAsync(mesh, 0, p.mesh_elems * sizeof(T), st));
  int h = prof_begin(st);
  int s = launch_spread<T>(b, pos, box, v, mesh, order, st);
  if (s) return s;
  prof_end(h, PK_SPREAD, na * 4 * sizeof(T) + mb, st);
  s = launch_fft_green<T>(p, mesh, spec, box, acc, ke, st, green);
  if (s) return s;
  h = prof_begin(st);
  s = launch_gather<T, false>(b, pos, box, v, mesh, pot, nullptr, acc, order, st);
  if (s) return s;
  prof_end(h, PK_GATHER, mb + na * 4 * sizeof(T) + na * sizeof(T), st);
  count_launches(2);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

}  // namespace admp
