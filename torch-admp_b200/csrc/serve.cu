// Batched serving entry points: many independent PME / QEq systems per launch,
// with per-slot state (positions, CSR neighbour rows, CG vectors and scalars)
// that persists in caller-owned pools between calls, so a scheduler can admit
// and retire systems between CG iterations (continuous batching).
#include "pme_host.h"
#include "qeq_kernels.cuh"
#include "serve_kernels.cuh"

namespace admp {

struct SrvLaunch {
  Batch b;
  long long pair_off[kMaxBatch];
  long long pair_cap[kMaxBatch];
  double rc[kMaxBatch];
  int cell_off[kMaxBatch];
};

// (Re)build the per-launch system table; `fresh` recomputes geometry and
// clears the status (neighbour build), otherwise status comes from slot_info.
__global__ void srv_table_kernel(SrvLaunch L, const void* box_v, int dbl, const int* __restrict__ slot_info,
                                 SrvSys* __restrict__ ss, int fresh) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= L.b.nsys) return;
  const SysDesc d = L.b.s[s];
  SrvSys& S = ss[s];
  S.pair_off = L.pair_off[s];
  S.pair_cap = L.pair_cap[s];
  S.rc = L.rc[s];
  S.kappa = d.kappa;
  S.kind = d.flags;
  S.slot = d.box_idx;
  S.cell_off = L.cell_off[s];
  if (!fresh) {
    if (dbl)
      load_box((const double*)box_v + (size_t)d.box_idx * 9, S.b);
    else
      load_box((const float*)box_v + (size_t)d.box_idx * 9, S.b);
    inv3(S.b, S.bi);
    S.status = slot_info ? slot_info[4 * d.box_idx + 2] : 0;
  }
}

// done flag, iterations, status and (optionally) the residual ||P grad||_2 / N
// of the latest iterate of each listed QEq slot
__global__ void slot_export_kernel(Batch b, const CGScal* __restrict__ sc, int* __restrict__ slot_info,
                                   double* __restrict__ slot_resid) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.nsys) return;
  const int sl = b.s[s].box_idx;
  slot_info[4 * sl + 0] = sc[sl].done;
  slot_info[4 * sl + 1] = sc[sl].iter;
  if (sc[sl].status) slot_info[4 * sl + 2] = sc[sl].status;
  if (slot_resid) {
    const double rr = sc[sl].rr_new;  // the latest residual (init and every update leave it there)
    slot_resid[sl] = sqrt(rr > 0.0 ? rr : 0.0) / (double)(b.s[s].natoms > 0 ? b.s[s].natoms : 1);
  }
}

__global__ void slot_reset_kernel(Batch b, CGScal* __restrict__ sc, int nc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.nsys) return;
  const int sl = b.s[s].box_idx;
  CGScal z;
  memset(&z, 0, sizeof(CGScal));
  z.n_const = nc;
  sc[sl] = z;
}

// zero the CG accumulators of the listed slots, keeping Ginv / b / constants
__global__ void slot_clear_acc_kernel(Batch b, CGScal* __restrict__ sc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.nsys) return;
  CGScal& S = sc[b.s[s].box_idx];
  S.rr = 0.0;
  S.rr_new = 0.0;
  S.pHp = 0.0;
  for (int c = 0; c < kMaxConst; ++c) S.Cv[c] = 0.0;
  S.sp = 0.0;
  S.spz = 0.0;
  S.spz2 = 0.0;
}

template <typename T>
__global__ void __launch_bounds__(256) cast_atoms_kernel(Batch b, const T* __restrict__ in, double* __restrict__ out,
                                                         int to_double, T* __restrict__ back,
                                                         const double* __restrict__ src) {
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    if (to_double)
      out[i] = (double)in[i];
    else
      back[i] = (T)src[i];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) zero_vec_kernel(Batch b, T* __restrict__ v) {
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) v[d.atom_off + a] = T(0);
}

struct SrvCtx {
  SrvLaunch L;
  size_t cells_need;
};

// per-system scratch of a call, after the system table at the head of sys_scratch
static SrvSys* srv_sys(const admp_pools* P) { return (SrvSys*)((char*)P->sys_scratch + sys_table_bytes()); }

template <typename T>
static int srv_build(const admp_pools* P, const admp_sys* sys, int nsys, RecipPlan<T>& plan, SrvCtx& c,
                     bool need_mesh, cudaStream_t stream) {
  if (nsys <= 0 || nsys > kMaxBatch) return fail(ADMP_ERR_BAD_ARG, "serve: %d systems per call (1..%d)", nsys, kMaxBatch);
  SysSpec spec[kMaxBatch];
  size_t coff = 0;
  for (int s = 0; s < nsys; ++s) {
    const admp_sys& a = sys[s];
    if (a.natoms <= 0 || a.atom_off < 0 || a.slot < 0) return fail(ADMP_ERR_BAD_ARG, "serve: bad system %d", s);
    spec[s].natoms = a.natoms;
    spec[s].atom_off = a.atom_off;
    for (int d = 0; d < 3; ++d) spec[s].K[d] = a.kmesh[d];
    spec[s].kappa = a.kappa;
    spec[s].box_idx = a.slot;
    spec[s].green_off = a.kind == ADMP_SYS_QEQ ? a.green_off : -1;
    if (a.kind == ADMP_SYS_QEQ && P->green) {
      const long long need = (long long)a.kmesh[0] * a.kmesh[1] * (a.kmesh[2] / 2 + 1);
      if (a.green_off < 0 || a.green_off + need > P->green_cap)
        return fail(ADMP_ERR_WORKSPACE, "serve: green region of system %d outside the pool", s);
    }
    c.L.pair_off[s] = a.pair_off;
    c.L.pair_cap[s] = a.pair_cap;
    c.L.rc[s] = a.rcut;
    c.L.cell_off[s] = (int)coff;
    coff += 3 * (size_t)(2 * a.natoms + 128 + 1);
  }
  c.cells_need = coff;
  int st = build_recip_plan<T>(spec, nsys, plan);
  if (st) return st;
  for (int s = 0; s < nsys; ++s) plan.hs[s].flags = sys[s].kind;
  if (need_mesh) {
    if ((long long)plan.mesh_elems > P->mesh_cap || (long long)plan.spec_elems > P->spec_cap || nsys > P->acc_cap)
      return fail(ADMP_ERR_WORKSPACE, "serve: mesh pool too small (need %zu real, %zu complex)", plan.mesh_elems,
                  plan.spec_elems);
  }
  if ((size_t)P->sys_scratch_bytes < sys_table_bytes() + sizeof(SrvSys) * nsys)
    return fail(ADMP_ERR_WORKSPACE, "serve: sys scratch too small");
  // the call's system table goes to the head of the sys scratch; its launches follow on the same stream
  st = bind_plan<T>(plan, (SysDesc*)P->sys_scratch, stream);
  if (st) return st;
  c.L.b = plan.b;
  return ADMP_OK;
}

template <typename T>
static int serve_neighbors_impl(const admp_pools* P, const admp_sys* sys, int nsys, cudaStream_t st) {
  RecipPlan<T> plan;
  SrvCtx c;
  int s = srv_build<T>(P, sys, nsys, plan, c, false, st);
  if (s) return s;
  if ((long long)c.cells_need > P->cells_cap) return fail(ADMP_ERR_WORKSPACE, "serve: cell pool too small (%zu)", c.cells_need);
  SrvSys* ss = srv_sys(P);
  const Batch& b = plan.b;
  typedef typename Vec4<T>::type V4;
  const int hn = prof_begin(st);
  srv_table_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(c.L, P->box, sizeof(T) == 8, nullptr, ss, 1);
  if (P->pos64 && !P->frac64) return fail(ADMP_ERR_BAD_ARG, "serve: pos64 needs a frac64 scratch");
  const double4* f64 = P->pos64 ? (const double4*)P->frac64 : nullptr;
  sn_setup_kernel<T><<<nsys, 256, 0, st>>>(b, ss, (const T*)P->box, P->box64, P->cells);
  sn_bin_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, ss, (const T*)P->pos, P->pos64, (V4*)P->frac,
                                                P->pos64 ? (double4*)P->frac64 : nullptr, P->cell_of, P->cells,
                                                P->pcnt, P->pstart);
  sn_scan_cells_kernel<<<nsys, 1024, 0, st>>>(ss, P->cells);
  sn_scatter_kernel<<<b.nblk_atom, 256, 0, st>>>(b, ss, P->cell_of, P->cells, P->sorted);
  sn_pairs_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, ss, (const V4*)P->frac, f64, P->cell_of, P->cells, P->sorted,
                                                  P->pcnt, P->pstart, P->col);
  sn_export_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(b, ss, P->slot_info);
  prof_end(hn, PK_NEIGHBORS, -1.0, st);
  count_launches(7);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

template <typename T>
static int serve_ef_impl(const admp_pools* P, const admp_sys* sys, int nsys, double ke, cudaStream_t st) {
  RecipPlan<T> plan;
  SrvCtx c;
  int s = srv_build<T>(P, sys, nsys, plan, c, true, st);
  if (s) return s;
  SrvSys* ss = srv_sys(P);
  const Batch& b = plan.b;
  typedef typename Vec4<T>::type V4;
  srv_table_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(c.L, P->box, sizeof(T) == 8, P->slot_info, ss, 0);
  zero_atoms_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, (T*)P->force, P->energy);
  int h = prof_begin(st);
  pair_ef_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, ss, (const V4*)P->frac,
                                                 P->pos64 ? (const double4*)P->frac64 : nullptr, (const T*)P->q,
                                                 (const T*)P->eta, P->pstart, P->pcnt, P->col, ke, (T*)P->force,
                                                 P->energy);
  prof_end(h, PK_PAIR_EF, plan_atoms(plan) * (sizeof(V4) + 2 * sizeof(T) + 12 + 3 * sizeof(T)), st);
  count_launches(6);
  ADMP_CUDA_TRY(cudaMemsetAsync(P->acc, 0, sizeof(double) * kAccStride * nsys, st));
  s = launch_recip<T>(plan, (const T*)P->pos, (const T*)P->box, (const T*)P->q, (T*)P->mesh, (Cplx<T>*)P->spec,
                      P->acc, ke, nullptr, (T*)P->force, st, P->sorted);
  if (s) return s;
  recip_finalize_kernel<T><<<(nsys + 127) / 128, 128, 0, st>>>(b, (const T*)P->box, P->acc, P->energy, nullptr);
  sys_terms_kernel<T><<<nsys, 512, 0, st>>>(b, ss, (const T*)P->q, (const T*)P->chi, (const T*)P->hardness,
                                            (const T*)P->eta, ke, P->energy);
  negate_atoms_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, (T*)P->force);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

// CSR SpMV (QEq real-space matrix times v) fused with the end of the matvec (as
// qeq_finish_kernel): per row h = (recip + J_real v)_i + diag_i v_i + nn sum(v)
// (+ slab terms), Hv_i = h, and the block sums of v.h and C.h into the CG
// scalars -- one pass over the rows instead of two.
template <typename T>
static __global__ void __launch_bounds__(256)
    csr_spmv_finish_kernel(Batch b, QEqParams prm, const long long* __restrict__ pstart, const int* __restrict__ pcnt,
                           const int* __restrict__ col, const T* __restrict__ coef, const T* __restrict__ v,
                           T* __restrict__ Hv, const double* __restrict__ diag, const double* __restrict__ zc,
                           CGScal* __restrict__ sc, double* __restrict__ hv_out) {
  __shared__ double red[5 * 32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  if (sc[s].done) return;
  const CGScal& S = sc[s];
  const double sp = S.sp, spz = S.spz, spz2 = S.spz2;
  const bool slab = (prm.flags & ADMP_QEQ_SLAB) != 0;
  const int nc = S.n_const;
  double accs[5] = {0, 0, 0, 0, 0};
  const int sub = threadIdx.x & (kSpmvLanes - 1);
  const int grp = threadIdx.x / kSpmvLanes, ngrp = blockDim.x / kSpmvLanes;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  long long st_next = 0;
  int n_next = 0;
  if (a0 + grp < a1) {
    st_next = pstart[d.atom_off + a0 + grp];
    n_next = pcnt[d.atom_off + a0 + grp];
  }
  for (int base = a0; base < a1; base += ngrp) {
    const int a = base + grp;
    const bool row = a < a1;
    const int i = d.atom_off + (row ? a : a0);
    const long long st = st_next;
    const int n = row ? n_next : 0;
    if (a + ngrp < a1) {
      st_next = pstart[i + ngrp];
      n_next = pcnt[i + ngrp];
    }
    T acc = 0;
    for (int k0 = 0; k0 < n; k0 += kSpmvLanes * kSpmvUnroll) {
      int c[kSpmvUnroll];
      T w[kSpmvUnroll];
#pragma unroll
      for (int u = 0; u < kSpmvUnroll; ++u) {
        const int k = k0 + sub + u * kSpmvLanes;
        const bool ok = k < n;
        c[u] = ok ? col[st + k] : -1;
        w[u] = ok ? coef[st + k] : T(0);
      }
      T vv[kSpmvUnroll];
#pragma unroll
      for (int u = 0; u < kSpmvUnroll; ++u) vv[u] = c[u] >= 0 ? v[c[u]] : T(0);
#pragma unroll
      for (int u = 0; u < kSpmvUnroll; ++u) acc += w[u] * vv[u];
    }
#pragma unroll
    for (int o = kSpmvLanes / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (row && sub == 0) {
      const T hv = Hv[i] + acc;
      const double x = (double)v[i];
      double h = (double)hv + diag[i] * x + S.nn * sp;
      if (slab) {
        const double z = zc[i];
        h += S.pre * (2.0 * z * spz - spz2 - z * z * sp - S.Lz2 / 6.0 * sp);
      }
      Hv[i] = (T)h;
      if (hv_out) hv_out[i] = h;
      accs[0] += x * h;
#pragma unroll
      for (int cc = 0; cc < kMaxConst; ++cc)  // serving constraints are total-charge rows
        if (cc < nc) accs[1 + cc] += h;
    }
  }
  double a1v[1] = {accs[0]};
  block_atomic_sum<1>(a1v, &sc[s].pHp, red);
  if (nc > 0) {
    double a4[4] = {accs[1], accs[2], accs[3], accs[4]};
    block_atomic_sum<4>(a4, sc[s].Cv, red);
  }
}

// H v for the listed systems: Hv must be zeroed, sums of v in the CG state.
template <typename T>
static int srv_matvec(const admp_pools* P, const RecipPlan<T>& plan, QEqParams prm, const T* v, T* Hv,
                      double* hv_out, double ke, cudaStream_t st) {
  const Batch& b = plan.b;
  int s = launch_recip_potential<T>(plan, (const T*)P->pos, (const T*)P->box, v, (T*)P->mesh, (Cplx<T>*)P->spec,
                                    P->acc, ke, Hv, st, P->sorted, (const T*)P->green);
  if (s) return s;
  int h = prof_begin(st);
  csr_spmv_finish_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, prm, P->pstart, P->pcnt, P->col, (const T*)P->coef, v,
                                                         Hv, P->cg_diag, P->cg_z, (CGScal*)P->cg_state, hv_out);
  prof_end(h, PK_CSR_SPMV, -1.0, st);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

static QEqParams srv_params(double tol, int max_iter, double ke) {
  QEqParams p;
  p.flags = ADMP_QEQ_KSPACE | ADMP_QEQ_RSPACE | ADMP_QEQ_DAMPING;
  p.axis = 2;
  p.max_iter = max_iter;
  p.tol = tol;
  p.ke = ke;
  return p;
}

template <typename T>
static int serve_qeq_init_impl(const admp_pools* P, const admp_sys* sys, int nsys, double tol, int max_iter,
                               double ke, cudaStream_t st) {
  RecipPlan<T> plan;
  SrvCtx c;
  int s = srv_build<T>(P, sys, nsys, plan, c, true, st);
  if (s) return s;
  SrvSys* ss = srv_sys(P);
  const Batch& b = plan.b;
  typedef typename Vec4<T>::type V4;
  CGScal* sc = (CGScal*)P->cg_state;
  const QEqParams prm = srv_params(tol, max_iter, ke);
  srv_table_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(c.L, P->box, sizeof(T) == 8, P->slot_info, ss, 0);
  slot_reset_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(b, sc, 1);
  qeq_setup_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, prm, (const T*)P->pos, (const T*)P->box, (const T*)P->chi,
                                                  (const T*)P->hardness, (const T*)P->eta, (const T*)nullptr,
                                                  P->cg_diag, P->cg_z, P->cg_chi, sc);
  if (P->green) {
    s = launch_green_build<T>(plan, (const T*)P->box, (T*)P->green, ke, st);
    if (s) return s;
  }
  // total-charge constraint: Gram = N
  qeq_gram_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, 1, (const T*)nullptr, 0, sc);
  qeq_gram_invert_kernel<<<(nsys + 31) / 32, 32, 0, st>>>(b, 1, sc);
  csr_coef_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, ss, (const V4*)P->frac, (const T*)P->eta, P->pstart, P->pcnt,
                                                  P->col, ke, (T*)P->coef);
  // x0 = P(q_warm)
  cast_atoms_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, (const T*)P->q, P->cg_x, 1, nullptr, nullptr);
  qeq_sums_kernel<T, double><<<b.nblk_atom, 256, 0, st>>>(b, P->cg_x, P->cg_z, (const T*)nullptr, 0, 1, 1, sc,
                                                          nullptr, nullptr);
  qeq_project_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, P->cg_x, (const T*)nullptr, 0, sc);
  slot_clear_acc_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(b, sc);
  // H x0
  qeq_sums_kernel<T, double><<<b.nblk_atom, 256, 0, st>>>(b, P->cg_x, P->cg_z, (const T*)nullptr, 0, 1, 0, sc,
                                                          (T*)P->cg_hp, (T*)P->cg_p);
  s = srv_matvec<T>(P, plan, prm, (const T*)P->cg_p, (T*)P->cg_hp, P->cg_hx, ke, st);
  if (s) return s;
  slot_clear_acc_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(b, sc);
  zero_vec_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, (T*)P->cg_hp);
  qeq_resid_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, P->cg_hx, P->cg_chi, (const T*)nullptr, 0, P->cg_z, P->cg_r,
                                                   (T*)P->cg_p, sc, 0);
  qeq_resid_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, P->cg_hx, P->cg_chi, (const T*)nullptr, 0, P->cg_z, P->cg_r,
                                                   (T*)P->cg_p, sc, 1);
  qeq_init_done_kernel<<<(nsys + 31) / 32, 32, 0, st>>>(b, prm, sc);
  slot_export_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(b, sc, P->slot_info, P->slot_resid);
  count_launches(18);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

template <typename T>
static int serve_qeq_iterate_impl(const admp_pools* P, const admp_sys* sys, int nsys, int niter, double tol,
                                  int max_iter, double ke, cudaStream_t st) {
  RecipPlan<T> plan;
  SrvCtx c;
  int s = srv_build<T>(P, sys, nsys, plan, c, true, st);
  if (s) return s;
  CGScal* sc = (CGScal*)P->cg_state;
  plan.b.done = &sc[0].done;
  plan.b.done_stride = (int)(sizeof(CGScal) / sizeof(int));
  plan.b.status_off = (int)((offsetof(CGScal, status) - offsetof(CGScal, done)) / sizeof(int));
  const Batch& b = plan.b;
  const QEqParams prm = srv_params(tol, max_iter, ke);
  for (int k = 0; k < niter; ++k) {
    count_launches(3);
    qeq_rotate_kernel<<<(nsys + 31) / 32, 32, 0, st>>>(b, sc);
    s = srv_matvec<T>(P, plan, prm, (const T*)P->cg_p, (T*)P->cg_hp, nullptr, ke, st);
    if (s) return s;
    const int hv = prof_begin(st);
    qeq_update_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, P->cg_x, P->cg_r, (const T*)P->cg_p, (T*)P->cg_hp,
                                                      (const T*)nullptr, 0, sc);
    qeq_direction_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, prm, P->cg_r, (T*)P->cg_p, P->cg_z, sc);
    prof_end(hv, PK_CG_VECTOR, -1.0, st);
  }
  slot_export_kernel<<<(nsys + 63) / 64, 64, 0, st>>>(b, sc, P->slot_info, P->slot_resid);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

template <typename T>
static int serve_qeq_finish_impl(const admp_pools* P, const admp_sys* sys, int nsys, cudaStream_t st) {
  RecipPlan<T> plan;
  SrvCtx c;
  int s = srv_build<T>(P, sys, nsys, plan, c, false, st);
  if (s) return s;
  const Batch& b = plan.b;
  cast_atoms_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, nullptr, nullptr, 0, (T*)P->q, P->cg_x);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

}  // namespace admp

using namespace admp;

extern "C" size_t admp_serve_slot_state_bytes(void) { return sizeof(CGScal); }
extern "C" size_t admp_serve_sys_scratch_bytes(int nsys) {
  return sys_table_bytes() + sizeof(SrvSys) * (size_t)(nsys > 0 ? nsys : 1);
}
extern "C" size_t admp_serve_cells_needed(const admp_sys* sys, int nsys) {
  size_t c = 0;
  for (int s = 0; s < nsys; ++s) c += 3 * (size_t)(2 * sys[s].natoms + 128 + 1);
  return c;
}

#define SERVE_DISPATCH(call_f64, call_f32)                   \
  do {                                                       \
    if (dtype == ADMP_F64) return call_f64;                  \
    if (dtype == ADMP_F32) return call_f32;                  \
    return fail(ADMP_ERR_BAD_ARG, "bad dtype");              \
  } while (0)

extern "C" int admp_serve_neighbors(int dtype, const admp_pools* P, const admp_sys* sys, int nsys, void* stream) {
  if (!P || !sys) return fail(ADMP_ERR_BAD_ARG, "serve: null pools/systems");
  cudaStream_t st = (cudaStream_t)stream;
  SERVE_DISPATCH(serve_neighbors_impl<double>(P, sys, nsys, st), serve_neighbors_impl<float>(P, sys, nsys, st));
}

extern "C" int admp_serve_energy_forces(int dtype, const admp_pools* P, const admp_sys* sys, int nsys, double ke,
                                        void* stream) {
  if (!P || !sys) return fail(ADMP_ERR_BAD_ARG, "serve: null pools/systems");
  cudaStream_t st = (cudaStream_t)stream;
  SERVE_DISPATCH(serve_ef_impl<double>(P, sys, nsys, ke, st), serve_ef_impl<float>(P, sys, nsys, ke, st));
}

extern "C" int admp_serve_qeq_init(int dtype, const admp_pools* P, const admp_sys* sys, int nsys, double tol,
                                   int max_iter, double ke, void* stream) {
  if (!P || !sys) return fail(ADMP_ERR_BAD_ARG, "serve: null pools/systems");
  cudaStream_t st = (cudaStream_t)stream;
  SERVE_DISPATCH(serve_qeq_init_impl<double>(P, sys, nsys, tol, max_iter, ke, st),
                 serve_qeq_init_impl<float>(P, sys, nsys, tol, max_iter, ke, st));
}

extern "C" int admp_serve_qeq_iterate(int dtype, const admp_pools* P, const admp_sys* sys, int nsys, int niter,
                                      double tol, int max_iter, double ke, void* stream) {
  if (!P || !sys || niter < 0) return fail(ADMP_ERR_BAD_ARG, "serve: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  SERVE_DISPATCH(serve_qeq_iterate_impl<double>(P, sys, nsys, niter, tol, max_iter, ke, st),
                 serve_qeq_iterate_impl<float>(P, sys, nsys, niter, tol, max_iter, ke, st));
}

extern "C" int admp_serve_qeq_finish(int dtype, const admp_pools* P, const admp_sys* sys, int nsys, void* stream) {
  if (!P || !sys) return fail(ADMP_ERR_BAD_ARG, "serve: null pools/systems");
  cudaStream_t st = (cudaStream_t)stream;
  SERVE_DISPATCH(serve_qeq_finish_impl<double>(P, sys, nsys, st), serve_qeq_finish_impl<float>(P, sys, nsys, st));
}
