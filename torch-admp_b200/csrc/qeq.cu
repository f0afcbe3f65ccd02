// admp_qeq_solve / admp_qeq_hvp: matrix-free projected CG for the QEq and
// electrode charges (replaces pgrad_optimize and the quadratic / LBFGS
// minimisers, qeq.py:1117-1527, electrode.py:456-560).
#include <vector>

#include "pme_host.h"
#include "qeq_kernels.cuh"

namespace admp {

template <typename T>
struct QEqWS {
  RecipPlan<T> plan;
  SysDesc* table;
  T* mesh;
  Cplx<T>* spec;
  T* green;
  double* acc;
  double *x, *r, *diag, *zc, *chi_eff, *hx;
  T *p, *Hp, *coef;
  CGScal* sc;
  size_t bytes;
};

// nf frames of N atoms each (frame f: atoms [f N, (f+1) N), box f, mesh
// kmesh[3 f .. 3 f + 2]); every per-atom vector spans all frames.
template <typename T>
static int qeq_carve(QEqWS<T>& w, void* ws, size_t bytes, int nf, int N, long long P, const int* kmesh,
                     double kappa, int flags) {
  if (nf <= 0 || nf > kMaxBatch) return fail(ADMP_ERR_BAD_ARG, "qeq: %d frames per call (1..%d)", nf, kMaxBatch);
  SysSpec sys[kMaxBatch];
  for (int f = 0; f < nf; ++f) {
    sys[f].natoms = N;
    sys[f].atom_off = f * N;
    for (int d = 0; d < 3; ++d) sys[f].K[d] = (flags & ADMP_QEQ_KSPACE) ? kmesh[3 * f + d] : 1;
    sys[f].kappa = kappa > 0 ? kappa : 1.0;
    sys[f].box_idx = f;
  }
  int s = build_recip_plan<T>(sys, nf, w.plan);
  if (s) return s;
  const size_t NT = (size_t)nf * N;
  Carver c(ws, bytes);
  w.table = reinterpret_cast<SysDesc*>(c.take<unsigned char>(sys_table_bytes()));
  w.mesh = c.take<T>((flags & ADMP_QEQ_KSPACE) ? w.plan.mesh_elems : 0);
  w.spec = c.take<Cplx<T>>((flags & ADMP_QEQ_KSPACE) ? w.plan.spec_elems : 0);
  w.green = c.take<T>((flags & ADMP_QEQ_KSPACE) ? w.plan.spec_elems : 0);
  w.acc = c.take<double>((size_t)kAccStride * nf);
  w.x = c.take<double>(NT);
  w.r = c.take<double>(NT);
  w.diag = c.take<double>(NT);
  w.zc = c.take<double>(NT);
  w.chi_eff = c.take<double>(NT);
  w.hx = c.take<double>(NT);
  w.p = c.take<T>(NT);
  w.Hp = c.take<T>(NT);
  w.coef = c.take<T>(P > 0 ? P : 0);
  w.sc = c.take<CGScal>(nf);
  w.bytes = c.off;
  return ADMP_OK;
}

template <typename T>
struct QEqCtx {
  QEqWS<T> w;
  QEqParams P;
  int nf;
  int N;
  long long Pn;
  const long long* pairs;
  const T* pos;
  const T* box;
  const T* C;
  int nc;
  cudaStream_t st;
  int atom_blocks;
};

// Hv = H v (Hv zeroed, sums of v already in sc); optional double copy.
template <typename T>
static int qeq_matvec(QEqCtx<T>& c, const T* v, T* Hv, double* hv_out) {
  const Batch& b = c.w.plan.b;
  if (c.P.flags & ADMP_QEQ_KSPACE) {
    int s = launch_recip_potential<T>(c.w.plan, c.pos, c.box, v, c.w.mesh, c.w.spec, c.w.acc, c.P.ke, Hv, c.st,
                                      nullptr, c.w.green);
    if (s) return s;
  }
  if (c.Pn > 0 && (c.P.flags & (ADMP_QEQ_RSPACE | ADMP_QEQ_DAMPING))) {
    long long blocks = (c.Pn + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    qeq_coo_spmv_kernel<T><<<(unsigned)blocks, 256, 0, c.st>>>(c.Pn, c.pairs, c.w.coef, v, Hv, c.w.sc, c.N);
  }
  qeq_finish_kernel<T><<<b.nblk_atom, 256, 0, c.st>>>(b, c.P, v, Hv, c.w.diag, c.w.zc, c.C, (long long)c.N,
                                                     c.w.sc, hv_out);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

template <typename T>
static int qeq_prepare(QEqCtx<T>& c, const T* chi, const T* hard, const T* eta, const T* shift, const T* ds,
                       const T* bs, double kappa) {
  const Batch& b = c.w.plan.b;
  ADMP_CUDA_TRY(cudaMemsetAsync(c.w.sc, 0, sizeof(CGScal) * c.nf, c.st));
  ADMP_CUDA_TRY(cudaMemsetAsync(c.w.Hp, 0, sizeof(T) * c.N * (size_t)c.nf, c.st));
  qeq_setup_kernel<T><<<b.nblk_atom, 256, 0, c.st>>>(b, c.P, c.pos, c.box, chi, hard, eta, shift, c.w.diag, c.w.zc,
                                                    c.w.chi_eff, c.w.sc);
  if (c.P.flags & ADMP_QEQ_KSPACE) {
    int s = launch_green_build<T>(c.w.plan, c.box, c.w.green, c.P.ke, c.st);
    if (s) return s;
  }
  if (c.nc > 0) {
    qeq_gram_kernel<T><<<b.nblk_atom, 256, 0, c.st>>>(b, c.nc, c.C, (long long)c.N, c.w.sc);
    qeq_gram_invert_kernel<<<(c.nf + 31) / 32, 32, 0, c.st>>>(b, c.nc, c.w.sc);
  }
  if (c.Pn > 0 && (c.P.flags & (ADMP_QEQ_RSPACE | ADMP_QEQ_DAMPING))) {
    DevError* err = scratch_error(c.st);
    long long blocks = (c.Pn + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    qeq_pair_coef_kernel<T><<<(unsigned)blocks, 256, 0, c.st>>>(c.N * c.nf, c.Pn, c.P.flags, kappa, c.P.ke, c.pairs,
                                                                ds, bs, eta, c.w.coef, err);
  }
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

template <typename T>
static int qeq_solve_impl(int flags, int nf, int N, const int* kmesh, const T* pos, const T* box, long long Pn,
                          const long long* pairs, const T* ds, const T* bs, const T* chi, const T* hard, const T* eta,
                          const T* shift, double kappa, double ke, int nc, const T* C, const double* bvals, T* q,
                          double tol, int max_iter, int* iters, double* resid, void* ws, size_t bytes,
                          cudaStream_t st) {
  QEqCtx<T> c;
  int s = qeq_carve<T>(c.w, ws, bytes, nf, N, Pn, kmesh, kappa, flags);
  if (s) return s;
  if (!ws || c.w.bytes > bytes) return fail(ADMP_ERR_WORKSPACE, "qeq workspace: need %zu bytes, got %zu", c.w.bytes, bytes);
  s = bind_plan<T>(c.w.plan, c.w.table, st);
  if (s) return s;
  c.P.flags = flags;
  c.P.axis = (flags >> 8) & 3;
  c.P.max_iter = max_iter;
  c.P.tol = tol;
  c.P.ke = ke;
  c.nf = nf;
  c.N = N;
  c.Pn = Pn;
  c.pairs = pairs;
  c.pos = pos;
  c.box = box;
  c.C = C;
  c.nc = nc;
  c.st = st;
  const Batch& b = c.w.plan.b;
  const long long NT = (long long)nf * N;
  const int sb = (nf + 63) / 64;
  s = qeq_prepare<T>(c, chi, hard, eta, shift, ds, bs, kappa);
  if (s) return s;
  double bv[4] = {0, 0, 0, 0};
  for (int k = 0; k < nc; ++k) bv[k] = bvals[k];
  qeq_set_b_kernel<<<sb, 64, 0, st>>>(nf, c.w.sc, nc, bv[0], bv[1], bv[2], bv[3]);
  // x0 (optionally projected onto C x = b)
  const int cb = (int)((NT + 255) / 256 < 2048 ? (NT + 255) / 256 : 2048);
  cast_kernel<T><<<cb > 0 ? cb : 1, 256, 0, st>>>(NT, q, c.w.x);
  if ((flags & ADMP_QEQ_PROJECT_Q0) && nc > 0) {
    qeq_sums_kernel<T, double><<<b.nblk_atom, 256, 0, st>>>(b, c.w.x, c.w.zc, C, (long long)N, nc, 1, c.w.sc, nullptr,
                                                            nullptr);
    qeq_project_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, c.w.x, C, (long long)N, c.w.sc);
    qeq_clear_acc_kernel<<<sb, 64, 0, st>>>(nf, c.w.sc);
  }
  // H x0 -> hx (double); the p buffer carries x0 in T for the matvec
  qeq_sums_kernel<T, double><<<b.nblk_atom, 256, 0, st>>>(b, c.w.x, c.w.zc, C, (long long)N, nc, 0, c.w.sc, c.w.Hp,
                                                          c.w.p);
  s = qeq_matvec<T>(c, c.w.p, c.w.Hp, c.w.hx);
  if (s) return s;
  qeq_clear_acc_kernel<<<sb, 64, 0, st>>>(nf, c.w.sc);
  ADMP_CUDA_TRY(cudaMemsetAsync(c.w.Hp, 0, sizeof(T) * NT, st));
  qeq_resid_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, c.w.hx, c.w.chi_eff, C, (long long)N, c.w.zc, c.w.r, c.w.p,
                                                   c.w.sc, 0);
  qeq_resid_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, c.w.hx, c.w.chi_eff, C, (long long)N, c.w.zc, c.w.r, c.w.p,
                                                   c.w.sc, 1);
  qeq_init_done_kernel<<<(nf + 31) / 32, 32, 0, st>>>(b, c.P, c.w.sc);
  ADMP_CUDA_TRY(cudaGetLastError());
  // iterate; read the per-frame done flags every `chunk` iterations
  RecipPlan<T> pl = c.w.plan;
  pl.b.done = &c.w.sc->done;
  pl.b.done_stride = (int)(sizeof(CGScal) / sizeof(int));
  pl.b.status_off = (int)((offsetof(CGScal, status) - offsetof(CGScal, done)) / sizeof(int));
  c.w.plan = pl;
  const int chunk = 8;
  int it = 0;
  std::vector<CGScal> h(nf);
  while (true) {
    for (int k = 0; k < chunk; ++k) {
      qeq_rotate_kernel<<<(nf + 31) / 32, 32, 0, st>>>(b, c.w.sc);
      s = qeq_matvec<T>(c, c.w.p, c.w.Hp, nullptr);
      if (s) return s;
      qeq_update_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, c.w.x, c.w.r, c.w.p, c.w.Hp, C, (long long)N, c.w.sc);
      qeq_direction_kernel<T><<<b.nblk_atom, 256, 0, st>>>(b, c.P, c.w.r, c.w.p, c.w.zc, c.w.sc);
    }
    ADMP_CUDA_TRY(cudaGetLastError());
    it += chunk;
    ADMP_CUDA_TRY(cudaMemcpyAsync(h.data(), c.w.sc, sizeof(CGScal) * nf, cudaMemcpyDeviceToHost, st));
    ADMP_CUDA_TRY(cudaStreamSynchronize(st));
    bool all = true;
    for (int f = 0; f < nf; ++f) all = all && h[f].done;
    if (all || it > max_iter + chunk) break;
  }
  cast_back_kernel<T><<<cb > 0 ? cb : 1, 256, 0, st>>>(NT, c.w.x, q);
  ADMP_CUDA_TRY(cudaGetLastError());
  int worst = ADMP_OK, worst_f = 0;
  for (int f = 0; f < nf; ++f) {
    if (iters) iters[f] = h[f].iter;
    if (resid) resid[f] = sqrt(h[f].rr_new > 0 ? h[f].rr_new : h[f].rr) / (N > 0 ? N : 1);
    const int stf = h[f].done ? h[f].status : ADMP_ERR_NOT_CONVERGED;
    if (stf && (worst == ADMP_OK || worst == ADMP_ERR_NOT_CONVERGED)) {
      worst = stf;
      worst_f = f;
    }
  }
  DevError* err = scratch_error(st);
  int e = err ? check_error(err, st) : ADMP_OK;
  if (e) return e;
  if (worst == ADMP_ERR_NOT_CONVERGED)
    return fail(ADMP_ERR_NOT_CONVERGED, "QEq CG did not converge in %d iterations (frame %d, residual %g)",
                h[worst_f].iter, worst_f, sqrt(h[worst_f].rr_new > 0 ? h[worst_f].rr_new : h[worst_f].rr) / N);
  if (worst) return fail(worst, "QEq solve failed (frame %d, status %d)", worst_f, worst);
  return ADMP_OK;
}

template <typename T>
static int qeq_hvp_impl(int flags, int nf, int N, const int* kmesh, const T* pos, const T* box, long long Pn,
                        const long long* pairs, const T* ds, const T* bs, const T* hard, const T* eta, double kappa,
                        double ke, const T* p, T* out, void* ws, size_t bytes, cudaStream_t st) {
  QEqCtx<T> c;
  int s = qeq_carve<T>(c.w, ws, bytes, nf, N, Pn, kmesh, kappa, flags);
  if (s) return s;
  if (!ws || c.w.bytes > bytes) return fail(ADMP_ERR_WORKSPACE, "qeq workspace: need %zu bytes, got %zu", c.w.bytes, bytes);
  s = bind_plan<T>(c.w.plan, c.w.table, st);
  if (s) return s;
  c.nf = nf;
  c.P.flags = flags;
  c.P.axis = (flags >> 8) & 3;
  c.P.max_iter = 0;
  c.P.tol = 0;
  c.P.ke = ke;
  c.N = N;
  c.Pn = Pn;
  c.pairs = pairs;
  c.pos = pos;
  c.box = box;
  c.C = nullptr;
  c.nc = 0;
  c.st = st;
  const Batch& b = c.w.plan.b;
  s = qeq_prepare<T>(c, nullptr, hard, eta, nullptr, ds, bs, kappa);
  if (s) return s;
  qeq_sums_kernel<T, T><<<b.nblk_atom, 256, 0, st>>>(b, p, c.w.zc, nullptr, (long long)N, 0, 0, c.w.sc, c.w.Hp,
                                                     nullptr);
  s = qeq_matvec<T>(c, p, c.w.Hp, nullptr);
  if (s) return s;
  ADMP_CUDA_TRY(cudaMemcpyAsync(out, c.w.Hp, sizeof(T) * N * (size_t)nf, cudaMemcpyDeviceToDevice, st));
  DevError* err = scratch_error(st);
  return err ? check_error(err, st) : ADMP_OK;
}

}  // namespace admp

using namespace admp;

static size_t qeq_ws_bytes(int dtype, int nframes, int natoms, long long npairs, const int* kmesh) {
  if (nframes <= 0 || nframes > kMaxBatch || natoms <= 0) return 0;
  std::vector<int> K(3 * (size_t)nframes, 1);
  if (kmesh)
    for (size_t k = 0; k < K.size(); ++k) K[k] = kmesh[k];
  const int fl = kmesh ? ADMP_QEQ_KSPACE : 0;
  if (dtype == ADMP_F32) {
    QEqWS<float> w;
    return qeq_carve<float>(w, nullptr, 0, nframes, natoms, npairs, K.data(), 1.0, fl) ? 0 : w.bytes;
  }
  QEqWS<double> w;
  return qeq_carve<double>(w, nullptr, 0, nframes, natoms, npairs, K.data(), 1.0, fl) ? 0 : w.bytes;
}

extern "C" size_t admp_qeq_workspace_size(int dtype, int natoms, long long npairs, const int* kmesh, int n_const) {
  (void)n_const;
  return qeq_ws_bytes(dtype, 1, natoms, npairs, kmesh);
}

extern "C" size_t admp_qeq_frames_workspace_size(int dtype, int nframes, int natoms, long long npairs,
                                                 const int* kmesh, int n_const) {
  (void)n_const;
  return qeq_ws_bytes(dtype, nframes, natoms, npairs, kmesh);
}

extern "C" int admp_qeq_solve_frames(int dtype, int flags, int nframes, int natoms, const int* kmesh, const void* pos,
                                     const void* box, long long npairs, const long long* pairs, const void* ds,
                                     const void* buffer_scales, const void* chi, const void* hardness,
                                     const void* eta, const void* rhs_shift, double kappa, double ke, int n_const,
                                     const void* C, const double* b, void* q, double tol, int max_iter, int* iters,
                                     double* resid, void* workspace, size_t workspace_bytes, void* stream) {
  if (nframes <= 0 || nframes > kMaxBatch)
    return fail(ADMP_ERR_BAD_ARG, "admp_qeq_solve: %d frames (1..%d)", nframes, kMaxBatch);
  if (natoms <= 0 || !pos || !box || !hardness || !q) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_solve: args");
  if (n_const < 0 || n_const > kMaxConst || (n_const > 0 && (!C || !b)))
    return fail(ADMP_ERR_BAD_ARG, "admp_qeq_solve: n_const must be in [0, %d] with C and b", kMaxConst);
  if ((flags & ADMP_QEQ_KSPACE) && (!kmesh || !(kappa > 0))) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_solve: kspace needs kmesh and kappa");
  if ((flags & ADMP_QEQ_DAMPING) && !eta) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_solve: damping needs eta");
  if (npairs > 0 && (!pairs || !ds || !buffer_scales)) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_solve: pairs");
  std::vector<int> K(3 * (size_t)nframes, 1);
  if (flags & ADMP_QEQ_KSPACE)
    for (size_t k = 0; k < K.size(); ++k) K[k] = kmesh[k];
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return qeq_solve_impl<double>(flags, nframes, natoms, K.data(), (const double*)pos, (const double*)box, npairs,
                                  pairs, (const double*)ds, (const double*)buffer_scales, (const double*)chi,
                                  (const double*)hardness, (const double*)eta, (const double*)rhs_shift, kappa, ke,
                                  n_const, (const double*)C, b, (double*)q, tol, max_iter, iters, resid, workspace,
                                  workspace_bytes, st);
  if (dtype == ADMP_F32)
    return qeq_solve_impl<float>(flags, nframes, natoms, K.data(), (const float*)pos, (const float*)box, npairs, pairs,
                                 (const float*)ds, (const float*)buffer_scales, (const float*)chi,
                                 (const float*)hardness, (const float*)eta, (const float*)rhs_shift, kappa, ke,
                                 n_const, (const float*)C, b, (float*)q, tol, max_iter, iters, resid, workspace,
                                 workspace_bytes, st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}

extern "C" int admp_qeq_solve(int dtype, int flags, int natoms, const int* kmesh, const void* pos, const void* box,
                              long long npairs, const long long* pairs, const void* ds, const void* buffer_scales,
                              const void* chi, const void* hardness, const void* eta, const void* rhs_shift,
                              double kappa, double ke, int n_const, const void* C, const double* b, void* q,
                              double tol, int max_iter, int* iters, double* resid, void* workspace,
                              size_t workspace_bytes, void* stream) {
  return admp_qeq_solve_frames(dtype, flags, 1, natoms, kmesh, pos, box, npairs, pairs, ds, buffer_scales, chi,
                               hardness, eta, rhs_shift, kappa, ke, n_const, C, b, q, tol, max_iter, iters, resid,
                               workspace, workspace_bytes, stream);
}

extern "C" int admp_qeq_hvp_frames(int dtype, int flags, int nframes, int natoms, const int* kmesh, const void* pos,
                                   const void* box, long long npairs, const long long* pairs, const void* ds,
                                   const void* buffer_scales, const void* hardness, const void* eta, double kappa,
                                   double ke, const void* p, void* out, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  if (nframes <= 0 || nframes > kMaxBatch)
    return fail(ADMP_ERR_BAD_ARG, "admp_qeq_hvp: %d frames (1..%d)", nframes, kMaxBatch);
  if (natoms <= 0 || !pos || !box || !hardness || !p || !out) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_hvp: args");
  if ((flags & ADMP_QEQ_KSPACE) && (!kmesh || !(kappa > 0))) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_hvp: kspace needs kmesh and kappa");
  if ((flags & ADMP_QEQ_DAMPING) && !eta) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_hvp: damping needs eta");
  if (npairs > 0 && (!pairs || !ds || !buffer_scales)) return fail(ADMP_ERR_BAD_ARG, "admp_qeq_hvp: pairs");
  std::vector<int> K(3 * (size_t)nframes, 1);
  if (flags & ADMP_QEQ_KSPACE)
    for (size_t k = 0; k < K.size(); ++k) K[k] = kmesh[k];
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return qeq_hvp_impl<double>(flags, nframes, natoms, K.data(), (const double*)pos, (const double*)box, npairs,
                                pairs, (const double*)ds, (const double*)buffer_scales, (const double*)hardness,
                                (const double*)eta, kappa, ke, (const double*)p, (double*)out, workspace,
                                workspace_bytes, st);
  if (dtype == ADMP_F32)
    return qeq_hvp_impl<float>(flags, nframes, natoms, K.data(), (const float*)pos, (const float*)box, npairs, pairs,
                               (const float*)ds, (const float*)buffer_scales, (const float*)hardness,
                               (const float*)eta, kappa, ke, (const float*)p, (float*)out, workspace, workspace_bytes,
                               st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}

extern "C" int admp_qeq_hvp(int dtype, int flags, int natoms, const int* kmesh, const void* pos, const void* box,
                            long long npairs, const long long* pairs, const void* ds, const void* buffer_scales,
                            const void* hardness, const void* eta, double kappa, double ke, const void* p, void* out,
                            void* workspace, size_t workspace_bytes, void* stream) {
  return admp_qeq_hvp_frames(dtype, flags, 1, natoms, kmesh, pos, box, npairs, pairs, ds, buffer_scales, hardness,
                             eta, kappa, ke, p, out, workspace, workspace_bytes, stream);
}
