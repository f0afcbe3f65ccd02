// Matrix-free projected conjugate gradient for the QEq charges.
//
// The reference minimises E(q) = site + Coulomb(PME) + damping under C q = b
// with a projected nonlinear CG and a parabolic line search (qeq.py:1374-1527)
// or LBFGS (qeq.py:1273-1371).  E is quadratic in q, so the same minimiser is
// the linear projected CG on  H q = -chi,  H = 2 diag(hardness) + J, where
//   J p = recip(p) [spread -> FFT -> G -> IFFT -> gather]
//       + sum_pairs ke s_p inv(d) (erfc(kappa d) - erfc(d / 2 eta_ij)) p_j
//       + diag(-2 kappa ke / sqrt(pi) + ke / (sqrt(pi) eta_i)) p
//       - pi ke / (V kappa^2) (sum p)                              (non-neutral)
//       + slab: pre (2 z_i sum(p z) - sum(p z^2) - z_i^2 sum p - Lz^2/6 sum p)
// The stopping rule is the reference's: ||P grad||_2 / N < tol (qeq.py:1516).
// Scalars (dots, alpha, beta, convergence) live on the device; every kernel
// skips systems whose `done` flag is set, so a batch of systems iterates in
// lock-step launches while each converges on its own.
#pragma once

#include "pme_kernels.cuh"

namespace admp {

constexpr int kMaxConst = 4;

// per-system scalar slots (double)
struct CGScal {
  double rr;          // current ||r||^2
  double rr_new;      // accumulating ||r_new||^2
  double pHp;         // p^T H p
  double Cv[kMaxConst];
  double sp, spz, spz2;  // sum p, sum p z, sum p z^2 (rank-1 terms)
  double Ginv[kMaxConst * kMaxConst];
  double b[kMaxConst];
  double pre, Lz2, nn;   // slab prefactor, Lz^2, non-neutral coefficient
  int done;
  int iter;
  int status;
  int n_const;
};

struct QEqParams {
  int flags;
  int axis;
  int max_iter;
  double tol;
  double ke;
};

template <typename T>
__device__ __forceinline__ bool sys_done(const CGScal* sc, int s) {
  return sc[s].done != 0;
}

// Constraint row c at atom i of a system (i counts within the system, so the
// frames of a multi-frame solve share one [n_const, N] matrix); a null matrix
// stands for the single all-ones row of the total-charge constraint.
template <typename T>
__device__ __forceinline__ double cval(const T* C, int c, long long cstride, int i) {
  return C ? (double)C[(long long)c * cstride + i] : 1.0;
}

// Setup per atom: diag_i, z_i, chi_eff_i; per system (block 0 thread 0 of the
// system's first block): slab / non-neutral constants.
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_setup_kernel(Batch b, QEqParams P, const T* __restrict__ pos, const T* __restrict__ box,
                     const T* __restrict__ chi, const T* __restrict__ hard, const T* __restrict__ eta,
                     const T* __restrict__ shift, double* __restrict__ diag, double* __restrict__ zc,
                     double* __restrict__ chi_eff, CGScal* __restrict__ sc) {
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const double kappa = d.kappa, ke = P.ke;
  if (threadIdx.x == 0 && blockIdx.x == d.blk_atom) {
    double bx[9], bi[9];
    load_box(box + (size_t)d.box_idx * 9, bx);
    const double V = inv3(bx, bi);
    const int ax = P.axis;
    sc[s].pre = 2.0 * kPi / V * ke;
    sc[s].Lz2 = bx[ax * 3] * bx[ax * 3] + bx[ax * 3 + 1] * bx[ax * 3 + 1] + bx[ax * 3 + 2] * bx[ax * 3 + 2];
    sc[s].nn = (P.flags & ADMP_QEQ_KSPACE) ? -kPi / (V * kappa * kappa) * ke : 0.0;
  }
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    double dg = 2.0 * (double)hard[i];
    if (P.flags & ADMP_QEQ_KSPACE) dg += -2.0 * kappa * ke / kSqrtPi;
    if (P.flags & ADMP_QEQ_DAMPING) {
      const double e = eta[i];
      dg += fabs(e) > 1e-4 ? ke / (kSqrtPi * e) : 0.0;
    }
    diag[i] = dg;
    zc[i] = pos[3 * (size_t)i + P.axis];
    chi_eff[i] = (chi ? (double)chi[i] : 0.0) + (shift ? (double)shift[i] : 0.0);
  }
}

// Gram matrix C C^T per system (accumulated into Ginv slots, inverted later).
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_gram_kernel(Batch b, int nc, const T* __restrict__ C, long long cstride, CGScal* __restrict__ sc) {
  __shared__ double red[16 * 32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  double v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = 0.0;
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    for (int r = 0; r < nc; ++r)
      for (int c = 0; c < nc; ++c) v[r * kMaxConst + c] += cval(C, r, cstride, i - d.atom_off) * cval(C, c, cstride, i - d.atom_off);
  }
  block_atomic_sum<16>(v, sc[s].Ginv, red);
}

// Invert the Gram matrices (one thread per system, Gauss-Jordan).
static __global__ void qeq_gram_invert_kernel(Batch b, int nc, CGScal* __restrict__ sc) {
  const int s0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (s0 >= b.nsys) return;
  const int s = b.s[s0].box_idx;
  double a[kMaxConst][2 * kMaxConst];
  for (int r = 0; r < nc; ++r)
    for (int c = 0; c < 2 * nc; ++c) a[r][c] = c < nc ? sc[s].Ginv[r * kMaxConst + c] : (c - nc == r ? 1.0 : 0.0);
  for (int c = 0; c < nc; ++c) {
    int piv = c;
    for (int r = c + 1; r < nc; ++r)
      if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
    for (int k = 0; k < 2 * nc; ++k) {
      double t = a[c][k];
      a[c][k] = a[piv][k];
      a[piv][k] = t;
    }
    const double inv = a[c][c] != 0.0 ? 1.0 / a[c][c] : 0.0;
    if (a[c][c] == 0.0) sc[s].status = ADMP_ERR_BAD_ARG;
    for (int k = 0; k < 2 * nc; ++k) a[c][k] *= inv;
    for (int r = 0; r < nc; ++r)
      if (r != c) {
        const double f = a[r][c];
        for (int k = 0; k < 2 * nc; ++k) a[r][k] -= f * a[c][k];
      }
  }
  for (int k = 0; k < kMaxConst * kMaxConst; ++k) sc[s].Ginv[k] = 0.0;
  for (int r = 0; r < nc; ++r)
    for (int c = 0; c < nc; ++c) sc[s].Ginv[r * kMaxConst + c] = a[r][nc + c];
  sc[s].n_const = nc;
}

// sums for rank-1 terms and C v (cv_slot) of a vector v; optional copy to vt.
template <typename T, typename V>
__global__ void __launch_bounds__(256)
    qeq_sums_kernel(Batch b, const V* __restrict__ v, const double* __restrict__ zc, const T* __restrict__ C,
                    long long cstride, int nc, int want_cv, CGScal* __restrict__ sc, T* __restrict__ hv_zero,
                    T* __restrict__ vt) {
  __shared__ double red[7 * 32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  if (sys_done<T>(sc, s)) return;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    const double x = (double)v[i];
    const double z = zc[i];
    acc[0] += x;
    acc[1] += x * z;
    acc[2] += x * z * z;
    if (want_cv)
      for (int c = 0; c < nc; ++c) acc[3 + c] += cval(C, c, cstride, i - d.atom_off) * x;
    if (hv_zero) hv_zero[i] = T(0);
    if (vt) vt[i] = (T)x;
  }
  double* dst = want_cv ? &sc[s].sp : &sc[s].sp;
  double a3[3] = {acc[0], acc[1], acc[2]};
  block_atomic_sum<3>(a3, dst, red);
  if (want_cv) {
    double a4[4] = {acc[3], acc[4], acc[5], acc[6]};
    block_atomic_sum<4>(a4, sc[s].Cv, red);
  }
}

// COO pair coefficients of J (drop-in list; pairs with scale 0 get 0).
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_pair_coef_kernel(int N, long long Pn, int flags, double kappa, double ke, const long long* __restrict__ pairs,
                         const T* __restrict__ ds, const T* __restrict__ bs, const T* __restrict__ eta,
                         T* __restrict__ coef, DevError* err) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < Pn; p += (long long)gridDim.x * blockDim.x) {
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    double c = 0.0;
    if (i < 0 || i >= N || j < 0 || j >= N) {
      report_error(err, ADMP_ERR_BAD_INDEX, 5, p);
    } else {
      const double dd = ds[p], s = bs[p];
      const double inv = fabs(dd) > 1e-4 ? 1.0 / dd : 0.0;
      if (s != 0.0 && inv != 0.0) {
        if (flags & ADMP_QEQ_RSPACE) c += erfc(kappa * dd);
        if (flags & ADMP_QEQ_DAMPING) {
          const double ei = eta[i], ej = eta[j];
          double eij = sqrt((ei * ei + ej * ej) / 2.0);
          if (eij == 0.0) eij = 1e-10;
          c -= erfc(dd / (2.0 * eij));
        }
        c *= ke * s * inv;
      }
    }
    coef[p] = (T)c;
  }
}

// Hv[i] += c_p v[j], Hv[j] += c_p v[i]  (COO over the frames of a batch:
// atom i belongs to frame i / natoms, whose CG state is sc[i / natoms])
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_coo_spmv_kernel(long long Pn, const long long* __restrict__ pairs, const T* __restrict__ coef,
                        const T* __restrict__ v, T* __restrict__ Hv, const CGScal* __restrict__ sc, int natoms) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < Pn; p += (long long)gridDim.x * blockDim.x) {
    const T c = coef[p];
    if (c == T(0)) continue;
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    if (sc[i / natoms].done) continue;
    atomicAdd(Hv + i, c * v[j]);
    atomicAdd(Hv + j, c * v[i]);
  }
}

// Hv += diag v + rank-1 terms; accumulate p^T Hv and C Hv.
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_finish_kernel(Batch b, QEqParams P, const T* __restrict__ v, T* __restrict__ Hv,
                      const double* __restrict__ diag, const double* __restrict__ zc, const T* __restrict__ C,
                      long long cstride, CGScal* __restrict__ sc, double* __restrict__ hv_out) {
  __shared__ double red[5 * 32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  if (sc[s].done) return;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const CGScal& S = sc[s];
  const double sp = S.sp, spz = S.spz, spz2 = S.spz2;
  const bool slab = (P.flags & ADMP_QEQ_SLAB) != 0;
  const int nc = S.n_const;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    const double x = (double)v[i];
    double h = (double)Hv[i] + diag[i] * x + S.nn * sp;
    if (slab) {
      const double z = zc[i];
      h += S.pre * (2.0 * z * spz - spz2 - z * z * sp - S.Lz2 / 6.0 * sp);
    }
    Hv[i] = (T)h;
    if (hv_out) hv_out[i] = h;
    acc[0] += x * h;
    for (int c = 0; c < nc; ++c) acc[1 + c] += cval(C, c, cstride, i - d.atom_off) * h;
  }
  double a1v[1] = {acc[0]};
  block_atomic_sum<1>(a1v, &sc[s].pHp, red);
  if (nc > 0) {
    double a4[4] = {acc[1], acc[2], acc[3], acc[4]};
    block_atomic_sum<4>(a4, sc[s].Cv, red);
  }
}

// x += alpha p ; r -= alpha P(Hp) ; rr_new += r^2 ; zero sp/spz/spz2.
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_update_kernel(Batch b, double* __restrict__ x, double* __restrict__ r, const T* __restrict__ p,
                      T* __restrict__ Hp, const T* __restrict__ C, long long cstride, CGScal* __restrict__ sc) {
  __shared__ double red[32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  if (sc[s].done) return;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const CGScal& S = sc[s];
  const int nc = S.n_const;
  const double alpha = S.pHp != 0.0 ? S.rr / S.pHp : 0.0;
  double lam[kMaxConst] = {0, 0, 0, 0};
  for (int r0 = 0; r0 < nc; ++r0)
    for (int c = 0; c < nc; ++c) lam[r0] += S.Ginv[r0 * kMaxConst + c] * S.Cv[c];
  double acc = 0.0;
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    double w = (double)Hp[i];
    Hp[i] = T(0);
    for (int c = 0; c < nc; ++c) w -= cval(C, c, cstride, i - d.atom_off) * lam[c];
    x[i] += alpha * (double)p[i];
    const double rn = r[i] - alpha * w;
    r[i] = rn;
    acc += rn * rn;
  }
  double v[1] = {acc};
  block_atomic_sum<1>(v, &sc[s].rr_new, red);
  if (threadIdx.x == 0 && blockIdx.x == d.blk_atom) {
    sc[s].sp = 0.0;
    sc[s].spz = 0.0;
    sc[s].spz2 = 0.0;
  }
}

// convergence check and p = r + beta p ; sums of the new p.
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_direction_kernel(Batch b, QEqParams P, const double* __restrict__ r, T* __restrict__ p,
                         const double* __restrict__ zc, CGScal* __restrict__ sc) {
  __shared__ double red[3 * 32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  if (sc[s].done) return;
  const CGScal& S = sc[s];
  const double rrn = S.rr_new;
  const bool conv = sqrt(rrn) / (double)(d.natoms > 0 ? d.natoms : 1) < P.tol;
  if (conv || S.iter >= P.max_iter) {
    if (threadIdx.x == 0) {
      sc[s].status = conv ? ADMP_OK : ADMP_ERR_NOT_CONVERGED;
      sc[s].done = 1;
    }
    return;
  }
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const double beta = S.rr != 0.0 ? rrn / S.rr : 0.0;
  double acc[3] = {0, 0, 0};
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    const double pn = r[i] + beta * (double)p[i];
    p[i] = (T)pn;
    const double z = zc[i];
    acc[0] += pn;
    acc[1] += pn * z;
    acc[2] += pn * z * z;
  }
  block_atomic_sum<3>(acc, &sc[s].sp, red);
}

// Start of an iteration: rotate scalars (rr <- rr_new), zero accumulators.
static __global__ void qeq_rotate_kernel(Batch b, CGScal* __restrict__ sc) {
  const int s0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (s0 >= b.nsys) return;
  const int s = b.s[s0].box_idx;
  if (sc[s].done) return;
  sc[s].rr = sc[s].rr_new;
  sc[s].rr_new = 0.0;
  sc[s].pHp = 0.0;
  for (int c = 0; c < kMaxConst; ++c) sc[s].Cv[c] = 0.0;
  sc[s].iter += 1;
}

// x0 <- x0 + C^T Ginv (b - C x0)   (vector_projection, utils.py:175-210)
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_project_kernel(Batch b, double* __restrict__ x, const T* __restrict__ C, long long cstride,
                       const CGScal* __restrict__ sc) {
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  const CGScal& S = sc[s];
  const int nc = S.n_const;
  double lam[kMaxConst] = {0, 0, 0, 0};
  for (int r0 = 0; r0 < nc; ++r0)
    for (int c = 0; c < nc; ++c) lam[r0] += S.Ginv[r0 * kMaxConst + c] * (S.b[c] - S.Cv[c]);
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    double v = x[i];
    for (int c = 0; c < nc; ++c) v += cval(C, c, cstride, i - d.atom_off) * lam[c];
    x[i] = v;
  }
}

// g = chi_eff + Hx (already in hv) -> r = -P g ; p = r ; rr ; sums of p.
template <typename T>
__global__ void __launch_bounds__(256)
    qeq_resid_kernel(Batch b, const double* __restrict__ hx, const double* __restrict__ chi_eff,
                     const T* __restrict__ C, long long cstride, const double* __restrict__ zc,
                     double* __restrict__ r, T* __restrict__ p, CGScal* __restrict__ sc, int pass) {
  __shared__ double red[4 * 32];
  const int s0 = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s0];
  const int s = d.box_idx;
  const CGScal& S = sc[s];
  const int nc = S.n_const;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  if (pass == 0) {  // accumulate C g
    double acc[4] = {0, 0, 0, 0};
    for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
      const int i = d.atom_off + a;
      const double g = chi_eff[i] + hx[i];
      for (int c = 0; c < nc; ++c) acc[c] += cval(C, c, cstride, i - d.atom_off) * g;
    }
    if (nc > 0) block_atomic_sum<4>(acc, sc[s].Cv, red);
    return;
  }
  double lam[kMaxConst] = {0, 0, 0, 0};
  for (int r0 = 0; r0 < nc; ++r0)
    for (int c = 0; c < nc; ++c) lam[r0] += S.Ginv[r0 * kMaxConst + c] * S.Cv[c];
  double acc[4] = {0, 0, 0, 0};
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    double g = chi_eff[i] + hx[i];
    for (int c = 0; c < nc; ++c) g -= cval(C, c, cstride, i - d.atom_off) * lam[c];
    const double rv = -g;
    r[i] = rv;
    p[i] = (T)rv;
    const double z = zc[i];
    acc[0] += rv * rv;
    acc[1] += rv;
    acc[2] += rv * z;
    acc[3] += rv * z * z;
  }
  double a1v[1] = {acc[0]};
  block_atomic_sum<1>(a1v, &sc[s].rr_new, red);
  double a3[3] = {acc[1], acc[2], acc[3]};
  block_atomic_sum<3>(a3, &sc[s].sp, red);
}

// Constraint values b (shared by every system of the batch) and their count.
static __global__ void qeq_set_b_kernel(int nsys, CGScal* __restrict__ sc, int nc, double b0, double b1, double b2,
                                        double b3) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  sc[s].b[0] = b0;
  sc[s].b[1] = b1;
  sc[s].b[2] = b2;
  sc[s].b[3] = b3;
  sc[s].n_const = nc;
}

// Zero the CG accumulators (rr .. spz2) of every system, keeping Ginv, b and
// the per-system constants.
static __global__ void qeq_clear_acc_kernel(int nsys, CGScal* __restrict__ sc) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys) return;
  CGScal& S = sc[s];
  S.rr = 0.0;
  S.rr_new = 0.0;
  S.pHp = 0.0;
  for (int c = 0; c < kMaxConst; ++c) S.Cv[c] = 0.0;
  S.sp = 0.0;
  S.spz = 0.0;
  S.spz2 = 0.0;
}

template <typename T>
__global__ void cast_kernel(long long n, const T* __restrict__ in, double* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

template <typename T>
__global__ void cast_back_kernel(long long n, const double* __restrict__ in, T* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (T)in[i];
}

static __global__ void qeq_init_done_kernel(Batch b, QEqParams P, CGScal* __restrict__ sc) {
  const int s0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (s0 >= b.nsys) return;
  const int s = b.s[s0].box_idx;
  const double n = b.s[s0].natoms > 0 ? b.s[s0].natoms : 1;
  sc[s].rr = sc[s].rr_new;
  sc[s].iter = 0;
  for (int c = 0; c < kMaxConst; ++c) sc[s].Cv[c] = 0.0;
  sc[s].pHp = 0.0;
  if (sqrt(sc[s].rr) / n < P.tol || P.max_iter <= 0) {
    sc[s].done = 1;
    sc[s].status = sqrt(sc[s].rr) / n < P.tol ? ADMP_OK : ADMP_ERR_NOT_CONVERGED;
  }
}

}  // namespace admp
