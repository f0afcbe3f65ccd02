// Pair-list and per-atom terms of the drop-in path.
//   admp_pair_energy      pme.py:312-349 (Ewald real), pme.py:529-561 (OBC),
//                         qeq.py:104-119 (Gaussian damping pair part)
//   admp_atom_terms       pme.py:448-527 (self, non-neutral, slab),
//                         qeq.py:121-126 (damping self), qeq.py:159-209 (site)
//   admp_pair_distances   nblist.py:517-551 with spatial.py:15-36
#include "admp_common.cuh"
#include "runtime.h"

namespace admp {

template <typename T, int MODE>
__global__ void __launch_bounds__(256)
    pair_list_kernel(int N, long long P, const long long* __restrict__ pairs, const T* __restrict__ ds,
                     const T* __restrict__ bs, const T* __restrict__ q, const T* __restrict__ eta, T kappa,
                     T ke, double* __restrict__ energy, T* __restrict__ dE_dds, T* __restrict__ dE_dq,
                     T* __restrict__ dE_deta, DevError* err) {
  __shared__ double red[32];
  const int f = blockIdx.y;
  pairs += (size_t)f * P * 2;
  ds += (size_t)f * P;
  bs += (size_t)f * P;
  q += (size_t)f * N;
  if (eta) eta += (size_t)f * N;
  if (dE_dds) dE_dds += (size_t)f * P;
  if (dE_dq) dE_dq += (size_t)f * N;
  if (dE_deta) dE_deta += (size_t)f * N;
  const T two_over_sqrtpi = T(2.0 / kSqrtPi);
  double e = 0.0;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    if (i < 0 || i >= N || j < 0 || j >= N) {
      report_error(err, ADMP_ERR_BAD_INDEX, 1, p);
      continue;
    }
    const T d = ds[p], s = bs[p];
    const T qi = q[i], qj = q[j];
    const T thr = MODE == ADMP_PAIR_OBC ? T(1e-8) : T(1e-4);
    const bool valid = fabs((double)d) > (double)thr;
    const T inv = valid ? T(1) / d : T(0);
    T ep, dd, c;
    if (MODE == ADMP_PAIR_EWALD) {
      const T x = kappa * d;
      const T er = erfc_t(x);
      ep = er * qi * qj * inv * s * ke;
      dd = valid ? (-two_over_sqrtpi * kappa * exp_t(-x * x) * inv - er * inv * inv) * qi * qj * s * ke : T(0);
      c = er * inv * s * ke;
    } else if (MODE == ADMP_PAIR_OBC) {
      ep = qi * qj * ke * inv * s;
      dd = valid ? -qi * qj * ke * inv * inv * s : T(0);
      c = ke * inv * s;
    } else {
      const T ei = eta[i], ej = eta[j];
      const T eij = sqrt_t((ei * ei + ej * ej) / T(2));
      const bool zero = eij == T(0);
      const T eijs = zero ? T(1e-10) : eij;
      const T x = d / (T(2) * eijs);
      const T er = erfc_t(x);
      const T ge = two_over_sqrtpi * exp_t(-x * x);
      ep = -er * qi * qj * inv * s * ke;
      dd = valid ? (ge / (T(2) * eijs) * inv + er * inv * inv) * qi * qj * s * ke : T(0);
      c = -er * inv * s * ke;
      if (dE_deta && !zero) {
        const T deij = -ge * d / (T(2) * eijs * eijs) * qi * qj * inv * s * ke;
        atomicAdd(dE_deta + i, deij * ei / (T(2) * eijs));
        atomicAdd(dE_deta + j, deij * ej / (T(2) * eijs));
      }
    }
    e += (double)ep;
    if (dE_dds) dE_dds[p] += dd;
    if (dE_dq && c != T(0)) {
      atomicAdd(dE_dq + i, c * qj);
      atomicAdd(dE_dq + j, c * qi);
    }
  }
  double v[1] = {e};
  if (energy) block_atomic_sum<1>(v, energy + f, red);
}

template <typename T>
__global__ void __launch_bounds__(512)
    atom_terms_kernel(int flags, int N, const T* __restrict__ pos, const T* __restrict__ box,
                      const T* __restrict__ q, const T* __restrict__ eta, const T* __restrict__ chi,
                      const T* __restrict__ hard, double kappa, double ke, double* __restrict__ energy,
                      double* __restrict__ terms, T* __restrict__ dq, T* __restrict__ dpos,
                      T* __restrict__ dbox, T* __restrict__ deta, T* __restrict__ dchi,
                      T* __restrict__ dhard) {
  __shared__ double red[6 * 32];
  __shared__ double sums[6];
  __shared__ double geo[20];  // box 9, binv 9, V, Lz
  const int f = blockIdx.x;
  const int axis = (flags >> 8) & 3;
  q += (size_t)f * N;
  if (pos) pos += (size_t)f * N * 3;
  if (eta) eta += (size_t)f * N;
  if (chi) chi += (size_t)f * N;
  if (hard) hard += (size_t)f * N;
  if (threadIdx.x < 6) sums[threadIdx.x] = 0.0;
  if (threadIdx.x == 0 && box) {
    double b[9], bi[9];
    load_box(box + (size_t)f * 9, b);
    double V = inv3(b, bi);
    for (int k = 0; k < 9; ++k) {
      geo[k] = b[k];
      geo[9 + k] = bi[k];
    }
    geo[18] = V;
    geo[19] = sqrt(b[axis * 3] * b[axis * 3] + b[axis * 3 + 1] * b[axis * 3 + 1] + b[axis * 3 + 2] * b[axis * 3 + 2]);
  }
  __syncthreads();
  // pass 1: Q, sum q^2, Mz, sum q z^2, damping self, site
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double qi = q[i];
    v[0] += qi;
    v[1] += qi * qi;
    if (flags & ADMP_TERM_SLAB) {
      const double z = pos[3 * (size_t)i + axis];
      v[2] += qi * z;
      v[3] += qi * z * z;
    }
    if (flags & ADMP_TERM_DAMP_SELF) {
      const double e = eta[i];
      const double einv = fabs(e) > 1e-4 ? 1.0 / e : 0.0;
      v[4] += einv / (2.0 * kSqrtPi) * qi * qi;
    }
    if (flags & ADMP_TERM_SITE) v[5] += (double)chi[i] * qi + (double)hard[i] * qi * qi;
  }
  block_atomic_sum<6>(v, sums, red);
  const double Q = sums[0], Sq2 = sums[1], Mz = sums[2], Sz2 = sums[3];
  double Eself = 0, Enn = 0, Eslab = 0, Eds = 0, Esite = 0, pre = 0, V = 0, Lz = 0;
  if (flags & ADMP_TERM_SELF) Eself = -ke * kappa / kSqrtPi * Sq2;
  if (box) {
    V = geo[18];
    Lz = geo[19];
  }
  if (flags & ADMP_TERM_NON_NEUTRAL) Enn = -kPi / (2.0 * V * kappa * kappa) * ke * Q * Q;
  if (flags & ADMP_TERM_SLAB) {
    pre = 2.0 * kPi / V * ke;
    Eslab = pre * (Mz * Mz - Q * Sz2 - Q * Q * Lz * Lz / 12.0);
  }
  if (flags & ADMP_TERM_DAMP_SELF) Eds = ke * sums[4];
  if (flags & ADMP_TERM_SITE) Esite = sums[5];
  if (threadIdx.x == 0) {
    if (energy) energy[f] += Eself + Enn + Eslab + Eds + Esite;
    if (terms) {
      terms[f * 5 + 0] += Eself;
      terms[f * 5 + 1] += Enn;
      terms[f * 5 + 2] += Eslab;
      terms[f * 5 + 3] += Eds;
      terms[f * 5 + 4] += Esite;
    }
    if (dbox) {
      double g[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const double Ev = Enn + Eslab;  // both scale as 1/V: dE/dbox = -E B^T
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) g[i * 3 + j] = -Ev * geo[9 + j * 3 + i];
      if ((flags & ADMP_TERM_SLAB) && Lz > 0) {
        const double dLz = pre * (-Q * Q * 2.0 * Lz / 12.0);
        for (int j = 0; j < 3; ++j) g[axis * 3 + j] += dLz * geo[axis * 3 + j] / Lz;
      }
      for (int k = 0; k < 9; ++k) dbox[(size_t)f * 9 + k] += (T)g[k];
    }
  }
  // pass 2: per-atom gradients
  const double cself = (flags & ADMP_TERM_SELF) ? -2.0 * ke * kappa / kSqrtPi : 0.0;
  const double cnn = (flags & ADMP_TERM_NON_NEUTRAL) ? -kPi / (V * kappa * kappa) * ke * Q : 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const double qi = q[i];
    double g = cself * qi + cnn;
    if (flags & ADMP_TERM_SLAB) {
      const double z = pos[3 * (size_t)i + axis];
      g += pre * (2.0 * Mz * z - Sz2 - Q * z * z - Q * Lz * Lz / 6.0);
      if (dpos) dpos[((size_t)f * N + i) * 3 + axis] += (T)(pre * (2.0 * Mz * qi - 2.0 * Q * qi * z));
    }
    if (flags & ADMP_TERM_DAMP_SELF) {
      const double e = eta[i];
      const bool ok = fabs(e) > 1e-4;
      const double einv = ok ? 1.0 / e : 0.0;
      g += ke * qi * einv / kSqrtPi;
      if (deta) deta[(size_t)f * N + i] += (T)(ok ? -ke * qi * qi / (2.0 * kSqrtPi) * einv * einv : 0.0);
    }
    if (flags & ADMP_TERM_SITE) {
      g += (double)chi[i] + 2.0 * (double)hard[i] * qi;
      if (dchi) dchi[(size_t)f * N + i] += (T)qi;
      if (dhard) dhard[(size_t)f * N + i] += (T)(qi * qi);
    }
    if (dq) dq[(size_t)f * N + i] += (T)g;
  }
}

template <typename T>
__device__ __forceinline__ void min_image(const double* b, const double* bi, double* dr, double* nimg) {
  double f[3];
#pragma unroll
  for (int e = 0; e < 3; ++e) f[e] = dr[0] * bi[0 * 3 + e] + dr[1] * bi[1 * 3 + e] + dr[2] * bi[2 * 3 + e];
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    nimg[e] = floor(f[e] + 0.5);
    f[e] -= nimg[e];
  }
#pragma unroll
  for (int e = 0; e < 3; ++e) dr[e] = f[0] * b[0 * 3 + e] + f[1] * b[1 * 3 + e] + f[2] * b[2 * 3 + e];
}

template <typename T>
__global__ void __launch_bounds__(256)
    pair_dist_kernel(int pbc, int N, long long P, const long long* __restrict__ pairs,
                     const T* __restrict__ pos, const T* __restrict__ box, T* __restrict__ ds,
                     DevError* err) {
  __shared__ double geo[18];
  if (threadIdx.x == 0 && pbc) {
    load_box(box, geo);
    inv3(geo, geo + 9);
  }
  __syncthreads();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    if (i < 0 || i >= N || j < 0 || j >= N) {
      report_error(err, ADMP_ERR_BAD_INDEX, 2, p);
      ds[p] = T(0);
      continue;
    }
    double dr[3], n[3];
    if (pbc) {
      for (int e = 0; e < 3; ++e) dr[e] = (double)pos[3 * i + e] - (double)pos[3 * j + e];
      min_image<T>(geo, geo + 9, dr, n);
    } else {
      for (int e = 0; e < 3; ++e) dr[e] = (double)pos[3 * j + e] - (double)pos[3 * i + e];
    }
    ds[p] = (T)sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
  }
}

template <typename T>
__global__ void __launch_bounds__(256)
    pair_dist_bwd_kernel(int pbc, int N, long long P, const long long* __restrict__ pairs,
                         const T* __restrict__ pos, const T* __restrict__ box, const T* __restrict__ g,
                         T* __restrict__ gpos, T* __restrict__ gbox, DevError* err) {
  __shared__ double geo[18];
  __shared__ double red[9 * 32];
  if (threadIdx.x == 0 && pbc) {
    load_box(box, geo);
    inv3(geo, geo + 9);
  }
  __syncthreads();
  double vb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P;
       p += (long long)gridDim.x * blockDim.x) {
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    if (i < 0 || i >= N || j < 0 || j >= N) {
      report_error(err, ADMP_ERR_BAD_INDEX, 3, p);
      continue;
    }
    const double gp = g[p];
    if (gp == 0.0) continue;
    double dr[3], n[3] = {0, 0, 0};
    if (pbc) {
      for (int e = 0; e < 3; ++e) dr[e] = (double)pos[3 * i + e] - (double)pos[3 * j + e];
      min_image<T>(geo, geo + 9, dr, n);
    } else {
      for (int e = 0; e < 3; ++e) dr[e] = (double)pos[3 * j + e] - (double)pos[3 * i + e];
    }
    const double d = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    if (d == 0.0) continue;
    const double s = gp / d;
    const long long a = pbc ? i : j, c = pbc ? j : i;
    for (int e = 0; e < 3; ++e) {
      const double v = s * dr[e];
      if (gpos) {
        atomicAdd(gpos + 3 * a + e, (T)v);
        atomicAdd(gpos + 3 * c + e, (T)(-v));
      }
      if (pbc)
        for (int k = 0; k < 3; ++k) vb[k * 3 + e] -= n[k] * v;
    }
  }
  if (pbc && gbox) {
    __shared__ double out[9];
    if (threadIdx.x < 9) out[threadIdx.x] = 0.0;
    __syncthreads();
    block_atomic_sum<9>(vb, out, red);
    if (threadIdx.x < 9 && out[threadIdx.x] != 0.0) atomicAdd(gbox + threadIdx.x, (T)out[threadIdx.x]);
  }
}

// ------------------------------------------------------------------ host side
template <typename T>
static int pair_energy_impl(int mode, int nf, int N, long long P, const long long* pairs, const void* ds,
                            const void* bs, const void* q, const void* eta, double kappa, double ke,
                            double* energy, void* dds, void* dq, void* deta, cudaStream_t st) {
  if (P == 0 || nf == 0) return ADMP_OK;
  DevError* err = scratch_error(st);
  if (!err) return ADMP_ERR_CUDA;
  long long blocks = (P + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  dim3 grid((unsigned)blocks, (unsigned)nf);
  const T* tds = (const T*)ds;
  const T* tbs = (const T*)bs;
  const T* tq = (const T*)q;
  const T* te = (const T*)eta;
  switch (mode) {
    case ADMP_PAIR_EWALD:
      pair_list_kernel<T, ADMP_PAIR_EWALD><<<grid, 256, 0, st>>>(N, P, pairs, tds, tbs, tq, te, (T)kappa, (T)ke,
                                                                  energy, (T*)dds, (T*)dq, (T*)deta, err);
      break;
    case ADMP_PAIR_OBC:
      pair_list_kernel<T, ADMP_PAIR_OBC><<<grid, 256, 0, st>>>(N, P, pairs, tds, tbs, tq, te, (T)kappa, (T)ke,
                                                                energy, (T*)dds, (T*)dq, (T*)deta, err);
      break;
    default:
      pair_list_kernel<T, ADMP_PAIR_DAMPING><<<grid, 256, 0, st>>>(N, P, pairs, tds, tbs, tq, te, (T)kappa,
                                                                    (T)ke, energy, (T*)dds, (T*)dq, (T*)deta, err);
  }
  ADMP_CUDA_TRY(cudaGetLastError());
  return check_error(err, st);
}

}  // namespace admp

using namespace admp;

extern "C" int admp_pair_energy(int dtype, int mode, int nframes, int natoms, long long npairs,
                                const long long* pairs, const void* ds, const void* buffer_scales,
                                const void* q, const void* eta, double kappa, double ke, double* energy,
                                void* dE_dds, void* dE_dq, void* dE_deta, void* stream) {
  if (mode < 0 || mode > 2 || nframes < 0 || natoms < 0 || npairs < 0) return fail(ADMP_ERR_BAD_ARG, "admp_pair_energy: bad mode/sizes");
  if (npairs > 0 && (!pairs || !ds || !buffer_scales || !q)) return fail(ADMP_ERR_BAD_ARG, "admp_pair_energy: null input");
  if (mode == ADMP_PAIR_DAMPING && npairs > 0 && !eta) return fail(ADMP_ERR_BAD_ARG, "admp_pair_energy: damping needs eta");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return pair_energy_impl<double>(mode, nframes, natoms, npairs, pairs, ds, buffer_scales, q, eta, kappa, ke,
                                    energy, dE_dds, dE_dq, dE_deta, st);
  if (dtype == ADMP_F32)
    return pair_energy_impl<float>(mode, nframes, natoms, npairs, pairs, ds, buffer_scales, q, eta, kappa, ke,
                                   energy, dE_dds, dE_dq, dE_deta, st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}

extern "C" int admp_atom_terms(int dtype, int flags, int nframes, int natoms, const void* pos, const void* box,
                               const void* q, const void* eta, const void* chi, const void* hardness,
                               double kappa, double ke, double* energy, double* terms, void* dE_dq,
                               void* dE_dpos, void* dE_dbox, void* dE_deta, void* dE_dchi, void* dE_dhard,
                               void* stream) {
  if (nframes <= 0 || natoms < 0) return nframes == 0 ? ADMP_OK : fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: sizes");
  if (!q) return fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: q is null");
  if ((flags & (ADMP_TERM_NON_NEUTRAL | ADMP_TERM_SLAB)) && !box) return fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: box needed");
  if ((flags & ADMP_TERM_SLAB) && !pos) return fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: pos needed");
  if ((flags & ADMP_TERM_DAMP_SELF) && !eta) return fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: eta needed");
  if ((flags & ADMP_TERM_SITE) && (!chi || !hardness)) return fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: chi/hardness needed");
  if (((flags >> 8) & 3) > 2) return fail(ADMP_ERR_BAD_ARG, "admp_atom_terms: slab axis");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64) {
    atom_terms_kernel<double><<<nframes, 512, 0, st>>>(flags, natoms, (const double*)pos, (const double*)box,
                                                       (const double*)q, (const double*)eta, (const double*)chi,
                                                       (const double*)hardness, kappa, ke, energy, terms,
                                                       (double*)dE_dq, (double*)dE_dpos, (double*)dE_dbox,
                                                       (double*)dE_deta, (double*)dE_dchi, (double*)dE_dhard);
  } else if (dtype == ADMP_F32) {
    atom_terms_kernel<float><<<nframes, 512, 0, st>>>(flags, natoms, (const float*)pos, (const float*)box,
                                                      (const float*)q, (const float*)eta, (const float*)chi,
                                                      (const float*)hardness, kappa, ke, energy, terms,
                                                      (float*)dE_dq, (float*)dE_dpos, (float*)dE_dbox,
                                                      (float*)dE_deta, (float*)dE_dchi, (float*)dE_dhard);
  } else {
    return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  }
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

extern "C" int admp_pair_distances(int dtype, int pbc, int natoms, long long npairs, const long long* pairs,
                                   const void* pos, const void* box, void* ds, void* stream) {
  if (npairs == 0) return ADMP_OK;
  if (npairs < 0 || !pairs || !pos || !ds || (pbc && !box)) return fail(ADMP_ERR_BAD_ARG, "admp_pair_distances: args");
  cudaStream_t st = (cudaStream_t)stream;
  DevError* err = scratch_error(st);
  if (!err) return ADMP_ERR_CUDA;
  long long blocks = (npairs + 255) / 256;
  if (blocks > 8192) blocks = 8192;
  if (dtype == ADMP_F64)
    pair_dist_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(pbc, natoms, npairs, pairs, (const double*)pos,
                                                               (const double*)box, (double*)ds, err);
  else if (dtype == ADMP_F32)
    pair_dist_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(pbc, natoms, npairs, pairs, (const float*)pos,
                                                              (const float*)box, (float*)ds, err);
  else
    return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  ADMP_CUDA_TRY(cudaGetLastError());
  return check_error(err, st);
}

extern "C" int admp_pair_distances_backward(int dtype, int pbc, int natoms, long long npairs,
                                            const long long* pairs, const void* pos, const void* box,
                                            const void* grad_ds, void* grad_pos, void* grad_box, void* stream) {
  if (npairs == 0) return ADMP_OK;
  if (npairs < 0 || !pairs || !pos || !grad_ds || (pbc && !box)) return fail(ADMP_ERR_BAD_ARG, "admp_pair_distances_backward: args");
  cudaStream_t st = (cudaStream_t)stream;
  DevError* err = scratch_error(st);
  if (!err) return ADMP_ERR_CUDA;
  long long blocks = (npairs + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  if (dtype == ADMP_F64)
    pair_dist_bwd_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(pbc, natoms, npairs, pairs, (const double*)pos,
                                                                   (const double*)box, (const double*)grad_ds,
                                                                   (double*)grad_pos, (double*)grad_box, err);
  else if (dtype == ADMP_F32)
    pair_dist_bwd_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(pbc, natoms, npairs, pairs, (const float*)pos,
                                                                  (const float*)box, (const float*)grad_ds,
                                                                  (float*)grad_pos, (float*)grad_box, err);
  else
    return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  ADMP_CUDA_TRY(cudaGetLastError());
  return check_error(err, st);
}
