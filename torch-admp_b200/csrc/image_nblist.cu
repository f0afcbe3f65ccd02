// Neighbour list over periodic images, for cutoffs above half the box
// (the pair set of dp_nblist, nblist.py:33-93 and make_local_pairs /
// make_ds, nblist.py:173-240): every periodic image j + n.B of atom j within
// rc of atom i gives one pair (i, j) with i < j (buffer scale 1), and every
// image i + n.B (n != 0) of atom i itself gives a pair (i, i) (scale 1/2);
// the pair distances are |r_j - r_i + n.B| with the image shift n stored per
// pair, so they are differentiable in the positions and the box.
//
// Atoms are wrapped into the cell for the search (fractional coordinates
// mod 1); the stored shift refers to the caller's unwrapped positions.  With
// wrapped coordinates |f_j - f_i| < 1, so images |n_d| <= ceil(rc / h_d) cover
// the cutoff (h_d = V / |b_e x b_f| the height of the cell along axis d).
// The search is O(N^2 x images) with one thread per atom i: meant for the
// small cells that need it.
#include "admp_common.cuh"
#include "runtime.h"

namespace admp {

struct ImgGeom {
  double b[9], bi[9];
  int m[3];
  int pbc;
};

// Open boundaries (pbc == 0, box unused): identity cell, no wrap, no images.
template <typename T>
__device__ __forceinline__ void img_geom(const T* box, int pbc, double rc, ImgGeom& g) {
  g.pbc = pbc;
  if (!pbc) {
    for (int k = 0; k < 9; ++k) g.b[k] = g.bi[k] = (k % 4 == 0) ? 1.0 : 0.0;
    g.m[0] = g.m[1] = g.m[2] = 0;
    return;
  }
  load_box(box, g.b);
  const double V = fabs(inv3(g.b, g.bi));
  for (int d = 0; d < 3; ++d) {
    const double* u = g.b + ((d + 1) % 3) * 3;
    const double* v = g.b + ((d + 2) % 3) * 3;
    const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
    const double h = V / sqrt(cx * cx + cy * cy + cz * cz);
    g.m[d] = (int)ceil(rc / h);
  }
}

// wrapped fractional coordinates and the integer cell offset of atom i
template <typename T>
__device__ __forceinline__ void img_frac(const T* pos, int i, const ImgGeom& g, double* f, int* k) {
  const double r0 = pos[3 * i], r1 = pos[3 * i + 1], r2 = pos[3 * i + 2];
  for (int e = 0; e < 3; ++e) {
    const double x = r0 * g.bi[0 * 3 + e] + r1 * g.bi[1 * 3 + e] + r2 * g.bi[2 * 3 + e];
    const double fl = g.pbc ? floor(x) : 0.0;
    f[e] = x - fl;
    k[e] = (int)fl;
  }
}

// Visit every image (j, n) within sqrt(thr2) of atom i (both orders, self
// images included, the atom itself excluded); emit(j, shift, r2) gets the
// shift relative to the caller's positions: r_j - r_i + n.B with
// n = (a, b, c) + k_i - k_j.
template <typename T, typename F>
__device__ __forceinline__ void img_visit(const T* __restrict__ pos, int N, int i, const ImgGeom& g, double thr2,
                                          F&& emit) {
  double fi[3];
  int ki[3];
  img_frac<T>(pos, i, g, fi, ki);
  for (int j = 0; j < N; ++j) {
    double fj[3];
    int kj[3];
    img_frac<T>(pos, j, g, fj, kj);
    for (int a = -g.m[0]; a <= g.m[0]; ++a)
      for (int bb = -g.m[1]; bb <= g.m[1]; ++bb)
        for (int c = -g.m[2]; c <= g.m[2]; ++c) {
          if (j == i && a == 0 && bb == 0 && c == 0) continue;
          const double df[3] = {fj[0] - fi[0] + a, fj[1] - fi[1] + bb, fj[2] - fi[2] + c};
          double r2 = 0.0;
          for (int e = 0; e < 3; ++e) {
            const double v = df[0] * g.b[0 * 3 + e] + df[1] * g.b[1 * 3 + e] + df[2] * g.b[2 * 3 + e];
            r2 += v * v;
          }
          if (r2 <= thr2) emit(j, a + ki[0] - kj[0], bb + ki[1] - kj[1], c + ki[2] - kj[2], r2);
        }
  }
}

template <typename T>
__device__ __forceinline__ int img_count_within(const T* pos, int N, int i, const ImgGeom& g, double thr2) {
  int n = 0;
  img_visit<T>(pos, N, i, g, thr2, [&](int, int, int, int, double) { ++n; });
  return n;
}

// Per atom: the squared radius that keeps its `nnei` nearest images (all of
// them when it has no more than nnei within rc).  The nnei-th smallest r^2 is
// found exactly by bisection over the bit patterns of non-negative doubles,
// which order like the values.  Then the (i, j >= i) pair counts.
template <typename T>
__global__ void __launch_bounds__(128) img_count_kernel(int N, const T* __restrict__ pos, const T* __restrict__ box,
                                                        int pbc, double rc, int nnei, double* __restrict__ thr,
                                                        int* __restrict__ cnt_ij, int* __restrict__ cnt_ii,
                                                        int* __restrict__ ntrunc) {
  __shared__ ImgGeom g;
  if (threadIdx.x == 0) img_geom<T>(box, pbc, rc, g);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double rc2 = rc * rc;
  double t2 = rc2;
  if (nnei >= 0 && img_count_within<T>(pos, N, i, g, rc2) > nnei) {
    atomicAdd(ntrunc, 1);
    if (nnei == 0) {
      t2 = -1.0;
    } else {
      unsigned long long lo = 0ull, hi = (unsigned long long)__double_as_longlong(rc2);
      while (lo < hi) {  // smallest bits with count(r2 <= value) >= nnei
        const unsigned long long mid = lo + (hi - lo) / 2;
        if (img_count_within<T>(pos, N, i, g, __longlong_as_double((long long)mid)) >= nnei)
          hi = mid;
        else
          lo = mid + 1;
      }
      t2 = __longlong_as_double((long long)lo);
    }
  }
  thr[i] = t2;
  int nij = 0, nii = 0;
  img_visit<T>(pos, N, i, g, t2, [&](int j, int, int, int, double) {
    if (j == i)
      ++nii;
    else if (j > i)
      ++nij;
  });
  cnt_ij[i] = nij;
  cnt_ii[i] = nii;
}

template <typename T>
__global__ void __launch_bounds__(128) img_fill_kernel(int N, const T* __restrict__ pos, const T* __restrict__ box,
                                                       int pbc, double rc, const double* __restrict__ thr,
                                                       const long long* __restrict__ off_ij,
                                                       const long long* __restrict__ off_ii, long long base_ii,
                                                       long long* __restrict__ pairs, int* __restrict__ shifts) {
  __shared__ ImgGeom g;
  if (threadIdx.x == 0) img_geom<T>(box, pbc, rc, g);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  long long pij = off_ij[i], pii = base_ii + off_ii[i];
  img_visit<T>(pos, N, i, g, thr[i], [&](int j, int na, int nb, int nc, double) {
    if (j < i) return;
    const long long p = (j == i) ? pii++ : pij++;
    pairs[2 * p] = i;
    pairs[2 * p + 1] = j;
    shifts[3 * p] = na;
    shifts[3 * p + 1] = nb;
    shifts[3 * p + 2] = nc;
  });
}

// ds = |r_j - r_i + n.B|
template <typename T>
__global__ void __launch_bounds__(256) img_dist_kernel(int N, long long P, const long long* __restrict__ pairs,
                                                       const int* __restrict__ shifts, const T* __restrict__ pos,
                                                       const T* __restrict__ box, T* __restrict__ ds, DevError* err) {
  __shared__ double b[9];
  if (threadIdx.x < 9) b[threadIdx.x] = box ? (double)box[threadIdx.x] : 0.0;
  __syncthreads();
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    if (i < 0 || i >= N || j < 0 || j >= N) {
      report_error(err, ADMP_ERR_BAD_INDEX, 4, p);
      ds[p] = T(0);
      continue;
    }
    double r2 = 0.0;
    for (int e = 0; e < 3; ++e) {
      const double v = (double)pos[3 * j + e] - (double)pos[3 * i + e] + shifts[3 * p] * b[e] +
                       shifts[3 * p + 1] * b[3 + e] + shifts[3 * p + 2] * b[6 + e];
      r2 += v * v;
    }
    ds[p] = (T)sqrt(r2);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) img_dist_bwd_kernel(int N, long long P, const long long* __restrict__ pairs,
                                                           const int* __restrict__ shifts, const T* __restrict__ pos,
                                                           const T* __restrict__ box, const T* __restrict__ g,
                                                           T* __restrict__ gpos, T* __restrict__ gbox, DevError* err) {
  __shared__ double b[9];
  __shared__ double red[9 * 32];
  if (threadIdx.x < 9) b[threadIdx.x] = box ? (double)box[threadIdx.x] : 0.0;
  __syncthreads();
  double vb[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const long long i = pairs[2 * p], j = pairs[2 * p + 1];
    if (i < 0 || i >= N || j < 0 || j >= N) {
      report_error(err, ADMP_ERR_BAD_INDEX, 5, p);
      continue;
    }
    const double gp = g[p];
    if (gp == 0.0) continue;
    const int n[3] = {shifts[3 * p], shifts[3 * p + 1], shifts[3 * p + 2]};
    double dr[3];
    for (int e = 0; e < 3; ++e)
      dr[e] = (double)pos[3 * j + e] - (double)pos[3 * i + e] + n[0] * b[e] + n[1] * b[3 + e] + n[2] * b[6 + e];
    const double d = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    if (d == 0.0) continue;
    const double s = gp / d;
    for (int e = 0; e < 3; ++e) {
      const double v = s * dr[e];
      if (gpos && i != j) {
        atomicAdd(gpos + 3 * j + e, (T)v);
        atomicAdd(gpos + 3 * i + e, (T)(-v));
      }
      for (int a = 0; a < 3; ++a) vb[a * 3 + e] += n[a] * v;
    }
  }
  if (gbox && box) {
    __shared__ double out[9];
    if (threadIdx.x < 9) out[threadIdx.x] = 0.0;
    __syncthreads();
    block_atomic_sum<9>(vb, out, red);
    if (threadIdx.x < 9 && out[threadIdx.x] != 0.0) atomicAdd(gbox + threadIdx.x, (T)out[threadIdx.x]);
  }
}

// single-block exclusive scan of n ints into long long offsets
static __global__ void img_scan_kernel(const int* __restrict__ in, long long* __restrict__ out, int n) {
  __shared__ long long part[1024];
  const int nt = blockDim.x, chunk = (n + nt - 1) / nt;
  const int b0 = threadIdx.x * chunk, b1 = min(b0 + chunk, n);
  long long s = 0;
  for (int i = b0; i < b1; ++i) s += in[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long acc = 0;
    for (int k = 0; k < nt; ++k) {
      const long long t = part[k];
      part[k] = acc;
      acc += t;
    }
    out[n] = acc;
  }
  __syncthreads();
  long long acc = part[threadIdx.x];
  for (int i = b0; i < b1; ++i) {
    out[i] = acc;
    acc += in[i];
  }
}

// workspace: thr [N] double, cnt_ij, cnt_ii [N] int, off_ij, off_ii [N+1]
// long long, truncated-atom count int
struct ImgWS {
  double* thr;
  int *cij, *cii, *ntrunc;
  long long *oij, *oii;
};

static size_t img_carve(void* ws, int N, ImgWS* w) {
  Carver c(ws, 0);
  w->thr = c.take<double>(N);
  w->cij = c.take<int>(N);
  w->cii = c.take<int>(N);
  w->oij = c.take<long long>(N + 1);
  w->oii = c.take<long long>(N + 1);
  w->ntrunc = c.take<int>(1);
  return c.off;
}

template <typename T>
static int img_count_impl(int pbc, int N, const T* pos, const T* box, double rc, int nnei, void* ws, size_t bytes,
                          long long* n_ij, long long* n_ii, int* n_truncated, cudaStream_t st) {
  ImgWS w;
  const size_t need = img_carve(ws, N, &w);
  if (!ws || need > bytes) return fail(ADMP_ERR_WORKSPACE, "image neighbour list: workspace needs %zu bytes", need);
  ADMP_CUDA_TRY(cudaMemsetAsync(w.ntrunc, 0, sizeof(int), st));
  img_count_kernel<T><<<(N + 127) / 128, 128, 0, st>>>(N, pos, box, pbc, rc, nnei, w.thr, w.cij, w.cii, w.ntrunc);
  img_scan_kernel<<<1, 1024, 0, st>>>(w.cij, w.oij, N);
  img_scan_kernel<<<1, 1024, 0, st>>>(w.cii, w.oii, N);
  count_launches(3);
  ADMP_CUDA_TRY(cudaGetLastError());
  long long tot[2];
  int nt = 0;
  ADMP_CUDA_TRY(cudaMemcpyAsync(&tot[0], w.oij + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaMemcpyAsync(&tot[1], w.oii + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaMemcpyAsync(&nt, w.ntrunc, sizeof(int), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaStreamSynchronize(st));
  *n_ij = tot[0];
  *n_ii = tot[1];
  if (n_truncated) *n_truncated = nt;
  return ADMP_OK;
}

template <typename T>
static int img_fill_impl(int pbc, int N, const T* pos, const T* box, double rc, void* ws, size_t bytes,
                         long long* pairs, int* shifts, long long capacity, cudaStream_t st) {
  ImgWS w;
  const size_t need = img_carve(ws, N, &w);
  if (!ws || need > bytes) return fail(ADMP_ERR_WORKSPACE, "image neighbour list: workspace needs %zu bytes", need);
  long long tot[2];
  ADMP_CUDA_TRY(cudaMemcpyAsync(&tot[0], w.oij + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaMemcpyAsync(&tot[1], w.oii + N, sizeof(long long), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaStreamSynchronize(st));
  if (tot[0] + tot[1] > capacity)
    return fail(ADMP_ERR_CAPACITY, "image neighbour list: %lld pairs, capacity %lld", tot[0] + tot[1], capacity);
  if (tot[0] + tot[1] == 0) return ADMP_OK;
  img_fill_kernel<T><<<(N + 127) / 128, 128, 0, st>>>(N, pos, box, pbc, rc, w.thr, w.oij, w.oii, tot[0], pairs,
                                                      shifts);
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

}  // namespace admp

using namespace admp;

extern "C" size_t admp_image_nblist_workspace_size(int natoms) {
  ImgWS w;
  return img_carve(nullptr, natoms < 0 ? 0 : natoms, &w);
}

extern "C" int admp_image_nblist_count(int dtype, int pbc, int natoms, const void* pos, const void* box,
                                       double cutoff, int nnei, void* workspace, size_t workspace_bytes,
                                       long long* n_ij, long long* n_ii, int* n_truncated, void* stream) {
  if (!n_ij || !n_ii) return fail(ADMP_ERR_BAD_ARG, "admp_image_nblist_count: null outputs");
  *n_ij = 0;
  *n_ii = 0;
  if (n_truncated) *n_truncated = 0;
  if (!(cutoff > 0)) return fail(ADMP_ERR_BAD_ARG, "rcut must be positive, got %g", cutoff);
  if (natoms == 0) return ADMP_OK;
  if (natoms < 0 || !pos || (pbc && !box)) return fail(ADMP_ERR_BAD_ARG, "admp_image_nblist_count: args");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return img_count_impl<double>(pbc, natoms, (const double*)pos, (const double*)box, cutoff, nnei, workspace,
                                  workspace_bytes, n_ij, n_ii, n_truncated, st);
  if (dtype == ADMP_F32)
    return img_count_impl<float>(pbc, natoms, (const float*)pos, (const float*)box, cutoff, nnei, workspace,
                                 workspace_bytes, n_ij, n_ii, n_truncated, st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}

extern "C" int admp_image_nblist_fill(int dtype, int pbc, int natoms, const void* pos, const void* box,
                                      double cutoff, void* workspace, size_t workspace_bytes, long long* pairs,
                                      int* shifts, long long capacity, void* stream) {
  if (natoms == 0) return ADMP_OK;
  if (natoms < 0 || !pos || (pbc && !box) || (capacity > 0 && (!pairs || !shifts)))
    return fail(ADMP_ERR_BAD_ARG, "admp_image_nblist_fill: args");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return img_fill_impl<double>(pbc, natoms, (const double*)pos, (const double*)box, cutoff, workspace,
                                 workspace_bytes, pairs, shifts, capacity, st);
  if (dtype == ADMP_F32)
    return img_fill_impl<float>(pbc, natoms, (const float*)pos, (const float*)box, cutoff, workspace,
                                workspace_bytes, pairs, shifts, capacity, st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}

extern "C" int admp_image_pair_distances(int dtype, int natoms, long long npairs, const long long* pairs,
                                         const int* shifts, const void* pos, const void* box, void* ds, void* stream) {
  if (npairs == 0) return ADMP_OK;
  if (npairs < 0 || !pairs || !shifts || !pos || !ds)
    return fail(ADMP_ERR_BAD_ARG, "admp_image_pair_distances: args");
  cudaStream_t st = (cudaStream_t)stream;
  DevError* err = scratch_error(st);
  if (!err) return ADMP_ERR_CUDA;
  long long blocks = (npairs + 255) / 256;
  if (blocks > 8192) blocks = 8192;
  if (dtype == ADMP_F64)
    img_dist_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(natoms, npairs, pairs, shifts, (const double*)pos,
                                                              (const double*)box, (double*)ds, err);
  else if (dtype == ADMP_F32)
    img_dist_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(natoms, npairs, pairs, shifts, (const float*)pos,
                                                             (const float*)box, (float*)ds, err);
  else
    return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return check_error(err, st);
}

extern "C" int admp_image_pair_distances_backward(int dtype, int natoms, long long npairs, const long long* pairs,
                                                  const int* shifts, const void* pos, const void* box,
                                                  const void* grad_ds, void* grad_pos, void* grad_box, void* stream) {
  if (npairs == 0) return ADMP_OK;
  if (npairs < 0 || !pairs || !shifts || !pos || !grad_ds)
    return fail(ADMP_ERR_BAD_ARG, "admp_image_pair_distances_backward: args");
  cudaStream_t st = (cudaStream_t)stream;
  DevError* err = scratch_error(st);
  if (!err) return ADMP_ERR_CUDA;
  long long blocks = (npairs + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  if (dtype == ADMP_F64)
    img_dist_bwd_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(natoms, npairs, pairs, shifts, (const double*)pos,
                                                                  (const double*)box, (const double*)grad_ds,
                                                                  (double*)grad_pos, (double*)grad_box, err);
  else if (dtype == ADMP_F32)
    img_dist_bwd_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(natoms, npairs, pairs, shifts, (const float*)pos,
                                                                 (const float*)box, (const float*)grad_ds,
                                                                 (float*)grad_pos, (float*)grad_box, err);
  else
    return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  count_launches(1);
  ADMP_CUDA_TRY(cudaGetLastError());
  return check_error(err, st);
}
