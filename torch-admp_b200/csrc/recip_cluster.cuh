// Cluster-resident reciprocal-space potential for the QEq CG matvec.
//
// One thread-block cluster per system holds the whole PME mesh of that system
// in the shared memory of its C CTAs (C = 1..16): CTA r owns the x planes
// [r P, r P + P), P = ceil(K0 / C).  One launch does, for every system:
//   1. spread   v -> real planes (shared-memory atomics; only the atoms whose
//               x stencil reaches the CTA's planes, found through the atoms'
//               x-key order built once per solve by xkey_sort_kernel)
//   2. z R2C of every pair of rows, then y FFT of every column, per plane
//   3. x FFT of every (y, kz) column across the cluster (distributed shared
//      memory), times the cached 2 G_s, inverse x FFT, written back in place
//   4. inverse y FFT per column, z C2R per pair of rows -> real potential
//   5. gather   dE/dq_i += sum_stencil w phi  (one global atomic per atom and
//               CTA; an atom's six planes span at most a few CTAs)
// Every line transform is done by one warp on its own (a per-warp scratch
// line, __syncwarp between stages), so the block synchronises only between
// the phases.  Each plane row holds K2 reals or K2/2 + 1 complex values in
// place (row stride RS complex, RS odd to spread the column accesses over
// the shared-memory banks).  This is the arithmetic of spread_kernel ->
// fft_slab_fwd_kernel -> fft_x_apply_kernel -> fft_slab_inv_kernel ->
// gather_kernel<T, false> (recip.py:216-308 with the Green's function of
// pme.py:410-443), but the mesh and its spectrum never leave the chip.
#pragma once

#include <cooperative_groups.h>

#include "pme_kernels.cuh"

namespace admp {

namespace cgx = cooperative_groups;

constexpr int kClusterThreads = 256;
constexpr int kClusterWarps = kClusterThreads / 32;
constexpr int kClusterMaxSize = 16;     // CTAs per cluster

// Systems of one launch (all with the same cluster size C).
struct ClusterList {
  int n;                   // clusters (systems) in this launch
  int C;                   // CTAs per cluster
  int sys[kMaxBatch];      // batch index of each cluster's system
};

// complex row stride of a plane: K2 / 2 + 1 rounded up to odd
__host__ __device__ inline int cluster_row_stride(int K2) { return (K2 / 2 + 1) | 1; }

template <typename T>
__host__ __device__ inline size_t cluster_smem_bytes(int K0, int K1, int K2, int C) {
  const int P = (K0 + C - 1) / C;
  int mk = K0 > K1 ? K0 : K1;
  mk = mk > K2 ? mk : K2;
  const size_t cs = sizeof(Cplx<T>);
  return ((size_t)K0 + K1 + K2 + (size_t)P * K1 * cluster_row_stride(K2) + 2 * (size_t)kClusterWarps * mk) * cs +
         (size_t)kClusterMaxSize * sizeof(void*);
}

// First mesh plane key of an atom along x: m0 mod K0 with m0 = ceil(K0 (r B^-1)_x),
// the same expression as make_stencil, so the atom's planes are key-3 .. key+2.
template <typename T>
__device__ __forceinline__ int xkey_of(const T* r, const Geom& g, int K0) {
  const double x = (double)K0 * ((double)r[0] * g.binv[0] + (double)r[1] * g.binv[3] + (double)r[2] * g.binv[6]);
  return wrap_index((int)ceil(x), K0);
}

// Block per system: counting sort of the system's atoms by x key into
// sorted[atom_off ..] (pool indices) and the key starts into
// xkey[slot * stride + k], k = 0..K0 (xkey[.. K0] = natoms).  Launch with
// (max K0 + 1) ints of dynamic shared memory.
template <typename T>
__global__ void __launch_bounds__(1024) xkey_sort_kernel(Batch b, const T* __restrict__ pos,
                                                         const T* __restrict__ box, int* __restrict__ sorted,
                                                         int* __restrict__ xkey, int stride) {
  extern __shared__ int cnt[];  // K0 + 1
  __shared__ Geom g;
  const SysDesc& d = b.s[blockIdx.x];
  const int K0 = d.K0, n = d.natoms;
  if (K0 + 1 > stride) return;  // no table for this slot: it keeps the mesh passes
  load_geom(box, d.box_idx, &g);
  for (int k = threadIdx.x; k <= K0; k += blockDim.x) cnt[k] = 0;
  __syncthreads();
  for (int a = threadIdx.x; a < n; a += blockDim.x)
    atomicAdd(&cnt[xkey_of(pos + 3 * (size_t)(d.atom_off + a), g, K0)], 1);
  __syncthreads();
  int* xs = xkey + (size_t)d.box_idx * stride;
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < K0; ++k) {
      const int c = cnt[k];
      cnt[k] = t;
      xs[k] = t;
      t += c;
    }
    xs[K0] = t;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < n; a += blockDim.x) {
    const int i = d.atom_off + a;
    const int key = xkey_of(pos + 3 * (size_t)i, g, K0);
    sorted[d.atom_off + atomicAdd(&cnt[key], 1)] = i;
  }
}

// Atoms whose stencil reaches planes [p0, p1) have keys in [p0 - 2, p1 + 3)
// (cyclic); one key of slack on each side keeps an atom whose key and stencil
// were rounded apart at an integer x inside the range.  Up to two ranges of
// the x-sorted order.
struct AtomRanges {
  int b0, e0, b1, e1;
  __device__ int count() const { return (e0 - b0) + (e1 - b1); }
  __device__ int at(int t) const { return t < e0 - b0 ? b0 + t : b1 + (t - (e0 - b0)); }
};

__device__ __forceinline__ AtomRanges atom_ranges(const int* xs, int K0, int n, int p0, int p1) {
  AtomRanges r{0, 0, 0, 0};
  if (p1 <= p0) return r;
  const int len = p1 - p0 + 7;
  if (len >= K0) {
    r.e0 = n;
    return r;
  }
  const int ks = wrap_index(p0 - 3, K0), ke = ks + len;
  if (ke <= K0) {
    r.b0 = xs[ks];
    r.e0 = xs[ke];
  } else {
    r.b0 = xs[ks];
    r.e0 = n;
    r.b1 = 0;
    r.e1 = xs[ke - K0];
  }
  return r;
}

template <typename T>
__global__ void __launch_bounds__(kClusterThreads, 2)
    recip_pot_cluster_kernel(Batch b, ClusterList cl, const T* __restrict__ pos, const T* __restrict__ box,
                             const T* __restrict__ v, const int* __restrict__ order, const int* __restrict__ xkey,
                             int xkey_stride, const T* __restrict__ green, T* __restrict__ pot) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Geom g;
  cgx::cluster_group cluster = cgx::this_cluster();
  const int C = cl.C;
  const int rank = (int)cluster.block_rank();
  const int s = cl.sys[blockIdx.x / C];
  if (skip_sys(b, s)) return;  // uniform over the cluster: every CTA leaves before any barrier
  const SysDesc& d = b.s[s];
  const int K0 = d.K0, K1 = d.K1, K2 = d.K2, K2h = d.K2h, np = (K1 + 1) / 2;
  const int RS = cluster_row_stride(K2);
  const int PS = K1 * RS;  // complex elements per plane
  const int P = (K0 + C - 1) / C;
  const int p0 = min(rank * P, K0), p1 = min(p0 + P, K0), npl = p1 - p0;
  const int mk = max(K0, max(K1, K2));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  Cplx<T>* W0 = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* W1 = W0 + K0;
  Cplx<T>* W2 = W1 + K1;
  Cplx<T>* planes = W2 + K2;
  Cplx<T>* wa = planes + (size_t)P * PS + (size_t)warp * 2 * mk;  // this warp's two scratch lines
  Cplx<T>* wb = wa + mk;
  Cplx<T>** rbase = reinterpret_cast<Cplx<T>**>(planes + (size_t)P * PS + (size_t)kClusterWarps * 2 * mk);

  make_twiddles(W0, K0);
  make_twiddles(W1, K1);
  make_twiddles(W2, K2);
  load_geom(box, d.box_idx, &g);
  for (int k = tid; k < npl * PS; k += kClusterThreads) {
    Cplx<T> z;
    z.x = T(0);
    z.y = T(0);
    planes[k] = z;
  }
  Radices R0, R1, R2;
  factor_radices(K0, R0);
  factor_radices(K1, R1);
  factor_radices(K2, R2);
  __syncthreads();

  const int* xs = xkey + (size_t)d.box_idx * xkey_stride;
  const AtomRanges ar = atom_ranges(xs, K0, d.natoms, p0, p1);
  const int na = ar.count();
  const int* ord = order + d.atom_off;
  T* pr = reinterpret_cast<T*>(planes);  // real view: value (lp, y, z) at ((lp K1 + y) RS) 2 + z

  // 1. spread into the owned planes
  for (int t = tid; t < na; t += kClusterThreads) {
    const int ga = ord[ar.at(t)];
    const T qa = v[ga];
    if (qa == T(0)) continue;
    T r[3] = {pos[3 * (size_t)ga], pos[3 * (size_t)ga + 1], pos[3 * (size_t)ga + 2]};
    Stencil<T> st;
    make_stencil<T>(r, g, K0, K1, K2, st);
#pragma unroll
    for (int dx = 0; dx < 6; ++dx) {
      const int lp = st.ix[dx] - p0;
      if (lp < 0 || lp >= npl) continue;
      const T wx = qa * st.w[0][dx];
#pragma unroll
      for (int dy = 0; dy < 6; ++dy) {
        T* row = pr + ((size_t)lp * K1 + st.iy[dy]) * RS * 2;
        const T wxy = wx * st.w[1][dy];
#pragma unroll
        for (int dz = 0; dz < 6; ++dz) atomicAdd(row + st.iz[dz], wxy * st.w[2][dz]);
      }
    }
  }
  __syncthreads();

  // 2a. z R2C: rows (2p, 2p+1) of a plane as one complex FFT, unpacked in place
  for (int task = warp; task < npl * np; task += kClusterWarps) {
    const int lp = task / np, p = task - lp * np;
    const int y0 = 2 * p, y1 = 2 * p + 1;
    Cplx<T>* r0 = planes + ((size_t)lp * K1 + y0) * RS;
    Cplx<T>* r1 = r0 + RS;
    const T* f0 = reinterpret_cast<const T*>(r0);
    const T* f1 = reinterpret_cast<const T*>(r1);
    for (int t = lane; t < K2; t += 32) {
      Cplx<T> z;
      z.x = f0[t];
      z.y = y1 < K1 ? f1[t] : T(0);
      wa[t] = z;
    }
    __syncwarp();
    const Cplx<T>* Z = warp_fft<T, false>(R2, wa, wb, K2, W2, lane);
    for (int k = lane; k < K2h; k += 32) {
      const Cplx<T> a = Z[k], m = Z[k == 0 ? 0 : K2 - k];
      Cplx<T> u, c;
      u.x = (a.x + m.x) * T(0.5);
      u.y = (a.y - m.y) * T(0.5);
      c.x = (a.y + m.y) * T(0.5);
      c.y = (m.x - a.x) * T(0.5);
      r0[k] = u;
      if (y1 < K1) r1[k] = c;
    }
    __syncwarp();
  }
  __syncthreads();

  // 2b. y FFT of every column (lp, kz)
  for (int task = warp; task < npl * K2h; task += kClusterWarps) {
    const int lp = task / K2h, kz = task - lp * K2h;
    Cplx<T>* col = planes + (size_t)lp * PS + kz;
    for (int y = lane; y < K1; y += 32) wa[y] = col[(size_t)y * RS];
    __syncwarp();
    const Cplx<T>* Y = warp_fft<T, false>(R1, wa, wb, K1, W1, lane);
    for (int y = lane; y < K1; y += 32) col[(size_t)y * RS] = Y[y];
    __syncwarp();
  }

  // 3. x FFT of the columns (y, kz) across the cluster
  cluster.sync();
  if (tid < C) rbase[tid] = cluster.map_shared_rank(planes, tid);
  __syncthreads();
  {
    const int ncol = K1 * K2h;
    const int cpr = (ncol + C - 1) / C;
    const int c_begin = min(rank * cpr, ncol), c_end = min(c_begin + cpr, ncol);
    const size_t gxs = (size_t)K1 * K2h;
    const T* G = green + d.green_off;
    for (int c = c_begin + warp; c < c_end; c += kClusterWarps) {
      const int y = c / K2h, kz = c - y * K2h;
      const size_t off = (size_t)y * RS + kz;
      for (int x = lane; x < K0; x += 32) {
        const int owner = x / P;
        wa[x] = rbase[owner][(size_t)(x - owner * P) * PS + off];
      }
      __syncwarp();
      Cplx<T>* X = warp_fft<T, false>(R0, wa, wb, K0, W0, lane);
      for (int x = lane; x < K0; x += 32) {
        const T gm = G[(size_t)x * gxs + c];
        X[x].x *= gm;
        X[x].y *= gm;
      }
      __syncwarp();
      Cplx<T>* F = X == wa ? wb : wa;
      const Cplx<T>* Q = warp_fft<T, true>(R0, X, F, K0, W0, lane);
      for (int x = lane; x < K0; x += 32) {
        const int owner = x / P;
        rbase[owner][(size_t)(x - owner * P) * PS + off] = Q[x];
      }
      __syncwarp();
    }
  }
  cluster.sync();  // the last access to other CTAs' shared memory is before this barrier

  // 4a. inverse y FFT of every column
  for (int task = warp; task < npl * K2h; task += kClusterWarps) {
    const int lp = task / K2h, kz = task - lp * K2h;
    Cplx<T>* col = planes + (size_t)lp * PS + kz;
    for (int y = lane; y < K1; y += 32) wa[y] = col[(size_t)y * RS];
    __syncwarp();
    const Cplx<T>* Y = warp_fft<T, true>(R1, wa, wb, K1, W1, lane);
    for (int y = lane; y < K1; y += 32) col[(size_t)y * RS] = Y[y];
    __syncwarp();
  }
  __syncthreads();

  // 4b. z C2R of rows (2p, 2p+1): one complex inverse FFT, real parts to row
  //     2p, imaginary parts to row 2p + 1 (both rows read before written)
  for (int task = warp; task < npl * np; task += kClusterWarps) {
    const int lp = task / np, p = task - lp * np;
    const int y0 = 2 * p, y1 = 2 * p + 1;
    Cplx<T>* r0 = planes + ((size_t)lp * K1 + y0) * RS;
    Cplx<T>* r1 = r0 + RS;
    for (int t = lane; t < K2; t += 32) {
      const bool lo = t < K2h;
      const int tt = lo ? t : K2 - t;
      Cplx<T> a = r0[tt], c;
      if (y1 < K1) {
        c = r1[tt];
      } else {
        c.x = T(0);
        c.y = T(0);
      }
      if (!lo) {
        a.y = -a.y;
        c.y = -c.y;
      }
      Cplx<T> z;
      z.x = a.x - c.y;
      z.y = a.y + c.x;
      wa[t] = z;
    }
    __syncwarp();
    const Cplx<T>* Z = warp_fft<T, true>(R2, wa, wb, K2, W2, lane);
    T* f0 = reinterpret_cast<T*>(r0);
    T* f1 = reinterpret_cast<T*>(r1);
    for (int t = lane; t < K2; t += 32) {
      f0[t] = Z[t].x;
      if (y1 < K1) f1[t] = Z[t].y;
    }
    __syncwarp();
  }
  __syncthreads();

  // 5. gather the partial potentials of the owned planes
  for (int t = tid; t < na; t += kClusterThreads) {
    const int ga = ord[ar.at(t)];
    T r[3] = {pos[3 * (size_t)ga], pos[3 * (size_t)ga + 1], pos[3 * (size_t)ga + 2]};
    Stencil<T> st;
    make_stencil<T>(r, g, K0, K1, K2, st);
    T acc = T(0);
    bool any = false;
#pragma unroll
    for (int dx = 0; dx < 6; ++dx) {
      const int lp = st.ix[dx] - p0;
      if (lp < 0 || lp >= npl) continue;
      any = true;
      T sx = T(0);
#pragma unroll
      for (int dy = 0; dy < 6; ++dy) {
        const T* row = pr + ((size_t)lp * K1 + st.iy[dy]) * RS * 2;
        T sy = T(0);
#pragma unroll
        for (int dz = 0; dz < 6; ++dz) sy += row[st.iz[dz]] * st.w[2][dz];
        sx += sy * st.w[1][dy];
      }
      acc += sx * st.w[0][dx];
    }
    if (any) atomicAdd(pot + ga, acc);
  }
}

}  // namespace admp
