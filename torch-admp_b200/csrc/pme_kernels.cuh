// Reciprocal-space PME kernels (order-6 B-splines, arbitrary mesh sizes),
// batched over independent systems described by a by-value launch descriptor.
//
//   spread      q -> mesh Q                  recip.py:216-252
//   fft_z_fwd   Q -> half spectrum along z   (two real lines per complex FFT)
//   fft_y       along y (forward / inverse)
//   fft_x_green along x, G(k)|S|^2 energy + k-space virial, S <- 2 G S, inverse x
//                                             pme.py:410-443, recip.py:255-308
//   fft_z_inv   half spectrum -> real potential mesh phi = dE/dQ
//   gather      phi -> dE/dq, dE/dpos, fractional-coordinate virial
//
// Mesh layout (per system): real Q[K0][K1][K2] row-major (the reference's
// flat index ((i0*K1)+i1)*K2+i2, recip.py:201-205); spectrum H[K0][K1][K2/2+1].
#pragma once

#include "admp_common.cuh"
#include "fft_smem.cuh"

namespace admp {

struct SysDesc {
  int32_t atom_off, natoms;
  int32_t K0, K1, K2, K2h;
  int32_t blk_atom, blk_z, blk_y, blk_x, blk_slab;
  int32_t blk_xt;  // first block of the tensor-core x pass (128 columns per block)
  int32_t blk_yt;  // first block of the tensor-core y passes (128 (x, kz) lines per block)
  int32_t blk_zt;  // first block of the tensor-core z passes (128 (x, y) lines per block)
  int64_t mesh_off, spec_off;
  int64_t green_off;  // cached 2 G_s (half-spectrum layout) for CG matvecs
  double kappa;
  int32_t box_idx;
  int32_t flags;
};

// Launch descriptor, passed by value (a few dozen bytes): block counts and
// tile sizes of the launch plus a pointer to the per-system table, which
// lives in device memory (uploaded once per library call, so the launches
// of a call do not each carry the whole table as a kernel parameter).
struct Batch {
  int nsys;
  int nblk_atom, nblk_z, nblk_y, nblk_x, nblk_slab, nblk_xt, nblk_yt, nblk_zt;
  int apb;  // atoms per block (atom kernels)
  int lp;   // line pairs per block (z passes)
  int zb;   // columns per block (y / x passes)
  int maxK0, maxK1, maxK2;
  const int* done;   // optional per-slot skip flags (done[slot * done_stride], slot = box_idx)
  int done_stride;
  int status_off;    // ints from a slot's done flag to its status word (errors of bounded waits)
  const SysDesc* s;  // device table [nsys]
  // first block of every system in the block family `fam` of this launch (a
  // copy of the table's blk_* column, ~1 KB): a block finds its system by
  // binary search over this parameter array (constant bank, broadcast)
  // instead of a chain of dependent global loads into the table
  int fam;
  int blk[kMaxBatch];
};

__device__ __forceinline__ bool skip_sys(const Batch& b, int s) {
  return b.done != nullptr && b.done[(size_t)b.s[s].box_idx * b.done_stride] != 0;
}

constexpr int kAccStride = 32;  // doubles per system in the accumulator array
// accumulator slots
constexpr int kAccErec = 0;     // reciprocal energy
constexpr int kAccVk = 1;       // 9: dE/dB (B = box^-1) through k vectors
constexpr int kAccWf = 10;      // 9: dE/dB through fractional coordinates
constexpr int kAccSlots = 19;

enum SysField { F_ATOM = 0, F_Z = 1, F_Y = 2, F_X = 3, F_SLAB = 4, F_XT = 5, F_YT = 6, F_ZT = 7 };

template <int F>
__device__ __forceinline__ int blk_of(const SysDesc& d) {
  return F == F_ATOM ? d.blk_atom
         : F == F_Z  ? d.blk_z
         : F == F_Y  ? d.blk_y
         : F == F_X  ? d.blk_x
         : F == F_XT ? d.blk_xt
         : F == F_YT ? d.blk_yt
         : F == F_ZT ? d.blk_zt
                     : d.blk_slab;
}

template <int F>
__device__ __forceinline__ int find_sys(const Batch& b, int blk) {
  int lo = 0, hi = b.nsys - 1;
  if (b.fam == F) {
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (b.blk[mid] <= blk)
        lo = mid;
      else
        hi = mid - 1;
    }
    return lo;
  }
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (blk_of<F>(b.s[mid]) <= blk)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int signed_k(int i, int K) { return i <= (K - 1) / 2 ? i : i - K; }

// Block-strided loop over items [0, n) that issues U items' global loads
// before using any of them: load(i) returns item i's value, use(i, v)
// consumes it.  In a plain loop each trip's consumer (a shared-memory store)
// waits for that trip's load, so a thread's loads would pay one memory
// latency each, one after another.
template <int U, typename V, typename L, typename S>
__device__ __forceinline__ void block_batched(int n, L&& load, S&& use) {
  for (int i0 = threadIdx.x; i0 < n; i0 += U * blockDim.x) {
    V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) v[u] = load(i);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) use(i, v[u]);
    }
  }
}

// Per-dimension B-spline structure factor used by the reference:
// theta_d(n) = sum_{m=-2..2} M6(m+3) cos(2 pi m n / K)   (pme.py:412-432)
__device__ __forceinline__ double theta_1d(int n, int K) {
  const double m4 = 26.0 / 120.0, m5 = 1.0 / 120.0, m3 = 66.0 / 120.0;
  double c1 = cospi(2.0 * (double)n / (double)K);
  double c2 = cospi(4.0 * (double)n / (double)K);
  return m3 + 2.0 * m4 * c1 + 2.0 * m5 * c2;
}

// Geometry of one system, computed by one thread into shared memory.
struct Geom {
  double box[9];
  double binv[9];
  double vol;
};

template <typename T>
__device__ __forceinline__ void load_geom(const T* box, int idx, Geom* g) {
  if (threadIdx.x == 0) {
    load_box(box + (size_t)idx * 9, g->box);
    g->vol = inv3(g->box, g->binv);
  }
}

// Stencil of one atom: mesh indices per dim and weights (+derivatives).
template <typename T>
struct Stencil {
  int ix[6], iy[6], iz[6];
  T w[3][6];
  T dw[3][6];
};

template <typename T>
__device__ __forceinline__ void make_stencil(const T* r, const Geom& g, int K0, int K1, int K2,
                                             Stencil<T>& st) {
  const int K[3] = {K0, K1, K2};
  const double x0 = r[0], x1 = r[1], x2 = r[2];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // x_d = K_d * (r @ box_inv)_d  (recip.py:33, 61)
    double x = (double)K[d] * (x0 * g.binv[0 * 3 + d] + x1 * g.binv[1 * 3 + d] + x2 * g.binv[2 * 3 + d]);
    double m0 = ceil(x);             // recip.py:62
    // u0 = m0 - x + 3 (recip.py:63); the stencil point s = k - 3 has u = (m0 - x) + k
    const T t = (T)(m0 - x);
    bspline6<T>(t, st.w[d], st.dw[d]);
    int base = (int)m0 - 3;
    int* idx = d == 0 ? st.ix : d == 1 ? st.iy : st.iz;
#pragma unroll
    for (int k = 0; k < 6; ++k) idx[k] = wrap_index(base + k, K[d]);
  }
}

// ---------------------------------------------------------------------------
// Warp-cooperative stencils: each lane builds the stencil of one atom (its
// 3x6 B-spline weights, derivatives and wrapped mesh indices) into shared
// memory, then the warp walks those 32 atoms with its lanes spread over the
// 36 (y, z) stencil columns, each lane looping over the 6 x offsets.  The
// optional `order` visits atoms in cell-sorted order so that neighbouring
// atoms touch neighbouring mesh lines.
// ---------------------------------------------------------------------------
// Per-warp shared layout (dynamic shared memory): for 32 atoms, the 18
// weights, optionally the 18 derivatives, x offsets ix*K1*K2 (6 ints), the
// wrapped y / z stencil bases, the charge and the atom index.
template <typename T, bool DERIV>
struct WarpStencil {
  T* w;     // [32][18]
  T* dw;    // [32][18]
  int* ox;  // [32][6]
  int* byz; // [32][2]
  T* q;     // [32]
  int* atom;// [32]
  __host__ __device__ static constexpr size_t bytes() {
    return 32 * 18 * sizeof(T) * (DERIV ? 2 : 1) + 32 * 6 * sizeof(int) + 32 * 2 * sizeof(int) + 32 * sizeof(T) +
           32 * sizeof(int) + 16;
  }
  __device__ void carve(unsigned char* base) {
    w = reinterpret_cast<T*>(base);
    T* e = w + 32 * 18;
    if (DERIV) {
      dw = e;
      e += 32 * 18;
    } else {
      dw = nullptr;
    }
    q = e;
    int* ip = reinterpret_cast<int*>(q + 32);
    ox = ip;
    byz = ox + 32 * 6;
    atom = byz + 32 * 2;
  }
};

template <typename T, bool DERIV>
__device__ __forceinline__ void warp_build_stencil(WarpStencil<T, DERIV>& ws, const SysDesc& d, const Geom& g,
                                                   const T* __restrict__ pos, const T* __restrict__ q,
                                                   const int* __restrict__ order, int a_first, int a_end, int lane) {
  const int a = a_first + lane;
  if (a < a_end) {
    const int ga = order ? order[d.atom_off + a] : d.atom_off + a;
    T r[3] = {pos[3 * (size_t)ga], pos[3 * (size_t)ga + 1], pos[3 * (size_t)ga + 2]};
    Stencil<T> st;
    make_stencil<T>(r, g, d.K0, d.K1, d.K2, st);
    T* w = ws.w + lane * 18;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      w[k] = st.w[0][k];
      w[6 + k] = st.w[1][k];
      w[12 + k] = st.w[2][k];
      ws.ox[lane * 6 + k] = st.ix[k] * d.K1 * d.K2;
    }
    if (DERIV) {
      T* dw = ws.dw + lane * 18;
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        dw[k] = st.dw[0][k];
        dw[6 + k] = st.dw[1][k];
        dw[12 + k] = st.dw[2][k];
      }
    }
    ws.byz[lane * 2] = st.iy[0];
    ws.byz[lane * 2 + 1] = st.iz[0];
    ws.q[lane] = q ? q[ga] : T(0);
    ws.atom[lane] = ga;
  }
  __syncwarp();
}

__device__ __forceinline__ int wrap_up(int i, int K) {
  while (i >= K) i -= K;
  return i;
}

// spread: q -> mesh (zeroed), atomic adds
template <typename T>
__global__ void __launch_bounds__(256) spread_kernel(Batch b, const T* __restrict__ pos,
                                                     const T* __restrict__ box,
                                                     const T* __restrict__ q, T* __restrict__ mesh,
                                                     const int* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Geom g;
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];  // a register copy would cost this kernel 10 registers
  load_geom(box, d.box_idx, &g);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int a_begin = (blockIdx.x - d.blk_atom) * b.apb;
  const int a_end = min(a_begin + b.apb, d.natoms);
  T* M = mesh + d.mesh_off;
  WarpStencil<T, false> ws;
  ws.carve(dsm + warp * WarpStencil<T, false>::bytes());
  // columns 0..31 of an atom: lane = 6 y + z; the last four columns (y 5, z 2..5) of eight
  // atoms at once: lane -> atom lane / 4, z 2 + lane % 4
  const int y0 = lane / 6, z0 = lane % 6, jt = lane >> 2, zt = 2 + (lane & 3);
  for (int a0 = a_begin + warp * 32; a0 < a_end; a0 += nw * 32) {
    warp_build_stencil<T, false>(ws, d, g, pos, q, order, a0, a_end, lane);
    const int na = min(32, a_end - a0);
    for (int j0 = 0; j0 < na; j0 += 8) {
      const int j1 = min(j0 + 8, na);
      for (int j = j0; j < j1; ++j) {
        const T qa = ws.q[j];
        if (qa == T(0)) continue;
        const T* w = ws.w + j * 18;
        const int* ox = ws.ox + j * 6;
        const T wyz = qa * w[6 + y0] * w[12 + z0];
        const int oyz = wrap_up(ws.byz[2 * j] + y0, d.K1) * d.K2 + wrap_up(ws.byz[2 * j + 1] + z0, d.K2);
#pragma unroll
        for (int dx = 0; dx < 6; ++dx) atomicAdd(M + ox[dx] + oyz, w[dx] * wyz);
      }
      const int j = j0 + jt;
      if (j < j1) {
        const T qa = ws.q[j];
        if (qa != T(0)) {
          const T* w = ws.w + j * 18;
          const int* ox = ws.ox + j * 6;
          const T wyz = qa * w[6 + 5] * w[12 + zt];
          const int oyz = wrap_up(ws.byz[2 * j] + 5, d.K1) * d.K2 + wrap_up(ws.byz[2 * j + 1] + zt, d.K2);
#pragma unroll
          for (int dx = 0; dx < 6; ++dx) atomicAdd(M + ox[dx] + oyz, w[dx] * wyz);
        }
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// z pass forward: two real lines -> one complex FFT -> two half spectra
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) fft_z_fwd_kernel(Batch b, const T* __restrict__ mesh,
                                                        Cplx<T>* __restrict__ spec) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = find_sys<F_Z>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K2 = d.K2, K2h = d.K2h, L = d.K0 * d.K1, npair = (L + 1) / 2;
  const FastDiv fdK2 = fast_div(K2), fdK2h = fast_div(K2h);
  const int p0 = (blockIdx.x - d.blk_z) * b.lp;
  const int np = min(b.lp, npair - p0);
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* A = W + b.maxK2;
  Cplx<T>* B = A + (size_t)b.lp * b.maxK2;
  make_twiddles(W, K2);
  const T* Q = mesh + d.mesh_off;
  for (int idx = threadIdx.x; idx < np * K2; idx += blockDim.x) {
    const int p = fdiv(idx, fdK2), t = idx - p * K2;
    const int l0 = 2 * (p0 + p), l1 = l0 + 1;
    Cplx<T> z;
    z.x = Q[(size_t)l0 * K2 + t];
    z.y = l1 < L ? Q[(size_t)l1 * K2 + t] : T(0);
    A[p * K2 + t] = z;
  }
  __syncthreads();
  Cplx<T>* R = fft_lines<T, false, false>(A, B, np, K2, K2, 1, W);
  Cplx<T>* H = spec + d.spec_off;
  for (int idx = threadIdx.x; idx < np * K2h; idx += blockDim.x) {
    const int p = fdiv(idx, fdK2h), k = idx - p * K2h;
    const Cplx<T> Z = R[p * K2 + k];
    const Cplx<T> Zm = R[p * K2 + (k == 0 ? 0 : K2 - k)];
    const int l0 = 2 * (p0 + p);
    Cplx<T> a, c;
    a.x = (Z.x + Zm.x) * T(0.5);
    a.y = (Z.y - Zm.y) * T(0.5);
    c.x = (Z.y + Zm.y) * T(0.5);
    c.y = (Zm.x - Z.x) * T(0.5);
    H[(size_t)l0 * K2h + k] = a;
    if (l0 + 1 < L) H[(size_t)(l0 + 1) * K2h + k] = c;
  }
}

// ---------------------------------------------------------------------------
// y pass (forward or inverse), in place on the spectrum
// ---------------------------------------------------------------------------
template <typename T, bool INV>
__global__ void __launch_bounds__(256) fft_y_kernel(Batch b, Cplx<T>* __restrict__ spec) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = find_sys<F_Y>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K1 = d.K1, K2h = d.K2h, zb = b.zb;
  const int ncb = (K2h + zb - 1) / zb;
  const int local = blockIdx.x - d.blk_y;
  const int x = local / ncb, cb = local - x * ncb;
  const int kz0 = cb * zb, nz = min(zb, K2h - kz0);
  const FastDiv fdnz = fast_div(nz);
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* A = W + b.maxK1;
  Cplx<T>* B = A + (size_t)zb * b.maxK1;
  make_twiddles(W, K1);
  Cplx<T>* H = spec + d.spec_off + (size_t)x * K1 * K2h + kz0;
  for (int idx = threadIdx.x; idx < K1 * nz; idx += blockDim.x) {
    const int y = fdiv(idx, fdnz), c = idx - y * nz;
    A[y * zb + c] = H[(size_t)y * K2h + c];
  }
  __syncthreads();
  Cplx<T>* R = fft_lines<T, true, INV>(A, B, nz, K1, 1, zb, W);
  for (int idx = threadIdx.x; idx < K1 * nz; idx += blockDim.x) {
    const int y = fdiv(idx, fdnz), c = idx - y * nz;
    H[(size_t)y * K2h + c] = R[y * zb + c];
  }
}

// ---------------------------------------------------------------------------
// x pass: forward FFT, Green's function (energy + virial), scale, inverse FFT
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) fft_x_green_kernel(Batch b, Cplx<T>* __restrict__ spec,
                                                          const T* __restrict__ box,
                                                          double* __restrict__ acc, double ke) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ Geom g;
  __shared__ double red[10 * 32];
  const int s = find_sys<F_X>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K0 = d.K0, K1 = d.K1, K2 = d.K2, K2h = d.K2h, zb = b.zb;
  // this block: columns [c0, c0 + nz) of the flattened (y, kz) index c = y K2h + kz
  const int c0 = (blockIdx.x - d.blk_x) * zb, nz = min(zb, K1 * K2h - c0);
  const FastDiv fdnz = fast_div(nz);
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* A = W + b.maxK0;
  Cplx<T>* B = A + (size_t)zb * b.maxK0;
  double* thx = reinterpret_cast<double*>(B + (size_t)zb * b.maxK0);
  double* thyz = thx + b.maxK0;   // theta_y theta_z per column
  double* wcol = thyz + zb;       // half-spectrum weight per column
  int* lab = reinterpret_cast<int*>(wcol + zb);  // per column: ny, mirror ny, nz, mirror nz
  make_twiddles(W, K0);
  load_geom(box, d.box_idx, &g);
  for (int i = threadIdx.x; i < K0; i += blockDim.x) thx[i] = theta_1d(signed_k(i, K0), K0);
  for (int i = threadIdx.x; i < nz; i += blockDim.x) {
    const int c = c0 + i, y = c / K2h, kz = c - y * K2h;
    // labels of the mirror indices -y, -kz (the reference labels K/2 as -K/2,
    // so a Nyquist index is its own mirror with the same label)
    const int ny = signed_k(y, K1), n2 = signed_k(kz, K2);
    lab[4 * i] = ny;
    lab[4 * i + 1] = signed_k(y == 0 ? 0 : K1 - y, K1);
    lab[4 * i + 2] = n2;
    lab[4 * i + 3] = signed_k(kz == 0 ? 0 : K2 - kz, K2);
    thyz[i] = theta_1d(ny, K1) * theta_1d(n2, K2);
    wcol[i] = (kz == 0 || (2 * kz == K2)) ? 1.0 : 2.0;
  }
  Cplx<T>* H = spec + d.spec_off + c0;
  const size_t xs = (size_t)K1 * K2h;
  block_batched<4, Cplx<T>>(
      K0 * nz,
      [&](int idx) {
        const int x = fdiv(idx, fdnz), c = idx - x * nz;
        return H[(size_t)x * xs + c];
      },
      [&](int idx, const Cplx<T>& v) {
        const int x = fdiv(idx, fdnz), c = idx - x * nz;
        A[x * zb + c] = v;
      });
  __syncthreads();
  Cplx<T>* R = fft_lines<T, true, false>(A, B, nz, K0, 1, zb, W);
  Cplx<T>* F = (R == A) ? B : A;
  const double kappa = d.kappa;
  const double inv4k2 = 1.0 / (4.0 * kappa * kappa);
  const double pref = ke * 2.0 * kPi / g.vol;
  double v[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) v[k] = 0.0;
  for (int idx = threadIdx.x; idx < K0 * nz; idx += blockDim.x) {
    const int x = fdiv(idx, fdnz), c = idx - x * nz;
    // A half-spectrum entry p stands for p and its mirror pb = -p (mod K); both
    // carry |S|^2 and the reference's own integer labels.  E = sum G(n)|S|^2
    // over the full spectrum equals sum over the half spectrum of
    // w * Gs * |S|^2 with Gs = (G(n_p) + G(n_pb)) / 2 and w = 2 (1 on the
    // kz = 0 and kz = K2/2 planes, whose mirrors are separate entries).
    const int ny = lab[4 * c], nyb = lab[4 * c + 1], n2 = lab[4 * c + 2], n2b = lab[4 * c + 3];
    const int n0 = signed_k(x, K0), n0b = signed_k(x == 0 ? 0 : K0 - x, K0);
    const double th = thx[x] * thyz[c];
    const double inv_th2 = 1.0 / (th * th);
    const double w = wcol[c];
    Cplx<T> S = R[x * zb + c];
    const double s2 = (double)S.x * (double)S.x + (double)S.y * (double)S.y;
    double Gs = 0.0;
    // the mirror label equals -n unless an x or y index is a Nyquist index; then
    // G(mirror) = G(n) and one evaluation counts twice
    const bool same = (n0b == -n0) && (nyb == -ny) && (n2b == -n2);
    const double mult = same ? 2.0 : 1.0;
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      if (m == 1 && same) break;
      const int a0 = m ? n0b : n0, a1 = m ? nyb : ny, a2 = m ? n2b : n2;
      if (a0 == 0 && a1 == 0 && a2 == 0) continue;  // k = 0 excluded (pme.py:435-438)
      double kv[3];
#pragma unroll
      for (int e = 0; e < 3; ++e)
        kv[e] = 2.0 * kPi * (a0 * g.binv[0 * 3 + e] + a1 * g.binv[1 * 3 + e] + a2 * g.binv[2 * 3 + e]);
      const double ksq = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      const double G = pref / ksq * exp(-ksq * inv4k2) * inv_th2;
      Gs += 0.5 * mult * G;
      const double Ek = 0.5 * mult * w * G * s2;
      v[0] += Ek;
      // dE/dB[a][e] = sum_k E_k (-(1/(4 kappa^2) + 1/k^2)) 2 k_e 2 pi n_a
      const double f = -4.0 * kPi * (inv4k2 + 1.0 / ksq) * Ek;
      const double nn[3] = {(double)a0, (double)a1, (double)a2};
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int e = 0; e < 3; ++e) v[1 + a * 3 + e] += f * nn[a] * kv[e];
    }
    // phi = dE/dQ = 2 * IFFT(Gs S)
    S.x = (T)(2.0 * Gs * (double)S.x);
    S.y = (T)(2.0 * Gs * (double)S.y);
    R[x * zb + c] = S;
  }
  block_atomic_sum<10>(v, acc + (size_t)s * kAccStride + kAccErec, red);
  Cplx<T>* P = fft_lines<T, true, true>(R, F, nz, K0, 1, zb, W);
  for (int idx = threadIdx.x; idx < K0 * nz; idx += blockDim.x) {
    const int x = fdiv(idx, fdnz), c = idx - x * nz;
    H[(size_t)x * xs + c] = P[x * zb + c];
  }
}

// ---------------------------------------------------------------------------
// Fused slab passes (a block takes ppb consecutive x planes when they fit in
// shared memory; small meshes get several planes per block so every FFT
// stage has enough lines for the whole block):
//   fft_slab_fwd: Q[x][y][z] -> z R2C (two real lines per complex FFT) -> y FFT
//                 -> H[x][y][kz]
//   fft_slab_inv: H[x][y][kz] -> inverse y FFT -> z C2R -> phi[x][y][z]
// In shared memory the z lines of the block's planes are packed back to back
// (line (pl, p) at (pl np + p) K2) and the y lines interleaved by plane
// (element (y, pl, kz) at (y npl + pl) K2h + kz), so each pass is one batch
// of equally strided lines.
// ---------------------------------------------------------------------------
// planes per block for a system whose plane needs PL complex values, given
// the launch's per-buffer capacity (the host computes block counts the same way)
__host__ __device__ inline int slab_ppb(int buf_elems, int PL, int K0) {
  int p = buf_elems / PL;
  p = p < 1 ? 1 : p;
  return p < K0 ? p : K0;
}

__host__ __device__ inline int slab_plane_elems(int K1, int K2) {
  const int a = ((K1 + 1) / 2) * K2, c = K1 * (K2 / 2 + 1);
  return a > c ? a : c;
}

template <typename T>
__global__ void __launch_bounds__(256) fft_slab_fwd_kernel(Batch b, const T* __restrict__ mesh,
                                                           Cplx<T>* __restrict__ spec, int buf_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = find_sys<F_SLAB>(b, blockIdx.x);  // a block per run of x planes
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K0 = d.K0, K1 = d.K1, K2 = d.K2, K2h = d.K2h;
  const int np = (K1 + 1) / 2;
  const int ppb = slab_ppb(buf_elems, slab_plane_elems(K1, K2), K0);
  const int x0 = (blockIdx.x - d.blk_slab) * ppb, npl = min(ppb, K0 - x0);
  const FastDiv fdK2 = fast_div(K2), fdK2h = fast_div(K2h), fdnp = fast_div(np), fdP = fast_div(K1 * K2h);
  Cplx<T>* W1 = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* W2 = W1 + b.maxK1;
  Cplx<T>* A = W2 + b.maxK2;
  Cplx<T>* B = A + buf_elems;
  make_twiddles(W1, K1);
  make_twiddles(W2, K2);
  const T* Q = mesh + d.mesh_off + (size_t)x0 * K1 * K2;
  const int nzl = npl * np;  // z line pairs of the block
  block_batched<4, Cplx<T>>(
      nzl * K2,
      [&](int idx) {
        const int line = fdiv(idx, fdK2), t = idx - line * K2;
        const int pl = fdiv(line, fdnp), p = line - pl * np;
        const T* Qp = Q + (size_t)pl * K1 * K2;
        Cplx<T> z;
        z.x = Qp[(size_t)(2 * p) * K2 + t];
        z.y = 2 * p + 1 < K1 ? Qp[(size_t)(2 * p + 1) * K2 + t] : T(0);
        return z;
      },
      [&](int idx, const Cplx<T>& z) { A[idx] = z; });
  __syncthreads();
  Cplx<T>* R = fft_lines<T, false, false>(A, B, nzl, K2, K2, 1, W2);
  Cplx<T>* U = (R == A) ? B : A;
  // unpack the two-for-one transforms into U[y][pl][kz]
  const int ys = npl * K2h;  // element stride of the y lines
  for (int idx = threadIdx.x; idx < nzl * K2h; idx += blockDim.x) {
    const int line = fdiv(idx, fdK2h), k = idx - line * K2h;
    const int pl = fdiv(line, fdnp), p = line - pl * np;
    const Cplx<T> Z = R[line * K2 + k];
    const Cplx<T> Zm = R[line * K2 + (k == 0 ? 0 : K2 - k)];
    Cplx<T> a, c;
    a.x = (Z.x + Zm.x) * T(0.5);
    a.y = (Z.y - Zm.y) * T(0.5);
    c.x = (Z.y + Zm.y) * T(0.5);
    c.y = (Zm.x - Z.x) * T(0.5);
    U[(2 * p) * ys + pl * K2h + k] = a;
    if (2 * p + 1 < K1) U[(2 * p + 1) * ys + pl * K2h + k] = c;
  }
  __syncthreads();
  Cplx<T>* V = fft_lines<T, true, false>(U, R, npl * K2h, K1, 1, ys, W1);
  Cplx<T>* H = spec + d.spec_off + (size_t)x0 * K1 * K2h;
  for (int idx = threadIdx.x; idx < npl * K1 * K2h; idx += blockDim.x) {
    const int pl = fdiv(idx, fdP), rem = idx - pl * (K1 * K2h);
    const int y = fdiv(rem, fdK2h), kz = rem - y * K2h;
    H[idx] = V[y * ys + pl * K2h + kz];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) fft_slab_inv_kernel(Batch b, const Cplx<T>* __restrict__ spec,
                                                           T* __restrict__ mesh, int buf_elems) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = find_sys<F_SLAB>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K0 = d.K0, K1 = d.K1, K2 = d.K2, K2h = d.K2h;
  const int np = (K1 + 1) / 2;
  const int ppb = slab_ppb(buf_elems, slab_plane_elems(K1, K2), K0);
  const int x0 = (blockIdx.x - d.blk_slab) * ppb, npl = min(ppb, K0 - x0);
  const FastDiv fdK2 = fast_div(K2), fdK2h = fast_div(K2h), fdnp = fast_div(np), fdP = fast_div(K1 * K2h);
  Cplx<T>* W1 = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* W2 = W1 + b.maxK1;
  Cplx<T>* A = W2 + b.maxK2;
  Cplx<T>* B = A + buf_elems;
  make_twiddles(W1, K1);
  make_twiddles(W2, K2);
  const int ys = npl * K2h;
  const Cplx<T>* H = spec + d.spec_off + (size_t)x0 * K1 * K2h;
  block_batched<4, Cplx<T>>(
      npl * K1 * K2h, [&](int idx) { return H[idx]; },
      [&](int idx, const Cplx<T>& v) {
        const int pl = fdiv(idx, fdP), rem = idx - pl * (K1 * K2h);
        const int y = fdiv(rem, fdK2h), kz = rem - y * K2h;
        A[y * ys + pl * K2h + kz] = v;
      });
  __syncthreads();
  Cplx<T>* V = fft_lines<T, true, true>(A, B, npl * K2h, K1, 1, ys, W1);
  Cplx<T>* Z = (V == A) ? B : A;
  const int nzl = npl * np;
  for (int idx = threadIdx.x; idx < nzl * K2; idx += blockDim.x) {
    const int line = fdiv(idx, fdK2), t = idx - line * K2;
    const int pl = fdiv(line, fdnp), p = line - pl * np;
    const bool lo = t < K2h;
    const int tt = lo ? t : K2 - t;
    Cplx<T> a = V[(2 * p) * ys + pl * K2h + tt];
    Cplx<T> c;
    if (2 * p + 1 < K1) {
      c = V[(2 * p + 1) * ys + pl * K2h + tt];
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
    Z[idx] = z;
  }
  __syncthreads();
  Cplx<T>* R = fft_lines<T, false, true>(Z, V, nzl, K2, K2, 1, W2);
  T* M = mesh + d.mesh_off + (size_t)x0 * K1 * K2;
  for (int idx = threadIdx.x; idx < nzl * K2; idx += blockDim.x) {
    const int line = fdiv(idx, fdK2), t = idx - line * K2;
    const int pl = fdiv(line, fdnp), p = line - pl * np;
    const Cplx<T> z = R[idx];
    T* Mp = M + (size_t)pl * K1 * K2;
    Mp[(size_t)(2 * p) * K2 + t] = z.x;
    if (2 * p + 1 < K1) Mp[(size_t)(2 * p + 1) * K2 + t] = z.y;
  }
}

// ---------------------------------------------------------------------------
// Cached Green's function for repeated matvecs (CG): green = 2 G_s over the
// half spectrum, with G_s symmetrised over the reference's mirror labels as in
// fft_x_green_kernel.  Box and mesh are fixed during a solve.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) green_build_kernel(Batch b, const T* __restrict__ box, T* __restrict__ green,
                                                          double ke) {
  __shared__ Geom g;
  const int s = find_sys<F_X>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const int K0 = d.K0, K1 = d.K1, K2 = d.K2, K2h = d.K2h, zb = b.zb;
  const int c0 = (blockIdx.x - d.blk_x) * zb, nz = min(zb, K1 * K2h - c0);
  const FastDiv fdnz = fast_div(nz);
  load_geom(box, d.box_idx, &g);
  __syncthreads();
  const double inv4k2 = 1.0 / (4.0 * d.kappa * d.kappa);
  const double pref = ke * 2.0 * kPi / g.vol;
  T* G = green + d.green_off + c0;
  for (int idx = threadIdx.x; idx < K0 * nz; idx += blockDim.x) {
    const int x = fdiv(idx, fdnz), c = idx - x * nz;
    const int cc = c0 + c, y = cc / K2h, kz = cc - y * K2h;
    const int ny = signed_k(y, K1), nyb = signed_k(y == 0 ? 0 : K1 - y, K1);
    const int n0 = signed_k(x, K0), n2 = signed_k(kz, K2);
    const int n0b = signed_k(x == 0 ? 0 : K0 - x, K0), n2b = signed_k(kz == 0 ? 0 : K2 - kz, K2);
    const double th = theta_1d(n0, K0) * theta_1d(ny, K1) * theta_1d(n2, K2);
    const bool same = (n0b == -n0) && (nyb == -ny) && (n2b == -n2);
    double Gs = 0.0;
    for (int m = 0; m < 2; ++m) {
      if (m == 1 && same) break;
      const int a0 = m ? n0b : n0, a1 = m ? nyb : ny, a2 = m ? n2b : n2;
      if (a0 == 0 && a1 == 0 && a2 == 0) continue;
      double kv[3];
      for (int e = 0; e < 3; ++e)
        kv[e] = 2.0 * kPi * (a0 * g.binv[0 * 3 + e] + a1 * g.binv[1 * 3 + e] + a2 * g.binv[2 * 3 + e]);
      const double ksq = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      Gs += (same ? 1.0 : 0.5) * pref / ksq * exp(-ksq * inv4k2) / (th * th);
    }
    G[(size_t)x * K1 * K2h + c] = (T)(2.0 * Gs);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) fft_x_apply_kernel(Batch b, Cplx<T>* __restrict__ spec,
                                                          const T* __restrict__ green) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = find_sys<F_X>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K0 = d.K0, K1 = d.K1, K2h = d.K2h, zb = b.zb;
  // this block: columns [c0, c0 + nz) of the flattened (y, kz) index c = y K2h + kz
  const int c0 = (blockIdx.x - d.blk_x) * zb, nz = min(zb, K1 * K2h - c0);
  const FastDiv fdnz = fast_div(nz);
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* A = W + b.maxK0;
  Cplx<T>* B = A + (size_t)zb * b.maxK0;
  make_twiddles(W, K0);
  Cplx<T>* H = spec + d.spec_off + c0;
  const T* G = green + d.green_off + c0;
  const size_t xs = (size_t)K1 * K2h;
  block_batched<4, Cplx<T>>(
      K0 * nz,
      [&](int idx) {
        const int x = fdiv(idx, fdnz), c = idx - x * nz;
        return H[(size_t)x * xs + c];
      },
      [&](int idx, const Cplx<T>& v) {
        const int x = fdiv(idx, fdnz), c = idx - x * nz;
        A[x * zb + c] = v;
      });
  __syncthreads();
  Cplx<T>* R = fft_lines<T, true, false>(A, B, nz, K0, 1, zb, W);
  Cplx<T>* F = (R == A) ? B : A;
  block_batched<4, T>(
      K0 * nz,
      [&](int idx) {
        const int x = fdiv(idx, fdnz), c = idx - x * nz;
        return G[(size_t)x * xs + c];
      },
      [&](int idx, T gm) {
        const int x = fdiv(idx, fdnz), c = idx - x * nz;
        Cplx<T> v = R[x * zb + c];
        v.x *= gm;
        v.y *= gm;
        R[x * zb + c] = v;
      });
  __syncthreads();
  Cplx<T>* P = fft_lines<T, true, true>(R, F, nz, K0, 1, zb, W);
  for (int idx = threadIdx.x; idx < K0 * nz; idx += blockDim.x) {
    const int x = fdiv(idx, fdnz), c = idx - x * nz;
    H[(size_t)x * xs + c] = P[x * zb + c];
  }
}

// ---------------------------------------------------------------------------
// z pass inverse: two half spectra -> one complex inverse FFT -> two real lines
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) fft_z_inv_kernel(Batch b, const Cplx<T>* __restrict__ spec,
                                                        T* __restrict__ mesh) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = find_sys<F_Z>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  const int K2 = d.K2, K2h = d.K2h, L = d.K0 * d.K1, npair = (L + 1) / 2;
  const FastDiv fdK2 = fast_div(K2);
  const int p0 = (blockIdx.x - d.blk_z) * b.lp;
  const int np = min(b.lp, npair - p0);
  Cplx<T>* W = reinterpret_cast<Cplx<T>*>(smem_raw);
  Cplx<T>* A = W + b.maxK2;
  Cplx<T>* B = A + (size_t)b.lp * b.maxK2;
  make_twiddles(W, K2);
  const Cplx<T>* H = spec + d.spec_off;
  for (int idx = threadIdx.x; idx < np * K2; idx += blockDim.x) {
    const int p = fdiv(idx, fdK2), t = idx - p * K2;
    const int l0 = 2 * (p0 + p), l1 = l0 + 1;
    const bool lo = t < K2h;
    const int tt = lo ? t : K2 - t;
    Cplx<T> a = H[(size_t)l0 * K2h + tt];
    Cplx<T> c;
    if (l1 < L) {
      c = H[(size_t)l1 * K2h + tt];
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
    A[p * K2 + t] = z;
  }
  __syncthreads();
  Cplx<T>* R = fft_lines<T, false, true>(A, B, np, K2, K2, 1, W);
  T* M = mesh + d.mesh_off;
  for (int idx = threadIdx.x; idx < np * K2; idx += blockDim.x) {
    const int p = fdiv(idx, fdK2), t = idx - p * K2;
    const int l0 = 2 * (p0 + p), l1 = l0 + 1;
    const Cplx<T> z = R[p * K2 + t];
    M[(size_t)l0 * K2 + t] = z.x;
    if (l1 < L) M[(size_t)l1 * K2 + t] = z.y;
  }
}

// ---------------------------------------------------------------------------
// gather: pot_i = sum phi theta; dE/du_d = q sum phi dtheta/du_d (warp-cooperative)
// ---------------------------------------------------------------------------
template <typename T, bool FORCES>
__global__ void __launch_bounds__(256) gather_kernel(Batch b, const T* __restrict__ pos,
                                                     const T* __restrict__ box,
                                                     const T* __restrict__ q,
                                                     const T* __restrict__ phi,
                                                     T* __restrict__ dE_dq, T* __restrict__ dE_dpos,
                                                     double* __restrict__ acc, T pot_scale,
                                                     const int* __restrict__ order) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Geom g;
  __shared__ double red[9 * 32];
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc d = b.s[s];
  load_geom(box, d.box_idx, &g);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int a_begin = (blockIdx.x - d.blk_atom) * b.apb;
  const int a_end = min(a_begin + b.apb, d.natoms);
  const T* M = phi + d.mesh_off;
  const int K[3] = {d.K0, d.K1, d.K2};
  WarpStencil<T, FORCES> ws;
  ws.carve(dsm + warp * WarpStencil<T, FORCES>::bytes());
  // column mapping as in spread_kernel: columns 0..31 per atom, the last four of eight atoms at once
  const int y0 = lane / 6, z0 = lane % 6, jt = lane >> 2, zt = 2 + (lane & 3);
  double wf[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) wf[k] = 0.0;
  for (int a0 = a_begin + warp * 32; a0 < a_end; a0 += nw * 32) {
    warp_build_stencil<T, FORCES>(ws, d, g, pos, FORCES ? q : nullptr, order, a0, a_end, lane);
    const int na = min(32, a_end - a0);
    T my_pot = 0, my_g0 = 0, my_g1 = 0, my_g2 = 0;
    for (int j0 = 0; j0 < na; j0 += 8) {
      const int j1 = min(j0 + 8, na);
      // GU atoms at a time: their 6 GU mesh loads are issued before the first reduction
      constexpr int GU = sizeof(T) == 8 ? 2 : 4;
      for (int jb = j0; jb < j1; jb += GU) {
        T fm[GU][6];
#pragma unroll
        for (int u = 0; u < GU; ++u) {
          const int j = jb + u;
          if (j < j1) {
            const int* ox = ws.ox + j * 6;
            const int oyz = wrap_up(ws.byz[2 * j] + y0, d.K1) * d.K2 + wrap_up(ws.byz[2 * j + 1] + z0, d.K2);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) fm[u][dx] = M[ox[dx] + oyz];
          }
        }
#pragma unroll
        for (int u = 0; u < GU; ++u) {
          const int j = jb + u;
          if (j >= j1) break;
          const T* w = ws.w + j * 18;
          const T wy = w[6 + y0], wz = w[12 + z0];
          T sw = 0, sdw = 0;
#pragma unroll
          for (int dx = 0; dx < 6; ++dx) {
            sw += fm[u][dx] * w[dx];
            if (FORCES) sdw += fm[u][dx] * ws.dw[j * 18 + dx];
          }
          T pot = sw * wy * wz, g0 = 0, g1 = 0, g2 = 0;
          pot = warp_sum(pot);
          if (FORCES) {
            g0 = warp_sum(sdw * wy * wz);
            g1 = warp_sum(sw * ws.dw[j * 18 + 6 + y0] * wz);
            g2 = warp_sum(sw * wy * ws.dw[j * 18 + 12 + z0]);
          }
          if (lane == j) {
            my_pot = pot;
            my_g0 = g0;
            my_g1 = g1;
            my_g2 = g2;
          }
        }
      }
      // the last four columns of atoms j0 .. j1-1, reduced over each atom's four lanes
      T pot = 0, g0 = 0, g1 = 0, g2 = 0;
      const int j = j0 + jt;
      if (j < j1) {
        const T* w = ws.w + j * 18;
        const int* ox = ws.ox + j * 6;
        const T wy = w[6 + 5], wz = w[12 + zt];
        const int oyz = wrap_up(ws.byz[2 * j] + 5, d.K1) * d.K2 + wrap_up(ws.byz[2 * j + 1] + zt, d.K2);
        T sw = 0, sdw = 0;
#pragma unroll
        for (int dx = 0; dx < 6; ++dx) {
          const T f = M[ox[dx] + oyz];
          sw += f * w[dx];
          if (FORCES) sdw += f * ws.dw[j * 18 + dx];
        }
        pot = sw * wy * wz;
        if (FORCES) {
          g0 = sdw * wy * wz;
          g1 = sw * ws.dw[j * 18 + 6 + 5] * wz;
          g2 = sw * wy * ws.dw[j * 18 + 12 + zt];
        }
      }
#pragma unroll
      for (int o = 1; o < 4; o <<= 1) {
        pot += __shfl_xor_sync(0xffffffffu, pot, o);
        if (FORCES) {
          g0 += __shfl_xor_sync(0xffffffffu, g0, o);
          g1 += __shfl_xor_sync(0xffffffffu, g1, o);
          g2 += __shfl_xor_sync(0xffffffffu, g2, o);
        }
      }
      // lane j0 + k takes the sums of atom j0 + k from lane 4 k
      const int src = 4 * ((lane - j0) & 7);
      pot = __shfl_sync(0xffffffffu, pot, src);
      if (FORCES) {
        g0 = __shfl_sync(0xffffffffu, g0, src);
        g1 = __shfl_sync(0xffffffffu, g1, src);
        g2 = __shfl_sync(0xffffffffu, g2, src);
      }
      if (lane >= j0 && lane < j1) {
        my_pot += pot;
        my_g0 += g0;
        my_g1 += g1;
        my_g2 += g2;
      }
    }
    if (lane < na) {
      const int ga = ws.atom[lane];
      if (dE_dq) dE_dq[ga] += my_pot * pot_scale;
      if (FORCES) {
        const T qa = ws.q[lane];
        // u = m0 - x + 3  ->  dE/dx_d = -q * dE/du_d ; x_d = K_d (r @ B)_d
        const double gx[3] = {-(double)qa * my_g0 * K[0], -(double)qa * my_g1 * K[1], -(double)qa * my_g2 * K[2]};
        if (dE_dpos) {
#pragma unroll
          for (int e = 0; e < 3; ++e) {
            const double v = gx[0] * g.binv[e * 3 + 0] + gx[1] * g.binv[e * 3 + 1] + gx[2] * g.binv[e * 3 + 2];
            dE_dpos[3 * (size_t)ga + e] += (T)v;
          }
        }
        const double r[3] = {(double)pos[3 * (size_t)ga], (double)pos[3 * (size_t)ga + 1],
                             (double)pos[3 * (size_t)ga + 2]};
#pragma unroll
        for (int e = 0; e < 3; ++e)
#pragma unroll
          for (int c = 0; c < 3; ++c) wf[e * 3 + c] += r[e] * gx[c];
      }
    }
    __syncwarp();
  }
  if (FORCES) block_atomic_sum<9>(wf, acc + (size_t)s * kAccStride + kAccWf, red);
}

// ---------------------------------------------------------------------------
// finalize: energy and dE/dbox = -B^T (dE/dB) B^T - E B^T   (one thread / system)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void recip_finalize_kernel(Batch b, const T* __restrict__ box, const double* __restrict__ acc,
                                      double* __restrict__ energy, T* __restrict__ dE_dbox) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.nsys) return;
  const SysDesc d = b.s[s];
  double bx[9], bi[9];
  load_box(box + (size_t)d.box_idx * 9, bx);
  inv3(bx, bi);
  const double* a = acc + (size_t)s * kAccStride;
  const double E = a[kAccErec];
  const int o = d.box_idx;
  if (energy) energy[o] += E;
  if (dE_dbox) {
    double dB[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) dB[k] = a[kAccVk + k] + a[kAccWf + k];
    // M = B^T dB B^T ; out = -M - E B^T
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double m = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
          for (int l = 0; l < 3; ++l) m += bi[k * 3 + i] * dB[k * 3 + l] * bi[j * 3 + l];
        dE_dbox[(size_t)o * 9 + i * 3 + j] += (T)(-m - E * bi[j * 3 + i]);
      }
  }
}

}  // namespace admp
