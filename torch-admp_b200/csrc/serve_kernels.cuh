// Batched kernels of the serving path: many independent systems per launch.
//
//   neighbours: per-system cell lists -> CSR rows (pstart, pcnt, col) in a
//               pair pool at caller-assigned offsets (nblist.py:335-445 set)
//   pair_ef   : warp per atom over its CSR row: Ewald real space (pme.py:312-349)
//               and Gaussian damping (qeq.py:104-119) energy, force, potential
//   csr_coef  : QEq real-space matrix entries ke (erfc(kappa r) - erfc(r / 2 eta_ij)) / r
//   sys_terms : per-system self / non-neutral / damping-self / site energies
#pragma once

#include "pme_kernels.cuh"

namespace admp {

struct SrvSys {          // per-system data of one launch (device array)
  double b[9], bi[9];
  int nc[3];
  int ncells;
  int cell_off;          // into the cell scratch
  int status;
  long long pair_off, pair_cap, pair_need;
  double rc, kappa;
  int kind;              // 0 PME, 1 QEq
  int slot;
};

template <typename T>
struct Vec4 {
  typedef float4 type;
};
template <>
struct Vec4<double> {
  typedef double4 type;
};

__device__ __forceinline__ double4 mk4(double a, double b, double c, double d) { return make_double4(a, b, c, d); }
__device__ __forceinline__ float4 mk4f(float a, float b, float c, float d) { return make_float4(a, b, c, d); }

template <typename T>
__device__ __forceinline__ typename Vec4<T>::type make_v4(T a, T b, T c, T d);
template <>
__device__ __forceinline__ float4 make_v4<float>(float a, float b, float c, float d) {
  return make_float4(a, b, c, d);
}
template <>
__device__ __forceinline__ double4 make_v4<double>(double a, double b, double c, double d) {
  return make_double4(a, b, c, d);
}

// one block per system: geometry, grid, zero the cell counters
template <typename T>
__global__ void sn_setup_kernel(Batch b, SrvSys* __restrict__ ss, const T* __restrict__ box,
                                const double* __restrict__ box64, int* __restrict__ cells) {
  const int s = blockIdx.x;
  SrvSys& S = ss[s];
  __shared__ int nc_sh[4];
  if (threadIdx.x == 0) {
    if (box64)
      load_box(box64 + (size_t)b.s[s].box_idx * 9, S.b);
    else
      load_box(box + (size_t)b.s[s].box_idx * 9, S.b);
    const double V = inv3(S.b, S.bi);
    double h[3];
    for (int d = 0; d < 3; ++d) {
      const double* u = S.b + ((d + 1) % 3) * 3;
      const double* v = S.b + ((d + 2) % 3) * 3;
      const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
      h[d] = fabs(V) / sqrt(cx * cx + cy * cy + cz * cz);
    }
    S.status = 0;
    S.pair_need = 0;
    if (!(S.rc <= fmin(h[0], fmin(h[1], h[2])) / 2.0)) S.status = ADMP_ERR_CUTOFF_TOO_LARGE;
    if (!isfinite(V) || V == 0.0) S.status = ADMP_ERR_NONFINITE;
    const int cap = 2 * b.s[s].natoms + 128;
    int nc[3];
    for (int d = 0; d < 3; ++d) {
      const double r = h[d] / S.rc;
      nc[d] = (r >= 1.0 && r < 1e6) ? (int)floor(r) : 1;
    }
    while ((long long)nc[0] * nc[1] * nc[2] > cap) {
      const int d = nc[0] >= nc[1] && nc[0] >= nc[2] ? 0 : (nc[1] >= nc[2] ? 1 : 2);
      nc[d] = (nc[d] + 1) / 2;
    }
    for (int d = 0; d < 3; ++d) S.nc[d] = nc[d];
    S.ncells = nc[0] * nc[1] * nc[2];
    nc_sh[0] = S.ncells;
  }
  __syncthreads();
  int* cnt = cells + S.cell_off;
  const int n = 3 * (nc_sh[0] + 1);
  for (int k = threadIdx.x; k < n; k += blockDim.x) cnt[k] = 0;
}

template <typename T>
static __global__ void __launch_bounds__(256)
    sn_bin_kernel(Batch b, SrvSys* __restrict__ ss, const T* __restrict__ pos, const double* __restrict__ pos64,
                  typename Vec4<T>::type* __restrict__ frac, double4* __restrict__ frac64, int* __restrict__ cell_of,
                  int* __restrict__ cells, int* __restrict__ pcnt, long long* __restrict__ pstart) {
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const SrvSys& S = ss[s];
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const long long row = S.pair_cap / (d.natoms > 0 ? d.natoms : 1);  // fixed row slot per atom
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    pcnt[i] = 0;
    pstart[i] = S.pair_off + (long long)a * row;
    if (S.status) {
      cell_of[i] = -1;
      continue;
    }
    const double r0 = pos64 ? pos64[3 * (size_t)i] : (double)pos[3 * (size_t)i];
    const double r1 = pos64 ? pos64[3 * (size_t)i + 1] : (double)pos[3 * (size_t)i + 1];
    const double r2 = pos64 ? pos64[3 * (size_t)i + 2] : (double)pos[3 * (size_t)i + 2];
    double f[3];
    int c[3];
    bool ok = isfinite(r0) && isfinite(r1) && isfinite(r2);
    for (int e = 0; e < 3; ++e) {
      f[e] = r0 * S.bi[0 * 3 + e] + r1 * S.bi[1 * 3 + e] + r2 * S.bi[2 * 3 + e];
      f[e] -= floor(f[e]);
      c[e] = ok ? min((int)(f[e] * S.nc[e]), S.nc[e] - 1) : 0;
    }
    frac[i] = make_v4<T>((T)f[0], (T)f[1], (T)f[2], T(0));
    if (frac64) frac64[i] = make_double4(f[0], f[1], f[2], 0.0);
    if (!ok) {
      cell_of[i] = -1;
      continue;
    }
    const int id = (c[0] * S.nc[1] + c[1]) * S.nc[2] + c[2];
    cell_of[i] = id;
    atomicAdd(cells + S.cell_off + id, 1);
  }
}

// block per system: exclusive scan of the cell counts -> starts
static __global__ void sn_scan_cells_kernel(SrvSys* __restrict__ ss, int* __restrict__ cells) {
  __shared__ int part[1024];
  const SrvSys& S = ss[blockIdx.x];
  const int n = S.ncells;
  int* cnt = cells + S.cell_off;
  int* start = cnt + (n + 1);
  const int nt = blockDim.x, chunk = (n + nt - 1) / nt;
  const int b0 = threadIdx.x * chunk, b1 = min(b0 + chunk, n);
  int acc = 0;
  for (int i = b0; i < b1; ++i) acc += cnt[i];
  part[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < nt; ++k) {
      const int v = part[k];
      part[k] = t;
      t += v;
    }
    start[n] = t;
  }
  __syncthreads();
  acc = part[threadIdx.x];
  for (int i = b0; i < b1; ++i) {
    start[i] = acc;
    acc += cnt[i];
  }
}

static __global__ void __launch_bounds__(256)
    sn_scatter_kernel(Batch b, const SrvSys* __restrict__ ss, const int* __restrict__ cell_of, int* __restrict__ cells,
                      int* __restrict__ sorted) {
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const SrvSys& S = ss[s];
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const int n = S.ncells;
  const int* start = cells + S.cell_off + (n + 1);
  int* cursor = cells + S.cell_off + 2 * (n + 1);
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const int i = d.atom_off + a;
    const int c = cell_of[i];
    if (c < 0) continue;
    sorted[d.atom_off + start[c] + atomicAdd(cursor + c, 1)] = i;
  }
}

__device__ __forceinline__ void sn_offsets(int nc, int* off, int& n) {
  if (nc >= 3) {
    off[0] = -1; off[1] = 0; off[2] = 1; n = 3;
  } else if (nc == 2) {
    off[0] = 0; off[1] = 1; n = 2;
  } else {
    off[0] = 0; n = 1;
  }
}

// Asynchronous 16-byte global -> shared copies (cp.async, sm_80+): the
// issuing warp does not wait for them until cp.async.wait_group.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Neighbour cells of a home cell, as a flat sequence of candidate chunks of
// up to 32 atoms (warp-uniform state).
struct SnChunk {
  int q;   // neighbour cell (index into the warp's table), nq when past the end
  int t0;  // first sorted position of the chunk
};
__device__ __forceinline__ SnChunk sn_first(const int* tb_begin, const int* tb_end, int nq) {
  SnChunk c{0, nq > 0 ? tb_begin[0] : 0};
  while (c.q < nq && c.t0 >= tb_end[c.q]) {
    ++c.q;
    if (c.q < nq) c.t0 = tb_begin[c.q];
  }
  return c;
}
__device__ __forceinline__ SnChunk sn_next(SnChunk c, const int* tb_begin, const int* tb_end, int nq) {
  if (c.q >= nq) return c;
  c.t0 += 32;
  while (c.q < nq && c.t0 >= tb_end[c.q]) {
    ++c.q;
    if (c.q < nq) c.t0 = tb_begin[c.q];
  }
  return c;
}

// Warp per home cell: lane l takes home atom l of the cell (chunks of 32).
// The warp streams the atoms of the (up to 27) neighbour cells through a
// double buffer in shared memory, 32 at a time: the sorted indices of chunk
// k + 2 are loaded and the positions of chunk k + 1 copied asynchronously
// while every lane tests its atom against chunk k with broadcast loads, so
// the search runs at instruction rate instead of waiting on dependent global
// loads per candidate.  Rows keep the order of a per-atom scan: neighbour
// cells in (x, y, z) offset order, candidates in sorted order.  One pass:
// each atom writes its neighbours into its fixed row slot col[pstart[i] ..]
// (pstart from sn_bin_kernel, row = pair_cap / natoms) and pcnt[i]; a row
// that would overflow its slot keeps the first `row` entries, sets the
// system's status to ADMP_ERR_CAPACITY and raises pair_need to natoms x
// (longest row).  Unbinned atoms keep pcnt = 0.
// The cutoff decision is the double-precision one (frac64) whenever frac64 is
// given: candidates are first tested in T with a margin far above T's
// rounding error of r^2, and only those inside the margin band around rc^2 or
// the 1e-4 overlap threshold are re-tested in double.
template <typename T>
static __global__ void __launch_bounds__(256)
    sn_pairs_kernel(Batch b, SrvSys* __restrict__ ss, const typename Vec4<T>::type* __restrict__ frac,
                    const double4* __restrict__ frac64, const int* __restrict__ cell_of, const int* __restrict__ cells,
                    const int* __restrict__ sorted, int* __restrict__ pcnt, const long long* __restrict__ pstart,
                    int* __restrict__ col) {
  typedef typename Vec4<T>::type V4;
  constexpr int kV4Chunks = sizeof(V4) / 16;
  __shared__ __align__(16) V4 cand[8][2][32];
  __shared__ int cand_j[8][2][32];
  __shared__ int tb_begin[8][27], tb_end[8][27], tb_shift[8][27];
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  SrvSys& S = ss[s];
  if (S.status) return;  // sn_bin_kernel left every count of a failed system at zero
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const long long row = S.pair_cap / (d.natoms > 0 ? d.natoms : 1);
  const int n = S.ncells;
  const int* start = cells + S.cell_off + (n + 1);
  const double rc2 = S.rc * S.rc;
  const int nc0 = S.nc[0], nc1 = S.nc[1], nc2 = S.nc[2];
  int n0, n1, n2;
  {
    int o[3];
    sn_offsets(nc0, o, n0);
    sn_offsets(nc1, o, n1);
    sn_offsets(nc2, o, n2);
  }
  const int nq = n0 * n1 * n2;
  T bt[9];
  double bsum = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    bt[k] = (T)S.b[k];
    bsum += fabs(S.b[k]);
  }
  const T rc2t = (T)rc2;
  // |r^2_T - r^2| <= 2 r |dr| with |dr| <= (a few ulp of a fraction) * sum |B|
  const T mg = frac64 ? (T)(1e-3 * rc2 + 1e-5 * S.rc * bsum) : T(0);
  const T lo = rc2t - mg, hi = rc2t + mg, small = frac64 ? T(2e-3) : T(1e-4);
  // with >= 3 cells on every axis the image of a candidate is fixed by its
  // cell's wrap, so no rounding to the nearest image is needed
  const bool fast = nc0 >= 3 && nc1 >= 3 && nc2 >= 3;
  const bool ortho = S.b[1] == 0.0 && S.b[2] == 0.0 && S.b[3] == 0.0 && S.b[5] == 0.0 && S.b[6] == 0.0 &&
                     S.b[7] == 0.0;
  const int* srt = sorted + d.atom_off;
  int* tbb = tb_begin[warp];
  int* tbe = tb_end[warp];
  int* tbs = tb_shift[warp];
  const int nwarps_sys = ((d.natoms + b.apb - 1) / b.apb) * nw;
  for (int c = (blockIdx.x - d.blk_atom) * nw + warp; c < n; c += nwarps_sys) {
    const int h_begin = start[c], h_end = start[c + 1];
    if (h_begin >= h_end) continue;
    const int c0 = c / (nc1 * nc2), c1 = (c / nc2) % nc1, c2 = c % nc2;
    // table of neighbour cells: lane q < nq takes offset q in (x, y, z) order
    __syncwarp();
    if (lane < nq) {
      const int q2 = lane % n2, q1 = (lane / n2) % n1, q0 = lane / (n1 * n2);
      int xyz[3] = {c0 + (n0 == 3 ? q0 - 1 : q0), c1 + (n1 == 3 ? q1 - 1 : q1), c2 + (n2 == 3 ? q2 - 1 : q2)};
      const int ncs[3] = {nc0, nc1, nc2};
      int code = 0;
#pragma unroll
      for (int e = 0; e < 3; ++e) {
        int sh = 0;
        if (xyz[e] < 0) {
          xyz[e] += ncs[e];
          sh = -1;
        } else if (xyz[e] >= ncs[e]) {
          xyz[e] -= ncs[e];
          sh = 1;
        }
        code |= (sh + 1) << (2 * e);
      }
      const int cc = (xyz[0] * nc1 + xyz[1]) * nc2 + xyz[2];
      tbb[lane] = start[cc];
      tbe[lane] = start[cc + 1];
      tbs[lane] = code;
    }
    __syncwarp();
    for (int h0 = h_begin; h0 < h_end; h0 += 32) {
      const bool home = h0 + lane < h_end;
      const int i = home ? srt[h0 + lane] : -1;
      V4 fi;
      if (home) {
        fi = frac[i];
      } else {
        fi.x = fi.y = fi.z = fi.w = T(0);
      }
      const long long base = home ? pstart[i] : 0;
      int cnt = 0;
      // prologue: indices of chunks 0 and 1, positions of chunk 0 in flight
      SnChunk cur = sn_first(tbb, tbe, nq);
      SnChunk nxt = sn_next(cur, tbb, tbe, nq);
      int bsel = 0;
      {
        const int j = (cur.q < nq && cur.t0 + lane < tbe[cur.q]) ? srt[cur.t0 + lane] : -1;
        cand_j[warp][0][lane] = j;
        if (j >= 0)
#pragma unroll
          for (int h = 0; h < kV4Chunks; ++h)
            cp_async16(reinterpret_cast<char*>(&cand[warp][0][lane]) + 16 * h,
                       reinterpret_cast<const char*>(frac + j) + 16 * h);
        cp_async_commit();
      }
      int jn = (nxt.q < nq && nxt.t0 + lane < tbe[nxt.q]) ? srt[nxt.t0 + lane] : -1;
      while (cur.q < nq) {
        const SnChunk nxt2 = sn_next(nxt, tbb, tbe, nq);
        // positions of the next chunk into the other buffer (one group per trip, empty at the end)
        cand_j[warp][bsel ^ 1][lane] = jn;
        if (jn >= 0)
#pragma unroll
          for (int h = 0; h < kV4Chunks; ++h)
            cp_async16(reinterpret_cast<char*>(&cand[warp][bsel ^ 1][lane]) + 16 * h,
                       reinterpret_cast<const char*>(frac + jn) + 16 * h);
        cp_async_commit();
        const int jn2 = (nxt2.q < nq && nxt2.t0 + lane < tbe[nxt2.q]) ? srt[nxt2.t0 + lane] : -1;
        cp_async_wait1();  // this chunk's copies have landed
        __syncwarp();
        if (home) {
          const int code = tbs[cur.q];
          const T s0 = T((code & 3) - 1), s1 = T(((code >> 2) & 3) - 1), s2 = T(((code >> 4) & 3) - 1);
          const T g0 = s0 - fi.x, g1 = s1 - fi.y, g2 = s2 - fi.z;
          const int nt = min(32, tbe[cur.q] - cur.t0);
          const V4* cw = cand[warp][bsel];
          const int* cj = cand_j[warp][bsel];
          for (int k = 0; k < nt; ++k) {
            const int j = cj[k];
            if (j == i) continue;
            const V4 fj = cw[k];
            T f0 = fj.x + g0, f1 = fj.y + g1, f2 = fj.z + g2;
            if (!fast) {
              f0 -= floor(f0 + T(0.5));
              f1 -= floor(f1 + T(0.5));
              f2 -= floor(f2 + T(0.5));
            }
            T r2;
            if (ortho) {
              const T v0 = f0 * bt[0], v1 = f1 * bt[4], v2 = f2 * bt[8];
              r2 = v0 * v0 + v1 * v1 + v2 * v2;
            } else {
              r2 = 0;
#pragma unroll
              for (int e = 0; e < 3; ++e) {
                const T v = f0 * bt[e] + f1 * bt[3 + e] + f2 * bt[6 + e];
                r2 += v * v;
              }
            }
            bool in;
            if (r2 > hi) {
              in = false;
            } else if (r2 < lo && r2 > small) {
              in = true;
            } else if (!frac64) {
              in = r2 < rc2t && r2 > T(1e-4);
            } else {
              const double4 gi = frac64[i], gj = frac64[j];
              double df[3] = {gj.x - gi.x, gj.y - gi.y, gj.z - gi.z};
              for (int e = 0; e < 3; ++e) df[e] -= floor(df[e] + 0.5);
              double rr = 0.0;
              for (int e = 0; e < 3; ++e) {
                const double v = df[0] * S.b[0 * 3 + e] + df[1] * S.b[1 * 3 + e] + df[2] * S.b[2 * 3 + e];
                rr += v * v;
              }
              in = rr < rc2 && rr > 1e-4;
            }
            if (in) {
              if (cnt < row) col[base + cnt] = j;
              ++cnt;
            }
          }
        }
        __syncwarp();  // this buffer is refilled two trips later
        cur = nxt;
        nxt = nxt2;
        jn = jn2;
        bsel ^= 1;
      }
      if (home) {
        pcnt[i] = cnt < row ? cnt : (int)row;
        if (cnt > row) {
          S.status = ADMP_ERR_CAPACITY;  // every writer stores the same value
          atomicMax(&S.pair_need, (long long)d.natoms * cnt);
        }
      }
    }
  }
}

// thread per system: status and the pair entries a system needs (natoms x
// longest row when a row overflowed its slot) to slot_info
static __global__ void sn_export_kernel(Batch b, const SrvSys* __restrict__ ss, int* __restrict__ slot_info) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= b.nsys || !slot_info) return;
  const SrvSys& S = ss[s];
  int* si = slot_info + 4 * b.s[s].box_idx;
  si[2] = S.status;
  const long long need = S.pair_need;
  si[3] = (int)(need < 2147483647LL ? need : 2147483647LL);
}

// minimum-image Cartesian displacement r_j - r_i from wrapped fractional coords
template <typename V4>
__device__ __forceinline__ void disp(const V4& fi, const V4& fj, const double* bx, float* dr) {
  float df[3] = {fj.x - fi.x, fj.y - fi.y, fj.z - fi.z};
#pragma unroll
  for (int e = 0; e < 3; ++e) df[e] -= floorf(df[e] + 0.5f);
#pragma unroll
  for (int e = 0; e < 3; ++e) dr[e] = df[0] * (float)bx[e] + df[1] * (float)bx[3 + e] + df[2] * (float)bx[6 + e];
}
template <typename V4>
__device__ __forceinline__ void disp(const V4& fi, const V4& fj, const double* bx, double* dr) {
  double df[3] = {fj.x - fi.x, fj.y - fi.y, fj.z - fi.z};
#pragma unroll
  for (int e = 0; e < 3; ++e) df[e] -= floor(df[e] + 0.5);
#pragma unroll
  for (int e = 0; e < 3; ++e) dr[e] = df[0] * bx[e] + df[1] * bx[3 + e] + df[2] * bx[6 + e];
}

// warp per atom: real-space Ewald (+ damping for QEq systems) energy, gradient, potential
template <typename T>
static __global__ void __launch_bounds__(256)
    pair_ef_kernel(Batch b, const SrvSys* __restrict__ ss, const typename Vec4<T>::type* __restrict__ frac,
                   const double4* __restrict__ frac64, const T* __restrict__ q, const T* __restrict__ eta,
                   const long long* __restrict__ pstart, const int* __restrict__ pcnt, const int* __restrict__ col,
                   double ke, T* __restrict__ grad, double* __restrict__ energy) {
  __shared__ double bx[9];
  __shared__ double red[32];
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const SrvSys& S = ss[s];
  if (threadIdx.x < 9) bx[threadIdx.x] = S.b[threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const T kappa = (T)S.kappa, kt = (T)ke;
  const T tsp = T(2.0 / kSqrtPi);
  const bool damp = S.kind == 1 && eta != nullptr;
  double e_acc = 0.0;
  if (!S.status) {
    for (int a = a0 + warp; a < a1; a += blockDim.x >> 5) {
      const int i = d.atom_off + a;
      const typename Vec4<T>::type fi = frac[i];
      const double4 fi64 = frac64 ? frac64[i] : make_double4(0, 0, 0, 0);
      const T qi = q[i];
      const T ei = damp ? eta[i] : T(0);
      const long long st = pstart[i];
      const int n = pcnt[i];
      T g0 = 0, g1 = 0, g2 = 0, e = 0;
      // three entries per lane per trip, their loads issued before any is used
      for (int k0 = 0; k0 < n; k0 += 96) {
        int jj[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int k = k0 + lane + 32 * u;
          jj[u] = k < n ? col[st + k] : -1;
        }
        T drr[3][3], qjj[3], ejj[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          const int j = jj[u] >= 0 ? jj[u] : i;
          if (frac64) {
            // displacement from double coordinates: close pairs keep full relative precision
            double d64[3];
            disp(fi64, frac64[j], bx, d64);
            drr[u][0] = (T)d64[0];
            drr[u][1] = (T)d64[1];
            drr[u][2] = (T)d64[2];
          } else {
            disp(fi, frac[j], bx, drr[u]);
          }
          qjj[u] = q[j];
          ejj[u] = damp ? eta[j] : T(0);
        }
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          if (jj[u] < 0) continue;
          const T* dr = drr[u];
          const T r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
          const T r = sqrt_t(r2);
          const T inv = T(1) / r;
          const T qq = qi * qjj[u] * kt;
          const T x = kappa * r;
          const T er = erfc_t(x);
          T ep = er * inv;
          T dd = -tsp * kappa * exp_t(-x * x) * inv - er * inv * inv;
          if (damp) {
            const T ej = ejj[u];
            T eij = sqrt_t((ei * ei + ej * ej) * T(0.5));
            if (eij == T(0)) eij = T(1e-10);
            const T y = r / (T(2) * eij);
            const T ed = erfc_t(y);
            ep -= ed * inv;
            dd += tsp * exp_t(-y * y) / (T(2) * eij) * inv + ed * inv * inv;
          }
          e += qq * ep;
          // dE/dr_i = dE/dr * d r / d r_i = dd * qq * (-(r_j - r_i) / r)
          const T gs = -dd * qq * inv;
          g0 += gs * dr[0];
          g1 += gs * dr[1];
          g2 += gs * dr[2];
        }
      }
      e = warp_sum(e);
      g0 = warp_sum(g0);
      g1 = warp_sum(g1);
      g2 = warp_sum(g2);
      if (lane == 0) {
        grad[3 * (size_t)i] += g0;
        grad[3 * (size_t)i + 1] += g1;
        grad[3 * (size_t)i + 2] += g2;
        e_acc += 0.5 * (double)e;  // each pair appears in both rows
      }
    }
  }
  double v[1] = {e_acc};
  block_atomic_sum<1>(v, energy + d.box_idx, red);
}

// QEq real-space matrix entries (CSR)
template <typename T>
static __global__ void __launch_bounds__(256)
    csr_coef_kernel(Batch b, const SrvSys* __restrict__ ss, const typename Vec4<T>::type* __restrict__ frac,
                    const T* __restrict__ eta, const long long* __restrict__ pstart, const int* __restrict__ pcnt,
                    const int* __restrict__ col, double ke, T* __restrict__ coef) {
  __shared__ double bx[9];
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const SrvSys& S = ss[s];
  if (threadIdx.x < 9) bx[threadIdx.x] = S.b[threadIdx.x];
  __syncthreads();
  if (S.status) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  const T kappa = (T)S.kappa;
  for (int a = a0 + warp; a < a1; a += blockDim.x >> 5) {
    const int i = d.atom_off + a;
    const typename Vec4<T>::type fi = frac[i];
    const T ei = eta[i];
    const long long st = pstart[i];
    const int n = pcnt[i];
    // three entries per lane per trip, their loads issued before any is used
    for (int k0 = 0; k0 < n; k0 += 96) {
      int jj[3];
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        const int k = k0 + lane + 32 * u;
        jj[u] = k < n ? col[st + k] : -1;
      }
      T drr[3][3], ejj[3];
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        const int j = jj[u] >= 0 ? jj[u] : i;
        disp(fi, frac[j], bx, drr[u]);
        ejj[u] = eta[j];
      }
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        if (jj[u] < 0) continue;
        const T* dr = drr[u];
        const T r = sqrt_t(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        T eij = sqrt_t((ei * ei + ejj[u] * ejj[u]) * T(0.5));
        if (eij == T(0)) eij = T(1e-10);
        coef[st + k0 + lane + 32 * u] = (T)ke * (erfc_t(kappa * r) - erfc_t(r / (T(2) * eij))) / r;
      }
    }
  }
}

// CSR SpMV layout (csr_spmv_finish_kernel): eight lanes per row, four rows
// per warp at a time; each lane issues the loads of up to kSpmvUnroll entries
// of its row before using any of them, so a row costs about three dependent
// memory latencies (row start, entries, gathered p) instead of three per 32
// entries: the SpMV is bound by the latency of those chains, not by bytes.
constexpr int kSpmvLanes = 8;
constexpr int kSpmvUnroll = 12;

// block per system: self + non-neutral (+ damping self + site for QEq systems)
template <typename T>
__global__ void __launch_bounds__(512)
    sys_terms_kernel(Batch b, const SrvSys* __restrict__ ss, const T* __restrict__ q, const T* __restrict__ chi,
                     const T* __restrict__ hard, const T* __restrict__ eta, double ke, double* __restrict__ energy) {
  __shared__ double red[4 * 32];
  __shared__ double sums[4];
  const SysDesc d = b.s[blockIdx.x];
  const SrvSys& S = ss[blockIdx.x];
  if (threadIdx.x < 4) sums[threadIdx.x] = 0.0;
  __syncthreads();
  const bool qeq = S.kind == 1;
  double v[4] = {0, 0, 0, 0};
  for (int a = threadIdx.x; a < d.natoms; a += blockDim.x) {
    const int i = d.atom_off + a;
    const double qi = q[i];
    v[0] += qi;
    v[1] += qi * qi;
    if (qeq) {
      const double e = eta[i];
      v[2] += (fabs(e) > 1e-4 ? 1.0 / e : 0.0) / (2.0 * kSqrtPi) * qi * qi;
      v[3] += (double)chi[i] * qi + (double)hard[i] * qi * qi;
    }
  }
  block_atomic_sum<4>(v, sums, red);
  if (threadIdx.x == 0) {
    const double V = fabs(S.b[0] * (S.b[4] * S.b[8] - S.b[5] * S.b[7]) - S.b[1] * (S.b[3] * S.b[8] - S.b[5] * S.b[6]) +
                          S.b[2] * (S.b[3] * S.b[7] - S.b[4] * S.b[6]));
    const double kap = S.kappa;
    double E = -ke * kap / kSqrtPi * sums[1] - kPi / (2.0 * V * kap * kap) * ke * sums[0] * sums[0];
    if (qeq) E += ke * sums[2] + sums[3];
    energy[d.box_idx] += E;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) zero_atoms_kernel(Batch b, T* __restrict__ a3, double* __restrict__ energy) {
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const size_t i = (size_t)(d.atom_off + a);
    a3[3 * i] = T(0);
    a3[3 * i + 1] = T(0);
    a3[3 * i + 2] = T(0);
  }
  if (threadIdx.x == 0 && blockIdx.x == d.blk_atom) energy[d.box_idx] = 0.0;
}

template <typename T>
__global__ void __launch_bounds__(256) negate_atoms_kernel(Batch b, T* __restrict__ a3) {
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  const SysDesc d = b.s[s];
  const int a0 = (blockIdx.x - d.blk_atom) * b.apb;
  const int a1 = min(a0 + b.apb, d.natoms);
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const size_t i = (size_t)(d.atom_off + a);
    a3[3 * i] = -a3[3 * i];
    a3[3 * i + 1] = -a3[3 * i + 1];
    a3[3 * i + 2] = -a3[3 * i + 2];
  }
}

}  // namespace admp
