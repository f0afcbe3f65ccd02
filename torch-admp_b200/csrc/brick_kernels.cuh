// Brick-privatised spread and gather for atoms binned in neighbour cells
// (the serving path, whose neighbour build sorts every system's atoms by
// cell).  Same arithmetic as spread_kernel / gather_kernel (recip.py:146-252
// and the autograd of pme.py:351-446); only the memory traffic differs.
//
// A brick is a run of G cells along z inside one (x, y) cell column.  The
// stencils of its atoms cover a box of mesh points ("tile"): the brick's
// mesh extent plus the 6-point stencil reach, or the whole period along an
// axis where that box would wrap onto itself.  spread accumulates the tile
// in shared memory and adds it to the mesh row by row (coalesced global
// reductions, one per tile point instead of 216 scattered ones per atom);
// gather loads the tile once and every atom reads its 216 points from shared
// memory.  An atom whose stencil falls outside its brick's tile (possible
// only within rounding of a cell face, since the binning and the stencil
// compute the fractional coordinate from different copies of the position)
// takes the direct global path, so the result never depends on the binning.
//
// Cell table per slot (written by the neighbour build): [0..2] cells per
// axis, [3] 1 when valid, [4 ..] start of each cell's atoms in the system's
// cell-sorted order (ncells + 1 entries).
#pragma once

#include "pme_kernels.cuh"

namespace admp {

constexpr int kCellHdr = 4;

// tile capacity (elements of T) per kernel: shared memory is the tile plus
// 8 warps' stencils, sized for two blocks per SM
template <typename T, bool FORCES>
__host__ __device__ constexpr int brick_cap() {
  return sizeof(T) == 4 ? (FORCES ? 16000 : 18000) : (FORCES ? 8000 : 9000);
}

struct TileAxis {
  int o, w, K;
  bool full;
};

// Tile axis for cells [c0, c1) of nc cells over K mesh points.  An atom of
// cell c has x = K f, f in [c / nc, (c + 1) / nc), so m0 = ceil(x) lies in
// [ceil(K c0 / nc), ceil(K c1 / nc)] and its stencil m0 - 3 .. m0 + 2.
__device__ __forceinline__ TileAxis tile_axis(int K, int nc, int c0, int c1) {
  TileAxis a;
  a.K = K;
  const int lo = (int)(((long long)K * c0 + nc - 1) / nc) - 3;
  const int hi = (int)(((long long)K * c1 + nc - 1) / nc) + 2;
  a.w = hi - lo + 1;
  a.full = a.w >= K;
  if (a.full) {
    a.o = 0;
    a.w = K;
  } else {
    a.o = wrap_index(lo, K);
  }
  return a;
}

// widest tile of g cells along an axis (any c0): ceil(K g / nc) + 6, at most K
__device__ __forceinline__ int tile_wmax(int K, int nc, int g) {
  const int w = (int)(((long long)K * g + nc - 1) / nc) + 6;
  return w < K ? w : K;
}

// tile coordinate of a wrapped stencil base b (0 <= b < K), or -1 when the
// six points b .. b + 5 do not all lie inside the tile
__device__ __forceinline__ int tile_start(const TileAxis& a, int b) {
  if (a.full) return b;
  int t = b - a.o;
  if (t < 0) t += a.K;
  return t + 5 < a.w ? t : -1;
}

__device__ __forceinline__ int tile_at(const TileAxis& a, int t, int k) {
  int v = t + k;
  if (a.full && v >= a.K) v -= a.K;
  return v;
}

// mesh index along the axis of tile coordinate t
__device__ __forceinline__ int tile_mesh(const TileAxis& a, int t) {
  if (a.full) return t;
  int v = a.o + t;
  return v >= a.K ? v - a.K : v;
}

// Brick layout of one system: G cells per brick along z, as many as fit the
// capacity; G = 0 when even one cell does not fit (the system then takes the
// direct kernels' path).
struct BrickPlan {
  int nc0, nc1, nc2, G, ngz, nbricks;
};

__device__ __forceinline__ BrickPlan brick_plan(const int* ct, const SysDesc& d, int cap) {
  BrickPlan p;
  p.nc0 = ct[0];
  p.nc1 = ct[1];
  p.nc2 = ct[2];
  p.G = 0;
  p.ngz = 0;
  p.nbricks = 0;
  if (ct[3] != 1 || p.nc0 <= 0 || p.nc1 <= 0 || p.nc2 <= 0) return p;
  const long long wxy = (long long)tile_wmax(d.K0, p.nc0, 1) * tile_wmax(d.K1, p.nc1, 1);
  for (int g = p.nc2; g >= 1; --g)
    if (wxy * tile_wmax(d.K2, p.nc2, g) <= cap) {
      p.G = g;
      break;
    }
  if (p.G > 0) {
    p.ngz = (p.nc2 + p.G - 1) / p.G;
    p.nbricks = p.nc0 * p.nc1 * p.ngz;
  }
  return p;
}

struct Brick {
  TileAxis ax, ay, az;
  int a0, a1;  // atom range in the system's cell-sorted order
};

__device__ __forceinline__ Brick brick_at(const int* ct, const SysDesc& d, const BrickPlan& p, int br) {
  Brick k;
  const int col = br / p.ngz, gz = br - col * p.ngz;
  const int cx = col / p.nc1, cy = col - cx * p.nc1;
  const int cz0 = gz * p.G, cz1 = min(cz0 + p.G, p.nc2);
  k.ax = tile_axis(d.K0, p.nc0, cx, cx + 1);
  k.ay = tile_axis(d.K1, p.nc1, cy, cy + 1);
  k.az = tile_axis(d.K2, p.nc2, cz0, cz1);
  const int* start = ct + kCellHdr;
  k.a0 = start[col * p.nc2 + cz0];
  k.a1 = start[col * p.nc2 + cz1];
  return k;
}

// Per-warp stencils of 32 atoms: 18 weights (and derivatives), the wrapped
// stencil bases per axis, the charge and the atom index.
template <typename T, bool DERIV>
struct BrickStencil {
  T* w;      // [32][18]
  T* dw;     // [32][18]
  T* q;      // [32]
  int* b3;   // [32][3]
  int* atom; // [32]
  __host__ __device__ static constexpr size_t bytes() {
    return 32 * 18 * sizeof(T) * (DERIV ? 2 : 1) + 32 * sizeof(T) + 32 * 3 * sizeof(int) + 32 * sizeof(int) + 16;
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
    b3 = reinterpret_cast<int*>(q + 32);
    atom = b3 + 32 * 3;
  }
};

template <typename T, bool DERIV>
__device__ __forceinline__ void brick_build_stencil(BrickStencil<T, DERIV>& ws, const SysDesc& d, const Geom& g,
                                                    const T* __restrict__ pos, const T* __restrict__ q,
                                                    const int* __restrict__ order, int a_first, int a_end,
                                                    int lane) {
  const int a = a_first + lane;
  if (a < a_end) {
    const int ga = order[d.atom_off + a];
    T r[3] = {pos[3 * (size_t)ga], pos[3 * (size_t)ga + 1], pos[3 * (size_t)ga + 2]};
    Stencil<T> st;
    make_stencil<T>(r, g, d.K0, d.K1, d.K2, st);
    T* w = ws.w + lane * 18;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      w[k] = st.w[0][k];
      w[6 + k] = st.w[1][k];
      w[12 + k] = st.w[2][k];
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
    ws.b3[lane * 3] = st.ix[0];
    ws.b3[lane * 3 + 1] = st.iy[0];
    ws.b3[lane * 3 + 2] = st.iz[0];
    ws.q[lane] = q ? q[ga] : T(0);
    ws.atom[lane] = ga;
  }
  __syncwarp();
}

template <typename T, bool FORCES>
inline size_t brick_smem() {
  return (size_t)brick_cap<T, FORCES>() * sizeof(T) + 8 * BrickStencil<T, FORCES>::bytes() + 64;
}

// ---------------------------------------------------------------------------
// spread into the zeroed mesh
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 2) spread_brick_kernel(Batch b, const T* __restrict__ pos,
                                                           const T* __restrict__ box, const T* __restrict__ q,
                                                           T* __restrict__ mesh, const int* __restrict__ order,
                                                           const int* __restrict__ cells, int cell_stride) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Geom g;
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];
  constexpr int cap = brick_cap<T, false>();
  T* tile = reinterpret_cast<T*>(dsm);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  BrickStencil<T, false> ws;
  ws.carve(dsm + (size_t)cap * sizeof(T) + warp * BrickStencil<T, false>::bytes());
  load_geom(box, d.box_idx, &g);
  __syncthreads();
  const int* ct = cells + (size_t)d.box_idx * cell_stride;
  const BrickPlan p = brick_plan(ct, d, cap);
  const int jb = blockIdx.x - d.blk_atom;
  const int nblk = (d.natoms + b.apb - 1) / b.apb;
  T* M = mesh + d.mesh_off;
  const int K1K2 = d.K1 * d.K2;
  // lanes over the first 32 (y, z) stencil columns; the last four columns of eight atoms in one pass
  const int y0 = lane / 6, z0 = lane % 6, jt = lane >> 2, zt = 2 + (lane & 3);
  if (p.G == 0) {  // no brick fits: this block's chunk of the sorted atoms with global reductions
    const int a_begin = jb * b.apb, a_end = min(a_begin + b.apb, d.natoms);
    for (int a0 = a_begin + warp * 32; a0 < a_end; a0 += nw * 32) {
      brick_build_stencil<T, false>(ws, d, g, pos, q, order, a0, a_end, lane);
      const int na = min(32, a_end - a0);
      for (int j = 0; j < na; ++j) {
        const T qa = ws.q[j];
        const T* w = ws.w + j * 18;
        for (int c = lane; c < 36; c += 32) {
          const int yy = c / 6, zz = c - 6 * (c / 6);
          const T wyz = qa * w[6 + yy] * w[12 + zz];
          const int oyz = wrap_up(ws.b3[3 * j + 1] + yy, d.K1) * d.K2 + wrap_up(ws.b3[3 * j + 2] + zz, d.K2);
#pragma unroll
          for (int dx = 0; dx < 6; ++dx) atomicAdd(M + wrap_up(ws.b3[3 * j] + dx, d.K0) * K1K2 + oyz, w[dx] * wyz);
        }
      }
      __syncwarp();
    }
    return;
  }
  for (int br = jb; br < p.nbricks; br += nblk) {
    const Brick k = brick_at(ct, d, p, br);
    const int n = k.ax.w * k.ay.w * k.az.w;
    const int wyz = k.ay.w * k.az.w;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tile[i] = T(0);
    __syncthreads();
    for (int a0 = k.a0 + warp * 32; a0 < k.a1; a0 += nw * 32) {
      brick_build_stencil<T, false>(ws, d, g, pos, q, order, a0, k.a1, lane);
      const int na = min(32, k.a1 - a0);
      for (int j0 = 0; j0 < na; j0 += 8) {
        const int j1 = min(j0 + 8, na);
        for (int j = j0; j < j1; ++j) {
          const T qa = ws.q[j];
          if (qa == T(0)) continue;
          const T* w = ws.w + j * 18;
          const int* bb = ws.b3 + 3 * j;
          const int tx = tile_start(k.ax, bb[0]), ty = tile_start(k.ay, bb[1]), tz = tile_start(k.az, bb[2]);
          const T v = qa * w[6 + y0] * w[12 + z0];
          if (tx >= 0 && ty >= 0 && tz >= 0) {
            const int oyz = tile_at(k.ay, ty, y0) * k.az.w + tile_at(k.az, tz, z0);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) atomicAdd(tile + tile_at(k.ax, tx, dx) * wyz + oyz, w[dx] * v);
          } else {
            const int oyz = wrap_up(bb[1] + y0, d.K1) * d.K2 + wrap_up(bb[2] + z0, d.K2);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) atomicAdd(M + wrap_up(bb[0] + dx, d.K0) * K1K2 + oyz, w[dx] * v);
          }
        }
        const int j = j0 + jt;
        if (j < j1) {
          const T qa = ws.q[j];
          if (qa != T(0)) {
            const T* w = ws.w + j * 18;
            const int* bb = ws.b3 + 3 * j;
            const int tx = tile_start(k.ax, bb[0]), ty = tile_start(k.ay, bb[1]), tz = tile_start(k.az, bb[2]);
            const T v = qa * w[6 + 5] * w[12 + zt];
            if (tx >= 0 && ty >= 0 && tz >= 0) {
              const int oyz = tile_at(k.ay, ty, 5) * k.az.w + tile_at(k.az, tz, zt);
#pragma unroll
              for (int dx = 0; dx < 6; ++dx) atomicAdd(tile + tile_at(k.ax, tx, dx) * wyz + oyz, w[dx] * v);
            } else {
              const int oyz = wrap_up(bb[1] + 5, d.K1) * d.K2 + wrap_up(bb[2] + zt, d.K2);
#pragma unroll
              for (int dx = 0; dx < 6; ++dx) atomicAdd(M + wrap_up(bb[0] + dx, d.K0) * K1K2 + oyz, w[dx] * v);
            }
          }
        }
      }
      __syncwarp();
    }
    __syncthreads();
    // add the tile to the mesh, one warp per tile row (consecutive z)
    for (int r = warp; r < k.ax.w * k.ay.w; r += nw) {
      const int tx = r / k.ay.w, ty = r - tx * k.ay.w;
      T* row = M + (size_t)tile_mesh(k.ax, tx) * K1K2 + (size_t)tile_mesh(k.ay, ty) * d.K2;
      const T* src = tile + (size_t)r * k.az.w;
      for (int tz = lane; tz < k.az.w; tz += 32) {
        const T v = src[tz];
        if (v != T(0)) atomicAdd(row + tile_mesh(k.az, tz), v);
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// gather: pot_i = sum phi theta; dE/du_d = q sum phi dtheta/du_d
// ---------------------------------------------------------------------------
template <typename T, bool FORCES>
__global__ void __launch_bounds__(256, 2) gather_brick_kernel(Batch b, const T* __restrict__ pos,
                                                           const T* __restrict__ box, const T* __restrict__ q,
                                                           const T* __restrict__ phi, T* __restrict__ dE_dq,
                                                           T* __restrict__ dE_dpos, double* __restrict__ acc,
                                                           T pot_scale, const int* __restrict__ order,
                                                           const int* __restrict__ cells, int cell_stride) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Geom g;
  __shared__ double red[9 * 32];
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];
  constexpr int cap = brick_cap<T, FORCES>();
  T* tile = reinterpret_cast<T*>(dsm);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  BrickStencil<T, FORCES> ws;
  ws.carve(dsm + (size_t)cap * sizeof(T) + warp * BrickStencil<T, FORCES>::bytes());
  load_geom(box, d.box_idx, &g);
  __syncthreads();
  const int* ct = cells + (size_t)d.box_idx * cell_stride;
  const BrickPlan p = brick_plan(ct, d, cap);
  const int jb = blockIdx.x - d.blk_atom;
  const int nblk = (d.natoms + b.apb - 1) / b.apb;
  const T* M = phi + d.mesh_off;
  const int K1K2 = d.K1 * d.K2;
  const int K[3] = {d.K0, d.K1, d.K2};
  const int y0 = lane / 6, z0 = lane % 6, jt = lane >> 2, zt = 2 + (lane & 3);
  double wf[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) wf[e] = 0.0;
  // without bricks (G = 0) the block makes one pass over its chunk of the sorted atoms, reading the mesh
  const bool direct = p.G == 0;
  const int first = direct ? 0 : jb, last = direct ? 1 : p.nbricks, step = direct ? 1 : nblk;
  for (int br = first; br < last; br += step) {
    Brick k;
    if (direct) {
      k.a0 = jb * b.apb;
      k.a1 = min(k.a0 + b.apb, d.natoms);
    } else {
      k = brick_at(ct, d, p, br);
      // load the tile, one warp per row of consecutive z
      for (int r = warp; r < k.ax.w * k.ay.w; r += nw) {
        const int tx = r / k.ay.w, ty = r - tx * k.ay.w;
        const T* row = M + (size_t)tile_mesh(k.ax, tx) * K1K2 + (size_t)tile_mesh(k.ay, ty) * d.K2;
        T* dst = tile + (size_t)r * k.az.w;
        for (int tz = lane; tz < k.az.w; tz += 32) dst[tz] = row[tile_mesh(k.az, tz)];
      }
      __syncthreads();
    }
    for (int a0 = k.a0 + warp * 32; a0 < k.a1; a0 += nw * 32) {
      brick_build_stencil<T, FORCES>(ws, d, g, pos, q, order, a0, k.a1, lane);
      const int na = min(32, k.a1 - a0);
      T my_pot = 0, my_g0 = 0, my_g1 = 0, my_g2 = 0;
      for (int j0 = 0; j0 < na; j0 += 8) {
        const int j1 = min(j0 + 8, na);
        for (int j = j0; j < j1; ++j) {
          const T* w = ws.w + j * 18;
          const int* bb = ws.b3 + 3 * j;
          T f[6];
          const int tx = direct ? -1 : tile_start(k.ax, bb[0]);
          const int ty = direct ? -1 : tile_start(k.ay, bb[1]);
          const int tz = direct ? -1 : tile_start(k.az, bb[2]);
          if (tx >= 0 && ty >= 0 && tz >= 0) {
            const int wyz = k.ay.w * k.az.w;
            const int oyz = tile_at(k.ay, ty, y0) * k.az.w + tile_at(k.az, tz, z0);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) f[dx] = tile[tile_at(k.ax, tx, dx) * wyz + oyz];
          } else {
            const int oyz = wrap_up(bb[1] + y0, d.K1) * d.K2 + wrap_up(bb[2] + z0, d.K2);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) f[dx] = M[wrap_up(bb[0] + dx, d.K0) * K1K2 + oyz];
          }
          const T wy = w[6 + y0], wz = w[12 + z0];
          T sw = 0, sdw = 0;
#pragma unroll
          for (int dx = 0; dx < 6; ++dx) {
            sw += f[dx] * w[dx];
            if (FORCES) sdw += f[dx] * ws.dw[j * 18 + dx];
          }
          T pot = warp_sum(sw * wy * wz), g0 = 0, g1 = 0, g2 = 0;
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
        // the last four columns of atoms j0 .. j1-1, reduced over each atom's four lanes
        T pot = 0, g0 = 0, g1 = 0, g2 = 0;
        const int j = j0 + jt;
        if (j < j1) {
          const T* w = ws.w + j * 18;
          const int* bb = ws.b3 + 3 * j;
          T f[6];
          const int tx = direct ? -1 : tile_start(k.ax, bb[0]);
          const int ty = direct ? -1 : tile_start(k.ay, bb[1]);
          const int tz = direct ? -1 : tile_start(k.az, bb[2]);
          if (tx >= 0 && ty >= 0 && tz >= 0) {
            const int wyz = k.ay.w * k.az.w;
            const int oyz = tile_at(k.ay, ty, 5) * k.az.w + tile_at(k.az, tz, zt);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) f[dx] = tile[tile_at(k.ax, tx, dx) * wyz + oyz];
          } else {
            const int oyz = wrap_up(bb[1] + 5, d.K1) * d.K2 + wrap_up(bb[2] + zt, d.K2);
#pragma unroll
            for (int dx = 0; dx < 6; ++dx) f[dx] = M[wrap_up(bb[0] + dx, d.K0) * K1K2 + oyz];
          }
          const T wy = w[6 + 5], wz = w[12 + zt];
          T sw = 0, sdw = 0;
#pragma unroll
          for (int dx = 0; dx < 6; ++dx) {
            sw += f[dx] * w[dx];
            if (FORCES) sdw += f[dx] * ws.dw[j * 18 + dx];
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
    __syncthreads();
  }
  if (FORCES) block_atomic_sum<9>(wf, acc + (size_t)s * kAccStride + kAccWf, red);
}

}  // namespace admp
