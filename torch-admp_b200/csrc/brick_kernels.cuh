// Brick-privatised spread for atoms binned in neighbour cells (the serving
// path, whose neighbour build sorts every system's atoms by cell).  Same
// arithmetic as spread_kernel (recip.py:146-252); only the memory traffic
// differs.
//
// A brick is a run of G cells along z inside one (x, y) cell column.  The
// stencils of its atoms cover a box of mesh points ("tile"): the brick's
// mesh extent plus the 6-point stencil reach, or the whole period along an
// axis where that box would wrap onto itself.  The kernel accumulates the
// tile in shared memory and adds it to the mesh row by row (coalesced global
// reductions, one per tile point instead of 216 scattered ones per atom).
// An atom whose stencil falls outside its brick's tile (possible
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

// Per-warp stencils of 32 atoms, laid out for the accumulation loop: the 18
// weights, the charge, the tile offsets of the atom's 6 x planes (-1 when
// the stencil does not fit the tile), of its 6 y rows and 6 z points, and
// the wrapped mesh bases for the atoms that take the direct path.
template <typename T>
struct BrickStencil {
  T* w;          // [32][18]
  T* q;          // [32]
  int* ox;       // [32][6]  tile offset of plane x (times wy wz)
  short* oy;     // [32][6]  tile offset of row y (times wz)
  short* oz;     // [32][6]  tile offset of point z
  int* b3;       // [32][3]  wrapped mesh bases
  __host__ __device__ static constexpr size_t bytes() {
    return 32 * 18 * sizeof(T) + 32 * sizeof(T) + 32 * 6 * sizeof(int) + 2 * 32 * 6 * sizeof(short) +
           32 * 3 * sizeof(int) + 16;
  }
  __device__ void carve(unsigned char* base) {
    w = reinterpret_cast<T*>(base);
    q = w + 32 * 18;
    ox = reinterpret_cast<int*>(q + 32);
    b3 = ox + 32 * 6;
    oy = reinterpret_cast<short*>(b3 + 32 * 3);
    oz = oy + 32 * 6;
  }
};

template <typename T>
__device__ __forceinline__ void brick_build_stencil(BrickStencil<T>& ws, const SysDesc& d, const Geom& g,
                                                    const Brick& k, const T* __restrict__ pos,
                                                    const T* __restrict__ q, const int* __restrict__ order,
                                                    int a_first, int a_end, int lane) {
  const int a = a_first + lane;
  if (a < a_end) {
    const int ga = order[d.atom_off + a];
    T r[3] = {pos[3 * (size_t)ga], pos[3 * (size_t)ga + 1], pos[3 * (size_t)ga + 2]};
    Stencil<T> st;
    make_stencil<T>(r, g, d.K0, d.K1, d.K2, st);
    T* w = ws.w + lane * 18;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      w[j] = st.w[0][j];
      w[6 + j] = st.w[1][j];
      w[12 + j] = st.w[2][j];
    }
    ws.q[lane] = q[ga];
    ws.b3[lane * 3] = st.ix[0];
    ws.b3[lane * 3 + 1] = st.iy[0];
    ws.b3[lane * 3 + 2] = st.iz[0];
    const int tx = tile_start(k.ax, st.ix[0]), ty = tile_start(k.ay, st.iy[0]), tz = tile_start(k.az, st.iz[0]);
    const bool fit = tx >= 0 && ty >= 0 && tz >= 0;
    const int wyz = k.ay.w * k.az.w;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      ws.ox[lane * 6 + j] = fit ? tile_at(k.ax, tx, j) * wyz : -1;
      ws.oy[lane * 6 + j] = (short)(fit ? tile_at(k.ay, ty, j) * k.az.w : 0);
      ws.oz[lane * 6 + j] = (short)(fit ? tile_at(k.az, tz, j) : 0);
    }
  }
  __syncwarp();
}

// tile capacity (elements of T) of the spread, and its dynamic shared memory:
// the tile plus 8 warps' stencils, sized for three blocks per SM
template <typename T>
__host__ __device__ constexpr int brick_cap() {
  return sizeof(T) == 4 ? 10000 : 5000;
}

template <typename T>
inline size_t brick_smem() {
  return (size_t)brick_cap<T>() * sizeof(T) + 8 * BrickStencil<T>::bytes() + 64;
}

// one stencil column (lanes y0, z0) of atom j: into the tile, or into the mesh
template <typename T>
__device__ __forceinline__ void brick_column(const BrickStencil<T>& ws, int j, int y0, int z0, T* tile, T* M,
                                             const SysDesc& d, int K1K2) {
  const T qa = ws.q[j];
  const T* w = ws.w + j * 18;
  const T v = qa * w[6 + y0] * w[12 + z0];
  const int* ox = ws.ox + j * 6;
  if (ox[0] >= 0) {
    T* t = tile + ws.oy[j * 6 + y0] + ws.oz[j * 6 + z0];
#pragma unroll
    for (int dx = 0; dx < 6; ++dx) atomicAdd(t + ox[dx], w[dx] * v);
  } else {
    const int* bb = ws.b3 + 3 * j;
    T* m = M + wrap_up(bb[1] + y0, d.K1) * d.K2 + wrap_up(bb[2] + z0, d.K2);
#pragma unroll
    for (int dx = 0; dx < 6; ++dx) atomicAdd(m + wrap_up(bb[0] + dx, d.K0) * K1K2, w[dx] * v);
  }
}

// ---------------------------------------------------------------------------
// spread into the zeroed mesh
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256, 3) spread_brick_kernel(Batch b, const T* __restrict__ pos,
                                                              const T* __restrict__ box, const T* __restrict__ q,
                                                              T* __restrict__ mesh, const int* __restrict__ order,
                                                              const int* __restrict__ cells, int cell_stride) {
  extern __shared__ __align__(16) unsigned char dsm[];
  __shared__ Geom g;
  const int s = find_sys<F_ATOM>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];
  constexpr int cap = brick_cap<T>();
  T* tile = reinterpret_cast<T*>(dsm);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  BrickStencil<T> ws;
  ws.carve(dsm + (size_t)cap * sizeof(T) + warp * BrickStencil<T>::bytes());
  load_geom(box, d.box_idx, &g);
  __syncthreads();
  const int* ct = cells + (size_t)d.box_idx * cell_stride;
  BrickPlan p = brick_plan(ct, d, cap);
  const int jb = blockIdx.x - d.blk_atom;
  const int nblk = (d.natoms + b.apb - 1) / b.apb;
  T* M = mesh + d.mesh_off;
  const int K1K2 = d.K1 * d.K2;
  // lanes over the first 32 (y, z) stencil columns; the last four columns of eight atoms in one pass
  const int y0 = lane / 6, z0 = lane % 6, jt = lane >> 2, zt = 2 + (lane & 3);
  // without bricks (G = 0) the block makes one pass over its chunk of the sorted atoms with every
  // stencil taking the direct path (an empty tile: nothing fits)
  const bool direct = p.G == 0;
  const int br0 = direct ? 0 : jb, br1 = direct ? 1 : p.nbricks, step = direct ? 1 : nblk;
  for (int br = br0; br < br1; br += step) {
    Brick k;
    if (direct) {
      k.a0 = jb * b.apb;
      k.a1 = min(k.a0 + b.apb, d.natoms);
      k.ax = {0, 0, d.K0, false};  // width 0: tile_start never fits
      k.ay = k.ax;
      k.az = k.ax;
    } else {
      k = brick_at(ct, d, p, br);
      const int n = k.ax.w * k.ay.w * k.az.w;
      for (int i = threadIdx.x; i < n; i += blockDim.x) tile[i] = T(0);
    }
    __syncthreads();
    for (int a0 = k.a0 + warp * 32; a0 < k.a1; a0 += nw * 32) {
      brick_build_stencil<T>(ws, d, g, k, pos, q, order, a0, k.a1, lane);
      const int na = min(32, k.a1 - a0);
      for (int j0 = 0; j0 < na; j0 += 8) {
        const int j1 = min(j0 + 8, na);
        for (int j = j0; j < j1; ++j) brick_column<T>(ws, j, y0, z0, tile, M, d, K1K2);
        if (j0 + jt < j1) brick_column<T>(ws, j0 + jt, 5, zt, tile, M, d, K1K2);
      }
      __syncwarp();
    }
    __syncthreads();
    if (!direct) {
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
}

}  // namespace admp
