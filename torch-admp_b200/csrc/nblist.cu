// Cell-list neighbour list: TorchNeighborList.forward (nblist.py:304-445 with
// image padding, 472-490 without a box) and check_cutoff (nblist.py:620-660).
//
// With a box the reference asserts rc <= half the minimum box height, so each
// pair has at most one periodic image inside rc and the pair SET equals the
// minimum-image set: atoms are binned by wrapped fractional coordinates into
// cells at least rc high, and every candidate in the (deduplicated) 27
// neighbouring cells is tested with the minimum-image distance
// (spatial.py:15-36 convention, floor(f + 0.5)).  Rows are sorted by j so the
// output is deterministic and sorted by (i, j).
#include "admp_common.cuh"
#include "runtime.h"

namespace admp {

struct NbMeta {
  double b[9], bi[9];
  double lo[3], hi[3], cs[3];
  int nc[3];
  int ncells;
  int status;
  int pad;
  long long npairs;
};

__device__ __forceinline__ void nb_offsets(int pbc, int nc, int* off, int& n) {
  if (!pbc || nc >= 3) {
    off[0] = -1; off[1] = 0; off[2] = 1; n = 3;
  } else if (nc == 2) {
    off[0] = 0; off[1] = 1; n = 2;
  } else {
    off[0] = 0; n = 1;
  }
}

template <typename T>
__global__ void nb_bounds_kernel(int N, const T* __restrict__ pos, NbMeta* meta) {
  __shared__ double smin[3][32], smax[3][32];
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int i = threadIdx.x; i < N; i += blockDim.x)
    for (int e = 0; e < 3; ++e) {
      double v = pos[3 * (size_t)i + e];
      mn[e] = fmin(mn[e], v);
      mx[e] = fmax(mx[e], v);
    }
  for (int e = 0; e < 3; ++e)
    for (int o = 16; o > 0; o >>= 1) {
      mn[e] = fmin(mn[e], __shfl_xor_sync(0xffffffffu, mn[e], o));
      mx[e] = fmax(mx[e], __shfl_xor_sync(0xffffffffu, mx[e], o));
    }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0)
    for (int e = 0; e < 3; ++e) {
      smin[e][w] = mn[e];
      smax[e][w] = mx[e];
    }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int e = 0; e < 3; ++e) {
      double a = 1e300, b = -1e300;
      for (int k = 0; k < nw; ++k) {
        a = fmin(a, smin[e][k]);
        b = fmax(b, smax[e][k]);
      }
      meta->lo[e] = a;
      meta->hi[e] = b;
    }
  }
}

template <typename T>
__global__ void nb_setup_kernel(int pbc, int N, const T* __restrict__ box, double rc, int maxcells, NbMeta* m) {
  m->status = 0;
  m->npairs = 0;
  int nc[3];
  if (pbc) {
    load_box(box, m->b);
    double V = inv3(m->b, m->bi);
    const double* a = m->b;
    double h[3];
    for (int d = 0; d < 3; ++d) {
      const double* u = a + ((d + 1) % 3) * 3;
      const double* v = a + ((d + 2) % 3) * 3;
      double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
      h[d] = fabs(V) / sqrt(cx * cx + cy * cy + cz * cz);
    }
    double mh = fmin(h[0], fmin(h[1], h[2])) / 2.0;
    if (!(rc <= mh)) m->status = ADMP_ERR_CUTOFF_TOO_LARGE;
    if (!isfinite(V) || V == 0.0) m->status = ADMP_ERR_NONFINITE;
    for (int d = 0; d < 3; ++d) {
      double r = h[d] / rc;
      nc[d] = r >= 1.0 && r < 1e6 ? (int)floor(r) : 1;
    }
  } else {
    for (int d = 0; d < 3; ++d) {
      double ext = m->hi[d] - m->lo[d];
      if (!isfinite(ext)) m->status = ADMP_ERR_NONFINITE;
      m->cs[d] = rc;
      double r = ext / rc;
      nc[d] = r < 1e6 ? (int)floor(r) + 1 : 1;
    }
  }
  // keep the grid at most `maxcells` cells (cells may grow beyond rc, never shrink)
  while ((long long)nc[0] * nc[1] * nc[2] > maxcells) {
    int d = nc[0] >= nc[1] && nc[0] >= nc[2] ? 0 : (nc[1] >= nc[2] ? 1 : 2);
    nc[d] = (nc[d] + 1) / 2;
  }
  for (int d = 0; d < 3; ++d) {
    m->nc[d] = nc[d];
    if (!pbc) m->cs[d] = fmax(rc, (m->hi[d] - m->lo[d]) / nc[d] * (1.0 + 1e-12) + 1e-300);
  }
  m->ncells = nc[0] * nc[1] * nc[2];
}

template <typename T>
__global__ void nb_bin_kernel(int pbc, int N, const T* __restrict__ pos, const NbMeta* __restrict__ m,
                              double4* __restrict__ coord, int* __restrict__ cell, int* __restrict__ count,
                              DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  if (m->status) {  // invalid box / cutoff: no atom is binned, later passes skip it
    cell[i] = -1;
    return;
  }
  double r[3] = {(double)pos[3 * (size_t)i], (double)pos[3 * (size_t)i + 1], (double)pos[3 * (size_t)i + 2]};
  if (!isfinite(r[0]) || !isfinite(r[1]) || !isfinite(r[2])) {
    report_error(err, ADMP_ERR_NONFINITE, 4, i);
    cell[i] = -1;
    return;
  }
  int c[3];
  double4 v;
  if (pbc) {
    double f[3];
    for (int e = 0; e < 3; ++e) {
      f[e] = r[0] * m->bi[0 * 3 + e] + r[1] * m->bi[1 * 3 + e] + r[2] * m->bi[2 * 3 + e];
      f[e] -= floor(f[e]);
      c[e] = min((int)(f[e] * m->nc[e]), m->nc[e] - 1);
    }
    v = make_double4(f[0], f[1], f[2], 0.0);
  } else {
    for (int e = 0; e < 3; ++e) c[e] = min(max((int)((r[e] - m->lo[e]) / m->cs[e]), 0), m->nc[e] - 1);
    v = make_double4(r[0], r[1], r[2], 0.0);
  }
  coord[i] = v;
  const int id = (c[0] * m->nc[1] + c[1]) * m->nc[2] + c[2];
  cell[i] = id;
  atomicAdd(count + id, 1);
}

// Single-block exclusive scan of n values (int or long long) -> out[0..n],
// out[n] = total.  Optionally stores the total to *total.
template <typename TI, typename TO>
__global__ void scan_kernel(const TI* __restrict__ in, TO* __restrict__ out, const int* n_ptr, int n_fixed,
                            long long* total) {
  __shared__ TO part[1024];
  const int n = n_ptr ? *n_ptr : n_fixed;
  const int nt = blockDim.x;
  const int chunk = (n + nt - 1) / nt;
  const int b0 = threadIdx.x * chunk, b1 = min(b0 + chunk, n);
  TO s = 0;
  for (int i = b0; i < b1; ++i) s += (TO)in[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    TO acc = 0;
    for (int k = 0; k < nt; ++k) {
      TO t = part[k];
      part[k] = acc;
      acc += t;
    }
    out[n] = acc;
    if (total) *total = (long long)acc;
  }
  __syncthreads();
  TO acc = part[threadIdx.x];
  for (int i = b0; i < b1; ++i) {
    TO t = (TO)in[i];
    out[i] = acc;
    acc += t;
  }
}

__global__ void nb_scatter_kernel(int N, const int* __restrict__ cell, const int* __restrict__ start,
                                  int* __restrict__ cursor, int* __restrict__ sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int c = cell[i];
  if (c < 0) return;
  sorted[start[c] + atomicAdd(cursor + c, 1)] = i;
}

template <bool FILL>
__global__ void nb_pairs_kernel(int pbc, int N, double rc, const NbMeta* __restrict__ m,
                                const double4* __restrict__ coord, const int* __restrict__ cell,
                                const int* __restrict__ start, const int* __restrict__ sorted,
                                long long* __restrict__ rowcnt, const long long* __restrict__ rowptr,
                                long long* __restrict__ pairs, long long* __restrict__ bscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int ci = m->status ? -1 : cell[i];
  if (ci < 0) {
    if (!FILL) rowcnt[i] = 0;
    return;
  }
  const int nc0 = m->nc[0], nc1 = m->nc[1], nc2 = m->nc[2];
  const int c0 = ci / (nc1 * nc2), c1 = (ci / nc2) % nc1, c2 = ci % nc2;
  int o0[3], o1[3], o2[3], n0, n1, n2;
  nb_offsets(pbc, nc0, o0, n0);
  nb_offsets(pbc, nc1, o1, n1);
  nb_offsets(pbc, nc2, o2, n2);
  const double4 ri = coord[i];
  long long cnt = 0;
  const long long base = FILL ? rowptr[i] : 0;
  for (int a = 0; a < n0; ++a) {
    int x = c0 + o0[a];
    if (pbc) x = (x + nc0) % nc0; else if (x < 0 || x >= nc0) continue;
    for (int b = 0; b < n1; ++b) {
      int y = c1 + o1[b];
      if (pbc) y = (y + nc1) % nc1; else if (y < 0 || y >= nc1) continue;
      for (int c = 0; c < n2; ++c) {
        int z = c2 + o2[c];
        if (pbc) z = (z + nc2) % nc2; else if (z < 0 || z >= nc2) continue;
        const int cc = (x * nc1 + y) * nc2 + z;
        for (int s = start[cc]; s < start[cc + 1]; ++s) {
          const int j = sorted[s];
          if (j == i) continue;
          const double4 rj = coord[j];
          double d2;
          if (pbc) {
            double df[3] = {rj.x - ri.x, rj.y - ri.y, rj.z - ri.z};
            for (int e = 0; e < 3; ++e) df[e] -= floor(df[e] + 0.5);
            double dr[3];
            for (int e = 0; e < 3; ++e) dr[e] = df[0] * m->b[0 * 3 + e] + df[1] * m->b[1 * 3 + e] + df[2] * m->b[2 * 3 + e];
            d2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
          } else {
            const double dx = rj.x - ri.x, dy = rj.y - ri.y, dz = rj.z - ri.z;
            d2 = dx * dx + dy * dy + dz * dz;
          }
          const double d = sqrt(d2);
          const bool keep = pbc ? (d < rc && d > 0.01) : (d < rc);
          if (keep) {
            if (FILL) {
              pairs[2 * (base + cnt)] = i;
              pairs[2 * (base + cnt) + 1] = j;
            }
            ++cnt;
          }
        }
      }
    }
  }
  if (!FILL) {
    rowcnt[i] = cnt;
    return;
  }
  // insertion sort of the row by j, then buffer scales (1 if i < j)
  long long* row = pairs + 2 * base;
  for (long long k = 1; k < cnt; ++k) {
    const long long v = row[2 * k + 1];
    long long t = k - 1;
    while (t >= 0 && row[2 * t + 1] > v) {
      row[2 * (t + 1) + 1] = row[2 * t + 1];
      --t;
    }
    row[2 * (t + 1) + 1] = v;
  }
  if (bscale)
    for (long long k = 0; k < cnt; ++k) bscale[base + k] = i < row[2 * k + 1] ? 1 : 0;
}

struct NbWS {
  NbMeta* meta;
  double4* coord;
  int* cell;
  int* count;
  int* start;
  int* cursor;
  int* sorted;
  long long* rowcnt;
  long long* rowptr;
};

static int max_cells(int N) { return 2 * N + 128; }

static NbWS carve_nb(void* ws, size_t bytes, int N, size_t* need) {
  Carver c(ws, bytes);
  NbWS w;
  const int mc = max_cells(N);
  w.meta = c.take<NbMeta>(1);
  w.coord = c.take<double4>(N);
  w.cell = c.take<int>(N);
  w.count = c.take<int>(mc + 1);
  w.start = c.take<int>(mc + 1);
  w.cursor = c.take<int>(mc + 1);
  w.sorted = c.take<int>(N);
  w.rowcnt = c.take<long long>(N + 1);
  w.rowptr = c.take<long long>(N + 1);
  *need = c.off;
  return w;
}

template <typename T>
static int nblist_count_impl(int pbc, int N, const T* pos, const T* box, double rc, void* ws, size_t bytes,
                             long long* npairs, cudaStream_t st) {
  size_t need;
  NbWS w = carve_nb(ws, bytes, N, &need);
  if (need > bytes || !ws) return fail(ADMP_ERR_WORKSPACE, "nblist workspace: need %zu bytes, got %zu", need, bytes);
  DevError* err = scratch_error(st);
  if (!err) return ADMP_ERR_CUDA;
  const int mc = max_cells(N);
  ADMP_CUDA_TRY(cudaMemsetAsync(w.count, 0, sizeof(int) * (mc + 1), st));
  ADMP_CUDA_TRY(cudaMemsetAsync(w.cursor, 0, sizeof(int) * (mc + 1), st));
  if (!pbc) nb_bounds_kernel<T><<<1, 1024, 0, st>>>(N, pos, w.meta);
  nb_setup_kernel<T><<<1, 1, 0, st>>>(pbc, N, box, rc, mc, w.meta);
  const int nb = (N + 255) / 256;
  nb_bin_kernel<T><<<nb, 256, 0, st>>>(pbc, N, pos, w.meta, w.coord, w.cell, w.count, err);
  scan_kernel<int, int><<<1, 1024, 0, st>>>(w.count, w.start, &w.meta->ncells, 0, nullptr);
  nb_scatter_kernel<<<nb, 256, 0, st>>>(N, w.cell, w.start, w.cursor, w.sorted);
  nb_pairs_kernel<false><<<nb, 256, 0, st>>>(pbc, N, rc, w.meta, w.coord, w.cell, w.start, w.sorted, w.rowcnt,
                                             nullptr, nullptr, nullptr);
  scan_kernel<long long, long long><<<1, 1024, 0, st>>>(w.rowcnt, w.rowptr, nullptr, N, &w.meta->npairs);
  ADMP_CUDA_TRY(cudaGetLastError());
  NbMeta h;
  ADMP_CUDA_TRY(cudaMemcpyAsync(&h, w.meta, sizeof(NbMeta), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaStreamSynchronize(st));
  if (h.status == ADMP_ERR_CUTOFF_TOO_LARGE)
    return fail(ADMP_ERR_CUTOFF_TOO_LARGE, "Cutoff %g is larger than half the minimum height of the box.", rc);
  if (h.status) return fail(h.status, "neighbour list: invalid box or positions");
  int s = check_error(err, st);
  if (s) return s;
  *npairs = h.npairs;
  return ADMP_OK;
}

template <typename T>
static int nblist_fill_impl(int pbc, int N, double rc, void* ws, size_t bytes, long long* pairs,
                            long long* bscale, long long cap, cudaStream_t st) {
  size_t need;
  NbWS w = carve_nb(ws, bytes, N, &need);
  if (need > bytes || !ws) return fail(ADMP_ERR_WORKSPACE, "nblist workspace too small");
  long long total = 0;
  ADMP_CUDA_TRY(cudaMemcpyAsync(&total, &w.meta->npairs, sizeof(long long), cudaMemcpyDeviceToHost, st));
  ADMP_CUDA_TRY(cudaStreamSynchronize(st));
  if (total > cap) return fail(ADMP_ERR_CAPACITY, "neighbour list: %lld pairs exceed capacity %lld", total, cap);
  if (total == 0) return ADMP_OK;
  const int nb = (N + 255) / 256;
  nb_pairs_kernel<true><<<nb, 256, 0, st>>>(pbc, N, rc, w.meta, w.coord, w.cell, w.start, w.sorted, w.rowcnt,
                                            w.rowptr, pairs, bscale);
  ADMP_CUDA_TRY(cudaGetLastError());
  return ADMP_OK;
}

}  // namespace admp

using namespace admp;

extern "C" size_t admp_nblist_workspace_size(int natoms) {
  size_t need;
  carve_nb(nullptr, 0, natoms < 0 ? 0 : natoms, &need);
  return need;
}

extern "C" int admp_nblist_count(int dtype, int pbc, int natoms, const void* pos, const void* box, double cutoff,
                                 void* workspace, size_t workspace_bytes, long long* npairs, void* stream) {
  if (!npairs) return fail(ADMP_ERR_BAD_ARG, "npairs is null");
  *npairs = 0;
  if (natoms == 0) return ADMP_OK;
  if (natoms < 0 || !pos || (pbc && !box) || !(cutoff > 0)) return fail(ADMP_ERR_BAD_ARG, "admp_nblist_count: args");
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == ADMP_F64)
    return nblist_count_impl<double>(pbc, natoms, (const double*)pos, (const double*)box, cutoff, workspace,
                                     workspace_bytes, npairs, st);
  if (dtype == ADMP_F32)
    return nblist_count_impl<float>(pbc, natoms, (const float*)pos, (const float*)box, cutoff, workspace,
                                    workspace_bytes, npairs, st);
  return fail(ADMP_ERR_BAD_ARG, "bad dtype");
}

extern "C" int admp_nblist_fill(int dtype, int pbc, int natoms, const void* pos, const void* box, double cutoff,
                                void* workspace, size_t workspace_bytes, long long* pairs, long long* buffer_scales,
                                long long capacity, void* stream) {
  (void)pos;
  (void)box;
  if (natoms == 0) return ADMP_OK;
  if (natoms < 0 || (capacity > 0 && !pairs)) return fail(ADMP_ERR_BAD_ARG, "admp_nblist_fill: args");
  if (dtype != ADMP_F64 && dtype != ADMP_F32) return fail(ADMP_ERR_BAD_ARG, "bad dtype");
  return nblist_fill_impl<double>(pbc, natoms, cutoff, workspace, workspace_bytes, pairs, buffer_scales, capacity,
                                  (cudaStream_t)stream);
}
