// Batched 1-D FFTs of arbitrary length in shared memory (Stockham autosort,
// runtime mixed radix).  The PME mesh sizes follow the reference's automatic
// rule ceil(2 kappa L / (3 ethresh^0.2)) (pme.py:390-392), so lengths such as
// 17, 79 (prime) or 658 = 2*7*47 must all work; radix-4/2 stages are used
// where they divide n, every other prime factor runs as a direct DFT stage.
#pragma once

#include "admp_common.cuh"

namespace admp {

struct Radices {
  int n;
  int ns;
  int r[24];
};

__device__ __forceinline__ void factor_radices(int n, Radices& R) {
  R.n = n;
  R.ns = 0;
  int m = n;
  while (m % 4 == 0 && R.ns < 24) { R.r[R.ns++] = 4; m /= 4; }
  while (m % 2 == 0 && R.ns < 24) { R.r[R.ns++] = 2; m /= 2; }
  for (int f = 3; f * f <= m; f += 2)
    while (m % f == 0 && R.ns < 24) { R.r[R.ns++] = f; m /= f; }
  if (m > 1) R.r[R.ns++] = m;
}

// W[e] = exp(-2 pi i e / n), e in [0, n); computed in double.
template <typename T>
__device__ __forceinline__ void make_twiddles(Cplx<T>* W, int n) {
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)e / (double)n, &s, &c);
    W[e].x = (T)c;
    W[e].y = (T)(-s);
  }
}

// One Stockham stage with radix r over nl lines of length n.
// Element (l, t) lives at buf[l * ls + t * es].
// LINE_FAST selects the thread mapping (consecutive threads -> consecutive
// lines, for layouts where the line stride is the unit stride).
template <typename T, bool LINE_FAST>
__device__ __forceinline__ void stockham_stage(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                               int nl, int n, int ls, int es, int Ns, int r,
                                               const Cplx<T>* __restrict__ W, bool inverse) {
  const int total = nl * n;
  const int nr = n / r;
  const int scale = n / (Ns * r);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int l, o;
    if (LINE_FAST) {
      l = idx % nl;
      o = idx / nl;
    } else {
      o = idx % n;
      l = idx / n;
    }
    const int q = o / (Ns * r);
    const int rem = o - q * (Ns * r);
    const int u = rem / Ns;
    const int k = rem - u * Ns;
    const int j = q * Ns + k;
    const int c = scale * (k + u * Ns);
    const Cplx<T>* src = in + (size_t)l * ls + (size_t)j * es;
    T sx = 0, sy = 0;
    int e = 0;
    for (int t = 0; t < r; ++t) {
      Cplx<T> x = src[(size_t)t * nr * es];
      Cplx<T> w = W[e];
      T wy = inverse ? -w.y : w.y;
      sx += x.x * w.x - x.y * wy;
      sy += x.x * wy + x.y * w.x;
      e += c;
      if (e >= n) e -= n;
    }
    Cplx<T> res;
    res.x = sx;
    res.y = sy;
    out[(size_t)l * ls + (size_t)o * es] = res;
  }
}

// Radix-4 stage, one thread per butterfly (4 outputs).
template <typename T, bool LINE_FAST>
__device__ __forceinline__ void stockham_r4(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                            int nl, int n, int ls, int es, int Ns,
                                            const Cplx<T>* __restrict__ W, bool inverse) {
  const int nb = n >> 2;
  const int total = nl * nb;
  const int scale = n / (Ns * 4);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int l, j;
    if (LINE_FAST) {
      l = idx % nl;
      j = idx / nl;
    } else {
      j = idx % nb;
      l = idx / nb;
    }
    const int k = j % Ns;
    const Cplx<T>* src = in + (size_t)l * ls;
    Cplx<T> v[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      Cplx<T> x = src[(size_t)(j + t * nb) * es];
      if (t == 0) {
        v[0] = x;
      } else {
        Cplx<T> w = W[scale * k * t];
        T wy = inverse ? -w.y : w.y;
        v[t].x = x.x * w.x - x.y * wy;
        v[t].y = x.x * wy + x.y * w.x;
      }
    }
    // 4-point DFT: forward uses -i, inverse +i
    T ax = v[0].x + v[2].x, ay = v[0].y + v[2].y;
    T bx = v[0].x - v[2].x, by = v[0].y - v[2].y;
    T cx = v[1].x + v[3].x, cy = v[1].y + v[3].y;
    T dx = v[1].x - v[3].x, dy = v[1].y - v[3].y;
    // (-i) * d = (dy, -dx); (+i) * d = (-dy, dx)
    T mdx = inverse ? -dy : dy;
    T mdy = inverse ? dx : -dx;
    const int base = (j / Ns) * Ns * 4 + k;
    Cplx<T>* dst = out + (size_t)l * ls;
    Cplx<T> o0, o1, o2, o3;
    o0.x = ax + cx; o0.y = ay + cy;
    o1.x = bx + mdx; o1.y = by + mdy;
    o2.x = ax - cx; o2.y = ay - cy;
    o3.x = bx - mdx; o3.y = by - mdy;
    dst[(size_t)(base) * es] = o0;
    dst[(size_t)(base + Ns) * es] = o1;
    dst[(size_t)(base + 2 * Ns) * es] = o2;
    dst[(size_t)(base + 3 * Ns) * es] = o3;
  }
}

// Radix-2 stage, one thread per butterfly.
template <typename T, bool LINE_FAST>
__device__ __forceinline__ void stockham_r2(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                            int nl, int n, int ls, int es, int Ns,
                                            const Cplx<T>* __restrict__ W, bool inverse) {
  const int nb = n >> 1;
  const int total = nl * nb;
  const int scale = n / (Ns * 2);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    int l, j;
    if (LINE_FAST) {
      l = idx % nl;
      j = idx / nl;
    } else {
      j = idx % nb;
      l = idx / nb;
    }
    const int k = j % Ns;
    const Cplx<T>* src = in + (size_t)l * ls;
    Cplx<T> a = src[(size_t)j * es];
    Cplx<T> x = src[(size_t)(j + nb) * es];
    Cplx<T> w = W[scale * k];
    T wy = inverse ? -w.y : w.y;
    Cplx<T> b;
    b.x = x.x * w.x - x.y * wy;
    b.y = x.x * wy + x.y * w.x;
    const int base = (j / Ns) * Ns * 2 + k;
    Cplx<T>* dst = out + (size_t)l * ls;
    Cplx<T> o0, o1;
    o0.x = a.x + b.x; o0.y = a.y + b.y;
    o1.x = a.x - b.x; o1.y = a.y - b.y;
    dst[(size_t)base * es] = o0;
    dst[(size_t)(base + Ns) * es] = o1;
  }
}

// Full transform; returns the buffer holding the result (a or b).
// Caller must __syncthreads() before (inputs written) -- this function
// synchronises between stages and after the last one.
template <typename T, bool LINE_FAST>
__device__ Cplx<T>* fft_lines(Cplx<T>* a, Cplx<T>* b, int nl, int n, int ls, int es,
                              const Cplx<T>* W, bool inverse) {
  Radices R;
  factor_radices(n, R);
  int Ns = 1;
  Cplx<T>* in = a;
  Cplx<T>* out = b;
  for (int s = 0; s < R.ns; ++s) {
    const int r = R.r[s];
    if (r == 4)
      stockham_r4<T, LINE_FAST>(in, out, nl, n, ls, es, Ns, W, inverse);
    else if (r == 2)
      stockham_r2<T, LINE_FAST>(in, out, nl, n, ls, es, Ns, W, inverse);
    else
      stockham_stage<T, LINE_FAST>(in, out, nl, n, ls, es, Ns, r, W, inverse);
    __syncthreads();
    Ns *= r;
    Cplx<T>* tmp = in;
    in = out;
    out = tmp;
  }
  return in;
}

}  // namespace admp
