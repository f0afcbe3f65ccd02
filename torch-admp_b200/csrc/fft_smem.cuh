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

// Division by a runtime but block-uniform divisor through a float reciprocal
// (operands stay far below 2^22, so the estimate is off by at most one and
// one correction step makes it exact).
struct FastDiv {
  int d;
  float inv;
};
__device__ __forceinline__ FastDiv fast_div(int d) {
  FastDiv f;
  f.d = d;
  f.inv = 1.0f / (float)d;
  return f;
}
__device__ __forceinline__ int fdiv(int x, const FastDiv& f) {
  int q = __float2int_rz((float)x * f.inv);
  const int r = x - q * f.d;
  if (r < 0)
    --q;
  else if (r >= f.d)
    ++q;
  return q;
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
  const FastDiv f_split = fast_div(LINE_FAST ? nl : n), f_nsr = fast_div(Ns * r), f_ns = fast_div(Ns);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int qd = fdiv(idx, f_split);
    const int rm = idx - qd * f_split.d;
    const int l = LINE_FAST ? rm : qd;
    const int o = LINE_FAST ? qd : rm;
    const int q = fdiv(o, f_nsr);
    const int rem = o - q * (Ns * r);
    const int u = fdiv(rem, f_ns);
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

// Radix-3 and radix-5 stages: one thread per butterfly, inputs twiddled from
// the table, then the small DFT with the exact cosines / sines of 2 pi / 3 and
// 2 pi / 5 (sign of the sines flips for the inverse transform).
template <typename T, bool LINE_FAST, int R>
__device__ __forceinline__ void stockham_r35(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                             int nl, int n, int ls, int es, int Ns,
                                             const Cplx<T>* __restrict__ W, bool inverse) {
  const int nb = n / R;
  const int total = nl * nb;
  const int scale = n / (Ns * R);
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns);
  const T sg = inverse ? T(-1) : T(1);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int qd = fdiv(idx, f_split);
    const int rm = idx - qd * f_split.d;
    const int l = LINE_FAST ? rm : qd;
    const int j = LINE_FAST ? qd : rm;
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = in + (size_t)l * ls;
    Cplx<T> v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) {
      const Cplx<T> x = src[(size_t)(j + t * nb) * es];
      if (t == 0) {
        v[0] = x;
      } else {
        const Cplx<T> w = W[scale * k * t];
        const T wy = inverse ? -w.y : w.y;
        v[t].x = x.x * w.x - x.y * wy;
        v[t].y = x.x * wy + x.y * w.x;
      }
    }
    Cplx<T> X[R];
    if (R == 3) {
      const T s3 = T(0.86602540378443864676) * sg;  // sin(2 pi / 3)
      const T ax = v[1].x + v[2].x, ay = v[1].y + v[2].y;
      const T bx = v[1].x - v[2].x, by = v[1].y - v[2].y;
      const T mx = v[0].x - T(0.5) * ax, my = v[0].y - T(0.5) * ay;
      X[0].x = v[0].x + ax;
      X[0].y = v[0].y + ay;
      // -i s b = (s b.y, -s b.x)
      X[1].x = mx + s3 * by;
      X[1].y = my - s3 * bx;
      X[2].x = mx - s3 * by;
      X[2].y = my + s3 * bx;
    } else {
      const T c1 = T(0.30901699437494742410), c2 = T(-0.80901699437494742410);  // cos(2pi/5), cos(4pi/5)
      const T s1 = T(0.95105651629515357212) * sg, s2 = T(0.58778525229247312917) * sg;  // sin(2pi/5), sin(4pi/5)
      const T a1x = v[1].x + v[4].x, a1y = v[1].y + v[4].y, b1x = v[1].x - v[4].x, b1y = v[1].y - v[4].y;
      const T a2x = v[2].x + v[3].x, a2y = v[2].y + v[3].y, b2x = v[2].x - v[3].x, b2y = v[2].y - v[3].y;
      X[0].x = v[0].x + a1x + a2x;
      X[0].y = v[0].y + a1y + a2y;
      const T p1x = v[0].x + c1 * a1x + c2 * a2x, p1y = v[0].y + c1 * a1y + c2 * a2y;
      const T q1x = s1 * b1x + s2 * b2x, q1y = s1 * b1y + s2 * b2y;   // X1 = p1 - i q1, X4 = p1 + i q1
      const T p2x = v[0].x + c2 * a1x + c1 * a2x, p2y = v[0].y + c2 * a1y + c1 * a2y;
      const T q2x = s2 * b1x - s1 * b2x, q2y = s2 * b1y - s1 * b2y;   // X2 = p2 - i q2, X3 = p2 + i q2
      X[1].x = p1x + q1y;
      X[1].y = p1y - q1x;
      X[4].x = p1x - q1y;
      X[4].y = p1y + q1x;
      X[2].x = p2x + q2y;
      X[2].y = p2y - q2x;
      X[3].x = p2x - q2y;
      X[3].y = p2y + q2x;
    }
    const int base = jq * Ns * R + k;
    Cplx<T>* dst = out + (size_t)l * ls;
#pragma unroll
    for (int u = 0; u < R; ++u) dst[(size_t)(base + u * Ns) * es] = X[u];
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
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int qd = fdiv(idx, f_split);
    const int rm = idx - qd * f_split.d;
    const int l = LINE_FAST ? rm : qd;
    const int j = LINE_FAST ? qd : rm;
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
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
    const int base = jq * Ns * 4 + k;
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
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns);
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const int qd = fdiv(idx, f_split);
    const int rm = idx - qd * f_split.d;
    const int l = LINE_FAST ? rm : qd;
    const int j = LINE_FAST ? qd : rm;
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = in + (size_t)l * ls;
    Cplx<T> a = src[(size_t)j * es];
    Cplx<T> x = src[(size_t)(j + nb) * es];
    Cplx<T> w = W[scale * k];
    T wy = inverse ? -w.y : w.y;
    Cplx<T> b;
    b.x = x.x * w.x - x.y * wy;
    b.y = x.x * wy + x.y * w.x;
    const int base = jq * Ns * 2 + k;
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
    else if (r == 3)
      stockham_r35<T, LINE_FAST, 3>(in, out, nl, n, ls, es, Ns, W, inverse);
    else if (r == 5)
      stockham_r35<T, LINE_FAST, 5>(in, out, nl, n, ls, es, Ns, W, inverse);
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
