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

// Division by a runtime but block-uniform divisor: q = (x * m) >> 32 is exact
// for 0 <= x < 2^16 whenever 2^32/d <= m < 2^32/d + 2^16/d (the error term
// x (m - 2^32/d) / 2^32 stays below 1/d).  On the device m comes from a
// rounded-up single-precision reciprocal, m = floor(ru(2^32 ru(1/d))) + 1,
// which lies in that window for 2 <= d <= 65000 (checked exhaustively over
// every d and x); the exact integer quotient is used on the host.  Every
// shared-memory index here is below 2^16 (a block never holds more than
// 227 KB / 8 B complex values).
struct FastDiv {
  int d;
  unsigned m;
};
__host__ __device__ __forceinline__ FastDiv fast_div(int d) {
  FastDiv f;
  f.d = d;
#ifdef __CUDA_ARCH__
  f.m = d > 1 ? (unsigned)__fmul_ru(4294967296.0f, __frcp_ru((float)d)) + 1u : 0u;
#else
  f.m = d > 1 ? 0xFFFFFFFFu / (unsigned)d + 1u : 0u;
#endif
  return f;
}
__device__ __forceinline__ int fdiv(int x, const FastDiv& f) {
  return f.d > 1 ? (int)__umulhi((unsigned)x, f.m) : x;
}

// Item idx of a stage -> (line l, butterfly j).  LINE_FAST: consecutive items
// take consecutive lines.  NL > 0 (a power of two) is the line count known at
// compile time, so the split is a mask and a shift.
template <bool LINE_FAST, int NL>
__device__ __forceinline__ void split_item(int idx, const FastDiv& f, int& l, int& j) {
  if constexpr (LINE_FAST && NL > 0) {
    l = idx & (NL - 1);
    j = idx / NL;
  } else {
    const int qd = fdiv(idx, f);
    const int rm = idx - qd * f.d;
    l = LINE_FAST ? rm : qd;
    j = LINE_FAST ? qd : rm;
  }
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

// Shared-memory offsets in these stages are 32-bit ints: a block never holds
// more than 227 KB, i.e. fewer than 2^16 complex values.
//
// One Stockham stage with an odd prime radix r >= 7 over nl lines of length n.
// Element (l, t) lives at buf[l * ls + t * es].  LINE_FAST selects the thread
// mapping (consecutive threads -> consecutive lines, for layouts where the
// line stride is the unit stride).
// The r-point DFT of each butterfly uses the pairing of inputs t and r - t:
//   X_k     = v_0 + sum_t s_t cos(2 pi t k / r) -/+ i sum_t d_t sin(2 pi t k / r)
//   X_{r-k} = v_0 + sum_t s_t cos(...)          +/- i sum_t d_t sin(...)
// with s_t = v_t + v_{r-t}, d_t = v_t - v_{r-t} (t = 1 .. (r-1)/2), which needs
// about r^2 / 4 complex-by-real products per butterfly instead of r^2 complex
// ones.  Step 1 twiddles and folds the inputs (in -> out, in the butterfly's
// own output slots), step 2 forms the output pairs (out -> in), so the result
// of this stage is left in `in`.
template <typename T, bool LINE_FAST, bool WARP, bool INV, int NL>
__device__ __forceinline__ void stockham_odd(Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                             int nl, int n, int ls, int es, int Ns, int r,
                                             const Cplx<T>* __restrict__ W, int tid, int nthr) {
  const int nb = n / r;
  const int h = (r - 1) >> 1;
  const int scale = n / (Ns * r);
  const int wr = n / r;  // W[e * wr] = exp(-2 pi i e / r)
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns), f_items = fast_div(nl * nb);
  const int total1 = nl * nb;
  for (int idx = tid; idx < total1; idx += nthr) {
    int l, j;
    split_item<LINE_FAST, NL>(idx, f_split, l, j);
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = in + (int)l * ls;
    Cplx<T>* dst = out + (int)l * ls;
    const int base = jq * Ns * r + k;
    dst[(int)base * es] = src[(int)j * es];
    for (int u = 1; u <= h; ++u) {
      const Cplx<T> a = src[(int)(j + u * nb) * es];
      const Cplx<T> c = src[(int)(j + (r - u) * nb) * es];
      T ax = a.x, ay = a.y, cx = c.x, cy = c.y;
      if (Ns > 1) {  // the first stage's twiddles are all 1
        const Cplx<T> wa = W[scale * k * u];
        const Cplx<T> wc = W[scale * k * (r - u)];
        const T way = INV ? -wa.y : wa.y, wcy = INV ? -wc.y : wc.y;
        ax = a.x * wa.x - a.y * way;
        ay = a.x * way + a.y * wa.x;
        cx = c.x * wc.x - c.y * wcy;
        cy = c.x * wcy + c.y * wc.x;
      }
      Cplx<T> sv, dv;
      sv.x = ax + cx;
      sv.y = ay + cy;
      dv.x = ax - cx;
      dv.y = ay - cy;
      dst[(int)(base + u * Ns) * es] = sv;
      dst[(int)(base + (h + u) * Ns) * es] = dv;
    }
  }
  if (WARP)
    __syncwarp();
  else
    __syncthreads();
  // step 2 items: class 0 forms X_0, class c >= 1 the output pairs
  // kk = 1 + QK (c - 1) .. QK c, which share each load of s_t and d_t
  // (4 and 8 pairs per item measured slower on the serving stream: fewer items per stage, more registers)
  constexpr int QK = 2;
  const int nq = (h + QK - 1) / QK;
  const int total2 = (nq + 1) * total1;
  for (int idx = tid; idx < total2; idx += nthr) {
    const int c = fdiv(idx, f_items);
    const int it = idx - c * f_items.d;
    int l, j;
    split_item<LINE_FAST, NL>(it, f_split, l, j);
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = out + (int)l * ls;
    Cplx<T>* dst = in + (int)l * ls;
    const int base = jq * Ns * r + k;
    const Cplx<T> v0 = src[(int)base * es];
    if (c == 0) {
      T ax = v0.x, ay = v0.y;
      for (int u = 1; u <= h; ++u) {
        const Cplx<T> sv = src[(int)(base + u * Ns) * es];
        ax += sv.x;
        ay += sv.y;
      }
      Cplx<T> X;
      X.x = ax;
      X.y = ay;
      dst[(int)base * es] = X;
      continue;
    }
    const int kk0 = 1 + (c - 1) * QK;
    T ax[QK], ay[QK], bx[QK], by[QK];
    int e[QK], kq[QK];
#pragma unroll
    for (int t = 0; t < QK; ++t) {
      kq[t] = min(kk0 + t, h);  // past h: computed, not stored
      e[t] = 0;
      ax[t] = v0.x;
      ay[t] = v0.y;
      bx[t] = T(0);
      by[t] = T(0);
    }
    for (int u = 1; u <= h; ++u) {
      const Cplx<T> sv = src[(int)(base + u * Ns) * es];
      const Cplx<T> dv = src[(int)(base + (h + u) * Ns) * es];
#pragma unroll
      for (int t = 0; t < QK; ++t) {
        e[t] += kq[t];
        if (e[t] >= r) e[t] -= r;
        const Cplx<T> w = W[e[t] * wr];  // (cos, -sin) of 2 pi e / r
        ax[t] += sv.x * w.x;
        ay[t] += sv.y * w.x;
        bx[t] -= dv.x * w.y;
        by[t] -= dv.y * w.y;
      }
    }
#pragma unroll
    for (int t = 0; t < QK; ++t) {
      const int kk = kk0 + t;
      if (kk > h) break;
      // forward: X_k = A - i B, X_{r-k} = A + i B (inverse: signs swapped); -i B = (B.y, -B.x)
      const T ibx = INV ? -by[t] : by[t], iby = INV ? bx[t] : -bx[t];
      Cplx<T> X1, X2;
      X1.x = ax[t] + ibx;
      X1.y = ay[t] + iby;
      X2.x = ax[t] - ibx;
      X2.y = ay[t] - iby;
      dst[(int)(base + kk * Ns) * es] = X1;
      dst[(int)(base + (r - kk) * Ns) * es] = X2;
    }
  }
}

// Radix-3 and radix-5 stages: one thread per butterfly, inputs twiddled from
// the table, then the small DFT with the exact cosines / sines of 2 pi / 3 and
// 2 pi / 5 (sign of the sines flips for the inverse transform).
template <typename T, bool LINE_FAST, int R, bool INV, int NL>
__device__ __forceinline__ void stockham_r35(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                             int nl, int n, int ls, int es, int Ns,
                                             const Cplx<T>* __restrict__ W, int tid, int nthr) {
  const int nb = n / R;
  const int total = nl * nb;
  const int scale = n / (Ns * R);
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns);
  const T sg = INV ? T(-1) : T(1);
  for (int idx = tid; idx < total; idx += nthr) {
    int l, j;
    split_item<LINE_FAST, NL>(idx, f_split, l, j);
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = in + (int)l * ls;
    Cplx<T> v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) {
      const Cplx<T> x = src[(int)(j + t * nb) * es];
      if (t == 0 || Ns == 1) {  // first stage: every twiddle is 1
        v[t] = x;
      } else {
        const Cplx<T> w = W[scale * k * t];
        const T wy = INV ? -w.y : w.y;
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
    Cplx<T>* dst = out + (int)l * ls;
#pragma unroll
    for (int u = 0; u < R; ++u) dst[(int)(base + u * Ns) * es] = X[u];
  }
}

// Radix-4 stage, one thread per butterfly (4 outputs).
template <typename T, bool LINE_FAST, bool INV, int NL>
__device__ __forceinline__ void stockham_r4(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                            int nl, int n, int ls, int es, int Ns,
                                            const Cplx<T>* __restrict__ W, int tid, int nthr) {
  const int nb = n >> 2;
  const int total = nl * nb;
  const int scale = n / (Ns * 4);
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns);
  for (int idx = tid; idx < total; idx += nthr) {
    int l, j;
    split_item<LINE_FAST, NL>(idx, f_split, l, j);
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = in + (int)l * ls;
    Cplx<T> v[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      Cplx<T> x = src[(int)(j + t * nb) * es];
      if (t == 0 || Ns == 1) {  // first stage: every twiddle is 1
        v[t] = x;
      } else {
        Cplx<T> w = W[scale * k * t];
        T wy = INV ? -w.y : w.y;
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
    T mdx = INV ? -dy : dy;
    T mdy = INV ? dx : -dx;
    const int base = jq * Ns * 4 + k;
    Cplx<T>* dst = out + (int)l * ls;
    Cplx<T> o0, o1, o2, o3;
    o0.x = ax + cx; o0.y = ay + cy;
    o1.x = bx + mdx; o1.y = by + mdy;
    o2.x = ax - cx; o2.y = ay - cy;
    o3.x = bx - mdx; o3.y = by - mdy;
    dst[(int)(base) * es] = o0;
    dst[(int)(base + Ns) * es] = o1;
    dst[(int)(base + 2 * Ns) * es] = o2;
    dst[(int)(base + 3 * Ns) * es] = o3;
  }
}

// Radix-2 stage, one thread per butterfly.
template <typename T, bool LINE_FAST, bool INV, int NL>
__device__ __forceinline__ void stockham_r2(const Cplx<T>* __restrict__ in, Cplx<T>* __restrict__ out,
                                            int nl, int n, int ls, int es, int Ns,
                                            const Cplx<T>* __restrict__ W, int tid, int nthr) {
  const int nb = n >> 1;
  const int total = nl * nb;
  const int scale = n / (Ns * 2);
  const FastDiv f_split = fast_div(LINE_FAST ? nl : nb), f_ns = fast_div(Ns);
  for (int idx = tid; idx < total; idx += nthr) {
    int l, j;
    split_item<LINE_FAST, NL>(idx, f_split, l, j);
    const int jq = fdiv(j, f_ns);
    const int k = j - jq * Ns;
    const Cplx<T>* src = in + (int)l * ls;
    Cplx<T> a = src[(int)j * es];
    Cplx<T> x = src[(int)(j + nb) * es];
    Cplx<T> b = x;
    if (Ns > 1) {  // the first stage's twiddles are all 1
      const Cplx<T> w = W[scale * k];
      const T wy = INV ? -w.y : w.y;
      b.x = x.x * w.x - x.y * wy;
      b.y = x.x * wy + x.y * w.x;
    }
    const int base = jq * Ns * 2 + k;
    Cplx<T>* dst = out + (int)l * ls;
    Cplx<T> o0, o1;
    o0.x = a.x + b.x; o0.y = a.y + b.y;
    o1.x = a.x - b.x; o1.y = a.y - b.y;
    dst[(int)base * es] = o0;
    dst[(int)(base + Ns) * es] = o1;
  }
}

// One pass of all stages over nl lines with threads tid, tid + nthr, ...;
// WARP: the calling threads are one warp (synchronised with __syncwarp),
// otherwise the whole block (__syncthreads).  Returns the buffer holding the
// result (a or b).
template <typename T, bool LINE_FAST, bool WARP, bool INV, int NL = 0>
__device__ __forceinline__ Cplx<T>* fft_run(const Radices& R, Cplx<T>* a, Cplx<T>* b, int nl, int n, int ls, int es,
                                            const Cplx<T>* W, int tid, int nthr) {
  int Ns = 1;
  Cplx<T>* in = a;
  Cplx<T>* out = b;
  for (int s = 0; s < R.ns; ++s) {
    const int r = R.r[s];
    if (r == 4)
      stockham_r4<T, LINE_FAST, INV, NL>(in, out, nl, n, ls, es, Ns, W, tid, nthr);
    else if (r == 2)
      stockham_r2<T, LINE_FAST, INV, NL>(in, out, nl, n, ls, es, Ns, W, tid, nthr);
    else if (r == 3)
      stockham_r35<T, LINE_FAST, 3, INV, NL>(in, out, nl, n, ls, es, Ns, W, tid, nthr);
    else if (r == 5)
      stockham_r35<T, LINE_FAST, 5, INV, NL>(in, out, nl, n, ls, es, Ns, W, tid, nthr);
    else
      stockham_odd<T, LINE_FAST, WARP, INV, NL>(in, out, nl, n, ls, es, Ns, r, W, tid, nthr);
    if (WARP)
      __syncwarp();
    else
      __syncthreads();
    Ns *= r;
    if (r <= 5) {  // the odd-radix stage leaves its result in `in`
      Cplx<T>* tmp = in;
      in = out;
      out = tmp;
    }
  }
  return in;
}

// Full transform by the whole block; returns the buffer holding the result (a or b).
// Caller must __syncthreads() before (inputs written) -- this function
// synchronises between stages and after the last one.
// INV: inverse (unnormalised) transform.  NL > 0: nl == NL lines (a power of
// two), known at compile time.
template <typename T, bool LINE_FAST, bool INV, int NL = 0>
__device__ Cplx<T>* fft_lines(Cplx<T>* a, Cplx<T>* b, int nl, int n, int ls, int es, const Cplx<T>* W) {
  Radices R;
  factor_radices(n, R);
  return fft_run<T, LINE_FAST, false, INV, NL>(R, a, b, nl, n, ls, es, W, threadIdx.x, blockDim.x);
}

}  // namespace admp
