// x pass of the CG matvec (FP32) on the tensor cores: for a tile of 128
// flattened (y, kz) columns of one system's half spectrum, the DFT along x,
// the product with the cached Green's function and the inverse DFT along x
// are two real matrix products on tcgen05 (kind::tf32, accumulators in TMEM)
// with the Green's-function product in between.  The reference computes the
// same potential with torch.fft (recip.py:216-252, pme.py:433-446).
//
// Matrix form.  For a column with values h_x = a_x + i b_x (x < K0), write
// the DFT through the real matrix Phi[x][j']:
//   j' <  40:  cos(2 pi x j' / K0)       for j' <= K0/2      (else 0)
//   j' >= 40:  sin(2 pi x (j'-40) / K0)  for 1 <= j'-40 <= (K0-1)/2 (else 0)
// Stage 1: E/O[c][j'] = sum_x (a or b)[c][x] Phi[x][j'] gives the even (cos)
// and odd (sin) parts of the spectrum: S_k = Ea + Ob + i (Eb - Oa) at k' = k,
// S_{K0-k} = Ea - Ob + i (Eb + Oa).  Between the stages T_k = g_k S_k and
// the folded inputs U_k = T_k + T_{K0-k}, V_k = T_k - T_{K0-k} are formed
// (k = 0 and the Nyquist index stand alone).  Stage 3: the unnormalised
// inverse transform, out = [U_re | -V_im] Phi^T + i [U_im | V_re] Phi^T.
//
// Precision: every operand is split into a TF32 head and a TF32 tail, and
// each product is head*head + head*tail + tail*head (three MMAs), so the
// result carries about 22 significand bits (relative error ~1e-6 measured
// on 80-term products against FP64), close to the FP32 FFT it replaces.
//
// Layout.  Operands are K-major without swizzle: an 8-row x 16-byte core
// matrix per (row group, 4 columns), 128 bytes apart along K (LBO) and
// kTcSbo bytes apart along M/N (SBO).  The contraction of each stage runs
// in two halves of 40 columns (x < 40 and x >= 40 in stage 1; the U and the
// V columns in stage 3), so a CTA holds only one half: A = 4 tiles of
// 128 x 40 (re / im, head / tail) and B = 2 tiles of 80 x 40 (head / tail),
// 105 KB of shared memory, and two CTAs share an SM, one CTA's loads and
// Green's-function step overlapping the other's products.  TMEM: 256
// columns per CTA (the real accumulator at column 0, the imaginary one at
// column 128).  The B halves (Phi^T for stage 1, Phi for stage 3, head and
// tail) of every mesh length are built once per device in global memory
// and copied into shared memory by 1-D bulk asynchronous copies (the TMA
// engine, no tensor map, no multicast) on an mbarrier.  Every wait is
// bounded; on expiry the system's CG status is set and the kernel returns
// after freeing its TMEM.
#pragma once

#include <cstddef>
#include <cstdint>

#include "pme_kernels.cuh"

namespace admp {

constexpr int kTcMaxK = 79;                       // longest x line of this path (40 cos + 40 sin columns)
constexpr int kTcRows = 128;                      // flattened columns per CTA (MMA M)
constexpr int kTcN = 80;                          // N of stage 1 (40 cos + 40 sin columns)
constexpr int kTcHalf = 40;                       // K columns of one half of a contraction
constexpr int kTcSbo = (kTcHalf / 4) * 128;       // bytes between 8-row groups
constexpr int kTcATile = kTcRows * kTcHalf * 4;   // bytes
constexpr int kTcBTile = kTcN * kTcHalf * 4;
constexpr int kTcSmem = 4 * kTcATile + 2 * kTcBTile;
constexpr int kTcImgWords = kTcN * kTcHalf;       // one B image (one half, head or tail)
constexpr long long kTcSpin = 1LL << 24;

// byte offset of (row r, column k) in a K-major no-swizzle tile kTcHalf columns wide
__host__ __device__ __forceinline__ int tc_off(int r, int k) {
  return (r >> 3) * kTcSbo + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

__device__ __forceinline__ uint32_t tc_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t tf32_head(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// shared-memory matrix descriptor (sm_100): start, LBO, SBO in 16-byte units, version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)((kTcSbo >> 4) & 0x3FFF) << 32) |
         (1ull << 46);
}

// instruction descriptor: D f32, A and B tf32, both K-major, M = 128, N = n
__device__ __forceinline__ uint32_t tc_idesc(int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kTcRows >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dt, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dt),
      "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(tc_smem(bar))
               : "memory");
}

__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok = 0;
  for (long long it = 0; it < kTcSpin && !ok; ++it)
    asm volatile(
        "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(ok)
        : "r"(tc_smem(bar)), "r"(parity)
        : "memory");
  return ok != 0;
}

// one B half (head and tail images, 2 x 12,800 bytes) by the bulk-copy engine
__device__ __forceinline__ void tc_load_b(unsigned char* dst, const uint32_t* src, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc_smem(bar)), "r"(2 * kTcBTile)
               : "memory");
  for (int h = 0; h < 2; ++h)
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            tc_smem(dst + h * kTcBTile)),
        "l"(src + (size_t)h * kTcImgWords), "r"(kTcBTile), "r"(tc_smem(bar))
        : "memory");
}

// The three-term products of one contraction half, issued by one thread: D_re += A_re B,
// D_im += A_im B over ks K-steps (8 columns each, 256 bytes apart in every tile, i.e. 16 in the
// descriptors' start-address field).  `acc`: accumulate onto the earlier half.
__device__ __forceinline__ void tc_products(uint32_t dre, uint32_t dim, const unsigned char* Arh,
                                            const unsigned char* Arl, const unsigned char* Aih,
                                            const unsigned char* Ail, const unsigned char* Bt, int ks, int n,
                                            bool acc) {
  const uint32_t id = tc_idesc(n);
  const uint64_t arh = tc_desc(tc_smem(Arh)), arl = tc_desc(tc_smem(Arl)), aih = tc_desc(tc_smem(Aih)),
                 ail = tc_desc(tc_smem(Ail)), bh = tc_desc(tc_smem(Bt)), bl = tc_desc(tc_smem(Bt + kTcBTile));
  for (int k = 0; k < ks; ++k) {
    const uint64_t o = (uint64_t)k * 16;
    const uint32_t first = (acc || k > 0) ? 1u : 0u;
    tc_mma(dre, arh + o, bh + o, id, first);  // head * head
    tc_mma(dim, aih + o, bh + o, id, first);
    tc_mma(dre, arh + o, bl + o, id, 1u);     // head * tail
    tc_mma(dim, aih + o, bl + o, id, 1u);
    tc_mma(dre, arl + o, bh + o, id, 1u);     // tail * head
    tc_mma(dim, ail + o, bh + o, id, 1u);
  }
}

#define ADMP_TC_LD4(taddr, v)                                                                           \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"                           \
               : "=r"((v)[0]), "=r"((v)[1]), "=r"((v)[2]), "=r"((v)[3])                               \
               : "r"(taddr))
#define ADMP_TC_LD8(taddr, v)                                                                           \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"               \
               : "=r"((v)[0]), "=r"((v)[1]), "=r"((v)[2]), "=r"((v)[3]), "=r"((v)[4]), "=r"((v)[5]),  \
                 "=r"((v)[6]), "=r"((v)[7])                                                           \
               : "r"(taddr))

// four values -> head / tail vectors at (row, k0 .. k0+3) of two tiles
__device__ __forceinline__ void tc_put4(unsigned char* hi, unsigned char* lo, int row, int k0, const float v[4]) {
  uint4 h, l;
  uint32_t* hp = &h.x;
  uint32_t* lp = &l.x;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    hp[t] = tf32_head(v[t]);
    lp[t] = tf32_head(v[t] - __uint_as_float(hp[t]));
  }
  const int o = tc_off(row, k0);
  *reinterpret_cast<uint4*>(hi + o) = h;
  *reinterpret_cast<uint4*>(lo + o) = l;
}

// The B images of every mesh length 1..kTcMaxK, [K0][part][head, tail][kTcImgWords] with parts
// 0, 1 = stage 1 (Phi^T restricted to x < 40, x >= 40) and 2, 3 = stage 3 (Phi restricted to
// j' < 40, j' >= 40) (dft_tc.cu): built on the current device at the first call (ordered on `st`
// and waited for, so any stream may read them afterwards).  nullptr if they cannot be built.  The first
// call on a device synchronises `st` (not allowed while `st` is being captured into a CUDA graph: make
// one uncaptured call first); the cached address is not valid across cudaDeviceReset.
const uint32_t* tc_tables(cudaStream_t st);

// One tile: 128 flattened columns of one system (block family F_XT).
struct TcTile {
  int K0, c0, nz, box_idx;
  size_t xs;
  int64_t spec_off, green_off;
};

__device__ __forceinline__ bool tc_tile(const Batch& b, int t, TcTile& T) {
  const int s = find_sys<F_XT>(b, t);
  if (skip_sys(b, s)) return false;
  const SysDesc& d = b.s[s];
  const int C = d.K1 * d.K2h;
  T.K0 = d.K0;
  T.c0 = (t - d.blk_xt) * kTcRows;
  T.nz = min(kTcRows, C - T.c0);
  T.box_idx = d.box_idx;
  T.xs = (size_t)C;
  T.spec_off = d.spec_off;
  T.green_off = d.green_off;
  return true;
}

// A thread's part of a tile's spectrum: column tid % 128, x runs (tid / 128) * 4 + 8 m (m < 10);
// runs m < 5 lie in the first contraction half (x < 40), m >= 5 in the second.
__device__ __forceinline__ void tc_fetch(const Cplx<float>* __restrict__ spec, const TcTile& T, int tid,
                                         Cplx<float> (&v)[10][4]) {
  const Cplx<float>* H = spec + T.spec_off + T.c0;
  const int ca = tid & (kTcRows - 1), xa = (tid >> 7) * 4;
  const bool la = ca < T.nz;
#pragma unroll
  for (int m = 0; m < 10; ++m)
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int x = xa + 8 * m + t;
      v[m][t].x = 0.f;
      v[m][t].y = 0.f;
      if (la && x < T.K0) v[m][t] = H[(size_t)x * T.xs + ca];
    }
}

// runs M0 .. M0+4 of the thread's values into the A tiles (columns x - 40 * (M0 / 5))
template <int M0>
__device__ __forceinline__ void tc_stage_a(unsigned char* Arh, unsigned char* Arl, unsigned char* Aih,
                                           unsigned char* Ail, int tid, const Cplx<float> (&v)[10][4]) {
  const int ca = tid & (kTcRows - 1), xa = (tid >> 7) * 4;
#pragma unroll
  for (int mm = 0; mm < 5; ++mm) {
    const int m = M0 + mm;
    float re[4], im[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      re[t] = v[m][t].x;
      im[t] = v[m][t].y;
    }
    tc_put4(Arh, Arl, ca, xa + 8 * mm, re);
    tc_put4(Aih, Ail, ca, xa + 8 * mm, im);
  }
}

// Two CTAs per SM (105 KB of shared memory each), one tile per CTA, 256 threads.
static __global__ void __launch_bounds__(256, 2)
    tc_x_apply_kernel(Batch b, Cplx<float>* __restrict__ spec, const float* __restrict__ green,
                      const uint32_t* __restrict__ tab) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bar_b, bar_m;
  __shared__ uint32_t tslot;
  unsigned char* Arh = tsm;
  unsigned char* Arl = Arh + kTcATile;
  unsigned char* Aih = Arl + kTcATile;
  unsigned char* Ail = Aih + kTcATile;
  unsigned char* Bt = Ail + kTcATile;  // head, tail
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  TcTile cur;
  if (!tc_tile(b, blockIdx.x, cur)) return;
  const int K0 = cur.K0, h0 = K0 / 2, ns = (K0 - 1) / 2;
  const size_t xs = cur.xs;
  const uint32_t* tb = tab + (size_t)K0 * 8 * kTcImgWords;  // [part][head, tail]
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_b)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_m)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_load_b(Bt, tb, &bar_b);  // stage 1, x < 40
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(tc_smem(&tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  Cplx<float> v[10][4];
  tc_fetch(spec, cur, tid, v);  // all 40 loads of a thread in flight before the first use
  tc_stage_a<0>(Arh, Arl, Aih, Ail, tid, v);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tslot;
  const uint32_t dre = tm, dim = tm + 128;
  const int q = warp & 3, half = warp >> 2, row = q * 32 + lane;
  const uint32_t lane_base = (uint32_t)(q * 32) << 16;
  const int c = cur.c0 + row;
  const bool live = row < cur.nz;
  uint32_t pb = 0, pm = 0;  // completed phases of bar_b and bar_m
  bool ok = true;
  // one contraction half: B copy awaited, products issued and committed by thread 0, then every
  // thread waits for them; the verdict is block-uniform
  auto run_half = [&](int ks, int n, bool acc) {
    if (tid == 0 && ok) {
      ok = tc_wait(&bar_b, pb & 1);
      if (ok) {
        tc_products(dre, dim, Arh, Arl, Aih, Ail, Bt, ks, n, acc);
        tc_commit(&bar_m);
      }
    }
    ++pb;
  };
  auto await_half = [&]() {
    ok = __syncthreads_and(ok) != 0;
    ok = __syncthreads_and(ok && tc_wait(&bar_m, pm & 1)) != 0;
    ++pm;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  };
  auto publish = [&]() {  // generic-proxy shared-memory writes -> the products
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  };
  // stage 1: D = A Phi over x < 40, then x >= 40
  run_half(min(5, (K0 + 7) >> 3), kTcN, false);
  await_half();
  if (K0 > kTcHalf) {
    if (tid == 0 && ok) tc_load_b(Bt, tb + 2 * (size_t)kTcImgWords, &bar_b);  // stage 1, x >= 40
    tc_stage_a<5>(Arh, Arl, Aih, Ail, tid, v);
    publish();
    run_half((K0 - kTcHalf + 7) >> 3, kTcN, true);
  }
  // the Green's function of this thread's row and k' range, loaded while the products run
  float g1[20], g2[20];
  {
    const float* G = green + cur.green_off + c;
#pragma unroll
    for (int u = 0; u < 20; ++u) {
      const int k = half * 20 + u;
      const bool in = live && k <= h0;
      g1[u] = in ? G[(size_t)k * xs] : 0.f;
      g2[u] = in ? G[(size_t)((K0 - k) % K0) * xs] : 0.f;
    }
  }
  if (K0 > kTcHalf) await_half();
  // stage 3 inputs: U (cos columns) into the A tiles now, V (sin columns) kept for the second half
  if (tid == 0 && ok) tc_load_b(Bt, tb + 4 * (size_t)kTcImgWords, &bar_b);  // stage 3, j' < 40
  const int nch = h0 >= half * 20 ? min(5, (h0 - half * 20) / 4 + 1) : 0;  // block-uniform
  float wr[20], wi[20];  // V_re, -V_im of k' = 20 half + u
  if (ok) {
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i >= nch) break;
      const int k0 = half * 20 + 4 * i;
      uint32_t ea[4], oa[4], eb[4], ob[4];
      ADMP_TC_LD4(dre + lane_base + k0, ea);
      ADMP_TC_LD4(dre + lane_base + 40 + k0, oa);
      ADMP_TC_LD4(dim + lane_base + k0, eb);
      ADMP_TC_LD4(dim + lane_base + 40 + k0, ob);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float ur[4], ui[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = k0 + u;
        const float Ea = __uint_as_float(ea[u]), Oa = __uint_as_float(oa[u]);
        const float Eb = __uint_as_float(eb[u]), Ob = __uint_as_float(ob[u]);
        const float ga = g1[4 * i + u], gb = g2[4 * i + u];
        if (k == 0 || 2 * k == K0) {  // stands alone: S = (Ea, Eb)
          ur[u] = ga * Ea;
          ui[u] = ga * Eb;
          wr[4 * i + u] = 0.f;
          wi[4 * i + u] = 0.f;
        } else {  // zero past K0 / 2 through g
          const float t1r = ga * (Ea + Ob), t1i = ga * (Eb - Oa);
          const float t2r = gb * (Ea - Ob), t2i = gb * (Eb + Oa);
          ur[u] = t1r + t2r;
          ui[u] = t1i + t2i;
          wr[4 * i + u] = t1r - t2r;
          wi[4 * i + u] = t2i - t1i;
        }
      }
      tc_put4(Arh, Arl, row, k0, ur);
      tc_put4(Aih, Ail, row, k0, ui);
    }
  }
  // chunks past K0 / 2 (and every chunk after a failed wait) hold no input: zero
  auto zero_rest = [&]() {
    for (int it = tid; it < kTcRows * (kTcHalf / 4); it += 256) {
      const int r = it & (kTcRows - 1), k4 = (it >> 7) * 4;
      if (ok && k4 <= h0) continue;
      const float z[4] = {0.f, 0.f, 0.f, 0.f};
      tc_put4(Arh, Arl, r, k4, z);
      tc_put4(Aih, Ail, r, k4, z);
    }
  };
  zero_rest();
  publish();
  // stage 3, U half: out = U Phi^T (cos columns); N = x rows, 16-aligned past K0
  const int n3 = ((K0 + 15) >> 4) << 4;
  run_half((h0 + 1 + 7) >> 3, n3, false);
  await_half();
  // V half (sin columns; V_0 = 0 and V is zero past (K0 - 1) / 2)
  if (ns >= 1) {
    if (tid == 0 && ok) tc_load_b(Bt, tb + 6 * (size_t)kTcImgWords, &bar_b);  // stage 3, j' >= 40
    if (ok) {
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        if (i >= nch) break;
        const int k0 = half * 20 + 4 * i;
        float a[4], bq[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a[u] = wi[4 * i + u];
          bq[u] = wr[4 * i + u];
        }
        tc_put4(Arh, Arl, row, k0, a);   // re row: -V_im
        tc_put4(Aih, Ail, row, k0, bq);  // im row:  V_re
      }
    }
    zero_rest();
    publish();
    run_half((ns + 1 + 7) >> 3, n3, true);
    await_half();
  }
  if (ok) {
    // epilogue: x in [40 half, 40 half + 40), eight at a time
    Cplx<float>* Ho = spec + cur.spec_off + c;
    const int nx = K0 > half * 40 ? min(5, (K0 - half * 40 + 7) / 8) : 0;  // block-uniform
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i >= nx) break;
      const int x0 = half * 40 + 8 * i;
      uint32_t vr[8], vi[8];
      ADMP_TC_LD8(dre + lane_base + x0, vr);
      ADMP_TC_LD8(dim + lane_base + x0, vi);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (live)
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int x = x0 + u;
          if (x < K0) {
            Cplx<float> o;
            o.x = __uint_as_float(vr[u]);
            o.y = __uint_as_float(vi[u]);
            Ho[(size_t)x * xs] = o;
          }
        }
    }
  } else if (tid == 0 && b.done) {
    atomicExch(const_cast<int*>(b.done) + (size_t)cur.box_idx * b.done_stride + b.status_off, ADMP_ERR_CUDA);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tm));
}

// y pass (forward, or inverse through conjugation: IDFT(h) = conj(DFT(conj(h)))) of the FP32 CG
// matvec on the tensor cores, in place on the half spectrum H[x][y][kz]: a tile is 128 lines
// r = (x, kz) of one system, line r holding H[x][.][kz] (stride K2h); stage 1 of the x pass without
// the Green's function and stage 3.  Two CTAs per SM.
template <bool INV>
static __global__ void __launch_bounds__(256, 2)
    tc_y_kernel(Batch b, Cplx<float>* __restrict__ spec, const uint32_t* __restrict__ tab) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bar_b, bar_m;
  __shared__ uint32_t tslot;
  unsigned char* Arh = tsm;
  unsigned char* Arl = Arh + kTcATile;
  unsigned char* Aih = Arl + kTcATile;
  unsigned char* Ail = Aih + kTcATile;
  unsigned char* Bt = Ail + kTcATile;  // head, tail
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = find_sys<F_YT>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];
  const int K1 = d.K1, K2h = d.K2h, h1 = K1 / 2;
  const int r0 = (blockIdx.x - d.blk_yt) * kTcRows, nz = min(kTcRows, d.K0 * K2h - r0);
  const size_t ys = (size_t)K2h, plane = (size_t)K1 * K2h;
  Cplx<float>* H = spec + d.spec_off;
  const FastDiv fk = fast_div(K2h);
  const uint32_t* tb = tab + (size_t)K1 * 8 * kTcImgWords;  // [part][head, tail]
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_b)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_m)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_load_b(Bt, tb, &bar_b);  // y < 40
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(tc_smem(&tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // the tile's lines as rows, y as columns (every load of a thread in flight before the first use)
  Cplx<float> v[10][4];
  {
    const int ca = tid & (kTcRows - 1), ya = (tid >> 7) * 4;
    const bool la = ca < nz;
    const int r = r0 + (la ? ca : 0), x = fdiv(r, fk);
    const Cplx<float>* L = H + (size_t)x * plane + (r - x * K2h);
#pragma unroll
    for (int m = 0; m < 10; ++m)
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int y = ya + 8 * m + t;
        v[m][t].x = 0.f;
        v[m][t].y = 0.f;
        if (la && y < K1) v[m][t] = L[(size_t)y * ys];
        if (INV) v[m][t].y = -v[m][t].y;
      }
  }
  tc_stage_a<0>(Arh, Arl, Aih, Ail, tid, v);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tslot;
  const uint32_t dre = tm, dim = tm + 128;
  const int q = warp & 3, half = warp >> 2, row = q * 32 + lane;
  const uint32_t lane_base = (uint32_t)(q * 32) << 16;
  uint32_t pb = 0, pm = 0;
  bool ok = true;
  auto run_half = [&](int ks, bool acc) {
    if (tid == 0 && ok) {
      ok = tc_wait(&bar_b, pb & 1);
      if (ok) {
        tc_products(dre, dim, Arh, Arl, Aih, Ail, Bt, ks, kTcN, acc);
        tc_commit(&bar_m);
      }
    }
    ++pb;
  };
  auto await_half = [&]() {
    ok = __syncthreads_and(ok) != 0;
    ok = __syncthreads_and(ok && tc_wait(&bar_m, pm & 1)) != 0;
    ++pm;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  };
  run_half(min(5, (K1 + 7) >> 3), false);
  await_half();
  if (K1 > kTcHalf) {
    if (tid == 0 && ok) tc_load_b(Bt, tb + 2 * (size_t)kTcImgWords, &bar_b);  // y >= 40
    tc_stage_a<5>(Arh, Arl, Aih, Ail, tid, v);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    run_half((K1 - kTcHalf + 7) >> 3, true);
    await_half();
  }
  if (ok) {
    // S_k = Ea + Ob + i (Eb - Oa) for k <= K1 / 2, S_{K1-k} = Ea - Ob + i (Eb + Oa) for 1 <= k < K1 / 2
    // (the sine columns of k = 0 and of the Nyquist index are zero)
    const bool live = row < nz;
    const int r = r0 + (live ? row : 0), x = fdiv(r, fk);
    Cplx<float>* L = H + (size_t)x * plane + (r - x * K2h);
    const int nch = h1 >= half * 20 ? min(5, (h1 - half * 20) / 4 + 1) : 0;  // block-uniform
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i >= nch) break;
      const int k0 = half * 20 + 4 * i;
      uint32_t ea[4], oa[4], eb[4], ob[4];
      ADMP_TC_LD4(dre + lane_base + k0, ea);
      ADMP_TC_LD4(dre + lane_base + 40 + k0, oa);
      ADMP_TC_LD4(dim + lane_base + k0, eb);
      ADMP_TC_LD4(dim + lane_base + 40 + k0, ob);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (live)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + u;
          if (k > h1) break;
          const float Ea = __uint_as_float(ea[u]), Oa = __uint_as_float(oa[u]);
          const float Eb = __uint_as_float(eb[u]), Ob = __uint_as_float(ob[u]);
          Cplx<float> o;
          o.x = Ea + Ob;
          o.y = INV ? Oa - Eb : Eb - Oa;
          L[(size_t)k * ys] = o;
          if (k >= 1 && 2 * k != K1) {
            o.x = Ea - Ob;
            o.y = INV ? -(Eb + Oa) : Eb + Oa;
            L[(size_t)(K1 - k) * ys] = o;
          }
        }
    }
  } else if (tid == 0 && b.done) {
    atomicExch(const_cast<int*>(b.done) + (size_t)d.box_idx * b.done_stride + b.status_off, ADMP_ERR_CUDA);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tm));
}

// Products of a real operand: D += A B over ks K-steps, head*head + head*tail + tail*head.
__device__ __forceinline__ void tc_products_real(uint32_t dt, const unsigned char* Ah, const unsigned char* Al,
                                                 const unsigned char* Bt, int ks, int n, bool acc) {
  const uint32_t id = tc_idesc(n);
  const uint64_t ah = tc_desc(tc_smem(Ah)), al = tc_desc(tc_smem(Al)), bh = tc_desc(tc_smem(Bt)),
                 bl = tc_desc(tc_smem(Bt + kTcBTile));
  for (int k = 0; k < ks; ++k) {
    const uint64_t o = (uint64_t)k * 16;
    tc_mma(dt, ah + o, bh + o, id, (acc || k > 0) ? 1u : 0u);
    tc_mma(dt, ah + o, bl + o, id, 1u);
    tc_mma(dt, al + o, bh + o, id, 1u);
  }
}

// Asynchronous global -> shared copies of 4 or 8 bytes (cp.async, no register round trip): a thread
// issues all of its copies before waiting, so the staging of a tile is one memory latency.
template <int BYTES>
__device__ __forceinline__ void tc_cp_async(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(tc_smem(smem)), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void tc_cp_async_wait() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Shared state of the z passes: a tile is 128 lines r = (x, y) of one system (contiguous in both
// the mesh, K2 reals a line, and the half spectrum, K2h complex a line), staged through shared
// memory so that global loads and stores are coalesced.  Layout: A head / tail (one 40-column half),
// the staging area (40 KB), B head / tail.  TMEM: one accumulator of 128 columns.
struct TcZ {
  unsigned char *Ah, *Al, *Bt;
  float* S;
  uint64_t *bar_b, *bar_m;
  uint32_t tm;
  uint32_t pb, pm;
  bool ok;
};

__device__ __forceinline__ void tc_z_half(TcZ& z, int tid, int ks, int n, bool acc) {
  if (tid == 0 && z.ok) {
    z.ok = tc_wait(z.bar_b, z.pb & 1);
    if (z.ok) {
      tc_products_real(z.tm, z.Ah, z.Al, z.Bt, ks, n, acc);
      tc_commit(z.bar_m);
    }
  }
  ++z.pb;
  z.ok = __syncthreads_and(z.ok) != 0;
  z.ok = __syncthreads_and(z.ok && tc_wait(z.bar_m, z.pm & 1)) != 0;
  ++z.pm;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_publish() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// z pass forward (real to half spectrum): H[r][kz] = sum_z q[r][z] (cos - i sin)(2 pi z kz / K2),
// i.e. D = A Phi with the cosine columns kz and the sine columns 40 + kz.  Two CTAs per SM.
static __global__ void __launch_bounds__(256, 2)
    tc_zf_kernel(Batch b, const float* __restrict__ mesh, Cplx<float>* __restrict__ spec,
                 const uint32_t* __restrict__ tab) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bar_b, bar_m;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = find_sys<F_ZT>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];
  const int K2 = d.K2, K2h = d.K2h;
  const int r0 = (blockIdx.x - d.blk_zt) * kTcRows, nz = min(kTcRows, d.K0 * d.K1 - r0);
  TcZ z;
  z.Ah = tsm;
  z.Al = z.Ah + kTcATile;
  z.S = reinterpret_cast<float*>(z.Al + kTcATile);
  z.Bt = z.Al + 3 * kTcATile;
  z.bar_b = &bar_b;
  z.bar_m = &bar_m;
  z.pb = z.pm = 0;
  z.ok = true;
  const uint32_t* tb = tab + (size_t)K2 * 8 * kTcImgWords;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_b)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_m)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_load_b(z.Bt, tb, &bar_b);  // z < 40
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(tc_smem(&tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  {
    const float* Q = mesh + d.mesh_off + (size_t)r0 * K2;
    const int n = nz * K2;
    for (int i = tid; i < n; i += 256) tc_cp_async<4>(z.S + i, Q + i);
    tc_cp_async_wait();
  }
  __syncthreads();
  z.tm = tslot;
  const int ca = tid & (kTcRows - 1), za = (tid >> 7) * 4;
  auto fill = [&](int hh) {
#pragma unroll
    for (int mm = 0; mm < 5; ++mm) {
      float v[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int zz = kTcHalf * hh + za + 8 * mm + t;
        v[t] = (ca < nz && zz < K2) ? z.S[ca * K2 + zz] : 0.f;
      }
      tc_put4(z.Ah, z.Al, ca, za + 8 * mm, v);
    }
  };
  fill(0);
  tc_publish();
  tc_z_half(z, tid, min(5, (K2 + 7) >> 3), kTcN, false);
  if (K2 > kTcHalf) {
    if (tid == 0 && z.ok) tc_load_b(z.Bt, tb + 2 * (size_t)kTcImgWords, &bar_b);  // z >= 40
    fill(1);
    tc_publish();
    tc_z_half(z, tid, (K2 - kTcHalf + 7) >> 3, kTcN, true);
  }
  // D -> H (cos, -sin) into the staging area as [row][kz], then coalesced stores
  const int q = warp & 3, half = warp >> 2, row = q * 32 + lane;
  const uint32_t lb = z.tm + ((uint32_t)(q * 32) << 16);
  Cplx<float>* Sc = reinterpret_cast<Cplx<float>*>(z.S);
  if (z.ok) {
    const int nch = K2h - 1 >= half * 20 ? min(5, (K2h - 1 - half * 20) / 4 + 1) : 0;  // block-uniform
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i >= nch) break;
      const int k0 = half * 20 + 4 * i;
      uint32_t c4[4], s4[4];
      ADMP_TC_LD4(lb + k0, c4);
      ADMP_TC_LD4(lb + 40 + k0, s4);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = k0 + u;
        if (k < K2h) {
          Cplx<float> o;
          o.x = __uint_as_float(c4[u]);
          o.y = -__uint_as_float(s4[u]);
          Sc[row * K2h + k] = o;
        }
      }
    }
  } else if (tid == 0 && b.done) {
    atomicExch(const_cast<int*>(b.done) + (size_t)d.box_idx * b.done_stride + b.status_off, ADMP_ERR_CUDA);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (z.ok) {
    Cplx<float>* H = spec + d.spec_off + (size_t)r0 * K2h;
    const int n = nz * K2h;
    for (int i = tid; i < n; i += 256) H[i] = Sc[i];
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(z.tm));
}

// z pass inverse (half spectrum to real, unnormalised): q[r][z] = sum_k w_k (Re S_k cos - Im S_k sin)
// with w = 1 at k = 0 and at the Nyquist index, 2 elsewhere, i.e. A = [w Re S | -w Im S] and
// q = A Phi^T (the cosine half, then the sine half).  Two CTAs per SM.
static __global__ void __launch_bounds__(256, 2)
    tc_zi_kernel(Batch b, const Cplx<float>* __restrict__ spec, float* __restrict__ mesh,
                 const uint32_t* __restrict__ tab) {
  extern __shared__ __align__(1024) unsigned char tsm[];
  __shared__ __align__(8) uint64_t bar_b, bar_m;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int s = find_sys<F_ZT>(b, blockIdx.x);
  if (skip_sys(b, s)) return;
  const SysDesc& d = b.s[s];
  const int K2 = d.K2, K2h = d.K2h, ns = (K2 - 1) / 2;
  const int r0 = (blockIdx.x - d.blk_zt) * kTcRows, nz = min(kTcRows, d.K0 * d.K1 - r0);
  TcZ z;
  z.Ah = tsm;
  z.Al = z.Ah + kTcATile;
  z.S = reinterpret_cast<float*>(z.Al + kTcATile);
  z.Bt = z.Al + 3 * kTcATile;
  z.bar_b = &bar_b;
  z.bar_m = &bar_m;
  z.pb = z.pm = 0;
  z.ok = true;
  const uint32_t* tb = tab + (size_t)K2 * 8 * kTcImgWords;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_b)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_m)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_load_b(z.Bt, tb + 4 * (size_t)kTcImgWords, &bar_b);  // cosine columns
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(tc_smem(&tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  Cplx<float>* Sc = reinterpret_cast<Cplx<float>*>(z.S);
  {
    const Cplx<float>* H = spec + d.spec_off + (size_t)r0 * K2h;
    const int n = nz * K2h;
    for (int i = tid; i < n; i += 256) tc_cp_async<8>(Sc + i, H + i);
    tc_cp_async_wait();
  }
  __syncthreads();
  z.tm = tslot;
  const int ca = tid & (kTcRows - 1), ka = (tid >> 7) * 4;
  // hh = 0: w Re S_k at column k (k <= K2 / 2); hh = 1: -w Im S_k at column k (1 <= k <= ns)
  auto fill = [&](int hh) {
#pragma unroll
    for (int mm = 0; mm < 5; ++mm) {
      float v[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int k = ka + 8 * mm + t;
        const bool in = ca < nz && (hh == 0 ? k < K2h : (k >= 1 && k <= ns));
        const float w = (k == 0 || 2 * k == K2) ? 1.f : 2.f;
        v[t] = 0.f;
        if (in) {
          const Cplx<float> e = Sc[ca * K2h + k];
          v[t] = hh == 0 ? w * e.x : -w * e.y;
        }
      }
      tc_put4(z.Ah, z.Al, ca, ka + 8 * mm, v);
    }
  };
  const int n3 = ((K2 + 15) >> 4) << 4;
  fill(0);
  tc_publish();
  tc_z_half(z, tid, (K2h + 7) >> 3, n3, false);
  if (ns >= 1) {
    if (tid == 0 && z.ok) tc_load_b(z.Bt, tb + 6 * (size_t)kTcImgWords, &bar_b);  // sine columns
    fill(1);
    tc_publish();
    tc_z_half(z, tid, (ns + 1 + 7) >> 3, n3, true);
  }
  // D -> q[row][z] into the staging area, then coalesced stores
  const int q = warp & 3, half = warp >> 2, row = q * 32 + lane;
  const uint32_t lb = z.tm + ((uint32_t)(q * 32) << 16);
  if (z.ok) {
    const int nx = K2 > half * 40 ? min(5, (K2 - half * 40 + 7) / 8) : 0;  // block-uniform
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      if (i >= nx) break;
      const int z0 = half * 40 + 8 * i;
      uint32_t v8[8];
      ADMP_TC_LD8(lb + z0, v8);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (z0 + u < K2) z.S[row * K2 + z0 + u] = __uint_as_float(v8[u]);
    }
  } else if (tid == 0 && b.done) {
    atomicExch(const_cast<int*>(b.done) + (size_t)d.box_idx * b.done_stride + b.status_off, ADMP_ERR_CUDA);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (z.ok) {
    float* Q = mesh + d.mesh_off + (size_t)r0 * K2;
    const int n = nz * K2;
    for (int i = tid; i < n; i += 256) Q[i] = z.S[i];
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(z.tm));
}

}  // namespace admp
