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
// kTcSbo bytes apart along M/N (SBO).  Each tile is 80 columns (K) wide.
// Per CTA: A = 4 tiles of 128 x 80 (re / im, head / tail), B = 2 tiles of
// 80 x 80 (head / tail), 210 KB of shared memory; TMEM: 256 columns (the
// real accumulator at column 0, the imaginary one at column 128).  The two
// B images per mesh length (Phi^T for stage 1, Phi for stage 3, head and
// tail) are built once per device in global memory and copied into shared
// memory by 1-D bulk asynchronous copies (the TMA engine, no tensor map,
// no multicast) on an mbarrier.  Every wait is bounded; on expiry the
// system's CG status is set and the kernel returns after freeing its TMEM.
#pragma once

#include <cstddef>
#include <cstdint>

#include "pme_kernels.cuh"

namespace admp {

constexpr int kTcMaxK = 79;               // longest x line of this path (40 cos + 40 sin columns)
constexpr int kTcRows = 128;              // flattened columns per CTA (MMA M)
constexpr int kTcCols = 80;               // K width of every operand tile, N of stage 1
constexpr int kTcSbo = (kTcCols / 4) * 128;
constexpr int kTcATile = kTcRows * kTcCols * 4;  // bytes
constexpr int kTcBTile = kTcCols * kTcCols * 4;
constexpr int kTcSmem = 4 * kTcATile + 2 * kTcBTile;
constexpr int kTcImgWords = kTcCols * kTcCols;   // one B image
constexpr long long kTcSpin = 1LL << 24;

// byte offset of (row r, column k) in a K-major no-swizzle tile
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

// the two B images (head, tail) of one stage: 2 x 25,600 bytes by the bulk-copy engine
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

// The B images of every mesh length 1..kTcMaxK, [K0][stage 1 head, stage 1
// tail, stage 3 head, stage 3 tail][kTcImgWords] (dft_tc.cu): built on the
// current device at the first call (ordered on `st` and waited for, so any
// stream may read them afterwards).  nullptr if they cannot be built.
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

// A thread's part of a tile's spectrum: column tid % 128, x runs (tid / 128) * 4 + 8 m (m < 10)
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

__device__ __forceinline__ void tc_stage_a(unsigned char* Arh, unsigned char* Arl, unsigned char* Aih,
                                           unsigned char* Ail, int tid, const Cplx<float> (&v)[10][4]) {
  const int ca = tid & (kTcRows - 1), xa = (tid >> 7) * 4;
#pragma unroll
  for (int m = 0; m < 10; ++m) {
    float re[4], im[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      re[t] = v[m][t].x;
      im[t] = v[m][t].y;
    }
    tc_put4(Arh, Arl, ca, xa + 8 * m, re);
    tc_put4(Aih, Ail, ca, xa + 8 * m, im);
  }
}

// One CTA per tile (210 KB of shared memory: one CTA per SM), 256 threads.  (A grid of one CTA per
// SM walking its tiles, loading the next tile's spectrum into registers during the current tile's
// products, measured 5% slower: static tile assignment over systems of unequal mesh length.)
static __global__ void __launch_bounds__(256, 1)
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
  const int K0 = cur.K0;
  const size_t xs = cur.xs;
  const uint32_t* tb = tab + (size_t)K0 * 4 * kTcImgWords;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_b)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem(&bar_m)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_load_b(Bt, tb, &bar_b);  // stage 1 images
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(tc_smem(&tslot)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  {
    Cplx<float> v[10][4];
    tc_fetch(spec, cur, tid, v);  // all 40 loads of a thread in flight before the first use
    tc_stage_a(Arh, Arl, Aih, Ail, tid, v);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tm = tslot;
  const uint32_t dre = tm, dim = tm + 128;
  const int q = warp & 3, half = warp >> 2, row = q * 32 + lane;
  const uint32_t lane_base = (uint32_t)(q * 32) << 16;
  bool ok = true;
  {
    // stage 1: D_re = A_re Phi, D_im = A_im Phi over ceil(K0 / 8) K-steps
    if (tid == 0) {
      ok = tc_wait(&bar_b, 0);
      if (ok) {
        const uint32_t id = tc_idesc(kTcCols);
        const uint32_t a_r[2] = {tc_smem(Arh), tc_smem(Arl)}, a_i[2] = {tc_smem(Aih), tc_smem(Ail)};
        const uint32_t bb[2] = {tc_smem(Bt), tc_smem(Bt + kTcBTile)};
        const int ks = (K0 + 7) >> 3;
        for (int k = 0; k < ks; ++k)
          for (int u = 0; u < 3; ++u) {  // head*head, head*tail, tail*head
            const int ia = u == 2 ? 1 : 0, ib = u == 1 ? 1 : 0;
            const uint32_t acc = (k > 0 || u > 0) ? 1u : 0u;
            tc_mma(dre, tc_desc(a_r[ia] + k * 256), tc_desc(bb[ib] + k * 256), id, acc);
            tc_mma(dim, tc_desc(a_i[ia] + k * 256), tc_desc(bb[ib] + k * 256), id, acc);
          }
        tc_commit(&bar_m);
      }
    }
    // the Green's function of this thread's row and k' range, loaded while the products run
    const int c = cur.c0 + row;
    const bool live = row < cur.nz;
    float g1[20], g2[20];
    {
      const float* G = green + cur.green_off + c;
#pragma unroll
      for (int u = 0; u < 20; ++u) {
        const int k = half * 20 + u;
        const bool in = live && k <= K0 / 2;
        g1[u] = in ? G[(size_t)k * xs] : 0.f;
        g2[u] = in ? G[(size_t)((K0 - k) % K0) * xs] : 0.f;
      }
    }
    ok = __syncthreads_and(ok) != 0;  // thread 0's verdict (the others hold true)
    ok = __syncthreads_and(ok && tc_wait(&bar_m, 0)) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // the B region is free once stage 1 has completed: stage 3 images
    if (tid == 0 && ok) tc_load_b(Bt, tb + 2 * (size_t)kTcImgWords, &bar_b);
    if (ok) {
      // epilogue 1: k' in [20 half, 20 half + 20), four at a time
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const int k0 = half * 20 + 4 * i;
        if (k0 > K0 / 2) break;  // block-uniform
        uint32_t ea[4], oa[4], eb[4], ob[4];
        ADMP_TC_LD4(dre + lane_base + k0, ea);
        ADMP_TC_LD4(dre + lane_base + 40 + k0, oa);
        ADMP_TC_LD4(dim + lane_base + k0, eb);
        ADMP_TC_LD4(dim + lane_base + 40 + k0, ob);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        float ur[4], ui[4], vr[4], nvi[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int k = k0 + u;
          const float Ea = __uint_as_float(ea[u]), Oa = __uint_as_float(oa[u]);
          const float Eb = __uint_as_float(eb[u]), Ob = __uint_as_float(ob[u]);
          const float ga = g1[4 * i + u], gb = g2[4 * i + u];
          if (k == 0 || 2 * k == K0) {  // stands alone: S = (Ea, Eb)
            ur[u] = ga * Ea;
            ui[u] = ga * Eb;
            vr[u] = 0.f;
            nvi[u] = 0.f;
          } else {  // zero past K0 / 2 through g
            const float t1r = ga * (Ea + Ob), t1i = ga * (Eb - Oa);
            const float t2r = gb * (Ea - Ob), t2i = gb * (Eb + Oa);
            ur[u] = t1r + t2r;
            ui[u] = t1i + t2i;
            vr[u] = t1r - t2r;
            nvi[u] = t2i - t1i;
          }
        }
        tc_put4(Arh, Arl, row, k0, ur);
        tc_put4(Arh, Arl, row, 40 + k0, nvi);
        tc_put4(Aih, Ail, row, k0, ui);
        tc_put4(Aih, Ail, row, 40 + k0, vr);
      }
    }
    // columns the loop above did not reach still hold stage 1 inputs: zero them (their B rows are
    // zero too, but stale tails could hold non-finite bit patterns)
    for (int it = tid; it < kTcRows * 20; it += 256) {
      const int r = it & (kTcRows - 1), k4 = (it >> 7) * 4;  // k4 in [0, 80)
      const int kk = k4 < 40 ? k4 : k4 - 40;
      if (ok && kk <= K0 / 2) continue;
      const float z[4] = {0.f, 0.f, 0.f, 0.f};
      tc_put4(Arh, Arl, r, k4, z);
      tc_put4(Aih, Ail, r, k4, z);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // stage 3: out_re = A3_re Phi^T, out_im = A3_im Phi^T (N = x rows, 16-aligned past K0)
    if (tid == 0 && ok) {
      ok = tc_wait(&bar_b, 1);
      if (ok) {
        const uint32_t id = tc_idesc(((K0 + 15) >> 4) << 4);
        const uint32_t a_r[2] = {tc_smem(Arh), tc_smem(Arl)}, a_i[2] = {tc_smem(Aih), tc_smem(Ail)};
        const uint32_t bb[2] = {tc_smem(Bt), tc_smem(Bt + kTcBTile)};
        for (int k = 0; k < kTcCols / 8; ++k)
          for (int u = 0; u < 3; ++u) {
            const int ia = u == 2 ? 1 : 0, ib = u == 1 ? 1 : 0;
            const uint32_t acc = (k > 0 || u > 0) ? 1u : 0u;
            tc_mma(dre, tc_desc(a_r[ia] + k * 256), tc_desc(bb[ib] + k * 256), id, acc);
            tc_mma(dim, tc_desc(a_i[ia] + k * 256), tc_desc(bb[ib] + k * 256), id, acc);
          }
        tc_commit(&bar_m);
      }
    }
    ok = __syncthreads_and(ok) != 0;
    ok = __syncthreads_and(ok && tc_wait(&bar_m, 1)) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
      // epilogue 3: x in [40 half, 40 half + 40), eight at a time
      Cplx<float>* Ho = spec + cur.spec_off + c;
#pragma unroll
      for (int i = 0; i < 5; ++i) {
        const int x0 = half * 40 + 8 * i;
        if (x0 >= K0) break;  // block-uniform
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
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tm));
}

}  // namespace admp
