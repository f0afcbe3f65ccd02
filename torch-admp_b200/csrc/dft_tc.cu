// Tables of the tensor-core x pass (dft_tc.cuh): the real DFT matrix Phi of
// every mesh length 1..kTcMaxK as shared-memory images (K-major, no swizzle),
// split into TF32 head and tail.
#include <mutex>

#include "dft_tc.cuh"

namespace admp {

static __device__ __align__(128) uint32_t g_tc_tab[kTcMaxK + 1][4][2][kTcImgWords];

// Phi[x][j']: cos(2 pi x j' / K0) for j' <= K0 / 2 (j' < 40); sin(2 pi x (j' - 40) / K0) for
// 1 <= j' - 40 <= (K0 - 1) / 2; zero elsewhere and for x >= K0.  Arguments reduced exactly mod K0.
__device__ double tc_phi(int K0, int x, int j) {
  if (x >= K0) return 0.0;
  double s, c;
  if (j < 40) {
    if (j > K0 / 2) return 0.0;
    sincospi(2.0 * (double)((x * j) % K0) / (double)K0, &s, &c);
    return c;
  }
  const int k = j - 40;
  if (k < 1 || k > (K0 - 1) / 2) return 0.0;
  sincospi(2.0 * (double)((x * k) % K0) / (double)K0, &s, &c);
  return s;
}

// Part 0 / 1: rows j' (0..79), columns x - 40 part (stage 1); part 2 / 3: rows x (0..79), columns
// j' - 40 (part - 2) (stage 3).  Head and tail images of each.
static __global__ void tc_table_kernel() {
  const int K0 = blockIdx.x + 1;
  for (int e = threadIdx.x; e < 4 * kTcN * kTcHalf; e += blockDim.x) {
    const int part = e / (kTcN * kTcHalf), rem = e % (kTcN * kTcHalf);
    const int r = rem / kTcHalf, k = rem % kTcHalf;
    const float p = part < 2 ? (float)tc_phi(K0, k + kTcHalf * part, r) : (float)tc_phi(K0, r, k + kTcHalf * (part - 2));
    const int w = tc_off(r, k) >> 2;
    const uint32_t h = tf32_head(p);
    g_tc_tab[K0][part][0][w] = h;
    g_tc_tab[K0][part][1][w] = tf32_head(p - __uint_as_float(h));
  }
}

const uint32_t* tc_tables(cudaStream_t st) {
  static std::mutex mu;
  static const uint32_t* base[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!base[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_tc_tab) != cudaSuccess) return nullptr;
    tc_table_kernel<<<kTcMaxK, 256, 0, st>>>();
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) return nullptr;
    base[dev] = (const uint32_t*)p;
  }
  return base[dev];
}

}  // namespace admp
