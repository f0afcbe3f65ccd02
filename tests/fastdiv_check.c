/* Exhaustive check of the FastDiv multiply-high division used for the
 * shared-memory FFT indexing (torch-admp_b200/csrc/fft_smem.cuh, fast_div /
 * fdiv): q = (x * m) >> 32 must equal x / d for every divisor 2 <= d <= DMAX
 * and every dividend 0 <= x < 2^16.
 *
 *   device form: m = (unsigned) ru(2^32 * ru(1 / d)) + 1, with ru() the
 *                single-precision operation rounded towards +infinity
 *                (__frcp_ru, __fmul_ru; both correctly rounded), emulated
 *                here with the FE_UPWARD rounding mode;
 *   host form:   m = floor((2^32 - 1) / d) + 1.
 *
 * Prints "ok <divisors>" and exits 0 when every quotient is exact; otherwise
 * prints the first failure and exits 1.  Build with -frounding-math so the
 * float operations are not folded under the default rounding mode. */
#include <fenv.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

static unsigned device_m(int d) {
  volatile float fd = (float)d;
  fesetround(FE_UPWARD);
  volatile float r = 1.0f / fd;
  volatile float p = 4294967296.0f * r;
  fesetround(FE_TONEAREST);
  return (unsigned)p + 1u;
}

static unsigned host_m(int d) { return 0xFFFFFFFFu / (unsigned)d + 1u; }

static int check(const char* form, int d, unsigned m) {
  for (uint32_t x = 0; x < 65536u; ++x) {
    const uint32_t q = (uint32_t)(((uint64_t)x * m) >> 32);
    if (q != x / (uint32_t)d) {
      printf("FAIL %s d=%d x=%u m=%u q=%u expected %u\n", form, d, x, m, q, x / (uint32_t)d);
      return 1;
    }
  }
  return 0;
}

int main(int argc, char** argv) {
  const int dmax = argc > 1 ? atoi(argv[1]) : 65000;
  int bad = 0;
  /* divisors in parallel when built with -fopenmp (the rounding mode is per thread) */
#pragma omp parallel for schedule(dynamic, 256) reduction(| : bad)
  for (int d = 2; d <= dmax; ++d) bad |= check("device", d, device_m(d)) | check("host", d, host_m(d));
  if (bad) return 1;
  printf("ok %d\n", dmax - 1);
  return 0;
}
