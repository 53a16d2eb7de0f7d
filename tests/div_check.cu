// div_check.cu -- FastDiv (hormone_b200/csrc/hmn_div.cuh) against IEEE
// division on the GPU: for every operand pair that FastDiv does not flag,
// its reciprocal must equal 1.0/b and its quotient a/b bit for bit.
//
//   div_check N SEED     N pairs per operand family; prints one line
//                        "<family> pairs=<n> flagged=<n> mismatches=<n>"
//                        per family and exits 1 on any mismatch.
//
// Families: random significands over the whole checked exponent range;
// operands near the range limits; significands with long runs of ones or
// zeros (where rounding is closest to a tie); b a power of two; a = 0 of
// either sign; quotients of nearly equal operands.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "hmn_div.cuh"

using hmn::div_rn;
using hmn::recip_rn;

__device__ __forceinline__ uint64_t mix(uint64_t x) {  // splitmix64
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

__device__ double make(uint64_t r, int fam, int which) {
  const uint64_t sign = (r >> 63) << 63;
  uint64_t mant = r & 0xfffffffffffffull;
  int e;
  switch (fam) {
    case 0:  // anywhere in [2^-520, 2^520]
      e = (int)((r >> 52) % 1041) - 520;
      break;
    case 1:  // at the checked limits 2^-500 and 2^500 and just outside
      e = (int)((r >> 52) % 8) - 4 + (((r >> 60) & 1) ? 500 : -500);
      break;
    case 2: {  // long runs of ones or zeros in the significand
      const int len = (int)((r >> 52) % 52) + 1;
      const uint64_t run = ((1ull << len) - 1) << (52 - len);
      mant = ((r >> 57) & 1) ? (mant | run) : (mant & ~run);
      e = (int)((r >> 58) % 41) - 20;
      break;
    }
    case 3:  // b a power of two (a random)
      if (which == 1) mant = 0;
      e = (int)((r >> 52) % 81) - 40;
      break;
    case 4:  // a = +0 or -0
      if (which == 0) return __longlong_as_double((long long)sign);
      e = (int)((r >> 52) % 81) - 40;
      break;
    default:  // a and b within a few ulps of each other
      e = (int)((r >> 52) % 21) - 10;
      break;
  }
  const uint64_t bits = sign | ((uint64_t)(e + 1023) << 52) | mant;
  return __longlong_as_double((long long)bits);
}

__global__ void check(int fam, long long n, unsigned long long seed, unsigned long long* bad,
                      unsigned long long* flagged, double* ex) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const uint64_t r0 = mix(seed * 0x100000001b3ull + 2 * (uint64_t)t), r1 = mix(r0 ^ 0x5bd1e995u);
    double a = make(r0, fam, 0), b = make(r1, fam, 1);
    if (fam == 5) {  // b = a moved by a few ulps
      const long long k = (long long)(r1 % 9) - 4;
      b = __longlong_as_double(__double_as_longlong(a) + k);
    }
    bool flag = false;
    const double y = recip_rn(b, flag);
    const double q = div_rn(a, b, y, flag);
    if (flag) {
      atomicAdd(flagged, 1ull);
      continue;
    }
    const double yr = 1.0 / b, qr = a / b;
    if (__double_as_longlong(y) != __double_as_longlong(yr) || __double_as_longlong(q) != __double_as_longlong(qr)) {
      if (atomicAdd(bad, 1ull) == 0) {
        ex[0] = a;
        ex[1] = b;
        ex[2] = q;
        ex[3] = qr;
      }
    }
  }
}

int main(int argc, char** argv) {
  const long long n = argc > 1 ? atoll(argv[1]) : (1ll << 24);
  const unsigned long long seed = argc > 2 ? strtoull(argv[2], nullptr, 10) : 1;
  unsigned long long *d_bad, *d_fl;
  double* d_ex;
  if (cudaMalloc(&d_bad, 8) != cudaSuccess || cudaMalloc(&d_fl, 8) != cudaSuccess ||
      cudaMalloc(&d_ex, 4 * sizeof(double)) != cudaSuccess) {
    fprintf(stderr, "cudaMalloc failed\n");
    return 2;
  }
  const char* names[6] = {"random", "range_limits", "runs_of_ones_or_zeros", "b_power_of_two", "a_zero",
                          "nearly_equal"};
  int fail = 0;
  for (int fam = 0; fam < 6; fam++) {
    cudaMemset(d_bad, 0, 8);
    cudaMemset(d_fl, 0, 8);
    check<<<148 * 8, 256>>>(fam, n, seed + 1000003ull * fam, d_bad, d_fl, d_ex);
    if (cudaDeviceSynchronize() != cudaSuccess) {
      fprintf(stderr, "kernel failed: %s\n", cudaGetErrorString(cudaGetLastError()));
      return 2;
    }
    unsigned long long bad = 0, fl = 0;
    double ex[4];
    cudaMemcpy(&bad, d_bad, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(&fl, d_fl, 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ex, d_ex, sizeof(ex), cudaMemcpyDeviceToHost);
    printf("%s pairs=%lld flagged=%llu mismatches=%llu\n", names[fam], n, fl, bad);
    if (bad) {
      printf("  e.g. a=%a b=%a fast=%a ieee=%a\n", ex[0], ex[1], ex[2], ex[3]);
      fail = 1;
    }
  }
  return fail;
}
