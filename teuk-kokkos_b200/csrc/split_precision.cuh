// Split-precision tensor-core arithmetic shared by the stage kernels and the
// second-order angular operators.
//
// Method (Ozaki, Ogita, Oishi & Rump, "Error-free transformations of matrix
// multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012): a real row of one operand and
// a real column of the other are scaled by powers of two to below 1 in
// modulus and cut into five signed 8-bit digits,
//     w = sum_s t_s 2^(-7-8s),   |t_s| <= 128   (s = 0..4),
// each exact in BF16.  A digit product is an integer below 2^14, and a sum
// over K <= 64 of up to five digit pairs stays below 2^24, so BF16 tensor-core
// products accumulated in FP32 (mma.sync m16n8k16) are exact.  The 15 pairs
// with s + t <= 4 go into five FP32 accumulators (one per u = s + t) and are
// recombined in FP64:
//     sum_k x_k y_k = 2^(E_x + E_y - 14) sum_u 2^(-8u) D_u.
// The dropped pairs (u >= 5) and the digit remainders leave an error of
// about 2^-40 of max|x| max|y| per product term.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

namespace teuk_b200 {
namespace split {

inline constexpr int kSlices = 5;

// D += A B for one m16n8k16 BF16 tile with FP32 accumulation.
__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4],
                                         const uint2 b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// The five digits of w (|w| < 1); every step is exact in binary64.
__device__ __forceinline__ void digits(const double w, float (&t)[kSlices]) {
  double r = w * 128.0;
#pragma unroll
  for (int s = 0; s < kSlices; ++s) {
    const double d = rint(r);
    t[s] = static_cast<float>(d);
    r = (r - d) * 256.0;
  }
}

// Two digits as BF16 in one register, `lo` in the low half (exact: they are
// integers of at most 8 bits).
__device__ __forceinline__ unsigned pack(const float lo, const float hi) {
  return (__float_as_uint(lo) >> 16) | (__float_as_uint(hi) & 0xffff0000u);
}

// e with m = f 2^e, f in [0.5, 1): 2^-e brings every |v| <= m below 1
// (0 for m = 0; at least -1000 so the scales stay finite).
__device__ __forceinline__ int exponent(const double m) {
  int e = 0;
  frexp(m, &e);
  return m == 0.0 ? 0 : max(e, -1000);
}

// FP64 value of the five accumulators: sum_u 2^(-8u) D_u (times the scales).
__device__ __forceinline__ double recombine(const float (&d)[kSlices][4],
                                            const int c) {
  double sum = static_cast<double>(d[kSlices - 1][c]);
#pragma unroll
  for (int u = kSlices - 2; u >= 0; --u) {
    sum = fma(sum, 1.0 / 256.0, static_cast<double>(d[u][c]));
  }
  return sum;
}

// ----------------------------------------------------------------- host
inline int host_exponent(const double m) {
  int e = 0;
  std::frexp(m, &e);
  return m == 0.0 ? 0 : (e < -1000 ? -1000 : e);
}

inline void host_digits(const double w, float (&t)[kSlices]) {
  double r = w * 128.0;
  for (int s = 0; s < kSlices; ++s) {
    const double d = std::nearbyint(r);
    t[s] = static_cast<float>(d);
    r = (r - d) * 256.0;
  }
}

inline unsigned host_pack(const float lo, const float hi) {
  unsigned a = 0, b = 0;
  std::memcpy(&a, &lo, sizeof(a));
  std::memcpy(&b, &hi, sizeof(b));
  return (a >> 16) | (b & 0xffff0000u);
}

}  // namespace split
}  // namespace teuk_b200
