// Integer division by a divisor fixed at launch time, for index decoding.
#pragma once
#include <cstdint>

namespace grb {

// Unsigned 32-bit division by an invariant divisor d >= 1 with one
// multiply-high (Granlund and Montgomery, "Division by Invariant Integers
// using Multiplication", PLDI 1994, section 4, Figure 4.1): with
// l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1,
// n / d = (t + ((n - t) >> min(l, 1))) >> max(l - 1, 0), t = mulhi(m, n),
// exact for every 32-bit n.  d = 0 marks an unset divisor.
struct FastDiv {
  uint32_t d = 0, m = 0;
  int s1 = 0, s2 = 0;
};
inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  int l = 0;
  while ((1ull << l) < d) ++l;
  f.d = d;
  f.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
  f.s1 = l < 1 ? l : 1;
  f.s2 = l > 1 ? l - 1 : 0;
  return f;
}
__host__ __device__ __forceinline__ uint32_t fast_div(uint32_t n, const FastDiv& f) {
#ifdef __CUDA_ARCH__
  const uint32_t t = __umulhi(f.m, n);
#else
  const uint32_t t = (uint32_t)(((uint64_t)f.m * n) >> 32);
#endif
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

}  // namespace grb
