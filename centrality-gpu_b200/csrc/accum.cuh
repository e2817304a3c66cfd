// Device helpers shared by the per-source kernels: IEEE-754 exponent
// arithmetic for power-of-two scaling, and the fixed-point BC counters
// (plain.h: kAccDigits digits of kAccDigitBits bits, kAccFrac fractional bits).
#pragma once
#include "common.cuh"
#include "plain.h"

namespace bcg {

// Biased IEEE-754 exponent field of a double (0: zero or subnormal, 2047: inf or NaN).
__device__ __forceinline__ int exp_bits(double v) {
  return (int)((unsigned long long)__double_as_longlong(v) >> 52) & 0x7ff;
}

// 2^e for -1022 <= e <= 1023, built from its IEEE-754 exponent field.
__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// v * 2^e: a multiplication by an exact power of two (exact unless the result
// leaves the normal range); |e| beyond one factor's range takes two factors.
// e == 0 leaves v untouched.
__device__ __forceinline__ double scale2(double v, int e) {
  if (e == 0) return v;
  if (e >= -1022 && e <= 1023) return v * pow2(e);
  const int h = max(-1022, min(1023, e / 2));
  return v * pow2(h) * pow2(max(-1022, min(1023, e - h)));
}

// Adds contribution c >= 0 to a vertex's fixed-point counters a4[0..kAccDigits):
// floor(c * 2^kAccFrac) split into kAccDigitBits-bit digits. The double's
// fields are read directly (IEEE-754 binary64: c = m * 2^(E - 1075) with the
// 53-bit integer m = mantissa | 2^52 for a normal number); a value below
// 2^-kAccFrac contributes nothing, one too large for the counters (or not
// finite) flags kDevOverflow.
__device__ __forceinline__ void acc_add(unsigned long long *a4, double c, int *err) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(c);
  const int E = (int)(bits >> 52) & 0x7ff;
  if (bits >> 63 || E == 0x7ff) { set_err(err, kDevOverflow); return; }  // negative, inf or NaN
  if (E == 0) return;                                                  // zero or subnormal: below 2^-kAccFrac
  unsigned long long m = (bits & ((1ull << 52) - 1)) | (1ull << 52);
  int s = E - 1075 + kAccFrac;  // c * 2^kAccFrac = m * 2^s
  if (s < 0) {
    if (s <= -53) return;
    m >>= -s;
    s = 0;
  }
  if (s + 53 > kAccDigits * kAccDigitBits) { set_err(err, kDevOverflow); return; }
  constexpr unsigned long long kMask = (1ull << kAccDigitBits) - 1;
  const int di = s / kAccDigitBits, off = s % kAccDigitBits;  // m * 2^off spans digits di .. di+2
  const unsigned long long d0 = (m << off) & kMask;
  const unsigned long long d1 = (m >> (kAccDigitBits - off)) & kMask;
  const int sh2 = 2 * kAccDigitBits - off;
  const unsigned long long d2 = sh2 < 53 ? m >> sh2 : 0ull;
  if (d0) atomicAdd(a4 + di, d0);
  if (d1) atomicAdd(a4 + di + 1, d1);  // nonzero only when digit di+1 exists (s + 53 <= digits * bits)
  if (d2) atomicAdd(a4 + di + 2, d2);
}

}  // namespace bcg
