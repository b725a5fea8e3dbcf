/* Ozaki scheme-1 digit rules shared by the dense GEMM and the stack form (device code).
   IEEE-754 split and 7-bit digits of the max-exponent-aligned significand
   (samples/ozaki/kernels/ozaki_common.cl:789-834): digit s (0..6) holds bits [46-7s, 52-7s] of the
   aligned significand, digit 7 holds bits [0,3] and is stored multiplied by 8, so digit s always
   weighs 2^(46-7s) and a value is sum_s digit_s * 2^(46-7s) * 2^(emax-1075). */
#pragma once

#include <stdint.h>

namespace xs_oz {

/* IEEE-754 split: sign, biased exponent, significand with the implicit bit; zero, subnormal, Inf
   and NaN give exponent 0 and significand 0 (ozaki_common.cl:789-806). */
__device__ __forceinline__ void ieee_split(double v, unsigned& sign, int& bexp, unsigned long long& mant) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
  sign = (unsigned)(bits >> 63);
  bexp = (int)((bits >> 52) & 2047u);
  mant = (bits & 0x000FFFFFFFFFFFFFull) | 0x0010000000000000ull;
  if (0 == bexp || 2047 == bexp) {
    bexp = 0;
    mant = 0;
  }
}

__device__ __forceinline__ int biased_exp(double v) {
  const int e = (int)(((unsigned long long)__double_as_longlong(v) >> 52) & 2047u);
  return (2047 == e) ? 0 : e;
}

/* Digit s (0..7) of an aligned significand, signed; digit 7 carries bits [0,3] times 8. */
__device__ __forceinline__ int slice_digit(unsigned long long aligned, unsigned sign, int s) {
  const int d = (s < 7) ? (int)((aligned >> (46 - 7 * s)) & 127u) : (int)((aligned & 15u) << 3);
  return sign ? -d : d;
}

}  // namespace xs_oz
