// pow(x, y) with the exact rounding sequence of the host C library's pow, for host and device code.
//
// Mycel.Core computes E_e = Emin + Math.Pow(rho, p) (E0 - Emin) (Fem/FemOperator.cs:100,133) and
// dE/drho = p Math.Pow(rho, p - 1) dE (Optimization/SensitivityAnalysis.cs:93-95). On Linux, .NET's Math.Pow
// calls the C library's pow: GNU libc 2.39 here, whose pow is the table-driven algorithm published by Arm
// (optimized-routines, 2018; libc sysdeps/ieee754/dbl-64/e_pow.c since 2.28). On x86-64 the library selects
// its FMA build at run time, in which the compiler fused every a*b + c of that source into one fma. This
// file restates that algorithm with each of those fusions written out, so host and device give the
// library's bits for every input (the GPU tests compare both on the same samples):
//
//   x = 2^k z, z in [0x1.69555p-1, 0x1.69555p0), c near z with 1/c a multiple of 2^-8:
//   log x = k ln2 + log c + log1p(z/c - 1), as a double-double hi + lo (log1p by a degree-8 polynomial);
//   x^y  = exp(y hi + y lo), exp(t) = 2^(j/128) 2^(m) exp(r) with t = (128 m + j) ln2/128 + r,
//          2^(j/128) from a 128-entry table, exp(r) - 1 by a degree-5 polynomial.
//
// The tables are built by gen_libm_pow_tables.py from the algorithm's construction rules; the polynomial
// coefficients and split constants are the algorithm's published values. Every operation rounds once:
// device code uses the _rn intrinsics (never contracted, whatever -fmad says) and host code must be compiled
// with -ffp-contract=off.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define MYCEL_POW_FN __device__ __forceinline__
#define MYCEL_POW_TABLE_QUAL static __device__ const
#else
#include <math.h>
#include <string.h>
#define MYCEL_POW_FN static inline
#define MYCEL_POW_TABLE_QUAL static const
#endif

#include "libm_pow_tables.h"

namespace mycel {
namespace libm_pow {

#if defined(__CUDACC__)
MYCEL_POW_FN double f_mul(double a, double b) { return __dmul_rn(a, b); }
MYCEL_POW_FN double f_add(double a, double b) { return __dadd_rn(a, b); }
MYCEL_POW_FN double f_sub(double a, double b) { return __dsub_rn(a, b); }
MYCEL_POW_FN double f_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
MYCEL_POW_FN double bits_d(uint64_t u) { return __longlong_as_double((long long)u); }
MYCEL_POW_FN uint64_t d_bits(double d) { return (uint64_t)__double_as_longlong(d); }
MYCEL_POW_FN double log_tab(int i, int c) { return __ldg(&kLogTab[i][c]); }
MYCEL_POW_FN uint64_t exp_tab(uint64_t i) { return __ldg((const unsigned long long*)&kExpTab[i]); }
#else
MYCEL_POW_FN double f_mul(double a, double b) { return a * b; }
MYCEL_POW_FN double f_add(double a, double b) { return a + b; }
MYCEL_POW_FN double f_sub(double a, double b) { return a - b; }
MYCEL_POW_FN double f_fma(double a, double b, double c) { return fma(a, b, c); }
MYCEL_POW_FN double bits_d(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }
MYCEL_POW_FN uint64_t d_bits(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
MYCEL_POW_FN double log_tab(int i, int c) { return kLogTab[i][c]; }
MYCEL_POW_FN uint64_t exp_tab(uint64_t i) { return kExpTab[i]; }
#endif

MYCEL_POW_FN uint32_t top12(double d) { return (uint32_t)(d_bits(d) >> 52); }

// log x = k ln2 + log c + log1p(r): ln2 split so that k*ln2_hi + logc is exact.
constexpr double kLn2Hi = 0x1.62e42fefa3800p-1;
constexpr double kLn2Lo = 0x1.ef35793c76730p-45;
constexpr uint64_t kLogOff = 0x3fe6955500000000ULL;  // bits of 0x1.69555p-1
// log1p(r) - r + r^2/2 = ar3 (B1 + B2 r + ar2 (B3 + B4 r + ar2 (B5 + B6 r))), ar = -r/2, ar2 = r ar,
// ar3 = r ar2: the degree-8 minimax coefficients, scaled for that evaluation.
constexpr double kLogB1 = 0x1.555555555556p-2 * -2;
constexpr double kLogB2 = -0x1.0000000000006p-2 * -2;
constexpr double kLogB3 = 0x1.999999959554ep-3 * 4;
constexpr double kLogB4 = -0x1.555555529a47ap-3 * 4;
constexpr double kLogB5 = 0x1.2495b9b4845e9p-3 * -8;
constexpr double kLogB6 = -0x1.0002b8b263fc3p-3 * -8;

// exp: t = (128 m + j) ln2/128 + r; ln2/128 split so that kd*hi is exact.
constexpr double kInvLn2x128 = 0x1.71547652b82fep0 * 128;
constexpr double kRoundShift = 0x1.8p52;
constexpr double kNegLn2HiOver128 = -0x1.62e42fefa0000p-8;
constexpr double kNegLn2LoOver128 = -0x1.cf79abc9e3b3ap-47;
// exp(r) - 1 - r = r^2 (E2 + E3 r) + r^4 (E4 + E5 r)
constexpr double kExpE2 = 0x1.ffffffffffdbdp-2;
constexpr double kExpE3 = 0x1.555555555543cp-3;
constexpr double kExpE4 = 0x1.55555cf172b91p-5;
constexpr double kExpE5 = 0x1.1111167a4d017p-7;
constexpr uint64_t kSignBias = 0x800ULL << 7;  // lands on the sign bit once shifted by 45

// log of the positive normal double with bits ix, as hi (returned) + *lo.
MYCEL_POW_FN double log_hi_lo(uint64_t ix, double* lo_out) {
  const uint64_t t = ix - kLogOff;
  const int i = (int)((t >> 45) & 127);
  const int64_t k = (int64_t)t >> 52;
  const double z = bits_d(ix - (t & (0xfffULL << 52)));
  const double kd = (double)k;
  const double invc = log_tab(i, 0), logc = log_tab(i, 1), logctail = log_tab(i, 2);
  const double r = f_fma(z, invc, -1.0);  // exact: 1/c has few bits and |z/c - 1| < 1/128
  const double t1 = f_fma(kd, kLn2Hi, logc);
  const double t2 = f_add(t1, r);
  const double lo1 = f_fma(kd, kLn2Lo, logctail);
  const double lo2 = f_add(f_sub(t1, t2), r);
  const double ar = f_mul(-0.5, r);
  const double ar2 = f_mul(r, ar);
  const double ar3 = f_mul(r, ar2);
  const double hi = f_add(t2, ar2);
  const double lo3 = f_fma(ar, r, -ar2);
  const double lo4 = f_add(f_sub(t2, hi), ar2);
  const double inner = f_fma(ar2, f_fma(r, kLogB6, kLogB5), f_fma(r, kLogB4, kLogB3));
  const double poly = f_fma(ar2, inner, f_fma(r, kLogB2, kLogB1));
  const double lo = f_fma(ar3, poly, f_add(f_add(f_add(lo1, lo2), lo3), lo4));
  const double y = f_add(hi, lo);
  *lo_out = f_add(f_sub(hi, y), lo);
  return y;
}

MYCEL_POW_FN double overflow_value(uint64_t sign) { return bits_d(0x7ff0000000000000ULL | (sign ? 1ULL << 63 : 0)); }
MYCEL_POW_FN double underflow_value(uint64_t sign) { return bits_d(sign ? 1ULL << 63 : 0); }

// exp(hi + lo) * (sign_bias ? -1 : 1) for the |hi| >= 512 scales that leave the normal range.
MYCEL_POW_FN double exp_scaled_edge(double tmp, uint64_t sbits, uint64_t ki) {
  if ((ki & 0x80000000ULL) == 0) {
    // positive exponent: the scale's exponent may have overflowed; take 2^1009 out first
    const double scale = bits_d(sbits - (1009ULL << 52));
    return f_mul(0x1p1009, f_fma(scale, tmp, scale));
  }
  // negative exponent: round once to the final precision before scaling into the subnormal range
  // (here the library's compiler kept scale * tmp as a separate rounded product: it feeds two sums, one of
  // them in the branch below)
  sbits += 1022ULL << 52;
  const double scale = bits_d(sbits);
  const double st = f_mul(scale, tmp);
  double y = f_add(scale, st);
  if ((y < 0.0 ? -y : y) < 1.0) {
    const double one = y < 0.0 ? -1.0 : 1.0;
    double lo = f_add(f_sub(scale, y), st);
    const double hi = f_add(one, y);
    lo = f_add(f_add(f_sub(one, hi), y), lo);
    y = f_sub(f_add(hi, lo), one);
    if (y == 0.0) y = bits_d(sbits & 0x8000000000000000ULL);
  }
  return f_mul(0x1p-1022, y);
}

// exp(x + xtail), negated when sign_bias is set.
MYCEL_POW_FN double exp_hi_lo(double x, double xtail, uint64_t sign_bias) {
  uint32_t abstop = top12(x) & 0x7ff;
  if (abstop - 0x3c9u >= 0x408u - 0x3c9u) {  // |x| < 2^-54 or |x| >= 512
    if (abstop - 0x3c9u >= 0x80000000u) {
      const double one = f_add(1.0, x);
      return sign_bias ? -one : one;
    }
    if (abstop >= 0x409u) return (d_bits(x) >> 63) ? underflow_value(sign_bias) : overflow_value(sign_bias);
    abstop = 0;  // large |x|: handled after the common part
  }
  double kd = f_fma(kInvLn2x128, x, kRoundShift);
  const uint64_t ki = d_bits(kd);
  kd = f_sub(kd, kRoundShift);
  double r = f_fma(kd, kNegLn2LoOver128, f_fma(kd, kNegLn2HiOver128, x));
  r = f_add(r, xtail);
  const uint64_t idx = 2 * (ki % 128);
  const uint64_t top = (ki + sign_bias) << 45;
  const double tail = bits_d(exp_tab(idx));
  const uint64_t sbits = exp_tab(idx + 1) + top;
  const double r2 = f_mul(r, r);
  const double tmp = f_fma(f_mul(r2, r2), f_fma(r, kExpE5, kExpE4), f_fma(r2, f_fma(r, kExpE3, kExpE2), f_add(tail, r)));
  if (abstop == 0) return exp_scaled_edge(tmp, sbits, ki);
  const double scale = bits_d(sbits);
  return f_fma(scale, tmp, scale);
}

// 0 if y (bits iy, non-zero finite) is not an integer, 1 if odd, 2 if even.
MYCEL_POW_FN int int_kind(uint64_t iy) {
  const int e = (int)((iy >> 52) & 0x7ff);
  if (e < 0x3ff) return 0;
  if (e > 0x3ff + 52) return 2;
  if (iy & ((1ULL << (0x3ff + 52 - e)) - 1)) return 0;
  if (iy & (1ULL << (0x3ff + 52 - e))) return 1;
  return 2;
}

MYCEL_POW_FN bool zero_inf_nan(uint64_t i) { return 2 * i - 1 >= 2 * 0x7ff0000000000000ULL - 1; }

MYCEL_POW_FN double pow(double x, double y) {
  uint64_t sign_bias = 0;
  uint64_t ix = d_bits(x);
  const uint64_t iy = d_bits(y);
  uint32_t topx = top12(x);
  const uint32_t topy = top12(y);
  if (topx - 0x001u >= 0x7ffu - 0x001u || (topy & 0x7ffu) - 0x3beu >= 0x43eu - 0x3beu) {
    // x zero, subnormal, negative, inf or nan; or |y| < 2^-65, |y| >= 2^63, inf or nan
    if (zero_inf_nan(iy)) {
      if (2 * iy == 0) return 1.0;
      if (ix == 0x3ff0000000000000ULL) return 1.0;
      if (2 * ix > 2 * 0x7ff0000000000000ULL || 2 * iy > 2 * 0x7ff0000000000000ULL) return f_add(x, y);
      if (2 * ix == 2 * 0x3ff0000000000000ULL) return 1.0;
      if ((2 * ix < 2 * 0x3ff0000000000000ULL) == !(iy >> 63)) return 0.0;
      return f_mul(y, y);
    }
    if (zero_inf_nan(ix)) {
      double x2 = f_mul(x, x);
      if ((ix >> 63) && int_kind(iy) == 1) x2 = -x2;
      return (iy >> 63) ? 1.0 / x2 : x2;
    }
    if (ix >> 63) {  // finite x < 0
      const int kind = int_kind(iy);
      if (kind == 0) return bits_d(0x7ff8000000000000ULL);  // invalid: a quiet NaN
      if (kind == 1) sign_bias = kSignBias;
      ix &= 0x7fffffffffffffffULL;
      topx &= 0x7ff;
    }
    if ((topy & 0x7ffu) - 0x3beu >= 0x43eu - 0x3beu) {
      if (ix == 0x3ff0000000000000ULL) return 1.0;
      if ((topy & 0x7ffu) < 0x3beu) return ix > 0x3ff0000000000000ULL ? f_add(1.0, y) : f_sub(1.0, y);
      return (ix > 0x3ff0000000000000ULL) == (topy < 0x800u) ? overflow_value(0) : underflow_value(0);
    }
    if (topx == 0) {  // subnormal x: normalise so the exponent goes negative
      ix = d_bits(f_mul(x, 0x1p52));
      ix &= 0x7fffffffffffffffULL;
      ix -= 52ULL << 52;
    }
  }
  double lo;
  const double hi = log_hi_lo(ix, &lo);
  const double ehi = f_mul(y, hi);
  const double elo = f_fma(y, lo, f_fma(y, hi, -ehi));
  return exp_hi_lo(ehi, elo, sign_bias);
}

}  // namespace libm_pow
}  // namespace mycel
