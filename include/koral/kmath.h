// kmath.h — the transcendental library shared by the CPU oracle and the
// sm_100a kernels.
//
// Why it exists: the plain-FP64 engine must reproduce the oracle bit for bit,
// and CUDA's libdevice and glibc round differently in the last place. Every
// function here is written from a published method using only IEEE
// +, -, *, /, sqrt and integer bit manipulation, so the same source compiled
// by gcc (-ffp-contract=off) and nvcc (--fmad=false) yields the same bits.
//
// Methods:
//   exp, log1p, cbrt, sin, cos, tan, atan, atanh — the fdlibm (FreeBSD msun)
//           algorithms, step for step: they are what Zig 0.16's std.math and
//           compiler-rt compute for the reference (details at their
//           definitions below).
//   log   — Tang's table-driven logarithm (ACM TOMS 16(4), 1990): m in
//           [0.75,1.5], F = j/128 nearest, log1p(f/F) Taylor series, the
//           k*ln2 + ln F head combined with Knuth's two-sum.
//   pow   — the exp(yf*log x) * x^yi by repeated squaring scheme of Go's
//           math.Pow, which is the scheme of Zig's std.math.pow that the
//           reference calls (koral/math/simd.zig:45, koral/physics/hydro.zig:36).
#pragma once
#include <stdint.h>
#include "kmath_tables.h"

#if defined(__CUDACC__)
#define KC_HD __host__ __device__ __forceinline__
#define KC_HDN __host__ __device__ __noinline__
#define KC_HDI __host__ __device__ inline  // host and device, inlining left to the compiler
// a loop kept rolled on the device (code size: the solver is instruction-fetch bound)
#define KC_ROLLED _Pragma("unroll 1")
#else
#include <string.h>
#include <math.h>
#define KC_HD inline
#define KC_HDN inline
#define KC_HDI inline
#define KC_ROLLED
#endif
// Mid-size helpers (p2u, the M1 closure, boosts, opacities' thermodynamics,
// the 4x4 inverse) are inlined.
#define KC_HDM KC_HD

namespace kmath {

#if defined(__CUDACC__)
static __device__ const double d_log_tab[194] = KM_LOG_TAB_INIT;
#endif
static const double h_log_tab[194] = KM_LOG_TAB_INIT;

KC_HD const double* log_tab() {
#if defined(__CUDA_ARCH__)
  return d_log_tab;
#else
  return h_log_tab;
#endif
}

KC_HD uint64_t to_bits(double x) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, 8);
  return u;
#endif
}
KC_HD double from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, 8);
  return x;
#endif
}

KC_HD double inf() { return from_bits(0x7ff0000000000000ULL); }
KC_HD double nan() { return from_bits(0x7ff8000000000000ULL); }
KC_HD bool isnan(double x) { return x != x; }
// |x| < inf: false for NaN and +-inf (std.math.isFinite)
KC_HD bool isfinite(double x) { return (to_bits(x) & 0x7ff0000000000000ULL) != 0x7ff0000000000000ULL; }
KC_HD bool isinf(double x) { return (to_bits(x) & 0x7fffffffffffffffULL) == 0x7ff0000000000000ULL; }
KC_HD double fabs(double x) { return from_bits(to_bits(x) & 0x7fffffffffffffffULL); }
KC_HD double copysign(double x, double s) {
  return from_bits((to_bits(x) & 0x7fffffffffffffffULL) | (to_bits(s) & 0x8000000000000000ULL));
}
// Inline: out of line (one copy of the IEEE square-root sequence per kernel)
// was measured 1% slower once the implicit kernel's warps became coherent
// (the phi-fastest cell order); KC_SQRT_ATTR=KC_HDN selects it.
#ifndef KC_SQRT_ATTR
#define KC_SQRT_ATTR KC_HD
#endif
KC_SQRT_ATTR double sqrt(double x) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(x);
#else
  return __builtin_sqrt(x);
#endif
}
// IEEE double division a / b through one out-of-line copy of the divide
// sequence. The opacity, four-force and implicit-solver code divides through
// this: their kernels are bound by instruction fetch (the solve's call graph
// is far larger than the instruction cache), and an inline double divide is
// ~30 instructions at every site. The result is the same correctly rounded
// quotient as `a / b`.
#ifndef KC_DIV_ATTR
#define KC_DIV_ATTR KC_HDN
#endif
KC_DIV_ATTR double div(double a, double b) { return a / b; }
// Zig's @min/@max on floats: the non-NaN operand wins (LLVM minnum/maxnum).
KC_HD double fmin(double a, double b) {
  if (a != a) return b;
  if (b != b) return a;
  return (b < a) ? b : a;
}
KC_HD double fmax(double a, double b) {
  if (a != a) return b;
  if (b != b) return a;
  return (b > a) ? b : a;
}
KC_HD double trunc(double x) {
#if defined(__CUDA_ARCH__)
  return ::trunc(x);
#else
  return __builtin_trunc(x);
#endif
}

// x * 2^n, exact unless the result is subnormal (then rounded once).
KC_HD double ldexp(double x, int n) {
  if (x == 0.0 || !isfinite(x)) return x;
  // bring n into range in steps that keep intermediates normal
  while (n > 1023) {
    x *= from_bits((uint64_t)(1023 + 1023) << 52);
    n -= 1023;
    if (isinf(x)) return x;
  }
  while (n < -1022) {
    // scale by 2^-969 (= 2^-1022 * 2^53) so a subnormal result rounds once
    x *= from_bits((uint64_t)(1023 - 969) << 52);
    n += 969;
    if (x == 0.0) return x;
  }
  return x * from_bits((uint64_t)(n + 1023) << 52);
}

// x = frac * 2^exp with |frac| in [0.5, 1) (Go / Zig frexp convention).
struct Frexp {
  double frac;
  int exp;
};
KC_HD Frexp frexp(double x) {
  Frexp r;
  if (x == 0.0 || !isfinite(x)) {
    r.frac = x;
    r.exp = 0;
    return r;
  }
  int e = 0;
  uint64_t b = to_bits(x);
  int be = (int)((b >> 52) & 0x7ff);
  if (be == 0) {  // subnormal: normalize
    x *= from_bits((uint64_t)(1023 + 54) << 52);
    e = -54;
    b = to_bits(x);
    be = (int)((b >> 52) & 0x7ff);
  }
  e += be - 1022;
  b = (b & 0x800fffffffffffffULL) | ((uint64_t)1022 << 52);
  r.frac = from_bits(b);
  r.exp = e;
  return r;
}

// Knuth two-sum: s + err == a + b exactly.
KC_HD void two_sum(double a, double b, double& s, double& err) {
  s = a + b;
  double bb = s - a;
  err = (a - (s - bb)) + (b - bb);
}

// ---- the fdlibm (FreeBSD msun) family -------------------------------------
// exp, log1p, cbrt, sin, cos, tan, atan and atanh below follow the fdlibm
// algorithms step for step: the same argument reductions, the same minimax
// polynomial coefficients (the published fdlibm values) and the same order of
// IEEE operations. That is what the reference's arithmetic is: Zig 0.16's
// std.math.cbrt / log1p / atan / atanh and its compiler-rt @exp / @sin / @cos
// / @tan (which the reference reaches through koral/math/simd.zig:45-84,
// koral/physics/hydro.zig:36, koral/solve/invert.zig:182 and the metric in
// koral/metric/coco.zig, forms.zig) are restatements of those fdlibm
// routines, so these give the reference's bits.

KC_HD uint32_t hi_word(double x) { return (uint32_t)(to_bits(x) >> 32); }
KC_HD double clear_lo_word(double x) { return from_bits(to_bits(x) & 0xffffffff00000000ULL); }

// exp: x = k ln2 + r with ln2 split in two (k ln2hi exact), |r| <= ln2/2;
// e^r from the Remez rational form 1 + r + r c(r) / (2 - c(r)), then 2^k.
KC_HDN double exp(double x) {
  const double ln2hi = 6.93147180369123816490e-01, ln2lo = 1.90821492927058770002e-10,
               invln2 = 1.44269504088896338700e+00;
  const double P1 = 1.66666666666666019037e-01, P2 = -2.77777777770155933842e-03,
               P3 = 6.61375632143793436117e-05, P4 = -1.65339022054652515390e-06,
               P5 = 4.13813679705723846039e-08;
  if (x != x) return x;
  uint32_t hx = hi_word(x);
  const int neg = (int)(hx >> 31);
  hx &= 0x7fffffff;
  if (hx >= 0x4086232b) {  // |x| >= 708.39
    if (x > 709.782712893383973096) return inf();
    if (x < -745.13321910194110842) return 0.0;
  }
  double hi, lo;
  int k;
  if (hx > 0x3fd62e42) {      // |x| > ln2/2
    if (hx >= 0x3ff0a2b2) {   // |x| >= 1.5 ln2
      k = (int)(invln2 * x + (neg ? -0.5 : 0.5));
    } else {
      k = neg ? -1 : 1;
    }
    hi = x - (double)k * ln2hi;
    lo = (double)k * ln2lo;
    x = hi - lo;
  } else if (hx > 0x3e300000) {  // |x| > 2^-28
    k = 0;
    hi = x;
    lo = 0.0;
  } else {
    return 1.0 + x;
  }
  const double xx = x * x;
  const double c = x - xx * (P1 + xx * (P2 + xx * (P3 + xx * (P4 + xx * P5))));
  const double y = 1.0 + (x * c / (2.0 - c) - lo + hi);
  return k == 0 ? y : ldexp(y, k);
}

// ---- log -------------------------------------------------------------------
// Tang's table-driven logarithm. Both reference scenarios that pin the Zig
// build end to end reproduce bit for bit with it (the fdlibm e_log form does
// not: it differs in the last place at some of their atmosphere radii).
KC_HD double log_core(int k, double m) {
  // m in [0.75, 1.5]
  int j = (int)(m * 128.0 + 0.5);
  double F = (double)j * 0.0078125;  // exact j/128
  double f = m - F;                   // exact
  double u = f / F;
  double u2 = u * u;
  const double c3 = 1.0 / 3.0, c5 = 1.0 / 5.0, c6 = 1.0 / 6.0, c7 = 1.0 / 7.0, c9 = 1.0 / 9.0;
  double poly = (u2 * u) * (c3 - u * (0.25 - u * (c5 - u * (c6 - u * (c7 - u * (0.125 - u * c9))))));
  double lo = poly - 0.5 * u2;
  const double* L = log_tab();
  double lhi = L[2 * (j - 96)];
  double llo = L[2 * (j - 96) + 1];
  double dk = (double)k;
  double s1, e1, s2, e2;
  two_sum(dk * KM_LN2_HI, lhi, s1, e1);
  two_sum(s1, u, s2, e2);
  return s2 + (e1 + e2 + ((dk * KM_LN2_LO + llo) + lo));
}

KC_HDN double log(double x) {
  if (x != x) return x;
  if (x < 0.0) return nan();
  if (x == 0.0) return -inf();
  if (isinf(x)) return x;
  int k = 0;
  if (x < 2.2250738585072014e-308) {
    x *= 18014398509481984.0;  // 2^54
    k = -54;
  }
  uint64_t b = to_bits(x);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  double m = from_bits((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);  // [1,2)
  if (m > 1.5) {
    m *= 0.5;
    e += 1;
  }
  return log_core(k + e, m);
}

// log1p: u = 1 + x = 2^k (1 + f) with 1 + f in [sqrt(2)/2, sqrt(2)), the
// rounding of u carried as c/u; log(1+f) = f - f^2/2 + s (f^2/2 + R(s^2)),
// s = f / (2 + f), R the fdlibm Lg1..Lg7 polynomial.
KC_HDN double log1p(double x) {
  const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
  const double Lg1 = 6.666666666666735130e-01, Lg2 = 3.999999999940941908e-01, Lg3 = 2.857142874366239149e-01,
               Lg4 = 2.222219843214978396e-01, Lg5 = 1.818357216161805012e-01, Lg6 = 1.531383769920937332e-01,
               Lg7 = 1.479819860511658591e-01;
  const uint32_t hx = hi_word(x);
  int k = 1;
  double c = 0.0, f = 0.0;
  if (hx < 0x3fda827a || (hx >> 31)) {  // 1 + x < sqrt(2)
    if (hx >= 0xbff00000) {             // x <= -1
      return x == -1.0 ? -inf() : nan();
    }
    if ((hx << 1) < (0x3ca00000u << 1)) return x;  // |x| < 2^-53
    if (hx <= 0xbfd2bec4) {                        // sqrt(2)/2 <= 1 + x
      k = 0;
      f = x;
    }
  } else if (hx >= 0x7ff00000) {
    return x;
  }
  if (k) {
    const double u = 1.0 + x;
    uint32_t hu = hi_word(u) + (0x3ff00000 - 0x3fe6a09e);
    k = (int)(hu >> 20) - 0x3ff;
    if (k < 54) {
      c = k >= 2 ? 1.0 - (u - x) : x - (u - 1.0);
      c /= u;
    }
    hu = (hu & 0x000fffff) + 0x3fe6a09e;
    f = from_bits(((uint64_t)hu << 32) | (to_bits(u) & 0xffffffffULL)) - 1.0;
  }
  const double hfsq = 0.5 * f * f;
  const double s = f / (2.0 + f);
  const double z = s * s;
  const double w = z * z;
  const double t1 = w * (Lg2 + w * (Lg4 + w * Lg6));
  const double t2 = z * (Lg1 + w * (Lg3 + w * (Lg5 + w * Lg7)));
  const double dk = (double)k;
  return s * (hfsq + (t2 + t1)) + (dk * ln2_lo + c) - hfsq + f + dk * ln2_hi;
}

// ---- cbrt ------------------------------------------------------------------
// Seed from the exponent divided by three, a polynomial step to ~23 bits,
// rounding to 22 bits (so t*t is exact), one Newton-like step in double.
KC_HDN double cbrt(double x) {
  const uint32_t B1 = 715094163, B2 = 696219795;
  const double P0 = 1.87595182427177009643, P1 = -1.88497979543377169875, P2 = 1.621429720105354466140,
               P3 = -0.758397934778766047437, P4 = 0.145996192886612446982;
  uint64_t b = to_bits(x);
  uint32_t hx = (uint32_t)(b >> 32) & 0x7fffffff;
  if (hx >= 0x7ff00000) return x + x;  // NaN, inf
  if (hx < 0x00100000) {               // zero or subnormal
    b = to_bits(x * 18014398509481984.0);  // 2^54
    hx = (uint32_t)(b >> 32) & 0x7fffffff;
    if (hx == 0) return x;
    hx = hx / 3 + B2;
  } else {
    hx = hx / 3 + B1;
  }
  double t = from_bits((b & 0x8000000000000000ULL) | ((uint64_t)hx << 32));
  double r = (t * t) * (t / x);
  t = t * ((P0 + r * (P1 + r * P2)) + ((r * r) * r) * (P3 + r * P4));
  t = from_bits((to_bits(t) + 0x80000000ULL) & 0xffffffffc0000000ULL);
  const double s = t * t;
  r = x / s;
  const double w = t + t;
  r = (r - t) / (w + r);
  return t + t * r;
}

// ---- trigonometric ---------------------------------------------------------
// Kernels on |x| <= pi/4 with the reduced argument's tail y.
KC_HD double sin_kernel(double x, double y, bool tail) {
  const double S1 = -1.66666666666666324348e-01, S2 = 8.33333333332248946124e-03,
               S3 = -1.98412698298579493134e-04, S4 = 2.75573137070700676789e-06,
               S5 = -2.50507602534068634195e-08, S6 = 1.58969099521155010221e-10;
  const double z = x * x;
  const double w = z * z;
  const double r = S2 + z * (S3 + z * S4) + z * w * (S5 + z * S6);
  const double v = z * x;
  if (!tail) return x + v * (S1 + z * r);
  return x - ((z * (0.5 * y - v * r) - y) - v * S1);
}
KC_HD double cos_kernel(double x, double y) {
  const double C1 = 4.16666666666666019037e-02, C2 = -1.38888888888741095749e-03,
               C3 = 2.48015872894767294178e-05, C4 = -2.75573143513906633035e-07,
               C5 = 2.08757232129817482790e-09, C6 = -1.13596475577881948265e-11;
  const double z = x * x;
  double w = z * z;
  const double r = z * (C1 + z * (C2 + z * C3)) + w * w * (C4 + z * (C5 + z * C6));
  const double hz = 0.5 * z;
  w = 1.0 - hz;
  return w + (((1.0 - w) - hz) + (z * r - x * y));
}
// tan(x + y) for odd == 0, -1/tan(x + y) for odd == 1
KC_HD double tan_kernel(double x, double y, int odd) {
  const double T0 = 3.33333333333334091986e-01, T1 = 1.33333333333201242699e-01,
               T2 = 5.39682539762260521377e-02, T3 = 2.18694882948595424599e-02,
               T4 = 8.86323982359930005737e-03, T5 = 3.59207910759131235356e-03,
               T6 = 1.45620945432529025516e-03, T7 = 5.88041240820264096874e-04,
               T8 = 2.46463134818469906812e-04, T9 = 7.81794442939557092300e-05,
               T10 = 7.14072491382608190305e-05, T11 = -1.85586374855275456654e-05,
               T12 = 2.59073051863633712884e-05;
  const double pio4 = 7.85398163397448278999e-01, pio4lo = 3.06161699786838301793e-17;
  const uint32_t hx = hi_word(x);
  const bool big = (hx & 0x7fffffff) >= 0x3fe59428;  // |x| >= 0.6744
  const bool neg = (hx >> 31) != 0;
  if (big) {
    if (neg) {
      x = -x;
      y = -y;
    }
    x = (pio4 - x) + (pio4lo - y);
    y = 0.0;
  }
  const double z = x * x;
  double w = z * z;
  double r = T1 + w * (T3 + w * (T5 + w * (T7 + w * (T9 + w * T11))));
  double v = z * (T2 + w * (T4 + w * (T6 + w * (T8 + w * (T10 + w * T12)))));
  double s = z * x;
  r = y + z * (s * (r + v) + y) + s * T0;
  w = x + r;
  if (big) {
    s = (double)(1 - 2 * odd);
    v = s - 2.0 * (x + (r - w * w / (w + s)));
    return neg ? -v : v;
  }
  if (!odd) return w;
  // -1/(x + r) accurately: both w and -1/w split at their low words
  const double w0 = clear_lo_word(w);
  v = r - (w0 - x);
  const double a = -1.0 / w;
  const double a0 = clear_lo_word(a);
  return a0 + a * (1.0 + a0 * w0 + a0 * v);
}

// x - n pi/2 = y0 + y1 for pi/4 < |x| < 2^20 pi/2 (Cody-Waite with pi/2 in
// 33-bit pieces, a second and third piece only when cancellation needs them).
KC_HD int rem_pio2(double x, double& y0, double& y1) {
  const double toint = 6755399441055744.0;  // 1.5 * 2^52
  const double pio4 = 7.85398163397448278999e-01, invpio2 = 6.36619772367581382433e-01;
  const double pio2_1 = 1.57079632673412561417e+00, pio2_1t = 6.07710050650619224932e-11;
  const double pio2_2 = 6.07710050630396597660e-11, pio2_2t = 2.02226624879595063154e-21;
  const double pio2_3 = 2.02226624871116645580e-21, pio2_3t = 8.47842766036889956997e-32;
  const uint64_t b = to_bits(x);
  const bool neg = (b >> 63) != 0;
  const uint32_t ix = (uint32_t)(b >> 32) & 0x7fffffff;
  // |x| <= 9pi/4 away from the multiples of pi/2 where cancellation is
  // deep: subtract n (pio2_1 + pio2_1t) directly
  int n = 0;
  if (ix <= 0x400f6a7a) {  // |x| <= 5pi/4
    if ((ix & 0xfffff) != 0x921fb) n = ix <= 0x4002d97c ? 1 : 2;
  } else if (ix <= 0x401c463b) {  // |x| <= 9pi/4
    if (ix <= 0x4015fdbc) {
      if (ix != 0x4012d97c) n = 3;
    } else if (ix != 0x401921fb) {
      n = 4;
    }
  }
  if (n != 0) {
    const double dn = (double)n;
    if (!neg) {
      const double z = x - dn * pio2_1;
      y0 = z - dn * pio2_1t;
      y1 = (z - y0) - dn * pio2_1t;
      return n;
    }
    const double z = x + dn * pio2_1;
    y0 = z + dn * pio2_1t;
    y1 = (z - y0) + dn * pio2_1t;
    return -n;
  }
  double fn = x * invpio2 + toint - toint;  // rint(x / (pi/2))
  n = (int)fn;
  double r = x - fn * pio2_1;
  double w = fn * pio2_1t;
  if (r - w < -pio4) {
    n--;
    fn--;
    r = x - fn * pio2_1;
    w = fn * pio2_1t;
  } else if (r - w > pio4) {
    n++;
    fn++;
    r = x - fn * pio2_1;
    w = fn * pio2_1t;
  }
  y0 = r - w;
  const int ex = (int)(ix >> 20);
  int ey = (int)((to_bits(y0) >> 52) & 0x7ff);
  if (ex - ey > 16) {
    double t = r;
    w = fn * pio2_2;
    r = t - w;
    w = fn * pio2_2t - ((t - r) - w);
    y0 = r - w;
    ey = (int)((to_bits(y0) >> 52) & 0x7ff);
    if (ex - ey > 49) {
      t = r;
      w = fn * pio2_3;
      r = t - w;
      w = fn * pio2_3t - ((t - r) - w);
      y0 = r - w;
    }
  }
  y1 = (r - y0) - w;
  return n;
}

KC_HDN double sin(double x) {
  const uint32_t ix = hi_word(x) & 0x7fffffff;
  if (ix <= 0x3fe921fb) {                  // |x| <= pi/4
    if (ix < 0x3e500000) return x;         // |x| < 2^-26
    return sin_kernel(x, 0.0, false);
  }
  if (ix >= 0x7ff00000) return x - x;      // NaN for inf and NaN
  double y0, y1;
  const int n = rem_pio2(x, y0, y1);
  switch (n & 3) {
    case 0: return sin_kernel(y0, y1, true);
    case 1: return cos_kernel(y0, y1);
    case 2: return -sin_kernel(y0, y1, true);
    default: return -cos_kernel(y0, y1);
  }
}
KC_HDN double cos(double x) {
  const uint32_t ix = hi_word(x) & 0x7fffffff;
  if (ix <= 0x3fe921fb) {
    if (ix < 0x3e46a09e) return 1.0;       // |x| < 2^-27 sqrt(2)
    return cos_kernel(x, 0.0);
  }
  if (ix >= 0x7ff00000) return x - x;
  double y0, y1;
  const int n = rem_pio2(x, y0, y1);
  switch (n & 3) {
    case 0: return cos_kernel(y0, y1);
    case 1: return -sin_kernel(y0, y1, true);
    case 2: return -cos_kernel(y0, y1);
    default: return sin_kernel(y0, y1, true);
  }
}
KC_HDN double tan(double x) {
  const uint32_t ix = hi_word(x) & 0x7fffffff;
  if (ix <= 0x3fe921fb) {
    if (ix < 0x3e400000) return x;         // |x| < 2^-27
    return tan_kernel(x, 0.0, 0);
  }
  if (ix >= 0x7ff00000) return x - x;
  double y0, y1;
  const int n = rem_pio2(x, y0, y1);
  return tan_kernel(y0, y1, n & 1);
}

// atan: reduce |x| to one of five intervals around 0, 0.5, 1, 1.5 and inf
// (atan of the centre as a double-double), then the odd polynomial.
KC_HDN double atan(double x) {
  const double aT0 = 3.33333333333329318027e-01, aT1 = -1.99999999998764832476e-01,
               aT2 = 1.42857142725034663711e-01, aT3 = -1.11111104054623557880e-01,
               aT4 = 9.09088713343650656196e-02, aT5 = -7.69187620504482999495e-02,
               aT6 = 6.66107313738753120669e-02, aT7 = -5.83357013379057348645e-02,
               aT8 = 4.97687799461593236017e-02, aT9 = -3.65315727442169155270e-02,
               aT10 = 1.62858201153657823623e-02;
  uint32_t ix = hi_word(x);
  const bool neg = (ix >> 31) != 0;
  ix &= 0x7fffffff;
  double hi = 0.0, lo = 0.0;
  bool centred = true;
  if (ix >= 0x44100000) {  // |x| >= 2^66
    if (x != x) return x;
    const double z = 1.57079632679489655800e+00;
    return neg ? -z : z;
  }
  if (ix < 0x3fdc0000) {                 // |x| < 0.4375
    if (ix < 0x3e400000) return x;       // |x| < 2^-27
    centred = false;
  } else {
    x = fabs(x);
    if (ix < 0x3ff30000) {               // |x| < 1.1875
      if (ix < 0x3fe60000) {             // 7/16 <= |x| < 11/16
        hi = 4.63647609000806093515e-01;
        lo = 2.26987774529616870924e-17;
        x = (2.0 * x - 1.0) / (2.0 + x);
      } else {                           // 11/16 <= |x| < 19/16
        hi = 7.85398163397448278999e-01;
        lo = 3.06161699786838301793e-17;
        x = (x - 1.0) / (x + 1.0);
      }
    } else if (ix < 0x40038000) {        // |x| < 2.4375
      hi = 9.82793723247329054082e-01;
      lo = 1.39033110312309984516e-17;
      x = (x - 1.5) / (1.0 + 1.5 * x);
    } else {                             // 2.4375 <= |x| < 2^66
      hi = 1.57079632679489655800e+00;
      lo = 6.12323399573676603587e-17;
      x = -1.0 / x;
    }
  }
  double z = x * x;
  const double w = z * z;
  const double s1 = z * (aT0 + w * (aT2 + w * (aT4 + w * (aT6 + w * (aT8 + w * aT10)))));
  const double s2 = w * (aT1 + w * (aT3 + w * (aT5 + w * (aT7 + w * aT9))));
  if (!centred) return x - x * (s1 + s2);
  z = hi - (x * (s1 + s2) - lo - x);
  return neg ? -z : z;
}

// atanh(x) = log1p(2x / (1 - x)) / 2, with the |x| < 0.5 form
// 2x + 2x^2/(1 - x) that keeps the argument's rounding small
KC_HD double atanh(double x) {
  const uint64_t b = to_bits(x);
  const unsigned e = (unsigned)((b >> 52) & 0x7ff);
  double y = from_bits(b & 0x7fffffffffffffffULL);
  if (y == 1.0) return copysign(inf(), x);
  if (e < 0x3ff - 1) {
    if (e >= 0x3ff - 32) y = 0.5 * log1p(2.0 * y + 2.0 * y * y / (1.0 - y));
  } else {
    y = 0.5 * log1p(2.0 * (y / (1.0 - y)));
  }
  return (b >> 63) ? -y : y;
}

// ---- pow: Go math.Pow / Zig std.math.pow scheme --------------------------
KC_HD bool is_odd_integer(double y) {
  if (!isfinite(y)) return false;
  double t = trunc(y);
  if (t != y) return false;
  if (fabs(y) >= 9007199254740992.0) return false;  // 2^53: all even
  double h = trunc(y * 0.5);
  return h * 2.0 != y;
}

KC_HDN double pow(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (x != x || y != y) return nan();
  if (y == 1.0) return x;
  if (x == 0.0) {
    if (y < 0.0) return is_odd_integer(y) ? copysign(inf(), x) : inf();
    return is_odd_integer(y) ? x : 0.0;
  }
  if (isinf(y)) {
    if (x == -1.0) return 1.0;
    if ((fabs(x) < 1.0) == (y > 0.0)) return 0.0;
    return inf();
  }
  if (isinf(x)) {
    if (x < 0.0) return pow(1.0 / x, -y);
    if (y < 0.0) return 0.0;
    return inf();
  }
  if (y == 0.5) return sqrt(x);
  if (y == -0.5) return 1.0 / sqrt(x);
  double ay = fabs(y);
  double yi = trunc(ay);
  double yf = ay - yi;
  if (yf != 0.0 && x < 0.0) return nan();
  if (yi >= 9223372036854775808.0) {  // 2^63
    if (x == -1.0) return 1.0;
    if ((fabs(x) < 1.0) == (y > 0.0)) return 0.0;
    return inf();
  }
  double a1 = 1.0;
  int ae = 0;
  if (yf != 0.0) {
    if (yf > 0.5) {
      yf -= 1.0;
      yi += 1.0;
    }
    a1 = exp(yf * log(x));
  }
  Frexp fr = frexp(x);
  double x1 = fr.frac;
  int xe = fr.exp;
  long long i = (long long)yi;
  while (i != 0) {
    if (xe < -4096 || 4096 < xe) {
      ae += xe;
      break;
    }
    if (i & 1) {
      a1 *= x1;
      ae += xe;
    }
    x1 *= x1;
    xe <<= 1;
    if (x1 < 0.5) {
      x1 += x1;
      xe -= 1;
    }
    i >>= 1;
  }
  if (y < 0.0) {
    a1 = 1.0 / a1;
    ae = -ae;
  }
  return ldexp(a1, ae);
}

}  // namespace kmath
