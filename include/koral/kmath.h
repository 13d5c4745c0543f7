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
//   exp   — Tang's table-driven method (ACM TOMS 15(2), 1989): x = (64k+j)
//           ln2/64 + r, 2^(j/64) from a double-double table, degree-6 Taylor
//           polynomial for e^r - 1 on |r| <= ln2/128.
//   log   — Tang's table-driven logarithm (ACM TOMS 16(4), 1990): m in
//           [0.75,1.5], F = j/128 nearest, log1p(f/F) Taylor series, the
//           k*ln2 + ln F head combined with Knuth's two-sum.
//   log1p — Taylor series for |x| <= 2^-8, else Goldberg's correction
//           log(1+x) = log(u) + (x-(u-1))/u with u = fl(1+x).
//   cbrt  — bit-level seed, Newton iterations, final residual step with
//           Dekker's exact product (Veltkamp splitting).
//   sin/cos/tan — Cody–Waite reduction by pi/2 (three-part constant), Taylor
//           polynomials on |r| <= pi/4.
//   atan  — reduction to |t| <= tan(pi/12) via atan(1/x) and the pi/6
//           addition formula, Taylor series.
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
// the 4x4 inverse): inlined unless KC_SHARED_HELPERS is 1, which compiles
// them as calls and so shrinks the code of the large solver kernels. Either
// way the arithmetic is the same (no contraction), so results are identical.
#if defined(KC_SHARED_HELPERS) && KC_SHARED_HELPERS
#define KC_HDM KC_HDN
#else
#define KC_HDM KC_HD
#endif

namespace kmath {

#if defined(__CUDACC__)
static __device__ const double d_exp_tab[128] = KM_EXP_TAB_INIT;
static __device__ const double d_log_tab[194] = KM_LOG_TAB_INIT;
#endif
static const double h_exp_tab[128] = KM_EXP_TAB_INIT;
static const double h_log_tab[194] = KM_LOG_TAB_INIT;

KC_HD const double* exp_tab() {
#if defined(__CUDA_ARCH__)
  return d_exp_tab;
#else
  return h_exp_tab;
#endif
}
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
// round-half-up to an integer-valued double, exact for |x| < 2^51
KC_HD double rint_half_up(double x) {
#if defined(__CUDA_ARCH__)
  return ::floor(x + 0.5);
#else
  return __builtin_floor(x + 0.5);
#endif
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

// Veltkamp split and Dekker product: p + err == a * b exactly (no FMA).
KC_HD void split(double a, double& hi, double& lo) {
  double c = 134217729.0 * a;  // 2^27 + 1
  double ab = c - a;
  hi = c - ab;
  lo = a - hi;
}
KC_HD void two_prod(double a, double b, double& p, double& err) {
  p = a * b;
  double ah, al, bh, bl;
  split(a, ah, al);
  split(b, bh, bl);
  err = ((ah * bh - p) + ah * bl + al * bh) + al * bl;
}

// ---- exp -------------------------------------------------------------------
KC_HDN double exp(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return inf();
  if (x < -745.1332191019412) return 0.0;
  double n = rint_half_up(x * KM_INV_L64);
  int N = (int)n;
  double r = (x - n * KM_L64_HI) - n * KM_L64_LO;
  int j = N & 63;
  int k = (N - j) / 64;
  const double* T = exp_tab();
  double thi = T[2 * j];
  double tlo = T[2 * j + 1];
  const double c6 = 1.0 / 720.0, c5 = 1.0 / 120.0, c4 = 1.0 / 24.0, c3 = 1.0 / 6.0;
  double p = r + (r * r) * (0.5 + r * (c3 + r * (c4 + r * (c5 + r * c6))));
  double y = thi + (tlo + thi * p);
  return ldexp(y, k);
}

// ---- log -------------------------------------------------------------------
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

KC_HDN double log1p(double x) {
  if (x != x) return x;
  if (x < -1.0) return nan();
  if (x == -1.0) return -inf();
  if (isinf(x)) return x;
  double ax = fabs(x);
  if (ax < 5.551115123125783e-17) return x;  // 2^-54: log1p(x) rounds to x
  if (ax <= 0.00390625) {
    double u = x;
    double u2 = u * u;
    const double c3 = 1.0 / 3.0, c5 = 1.0 / 5.0, c6 = 1.0 / 6.0, c7 = 1.0 / 7.0, c9 = 1.0 / 9.0;
    double poly = (u2 * u) * (c3 - u * (0.25 - u * (c5 - u * (c6 - u * (c7 - u * (0.125 - u * c9))))));
    return u + (poly - 0.5 * u2);
  }
  double u = 1.0 + x;
  double c = (x - (u - 1.0)) / u;
  return log(u) + c;
}

// ---- cbrt ------------------------------------------------------------------
KC_HDN double cbrt(double x) {
  if (x == 0.0 || !isfinite(x)) return x;
  double a = fabs(x);
  int k = 0;
  if (a < 2.2250738585072014e-308) {
    a *= 18014398509481984.0;  // 2^54
    k = -18;                    // cube root of 2^-54
  }
  // seed: divide the biased exponent by three
  uint64_t b = to_bits(a);
  uint64_t hb = (b >> 32);
  hb = hb / 3 + 715094163;  // 0x2a9f7893
  double t = from_bits(hb << 32);
  for (int it = 0; it < 5; ++it) t = t - (t * t * t - a) / (3.0 * t * t);
  // final residual step: r = t^3 - a computed exactly to double-double
  double p, pe, q, qe;
  two_prod(t, t, p, pe);
  two_prod(p, t, q, qe);
  double r = (q - a) + (qe + pe * t);
  t = t - r / (3.0 * t * t);
  if (k != 0) t = ldexp(t, k);
  return (x < 0.0) ? -t : t;
}

// ---- trigonometric ---------------------------------------------------------
// The reduced argument is carried as a double-double r = rh + rl and the
// leading polynomial terms are formed exactly (two_prod), so sin/cos come out
// within ~0.55 ulp and tan (a double-double quotient) within ~0.6 ulp.
struct Reduced {
  double rh, rl;
  int q;
};
KC_HD Reduced reduce_pio2(double x) {
  Reduced o;
  if (fabs(x) <= 0.7853981633974483) {
    o.rh = x;
    o.rl = 0.0;
    o.q = 0;
    return o;
  }
  double n = rint_half_up(x * KM_2OPI);
  double t = x - n * KM_PIO2_1;  // exact (Sterbenz; n*P1 exact)
  double s, e;
  two_sum(t, -(n * KM_PIO2_2), s, e);
  double lo = e - n * KM_PIO2_3;
  two_sum(s, lo, o.rh, o.rl);
  o.q = ((int)n) & 3;
  return o;
}
// sin(rh + rl) as a double-double (hi, lo)
KC_HD void sin_dd(double rh, double rl, double& hi, double& lo) {
  double w = rh * rh;
  const double s3 = -1.0 / 6.0, s5 = 1.0 / 120.0, s7 = -1.0 / 5040.0, s9 = 1.0 / 362880.0,
               s11 = -1.0 / 39916800.0, s13 = 1.0 / 6227020800.0, s15 = -1.0 / 1307674368000.0,
               s17 = 1.0 / 355687428096000.0;
  double p = s3 + w * (s5 + w * (s7 + w * (s9 + w * (s11 + w * (s13 + w * (s15 + w * s17))))));
  // sin(rh+rl) = sin(rh) + rl*cos(rh) ~ rh + rh*w*p + rl*(1 - w/2)
  double tail = (rh * w) * p + rl * (1.0 - 0.5 * w);
  two_sum(rh, tail, hi, lo);
}
// cos(rh + rl) as a double-double (hi, lo)
KC_HD void cos_dd(double rh, double rl, double& hi, double& lo) {
  double wh, wl;
  two_prod(rh, rh, wh, wl);
  double w = wh;
  const double c4 = 1.0 / 24.0, c6 = -1.0 / 720.0, c8 = 1.0 / 40320.0, c10 = -1.0 / 3628800.0,
               c12 = 1.0 / 479001600.0, c14 = -1.0 / 87178291200.0, c16 = 1.0 / 20922789888000.0,
               c18 = -1.0 / 6402373705728000.0;
  double p = c4 + w * (c6 + w * (c8 + w * (c10 + w * (c12 + w * (c14 + w * (c16 + w * c18))))));
  double hz = 0.5 * wh;  // exact
  double a = 1.0 - hz;
  double corr = ((1.0 - a) - hz) - 0.5 * wl - rh * rl;
  double tail = corr + (w * w) * p;
  two_sum(a, tail, hi, lo);
}
KC_HDN double sin(double x) {
  if (!isfinite(x)) return nan();
  Reduced rd = reduce_pio2(x);
  double h, l;
  if (rd.q & 1) cos_dd(rd.rh, rd.rl, h, l);
  else sin_dd(rd.rh, rd.rl, h, l);
  double v = h + l;
  return (rd.q & 2) ? -v : v;
}
KC_HDN double cos(double x) {
  if (!isfinite(x)) return nan();
  Reduced rd = reduce_pio2(x);
  double h, l;
  if (rd.q & 1) sin_dd(rd.rh, rd.rl, h, l);
  else cos_dd(rd.rh, rd.rl, h, l);
  double v = h + l;
  return (((rd.q + 1) & 2) != 0) ? -v : v;
}
KC_HDN double tan(double x) {
  if (!isfinite(x)) return nan();
  Reduced rd = reduce_pio2(x);
  double sh, sl, ch, cl;
  sin_dd(rd.rh, rd.rl, sh, sl);
  cos_dd(rd.rh, rd.rl, ch, cl);
  double nh = sh, nl = sl, dh = ch, dl = cl;
  if (rd.q & 1) {  // tan = -cos/sin
    nh = -ch;
    nl = -cl;
    dh = sh;
    dl = sl;
  }
  double q0 = nh / dh;
  double p, pe;
  two_prod(q0, dh, p, pe);
  double r = (((nh - p) - pe) + nl) - q0 * dl;
  return q0 + r / dh;
}

KC_HDN double atan(double x) {
  if (x != x) return x;
  bool neg = x < 0.0;
  double a = fabs(x);
  if (isinf(a)) return neg ? -KM_PIO2_HI : KM_PIO2_HI;
  bool inv = a > 1.0;
  if (inv) a = 1.0 / a;
  double off_hi = 0.0, off_lo = 0.0, t = a;
  if (a > KM_TAN_PIO12) {
    t = (a * KM_SQRT3 - 1.0) / (a + KM_SQRT3);
    off_hi = KM_PIO6_HI;
    off_lo = KM_PIO6_LO;
  }
  double w = t * t;
  double p = 0.0;
  for (int n = 14; n >= 1; --n) {
    double c = ((n & 1) ? -1.0 : 1.0) / (double)(2 * n + 1);
    p = c + w * p;
  }
  double tail = (t * w) * p;
  double res = off_hi + (t + (off_lo + tail));
  if (inv) res = KM_PIO2_HI + (KM_PIO2_LO - res);
  return neg ? -res : res;
}

KC_HD double atanh(double x) {
  // 0.5 * log1p(2x / (1 - x)), defined for |x| < 1
  return 0.5 * log1p((x + x) / (1.0 - x));
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
