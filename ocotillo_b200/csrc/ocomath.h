/*
 * ocomath.h -- bit-reproducible double-precision exp, log, log10 and pow for host C/C++
 * and CUDA device code.
 *
 * Why: the reference evaluates its physics with the C library's exp/log/log10/pow
 * (gfortran calls glibc), and its tridiagonal solve amplifies a 1-ulp change in an
 * opacity by up to ~1e5 in the mean intensity.  A GPU and a CPU that disagree by one ulp
 * in a single exp therefore disagree visibly in the output.  This header gives the GPU
 * kernels and the CPU oracle the SAME function, built only from IEEE-754 basic operations
 * (+, -, *, /) and explicit fused multiply-adds, so the two produce identical bits.
 *
 * Method (published algorithms, written from their descriptions):
 *   exp: fast phase (Ziv): reduction by ln2/1024 with a 1024-entry table, accurate to
 *        2^-73 with a rounding test; when the test cannot decide (probability ~4e-6),
 *        table-driven reduction x = (128k + j) ln2/128 + r, |r| <= ln2/256
 *        (Tang, ACM TOMS 15(2) 1989), with a three-part Cody-Waite split of ln2/128,
 *        2^(j/128) stored as a double-double, and e^r - 1 evaluated in double-double up
 *        to r^2 and by FMA Horner to r^7.  Pre-rounding relative error < 2^-75.
 *   log: x = 2^e m, m in [0.75, 1.5), F = 1 + j/128 nearest to m, f = m - F exact,
 *        log x = e ln2 + log F + log1p(f/F) (Tang, ACM TOMS 16(4) 1990), with 1/F and
 *        log F as double-doubles and log1p by a degree-11 series whose first two terms
 *        are double-double (the rest by FMA Horner).  Pre-rounding relative error < 2^-78.
 *   pow: exp(y log|x|) with log|x| carried as a double-double; x == 10 uses a
 *        double-double ln10.  C99 Annex F special cases.
 * The results are correctly rounded except in rare hard cases (the exact value within
 * ~2^-75 relative of a rounding boundary).  Error-free transforms (TwoSum, Fast2Sum,
 * TwoProduct via FMA) follow Muller et al., "Handbook of Floating-Point Arithmetic",
 * 2nd ed., ch. 4-5.
 *
 * Build rules: host code must be compiled without FMA contraction (-ffp-contract=off);
 * device code uses __dmul_rn/__dadd_rn, which the compiler never contracts, so the
 * device result does not depend on -fmad.
 */
#ifndef OCOMATH_H
#define OCOMATH_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#ifdef __CUDACC__
#define OCO_HD static __host__ __device__ __forceinline__
#else
#define OCO_HD static inline
#endif

/* Host copy of the tables. */
#define OCO_MATH_TABLE(name, n) static const double name##_h[n]
#include "ocomath_tables.h"
#undef OCO_MATH_TABLE
/* Device copy of the tables. */
#ifdef __CUDACC__
#define OCO_MATH_TABLE(name, n) static __device__ const double name##_d[n]
#include "ocomath_tables.h"
#undef OCO_MATH_TABLE
#endif

#ifdef __CUDA_ARCH__
#define OCO_TAB(name, i) __ldg(&name##_d[(i)])
#define OCO_M(a, b) __dmul_rn((a), (b))
#define OCO_A(a, b) __dadd_rn((a), (b))
#define OCO_S(a, b) __dsub_rn((a), (b))
#define OCO_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define OCO_TAB(name, i) (name##_h[(i)])
#define OCO_M(a, b) ((a) * (b))
#define OCO_A(a, b) ((a) + (b))
#define OCO_S(a, b) ((a) - (b))
#define OCO_FMA(a, b, c) fma((a), (b), (c))
#endif

OCO_HD uint64_t oco_d2u(double x) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  return u;
#endif
}

OCO_HD double oco_u2d(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double x;
  memcpy(&x, &u, sizeof x);
  return x;
#endif
}

OCO_HD int oco_isnan(double x) { return x != x; }
OCO_HD int oco_isinf(double x) { return (oco_d2u(x) & 0x7fffffffffffffffULL) == 0x7ff0000000000000ULL; }
OCO_HD double oco_inf(void) { return oco_u2d(0x7ff0000000000000ULL); }
OCO_HD double oco_nan(void) { return oco_u2d(0x7ff8000000000000ULL); }

/* 2^k for -1022 <= k <= 1023, built from the exponent bits. */
OCO_HD double oco_pow2i(int k) { return oco_u2d((uint64_t)(int64_t)(k + 1023) << 52); }

/* Fast phase of e^(xh + xl) (Ziv's strategy): table of 2^(j/1024); the reduced argument
 * r = xh - k ln2/1024 (|r| <= 2^-11.5) as rh + rl from a three-part Cody-Waite split (head
 * exact, rl the exact residual of rh up to 2^-128); e^r - 1 = rh + ql with
 * ql = rl + rh^2 (1/2 + rh/6 + rh^2/24 + rh^3/120); xl (|xl| <= 2^-44) enters as the factor
 * 1 + xl, i.e. ql += xl (1 + rh + ql); the result T (1 + q) as hi + lo.  Error of hi + lo
 * relative to the result below 2^-73.4 (r^6/720 < 2^-78.3; rounding of rh^2 < 2^-77; 2 rh rl
 * omitted < 2^-76.6; Tl ql omitted < 2^-76; roundings of ql and P < 2^-77, 2^-78).  Returns 1
 * and the correctly rounded value in *res when the remainder of hi + lo after rounding to
 * nearest stays more than 2^(e-71) (result in [2^e, 2^(e+1))) inside half an ulp, so that
 * no value within the error bound rounds differently; returns 0 otherwise (the
 * double-double phase below then decides).  Normal results only. */
OCO_HD int oco_exp_fast(double xh, double xl, double *res) {
  const double shift = 0x1.8p52;
  const double ks = OCO_FMA(xh, OCO_EXPF_INVLN2N, shift);
  const double kd = OCO_S(ks, shift);
  const int ki = (int)(uint32_t)oco_d2u(ks);
  const int j = ki & (OCO_EXPF_N - 1);
  const int k = ki >> 10; /* floor(ki / 1024) */
  if (k <= -1021 || k >= 1023) return 0;
  const double d = OCO_FMA(-kd, OCO_EXPF_L1, xh); /* exact: k L1 has <= 53 bits, Sterbenz */
  const double rh = OCO_FMA(-kd, OCO_EXPF_L2, d);
  double rl = OCO_FMA(-kd, OCO_EXPF_L2, OCO_S(d, rh)); /* d - k L2 - rh, one rounding */
  rl = OCO_FMA(-kd, OCO_EXPF_L3, rl);
  const double s = OCO_M(rh, rh);
  double P = OCO_FMA(rh, OCO_EXP_C5, OCO_EXP_C4);
  P = OCO_FMA(rh, P, OCO_EXP_C3);
  P = OCO_FMA(rh, P, 0.5);
  double ql = OCO_FMA(s, P, rl);
  ql = OCO_A(ql, OCO_FMA(xl, OCO_A(rh, ql), xl)); /* (1 + q)(1 + xl) - 1 - rh */
  const double Th = OCO_TAB(oco_expf_tab, 2 * j), Tl = OCO_TAB(oco_expf_tab, 2 * j + 1);
  const double m = OCO_M(Th, rh);
  const double me = OCO_FMA(Th, rh, -m);
  const double hh = OCO_A(Th, m); /* Fast2Sum, |Th| >= 1 > |m| */
  const double e2 = OCO_S(m, OCO_S(hh, Th));
  const double lo = OCO_A(e2, OCO_A(me, OCO_FMA(Th, ql, OCO_FMA(Tl, rh, Tl))));
  const double v = OCO_A(hh, lo);
  const double t = OCO_S(lo, OCO_S(v, hh)); /* exact: v + t = hh + lo */
  const uint64_t vb = oco_d2u(v);
  const int ve = (int)(vb >> 52); /* v in (0.99, 2.01): positive, normal */
  double half = oco_u2d((uint64_t)(ve - 53) << 52);
  if ((vb & 0x000fffffffffffffULL) == 0 && t < 0.0) half = OCO_M(half, 0.5); /* power of two: finer grid below */
  const double bound = OCO_S(half, oco_u2d((uint64_t)(ve - 71) << 52));
  if (!(fabs(t) < bound)) return 0;
  *res = OCO_M(v, oco_pow2i(k));
  return 1;
}

/* The fast phase above without branches: the same operations on every input (the table
 * index is always in range; an out-of-range k or a non-finite input only makes *res
 * meaningless), and 1 exactly when oco_exp_fast would return 1 with the same *res.  Several
 * of these can be interleaved by the compiler; a caller falls back to oco_exp_dd on 0, which
 * makes the pair identical to oco_exp_dd for every input. */
OCO_HD int oco_exp_fast_nb(double xh, double xl, double *res) {
  const double shift = 0x1.8p52;
  const double ks = OCO_FMA(xh, OCO_EXPF_INVLN2N, shift);
  const double kd = OCO_S(ks, shift);
  const int ki = (int)(uint32_t)oco_d2u(ks);
  const int j = ki & (OCO_EXPF_N - 1);
  const int k = ki >> 10;
  const int kok = (k > -1021) & (k < 1023);
  const double d = OCO_FMA(-kd, OCO_EXPF_L1, xh);
  const double rh = OCO_FMA(-kd, OCO_EXPF_L2, d);
  double rl = OCO_FMA(-kd, OCO_EXPF_L2, OCO_S(d, rh));
  rl = OCO_FMA(-kd, OCO_EXPF_L3, rl);
  const double s = OCO_M(rh, rh);
  double P = OCO_FMA(rh, OCO_EXP_C5, OCO_EXP_C4);
  P = OCO_FMA(rh, P, OCO_EXP_C3);
  P = OCO_FMA(rh, P, 0.5);
  double ql = OCO_FMA(s, P, rl);
  ql = OCO_A(ql, OCO_FMA(xl, OCO_A(rh, ql), xl));
  const double Th = OCO_TAB(oco_expf_tab, 2 * j), Tl = OCO_TAB(oco_expf_tab, 2 * j + 1);
  const double m = OCO_M(Th, rh);
  const double me = OCO_FMA(Th, rh, -m);
  const double hh = OCO_A(Th, m);
  const double e2 = OCO_S(m, OCO_S(hh, Th));
  const double lo = OCO_A(e2, OCO_A(me, OCO_FMA(Th, ql, OCO_FMA(Tl, rh, Tl))));
  const double v = OCO_A(hh, lo);
  const double t = OCO_S(lo, OCO_S(v, hh));
  const uint64_t vb = oco_d2u(v);
  const int ve = (int)(vb >> 52) & 0x7ff;
  double half = oco_u2d((uint64_t)(ve - 53) << 52);
  half = ((vb & 0x000fffffffffffffULL) == 0 && t < 0.0) ? OCO_M(half, 0.5) : half;
  const double bound = OCO_S(half, oco_u2d((uint64_t)(ve - 71) << 52));
  *res = OCO_M(v, oco_pow2i(kok ? k : 0));
  return kok & (fabs(t) < bound) & (ve >= 0x3fe) & (ve <= 0x400);
}

/* e^(xh + xl) for a double-double argument with |xl| <= ulp(xh). */
OCO_HD double oco_exp_dd(double xh, double xl) {
  if (oco_isnan(xh)) return OCO_A(xh, xh);
  if (xh > 709.8) return oco_inf();
  if (xh < -746.0) return 0.0;
  double fast;
  if (oco_exp_fast(xh, xl, &fast)) return fast;
  /* kd = nearest integer to x * 128/ln2; its value also sits in the low bits of the
   * shifted sum (|kd| < 2^18), which gives j and k without a conversion. */
  const double shift = 0x1.8p52;
  double ks = OCO_A(OCO_M(xh, OCO_EXP_INVLN2N), shift);
  double kd = OCO_S(ks, shift);
  int ki = (int)(uint32_t)oco_d2u(ks);
  int j = ki & (OCO_EXP_N - 1);
  int k = ki >> 7; /* floor(ki / 128) */
  /* r = x - kd ln2/128 as a double-double.  kd*L1 is exact (35 + 18 bits) and the
   * subtraction is exact by Sterbenz's lemma. */
  double d = OCO_S(xh, OCO_M(kd, OCO_EXP_L1));
  double p2 = OCO_M(kd, OCO_EXP_L2);
  double p2e = OCO_FMA(kd, OCO_EXP_L2, -p2);
  double rh = OCO_S(d, p2); /* TwoSum(d, -p2) */
  double bb = OCO_S(rh, d);
  double t = OCO_A(OCO_S(d, OCO_S(rh, bb)), OCO_S(-p2, bb));
  double rl = OCO_A(OCO_S(OCO_S(t, p2e), OCO_M(kd, OCO_EXP_L3)), xl);
  double r0 = OCO_A(rh, rl); /* TwoSum renormalisation (needed when xl is not 0) */
  bb = OCO_S(r0, rh);
  rl = OCO_A(OCO_S(rh, OCO_S(r0, bb)), OCO_S(rl, bb));
  rh = r0;
  /* e^r - 1 = r + r^2/2 + r^3 (1/6 + r/24 + ...), |r| < 2^-8.5. */
  double s = OCO_M(rh, rh);
  double se = OCO_FMA(rh, rh, -s);
  double half = OCO_M(0.5, s);
  double halfe = OCO_A(OCO_M(0.5, se), OCO_M(rh, rl));
  double P = OCO_FMA(rh, OCO_EXP_C7, OCO_EXP_C6);
  P = OCO_FMA(rh, P, OCO_EXP_C5);
  P = OCO_FMA(rh, P, OCO_EXP_C4);
  P = OCO_FMA(rh, P, OCO_EXP_C3);
  P = OCO_M(OCO_M(s, rh), P);
  double qh = OCO_A(rh, half); /* Fast2Sum, |rh| >= |half| */
  double ql = OCO_A(OCO_S(half, OCO_S(qh, rh)), OCO_A(rl, OCO_A(halfe, P)));
  /* 2^(j/128) (1 + q) as a double-double (h, lo). */
  double Th = OCO_TAB(oco_exp_tab, 2 * j);
  double Tl = OCO_TAB(oco_exp_tab, 2 * j + 1);
  double m = OCO_M(Th, qh);
  double me = OCO_FMA(Th, qh, -m);
  double h = OCO_A(Th, m); /* Fast2Sum, |Th| >= 1 > |m| */
  double e2 = OCO_S(m, OCO_S(h, Th));
  double lo = OCO_A(e2, OCO_A(me, OCO_A(Tl, OCO_A(OCO_M(Th, ql), OCO_M(Tl, qh)))));
  if (k > -1022) {
    double v = OCO_A(h, lo);
    if (k < 1023) return OCO_M(v, oco_pow2i(k));
    return OCO_M(OCO_M(v, oco_pow2i(k - 1)), 2.0);
  }
  /* Result at or below 2^-1022: round once on the subnormal grid by adding 1 in units of
   * 2^-1022 (so that the ulp of the sum is the subnormal ulp), then remove it exactly. */
  double sc = oco_pow2i(k + 1022);
  double b = OCO_M(h, sc);
  double bl = OCO_M(lo, sc);
  if (b >= 1.0) return OCO_M(OCO_A(h, lo), 0x1p-1022);
  double tt = OCO_A(1.0, b);
  double te = OCO_A(OCO_S(1.0, tt), b);
  double sum = OCO_A(tt, OCO_A(te, bl));
  return OCO_M(OCO_S(sum, 1.0), 0x1p-1022);
}

/* log(x) as a double-double for finite x > 0. */
OCO_HD void oco_log_dd(double x, double *lh, double *ll) {
  uint64_t u = oco_d2u(x);
  int e = 0;
  if (u < 0x0010000000000000ULL) { /* subnormal */
    x = OCO_M(x, 0x1p54);
    u = oco_d2u(x);
    e = -54;
  }
  e += (int)(u >> 52) - 1023;
  double m = oco_u2d((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m >= 1.5) {
    m = OCO_M(m, 0.5);
    e += 1;
  }
  const double shift = 0x1.8p52;
  double jd = OCO_S(OCO_A(OCO_M(OCO_S(m, 1.0), (double)OCO_LOG_N), shift), shift);
  int j = (int)jd;
  double F = OCO_A(1.0, OCO_M(jd, 1.0 / OCO_LOG_N));
  double f = OCO_S(m, F); /* exact */
  int idx = 2 * (j - OCO_LOG_JMIN);
  double ih = OCO_TAB(oco_invF_tab, idx), il = OCO_TAB(oco_invF_tab, idx + 1);
  double uh = OCO_M(f, ih);
  double ue = OCO_FMA(f, ih, -uh);
  double ul = OCO_A(ue, OCO_M(f, il));
  double u0 = OCO_A(uh, ul); /* Fast2Sum */
  ul = OCO_S(ul, OCO_S(u0, uh));
  uh = u0;
  /* log1p(u) = u - u^2/2 + u^3 (1/3 - u/4 + ... - u^8/11), |u| < 2^-7.5. */
  double s = OCO_M(uh, uh);
  double se = OCO_FMA(uh, uh, -s);
  double half = OCO_M(0.5, s);
  double halfe = OCO_A(OCO_M(0.5, se), OCO_M(uh, ul));
  double P = OCO_FMA(-uh, OCO_LOG_C11, OCO_LOG_C10);
  P = OCO_FMA(-uh, P, OCO_LOG_C9);
  P = OCO_FMA(-uh, P, OCO_LOG_C8);
  P = OCO_FMA(-uh, P, OCO_LOG_C7);
  P = OCO_FMA(-uh, P, OCO_LOG_C6);
  P = OCO_FMA(-uh, P, OCO_LOG_C5);
  P = OCO_FMA(-uh, P, OCO_LOG_C4);
  P = OCO_FMA(-uh, P, OCO_LOG_C3);
  P = OCO_M(OCO_M(s, uh), P);
  double qh = OCO_S(uh, half); /* Fast2Sum, |uh| >= |half| */
  double ql = OCO_A(OCO_S(OCO_S(uh, qh), half), OCO_A(OCO_S(ul, halfe), P));
  /* e ln2 + log F + log1p(u). */
  double ed = (double)e;
  double A = OCO_M(ed, OCO_LN2_HI); /* exact */
  double B = OCO_TAB(oco_logF_tab, idx);
  double s1 = OCO_A(A, B); /* TwoSum */
  double bb = OCO_S(s1, A);
  double t1 = OCO_A(OCO_S(A, OCO_S(s1, bb)), OCO_S(B, bb));
  double s2 = OCO_A(s1, qh); /* TwoSum */
  bb = OCO_S(s2, s1);
  double t2 = OCO_A(OCO_S(s1, OCO_S(s2, bb)), OCO_S(qh, bb));
  double lo = OCO_A(OCO_A(t1, t2),
                    OCO_A(OCO_A(OCO_M(ed, OCO_LN2_LO), OCO_TAB(oco_logF_tab, idx + 1)), ql));
  double r = OCO_A(s2, lo);
  *lh = r;
  *ll = OCO_S(lo, OCO_S(r, s2));
}

/* Natural exponential. */
OCO_HD double oco_exp(double x) { return oco_exp_dd(x, 0.0); }

/* Natural logarithm. */
OCO_HD double oco_log(double x) {
  if (oco_isnan(x)) return OCO_A(x, x);
  if (x < 0.0) return oco_nan();
  if (x == 0.0) return -oco_inf();
  if (oco_isinf(x)) return x;
  double lh, ll;
  oco_log_dd(x, &lh, &ll);
  return lh;
}

/* Base-10 logarithm. */
OCO_HD double oco_log10(double x) {
  if (oco_isnan(x)) return OCO_A(x, x);
  if (x < 0.0) return oco_nan();
  if (x == 0.0) return -oco_inf();
  if (oco_isinf(x)) return x;
  double lh, ll;
  oco_log_dd(x, &lh, &ll);
  double p = OCO_M(lh, OCO_LOG10E_HI);
  double pe = OCO_FMA(lh, OCO_LOG10E_HI, -p);
  return OCO_A(p, OCO_A(pe, OCO_A(OCO_M(lh, OCO_LOG10E_LO), OCO_M(ll, OCO_LOG10E_HI))));
}

/* 1 if y is an odd integer, 0 if an even integer, -1 if not an integer (y finite). */
OCO_HD int oco_int_class(double y) {
  if (y != trunc(y)) return -1;
  if (fabs(y) >= 0x1p53) return 0;
  return (int)((int64_t)y & 1);
}

/* 10^y: exactly the x == 10 path of oco_pow below (same operations, same result), without
 * the special-case ladder: y = +-0 gives 1, NaN gives NaN, +-inf give inf and 0 through
 * oco_exp_dd itself. */
OCO_HD double oco_pow10(double y) {
  double ph = OCO_M(y, OCO_LN10_HI);
  double pl = OCO_A(OCO_FMA(y, OCO_LN10_HI, -ph), OCO_M(y, OCO_LN10_LO));
  return OCO_M(1.0, oco_exp_dd(ph, pl));
}

/* x^y with the C99 Annex F special cases. */
OCO_HD double oco_pow(double x, double y) {
  if (y == 0.0 || x == 1.0) return 1.0;
  if (oco_isnan(x) || oco_isnan(y)) return OCO_A(x, y);
  double ay = fabs(y), ax = fabs(x);
  if (oco_isinf(y)) {
    if (ax == 1.0) return 1.0;
    return ((ax < 1.0) == (y < 0.0)) ? oco_inf() : 0.0;
  }
  int yc = oco_int_class(y);
  if (x == 0.0 || oco_isinf(x)) {
    int neg = (oco_d2u(x) >> 63) && (yc == 1);
    int big = (x == 0.0) ? (y < 0.0) : (y > 0.0);
    double r = big ? oco_inf() : 0.0;
    return neg ? -r : r;
  }
  double sign = 1.0;
  if (x < 0.0) {
    if (yc < 0) return oco_nan();
    if (yc == 1) sign = -1.0;
  }
  double ph, pl;
  if (x == 10.0) {
    ph = OCO_M(y, OCO_LN10_HI);
    pl = OCO_A(OCO_FMA(y, OCO_LN10_HI, -ph), OCO_M(y, OCO_LN10_LO));
  } else {
    double lh, ll;
    oco_log_dd(ax, &lh, &ll);
    ph = OCO_M(y, lh);
    pl = OCO_A(OCO_FMA(y, lh, -ph), OCO_M(y, ll));
  }
  (void)ay;
  return OCO_M(sign, oco_exp_dd(ph, pl));
}

#endif /* OCOMATH_H */
