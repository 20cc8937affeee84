/*
 * mathcheck.c -- reference values for testing the ocomath functions (TEST INFRASTRUCTURE).
 * Evaluates exp/log/log10/pow element-wise with (a) glibc, (b) quad precision (libquadmath,
 * 113-bit significand) rounded to double -- a correctly rounded reference except within
 * 2^-113 of a rounding boundary -- and (c) the host build of ocomath.
 * fn: 0 exp(x), 1 log(x), 2 log10(x), 3 pow(x, y), 4 10^y (ocomath's dedicated oco_pow10).
 */
#include <math.h>
#include <quadmath.h>
#include <stdint.h>

#include "ocomath.h"

void mc_glibc(int fn, const double *x, const double *y, double *out, int64_t n) {
  for (int64_t i = 0; i < n; i++)
    out[i] = fn == 0 ? exp(x[i]) : fn == 1 ? log(x[i]) : fn == 2 ? log10(x[i]) : pow(x[i], y[i]);
}

void mc_quad(int fn, const double *x, const double *y, double *out, int64_t n) {
  for (int64_t i = 0; i < n; i++) {
    __float128 a = (__float128)x[i];
    __float128 r = fn == 0 ? expq(a) : fn == 1 ? logq(a) : fn == 2 ? log10q(a) : powq(a, (__float128)y[i]);
    out[i] = (double)r;
  }
}

void mc_ocomath(int fn, const double *x, const double *y, double *out, int64_t n) {
  for (int64_t i = 0; i < n; i++)
    out[i] = fn == 0 ? oco_exp(x[i]) : fn == 1 ? oco_log(x[i]) : fn == 2 ? oco_log10(x[i])
             : fn == 3 ? oco_pow(x[i], y[i]) : oco_pow10(y[i]);
}
