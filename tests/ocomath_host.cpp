/* Host build of the exponential's branch-free fast phase (ocomath.h) for the CPU tests: the
 * plain kernels take oco_exp_fast_nb's result when it reports success and fall back to
 * oco_exp_dd otherwise, so the two must agree bit for bit wherever the fast phase succeeds. */
#include <cstdint>

#include "ocomath.h"

extern "C" void exp_fast_and_dd(const double *xh, const double *xl, int64_t n, double *fast, int32_t *ok,
                                double *dd) {
  for (int64_t i = 0; i < n; i++) {
    ok[i] = oco_exp_fast_nb(xh[i], xl[i], &fast[i]);
    dd[i] = oco_exp_dd(xh[i], xl[i]);
  }
}
