/* Host build of the batch descriptor checks (batch_layout.h) for the CPU tests. */
#include <cstdint>
#include <vector>

#include "batch_layout.h"

extern "C" void batch_first_overlap(const int64_t *off, const int64_t *len, int64_t n, int64_t *pair) {
  std::vector<int64_t> o(off, off + n), l(len, len + n);
  const auto pr = oco::first_overlap(o, l);
  pair[0] = pr.first;
  pair[1] = pr.second;
}
