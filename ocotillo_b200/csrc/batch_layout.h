/* Host-side checks of a ragged batch's column descriptors (oco_batch_create).  Plain C++,
 * no CUDA, so that a host test compiles it directly. */
#pragma once

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <utility>
#include <vector>

namespace oco {

/* Largest element offset a column descriptor may carry: 2^56 doubles (512 PiB) is far beyond
 * any device array, and offset + (nz + 6) * nw < 2^56 + 2^62 then stays inside int64. */
constexpr int64_t kBatchMaxOffset = int64_t(1) << 56;

/* The first pair of columns (lower index first) whose element ranges [off[i], off[i] + len[i])
 * intersect, or {-1, -1} when they are pairwise disjoint.  Empty ranges intersect nothing.
 * One sort by start; a range that starts before the furthest end seen so far meets the range
 * that reaches there. */
inline std::pair<int64_t, int64_t> first_overlap(const std::vector<int64_t> &off, const std::vector<int64_t> &len) {
  std::vector<int64_t> idx(off.size());
  std::iota(idx.begin(), idx.end(), int64_t(0));
  std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return off[a] != off[b] ? off[a] < off[b] : a < b; });
  bool any = false;
  int64_t end = 0, owner = -1;
  for (int64_t k : idx) {
    if (len[k] <= 0) continue;
    if (any && off[k] < end) return {std::min(owner, k), std::max(owner, k)};
    if (!any || off[k] + len[k] > end) {
      end = off[k] + len[k];
      owner = k;
    }
    any = true;
  }
  return {-1, -1};
}

}  // namespace oco
