/* Fortran unformatted sequential records as gfortran writes them (io.f90's binary outputs):
 * a 4-byte length marker before and after the data.  A record longer than the largest
 * subrecord (gfortran's default, 2147483639 bytes) is split into subrecords whose leading
 * marker is negative when more follow and whose trailing marker is negative when one
 * precedes.  Host-only, no CUDA. */
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdio>

namespace oco {

constexpr size_t kFortranMaxSubrecord = 2147483639u;

/* Appends one record of `bytes` bytes; max_sub (1 .. kFortranMaxSubrecord) is the largest
 * subrecord, smaller only to test the splitting.  False on a write error or a bad max_sub. */
inline bool write_fortran_record(FILE *fp, const void *data, size_t bytes, size_t max_sub = kFortranMaxSubrecord) {
  if (max_sub == 0 || max_sub > kFortranMaxSubrecord) return false;
  const char *p = (const char *)data;
  size_t left = bytes;
  bool first = true;
  do {
    const size_t len = left > max_sub ? max_sub : left;
    const bool last = left == len;
    const int32_t lead = last ? (int32_t)len : -(int32_t)len;
    const int32_t trail = first ? (int32_t)len : -(int32_t)len;
    if (fwrite(&lead, 4, 1, fp) != 1) return false;
    if (len && fwrite(p, 1, len, fp) != len) return false;
    if (fwrite(&trail, 4, 1, fp) != 1) return false;
    p += len;
    left -= len;
    first = false;
  } while (left > 0);
  return true;
}

}  // namespace oco
