// Host build of the disk generator's random numbers (disk_core.h) for the CPU tests.
#include "disk_core.h"

extern "C" void philox_host(const unsigned *ctr, unsigned k0, unsigned k1, unsigned *out) {
  oco::disk::philox4x32_10(ctr, k0, k1, out);
}
extern "C" void normals_host(unsigned long long seed, long long n, double *out) {
  for (long long i = 0; i < n; i++) out[i] = oco::disk::normal(seed, (uint64_t)i);
}
