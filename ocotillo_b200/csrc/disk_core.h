/*
 * disk_core.h -- synthetic disk columns (the reference's disk model) with a seeded lognormal
 * density perturbation, for the host and the device from one source.
 *
 * Per cell (column c, level i = 1..nz), as source/disk.f90 computes it:
 *   calc_grid (:42-62)          dz = (z1 - z0)/(nz - 1),  z_i = z0 + (i - 1)*dz
 *   calc_density (:111-129)     rho_i = rho0*exp(-((0.5*z_i**2)/H**2)), floored at rho_floor
 *   calc_temperature (:64-109)  T_i = midTemp; where T_i < switchTemp = (1 + 2^-52)*isoTemp
 *                               (disk.f90:28), T_i = Tgauss_i if Tgauss_i > floorTemp else
 *                               floorTemp, Tgauss_i = midTemp*exp(-((0.5*z_i**2)/sigma**2))
 * then rho_i *= 10^(sigma_dex*N) with N a standard normal drawn for the cell: Philox4x32-10
 * (Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11), key =
 * seed, counter = (cell index, attempt), two 53-bit uniforms per draw, Marsaglia's polar method
 * (Marsaglia & Bray 1964) for N.  Every operation is an IEEE basic operation or a correctly
 * rounded ocomath function, with no FMA contraction (host: -ffp-contract=off; device:
 * -fmad=false), so host and device produce the same bits.
 */
#ifndef OCO_DISK_CORE_H
#define OCO_DISK_CORE_H

#include <stdint.h>

#include "ocomath.h"

#ifdef __CUDACC__
#define DK_HD static __host__ __device__ __forceinline__
#else
#define DK_HD static inline
#endif

namespace oco {
namespace disk {

struct Params {
  int64_t ncol;
  int nz;
  double z0, z1;
  double rho0, H, rho_floor;
  double midTemp, sigma, floorTemp, switchTemp;
  double sigma_dex;
  uint64_t seed;
};

/* Philox4x32-10: ten rounds of the published S-box (multipliers 0xD2511F53, 0xCD9E8D57; key
 * schedule constants 0x9E3779B9, 0xBB67AE85). */
DK_HD void mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}
DK_HD void philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c0, hi0, lo0);
    mulhilo(0xCD9E8D57u, c2, hi1, lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
    c0 = n0, c1 = n1, c2 = n2, c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0, out[1] = c1, out[2] = c2, out[3] = c3;
}

/* A uniform double in [0, 1) from two words: 53 random bits times 2^-53 (exact). */
DK_HD double u53(uint32_t hi, uint32_t lo) {
  const uint64_t m = ((uint64_t)(hi >> 5) << 26) | (uint64_t)(lo >> 6);
  return (double)m * 0x1p-53;
}

/* Standard normal for cell `cell`: polar method on successive Philox blocks (attempts). */
DK_HD double normal(uint64_t seed, uint64_t cell) {
  for (uint32_t attempt = 0;; attempt++) {
    const uint32_t ctr[4] = {(uint32_t)cell, (uint32_t)(cell >> 32), attempt, 0x6f636f74u};
    uint32_t r[4];
    philox4x32_10(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), r);
    const double v1 = 2.0 * u53(r[0], r[1]) - 1.0, v2 = 2.0 * u53(r[2], r[3]) - 1.0;
    const double s = v1 * v1 + v2 * v2;
    if (s < 1.0 && s > 0.0) return v1 * sqrt((-2.0 * oco_log(s)) / s);
  }
}

/* rho and T of cell i (0-based level) of column c. */
DK_HD void cell(const Params &p, int64_t c, int i, double &rho, double &T) {
  const double dz = (p.z1 - p.z0) / (double)(p.nz - 1);
  const double z = p.z0 + (double)i * dz;
  double r = p.rho0 * oco_exp(-((0.5 * (z * z)) / (p.H * p.H)));
  if (r < p.rho_floor) r = p.rho_floor;
  double t = p.midTemp;
  if (t < p.switchTemp) {
    const double tg = p.midTemp * oco_exp(-((0.5 * (z * z)) / (p.sigma * p.sigma)));
    t = tg > p.floorTemp ? tg : p.floorTemp;
  }
  if (p.sigma_dex != 0.0) r = r * oco_pow10(p.sigma_dex * normal(p.seed, (uint64_t)c * (uint64_t)p.nz + (uint64_t)i));
  rho = r;
  T = t;
}

}  // namespace disk
}  // namespace oco

#endif
