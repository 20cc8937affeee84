/*
 * kernels_inputs.cu -- synthetic disk inputs generated where they are used (disk_core.h):
 *
 *   k_disk_inputs   one thread per (column, z): the reference's disk model (calc_grid,
 *                   calc_density, calc_temperature of source/disk.f90:42-129) times the
 *                   seeded lognormal density perturbation, written in the reference layout
 *                   (nz, ny, nx) so that a block's rho and T need not cross PCIe.
 *
 * oco_disk_inputs (host) and oco_disk_inputs_device give the same bits: both evaluate
 * disk_core.h with IEEE basic operations and ocomath, without FMA contraction (this unit is
 * compiled with -fmad=false; its host code with -ffp-contract=off).
 */
#include <cuda_runtime.h>

#include <cmath>

#include "disk_core.h"
#include "oco_ctx.h"
#include "oco_internal.h"

namespace oco {

__global__ void __launch_bounds__(256) k_disk_inputs(const disk::Params p, double *__restrict__ rho,
                                                     double *__restrict__ T) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= p.ncol * p.nz) return;
  double r, t;
  disk::cell(p, i / p.nz, (int)(i % p.nz), r, t);
  rho[i] = r;
  T[i] = t;
}

}  // namespace oco

using namespace oco;

static int disk_params(const oco_disk_params *q, disk::Params &p) {
  if (!q || q->nx < 1 || q->ny < 1 || q->nz < 2) return OCO_EINVAL;
  const double v[] = {q->z0, q->z1, q->rho0, q->H, q->rho_floor, q->midTemp, q->sigma, q->floorTemp, q->isoTemp,
                      q->sigma_dex};
  for (double x : v)
    if (!std::isfinite(x)) return OCO_EINVAL;
  if (!(q->H > 0.0) || !(q->sigma > 0.0) || q->reserved != 0) return OCO_EINVAL;
  p.ncol = (int64_t)q->nx * q->ny;
  p.nz = q->nz;
  p.z0 = q->z0;
  p.z1 = q->z1;
  p.rho0 = q->rho0;
  p.H = q->H;
  p.rho_floor = q->rho_floor;
  p.midTemp = q->midTemp;
  p.sigma = q->sigma;
  p.floorTemp = q->floorTemp;
  p.switchTemp = (1.0 + 0x1p-52) * q->isoTemp; /* disk.f90:28, epsilon of a double */
  p.sigma_dex = q->sigma_dex;
  p.seed = q->seed;
  return OCO_OK;
}

extern "C" int oco_disk_inputs(const oco_disk_params *q, double *rho, double *T, double *dz) {
  disk::Params p;
  if (disk_params(q, p) != OCO_OK || !rho || !T)
    return oco_set_err(nullptr, OCO_EINVAL, "oco_disk_inputs: bad parameters (nx, ny >= 1, nz >= 2, H, sigma > 0, finite)");
  for (int64_t i = 0; i < p.ncol * p.nz; i++) disk::cell(p, i / p.nz, (int)(i % p.nz), rho[i], T[i]);
  if (dz) *dz = (p.z1 - p.z0) / (double)(p.nz - 1);
  return OCO_OK;
}

extern "C" int oco_disk_inputs_device(oco_ctx *c, const oco_disk_params *q, double *rho, double *T, void *stream) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  disk::Params p;
  if (disk_params(q, p) != OCO_OK || !rho || !T)
    return oco_set_err(c, OCO_EINVAL,
                       "oco_disk_inputs_device: bad parameters (nx, ny >= 1, nz >= 2, H, sigma > 0, finite)");
  if ((double)p.ncol * p.nz > 72057594037927936.0) return oco_set_err(c, OCO_EINVAL, "oco_disk_inputs_device: too many cells");
  CU(cudaSetDevice(c->device));
  const int64_t n = p.ncol * p.nz;
  k_disk_inputs<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(p, rho, T);
  CU(cudaGetLastError());
  c->launches += 1;
  return OCO_OK;
}

/* ---- Athena snapshots into HBM ------------------------------------------------------------
 * The device half of oco_deck_block_inputs_device: the host reads each z-block file's five raw
 * fields (rho, the three momenta, E; x fastest, read_athena.f90:169-201) into device memory,
 * and these kernels reassemble the block and apply the reader's physics with the host
 * reader's operations, so the results are bit-identical. */
namespace oco {

/* One z-block: cell (ix, iy, iz) of the file goes to (ix, iy, iz0 + iz) of the block
 * (nz, nyl, nxl); T receives E/rho minus the kinetic part (:174-202), momenta below 2^-52 in
 * magnitude skipped when lavoid (fix_momentum_underflow, :213-228). One thread per file cell
 * (coalesced reads). */
__global__ void __launch_bounds__(256) k_athena_zblock(const AthenaZBlock b) {
  const int64_t nc = (int64_t)b.nxl * b.nyl * b.nzl;
  const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f >= nc) return;
  const int ix = (int)(f % b.nxl), iy = (int)((f / b.nxl) % b.nyl), iz = (int)(f / ((int64_t)b.nxl * b.nyl));
  const int64_t q = ((int64_t)ix * b.nyl + iy) * b.nz + (b.iz0 + iz);
  const double r = b.raw[f];
  double t = 0.0;
#pragma unroll
  for (int comp = 1; comp <= 3; comp++) {
    const double pp = b.raw[comp * nc + f];
    if (!b.lavoid || fabs(pp) >= 0x1p-52) t = t + (0.5 * (pp * pp)) / r;
  }
  b.rho[q] = r;
  b.T[q] = (b.raw[4 * nc + f] - t) / r;
}

/* postprocess_athena_values (:230-277) and calc_temperature (disk.f90:64-109) on the block:
 * rho in cgs with its floor, T = T gamma1 unit_T, then T below switchTemp replaced by the
 * Gaussian profile Tgauss[iz] or the floor. */
__global__ void __launch_bounds__(256) k_athena_post(double *__restrict__ rho, double *__restrict__ T, int64_t n,
                                                     int nz, double unit_density, double rho_floor, double gamma1,
                                                     double unit_T, const double *__restrict__ Tgauss,
                                                     double switchTemp, double floorTemp) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r = rho[i] * unit_density;
  if (r < rho_floor) r = rho_floor;
  double t = (T[i] * gamma1) * unit_T;
  if (t < switchTemp) {
    const double tg = Tgauss[i % nz];
    t = tg > floorTemp ? tg : floorTemp;
  }
  rho[i] = r;
  T[i] = t;
}

cudaError_t launch_athena_zblock(const AthenaZBlock &b, cudaStream_t s) {
  const int64_t nc = (int64_t)b.nxl * b.nyl * b.nzl;
  if (nc == 0) return cudaSuccess;
  k_athena_zblock<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_athena_post(double *rho, double *T, int64_t n, int nz, double unit_density, double rho_floor,
                               double gamma1, double unit_T, const double *Tgauss, double switchTemp, double floorTemp,
                               cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  k_athena_post<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rho, T, n, nz, unit_density, rho_floor, gamma1, unit_T,
                                                          Tgauss, switchTemp, floorTemp);
  return cudaGetLastError();
}

}  // namespace oco
