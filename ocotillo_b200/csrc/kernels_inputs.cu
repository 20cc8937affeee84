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
