/*
 * kernels_mixed_pillars.cu -- per-(column, z) records of the mixed-precision form.
 *
 *   k_pillars_mixed        one thread per (column, z): Saha ionization and the z-only factors
 *                          in FP64, written as the FP32 log2 record of mixed_core.h (MixedZ,
 *                          256 B; large logarithms as integer + fraction).
 *   k_pillars_mixed_batch  the same for the columns of a ragged batch.
 * Both mark the columns that the solve kernels must re-solve in FP64 (mx::pillar).
 *
 * Compiled with -fmad=false like the FP64 kernels: the Saha quadratic
 * 0.5*(sqrt(C^2 + 4C) - C) (gas_state.f90:63) cancels as the gas approaches full ionization
 * (1 - x ~ 1e-7 carries ~1% rounding error in FP64, as the reference's own comment notes), so
 * the FP64 form of this arithmetic must be the reference's, operation for operation, for the
 * mixed form to agree with the FP64 forms there.
 */
#include <cuda_runtime.h>

#include "mixed_core.h"
#include "oco_internal.h"

namespace oco {
using namespace oco::mx;

/* colflag[col] is set to 1 when a cell of the column has a negative neutral fraction (see
 * mx::pillar); the caller clears it first. */
__global__ void __launch_bounds__(256) k_pillars_mixed(const double *__restrict__ rho, const double *__restrict__ T,
                                                       int64_t n, int nz, double fully_ionized_T, float *__restrict__ rec,
                                                       unsigned *__restrict__ colflag) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float r[MZN];
  if (pillar(rho[i], T[i], fully_ionized_T, r)) colflag[i / nz] = 1u;
  float4 *o = reinterpret_cast<float4 *>(rec + i * MZN);
#pragma unroll
  for (int k = 0; k < MZN / 4; k++) o[k] = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
}

static_assert(MZN == MIXED_ZN, "mixed record size");

cudaError_t launch_pillars_mixed(const double *rho, const double *T, int64_t ncol, int nz, double fully_ionized_T,
                                 float *rec, unsigned *colflag, cudaStream_t s) {
  const int64_t n = ncol * nz;
  if (n == 0) return cudaSuccess;
  k_pillars_mixed<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(rho, T, n, nz, fully_ionized_T, rec, colflag);
  return cudaGetLastError();
}

/* Batch records: thread i is record i of the dense [sum nz] list; its column comes from a
 * binary search of the nz prefix sums rec_pre[0..ncol]. */
__global__ void __launch_bounds__(256) k_pillars_mixed_batch(const double *__restrict__ rho,
                                                             const double *__restrict__ T,
                                                             const MBatchCol *__restrict__ cols,
                                                             const int64_t *__restrict__ rec_pre, int64_t ncol,
                                                             int64_t n, double fully_ionized_T,
                                                             float *__restrict__ rec, unsigned *__restrict__ colflag) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int64_t lo = 0, hi = ncol;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (rec_pre[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  const int64_t src = cols[lo].in_off + (i - rec_pre[lo]);
  float r[MZN];
  if (pillar(rho[src], T[src], fully_ionized_T, r)) colflag[lo] = 1u;
  float4 *o = reinterpret_cast<float4 *>(rec + i * MZN);
#pragma unroll
  for (int k = 0; k < MZN / 4; k++) o[k] = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
}

cudaError_t launch_pillars_mixed_batch(const double *rho, const double *T, const MBatchCol *cols,
                                       const int64_t *rec_pre, int64_t ncol, int64_t nrec, double fully_ionized_T,
                                       float *rec, unsigned *colflag, cudaStream_t s) {
  if (nrec == 0) return cudaSuccess;
  k_pillars_mixed_batch<<<(unsigned)((nrec + 255) / 256), 256, 0, s>>>(rho, T, cols, rec_pre, ncol, nrec,
                                                                       fully_ionized_T, rec, colflag);
  return cudaGetLastError();
}

}  // namespace oco
