/*
 * kernels_mixed_pillars.cu -- per-(column, z) records of the mixed-precision form.
 *
 *   k_pillars_mixed        one thread per (column, z): Saha ionization and the z-only factors
 *                          in FP64, written as the FP32 log2 record of mixed_core.h (MixedZ,
 *                          256 B; large logarithms as integer + fraction).
 *   k_pillars_mixed_batch  the same for the columns of a ragged batch.
 * Both mark the columns that the solve kernels must re-solve in FP64 (mx::pillar), and write
 * each warp's 32 consecutive records through shared memory with coalesced stores.
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

constexpr int PM_THREADS = 128;
constexpr int PM_STRIDE = MZN + 4; /* floats per record in shared memory (16-byte rows, no bank conflicts) */

/* Writes the warp's records (lane l: record i0 + l, held in r) to rec with coalesced 512-byte
 * stores: each lane puts its record in the warp's shared buffer, then the warp copies the
 * 32 consecutive records out float4 by float4 (records at or beyond n are not written). */
__device__ __forceinline__ void store_records(const float *r, float *__restrict__ buf, float *__restrict__ rec,
                                              int64_t i0, int64_t n) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < MZN / 4; k++)
    *reinterpret_cast<float4 *>(buf + lane * PM_STRIDE + 4 * k) = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
  __syncwarp();
  float4 *o = reinterpret_cast<float4 *>(rec + i0 * MZN);
#pragma unroll
  for (int m = 0; m < MZN / 4; m++) {
    const int j = lane + 32 * m, q = j / (MZN / 4), part = j % (MZN / 4);
    if (i0 + q < n) o[j] = *reinterpret_cast<const float4 *>(buf + q * PM_STRIDE + 4 * part);
  }
}

/* colflag[col] is set to 1 when a cell of the column has a negative neutral fraction (see
 * mx::pillar); the caller clears it first. */
__global__ void __launch_bounds__(PM_THREADS) k_pillars_mixed(const double *__restrict__ rho,
                                                              const double *__restrict__ T, int64_t n, int nz,
                                                              double fully_ionized_T, float *__restrict__ rec,
                                                              unsigned *__restrict__ colflag) {
  __shared__ __align__(16) float s_buf[PM_THREADS / 32][32 * PM_STRIDE];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i0 = i - (threadIdx.x & 31);
  if (i0 >= n) return; /* whole warp past the end */
  float r[MZN];
  if (i < n) {
    if (pillar(rho[i], T[i], fully_ionized_T, r)) colflag[i / nz] = 1u;
  } else {
#pragma unroll
    for (int k = 0; k < MZN; k++) r[k] = 0.0f; /* not stored */
  }
  store_records(r, s_buf[threadIdx.x >> 5], rec, i0, n);
}

static_assert(MZN == MIXED_ZN, "mixed record size");

cudaError_t launch_pillars_mixed(const double *rho, const double *T, int64_t ncol, int nz, double fully_ionized_T,
                                 float *rec, unsigned *colflag, cudaStream_t s) {
  const int64_t n = ncol * nz;
  if (n == 0) return cudaSuccess;
  k_pillars_mixed<<<(unsigned)((n + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(rho, T, n, nz, fully_ionized_T,
                                                                                      rec, colflag);
  return cudaGetLastError();
}

/* Batch records: thread i is record i of the dense [sum nz] list; its column comes from a
 * binary search of the nz prefix sums rec_pre[0..ncol]. */
__global__ void __launch_bounds__(PM_THREADS) k_pillars_mixed_batch(const double *__restrict__ rho,
                                                             const double *__restrict__ T,
                                                             const MBatchCol *__restrict__ cols,
                                                             const int64_t *__restrict__ rec_pre, int64_t ncol,
                                                             int64_t n, double fully_ionized_T,
                                                             float *__restrict__ rec, unsigned *__restrict__ colflag) {
  __shared__ __align__(16) float s_buf[PM_THREADS / 32][32 * PM_STRIDE];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i0 = i - (threadIdx.x & 31);
  if (i0 >= n) return; /* whole warp past the end */
  float r[MZN];
  if (i < n) {
    int64_t lo = 0, hi = ncol;
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if (rec_pre[mid] <= i)
        lo = mid;
      else
        hi = mid;
    }
    const int64_t src = cols[lo].in_off + (i - rec_pre[lo]);
    if (pillar(rho[src], T[src], fully_ionized_T, r)) colflag[lo] = 1u;
  } else {
#pragma unroll
    for (int k = 0; k < MZN; k++) r[k] = 0.0f; /* not stored */
  }
  store_records(r, s_buf[threadIdx.x >> 5], rec, i0, n);
}

cudaError_t launch_pillars_mixed_batch(const double *rho, const double *T, const MBatchCol *cols,
                                       const int64_t *rec_pre, int64_t ncol, int64_t nrec, double fully_ionized_T,
                                       float *rec, unsigned *colflag, cudaStream_t s) {
  if (nrec == 0) return cudaSuccess;
  k_pillars_mixed_batch<<<(unsigned)((nrec + PM_THREADS - 1) / PM_THREADS), PM_THREADS, 0, s>>>(
      rho, T, cols, rec_pre, ncol, nrec, fully_ionized_T, rec, colflag);
  return cudaGetLastError();
}

}  // namespace oco
