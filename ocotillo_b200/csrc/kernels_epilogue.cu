/*
 * kernels_epilogue.cu -- per-(column, wavelength) quantities derived from a solved block, on
 * the device where the block's arrays already are:
 *   k_intensities     I+ = U + V and I- = U - V on the interior z (auxiliary.f90:80-94,
 *                     calc_intensity: upward and downward intensities);
 *   k_optical_depth   tau(z) = cumulative sum over z from index 1 of kappa rho dz, and the
 *                     first z index where tau reaches a target (tools/ocoutils/ReadOcotillo.py:
 *                     248-293, calculate_optical_depth and find_photosphere), -1 if never.
 *   k_integrated_flux the wavelength-integrated emergent flux per column, the trapezoid rule
 *                     over the wavelength grid as a weighted sum (weights in cm) in increasing
 *                     wavelength index; one thread per column, so a warp reads 32 adjacent
 *                     columns of a [lambda][column] flux plane (coalesced) and the sum order is
 *                     fixed.  No reference counterpart (the reference writes per-lambda planes
 *                     only); the bolometric emergent flux of each column.
 * One thread per item, z loop inside; compiled without FMA contraction so that the products
 * and the running sum round as the reference tools' array arithmetic does.
 */
#include <cuda_runtime.h>

#include <algorithm>

#include <cstdint>

#include "oco_internal.h"

namespace oco {

/* Address arithmetic of one block's arrays (see EpilogueArgs). */
__device__ __forceinline__ void item_bases(const EpilogueArgs &a, int64_t item, int64_t &iu, int64_t &iz,
                                           int64_t &zs_u, int64_t &zs) {
  const int64_t ncol = a.ncol;
  const int64_t col = item % ncol, iw = item / ncol; /* item = iw * ncol + col */
  if (a.layout == 0) {                               /* (nw, ncol, nz[+6]), z fastest */
    iu = (iw * ncol + col) * (a.nz + 6);
    iz = (iw * ncol + col) * a.nz;
    zs_u = zs = 1;
  } else { /* [z][col][lambda] */
    iu = iz = col * a.nw + iw;
    zs_u = zs = ncol * a.nw;
  }
}

__global__ void __launch_bounds__(256) k_intensities(const EpilogueArgs a) {
  const int64_t items = a.ncol * a.nw;
  for (int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; item < items;
       item += (int64_t)gridDim.x * blockDim.x) {
    int64_t iu, iz, zs_u, zs;
    item_bases(a, item, iu, iz, zs_u, zs);
    for (int z = 0; z < a.nz; z++) {
      const double u = a.U[iu + (int64_t)(z + 3) * zs_u], v = a.V[iz + (int64_t)z * zs];
      if (a.Ip) a.Ip[iz + (int64_t)z * zs] = u + v;
      if (a.Im) a.Im[iz + (int64_t)z * zs] = u - v;
    }
  }
}

__global__ void __launch_bounds__(256) k_optical_depth(const EpilogueArgs a) {
  const int64_t items = a.ncol * a.nw;
  for (int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; item < items;
       item += (int64_t)gridDim.x * blockDim.x) {
    int64_t iu, iz, zs_u, zs;
    item_bases(a, item, iu, iz, zs_u, zs);
    const int64_t col = item % a.ncol;
    const double *rho = a.rho + col * a.nz;
    double tau = 0.0;
    int photo = -1;
    for (int z = 0; z < a.nz; z++) {
      tau = tau + (a.K[iz + (int64_t)z * zs] * rho[z]) * a.dz;
      if (a.tau) a.tau[iz + (int64_t)z * zs] = tau;
      if (photo < 0 && tau >= a.target) photo = z;
    }
    if (a.photo) a.photo[item] = photo;
  }
}

__global__ void __launch_bounds__(256) k_integrated_flux(const double *__restrict__ V, const double *__restrict__ w,
                                                         int64_t ncol, int nw, int64_t ld_col, double *__restrict__ F) {
  for (int64_t col = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; col < ncol;
       col += (int64_t)gridDim.x * blockDim.x) {
    double f = 0.0;
    for (int iw = 0; iw < nw; iw++) f = f + __ldg(&w[iw]) * V[(int64_t)iw * ld_col + col];
    F[col] = f;
  }
}

cudaError_t launch_integrated_flux(const double *V, const double *w, int64_t ncol, int nw, int64_t ld_col, double *F,
                                   int blocks, cudaStream_t s) {
  k_integrated_flux<<<blocks, 256, 0, s>>>(V, w, ncol, nw, ld_col, F);
  return cudaGetLastError();
}

cudaError_t launch_intensities(const EpilogueArgs &a, int blocks, cudaStream_t s) {
  k_intensities<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_optical_depth(const EpilogueArgs &a, int blocks, cudaStream_t s) {
  k_optical_depth<<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace oco

namespace oco {

/* Reference-layout output from a lambda-fastest chunk: for each column col of the chunk, the
 * (rows x nw) plane src[z * src_zs + col * nw + iw] goes to dst[(iw * ld_col + c_off + col) *
 * rows + z].  Tiles of 64 z x 32 wavelengths through shared memory, so that the reads run along
 * lambda and the writes along z (256-byte runs both ways).  A persistent grid walks the tiles
 * (lambda tiles fastest, then z tiles, then columns), each block loading its next tile into
 * registers while it writes the current one out of shared memory, so that every block keeps a
 * tile's loads in flight throughout.  Block (32, 8). */
constexpr int TZ = 64; /* z rows per tile */
__global__ void __launch_bounds__(256) k_lambda_to_reference(const double *__restrict__ src, int64_t src_zs,
                                                             double *__restrict__ dst, int64_t ld_col,
                                                             int64_t c_off, int64_t nb, int rows, int nw) {
  __shared__ double tile[TZ][33];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ntw = (nw + 31) / 32, ntz = (rows + TZ - 1) / TZ;
  const int64_t per_col = (int64_t)ntw * ntz, ntiles = nb * per_col;
  int64_t t = blockIdx.x;
  if (t >= ntiles) return;
  double v[TZ / 8];
  auto coords = [&](int64_t tt, int64_t &col, int &z0, int &w0) {
    col = tt / per_col;
    const int r = (int)(tt - col * per_col);
    const int zt = r / ntw;
    z0 = zt * TZ;
    w0 = (r - zt * ntw) * 32;
  };
  auto load = [&](int64_t tt) {
    int64_t col;
    int z0, w0;
    coords(tt, col, z0, w0);
#pragma unroll
    for (int i = 0; i < TZ / 8; i++) {
      const int z = z0 + ty + 8 * i, iw = w0 + tx;
      v[i] = (z < rows && iw < nw) ? src[(int64_t)z * src_zs + col * nw + iw] : 0.0;
    }
  };
  load(t);
  for (;;) {
    int64_t col;
    int z0, w0;
    coords(t, col, z0, w0);
#pragma unroll
    for (int i = 0; i < TZ / 8; i++) tile[ty + 8 * i][tx] = v[i];
    __syncthreads();
    const int64_t tn = t + gridDim.x;
    if (tn < ntiles) load(tn); /* the next tile's loads in flight during this tile's stores */
#pragma unroll
    for (int j = 0; j < TZ / 8; j++) {
      const int lw = ty + 8 * (j >> 1), zz = tx + 32 * (j & 1);
      const int iw = w0 + lw, z = z0 + zz;
      if (z < rows && iw < nw) dst[((int64_t)iw * ld_col + c_off + col) * rows + z] = tile[zz][lw];
    }
    __syncthreads();
    if (tn >= ntiles) break;
    t = tn;
  }
}

cudaError_t launch_lambda_to_reference(const double *src, int64_t src_zs, double *dst, int64_t ld_col, int64_t c_off,
                                       int64_t nb, int rows, int nw, int num_sms, cudaStream_t s) {
  if (nb <= 0) return cudaSuccess;
  const int64_t ntiles = nb * ((nw + 31) / 32) * (int64_t)((rows + TZ - 1) / TZ);
  const int64_t blocks = std::min<int64_t>(ntiles, (int64_t)num_sms * 8); /* 8 resident blocks of 256 per SM */
  k_lambda_to_reference<<<(unsigned)blocks, dim3(32, 8), 0, s>>>(src, src_zs, dst, ld_col, c_off, nb, rows, nw);
  return cudaGetLastError();
}

}  // namespace oco
