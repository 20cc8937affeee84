/*
 * kernels_repair.cu -- k_repair: the FP64 re-solve (stable form) of the (column, wavelength)
 * items the mixed kernels flag.
 *
 * The mixed form's emergent flux is a weighted sum of boundary differences of U that FP32 can
 * resolve only where the sum is well conditioned; the mixed kernels append the other items to a
 * list (kernels_mixed.cu, push_flagged).  This kernel re-solves them and stores the results over
 * the mixed ones.  One warp per item (a persistent grid walks the list):
 *   1. the 32 lanes compute the column's FP64 records (pillar_record) and the item's opacity,
 *      absorption fraction and source function (opacity_at) for 32 levels at a time, and store
 *      kappa;
 *   2. the lanes compute every row's coefficients that do not depend on the elimination
 *      (1/kappa, a, c, the right-hand side and the diagonal excess of fill_center_coeffs /
 *      fill_boundary_coeffs, auxiliary.f90:125-201);
 *   3. lane 0 runs the difference-form elimination (the only recurrence) and the reverse sweep
 *      (solve_reverse: back-substitution, ghosts, flux).
 * Every expression is solve_item's (fp64_core.h) for the stable form with its operand order, and
 * this unit is compiled with -fmad=false, so a re-solved item equals the block solve's stable
 * form bit for bit.  An item costs the serial recurrence (three divisions per level) plus 1/32
 * of the per-level work, instead of the full per-level work of one thread.
 */
#include <cuda_runtime.h>

#include "fp64_core.h"
#include "oco_internal.h"

namespace oco {

/* A flagged item of a block chunk in the item interface of solve_reverse (cf. BlockItem). */
struct RBlockItem {
  const RepairArgs &a;
  int64_t cl;
  int w;
  __device__ __forceinline__ int64_t idx() const {
    return (a.layout == 0) ? (int64_t)w * a.ld_col + a.c_off + cl : (a.c_off + cl) * a.nw + w;
  }
  __device__ __forceinline__ int64_t pidx() const { return (int64_t)w * a.ld_col + a.c_off + cl; }
  __device__ __forceinline__ const double *lam() const { return a.lam64; }
  __device__ __forceinline__ int nz() const { return a.nz; }
  __device__ __forceinline__ int nw() const { return a.nw; }
  __device__ __forceinline__ int iw() const { return w; }
  __device__ __forceinline__ double dz() const { return a.dz; }
  __device__ __forceinline__ double dz2() const { return a.dz2; }
  __device__ __forceinline__ double dz1() const { return a.dz1; }
  __device__ __forceinline__ double *U() const { return a.U ? a.U + idx() * a.U_is : nullptr; }
  __device__ __forceinline__ double *K() const { return a.K ? a.K + idx() * a.K_is : nullptr; }
  __device__ __forceinline__ double *V() const { return a.V ? a.V + idx() * a.V_is : nullptr; }
  __device__ __forceinline__ int64_t uz() const { return a.U_zs; }
  __device__ __forceinline__ int64_t kz() const { return a.K_zs; }
  __device__ __forceinline__ int64_t vz() const { return a.V_zs; }
  __device__ __forceinline__ double *vtop() const { return a.Vtop ? a.Vtop + pidx() : nullptr; }
  __device__ __forceinline__ double *vbot() const { return a.Vbot ? a.Vbot + pidx() : nullptr; }
  __device__ __forceinline__ int64_t ss() const { return 1; }
  __device__ __forceinline__ const double *rho() const { return a.rho + cl * a.nz; }
  __device__ __forceinline__ const double *T() const { return a.T + cl * a.nz; }
  __device__ __forceinline__ unsigned long long id() const { return (unsigned long long)((a.c_off + cl) * a.nw + w); }
};

/* A flagged item of a ragged batch (cf. BatchItem in kernels_fp64.cu). */
struct RBatchItem {
  const RepairArgs &a;
  const MBatchCol &c;
  int64_t col;
  int w;
  __device__ __forceinline__ int nz() const { return c.nz; }
  __device__ __forceinline__ int nw() const { return c.nw; }
  __device__ __forceinline__ int iw() const { return w; }
  __device__ __forceinline__ const double *lam() const { return a.lam64 + c.lam_off / MIXED_LN * NL; }
  __device__ __forceinline__ double dz() const { return c.dz; }
  __device__ __forceinline__ double dz2() const { return c.dz2; }
  __device__ __forceinline__ double dz1() const { return c.dz1; }
  __device__ __forceinline__ int64_t zoff(int64_t base, int rows) const {
    return a.layout == 0 ? base + (int64_t)w * rows : base + w;
  }
  __device__ __forceinline__ double *U() const { return a.U ? a.U + zoff(c.u_off, c.nz + 6) : nullptr; }
  __device__ __forceinline__ double *K() const { return a.K ? a.K + zoff(c.kv_off, c.nz) : nullptr; }
  __device__ __forceinline__ double *V() const { return a.V ? a.V + zoff(c.kv_off, c.nz) : nullptr; }
  __device__ __forceinline__ int64_t uz() const { return a.layout == 0 ? 1 : c.nw; }
  __device__ __forceinline__ int64_t kz() const { return uz(); }
  __device__ __forceinline__ int64_t vz() const { return uz(); }
  __device__ __forceinline__ double *vtop() const { return a.Vtop ? a.Vtop + c.flux_off + w : nullptr; }
  __device__ __forceinline__ double *vbot() const { return a.Vbot ? a.Vbot + c.flux_off + w : nullptr; }
  __device__ __forceinline__ int64_t ss() const { return 1; }
  __device__ __forceinline__ const double *rho() const { return a.rho + c.in_off; }
  __device__ __forceinline__ const double *T() const { return a.T + c.in_off; }
  __device__ __forceinline__ unsigned long long id() const { return ((unsigned long long)col << 32) | (unsigned)w; }
};

/* The warp's scratch: eleven arrays of max_nz doubles. */
struct RScratch {
  double *op, *oma, *S, *o1, *aa, *cc, *dd, *ee, *gam, *uu, *qs;
  __device__ __forceinline__ RScratch(double *base, int max_nz) {
    double *p[11];
#pragma unroll
    for (int k = 0; k < 11; k++) p[k] = base + (int64_t)k * max_nz;
    op = p[0], oma = p[1], S = p[2], o1 = p[3], aa = p[4], cc = p[5], dd = p[6], ee = p[7], gam = p[8], uu = p[9],
    qs = p[10];
  }
};

template <class IT>
__device__ __forceinline__ void repair_item(const IT &it, double fit, const RScratch &r, unsigned long long *status) {
  const int lane = threadIdx.x & 31;
  const int nz = it.nz();
  const double dz = it.dz(), dz2 = it.dz2();
  const double *rho = it.rho(), *T = it.T();
  const LamR L(it, nullptr);
  double *Kb = it.K();
  const int64_t kz = it.kz();
  /* 1. records and opacities, 32 levels at a time */
  for (int z = lane; z < nz; z += 32) {
    double rec[NF];
    pillar_record(rho[z], T[z], fit, 0, rec);
    const Opac o = opacity_at<true>(SharedRec{rec}, L);
    r.op[z] = o.op;
    r.oma[z] = o.oma;
    r.S[z] = o.S;
    if (Kb) Kb[z * kz] = o.op;
  }
  __syncwarp();
  /* 2. the rows' coefficients (solve_item's forward sweep, stable form, without the recurrence):
   * row 0 stores h_0 in ee and the right-hand side numerator in dd; c of row j in cc */
  for (int j = lane; j < nz; j += 32) {
    const double op = r.op[j];
    const double o2 = op * op;
    r.o1[j] = 1.0 / op;
    if (j == 0) {
      const double zeta = ((op * dz2) * r.oma[0]) * 0.25;
      r.ee[0] = (dz + zeta) * o2;
      r.dd[0] = -((r.S[0] * zeta) * o2);
      r.cc[0] = op;
    } else if (j < nz - 1) {
      const double kh_prev = 0.5 * (op + r.op[j - 1]);
      const double kh = 0.5 * (r.op[j + 1] + op);
      r.aa[j] = o2 / kh_prev;
      r.cc[j] = o2 / kh;
      const double z3 = (dz2 * (op * (op * op))) * r.oma[j];
      r.dd[j] = -(r.S[j] * z3);
      r.ee[j] = z3;
    } else {
      r.aa[j] = op;
      const double zt = ((op * dz2) * r.oma[j]) * 0.25;
      r.cc[j] = 0.0;
      r.dd[j] = -((r.S[j] * zt) * o2);
      r.ee[j] = (dz + zt) * o2;
    }
  }
  __syncwarp();
  if (lane != 0) return;
  /* 3. the difference-form elimination and the reverse sweep */
  double h = r.ee[0];
  double bet = -(r.cc[0] + h);
  bool bad = bet == 0.0;
  double u = r.dd[0] / bet;
  r.uu[0] = u;
  double c_prev = r.cc[0];
  for (int j = 1; j < nz; j++) {
    const double aa = r.aa[j], cc = r.cc[j];
    const double den = c_prev + h;
    const double g = -(c_prev / den);
    r.qs[j - 1] = h / den;
    h = r.ee[j] + (aa * h) / den;
    bet = -(cc + h);
    if (bet == 0.0) bad = true;
    u = (r.dd[j] - aa * u) / bet;
    r.gam[j] = g;
    r.uu[j] = u;
    c_prev = cc;
  }
  if (bad) {
    atomicAdd(&status[0], 1ull);
    atomicMin(&status[1], it.id());
  }
  solve_reverse<1>(it, u, r.gam, r.uu, r.o1, r.qs);
}

__global__ void __launch_bounds__(128) k_repair(const RepairArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t n = (int64_t)*a.count;
  if (warp == 0 && lane == 0 && n) atomicAdd(a.repairs, (unsigned long long)n);
  const RScratch r(a.scratch + warp * 11 * (int64_t)a.max_nz, a.max_nz);
  for (int64_t k = warp; k < n; k += nwarps) {
    const unsigned long long id = a.list[k];
    if (a.block) {
      const int64_t cl = (int64_t)(id / (unsigned long long)a.nw);
      repair_item(RBlockItem{a, cl, (int)(id - (unsigned long long)cl * a.nw)}, a.fully_ionized_T, r, a.status);
    } else {
      const int64_t col = (int64_t)(id >> 32);
      repair_item(RBatchItem{a, a.cols[col], col, (int)(id & 0xffffffffu)}, a.fully_ionized_T, r, a.status);
    }
    __syncwarp();
  }
}

cudaError_t launch_repair(const RepairArgs &a, int num_sms, cudaStream_t s) {
  k_repair<<<num_sms * REPAIR_WARPS_PER_SM / 4, 128, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace oco
