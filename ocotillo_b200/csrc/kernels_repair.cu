/*
 * kernels_repair.cu -- the FP64 re-solve (stable form) of the (column, wavelength) items the
 * mixed kernels flag.
 *
 * The mixed form's emergent flux is a weighted sum of boundary differences of U that FP32 can
 * resolve only where the sum is well conditioned.  The mixed kernels list the other items
 * (kernels_mixed.cu): each item's id in an item list, whose index is the item's slot; each
 * item's bit in a word per (column, 32 wavelengths), with its slot beside the bit; and every
 * word that holds a bit, once, in a word list.  Two kernels then re-solve the items in the
 * stable FP64 form, split the way the work parallelises:
 *
 *   k_repair_coef   everything that is independent along z, fully parallel: a warp takes one
 *                   listed word and one chunk of CZ levels, its lanes compute the column's FP64
 *                   records (pillar_record) once for the chunk and, for every flagged item of
 *                   the word, the opacities (opacity_at) and the rows' coefficients a, c, the
 *                   right-hand side and the diagonal excess (fill_center_coeffs /
 *                   fill_boundary_coeffs, auxiliary.f90:125-201), stored in the item's slot
 *                   with 1/kappa, and kappa in the output;
 *   k_repair_solve  the recurrences: one lane per slot runs the difference-form elimination over
 *                   the stored coefficients (loads of 8 levels hoisted off the serial chain),
 *                   then the stable form's reverse sweep (solve_reverse: back-substitution,
 *                   ghosts, flux), storing over the mixed results.
 *
 * An item's critical path is thus its elimination alone (two dependent divisions per level)
 * instead of its whole per-level work, and the per-level work of all items runs at the GPU's
 * throughput.  Items beyond the slots' capacity (the mixed solve's scratch, free once that
 * kernel has finished) are re-solved one warp per item by k_repair_solve (repair_one: the same
 * phases per segment of RSEG levels, in the warp's shared memory).  Every expression is
 * solve_item's (fp64_core.h) for the stable form with its operand order, and this unit is
 * compiled with -fmad=false like the FP64 kernels, so a re-solved item equals OCO_FORM_STABLE
 * bit for bit.
 */
#include <cuda_runtime.h>

#include "fp64_core.h"
#include "oco_internal.h"

namespace oco {

/* A flagged item of a block chunk in the item interface of solve_item (cf. BlockItem). */
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
  __device__ __forceinline__ double sigma_grey() const { return 0.0; }
  __device__ __forceinline__ double *U() const { return a.U ? a.U + idx() * a.U_is : nullptr; }
  __device__ __forceinline__ double *K() const { return a.K ? a.K + idx() * a.K_is : nullptr; }
  __device__ __forceinline__ double *V() const { return a.V ? a.V + idx() * a.V_is : nullptr; }
  __device__ __forceinline__ int64_t uz() const { return a.U_zs; }
  __device__ __forceinline__ int64_t kz() const { return a.K_zs; }
  __device__ __forceinline__ int64_t vz() const { return a.V_zs; }
  __device__ __forceinline__ double *vtop() const { return a.Vtop ? a.Vtop + pidx() : nullptr; }
  __device__ __forceinline__ double *vbot() const { return a.Vbot ? a.Vbot + pidx() : nullptr; }
  __device__ __forceinline__ int64_t ss() const { return 32; }
  __device__ __forceinline__ unsigned long long *status() const { return a.status; }
  __device__ __forceinline__ unsigned long long id() const { return (unsigned long long)((a.c_off + cl) * a.nw + w); }
  __device__ __forceinline__ const double *rho() const { return a.rho + cl * a.nz; }
  __device__ __forceinline__ const double *T() const { return a.T + cl * a.nz; }
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
  __device__ __forceinline__ double sigma_grey() const { return 0.0; }
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
  __device__ __forceinline__ int64_t ss() const { return 32; }
  __device__ __forceinline__ unsigned long long *status() const { return a.status; }
  __device__ __forceinline__ unsigned long long id() const { return ((unsigned long long)col << 32) | (unsigned)w; }
  __device__ __forceinline__ const double *rho() const { return a.rho + c.in_off; }
  __device__ __forceinline__ const double *T() const { return a.T + c.in_off; }
};

/* An item whose scratch is one lane's contiguous arrays (the by-item path). */
template <class IT>
struct UnitStride : IT {
  __device__ __forceinline__ int64_t ss() const { return 1; }
};

/* ---- by item (items beyond the slots' capacity) ---------------------------------------- */
/* Levels per segment of the by-item path. */
constexpr int RSEG = 128;
constexpr int RWARPS = REPAIR_THREADS / 32;

/* The warp's shared buffers for one segment: opacity, absorption fraction and source function
 * of levels z0-1 .. z0+RSEG (index + 1), and the row coefficients of levels z0 .. z0+RSEG-1. */
struct RSeg {
  double op[RSEG + 2], oma[RSEG + 2], S[RSEG + 2];
  double aa[RSEG], cc[RSEG], dd[RSEG], ee[RSEG];
};

template <class IT>
__device__ __forceinline__ void repair_one(const IT &it, double fit, RSeg &g, double *gam, double *uu, double *o1,
                                           double *qs) {
  const int lane = threadIdx.x & 31;
  const int nz = it.nz();
  const double dz = it.dz(), dz2 = it.dz2();
  const double *rho = it.rho(), *T = it.T();
  const LamR L(it, nullptr);
  double *Kb = it.K();
  const int64_t kz = it.kz();
  double h = 0.0, u = 0.0, c_prev = 0.0; /* recurrence state (lane 0) */
  bool bad = false;
  for (int z0 = 0; z0 < nz; z0 += RSEG) {
    const int n = min(RSEG, nz - z0);
    /* 1. records and opacities of levels z0-1 .. z0+n (those that exist), 32 at a time */
    for (int k = lane; k < n + 2; k += 32) {
      const int z = z0 - 1 + k;
      if (z < 0 || z >= nz) continue;
      double rec[NF];
      pillar_record(rho[z], T[z], fit, 0, rec);
      const Opac o = opacity_at<true>(SharedRec{rec}, L);
      g.op[k] = o.op;
      g.oma[k] = o.oma;
      g.S[k] = o.S;
      if (Kb && k >= 1 && k <= n) Kb[z * kz] = o.op;
    }
    __syncwarp();
    /* 2. the rows' coefficients (solve_item's forward sweep, stable form, without the
     * recurrence): row 0 stores h_0 in ee and its right-hand side in dd; c of the row in cc */
    for (int k = lane; k < n; k += 32) {
      const int j = z0 + k;
      const double op = g.op[k + 1];
      const double o2 = op * op;
      o1[j] = 1.0 / op;
      if (j == 0) {
        const double zeta = ((op * dz2) * g.oma[1]) * 0.25;
        g.ee[k] = (dz + zeta) * o2;
        g.dd[k] = -((g.S[1] * zeta) * o2);
        g.cc[k] = op;
      } else if (j < nz - 1) {
        const double kh_prev = 0.5 * (op + g.op[k]);
        const double kh = 0.5 * (g.op[k + 2] + op);
        g.aa[k] = o2 / kh_prev;
        g.cc[k] = o2 / kh;
        const double z3 = (dz2 * (op * (op * op))) * g.oma[k + 1];
        g.dd[k] = -(g.S[k + 1] * z3);
        g.ee[k] = z3;
      } else {
        g.aa[k] = op;
        const double zt = ((op * dz2) * g.oma[k + 1]) * 0.25;
        g.cc[k] = 0.0;
        g.dd[k] = -((g.S[k + 1] * zt) * o2);
        g.ee[k] = (dz + zt) * o2;
      }
    }
    __syncwarp();
    /* 3. the difference-form elimination over the segment (lane 0) */
    if (lane == 0) {
      int k = 0;
      if (z0 == 0) {
        h = g.ee[0];
        const double bet = -(g.cc[0] + h);
        bad = bet == 0.0;
        u = g.dd[0] / bet;
        uu[0] = u;
        c_prev = g.cc[0];
        k = 1;
      }
      for (; k < n; k++) {
        const int j = z0 + k;
        const double aa = g.aa[k], cc = g.cc[k];
        const double den = c_prev + h;
        const double gj = -(c_prev / den);
        qs[j - 1] = h / den;
        h = g.ee[k] + (aa * h) / den;
        const double bet = -(cc + h);
        if (bet == 0.0) bad = true;
        u = (g.dd[k] - aa * u) / bet;
        gam[j] = gj;
        uu[j] = u;
        c_prev = cc;
      }
    }
    __syncwarp();
  }
  if (lane != 0) return;
  if (bad) {
    atomicAdd(&it.status()[0], 1ull);
    atomicMin(&it.status()[1], it.id());
  }
  /* 4. the reverse sweep: back-substitution, ghosts, flux (scratch at stride 1) */
  solve_reverse<1>(UnitStride<IT>{it}, u, gam, uu, o1, qs);
}

/* ---- coefficient slots ------------------------------------------------------------------ */
/* Slot pos of the coefficient arrays: level z of slot pos at ((pos / 32) * max_nz + z) * 32 +
 * pos % 32, so that 32 consecutive slots read one level as one 256-byte row. */
struct Slots {
  double *aa, *cc, *dd, *ee, *o1;
  int64_t max_nz;
  __device__ __forceinline__ Slots(const RepairArgs &a) {
    const int64_t n = a.cap * (int64_t)a.max_nz;
    aa = a.scratch;
    cc = aa + n;
    dd = cc + n;
    ee = dd + n;
    o1 = ee + n;
    max_nz = a.max_nz;
  }
  __device__ __forceinline__ int64_t at(int64_t pos, int z) const { return ((pos >> 5) * max_nz + z) * 32 + (pos & 31); }
};

/* Levels per coefficient task: lanes 1..CZ hold the task's levels, lanes 0 and CZ+1 their
 * neighbours (whose opacities the rows need). */
constexpr int CZ = 30;

/* One flagged item's rows for the task's levels: lane l holds level zl = c*CZ - 1 + l and its
 * record rec (valid: 0 <= zl < nz). */
template <class IT>
__device__ __forceinline__ void coef_item(const IT &it, const double *rec, int zl, bool valid, const Slots &S,
                                          int64_t pos) {
  const int lane = threadIdx.x & 31;
  const LamR L(it, nullptr);
  Opac o{0.0, 0.0, 0.0, 0.0};
  if (valid) o = opacity_at<true>(SharedRec{rec}, L);
  const double op_lo = __shfl_up_sync(0xffffffffu, o.op, 1), op_hi = __shfl_down_sync(0xffffffffu, o.op, 1);
  if (!valid || lane == 0 || lane > CZ) return;
  const int nz = it.nz(), j = zl;
  const double dz = it.dz(), dz2 = it.dz2();
  const double op = o.op, o2 = op * op;
  const int64_t q = S.at(pos, j);
  S.o1[q] = 1.0 / op;
  if (double *Kb = it.K()) Kb[j * it.kz()] = op;
  if (j == 0) { /* fill_boundary_coeffs :187-191; h_0 in ee */
    const double zeta = ((op * dz2) * o.oma) * 0.25;
    S.ee[q] = (dz + zeta) * o2;
    S.dd[q] = -((o.S * zeta) * o2);
    S.cc[q] = op;
  } else if (j < nz - 1) { /* fill_center_coeffs :159-165 */
    const double kh_prev = 0.5 * (op + op_lo);
    const double kh = 0.5 * (op_hi + op);
    S.aa[q] = o2 / kh_prev;
    S.cc[q] = o2 / kh;
    const double z3 = (dz2 * (op * (op * op))) * o.oma;
    S.dd[q] = -(o.S * z3);
    S.ee[q] = z3;
  } else { /* fill_boundary_coeffs :193-197 */
    S.aa[q] = op;
    const double zt = ((op * dz2) * o.oma) * 0.25;
    S.cc[q] = 0.0;
    S.dd[q] = -((o.S * zt) * o2);
    S.ee[q] = (dz + zt) * o2;
  }
}

constexpr int CWARPS = 4; /* warps per block of k_repair_coef */

__global__ void __launch_bounds__(CWARPS * 32, 4) k_repair_coef(const RepairArgs a) {
  __shared__ __align__(16) double s_rec[CWARPS][32 * NF];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t n_words = (int64_t)*a.count;
  const int nch = (a.max_nz + CZ - 1) / CZ;
  const unsigned long long ntasks = (unsigned long long)(n_words * nch);
  const Slots S(a);
  double *rec = &s_rec[wib][lane * NF]; /* each lane reads only its own record */
  /* tasks from a device counter, chunk-major (task t: chunk t / n_words of word t % n_words):
   * a task's cost grows with its word's flagged items, so a fixed assignment would leave some
   * warps with several times the mean */
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(a.queue, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= ntasks) break;
    const int c = (int)(t / (unsigned long long)n_words);
    const int64_t k = (int64_t)(t - (unsigned long long)c * n_words);
    const int64_t w = (int64_t)a.list[k];
    const int64_t col = w / a.wstride;
    const int word = (int)(w - col * a.wstride);
    const MBatchCol *bc = a.block ? nullptr : &a.cols[col];
    const int nz = a.block ? a.nz : bc->nz;
    if (c * CZ >= nz) continue;
    const double *rho = a.block ? a.rho + col * a.nz : a.rho + bc->in_off;
    const double *T = a.block ? a.T + col * a.nz : a.T + bc->in_off;
    const int zl = c * CZ - 1 + lane;
    const bool valid = zl >= 0 && zl < nz && lane <= CZ + 1;
    if (valid) pillar_record(rho[zl], T[zl], a.fully_ionized_T, 0, rec);
    for (unsigned m = a.bits[w]; m; m &= m - 1) {
      const int b = __ffs(m) - 1;
      const int64_t pos = a.slot[w * 32 + b];
      if (pos >= a.cap) continue; /* re-solved by item in k_repair_solve */
      if (a.block)
        coef_item(RBlockItem{a, col, word * 32 + b}, rec, zl, valid, S, pos);
      else
        coef_item(RBatchItem{a, *bc, col, word * 32 + b}, rec, zl, valid, S, pos);
    }
  }
}

/* The elimination over slot pos's coefficients (solve_item's recurrence for the stable form),
 * in place: gamma over a, u over the right-hand side, q_{j-1} over e_{j-1}; then the reverse
 * sweep. */
template <class IT>
__device__ __forceinline__ void chain_item(const IT &it, const Slots &S, int64_t pos) {
  const int nz = it.nz();
  const int64_t q0 = S.at(pos, 0);
  double *aa = S.aa + q0, *dd = S.dd + q0, *ee = S.ee + q0;
  const double *cc = S.cc + q0;
  double h = ee[0];
  double bet = -(cc[0] + h);
  bool bad = bet == 0.0;
  double u = dd[0] / bet;
  dd[0] = u;
  double c_prev = cc[0];
  auto step = [&](int j, double a_, double c_, double d_, double e_) {
    const double den = c_prev + h;
    const double g = -(c_prev / den);
    ee[(j - 1) * 32] = h / den; /* q_{j-1} = h_{j-1}/(c_{j-1} + h_{j-1}) */
    h = e_ + (a_ * h) / den;
    bet = -(c_ + h);
    if (bet == 0.0) bad = true;
    u = (d_ - a_ * u) / bet;
    aa[j * 32] = g;
    dd[j * 32] = u;
    c_prev = c_;
  };
  int j = 1;
  for (; j + 8 <= nz; j += 8) { /* the coefficients of 8 levels loaded ahead of the serial chain */
    for (int t = 16; t < 24 && j + t < nz; t++) { /* the block after next into L2 */
      prefetch_l2(&aa[(j + t) * 32]);
      prefetch_l2(&cc[(j + t) * 32]);
      prefetch_l2(&dd[(j + t) * 32]);
      prefetch_l2(&ee[(j + t) * 32]);
    }
    double ab[8], cb[8], db[8], eb[8];
#pragma unroll
    for (int t = 0; t < 8; t++) {
      ab[t] = aa[(j + t) * 32];
      cb[t] = cc[(j + t) * 32];
      db[t] = dd[(j + t) * 32];
      eb[t] = ee[(j + t) * 32];
    }
#pragma unroll
    for (int t = 0; t < 8; t++) step(j + t, ab[t], cb[t], db[t], eb[t]);
  }
  for (; j < nz; j++) step(j, aa[j * 32], cc[j * 32], dd[j * 32], ee[j * 32]);
  if (bad) {
    atomicAdd(&it.status()[0], 1ull);
    atomicMin(&it.status()[1], it.id());
  }
  solve_reverse<1, IT, true>(it, u, aa, dd, S.o1 + q0, ee);
}

__global__ void __launch_bounds__(REPAIR_THREADS, 6) k_repair_solve(const RepairArgs a) {
  __shared__ __align__(16) double s_seg[RWARPS][sizeof(RSeg) / sizeof(double)];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t n = (int64_t)*a.icount;
  const int64_t nfit = n < a.cap ? n : a.cap;
  if (warp == 0 && lane == 0 && n) atomicAdd(a.repairs, (unsigned long long)n);
  const Slots S(a);
  for (int64_t g = warp; g * 32 < nfit; g += nwarps) {
    const int64_t pos = g * 32 + lane;
    if (pos >= nfit) continue;
    const unsigned long long id = a.ilist[pos];
    if (a.block) {
      const int64_t cl = (int64_t)(id / (unsigned long long)a.nw);
      chain_item(RBlockItem{a, cl, (int)(id - (unsigned long long)cl * a.nw)}, S, pos);
    } else {
      const int64_t col = (int64_t)(id >> 32);
      chain_item(RBatchItem{a, a.cols[col], col, (int)(id & 0xffffffffu)}, S, pos);
    }
  }
  /* items beyond the slots: one warp per item, scratch after the slots */
  if (n <= nfit) return;
  RSeg &sg = *reinterpret_cast<RSeg *>(s_seg[wib]);
  double *base = a.scratch + 5 * a.cap * (int64_t)a.max_nz + warp * 4 * (int64_t)a.max_nz;
  double *gam = base, *uu = base + a.max_nz, *o1 = base + 2 * (int64_t)a.max_nz, *qs = base + 3 * (int64_t)a.max_nz;
  __syncwarp();
  for (int64_t k = nfit + warp; k < n; k += nwarps) {
    const unsigned long long id = a.ilist[k];
    if (a.block) {
      const int64_t cl = (int64_t)(id / (unsigned long long)a.nw);
      repair_one(RBlockItem{a, cl, (int)(id - (unsigned long long)cl * a.nw)}, a.fully_ionized_T, sg, gam, uu, o1, qs);
    } else {
      const int64_t col = (int64_t)(id >> 32);
      repair_one(RBatchItem{a, a.cols[col], col, (int)(id & 0xffffffffu)}, a.fully_ionized_T, sg, gam, uu, o1, qs);
    }
    __syncwarp();
  }
}

int64_t repair_capacity(size_t scratch_bytes, int max_nz, int solve_blocks) {
  const int64_t over = (int64_t)solve_blocks * RWARPS * 4 * max_nz * (int64_t)sizeof(double);
  const int64_t per = 5 * (int64_t)max_nz * (int64_t)sizeof(double);
  const int64_t cap = ((int64_t)scratch_bytes - over) / per;
  return cap > 0 ? cap & ~(int64_t)31 : 0;
}

cudaError_t launch_repair(const RepairArgs &a, int coef_blocks, int solve_blocks, cudaStream_t s) {
  k_repair_coef<<<coef_blocks, CWARPS * 32, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_repair_solve<<<solve_blocks, REPAIR_THREADS, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace oco
