/*
 * kernels_fp64.cu -- the FP64 hot path on sm_100a.
 *
 *   k_pillars   one thread per (column, z): Saha ionization and every factor of the
 *               reference's per-(z, lambda) opacity that depends on z only
 *               (gas_state.f90:30-110, continuous_opacity.f90:143-163 and the z-only
 *               parts of :203-300).  Hoisting changes no bits: each hoisted expression is
 *               the reference's expression with its operand order.
 *   k_solve     persistent kernel, one thread per (column, wavelength), warps take tasks
 *               of 32 consecutive items (lambda fastest) from a device counter.  Per item:
 *               opacity, albedo and source function (continuous_opacity.f90:175-201,
 *               :377-409), tridiagonal coefficients (auxiliary.f90:111-201), the Thomas
 *               forward sweep (auxiliary.f90:14-41) streaming gamma, u and 1/kappa to a
 *               per-warp-slot scratch, then the back-substitution (:43-45), ghost zones
 *               (:49-62) and 6th-order flux (:64-109) in one reverse sweep with a 7-point
 *               register window.
 *
 * Output stores (U, kappa, V and the emergent flux) use the streaming cache hint (st.global.cs,
 * evict first): they are never read back, and L2 then keeps more of the forward sweep's scratch
 * for the reverse sweep.
 *
 * This translation unit is compiled with -fmad=false (no FMA contraction) and IEEE
 * division/square root, and calls the ocomath functions, so FORM_PLAIN reproduces the CPU
 * oracle (ocomath back-end) bit for bit.  FORM_STABLE replaces the pivot recursion
 * bet_j = b_j - a_j*gam_j by its difference form (no cancellation; same linear system).
 */
#include <cuda_runtime.h>

#include "fp64_core.h"

namespace oco {

#if defined(__CUDACC__) && !defined(__CUDACC_RTC__)
#if defined(__FMA__) || defined(__USE_FAST_MATH__)
#error "kernels_fp64.cu must be compiled without fast math"
#endif
#endif

constexpr int PIL_THREADS = 128;
constexpr int PIL_STRIDE = NF + 1; /* doubles per record in shared memory (odd: no bank conflicts) */

/* Writes the warp's records (lane l: record i0 + l, held in r) to pil with coalesced stores:
 * each lane puts its record in the warp's shared buffer, then the warp copies the 32
 * consecutive records out (records at or beyond n are not written). */
__device__ __forceinline__ void store_pillars(const double *r, double *__restrict__ buf, double *__restrict__ pil,
                                              int64_t i0, int64_t n) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NF; k++) buf[lane * PIL_STRIDE + k] = r[k];
  __syncwarp();
  double *o = pil + i0 * NF;
#pragma unroll
  for (int m = 0; m < NF; m++) {
    const int j = lane + 32 * m, q = j / NF, f = j % NF;
    if (i0 + q < n) o[j] = buf[q * PIL_STRIDE + f];
  }
}

__global__ void __launch_bounds__(PIL_THREADS) k_pillars(const double *__restrict__ rho,
                                                         const double *__restrict__ T, int64_t n,
                                                         double fully_ionized_T, int grey,
                                                         double *__restrict__ pil) {
  __shared__ double s_buf[PIL_THREADS / 32][32 * PIL_STRIDE];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i0 = i - (threadIdx.x & 31);
  if (i0 >= n) return; /* whole warp past the end */
  double r[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) r[k] = 0.0; /* grey records set three fields */
  if (i < n) pillar_record(rho[i], T[i], fully_ionized_T, grey, r);
  store_pillars(r, s_buf[threadIdx.x >> 5], pil, i0, n);
}

/* Batch records: thread i is record i of the dense [sum nz] list; its column comes from a
 * binary search of the nz prefix sums rec_pre[0..ncol]. */
__global__ void __launch_bounds__(PIL_THREADS) k_pillars_batch(const double *__restrict__ rho,
                                                               const double *__restrict__ T,
                                                               const MBatchCol *__restrict__ cols,
                                                               const int64_t *__restrict__ rec_pre, int64_t ncol,
                                                               int64_t n, double fully_ionized_T,
                                                               double *__restrict__ pil) {
  __shared__ double s_buf[PIL_THREADS / 32][32 * PIL_STRIDE];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t i0 = i - (threadIdx.x & 31);
  if (i0 >= n) return; /* whole warp past the end */
  double r[NF];
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
    pillar_record(rho[src], T[src], fully_ionized_T, 0, r);
  } else {
#pragma unroll
    for (int k = 0; k < NF; k++) r[k] = 0.0; /* not stored */
  }
  store_pillars(r, s_buf[threadIdx.x >> 5], pil, i0, n);
}

/* ---- pillar access ------------------------------------------------------------------- */
/* Generic path: each lane reads its own column's records through the read-only cache. */
struct DirectPillars {
  const double *base;
  __device__ __forceinline__ GlobalRec at(int z) { return GlobalRec{base + (int64_t)z * NF}; }
};

constexpr int ZC = 16;            /* z records per staged chunk */
constexpr int WARPS_PER_BLOCK = 4; /* k_solve runs 128-thread blocks */
constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

/* Staged path: all 32 lanes of the warp work on one column.  Lane 0 streams the column's
 * pillar records in chunks of ZC z with a bulk (TMA) copy into one of two shared-memory
 * buffers per warp; an mbarrier per buffer signals arrival.  Records are read in increasing
 * z, one at a time: entering chunk c frees the buffer of chunk c-1, which then receives
 * chunk c+1.  Waits are bounded; on timeout the warp records the failure and stops. */
struct StagedPillars {
  double *buf;    /* shared: [2][ZC*NF] */
  uint32_t bar0;  /* shared address of two mbarriers (8 B each) */
  const double *src;
  int nz, nchunks, cur;
  uint32_t waits;    /* bit b: parity of the next wait on buffer b */
  uint32_t inflight; /* bit b: a copy into buffer b has been issued and not yet waited for */
  bool failed;

  __device__ __forceinline__ void issue(int c) {
    const int rows = min(ZC, nz - c * ZC);
    const uint32_t bytes = (uint32_t)(rows * NF * sizeof(double));
    const uint32_t bar = bar0 + 8u * (c & 1);
    const uint32_t dst = smem_addr(buf + (c & 1) * (ZC * NF));
    const size_t g = __cvta_generic_to_global(src + (int64_t)c * ZC * NF);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(g), "r"(bytes), "r"(bar)
                 : "memory");
  }
  /* Waits (bounded) for the copy into buffer b.  Every lane tracks the same state. */
  __device__ __forceinline__ bool wait(int b) {
    if (!((inflight >> b) & 1u)) return true;
    const uint32_t bar = bar0 + 8u * b;
    const uint32_t parity = (waits >> b) & 1u;
    long long spins = 0;
    while (!mbar_try_wait(bar, parity))
      if (++spins > kSpinLimit) return false;
    waits ^= 1u << b;
    inflight &= ~(1u << b);
    return true;
  }
  __device__ __forceinline__ void note_issue(int c) { inflight |= 1u << (c & 1); }
  __device__ __forceinline__ void begin(const double *column, int lane) {
    src = column;
    cur = -1;
    nchunks = (nz + ZC - 1) / ZC;
    __syncwarp();
    if (lane == 0) issue(0);
    note_issue(0);
  }
  __device__ __forceinline__ SharedRec at(int z) {
    const int c = z / ZC;
    if (c != cur) { /* c == cur + 1 */
      __syncwarp();
      if (!failed && c + 1 < nchunks) {
        if ((threadIdx.x & 31) == 0) issue(c + 1);
        note_issue(c + 1);
      }
      if (!failed && !wait(c & 1)) failed = true;
      cur = c;
    }
    return SharedRec{buf + (c & 1) * (ZC * NF) + (z - c * ZC) * NF};
  }
};

/* What one (column, wavelength) item needs besides its records, as an accessor read on
 * demand (kernel parameters and descriptors stay in their state spaces instead of registers).
 * Block kernels: column cl of the chunk, wavelength iw. */
struct BlockItem {
  const SolveArgs &a;
  int64_t cl;
  int w;
  __device__ __forceinline__ int64_t idx() const {
    return (a.layout == 0) ? (int64_t)w * a.ld_col + a.c_off + cl : (a.c_off + cl) * a.nw + w;
  }
  __device__ __forceinline__ int64_t pidx() const { return (int64_t)w * a.ld_col + a.c_off + cl; }
  __device__ __forceinline__ const double *lam() const { return a.lam; }
  __device__ __forceinline__ int nz() const { return a.nz; }
  __device__ __forceinline__ int nw() const { return a.nw; }
  __device__ __forceinline__ int iw() const { return w; }
  __device__ __forceinline__ double dz() const { return a.dz; }
  __device__ __forceinline__ double dz2() const { return a.dz2; }
  __device__ __forceinline__ double dz1() const { return a.dz1; }
  __device__ __forceinline__ double sigma_grey() const { return a.sigma_grey; }
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
  __device__ __forceinline__ unsigned long long id() const {
    return (unsigned long long)((a.c_off + cl) * a.nw + w);
  }
};

/* Generic path: warp tasks are 32 consecutive items of the flattened (column, lambda) index. */
template <int FORM, bool GREY>
__global__ void __launch_bounds__(128) k_solve(const SolveArgs a) {
  const int lane = threadIdx.x & 31;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nitems = a.ncol * a.nw;
  const unsigned long long ntasks = (unsigned long long)((nitems + 31) / 32);
  const int64_t wbase = slot * 32 * (int64_t)a.nz + lane; /* each warp's scratch [z][lane], contiguous */
  double *gam = a.gam + wbase;
  double *uu = a.uu + wbase;
  double *o1 = a.o1 + wbase;
  double *qs = a.q + wbase;
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(a.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int64_t item = (int64_t)task * 32 + lane;
    if (item < nitems) {
      const int64_t cl = item / a.nw;
      const int iw = (int)(item - cl * a.nw);
      DirectPillars pa{a.pil + cl * (int64_t)a.nz * NF};
      solve_item<FORM, GREY>(BlockItem{a, cl, iw}, true, pa, gam, uu, o1, qs);
    }
  }
}

/* Staged path: warp tasks are (column, tile of 32 wavelengths); the column's pillar records
 * are streamed into shared memory by bulk copies (see StagedPillars). */
template <int FORM, bool GREY>
__global__ void __launch_bounds__(128, 4) k_solve_staged(const SolveArgs a) {
  __shared__ __align__(128) double s_pil[WARPS_PER_BLOCK][2 * ZC * NF];
  __shared__ __align__(16) double s_lam[WARPS_PER_BLOCK][NLF * 32]; /* the task's 32 wavelengths' constants */
  __shared__ __align__(8) unsigned long long s_bar[WARPS_PER_BLOCK][2];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int ntiles = (a.nw + 31) / 32;
  const unsigned long long ntasks = (unsigned long long)a.ncol * ntiles;
  const int64_t wbase = slot * 32 * (int64_t)a.nz + lane; /* each warp's scratch [z][lane], contiguous */
  double *gam = a.gam + wbase;
  double *uu = a.uu + wbase;
  double *o1 = a.o1 + wbase;
  double *qs = a.q + wbase;
  StagedPillars pa;
  pa.buf = s_pil[wib];
  pa.bar0 = smem_addr(&s_bar[wib][0]);
  pa.nz = a.nz;
  pa.waits = 0;
  pa.inflight = 0;
  pa.failed = false;
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(a.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= ntasks) break;
    const int64_t cl = (int64_t)(task / ntiles);
    const int tile = (int)(task - (unsigned long long)cl * ntiles);
    const int iw_raw = tile * 32 + lane;
    const bool active = iw_raw < a.nw;
    const int iw = active ? iw_raw : a.nw - 1;
    pa.begin(a.pil + cl * (int64_t)a.nz * NF, lane);
    if (!GREY) store_lam_shared(&s_lam[wib][lane], a.lam, iw, a.nw);
    __syncwarp();
    solve_item<FORM, GREY, BlockItem, StagedPillars, LamS>(BlockItem{a, cl, iw}, active, pa, gam, uu, o1, qs,
                                                          &s_lam[wib][lane]);
    if (__any_sync(0xffffffffu, pa.failed)) {
      if (lane == 0) atomicOr(&a.status[2], 1ull);
      /* let copies still in flight land (bounded) before the block's shared memory is released */
      pa.wait(0);
      pa.wait(1);
      return;
    }
  }
}

/* ---- ragged batches (FP64 forms) -------------------------------------------------------- */
/* Item of a batch: wavelength w of column *c (descriptor read through the read-only cache). */
struct BatchItem {
  const FP64BatchArgs &b;
  const MBatchCol *c;
  int64_t col;
  int w;
  __device__ __forceinline__ int nz() const { return __ldg(&c->nz); }
  __device__ __forceinline__ int nw() const { return __ldg(&c->nw); }
  __device__ __forceinline__ int iw() const { return w; }
  __device__ __forceinline__ const double *lam() const { return b.lam + __ldg(&c->lam_off); }
  __device__ __forceinline__ double dz() const { return __ldg(&c->dz); }
  __device__ __forceinline__ double dz2() const { return __ldg(&c->dz2); }
  __device__ __forceinline__ double dz1() const { return __ldg(&c->dz1); }
  __device__ __forceinline__ double sigma_grey() const { return 0.0; }
  __device__ __forceinline__ int64_t zoff(int64_t base, int rows) const { /* element z = 0 */
    return b.layout == 0 ? base + (int64_t)w * rows : base + w;
  }
  __device__ __forceinline__ double *U() const { return b.U ? b.U + zoff(__ldg(&c->u_off), nz() + 6) : nullptr; }
  __device__ __forceinline__ double *K() const { return b.K ? b.K + zoff(__ldg(&c->kv_off), nz()) : nullptr; }
  __device__ __forceinline__ double *V() const { return b.V ? b.V + zoff(__ldg(&c->kv_off), nz()) : nullptr; }
  __device__ __forceinline__ int64_t uz() const { return b.layout == 0 ? 1 : nw(); }
  __device__ __forceinline__ int64_t kz() const { return uz(); }
  __device__ __forceinline__ int64_t vz() const { return uz(); }
  __device__ __forceinline__ double *vtop() const { return b.Vtop ? b.Vtop + __ldg(&c->flux_off) + w : nullptr; }
  __device__ __forceinline__ double *vbot() const { return b.Vbot ? b.Vbot + __ldg(&c->flux_off) + w : nullptr; }
  __device__ __forceinline__ int64_t ss() const { return 32; }
  __device__ __forceinline__ unsigned long long *status() const { return b.status; }
  __device__ __forceinline__ unsigned long long id() const { return ((unsigned long long)col << 32) | (unsigned)w; }
};

/* Warp-column tiling: tasks (column, 32-wavelength tile) from the device queue, longest
 * columns first; the column's records stream through the warp's shared-memory buffers and
 * the tile's wavelength constants sit in the warp's shared-memory table (as k_solve_staged). */
template <int FORM>
__global__ void __launch_bounds__(128, 4) k_batch_fp64_staged(const FP64BatchArgs b) {
  __shared__ __align__(128) double s_pil[WARPS_PER_BLOCK][2 * ZC * NF];
  __shared__ __align__(16) double s_lam[WARPS_PER_BLOCK][NLF * 32]; /* the task's 32 wavelengths' constants */
  __shared__ __align__(8) unsigned long long s_bar[WARPS_PER_BLOCK][2];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t slot = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t wbase = slot * 32 * (int64_t)b.max_nz + lane; /* each warp's scratch [z][lane], contiguous */
  double *gam = b.gam + wbase;
  double *uu = b.uu + wbase;
  double *o1 = b.o1 + wbase;
  double *qs = b.q + wbase;
  StagedPillars pa;
  pa.buf = s_pil[wib];
  pa.bar0 = smem_addr(&s_bar[wib][0]);
  pa.waits = 0;
  pa.inflight = 0;
  pa.failed = false;
  if (lane == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pa.bar0 + 8u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  for (;;) {
    unsigned long long task = 0;
    if (lane == 0) task = atomicAdd(b.work, 1ull);
    task = __shfl_sync(0xffffffffu, task, 0);
    if (task >= (unsigned long long)b.ntasks) break;
    const uint2 t = b.tasks[task];
    const MBatchCol *c = b.cols + t.x;
    const int nw = __ldg(&c->nw);
    const int iw_raw = (int)t.y * 32 + lane;
    const bool active = iw_raw < nw;
    const int iw = active ? iw_raw : nw - 1;
    pa.nz = __ldg(&c->nz);
    pa.begin(b.pil + __ldg(&c->rec_off) * NF, lane);
    store_lam_shared(&s_lam[wib][lane], b.lam + __ldg(&c->lam_off), iw, nw);
    __syncwarp();
    solve_item<FORM, false, BatchItem, StagedPillars, LamS>(BatchItem{b, c, (int64_t)t.x, iw}, active, pa, gam, uu, o1,
                                                           qs, &s_lam[wib][lane]);
    if (__any_sync(0xffffffffu, pa.failed)) {
      if (lane == 0) atomicOr(&b.status[2], 1ull);
      pa.wait(0);
      pa.wait(1);
      return;
    }
  }
}

cudaError_t launch_pillars_batch(const double *rho, const double *T, const MBatchCol *cols, const int64_t *rec_pre,
                                 int64_t ncol, int64_t nrec, double fully_ionized_T, double *pil, cudaStream_t s) {
  if (nrec == 0) return cudaSuccess;
  k_pillars_batch<<<(unsigned)((nrec + PIL_THREADS - 1) / PIL_THREADS), PIL_THREADS, 0, s>>>(
      rho, T, cols, rec_pre, ncol, nrec, fully_ionized_T, pil);
  return cudaGetLastError();
}

cudaError_t launch_batch_fp64(const FP64BatchArgs &a, int form, int blocks, int threads, cudaStream_t s) {
  if (form == 0)
    k_batch_fp64_staged<0><<<blocks, threads, 0, s>>>(a);
  else
    k_batch_fp64_staged<1><<<blocks, threads, 0, s>>>(a);
  return cudaGetLastError();
}

int batch_fp64_max_blocks_per_sm(int form, int threads) {
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &n, form == 0 ? (const void *)k_batch_fp64_staged<0> : (const void *)k_batch_fp64_staged<1>, threads, 0);
  return (e == cudaSuccess && n > 0) ? n : 1;
}

cudaError_t launch_pillars(const double *rho, const double *T, int64_t ncol, int nz,
                           double fully_ionized_T, int grey, double *pil, cudaStream_t s) {
  int64_t n = ncol * nz;
  if (n == 0) return cudaSuccess;
  const int64_t blocks = (n + PIL_THREADS - 1) / PIL_THREADS;
  k_pillars<<<(unsigned)blocks, PIL_THREADS, 0, s>>>(rho, T, n, fully_ionized_T, grey, pil);
  return cudaGetLastError();
}

bool solve_uses_staging(int nw) { return nw >= 64 || (nw % 32) == 0; }

static const void *solve_fn(int form, int grey, bool staged) {
  if (staged) {
    if (form == 0) return grey ? (const void *)k_solve_staged<0, true> : (const void *)k_solve_staged<0, false>;
    return grey ? (const void *)k_solve_staged<1, true> : (const void *)k_solve_staged<1, false>;
  }
  if (form == 0) return grey ? (const void *)k_solve<0, true> : (const void *)k_solve<0, false>;
  return grey ? (const void *)k_solve<1, true> : (const void *)k_solve<1, false>;
}

int solve_fp64_max_blocks_per_sm(int form, int grey, int threads) {
  int nb = 0, nb2 = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, solve_fn(form, grey, false), threads, 0) != cudaSuccess)
    nb = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb2, solve_fn(form, grey, true), threads, 0) != cudaSuccess)
    nb2 = 1;
  nb = nb > nb2 ? nb : nb2;
  return nb > 0 ? nb : 1;
}

/* Diagnostic: the staged kernels' bounded mbarrier wait, on a barrier phase that no copy or
 * arrival completes, so the wait runs out after `limit` polls and the timeout is reported in
 * status[2] as the solve kernels report it.  Nothing is in flight when the block exits. */
__global__ void k_bounded_wait_check(long long limit, unsigned long long *status) {
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t b = smem_addr(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  long long spins = 0;
  bool done = true;
  while (!mbar_try_wait(b, 0u))
    if (++spins > limit) {
      done = false;
      break;
    }
  if (__any_sync(0xffffffffu, !done) && threadIdx.x == 0) atomicOr(&status[2], 1ull);
}

cudaError_t launch_bounded_wait_check(long long limit, unsigned long long *status, cudaStream_t s) {
  k_bounded_wait_check<<<1, 32, 0, s>>>(limit, status);
  return cudaGetLastError();
}

cudaError_t launch_solve_fp64(const SolveArgs &a, int form, int grey, int blocks, int threads, cudaStream_t s) {
  const bool staged = !grey && solve_uses_staging(a.nw);
  void *args[] = {(void *)&a};
  return cudaLaunchKernel(solve_fn(form, grey, staged), dim3(blocks), dim3(threads), args, 0, s);
}

}  // namespace oco
