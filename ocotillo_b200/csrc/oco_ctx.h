/*
 * oco_ctx.h -- the context behind the C ABI's opaque oco_ctx (internal to the library):
 * device buffers, streams, wavelength tables, workspace and error reporting, shared by the
 * block solve (oco_api.cu), the ragged batch (oco_batch.cu) and the serving loop
 * (oco_server.cu).
 */
#ifndef OCO_CTX_H
#define OCO_CTX_H

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/oco.h"

struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T *as() const {
    return (T *)p;
  }
};

/* Per-chunk staging for the host-array path (two sets, used alternately). */
struct Stage {
  DevBuf rho, T, U, K, V, top, bot;
  cudaEvent_t done = nullptr; /* copy-back of this set finished */
};

struct oco_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr; /* kernels */
  cudaStream_t copy = nullptr;   /* host<->device copies of the host-array path */
  std::string err;
  /* wavelength tables (FP64 and the mixed form's FP32 log table) */
  int nw = 0;
  std::vector<double> wa;
  DevBuf lam, lam32;
  DevBuf trapw; /* trapezoid weights of the wavelength grid, cm (oco_integrated_flux_device) */
  /* workspace */
  DevBuf pil, scratch, work, status;
  /* mixed form: a chunk's flag words (one bit per item) with each flagged item's slot beside its
   * bit, the lists of words holding flags and of flagged items, column marks, and counters ([0] items re-solved since the last
   * oco_mixed_repairs, [1] words and [2] items listed in the current chunk) */
  DevBuf rbits, rslot, stats, colflag, rlist, ilist;
  float repair_cond = 100.0f; /* oco_set_mixed_repair */
  int64_t repair_slots_max = -1; /* OCO_REPAIR_SLOTS: caps the re-solve's slots (the rest go one warp per item) */
  Stage stage[2];
  int64_t launches = 0;
  size_t budget_bytes = 8ull << 30; /* chunk budget for pillars + staged outputs */
  int max_blocks = 0;               /* cap on the persistent grid (0: occupancy limit x SMs) */
  /* reference-layout device outputs: solve into lambda-fastest temporaries and transpose
   * (true), or store directly from the solve kernel (OCO_REFERENCE_STORES=direct) */
  bool ref_transpose = true;
  DevBuf tmpU, tmpK, tmpV;
  /* kernel timing (oco_set_profiling) */
  bool prof = false;
  /* device-array calls defer the zero-pivot check to oco_synchronize */
  bool status_pending = false;
  cudaStream_t status_stream = nullptr;
  oco_params status_params{};  /* the first pending call's, which locate the first bad item */
  bool status_dims_mixed = false; /* pending calls of different nx, ny or nw: no location */
  cudaEvent_t order_ev = nullptr; /* orders a device call on another stream after the pending one */
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_solve, ev_pil;
  cudaEvent_t take_event() {
    if (!ev_pool.empty()) {
      cudaEvent_t e = ev_pool.back();
      ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
};

/* Enqueues columns [c0, c0 + nb) of a block on stream s: the record kernel and the persistent
 * solve, with the solve grid capped at max_blocks (0: no cap).  Outputs (device arrays of the
 * whole block, layout p->layout; any may be NULL) are written for those columns only.  Zero
 * pivots and timeouts accumulate in the context's status until oco_ctx_read_status. */
int oco_ctx_run_columns(oco_ctx *c, const oco_params *p, const double *rho, const double *T, int64_t c0, int64_t nb,
                        double *U, double *kappa, double *V, double *Vtop, double *Vbot, int max_blocks,
                        cudaStream_t s);
/* Clears the context's status (zero-pivot count, first bad item, timeout flag) on stream s. */
int oco_ctx_reset_status(oco_ctx *c, cudaStream_t s);
/* Reads the status after the work on s: OCO_OK, OCO_EZEROPIVOT or OCO_ETIMEDOUT. */
int oco_ctx_read_status(oco_ctx *c, cudaStream_t s, const oco_params *p);
/* Validates p and the context's wavelength table for it (OCO_OK or an error code). */
int oco_ctx_check_params(oco_ctx *c, const oco_params *p);
/* Full device-resident persistent grid of a form (blocks). */
int oco_ctx_full_blocks(oco_ctx *c, int form, int grey);
/* The mixed re-solve's slots: a scratch capacity, capped by the context's OCO_REPAIR_SLOTS (the
 * environment variable read at creation; rounded down to a multiple of 32).  Items beyond the
 * slots are re-solved one warp per item; the cap lets tests reach that path. */
int64_t oco_ctx_repair_slots(const oco_ctx *c, int64_t cap);

/* Records a message for oco_last_error (on the context, if any, and the calling thread) and
 * returns code. */
int oco_set_err(oco_ctx *c, int code, const char *fmt, ...);

/* Returns the mapped error code from the enclosing function when a CUDA call fails; needs a
 * variable c (oco_ctx *, may be NULL) in scope. */
#define CU(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return oco_set_err(c, e_ == cudaErrorMemoryAllocation ? OCO_ENOMEM : OCO_ECUDA,        \
                         "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

#endif
