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
  /* workspace */
  DevBuf pil, scratch, work, status;
  Stage stage[2];
  int64_t launches = 0;
  size_t budget_bytes = 8ull << 30; /* chunk budget for pillars + staged outputs */
  /* kernel timing (oco_set_profiling) */
  bool prof = false;
  /* device-array calls defer the zero-pivot check to oco_synchronize */
  bool status_pending = false;
  cudaStream_t status_stream = nullptr;
  oco_params status_params{};
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
