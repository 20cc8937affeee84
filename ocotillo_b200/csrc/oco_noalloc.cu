/*
 * oco_noalloc.cu -- oco_solve_block_noalloc: the device-array block solve for callers that
 * cannot allocate GPU memory.
 *
 * Who needs it: code that runs where cudaMalloc is not allowed or not wanted -- inside an
 * allocator-free host application (a Fortran driver linked against a runtime that owns the
 * device heap), a plugin whose host forbids device allocation after start-up, or a caller
 * that budgets GPU memory up front and must not see a call grow it.  The regular entry
 * points allocate their workspace (pillars, Thomas scratch, wavelength table) on first use;
 * this one uses a fixed workspace compiled into the library instead.
 *
 * The workspace is the file-scope array g_noalloc_ws below (OCO_NOALLOC_WORKSPACE_BYTES,
 * 32 MiB): every GPU that loads the library holds it until the process exits.  Host code
 * cannot use the array's name as a device address; the first call on each device, with that
 * device current, asks the runtime for the address (cudaGetSymbolAddress) and caches it.
 * That first call should therefore come before any stream capture.
 *
 * All calls on a device share its workspace, which keeps the previous call's contents: the
 * work counter and the status words are cleared at the start of every call, everything else
 * is fully rewritten before it is read.  Calls whose GPU work overlapped would race on it, so
 * each call holds a lock of its device until its work on the stream is done (calls on
 * different devices run in parallel), and a call that fails after enqueueing work waits for
 * that work before it returns.
 *
 * Sizes: the scratch takes at most half of the workspace left after the wavelength table,
 * and always at least one 128-thread block, which together with one column of pillar
 * records fits every nz <= OCO_NOALLOC_MAX_NZ at nw <= OCO_NOALLOC_MAX_NW (checked at compile
 * time below); columns beyond what the rest holds are solved in further chunks.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/oco.h"
#include "oco_internal.h"

using namespace oco;

static __device__ __align__(256) unsigned char g_noalloc_ws[OCO_NOALLOC_WORKSPACE_BYTES];

namespace {

const int kMaxDevices = 64;
const int kThreads = 128;

/* The workspace is per device, so calls on different devices do not serialise: one mutex per
 * device guards its copy of g_noalloc_ws for the whole call; the host staging table (one, shared)
 * is guarded only while it is filled and copied out. */
std::mutex g_dev_mu[kMaxDevices];
std::mutex g_table_mu;
std::mutex g_addr_mu;
void *g_ws_addr[kMaxDevices];                       /* device address of g_noalloc_ws, per device */
double g_host_table[NL * OCO_NOALLOC_MAX_NW];       /* host staging of the wavelength table */
thread_local char g_msg[512];

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof g_msg, fmt, ap);
  va_end(ap);
  return code;
}

#define CUN(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(OCO_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

constexpr size_t round256(size_t n) { return (n + 255) & ~(size_t)255; }

/* Bytes of one 128-thread block of Thomas scratch (gamma, u, 1/kappa, q: 4 doubles per z per
 * thread) and of one column of pillar records. */
constexpr size_t scratch_block_bytes(size_t nz) { return nz * 4 * sizeof(double) * kThreads; }
constexpr size_t pillar_column_bytes(size_t nz) { return nz * NF * sizeof(double); }

/* The documented limits always fit: counters, the largest wavelength table, one block of
 * scratch and one column of pillars at nz = OCO_NOALLOC_MAX_NZ. */
static_assert(256 + round256((size_t)NL * OCO_NOALLOC_MAX_NW * sizeof(double)) +
                      round256(scratch_block_bytes(OCO_NOALLOC_MAX_NZ)) + pillar_column_bytes(OCO_NOALLOC_MAX_NZ) <=
                  OCO_NOALLOC_WORKSPACE_BYTES,
              "OCO_NOALLOC_MAX_NZ / OCO_NOALLOC_MAX_NW do not fit the static workspace");

}  // namespace

extern "C" const char *oco_noalloc_last_error(void) { return g_msg; }

extern "C" int oco_solve_block_noalloc(const oco_params *p, const double *wa_angstrom, const double *rho,
                                       const double *T, double *U, double *kappa, double *V, double *Vtop,
                                       double *Vbot, void *stream) {
  g_msg[0] = 0;
  if (!p || !rho || !T) return fail(OCO_EINVAL, "params, rho and T are required");
  if (p->nx < 1 || p->ny < 1 || p->nz < 2 || p->nw < 1)
    return fail(OCO_EINVAL, "bad dimensions nx=%d ny=%d nz=%d nw=%d (need nz >= 2)", p->nx, p->ny, p->nz, p->nw);
  if (p->lgrey && p->nw != 1) return fail(OCO_EGREY, "For Grey RT use only one wavelength");
  if (p->form != OCO_FORM_PLAIN && p->form != OCO_FORM_STABLE)
    return fail(OCO_EINVAL, "oco_solve_block_noalloc supports the plain and stable FP64 forms only");
  if (p->layout != OCO_LAYOUT_REFERENCE && p->layout != OCO_LAYOUT_LAMBDA_FASTEST)
    return fail(OCO_EINVAL, "unknown layout %d", p->layout);
  if (!(p->dz > 0.0) || !std::isfinite(p->dz)) return fail(OCO_EINVAL, "dz must be positive and finite");
  if (!block_elements_fit(p->nx, p->ny, p->nz, p->nw))
    return fail(OCO_EINVAL, "block too large: nx*ny*nw*(nz+6) exceeds 2^56 elements");
  if (!p->lgrey && !wa_angstrom) return fail(OCO_ENOWAVES, "wavelengths are required");
  if (p->nz > OCO_NOALLOC_MAX_NZ || p->nw > OCO_NOALLOC_MAX_NW)
    return fail(OCO_EINVAL, "oco_solve_block_noalloc: nz=%d nw=%d exceed the static workspace limits nz <= %d, nw <= %d",
                p->nz, p->nw, OCO_NOALLOC_MAX_NZ, OCO_NOALLOC_MAX_NW);
  if (!p->lgrey)
    for (int i = 0; i < p->nw; i++)
      if (!(wa_angstrom[i] > 0.0) || !std::isfinite(wa_angstrom[i]))
        return fail(OCO_EINVAL, "wavelength %d is not positive and finite", i);
  const int grey = p->lgrey ? 1 : 0;
  const int nz = p->nz, nw = p->nw;
  cudaStream_t s = (cudaStream_t)stream;

  int dev = 0;
  CUN(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(OCO_EINVAL, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_dev_mu[dev]);
  {
    std::lock_guard<std::mutex> al(g_addr_mu);
    if (!g_ws_addr[dev]) { /* once per device, with that device current */
      void *ptr = nullptr;
      CUN(cudaGetSymbolAddress(&ptr, g_noalloc_ws));
      g_ws_addr[dev] = ptr;
    }
  }
  unsigned char *ws = (unsigned char *)g_ws_addr[dev];

  /* workspace layout: [counters 256 B][wavelength table][Thomas scratch][pillars].  The scratch
   * takes at most half of what the table leaves, but always at least one block, which with one
   * column of pillars fits up to OCO_NOALLOC_MAX_NZ (static_assert above). */
  const size_t tab_bytes = grey ? 0 : round256((size_t)NL * nw * sizeof(double));
  const size_t avail = OCO_NOALLOC_WORKSPACE_BYTES - 256 - tab_bytes;
  int nsm = 0, bps = solve_fp64_max_blocks_per_sm(p->form == OCO_FORM_STABLE ? 1 : 0, grey, kThreads);
  CUN(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t per_block = scratch_block_bytes((size_t)nz), per_col = pillar_column_bytes((size_t)nz);
  const int64_t ncol = (int64_t)p->nx * p->ny;
  const int64_t need_blocks = (ncol * nw + kThreads - 1) / kThreads;
  const int64_t half_blocks = (int64_t)(avail / 2 / per_block);
  int64_t blocks = std::min<int64_t>({(int64_t)nsm * bps, need_blocks, std::max<int64_t>(half_blocks, 1)});
  const size_t scratch_bytes = round256((size_t)blocks * per_block);
  if (scratch_bytes + per_col > avail) return fail(OCO_EINVAL, "nz=%d does not fit the static workspace", nz);
  const int64_t chunk = std::min<int64_t>(ncol, (int64_t)((avail - scratch_bytes) / per_col));

  unsigned long long *ctr = (unsigned long long *)ws; /* [0] work, [1] zero-pivot count, [2] first bad item, [3] timeout */
  double *lam = (double *)(ws + 256);
  double *scr = (double *)(ws + 256 + tab_bytes);
  double *pil = (double *)(ws + 256 + tab_bytes + scratch_bytes);

  /* From the first enqueued operation on, an error return first waits for what was queued, so
   * that no kernel of this call still uses the workspace when the device lock is released. */
  auto drained = [&](int rc) {
    if (rc != OCO_OK) cudaStreamSynchronize(s);
    return rc;
  };
  if (!grey) { /* stage the table; a pageable-source copy has consumed the buffer when it returns */
    std::lock_guard<std::mutex> tl(g_table_mu);
    fill_lambda_table(wa_angstrom, nw, g_host_table);
    CUN(cudaMemcpyAsync(lam, g_host_table, (size_t)NL * nw * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  const int rc = drained([&]() -> int {
    CUN(cudaMemsetAsync(ctr + 1, 0, sizeof(unsigned long long), s));
    CUN(cudaMemsetAsync(ctr + 2, 0xff, sizeof(unsigned long long), s));
    CUN(cudaMemsetAsync(ctr + 3, 0, sizeof(unsigned long long), s));

    SolveArgs a{};
    a.nz = nz;
    a.nw = nw;
    a.dz = p->dz;
    a.dz1 = 1.0 / p->dz;
    a.dz2 = p->dz * p->dz;
    a.sigma_grey = p->sigma_grey;
    a.layout = p->layout;
    a.ld_col = ncol;
    const int64_t mz = nz + 6;
    if (p->layout == OCO_LAYOUT_REFERENCE) {
      a.U_zs = 1, a.U_is = mz, a.K_zs = 1, a.K_is = nz, a.V_zs = 1, a.V_is = nz;
    } else {
      const int64_t items = ncol * nw;
      a.U_zs = items, a.U_is = 1, a.K_zs = items, a.K_is = 1, a.V_zs = items, a.V_is = 1;
    }
    a.U = U, a.K = kappa, a.V = V, a.Vtop = Vtop, a.Vbot = Vbot;
    a.pil = pil;
    a.lam = grey ? nullptr : lam;
    const size_t slots = (size_t)blocks * kThreads;
    a.gam = scr;
    a.uu = scr + slots * nz;
    a.o1 = scr + 2 * slots * nz;
    a.q = scr + 3 * slots * nz;
    a.slot_stride = (int64_t)slots;
    a.work = ctr;
    a.status = ctr + 1;
    for (int64_t c0 = 0; c0 < ncol; c0 += chunk) {
      const int64_t nb = std::min(chunk, ncol - c0);
      a.ncol = nb;
      a.c_off = c0;
      CUN(launch_pillars(rho + c0 * nz, T + c0 * nz, nb, nz, p->fully_ionized_T, grey, pil, s));
      CUN(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), s));
      const int64_t nblk = std::min<int64_t>(blocks, (nb * nw + kThreads - 1) / kThreads);
      CUN(launch_solve_fp64(a, p->form == OCO_FORM_STABLE ? 1 : 0, grey, (int)nblk, kThreads, s));
    }
    return OCO_OK;
  }());
  if (rc != OCO_OK) return rc;
  unsigned long long st[3] = {0, 0, 0};
  const cudaError_t ce = cudaMemcpyAsync(st, ctr + 1, sizeof st, cudaMemcpyDeviceToHost, s);
  const cudaError_t se = cudaStreamSynchronize(s); /* also when the copy failed: drains the call's work */
  if (ce != cudaSuccess || se != cudaSuccess)
    return fail(OCO_ECUDA, "status read-back: %s", cudaGetErrorString(ce != cudaSuccess ? ce : se));
  if (st[2]) return fail(OCO_ETIMEDOUT, "a bounded wait for a pillar copy ran out; results are incomplete");
  if (st[0]) {
    long long col = (long long)(st[1] / (unsigned long long)nw), iw = (long long)(st[1] % nw);
    return fail(OCO_EZEROPIVOT, "ERROR tridiag: bet == 0 in %llu items; first: ix=%lld iy=%lld iw=%lld", st[0],
                col / p->ny + 1, col % p->ny + 1, iw + 1);
  }
  return OCO_OK;
}
