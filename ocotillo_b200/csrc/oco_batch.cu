/*
 * oco_batch.cu -- ragged batches (include/oco.h, "Ragged batches"): many independent columns
 * of different nz, dz and wavelength grids in one persistent launch, replayed as a CUDA graph.
 *
 * Work queue.  The kernels pull warp tasks from one device counter.  Tasks are ordered
 * longest column first, so the short columns fill the tail of the launch (a greedy
 * longest-processing-time schedule over the resident warps).  Two tilings:
 *   OCO_TILING_WARP_COLUMN  task = (column, 32-wavelength tile); the column's records stream
 *                           into the warp's shared memory (bulk copies); lanes past the
 *                           column's nw idle;
 *   OCO_TILING_PACKED       task = 32 consecutive (column, wavelength) items of the list of
 *                           columns sorted by nz; no idle lanes, records read through L1.
 * The autotuner (oco_batch_tune) times every (tiling, resident blocks per SM) candidate on
 * the bound arrays and keeps the fastest.
 *
 * The FP64 forms (plain, stable) run the warp-column tiling only, with the FP64 records and
 * the block solve's per-item arithmetic (bit-identical to it, and so to the oracle).
 *
 * Graph.  oco_batch_bind captures: counter reset, status reset, the record kernel over all
 * columns' z values, the solve kernel.  oco_batch_run replays it on the caller's stream.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <new>
#include <numeric>
#include <utility>
#include <vector>

#include "../../include/oco.h"
#include "batch_layout.h"
#include "mixed_core.h"
#include "oco_ctx.h"
#include "oco_internal.h"

using namespace oco;

static const int kBatchThreads = 128;

struct oco_batch {
  oco_ctx *c = nullptr;
  int form = OCO_FORM_MIXED;
  int layout = OCO_LAYOUT_LAMBDA_FASTEST;
  double fully_ionized_T = 2e4;
  int64_t ncol = 0, npoints = 0, nrec = 0, nitems = 0, ntasks_tile = 0, ntasks_packed = 0;
  int max_nz = 0, max_nw = 0;
  int64_t need_in = 0, need_u = 0, need_kv = 0, need_flux = 0; /* element counts the arrays must hold */
  /* first pair of columns whose output ranges overlap, per array family (U; kappa and V;
     Vtop and Vbot), {-1, -1} if none: binding an array of an overlapping family fails */
  int64_t overlap[3][2] = {{-1, -1}, {-1, -1}, {-1, -1}};
  DevBuf cols, rec_pre, tasks, order, item_pre, lam, rec, scratch, work, status;
  DevBuf lam64, colflag, rbits, rslot, rlist, ilist; /* mixed form: FP64 tables, column marks, flag words, slots, listed words and items of the re-solve */
  int64_t slots = 0; /* scratch slots (threads of the largest persistent grid) */
  int tiling = OCO_TILING_WARP_COLUMN, bps = 1, max_bps[2] = {1, 1}; /* max_bps 0: tiling not available */
  /* bound arrays */
  bool bound = false;
  const double *rho = nullptr, *T = nullptr;
  double *U = nullptr, *K = nullptr, *V = nullptr, *Vtop = nullptr, *Vbot = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t last = nullptr;
  bool pending = false;
  cudaEvent_t after_last = nullptr; /* orders a replay on another stream after the pending one */
  oco_batch_info info{};
};

static MixedBatchArgs batch_args(const oco_batch *b) {
  MixedBatchArgs a{};
  a.rec = b->rec.as<float>();
  a.lam = b->lam.as<float>();
  a.cols = b->cols.as<MBatchCol>();
  a.tasks = b->tasks.as<uint2>();
  a.order = b->order.as<int32_t>();
  a.item_pre = b->item_pre.as<int64_t>();
  a.ncol = b->ncol;
  a.ntasks = b->tiling == OCO_TILING_PACKED ? b->ntasks_packed : b->ntasks_tile;
  a.nitems = b->nitems;
  a.U = b->U;
  a.K = b->K;
  a.V = b->V;
  a.Vtop = b->Vtop;
  a.Vbot = b->Vbot;
  a.layout = b->layout;
  a.s4 = b->scratch.as<float4>();
  a.slot_stride = b->slots;
  a.max_nz = b->max_nz;
  a.work = b->work.as<unsigned long long>();
  a.status = b->status.as<unsigned long long>();
  a.repair_cond = b->c->repair_cond;
  a.colflag = b->colflag.as<unsigned>();
  a.rbits = b->rbits.as<unsigned>();
  a.rslot = b->rslot.as<int>();
  a.rwstride = (b->max_nw + 31) / 32;
  a.rlist = b->rlist.as<unsigned long long>();
  a.rcount = b->status.as<unsigned long long>() + 4;
  a.ilist = b->ilist.as<unsigned long long>();
  a.icount = b->status.as<unsigned long long>() + 5;
  return a;
}

/* The FP64 re-solve of the items the mixed batch kernel flags (stable form). */
static RepairArgs repair_args(const oco_batch *b) {
  RepairArgs r{};
  r.list = b->rlist.as<unsigned long long>();
  r.count = b->status.as<unsigned long long>() + 4;
  r.ilist = b->ilist.as<unsigned long long>();
  r.icount = b->status.as<unsigned long long>() + 5;
  r.bits = b->rbits.as<unsigned>();
  r.slot = b->rslot.as<int>();
  r.wstride = (b->max_nw + 31) / 32;
  r.block = 0;
  r.rho = b->rho;
  r.T = b->T;
  r.U = b->U, r.K = b->K, r.V = b->V, r.Vtop = b->Vtop, r.Vbot = b->Vbot;
  r.layout = b->layout;
  r.cols = b->cols.as<MBatchCol>();
  r.lam64 = b->lam64.as<double>();
  r.fully_ionized_T = b->fully_ionized_T;
  r.scratch = b->scratch.as<double>(); /* the mixed solve's */
  r.max_nz = b->max_nz;
  r.cap = oco_ctx_repair_slots(b->c, repair_capacity(b->scratch.n, b->max_nz, REPAIR_SOLVE_BLOCKS_PER_SM * b->c->num_sms));
  r.queue = b->status.as<unsigned long long>() + 6;
  r.repairs = b->c->stats.as<unsigned long long>();
  r.status = b->status.as<unsigned long long>();
  return r;
}

static FP64BatchArgs fp64_args(const oco_batch *b) {
  FP64BatchArgs a{};
  a.pil = b->rec.as<double>();
  a.lam = b->lam.as<double>();
  a.cols = b->cols.as<MBatchCol>();
  a.tasks = b->tasks.as<uint2>();
  a.ntasks = b->ntasks_tile;
  a.U = b->U;
  a.K = b->K;
  a.V = b->V;
  a.Vtop = b->Vtop;
  a.Vbot = b->Vbot;
  a.layout = b->layout;
  const size_t plane = (size_t)b->slots * b->max_nz;
  double *sc = b->scratch.as<double>();
  a.gam = sc;
  a.uu = sc + plane;
  a.o1 = sc + 2 * plane;
  a.q = sc + 3 * plane;
  a.slot_stride = b->slots;
  a.max_nz = b->max_nz;
  a.work = b->work.as<unsigned long long>();
  a.status = b->status.as<unsigned long long>();
  return a;
}

/* Enqueues one run (counter and status reset, records, solve) on s. */
static int enqueue_run(oco_batch *b, cudaStream_t s) {
  oco_ctx *c = b->c;
  CU(cudaMemsetAsync(b->work.p, 0, sizeof(unsigned long long), s));
  CU(cudaMemsetAsync(b->status.p, 0, 3 * sizeof(unsigned long long), s));
  CU(cudaMemsetAsync(b->status.as<unsigned long long>() + 1, 0xff, sizeof(unsigned long long), s)); /* atomicMin */
  const int blocks = b->bps * c->num_sms;
  if (b->form == OCO_FORM_MIXED) {
    CU(cudaMemsetAsync(b->colflag.p, 0, (size_t)b->ncol * sizeof(unsigned), s));
    CU(launch_pillars_mixed_batch(b->rho, b->T, b->cols.as<MBatchCol>(), b->rec_pre.as<int64_t>(), b->ncol, b->nrec,
                                  b->fully_ionized_T, b->rec.as<float>(), b->colflag.as<unsigned>(), s));
    const MixedBatchArgs a = batch_args(b);
    CU(cudaMemsetAsync(a.rcount, 0, 3 * sizeof(unsigned long long), s)); /* rcount, icount, the re-solve's queue */
    CU(cudaMemsetAsync(a.rbits, 0, (size_t)b->ncol * a.rwstride * sizeof(unsigned), s));
    CU(launch_batch_mixed(a, b->tiling == OCO_TILING_PACKED ? BATCH_TILING_PACKED : BATCH_TILING_WARP_COLUMN, blocks,
                          kBatchThreads, s));
    CU(launch_repair(repair_args(b), REPAIR_COEF_BLOCKS_PER_SM * c->num_sms, REPAIR_SOLVE_BLOCKS_PER_SM * c->num_sms, s));
  } else {
    CU(launch_pillars_batch(b->rho, b->T, b->cols.as<MBatchCol>(), b->rec_pre.as<int64_t>(), b->ncol, b->nrec,
                            b->fully_ionized_T, b->rec.as<double>(), s));
    CU(launch_batch_fp64(fp64_args(b), b->form == OCO_FORM_STABLE ? 1 : 0, blocks, kBatchThreads, s));
  }
  return OCO_OK;
}

static void drop_graph(oco_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

static int capture(oco_batch *b) {
  oco_ctx *c = b->c;
  drop_graph(b);
  CU(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_run(b, b->cap);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->cap, &g);
  if (rc != OCO_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  CU(e);
  b->graph = g;
  CU(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return OCO_OK;
}

/* Reads the last run's status: OCO_ETIMEDOUT, then (report_pivots, FP64 forms)
 * OCO_EZEROPIVOT. */
static int check_status(oco_batch *b, bool report_pivots = true) {
  oco_ctx *c = b->c;
  unsigned long long st[3];
  CU(cudaMemcpy(st, b->status.p, sizeof st, cudaMemcpyDeviceToHost));
  if (st[2]) return oco_set_err(c, OCO_ETIMEDOUT, "batch: a bounded wait for a record copy ran out; results are incomplete");
  if (report_pivots && b->form != OCO_FORM_MIXED && st[0])
    return oco_set_err(c, OCO_EZEROPIVOT,
                       "ERROR tridiag: bet == 0 in %llu (column, wavelength) items; first: column %llu, iw=%llu",
                       st[0], st[1] >> 32, (st[1] & 0xffffffffull) + 1);
  return OCO_OK;
}

static int batch_create(oco_ctx *c, const oco_batch_column *cols, int64_t ncol, const double *waves, int64_t nwaves,
                        int32_t form, int32_t layout, double fully_ionized_T, oco_batch **out) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_create: NULL context");
  if (!out) return oco_set_err(c, OCO_EINVAL, "oco_batch_create: out is NULL");
  *out = nullptr;
  if (form != OCO_FORM_MIXED && form != OCO_FORM_PLAIN && form != OCO_FORM_STABLE)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_create: bad form %d", form);
  if (layout != OCO_LAYOUT_REFERENCE && layout != OCO_LAYOUT_LAMBDA_FASTEST)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_create: bad layout %d", layout);
  if (!cols || ncol < 1 || ncol > (int64_t)INT32_MAX)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_create: need 1 <= ncol <= 2^31-1 column descriptors");
  if (!waves || nwaves < 1) return oco_set_err(c, OCO_EINVAL, "oco_batch_create: no wavelengths");
  if (!std::isfinite(fully_ionized_T)) return oco_set_err(c, OCO_EINVAL, "oco_batch_create: fully_ionized_T not finite");
  for (int64_t i = 0; i < nwaves; i++)
    if (!(waves[i] > 0.0) || !std::isfinite(waves[i]))
      return oco_set_err(c, OCO_EINVAL, "oco_batch_create: wavelength %lld is not positive", (long long)i);

  oco_batch *b = new (std::nothrow) oco_batch();
  if (!b) return oco_set_err(c, OCO_ENOMEM, "oco_batch_create: out of host memory");
  std::unique_ptr<oco_batch, void (*)(oco_batch *)> guard(b, oco_batch_destroy);
  b->c = c;
  b->form = form;
  b->layout = layout;
  b->fully_ionized_T = fully_ionized_T;
  b->ncol = ncol;

  /* descriptors, wavelength tables (one per distinct grid), record prefix sums */
  std::vector<MBatchCol> dc((size_t)ncol);
  std::vector<int64_t> rpre((size_t)ncol + 1, 0);
  std::map<std::pair<int64_t, int32_t>, int64_t> grids;
  const bool fp64 = form != OCO_FORM_MIXED;
  std::vector<float> lam;     /* mixed tables */
  std::vector<double> lam64;  /* FP64 tables */
  std::vector<double> tab;
  for (int64_t i = 0; i < ncol; i++) {
    const oco_batch_column &q = cols[i];
    const auto off_ok = [](int64_t o) { return o >= 0 && o <= kBatchMaxOffset; };
    if (q.nz < 2 || q.nw < 1 || !(q.dz > 0.0) || !std::isfinite(q.dz) || !off_ok(q.in_off) || !off_ok(q.u_off) ||
        !off_ok(q.kv_off) || !off_ok(q.flux_off) || q.wave_off < 0 || q.wave_off > nwaves - q.nw)
      return oco_set_err(c, OCO_EINVAL,
                         "oco_batch_create: column %lld: need nz >= 2, nw >= 1, dz > 0, 0 <= offsets <= 2^56 and "
                         "wave_off + nw <= nwaves",
                         (long long)i);
    auto key = std::make_pair(q.wave_off, q.nw);
    auto it = grids.find(key);
    int64_t loff;
    if (it == grids.end()) {
      tab.assign((size_t)NL * q.nw, 0.0);
      fill_lambda_table(waves + q.wave_off, q.nw, tab.data());
      if (fp64) {
        loff = (int64_t)lam64.size();
        lam64.insert(lam64.end(), tab.begin(), tab.end());
      } else { /* mixed tables; the FP64 ones follow in step (offset lam_off / MIXED_LN * NL) */
        loff = (int64_t)lam.size();
        lam.resize(lam.size() + (size_t)MIXED_LN * q.nw);
        fill_mixed_lambda_table(tab.data(), q.nw, lam.data() + loff);
        lam64.insert(lam64.end(), tab.begin(), tab.end());
      }
      grids.emplace(key, loff);
    } else {
      loff = it->second;
    }
    MBatchCol &d = dc[(size_t)i];
    d.in_off = q.in_off;
    d.rec_off = rpre[(size_t)i];
    d.u_off = q.u_off;
    d.kv_off = q.kv_off;
    d.flux_off = q.flux_off;
    d.lam_off = loff;
    d.nz = q.nz;
    d.nw = q.nw;
    d.dzf = (float)q.dz;
    mx::ldz2_split(q.dz, d.ldz2i, d.ldz2f);
    d.dz1 = 1.0 / q.dz;
    d.dz = q.dz;
    d.dz2 = q.dz * q.dz;
    rpre[(size_t)i + 1] = rpre[(size_t)i] + q.nz;
    b->npoints += (int64_t)q.nz * q.nw;
    b->nitems += q.nw;
    b->max_nz = std::max(b->max_nz, (int)q.nz);
    b->max_nw = std::max(b->max_nw, (int)q.nw);
    b->need_in = std::max(b->need_in, q.in_off + q.nz);
    b->need_u = std::max(b->need_u, q.u_off + (int64_t)(q.nz + 6) * q.nw);
    b->need_kv = std::max(b->need_kv, q.kv_off + (int64_t)q.nz * q.nw);
    b->need_flux = std::max(b->need_flux, q.flux_off + q.nw);
  }
  b->nrec = rpre[(size_t)ncol];
  if (!fp64 && b->nitems > INT32_MAX) /* the FP64 re-solve indexes flagged items with 32-bit slots */
    return oco_set_err(c, OCO_EINVAL, "oco_batch_create: a mixed batch holds at most 2^31-1 (column, wavelength) "
                       "items (got %lld)", (long long)b->nitems);
  {
    std::vector<int64_t> off((size_t)ncol), len((size_t)ncol);
    for (int f = 0; f < 3; f++) {
      for (int64_t i = 0; i < ncol; i++) {
        const oco_batch_column &q = cols[i];
        off[(size_t)i] = f == 0 ? q.u_off : f == 1 ? q.kv_off : q.flux_off;
        len[(size_t)i] = f == 0 ? (int64_t)(q.nz + 6) * q.nw : f == 1 ? (int64_t)q.nz * q.nw : q.nw;
      }
      const auto pr = first_overlap(off, len);
      b->overlap[f][0] = pr.first;
      b->overlap[f][1] = pr.second;
    }
  }

  /* work lists, longest column first */
  std::vector<int32_t> order((size_t)ncol);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return cols[x].nz > cols[y].nz; });
  std::vector<int64_t> ipre((size_t)ncol + 1, 0);
  std::vector<uint2> tasks;
  for (int64_t k = 0; k < ncol; k++) {
    const int32_t i = order[(size_t)k];
    ipre[(size_t)k + 1] = ipre[(size_t)k] + cols[i].nw;
    const int ntile = (cols[i].nw + 31) / 32;
    for (int t = 0; t < ntile; t++) tasks.push_back(make_uint2((unsigned)i, (unsigned)t));
  }
  b->ntasks_tile = (int64_t)tasks.size();
  b->ntasks_packed = (b->nitems + 31) / 32;

  /* device state */
  CU(cudaSetDevice(c->device));
  CU(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  if (fp64) {
    b->max_bps[0] = batch_fp64_max_blocks_per_sm(form == OCO_FORM_STABLE ? 1 : 0, kBatchThreads);
    b->max_bps[1] = 0;
  } else {
    b->max_bps[0] = batch_mixed_max_blocks_per_sm(BATCH_TILING_WARP_COLUMN, kBatchThreads);
    b->max_bps[1] = batch_mixed_max_blocks_per_sm(BATCH_TILING_PACKED, kBatchThreads);
  }
  b->slots = (int64_t)std::max(b->max_bps[0], b->max_bps[1]) * c->num_sms * kBatchThreads;
  b->tiling = OCO_TILING_WARP_COLUMN;
  b->bps = b->max_bps[0];
  CU(b->cols.ensure(dc.size() * sizeof(MBatchCol)));
  CU(b->rec_pre.ensure(rpre.size() * sizeof(int64_t)));
  CU(b->tasks.ensure(tasks.size() * sizeof(uint2)));
  CU(b->order.ensure(order.size() * sizeof(int32_t)));
  CU(b->item_pre.ensure(ipre.size() * sizeof(int64_t)));
  if (fp64) {
    CU(b->lam.ensure(lam64.size() * sizeof(double)));
    CU(b->rec.ensure((size_t)b->nrec * NF * sizeof(double)));
    CU(b->scratch.ensure((size_t)4 * b->slots * b->max_nz * sizeof(double)));
  } else {
    CU(b->lam.ensure(lam.size() * sizeof(float)));
    CU(b->rec.ensure((size_t)b->nrec * MIXED_ZN * sizeof(float)));
    CU(b->scratch.ensure(std::max((size_t)b->slots * sizeof(float4),
                                  ((size_t)REPAIR_SOLVE_BLOCKS_PER_SM * c->num_sms * (REPAIR_THREADS / 32) * 4 + 32 * 5) *
                                      sizeof(double)) *
                         b->max_nz)); /* the re-solve takes it over after the mixed solve */
    CU(b->lam64.ensure(lam64.size() * sizeof(double)));
    CU(b->colflag.ensure((size_t)ncol * sizeof(unsigned)));
    const size_t words = (size_t)ncol * ((b->max_nw + 31) / 32);
    CU(b->rbits.ensure(words * sizeof(unsigned)));
    CU(b->rlist.ensure(words * sizeof(unsigned long long)));
    CU(b->ilist.ensure((size_t)b->nitems * sizeof(unsigned long long)));
    CU(b->rslot.ensure(words * 32 * sizeof(int)));
  }
  CU(b->work.ensure(64));
  CU(b->status.ensure(64));
  CU(cudaMemcpy(b->cols.p, dc.data(), dc.size() * sizeof(MBatchCol), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->rec_pre.p, rpre.data(), rpre.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->tasks.p, tasks.data(), tasks.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->order.p, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  CU(cudaMemcpy(b->item_pre.p, ipre.data(), ipre.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  if (fp64)
    CU(cudaMemcpy(b->lam.p, lam64.data(), lam64.size() * sizeof(double), cudaMemcpyHostToDevice));
  else {
    CU(cudaMemcpy(b->lam.p, lam.data(), lam.size() * sizeof(float), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(b->lam64.p, lam64.data(), lam64.size() * sizeof(double), cudaMemcpyHostToDevice));
  }
  CU(cudaMemset(b->status.p, 0, 64));

  b->info.ncol = ncol;
  b->info.npoints = b->npoints;
  b->info.max_nz = b->max_nz;
  b->info.max_nw = b->max_nw;
  *out = guard.release();
  return OCO_OK;
}

/* Host work lists grow with ncol and nw: a failed allocation is OCO_ENOMEM (the partly built
 * batch is released by its guard while the exception unwinds), never an exception through
 * the C ABI. */
extern "C" int oco_batch_create(oco_ctx *c, const oco_batch_column *cols, int64_t ncol, const double *waves,
                                int64_t nwaves, int32_t form, int32_t layout, double fully_ionized_T,
                                oco_batch **out) {
  try {
    return batch_create(c, cols, ncol, waves, nwaves, form, layout, fully_ionized_T, out);
  } catch (const std::bad_alloc &) {
    return oco_set_err(c, OCO_ENOMEM, "oco_batch_create: out of host memory for %lld columns", (long long)ncol);
  }
}

extern "C" int oco_batch_bind(oco_batch *b, const double *rho, const double *T, int64_t n_in, double *U, int64_t n_u,
                              double *kappa, double *V, int64_t n_kv, double *Vtop, double *Vbot, int64_t n_flux) {
  if (!b) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_bind: NULL batch");
  oco_ctx *c = b->c;
  if (!rho || !T) return oco_set_err(c, OCO_EINVAL, "oco_batch_bind: rho and T are required");
  if (n_in < b->need_in) return oco_set_err(c, OCO_EINVAL, "oco_batch_bind: inputs need %lld elements", (long long)b->need_in);
  if (U && n_u < b->need_u) return oco_set_err(c, OCO_EINVAL, "oco_batch_bind: U needs %lld elements", (long long)b->need_u);
  if ((kappa || V) && n_kv < b->need_kv)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_bind: kappa and V need %lld elements", (long long)b->need_kv);
  if ((Vtop || Vbot) && n_flux < b->need_flux)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_bind: Vtop and Vbot need %lld elements", (long long)b->need_flux);
  const bool bound_family[3] = {U != nullptr, kappa || V, Vtop || Vbot};
  static const char *family[3] = {"U", "kappa/V", "Vtop/Vbot"};
  for (int f = 0; f < 3; f++)
    if (bound_family[f] && b->overlap[f][0] >= 0)
      return oco_set_err(c, OCO_EINVAL, "oco_batch_bind: columns %lld and %lld have overlapping %s ranges",
                         (long long)b->overlap[f][0], (long long)b->overlap[f][1], family[f]);
  CU(cudaSetDevice(c->device));
  if (b->pending) CU(cudaStreamSynchronize(b->last));
  b->rho = rho;
  b->T = T;
  b->U = U;
  b->K = kappa;
  b->V = V;
  b->Vtop = Vtop;
  b->Vbot = Vbot;
  b->bound = true;
  return capture(b);
}

extern "C" int oco_batch_tune(oco_batch *b) {
  if (!b) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_tune: NULL batch");
  oco_ctx *c = b->c;
  if (!b->bound) return oco_set_err(c, OCO_EINVAL, "oco_batch_tune: bind the arrays first");
  CU(cudaSetDevice(c->device));
  if (b->pending) CU(cudaStreamSynchronize(b->last));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  struct Cand {
    int tiling, bps;
    float ms;
  };
  std::vector<Cand> cands;
  for (int t = 0; t < 2; t++)
    for (int d = 0; d < 3; d++) {
      const int bps = b->max_bps[t] - d; /* max_bps 0: tiling not available for the form */
      if (bps >= 1) cands.push_back({t, bps, 0.0f});
    }
  if (cands.size() > 16) cands.resize(16);
  const int tiling0 = b->tiling, bps0 = b->bps; /* the captured graph's setting, kept on failure */
  int rc = OCO_OK;
  bool warm = false;
  for (auto &k : cands) {
    b->tiling = k.tiling;
    b->bps = k.bps;
    if (!warm) { /* first touch of the outputs and the code */
      rc = enqueue_run(b, b->cap);
      warm = true;
      if (rc) break;
    }
    cudaEventRecord(e0, b->cap);
    rc = enqueue_run(b, b->cap);
    if (rc) break;
    cudaEventRecord(e1, b->cap);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      rc = oco_set_err(c, OCO_ECUDA, "oco_batch_tune: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    cudaEventElapsedTime(&k.ms, e0, e1);
    if ((rc = check_status(b, false))) break; /* zero pivots are reported by oco_batch_wait */
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    b->tiling = tiling0;
    b->bps = bps0;
    return rc;
  }
  const Cand *best = &cands[0];
  for (auto &k : cands)
    if (k.ms < best->ms) best = &k;
  b->tiling = best->tiling;
  b->bps = best->bps;
  b->info.ncandidates = (int32_t)cands.size();
  for (size_t i = 0; i < cands.size(); i++) {
    b->info.cand_tiling[i] = cands[i].tiling;
    b->info.cand_blocks_per_sm[i] = cands[i].bps;
    b->info.cand_ms[i] = cands[i].ms;
  }
  b->info.tuned = 1;
  return capture(b);
}

extern "C" int oco_batch_set_tiling(oco_batch *b, int32_t tiling, int32_t blocks_per_sm) {
  if (!b) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_set_tiling: NULL batch");
  oco_ctx *c = b->c;
  if (tiling != OCO_TILING_WARP_COLUMN && tiling != OCO_TILING_PACKED)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_set_tiling: bad tiling %d", tiling);
  const int lim = b->max_bps[tiling];
  if (lim == 0) return oco_set_err(c, OCO_EINVAL, "oco_batch_set_tiling: the packed tiling runs the mixed form only");
  if (blocks_per_sm < 0 || blocks_per_sm > lim)
    return oco_set_err(c, OCO_EINVAL, "oco_batch_set_tiling: blocks_per_sm must be 0..%d", lim);
  CU(cudaSetDevice(c->device));
  if (b->pending) CU(cudaStreamSynchronize(b->last));
  b->tiling = tiling;
  b->bps = blocks_per_sm ? blocks_per_sm : lim;
  return b->bound ? capture(b) : OCO_OK;
}

extern "C" int oco_batch_run(oco_batch *b, void *stream) {
  if (!b) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_run: NULL batch");
  oco_ctx *c = b->c;
  if (!b->bound || !b->exec) return oco_set_err(c, OCO_EINVAL, "oco_batch_run: bind the arrays first");
  CU(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream;
  if (b->pending && b->last != s) { /* replays share the work queue: no overlap across streams */
    if (!b->after_last) CU(cudaEventCreateWithFlags(&b->after_last, cudaEventDisableTiming));
    CU(cudaEventRecord(b->after_last, b->last));
    CU(cudaStreamWaitEvent(s, b->after_last, 0));
  }
  CU(cudaGraphLaunch(b->exec, s));
  b->last = s;
  b->pending = true;
  b->info.graph_launches++;
  c->launches += b->form == OCO_FORM_MIXED ? 4 : 2; /* records, solve (+ the re-solve's two kernels) */
  return OCO_OK;
}

extern "C" int oco_batch_wait(oco_batch *b) {
  if (!b) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_wait: NULL batch");
  oco_ctx *c = b->c;
  if (!b->pending) return OCO_OK;
  CU(cudaSetDevice(c->device));
  CU(cudaStreamSynchronize(b->last));
  b->pending = false;
  return check_status(b);
}

extern "C" int oco_batch_get_info(const oco_batch *b, oco_batch_info *info) {
  if (!b || !info) return oco_set_err(nullptr, OCO_EINVAL, "oco_batch_get_info: NULL argument");
  *info = b->info;
  info->tiling = b->tiling;
  info->blocks_per_sm = b->bps;
  return OCO_OK;
}

extern "C" void oco_batch_destroy(oco_batch *b) {
  if (!b) return;
  if (b->c) cudaSetDevice(b->c->device);
  if (b->pending) cudaStreamSynchronize(b->last); /* a null stream is the default stream */
  if (b->cap) cudaStreamSynchronize(b->cap);
  drop_graph(b);
  for (DevBuf *d : {&b->lam64, &b->colflag, &b->rbits, &b->rslot, &b->rlist, &b->ilist, &b->cols, &b->rec_pre, &b->tasks, &b->order, &b->item_pre, &b->lam, &b->rec, &b->scratch,
                    &b->work, &b->status})
    d->release();
  if (b->after_last) cudaEventDestroy(b->after_last);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
}
