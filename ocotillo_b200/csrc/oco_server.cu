/*
 * oco_server.cu -- the serving loop (include/oco.h, "Serving loop").
 *
 * One scheduler thread per server drives every CUDA call of the running jobs.  Each job slot
 * is a context (oco_ctx: stream, wavelength tables, record and Thomas workspace), so jobs in
 * different slots run on different streams and their launches overlap on the device.  Per
 * pass the scheduler
 *   1. admits queued jobs (first come first served) while a slot is free and the job's
 *      footprint fits the remaining budget: allocates its device arrays (stream-ordered
 *      allocator), copies its inputs, builds its wavelength tables;
 *   2. tops up every running job to two launches in flight, each covering the next
 *      chunk_points of the job's columns with the persistent grid capped at the job's share
 *      (full grid / jobs with work left), so a job admitted mid-run gets SMs at the next
 *      launch boundary of the others;
 *   3. retires finished launches (event queries), completes jobs, frees their slots and
 *      their inputs; results stay on the device until oco_server_fetch.
 * It sleeps on a condition variable when it has nothing to issue (0.1 ms polls while work
 * is in flight).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <exception>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/oco.h"
#include "oco_ctx.h"
#include "oco_internal.h"

namespace {

thread_local std::string g_server_err;

int serr(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_server_err = buf;
  return code;
}

/* CUDA check for the client-facing calls (message for oco_server_last_error). */
#define SCU(call)                                                                                     \
  do {                                                                                                \
    cudaError_t e_ = (call);                                                                          \
    if (e_ != cudaSuccess)                                                                            \
      return serr(e_ == cudaErrorMemoryAllocation ? OCO_ENOMEM : OCO_ECUDA, "%s: %s", #call,           \
                  cudaGetErrorString(e_));                                                            \
  } while (0)

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

constexpr int kInFlight = 2;             /* launches in flight per job */
constexpr int64_t kMaxChunkCols = 4096;  /* record buffer bound */
constexpr size_t kRecordBytesMax = 26 * sizeof(double);

struct Job {
  int64_t id = 0;
  oco_params p{};
  int want_fields = 0;
  const double *rho_in = nullptr, *T_in = nullptr;
  std::vector<double> waves;
  /* state (guarded by the server mutex) */
  int state = OCO_JOB_QUEUED, error = OCO_OK, inputs_consumed = 0;
  bool fetching = false; /* one oco_server_fetch owns the done job's arrays */
  std::string msg;
  int64_t bytes = 0, input_bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  /* scheduler-owned */
  int slot = -1;
  double *rho = nullptr, *T = nullptr, *Vtop = nullptr, *Vbot = nullptr, *U = nullptr, *K = nullptr, *V = nullptr;
  int64_t ncol = 0, next_col = 0, chunk_cols = 1;
  cudaEvent_t inputs_done = nullptr;
  std::deque<cudaEvent_t> inflight;
};

struct Slot {
  oco_ctx *ctx = nullptr;
  Job *job = nullptr;
  std::vector<cudaEvent_t> pool;
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    return e;
  }
};

int64_t footprint(const oco_params &p, int want_fields, int64_t *input_bytes) {
  const int64_t ncol = (int64_t)p.nx * p.ny;
  const int64_t in = ncol * p.nz * 2 * (int64_t)sizeof(double);
  int64_t out = ncol * p.nw * 2 * (int64_t)sizeof(double);
  if (want_fields) out += ncol * p.nw * ((int64_t)(p.nz + 6) + 2 * (int64_t)p.nz) * (int64_t)sizeof(double);
  if (input_bytes) *input_bytes = in;
  return in + out;
}

}  // namespace

struct oco_server {
  int device = 0;
  bool trace = false; /* OCO_SERVER_TRACE=1: one stderr line per scheduler step slower than 1 ms */
  int64_t chunk_points = 1ll << 28;
  double budget = 0, used = 0;
  std::vector<Slot> slots;
  int full_blocks[3] = {1, 1, 1};
  cudaStream_t misc = nullptr; /* frees of fetched jobs */
  cudaMemPool_t pool = nullptr; /* job arrays; keeps freed memory mapped for the next job */
  std::mutex mu;
  std::condition_variable cv;      /* wakes the scheduler */
  std::condition_variable cv_done; /* wakes waiters */
  std::deque<Job *> queue;
  std::unordered_map<int64_t, std::unique_ptr<Job>> jobs;
  int64_t next_id = 1;
  bool closing = false;
  std::thread th;
  void loop();
  int admit(Job *j, Slot &s);
  void release_inputs(Job *j);
  void fail(Job *j, int code, const std::string &msg);
};

/* Frees a job's input arrays (called once their copies are done). */
void oco_server::release_inputs(Job *j) {
  cudaStream_t s = j->slot >= 0 ? slots[(size_t)j->slot].ctx->stream : misc;
  if (j->rho) cudaFreeAsync(j->rho, s);
  if (j->T) cudaFreeAsync(j->T, s);
  j->rho = j->T = nullptr;
}

/* Marks j failed (mutex held by the caller) and frees all its device memory. */
void oco_server::fail(Job *j, int code, const std::string &msg) {
  cudaStream_t s = j->slot >= 0 ? slots[(size_t)j->slot].ctx->stream : misc;
  if (j->slot >= 0) cudaStreamSynchronize(s);
  for (double **p : {&j->rho, &j->T, &j->Vtop, &j->Vbot, &j->U, &j->K, &j->V})
    if (*p) {
      cudaFreeAsync(*p, s);
      *p = nullptr;
    }
  if (j->state == OCO_JOB_RUNNING) used -= (double)j->bytes;
  j->state = OCO_JOB_FAILED;
  j->error = code;
  j->msg = msg;
  j->inputs_consumed = 1;
  j->t_done = now_s();
  if (j->slot >= 0) { /* its events are complete after the synchronize: back to the slot's pool */
    Slot &sl = slots[(size_t)j->slot];
    sl.pool.insert(sl.pool.end(), j->inflight.begin(), j->inflight.end());
    sl.job = nullptr;
  }
  j->inflight.clear();
  j->slot = -1;
  cv_done.notify_all();
}

int oco_server::admit(Job *j, Slot &sl) {
  oco_ctx *c = sl.ctx;
  cudaStream_t s = c->stream;
  const double t0 = now_s();
  int rc = oco_set_wavelengths(c, j->waves.data(), j->p.nw);
  if (rc) return rc;
  if ((rc = oco_ctx_check_params(c, &j->p))) return rc;
  const double t1 = now_s();
  const int64_t ncol = (int64_t)j->p.nx * j->p.ny;
  const size_t nin = (size_t)ncol * j->p.nz * sizeof(double);
  const size_t nfl = (size_t)ncol * j->p.nw * sizeof(double);
  CU(cudaMallocFromPoolAsync((void **)&j->rho, nin, pool, s));
  CU(cudaMallocFromPoolAsync((void **)&j->T, nin, pool, s));
  CU(cudaMallocFromPoolAsync((void **)&j->Vtop, nfl, pool, s));
  CU(cudaMallocFromPoolAsync((void **)&j->Vbot, nfl, pool, s));
  if (j->want_fields) {
    CU(cudaMallocFromPoolAsync((void **)&j->U, (size_t)ncol * j->p.nw * (j->p.nz + 6) * sizeof(double), pool, s));
    CU(cudaMallocFromPoolAsync((void **)&j->K, (size_t)ncol * j->p.nw * j->p.nz * sizeof(double), pool, s));
    CU(cudaMallocFromPoolAsync((void **)&j->V, (size_t)ncol * j->p.nw * j->p.nz * sizeof(double), pool, s));
  }
  const double t2 = now_s();
  CU(cudaMemcpyAsync(j->rho, j->rho_in, nin, cudaMemcpyDefault, s));
  CU(cudaMemcpyAsync(j->T, j->T_in, nin, cudaMemcpyDefault, s));
  if (!j->inputs_done) CU(cudaEventCreateWithFlags(&j->inputs_done, cudaEventDisableTiming));
  CU(cudaEventRecord(j->inputs_done, s));
  if ((rc = oco_ctx_reset_status(c, s))) return rc;
  if (trace)
    fprintf(stderr, "[oco_server] admit job %lld: tables %.3f ms, allocation %.3f ms, copies %.3f ms\n",
            (long long)j->id, 1e3 * (t1 - t0), 1e3 * (t2 - t1), 1e3 * (now_s() - t2));
  j->ncol = ncol;
  j->next_col = 0;
  const int64_t per_col = (int64_t)j->p.nz * j->p.nw;
  j->chunk_cols = std::max<int64_t>(1, std::min<int64_t>({ncol, chunk_points / per_col, kMaxChunkCols}));
  return OCO_OK;
}

void oco_server::loop() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    bool progress = false;
    /* 1. admission */
    for (;;) {
      if (queue.empty()) break;
      int free_slot = -1;
      for (size_t i = 0; i < slots.size(); i++)
        if (!slots[i].job) {
          free_slot = (int)i;
          break;
        }
      if (free_slot < 0) break;
      Job *j = queue.front();
      if (used + (double)j->bytes > budget) break; /* first come first served: the head waits for memory */
      queue.pop_front();
      Slot &sl = slots[(size_t)free_slot];
      sl.job = j;
      j->slot = free_slot;
      j->state = OCO_JOB_RUNNING;
      j->t_admit = now_s();
      used += (double)j->bytes;
      lk.unlock();
      const double ta = now_s();
      const int rc = admit(j, sl);
      if (trace) fprintf(stderr, "[oco_server] %.6f admit job %lld: %.3f ms\n", ta, (long long)j->id, 1e3 * (now_s() - ta));
      lk.lock();
      if (rc) fail(j, rc, std::string("admission: ") + oco_last_error(sl.ctx));
      progress = true;
    }
    if (closing && queue.empty()) {
      bool any = false;
      for (auto &sl : slots) any |= sl.job != nullptr;
      if (!any) break;
    }
    /* 2. dispatch */
    int with_work = 0;
    for (auto &sl : slots)
      if (sl.job && sl.job->next_col < sl.job->ncol) with_work++;
    lk.unlock();
    for (auto &sl : slots) {
      Job *j = sl.job;
      if (!j || j->state != OCO_JOB_RUNNING) continue;
      while ((int)j->inflight.size() < kInFlight && j->next_col < j->ncol) {
        const int64_t nb = std::min(j->chunk_cols, j->ncol - j->next_col);
        const int share = std::max(1, full_blocks[j->p.form] / std::max(1, with_work));
        const double tl = now_s();
        int rc = oco_ctx_run_columns(sl.ctx, &j->p, j->rho, j->T, j->next_col, nb, j->U, j->K, j->V, j->Vtop,
                                     j->Vbot, share, sl.ctx->stream);
        cudaEvent_t e = sl.take();
        if (!rc && cudaEventRecord(e, sl.ctx->stream) != cudaSuccess) rc = OCO_ECUDA;
        if (rc) {
          sl.pool.push_back(e);
          lk.lock();
          fail(j, rc, std::string("launch: ") + oco_last_error(sl.ctx));
          lk.unlock();
          break;
        }
        j->inflight.push_back(e);
        j->next_col += nb;
        progress = true;
        if (trace && now_s() - tl > 1e-3)
          fprintf(stderr, "[oco_server] %.6f launch job %lld cols %lld+%lld grid %d: %.3f ms\n", tl, (long long)j->id,
                  (long long)(j->next_col - nb), (long long)nb, share, 1e3 * (now_s() - tl));
      }
    }
    /* 3. retire */
    for (auto &sl : slots) {
      Job *j = sl.job;
      if (!j || j->state != OCO_JOB_RUNNING) continue;
      if (j->rho && cudaEventQuery(j->inputs_done) == cudaSuccess && !j->inputs_consumed) {
        lk.lock();
        j->inputs_consumed = 1;
        lk.unlock();
        progress = true;
      }
      while (!j->inflight.empty()) {
        const cudaError_t q = cudaEventQuery(j->inflight.front());
        if (q == cudaErrorNotReady) break;
        sl.pool.push_back(j->inflight.front());
        j->inflight.pop_front();
        progress = true;
        if (q != cudaSuccess) {
          lk.lock();
          fail(j, OCO_ECUDA, std::string("kernel: ") + cudaGetErrorString(q));
          lk.unlock();
          j = nullptr;
          break;
        }
      }
      if (!j || !j->inflight.empty() || j->next_col < j->ncol) continue;
      /* all launches done */
      const double tr = now_s();
      const int rc = oco_ctx_read_status(sl.ctx, sl.ctx->stream, &j->p);
      if (trace) fprintf(stderr, "[oco_server] %.6f done job %lld: status read %.3f ms\n", tr, (long long)j->id, 1e3 * (now_s() - tr));
      lk.lock();
      if (rc && rc != OCO_EZEROPIVOT) {
        fail(j, rc, oco_last_error(sl.ctx));
      } else {
        release_inputs(j);
        used -= (double)j->input_bytes;
        j->bytes -= j->input_bytes;
        j->error = rc;
        j->inputs_consumed = 1;
        j->state = OCO_JOB_DONE;
        j->t_done = now_s();
        sl.job = nullptr;
        j->slot = -1;
        cv_done.notify_all();
      }
      lk.unlock();
      progress = true;
    }
    lk.lock();
    if (!progress) {
      bool inflight = false;
      for (auto &sl : slots) inflight |= sl.job != nullptr;
      if (inflight)
        cv.wait_for(lk, std::chrono::microseconds(100));
      else if (queue.empty() && !closing)
        cv.wait_for(lk, std::chrono::milliseconds(50));
      else if (!queue.empty())
        cv.wait_for(lk, std::chrono::milliseconds(1)); /* head waits for memory: fetches wake us */
    }
  }
}

static void free_server(oco_server *s) {
  for (auto &sl : s->slots) {
    for (auto e : sl.pool) cudaEventDestroy(e);
    if (sl.ctx) oco_destroy(sl.ctx);
  }
  if (s->misc) cudaStreamDestroy(s->misc);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
}

static int setup_server(oco_server *srv, const oco_server_config *cfg) {
  SCU(cudaSetDevice(cfg->device));
  SCU(cudaStreamCreateWithFlags(&srv->misc, cudaStreamNonBlocking));
  srv->slots.resize((size_t)cfg->max_jobs);
  for (auto &sl : srv->slots) {
    const int rc = oco_create(&sl.ctx, cfg->device);
    if (rc) return serr(rc, "oco_server_create: %s", oco_last_error(nullptr));
    /* jobs' reference-layout fields are stored directly: transpose temporaries would be sized
     * by the launch (up to chunk_points) and allocated while other jobs run */
    sl.ctx->ref_transpose = false;
  }
  for (int f = 0; f < 3; f++) srv->full_blocks[f] = oco_ctx_full_blocks(srv->slots[0].ctx, f, 0);
  /* workspace reserved up front, so that admissions do not reallocate (a free synchronizes
   * the device): wavelength tables for up to 4096 wavelengths and, for nz <= max_nz, the
   * records of one launch and the Thomas scratch of a full grid */
  const int fb = std::max({srv->full_blocks[0], srv->full_blocks[1], srv->full_blocks[2]});
  for (auto &sl : srv->slots) {
    oco_ctx *c = sl.ctx;
    SCU(c->lam.ensure((size_t)oco::NL * 4096 * sizeof(double)));
    SCU(c->lam32.ensure((size_t)oco::MIXED_LN * 4096 * sizeof(float)));
    if (cfg->max_nz > 0) {
      SCU(c->scratch.ensure((size_t)fb * 128 * cfg->max_nz * 4 * sizeof(double)));
      SCU(c->pil.ensure((size_t)kMaxChunkCols * cfg->max_nz * kRecordBytesMax));
    }
  }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = cfg->device;
  SCU(cudaMemPoolCreate(&srv->pool, &props));
  uint64_t keep = UINT64_MAX;
  SCU(cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  if (cfg->reserve_bytes > 0) { /* grow the pool once; freed blocks stay mapped */
    void *r = nullptr;
    SCU(cudaMallocFromPoolAsync(&r, (size_t)cfg->reserve_bytes, srv->pool, srv->misc));
    SCU(cudaFreeAsync(r, srv->misc));
    SCU(cudaStreamSynchronize(srv->misc));
  }
  size_t fr = 0, tot = 0;
  SCU(cudaMemGetInfo(&fr, &tot));
  srv->budget = cfg->budget_bytes > 0 ? cfg->budget_bytes : 0.85 * (double)fr;
  return OCO_OK;
}

extern "C" int oco_server_create(const oco_server_config *cfg, oco_server **out) {
  if (!cfg || !out) return serr(OCO_EINVAL, "oco_server_create: NULL argument");
  *out = nullptr;
  if (cfg->max_jobs < 1 || cfg->max_nz < 0 || cfg->reserved != 0 || cfg->budget_bytes < 0 || cfg->chunk_points < 0 ||
      cfg->reserve_bytes < 0)
    return serr(OCO_EINVAL, "oco_server_create: need max_jobs >= 1, max_nz >= 0, budget >= 0, reserved = 0");
  oco_server *srv = new (std::nothrow) oco_server();
  if (!srv) return serr(OCO_ENOMEM, "oco_server_create: out of host memory");
  srv->device = cfg->device;
  if (cfg->chunk_points > 0) srv->chunk_points = cfg->chunk_points;
  if (const char *t = getenv("OCO_SERVER_TRACE")) srv->trace = t[0] == '1';
  int rc;
  try { /* host allocations grow with max_jobs; thread creation can fail */
    rc = setup_server(srv, cfg);
    if (!rc) srv->th = std::thread([srv] { srv->loop(); });
  } catch (const std::bad_alloc &) {
    rc = serr(OCO_ENOMEM, "oco_server_create: out of host memory");
  } catch (const std::exception &e) {
    rc = serr(OCO_EINVAL, "oco_server_create: %s", e.what());
  }
  if (rc) {
    free_server(srv);
    return rc;
  }
  *out = srv;
  return OCO_OK;
}

extern "C" int oco_server_submit(oco_server *s, const oco_job *job, int64_t *job_id) {
  if (!s || !job || !job_id) return serr(OCO_EINVAL, "oco_server_submit: NULL argument");
  if (job->nx < 1 || job->ny < 1 || job->nz < 2 || job->nw < 1 || !(job->dz > 0.0) || !std::isfinite(job->dz) ||
      !job->rho || !job->T || !job->waves)
    return serr(OCO_EINVAL, "oco_server_submit: bad job (need nx, ny >= 1, nz >= 2, nw >= 1, finite dz > 0, arrays)");
  if (!oco::block_elements_fit(job->nx, job->ny, job->nz, job->nw))
    return serr(OCO_EINVAL, "oco_server_submit: job too large: nx*ny*nw*(nz+6) exceeds 2^56 elements");
  for (int i = 0; i < job->nw; i++)
    if (!(job->waves[i] > 0.0) || !std::isfinite(job->waves[i]))
      return serr(OCO_EINVAL, "oco_server_submit: wavelength %d is not positive and finite", i);
  if (job->form != OCO_FORM_PLAIN && job->form != OCO_FORM_STABLE && job->form != OCO_FORM_MIXED)
    return serr(OCO_EINVAL, "oco_server_submit: unknown form %d", job->form);
  std::unique_ptr<Job> j;
  try {
    j = std::make_unique<Job>();
    j->waves.assign(job->waves, job->waves + job->nw);
  } catch (const std::bad_alloc &) {
    return serr(OCO_ENOMEM, "oco_server_submit: out of host memory");
  }
  j->p.nx = job->nx;
  j->p.ny = job->ny;
  j->p.nz = job->nz;
  j->p.nw = job->nw;
  j->p.dz = job->dz;
  j->p.sigma_grey = 0.4;
  j->p.fully_ionized_T = job->fully_ionized_T;
  j->p.lgrey = 0;
  j->p.form = job->form;
  j->p.layout = OCO_LAYOUT_REFERENCE;
  j->want_fields = job->want_fields ? 1 : 0;
  j->rho_in = job->rho;
  j->T_in = job->T;
  j->bytes = footprint(j->p, j->want_fields, &j->input_bytes);
  std::lock_guard<std::mutex> g(s->mu);
  if (s->closing) return serr(OCO_ECLOSED, "oco_server_submit: the server is shutting down");
  if ((double)j->bytes > s->budget)
    return serr(OCO_EADMIT, "oco_server_submit: footprint %.3g GB exceeds the admission budget %.3g GB",
                (double)j->bytes / 1e9, s->budget / 1e9);
  const int64_t id = s->next_id;
  j->id = id;
  j->t_submit = now_s();
  try { /* the job table owns the job before the queue refers to it, and loses it if queueing fails */
    auto it = s->jobs.emplace(id, std::move(j)).first;
    try {
      s->queue.push_back(it->second.get());
    } catch (...) {
      s->jobs.erase(it);
      throw;
    }
  } catch (const std::bad_alloc &) {
    return serr(OCO_ENOMEM, "oco_server_submit: out of host memory");
  }
  s->next_id++;
  *job_id = id;
  s->cv.notify_all();
  return OCO_OK;
}

extern "C" int oco_server_status(oco_server *s, int64_t id, oco_job_status *st) {
  if (!s || !st) return serr(OCO_EINVAL, "oco_server_status: NULL argument");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return serr(OCO_EINVAL, "oco_server_status: unknown job %lld", (long long)id);
  const Job *j = it->second.get();
  *st = oco_job_status{};
  st->state = j->state;
  st->error = j->error;
  st->inputs_consumed = j->inputs_consumed;
  st->bytes = j->bytes;
  st->submit_s = j->t_submit;
  st->admit_s = j->t_admit;
  st->done_s = j->t_done;
  return OCO_OK;
}

extern "C" int oco_server_wait(oco_server *s, int64_t id, double timeout_s) {
  if (!s) return serr(OCO_EINVAL, "oco_server_wait: NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return serr(OCO_EINVAL, "oco_server_wait: unknown job %lld", (long long)id);
  Job *j = it->second.get();
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(std::max(0.0, timeout_s));
  while (j->state != OCO_JOB_DONE && j->state != OCO_JOB_FAILED)
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout && j->state != OCO_JOB_DONE &&
        j->state != OCO_JOB_FAILED)
      return serr(OCO_EAGAIN, "oco_server_wait: job %lld not done", (long long)id);
  if (j->state == OCO_JOB_FAILED) return serr(j->error, "job %lld failed: %s", (long long)id, j->msg.c_str());
  return OCO_OK;
}

/* Copies a done job's results into the caller's host arrays (any may be NULL). */
static int copy_results(oco_server *s, const Job *j, double *Vtop, double *Vbot, double *U, double *kappa, double *V) {
  const int64_t ncol = (int64_t)j->p.nx * j->p.ny;
  const size_t nfl = (size_t)ncol * j->p.nw * sizeof(double);
  const size_t nkv = (size_t)ncol * j->p.nw * j->p.nz * sizeof(double);
  SCU(cudaSetDevice(s->device));
  if (Vtop) SCU(cudaMemcpyAsync(Vtop, j->Vtop, nfl, cudaMemcpyDeviceToHost, s->misc));
  if (Vbot) SCU(cudaMemcpyAsync(Vbot, j->Vbot, nfl, cudaMemcpyDeviceToHost, s->misc));
  if (U && j->U) SCU(cudaMemcpyAsync(U, j->U, (size_t)ncol * j->p.nw * (j->p.nz + 6) * sizeof(double),
                                    cudaMemcpyDeviceToHost, s->misc));
  if (kappa && j->K) SCU(cudaMemcpyAsync(kappa, j->K, nkv, cudaMemcpyDeviceToHost, s->misc));
  if (V && j->V) SCU(cudaMemcpyAsync(V, j->V, nkv, cudaMemcpyDeviceToHost, s->misc));
  SCU(cudaStreamSynchronize(s->misc));
  return OCO_OK;
}

extern "C" int oco_server_fetch(oco_server *s, int64_t id, double *Vtop, double *Vbot, double *U, double *kappa,
                                double *V) {
  if (!s) return serr(OCO_EINVAL, "oco_server_fetch: NULL server");
  Job *j = nullptr;
  {
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return serr(OCO_EINVAL, "oco_server_fetch: unknown job %lld", (long long)id);
    j = it->second.get();
    if (j->state == OCO_JOB_FAILED) return serr(j->error, "job %lld failed: %s", (long long)id, j->msg.c_str());
    if (j->state != OCO_JOB_DONE) return serr(OCO_EAGAIN, "oco_server_fetch: job %lld not done", (long long)id);
    if (j->fetching) return serr(OCO_EAGAIN, "oco_server_fetch: job %lld is being fetched by another call", (long long)id);
    j->fetching = true;
  }
  const int rc = copy_results(s, j, Vtop, Vbot, U, kappa, V);
  if (!rc && ((U && !j->U) || (kappa && !j->K) || (V && !j->V)))
    serr(OCO_OK, "oco_server_fetch: job %lld kept no fields; only the emergent flux was copied", (long long)id);
  std::lock_guard<std::mutex> g(s->mu);
  if (rc) { /* the job stays done and fetchable */
    j->fetching = false;
    return rc;
  }
  for (double **p : {&j->Vtop, &j->Vbot, &j->U, &j->K, &j->V})
    if (*p) {
      cudaFreeAsync(*p, s->misc);
      *p = nullptr;
    }
  if (j->inputs_done) cudaEventDestroy(j->inputs_done);
  s->used -= (double)j->bytes;
  s->jobs.erase(id);
  s->cv.notify_all();
  return OCO_OK;
}

extern "C" void oco_server_destroy(oco_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->closing = true;
    while (!s->queue.empty()) {
      Job *j = s->queue.front();
      s->queue.pop_front();
      j->state = OCO_JOB_FAILED;
      j->error = OCO_ECLOSED;
      j->msg = "server shut down before admission";
      j->inputs_consumed = 1;
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
  }
  if (s->th.joinable()) s->th.join();
  cudaSetDevice(s->device);
  for (auto &kv : s->jobs) {
    Job *j = kv.second.get();
    for (double **p : {&j->rho, &j->T, &j->Vtop, &j->Vbot, &j->U, &j->K, &j->V})
      if (*p) cudaFreeAsync(*p, s->misc);
    if (j->inputs_done) cudaEventDestroy(j->inputs_done);
  }
  cudaStreamSynchronize(s->misc);
  free_server(s);
}

extern "C" const char *oco_server_last_error(void) { return g_server_err.c_str(); }
