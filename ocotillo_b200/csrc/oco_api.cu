/*
 * oco_api.cu -- the C ABI (include/oco.h): context, wavelength tables, workspace, and the
 * block solve on host or device arrays.
 *
 * A block solve runs in column chunks.  For each chunk: the pillar kernel computes the
 * wavelength-independent per-(column, z) quantities, then the persistent solve kernel
 * processes the chunk's (column, wavelength) items.  The device-array entry point writes
 * straight into the caller's arrays (either layout); the host-array entry point stages
 * each chunk through device buffers in the reference layout and copies them back with one
 * pitched copy per output, overlapping the next chunk's kernels with the copy-back.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/oco.h"
#include "mixed_core.h"
#include "ocomath.h"
#include "oco_consts.h"
#include "oco_ctx.h"
#include "oco_internal.h"

using namespace oco;

static thread_local std::string g_thread_err;

int oco_set_err(oco_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  g_thread_err = buf;
  return code;
}

extern "C" int oco_abi_version(void) { return OCO_ABI_VERSION; }

extern "C" const char *oco_last_error(const oco_ctx *c) {
  return c ? c->err.c_str() : g_thread_err.c_str();
}

extern "C" int oco_create(oco_ctx **out, int device) {
  oco_ctx *c = nullptr;
  if (!out) return oco_set_err(nullptr, OCO_EINVAL, "oco_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return oco_set_err(nullptr, OCO_ECUDA, "oco_create: no CUDA device");
  if (device < 0 || device >= ndev) return oco_set_err(nullptr, OCO_EINVAL, "oco_create: bad device %d", device);
  c = new (std::nothrow) oco_ctx();
  if (!c) return oco_set_err(nullptr, OCO_ENOMEM, "oco_create: out of host memory");
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking);
  for (int i = 0; i < 2 && e == cudaSuccess; i++)
    e = cudaEventCreateWithFlags(&c->stage[i].done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = c->work.ensure(64);
  if (e == cudaSuccess) e = c->status.ensure(64);
  if (e == cudaSuccess) e = c->stats.ensure(64);
  if (e == cudaSuccess) e = cudaMemset(c->stats.p, 0, 64);
  c->repair_cond = MIXED_REPAIR_COND;
  if (e != cudaSuccess) {
    int code = oco_set_err(nullptr, OCO_ECUDA, "oco_create: %s", cudaGetErrorString(e));
    oco_destroy(c);
    return code;
  }
  if (const char *r = getenv("OCO_REFERENCE_STORES")) c->ref_transpose = strcmp(r, "direct") != 0;
  if (const char *g = getenv("OCO_WORKSPACE_GB")) {
    double gb = atof(g);
    if (gb > 0.0) c->budget_bytes = std::max<size_t>((size_t)(gb * (1ull << 30)), 1);
  }
  if (const char *r = getenv("OCO_REPAIR_SLOTS")) c->repair_slots_max = std::max<int64_t>(0, atoll(r));
  *out = c;
  return OCO_OK;
}

extern "C" void oco_destroy(oco_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->status_pending) cudaStreamSynchronize(c->status_stream); /* a device-array call in flight */
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy) cudaStreamSynchronize(c->copy);
  c->lam.release();
  c->lam32.release();
  c->trapw.release();
  c->pil.release();
  c->scratch.release();
  c->tmpU.release();
  c->tmpK.release();
  c->tmpV.release();
  c->work.release();
  c->status.release();
  c->rbits.release();
  c->ilist.release();
  c->rslot.release();
  c->stats.release();
  c->colflag.release();
  c->rlist.release();
  for (auto &s : c->stage) {
    s.rho.release();
    s.T.release();
    s.U.release();
    s.K.release();
    s.V.release();
    s.top.release();
    s.bot.release();
    if (s.done) cudaEventDestroy(s.done);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy) cudaStreamDestroy(c->copy);
  for (auto *v : {&c->ev_solve, &c->ev_pil})
    for (auto &pr : *v) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  if (c->order_ev) cudaEventDestroy(c->order_ev);
  delete c;
}

extern "C" int oco_calc_wavelength(double w1, double w0, int32_t nw, double *wa) {
  if (nw < 1 || !wa) return oco_set_err(nullptr, OCO_EINVAL, "oco_calc_wavelength: nw < 1 or NULL wa");
  if (nw > 1) { /* continuous_opacity.f90:48-54 */
    double dw = (w1 - w0) / (double)(nw - 1);
    for (int i = 1; i <= nw; i++) wa[i - 1] = w0 + (double)(i - 1) * dw;
  } else {
    wa[0] = w0;
  }
  return OCO_OK;
}

/* Right-to-left binary powering: the operation order of the library routine gfortran
 * calls for REAL**INTEGER with a non-constant exponent (continuous_opacity.f90:108, :136). */
static double powi_var(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

/* gaunt, continuous_opacity.f90:343-375 */
static double gaunt_bf(int n, double wave_cm) {
  double lam_n = (double)(n * n) * k::hcR1;
  if (wave_cm <= lam_n) {
    double t = (wave_cm / lam_n) - 1.0;
    double eps2 = t * t;
    return 1.0 - (0.17285714285714285 * (1.0 - eps2)) * std::pow((double)n * (1.0 + eps2), -k::two_thirds);
  }
  return 0.0;
}

/* pre_calc_opacity_quantities (continuous_opacity.f90:64-141) with the C library's pow and
 * log10, as the reference; then the hot loop's lambda-only factors (ocomath, as the
 * device computes everything inside the loop). */
void oco::fill_lambda_table(const double *waves, int nw, double *tab) {
  static const double a_coeff[7] = {+1.99654,     -1.18267e-6,  +2.62423e-7, -4.40524e-11,
                                    +3.23992e-15, -1.39568e-19, +2.78701e-24};
  static const double b_coeff[3][5] = {{-2.276300, -1.685000, +0.766610, -0.053356, +0.000000},
                                       {+15.28270, -9.284600, +1.993810, -0.142631, +0.000000},
                                       {-197.789, +190.266, -67.9775, +10.6913, -0.62515}};
  auto T = [&](int f, int iw) -> double & { return tab[(size_t)f * nw + iw]; };
  for (int iw = 0; iw < nw; iw++) {
    const double wa = waves[iw];
    const double wcm = wa * 1e-8;
    const double wcm1 = 1.0 / wcm;
    const double nu = k::c_light * wcm1;
    const double chi = 1.2398e4 / wa;
    const double x2 = wcm1 * wcm1;
    const double w1cm5 = x2 * (wcm1 * x2);
    double s = 0.0;
    for (int i = 1; i <= 7; i++) s = s + (1e-17 * a_coeff[i - 1]) * powi_var(wa, i - 1);
    const double lg = std::log10(wa);
    T(L_CHI, iw) = chi;
    T(L_CHI1, iw) = 1.0 / chi;
    T(L_GFF, iw) = 0.3456 * std::pow(wa * k::Rangstrom, -k::one_third);
    T(L_WA3, iw) = wa * (wa * wa);
    T(L_SCOEF, iw) = s;
    T(L_HMON, iw) = (wa < 16000.0) ? 1.0 : 0.0;
    for (int i = 0; i < 3; i++) {
      double f = 0.0;
      for (int j = 1; j <= 5; j++) f = f + powi_var(lg, j - 1) * b_coeff[i][j - 1];
      T(L_F1 + i, iw) = f;
    }
    for (int n = 1; n <= 6; n++) {
      double n1 = 1.0 / (double)n;
      T(L_GN1 + n - 1, iw) = gaunt_bf(n, wcm) * (n1 * (n1 * n1));
    }
    T(L_NU9, iw) = nu * 1e-9;
    T(L_L3NU, iw) = 3.0 * oco_log(nu);
    T(L_HNUK, iw) = (k::h_planck * nu) * k::k1_cgs;
    T(L_WCM1, iw) = wcm1;
    T(L_SW5, iw) = k::source_function_const * w1cm5;
    T(L_LNSW5, iw) = std::log(k::source_function_const * w1cm5);
  }
}

static_assert(mx::MLN == MIXED_LN && mx::MZN == MIXED_ZN, "mixed record sizes");

void oco::fill_mixed_lambda_table(const double *tab, int nw, float *tab32) {
  for (int iw = 0; iw < nw; iw++) {
    auto T = [&](int f) { return tab[(size_t)f * nw + iw]; };
    mx::LamIn li;
    li.chi = T(L_CHI);
    li.gff = T(L_GFF);
    li.chi1 = T(L_CHI1);
    li.wa3 = T(L_WA3);
    li.s = T(L_SCOEF);
    li.hmon = T(L_HMON);
    li.f1 = T(L_F1);
    li.f2 = T(L_F2);
    li.f3 = T(L_F3);
    for (int q = 0; q < 6; q++) li.gn[q] = T(L_GN1 + q);
    li.nu9 = T(L_NU9);
    li.l3nu = T(L_L3NU);
    li.hnuk = T(L_HNUK);
    li.wcm1 = T(L_WCM1);
    li.sw5 = T(L_SW5);
    float rec[mx::MLN];
    mx::lambda_record(li, rec);
    for (int f = 0; f < mx::MLN; f++) tab32[(size_t)f * nw + iw] = rec[f];
  }
}

/* Every host table is built before the context changes, so a failed host allocation leaves
 * the previous grid in place. */
static int set_wavelengths(oco_ctx *c, const double *wa, int32_t nw) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "oco_set_wavelengths: NULL context");
  if (!wa || nw < 1) return oco_set_err(c, OCO_EINVAL, "oco_set_wavelengths: nw < 1 or NULL wa");
  for (int i = 0; i < nw; i++)
    if (!(wa[i] > 0.0) || !std::isfinite(wa[i]))
      return oco_set_err(c, OCO_EINVAL, "oco_set_wavelengths: wavelength %d is not positive", i);
  std::vector<double> tab((size_t)NL * nw, 0.0);
  fill_lambda_table(wa, nw, tab.data());
  std::vector<float> tab32((size_t)mx::MLN * nw);
  fill_mixed_lambda_table(tab.data(), nw, tab32.data());
  /* trapezoid weights over the grid as given (cm): w_i = (wa_{i+1} - wa_{i-1}) / 2, halved
   * differences at the ends; a single wavelength integrates to 0 */
  std::vector<double> tw((size_t)nw, 0.0);
  for (int i = 0; i + 1 < nw; i++) {
    const double h = 0.5 * ((wa[i + 1] - wa[i]) * 1e-8);
    tw[(size_t)i] += h;
    tw[(size_t)i + 1] += h;
  }
  std::vector<double> wcopy(wa, wa + nw);
  CU(cudaSetDevice(c->device));
  CU(cudaStreamSynchronize(c->stream));
  if (c->status_pending) CU(cudaStreamSynchronize(c->status_stream)); /* a device-array call may read the tables */
  CU(c->lam.ensure(tab.size() * sizeof(double)));
  CU(cudaMemcpy(c->lam.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
  CU(c->lam32.ensure(tab32.size() * sizeof(float)));
  CU(cudaMemcpy(c->lam32.p, tab32.data(), tab32.size() * sizeof(float), cudaMemcpyHostToDevice));
  CU(c->trapw.ensure(tw.size() * sizeof(double)));
  CU(cudaMemcpy(c->trapw.p, tw.data(), tw.size() * sizeof(double), cudaMemcpyHostToDevice));
  c->wa.swap(wcopy);
  c->nw = nw;
  return OCO_OK;
}

extern "C" int oco_set_wavelengths(oco_ctx *c, const double *wa, int32_t nw) {
  try {
    return set_wavelengths(c, wa, nw);
  } catch (const std::bad_alloc &) {
    return oco_set_err(c, OCO_ENOMEM, "oco_set_wavelengths: out of host memory for %d wavelengths", nw);
  }
}

static int check_params(oco_ctx *c, const oco_params *p) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  if (!p) return oco_set_err(c, OCO_EINVAL, "NULL params");
  if (p->nx < 1 || p->ny < 1 || p->nz < 2 || p->nw < 1)
    return oco_set_err(c, OCO_EINVAL, "bad dimensions nx=%d ny=%d nz=%d nw=%d (need nz >= 2)", p->nx, p->ny,
                   p->nz, p->nw);
  if (!block_elements_fit(p->nx, p->ny, p->nz, p->nw))
    return oco_set_err(c, OCO_EINVAL, "block too large: nx*ny*nw*(nz+6) exceeds 2^56 elements");
  if (p->lgrey && p->nw != 1)
    return oco_set_err(c, OCO_EGREY, "For Grey RT use only one wavelength. Switch nw=1 in resolution.in");
  if (!p->lgrey && (c->nw != p->nw))
    return oco_set_err(c, OCO_ENOWAVES, "wavelength tables hold %d wavelengths, block has nw=%d", c->nw, p->nw);
  if (p->form != OCO_FORM_PLAIN && p->form != OCO_FORM_STABLE && p->form != OCO_FORM_MIXED)
    return oco_set_err(c, OCO_EINVAL, "unknown form %d", p->form);
  if (p->layout != OCO_LAYOUT_REFERENCE && p->layout != OCO_LAYOUT_LAMBDA_FASTEST)
    return oco_set_err(c, OCO_EINVAL, "unknown layout %d", p->layout);
  if (!(p->dz > 0.0) || !std::isfinite(p->dz)) return oco_set_err(c, OCO_EINVAL, "dz must be positive and finite");
  return OCO_OK;
}

static const int kSolveThreads = 128;

/* Grid of the persistent solve kernel and its scratch: per resident thread and z, FP64
 * gamma, u, 1/kappa, q (32 B) or, for the mixed form, one record of at most 16 B. */
static int prepare_solve(oco_ctx *c, int form, int grey, int64_t nitems, int nz, int *blocks) {
  const bool mixed = form == OCO_FORM_MIXED;
  int bps = mixed ? solve_mixed_max_blocks_per_sm(kSolveThreads, c->nw)
                  : solve_fp64_max_blocks_per_sm(form == OCO_FORM_STABLE ? 1 : 0, grey, kSolveThreads);
  int64_t maxb = (int64_t)bps * c->num_sms;
  if (c->max_blocks > 0) maxb = std::min<int64_t>(maxb, c->max_blocks);
  int64_t need = (nitems + kSolveThreads - 1) / kSolveThreads;
  *blocks = (int)std::max<int64_t>(1, std::min(maxb, need));
  size_t slots = (size_t)(*blocks) * kSolveThreads;
  CU(c->scratch.ensure(slots * (size_t)nz * (mixed ? 16 : 4 * sizeof(double))));
  return OCO_OK;
}

/* Reference-layout outputs of a device solve go through lambda-fastest temporaries and a
 * tiled transpose (coalesced stores) unless disabled or pointless (grey / few wavelengths). */
static bool uses_transpose(const oco_ctx *c, const oco_params *p, bool u, bool k, bool v) {
  return c->ref_transpose && p->layout == OCO_LAYOUT_REFERENCE && !p->lgrey && p->nw >= 8 && (u || k || v);
}

/* Bytes of the per-(column, z) record of a form: the FP64 pillar or the mixed record. */
static size_t record_bytes(int form) {
  return form == OCO_FORM_MIXED ? MIXED_ZN * sizeof(float) : NF * sizeof(double);
}

/* Columns per chunk so that pillars (+ staged outputs on the host path) fit the budget. */
static int64_t chunk_columns(oco_ctx *c, const oco_params *p, bool host_path, bool u = true, bool k = true,
                             bool v = true, bool planes = true) {
  const int64_t ncol = (int64_t)p->nx * p->ny;
  size_t per_col = (size_t)p->nz * record_bytes(p->form);
  if (host_path) { /* two staging sets of the requested outputs */
    const size_t per_w = (u ? (size_t)(p->nz + 6) : 0) + (k ? (size_t)p->nz : 0) + (v ? (size_t)p->nz : 0) +
                         (planes ? 2 : 0);
    per_col += 2 * ((size_t)p->nz * 2 + (size_t)p->nw * per_w) * sizeof(double);
  }
  if (!host_path && uses_transpose(c, p, u, k, v)) /* lambda-fastest temporaries of the chunk */
    per_col += (size_t)p->nw * ((u ? (size_t)(p->nz + 6) : 0) + (k ? (size_t)p->nz : 0) + (v ? (size_t)p->nz : 0)) *
               sizeof(double);
  int64_t ch = (int64_t)std::max<size_t>(1, c->budget_bytes / per_col);
  if (p->form == OCO_FORM_MIXED) /* the FP64 re-solve indexes a chunk's flagged items with 32-bit slots */
    ch = std::min<int64_t>(ch, std::max<int64_t>(1, INT32_MAX / p->nw));
  return std::min(ch, ncol);
}

int64_t oco_ctx_repair_slots(const oco_ctx *c, int64_t cap) {
  if (c->repair_slots_max >= 0 && c->repair_slots_max < cap) cap = c->repair_slots_max & ~(int64_t)31;
  return cap;
}

/* One chunk: pillars + persistent solve. Outputs described by the strides in a. */
static int run_chunk_mixed(oco_ctx *c, const oco_params *p, const double *rho, const double *T, int64_t nb,
                           const SolveArgs &a64, cudaStream_t s) {
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
  if (c->prof) {
    e0 = c->take_event();
    e1 = c->take_event();
    e2 = c->take_event();
    e3 = c->take_event();
    CU(cudaEventRecord(e0, s));
  }
  float *rec = c->pil.as<float>();
  CU(c->colflag.ensure((size_t)nb * sizeof(unsigned)));
  CU(cudaMemsetAsync(c->colflag.p, 0, (size_t)nb * sizeof(unsigned), s));
  CU(launch_pillars_mixed(rho, T, nb, p->nz, p->fully_ionized_T, rec, c->colflag.as<unsigned>(), s));
  if (c->prof) {
    CU(cudaEventRecord(e1, s));
    c->ev_pil.emplace_back(e0, e1);
  }
  int blocks = 0;
  int rc = prepare_solve(c, OCO_FORM_MIXED, 0, nb * p->nw, p->nz, &blocks);
  if (rc) return rc;
  const size_t slots = (size_t)blocks * kSolveThreads;
  /* the re-solve takes over the mixed solve's scratch: at least its per-warp arrays and 32 slots */
  const int rsolve_blocks = REPAIR_SOLVE_BLOCKS_PER_SM * c->num_sms, rcoef_blocks = REPAIR_COEF_BLOCKS_PER_SM * c->num_sms;
  CU(c->scratch.ensure(((size_t)rsolve_blocks * (REPAIR_THREADS / 32) * 4 + 32 * 5) * p->nz * sizeof(double)));
  MixedArgs a{};
  a.rec = rec;
  a.lam = c->lam32.as<float>();
  a.ncol = nb;
  a.nz = p->nz;
  a.nw = p->nw;
  a.dz = p->dz;
  mx::ldz2_split(p->dz, a.ldz2i, a.ldz2f);
  a.U = a64.U, a.U_zs = a64.U_zs, a.U_is = a64.U_is;
  a.K = a64.K, a.K_zs = a64.K_zs, a.K_is = a64.K_is;
  a.V = a64.V, a.V_zs = a64.V_zs, a.V_is = a64.V_is;
  a.Vtop = a64.Vtop, a.Vbot = a64.Vbot;
  a.ld_col = a64.ld_col, a.c_off = a64.c_off, a.layout = a64.layout;
  a.s4 = c->scratch.as<float4>();
  a.slot_stride = (int64_t)slots;
  a.work = c->work.as<unsigned long long>();
  a.status = c->status.as<unsigned long long>();
  a.repair_cond = c->repair_cond;
  a.colflag = c->colflag.as<unsigned>();
  const int64_t nwords = (p->nw + 31) / 32;
  CU(c->rbits.ensure((size_t)nb * nwords * sizeof(unsigned)));
  CU(c->rlist.ensure((size_t)nb * nwords * sizeof(unsigned long long)));
  CU(c->ilist.ensure((size_t)nb * p->nw * sizeof(unsigned long long)));
  CU(c->rslot.ensure((size_t)nb * nwords * 32 * sizeof(int)));
  a.rbits = c->rbits.as<unsigned>();
  a.rslot = c->rslot.as<int>();
  a.rlist = c->rlist.as<unsigned long long>();
  a.rcount = c->stats.as<unsigned long long>() + 1;
  a.ilist = c->ilist.as<unsigned long long>();
  a.icount = c->stats.as<unsigned long long>() + 2;
  CU(cudaMemsetAsync(a.rcount, 0, 3 * sizeof(unsigned long long), s)); /* rcount, icount, the re-solve's queue */
  CU(cudaMemsetAsync(a.rbits, 0, (size_t)nb * nwords * sizeof(unsigned), s));
  CU(cudaMemsetAsync(a.work, 0, sizeof(unsigned long long), s));
  /* the FP64 re-solve of the flagged items (stable form), after the mixed solve */
  RepairArgs r{};
  r.list = a.rlist;
  r.count = a.rcount;
  r.ilist = a.ilist;
  r.icount = a.icount;
  r.bits = a.rbits;
  r.slot = a.rslot;
  r.wstride = nwords;
  r.block = 1;
  r.rho = rho;
  r.T = T;
  r.nz = p->nz;
  r.nw = p->nw;
  r.dz = p->dz;
  r.dz1 = a64.dz1;
  r.dz2 = a64.dz2;
  r.U = a64.U, r.U_zs = a64.U_zs, r.U_is = a64.U_is;
  r.K = a64.K, r.K_zs = a64.K_zs, r.K_is = a64.K_is;
  r.V = a64.V, r.V_zs = a64.V_zs, r.V_is = a64.V_is;
  r.Vtop = a64.Vtop, r.Vbot = a64.Vbot;
  r.ld_col = a64.ld_col, r.c_off = a64.c_off, r.layout = a64.layout;
  r.lam64 = c->lam.as<double>();
  r.fully_ionized_T = p->fully_ionized_T;
  r.scratch = c->scratch.as<double>(); /* the mixed solve's */
  r.max_nz = p->nz;
  r.cap = oco_ctx_repair_slots(c, repair_capacity(c->scratch.n, p->nz, rsolve_blocks));
  r.queue = c->stats.as<unsigned long long>() + 3;
  r.repairs = c->stats.as<unsigned long long>();
  r.status = c->status.as<unsigned long long>();
  if (c->prof) CU(cudaEventRecord(e2, s));
  CU(launch_solve_mixed(a, blocks, kSolveThreads, s));
  CU(launch_repair(r, rcoef_blocks, rsolve_blocks, s));
  if (c->prof) {
    CU(cudaEventRecord(e3, s));
    c->ev_solve.emplace_back(e2, e3);
  }
  c->launches += 4;
  return OCO_OK;
}

static int run_chunk(oco_ctx *c, const oco_params *p, const double *rho, const double *T, int64_t nb,
                     SolveArgs a, cudaStream_t s) {
  if (p->form == OCO_FORM_MIXED) return run_chunk_mixed(c, p, rho, T, nb, a, s);
  const int grey = p->lgrey ? 1 : 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
  if (c->prof) {
    e0 = c->take_event();
    e1 = c->take_event();
    e2 = c->take_event();
    e3 = c->take_event();
    CU(cudaEventRecord(e0, s));
  }
  CU(launch_pillars(rho, T, nb, p->nz, p->fully_ionized_T, grey, c->pil.as<double>(), s));
  if (c->prof) {
    CU(cudaEventRecord(e1, s));
    c->ev_pil.emplace_back(e0, e1);
  }
  int blocks = 0;
  int rc = prepare_solve(c, p->form, grey, nb * p->nw, p->nz, &blocks);
  if (rc) return rc;
  size_t slots = (size_t)blocks * kSolveThreads;
  a.pil = c->pil.as<double>();
  a.lam = grey ? nullptr : c->lam.as<double>();
  a.ncol = nb;
  a.gam = c->scratch.as<double>();
  a.uu = a.gam + slots * p->nz;
  a.o1 = a.uu + slots * p->nz;
  a.q = a.o1 + slots * p->nz;
  a.slot_stride = (int64_t)slots;
  a.work = c->work.as<unsigned long long>();
  a.status = c->status.as<unsigned long long>();
  CU(cudaMemsetAsync(a.work, 0, sizeof(unsigned long long), s));
  if (c->prof) CU(cudaEventRecord(e2, s));
  CU(launch_solve_fp64(a, p->form == OCO_FORM_STABLE ? 1 : 0, grey, blocks, kSolveThreads, s));
  if (c->prof) {
    CU(cudaEventRecord(e3, s));
    c->ev_solve.emplace_back(e2, e3);
  }
  c->launches += 2;
  return OCO_OK;
}

/* status[0] = number of items with a zero pivot, status[1] = smallest such item index. */
static int reset_status(oco_ctx *c, cudaStream_t s) {
  if (c->status_pending) return OCO_OK; /* accumulate until the pending status is read */
  CU(cudaMemsetAsync(c->status.p, 0, sizeof(unsigned long long), s));
  CU(cudaMemsetAsync(c->status.as<unsigned long long>() + 1, 0xff, sizeof(unsigned long long), s));
  CU(cudaMemsetAsync(c->status.as<unsigned long long>() + 2, 0, sizeof(unsigned long long), s));
  return OCO_OK;
}

static int read_status(oco_ctx *c, cudaStream_t s, const oco_params *p) {
  unsigned long long st[3];
  c->status_pending = false;
  CU(cudaMemcpyAsync(st, c->status.p, sizeof st, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (st[2])
    return oco_set_err(c, OCO_ETIMEDOUT, "a bounded wait for a pillar copy ran out; results are incomplete");
  const bool mixed = c->status_dims_mixed;
  c->status_dims_mixed = false;
  if (st[0] && mixed)
    return oco_set_err(c, OCO_EZEROPIVOT,
                       "ERROR tridiag: bet == 0 in %llu (column, wavelength) items of pending calls with different "
                       "block dimensions; the first item's location is not known",
                       st[0]);
  if (st[0]) {
    unsigned long long item = st[1];
    long long col = (long long)(item / (unsigned long long)p->nw), iw = (long long)(item % p->nw);
    return oco_set_err(c, OCO_EZEROPIVOT,
                   "ERROR tridiag: bet == 0 in %llu (column, wavelength) items; first: ix=%lld iy=%lld iw=%lld",
                   st[0], col / p->ny + 1, col % p->ny + 1, iw + 1);
  }
  return OCO_OK;
}

static void fill_strides(SolveArgs &a, const oco_params *p, int layout, int64_t ld_col) {
  const int64_t mz = p->nz + 6, nz = p->nz;
  a.layout = layout;
  a.ld_col = ld_col;
  if (layout == OCO_LAYOUT_REFERENCE) {
    a.U_zs = 1;
    a.U_is = mz;
    a.K_zs = 1;
    a.K_is = nz;
    a.V_zs = 1;
    a.V_is = nz;
  } else {
    const int64_t items = ld_col * p->nw;
    a.U_zs = items;
    a.U_is = 1;
    a.K_zs = items;
    a.K_is = 1;
    a.V_zs = items;
    a.V_is = 1;
  }
}

/* One chunk [c0, c0 + nb) of a device solve into the caller's arrays (whole-block strides, layout
 * p->layout); reference-layout U, kappa, V go through lambda-fastest temporaries and a transpose. */
static int device_chunk(oco_ctx *c, const oco_params *p, const double *rho, const double *T, int64_t c0, int64_t nb,
                        double *U, double *kappa, double *V, double *Vtop, double *Vbot, cudaStream_t s) {
  const int64_t ncol = (int64_t)p->nx * p->ny;
  SolveArgs a{};
  a.nz = p->nz;
  a.nw = p->nw;
  a.dz = p->dz;
  a.dz1 = 1.0 / p->dz;
  a.dz2 = p->dz * p->dz;
  a.sigma_grey = p->sigma_grey;
  if (!uses_transpose(c, p, U != nullptr, kappa != nullptr, V != nullptr)) {
    fill_strides(a, p, p->layout, ncol);
    a.U = U;
    a.K = kappa;
    a.V = V;
    a.Vtop = Vtop;
    a.Vbot = Vbot;
    a.c_off = c0;
    return run_chunk(c, p, rho + c0 * p->nz, T + c0 * p->nz, nb, a, s);
  }
  const int nz = p->nz, nw = p->nw, mz = nz + 6;
  const int64_t items = nb * nw;
  if (U) CU(c->tmpU.ensure((size_t)items * mz * sizeof(double)));
  if (kappa) CU(c->tmpK.ensure((size_t)items * nz * sizeof(double)));
  if (V) CU(c->tmpV.ensure((size_t)items * nz * sizeof(double)));
  a.layout = OCO_LAYOUT_LAMBDA_FASTEST;
  a.ld_col = ncol; /* emergent planes: caller's plane, offset below */
  a.c_off = 0;
  a.U_zs = a.K_zs = a.V_zs = items;
  a.U_is = a.K_is = a.V_is = 1;
  a.U = U ? c->tmpU.as<double>() : nullptr;
  a.K = kappa ? c->tmpK.as<double>() : nullptr;
  a.V = V ? c->tmpV.as<double>() : nullptr;
  a.Vtop = Vtop ? Vtop + c0 : nullptr;
  a.Vbot = Vbot ? Vbot + c0 : nullptr;
  int rc = run_chunk(c, p, rho + c0 * p->nz, T + c0 * p->nz, nb, a, s);
  if (rc) return rc;
  if (U) CU(launch_lambda_to_reference(c->tmpU.as<double>(), items, U, ncol, c0, nb, mz, nw, c->num_sms, s));
  if (kappa) CU(launch_lambda_to_reference(c->tmpK.as<double>(), items, kappa, ncol, c0, nb, nz, nw, c->num_sms, s));
  if (V) CU(launch_lambda_to_reference(c->tmpV.as<double>(), items, V, ncol, c0, nb, nz, nw, c->num_sms, s));
  c->launches += (U ? 1 : 0) + (kappa ? 1 : 0) + (V ? 1 : 0);
  return OCO_OK;
}

extern "C" int oco_solve_block_device(oco_ctx *c, const oco_params *p, const double *rho, const double *T,
                                      double *U, double *kappa, double *V, double *Vtop, double *Vbot,
                                      void *stream) {
  int rc = check_params(c, p);
  if (rc) return rc;
  if (p->form == OCO_FORM_MIXED && p->lgrey) return oco_set_err(c, OCO_EINVAL, "the mixed form has no grey variant");
  if (!rho || !T) return oco_set_err(c, OCO_EINVAL, "rho and T are required");
  CU(cudaSetDevice(c->device));
  cudaStream_t s = (cudaStream_t)stream; /* NULL is the CUDA default stream */
  if (c->status_pending && c->status_stream != s) {
    /* the context's records, Thomas scratch and status serve one call at a time: a call on
       another stream waits for the pending one on the device (the host does not block) */
    if (!c->order_ev) CU(cudaEventCreateWithFlags(&c->order_ev, cudaEventDisableTiming));
    CU(cudaEventRecord(c->order_ev, c->status_stream));
    CU(cudaStreamWaitEvent(s, c->order_ev, 0));
  }
  const int64_t ncol = (int64_t)p->nx * p->ny;
  const int64_t ch = chunk_columns(c, p, false, U != nullptr, kappa != nullptr, V != nullptr, Vtop || Vbot);
  CU(c->pil.ensure((size_t)ch * p->nz * record_bytes(p->form)));
  if ((rc = reset_status(c, s))) return rc;
  for (int64_t c0 = 0; c0 < ncol; c0 += ch) {
    const int64_t nb = std::min(ch, ncol - c0);
    if ((rc = device_chunk(c, p, rho, T, c0, nb, U, kappa, V, Vtop, Vbot, s))) return rc;
  }
  if (!c->status_pending) {
    c->status_params = *p;
    c->status_dims_mixed = false;
  } else if (c->status_params.nx != p->nx || c->status_params.ny != p->ny || c->status_params.nw != p->nw) {
    c->status_dims_mixed = true;
  }
  c->status_pending = true;
  c->status_stream = s;
  return OCO_OK;
}

int oco_ctx_run_columns(oco_ctx *c, const oco_params *p, const double *rho, const double *T, int64_t c0, int64_t nb,
                        double *U, double *kappa, double *V, double *Vtop, double *Vbot, int max_blocks,
                        cudaStream_t s) {
  CU(c->pil.ensure((size_t)nb * p->nz * record_bytes(p->form)));
  c->max_blocks = max_blocks;
  const int rc = device_chunk(c, p, rho, T, c0, nb, U, kappa, V, Vtop, Vbot, s);
  c->max_blocks = 0;
  return rc;
}

int oco_ctx_reset_status(oco_ctx *c, cudaStream_t s) {
  c->status_pending = false;
  return reset_status(c, s);
}

int oco_ctx_read_status(oco_ctx *c, cudaStream_t s, const oco_params *p) { return read_status(c, s, p); }

int oco_ctx_check_params(oco_ctx *c, const oco_params *p) {
  const int rc = check_params(c, p);
  if (rc) return rc;
  if (p->form == OCO_FORM_MIXED && p->lgrey) return oco_set_err(c, OCO_EINVAL, "the mixed form has no grey variant");
  return OCO_OK;
}

int oco_ctx_full_blocks(oco_ctx *c, int form, int grey) {
  const int bps = form == OCO_FORM_MIXED ? solve_mixed_max_blocks_per_sm(kSolveThreads, 64)
                                         : solve_fp64_max_blocks_per_sm(form == OCO_FORM_STABLE ? 1 : 0, grey,
                                                                        kSolveThreads);
  return bps * c->num_sms;
}

extern "C" int oco_solve_block(oco_ctx *c, const oco_params *p, const double *rho, const double *T, double *U,
                               double *kappa, double *V, double *Vtop, double *Vbot) {
  int rc = check_params(c, p);
  if (rc) return rc;
  if (p->form == OCO_FORM_MIXED && p->lgrey) return oco_set_err(c, OCO_EINVAL, "the mixed form has no grey variant");
  if (!rho || !T) return oco_set_err(c, OCO_EINVAL, "rho and T are required");
  CU(cudaSetDevice(c->device));
  const int64_t ncol = (int64_t)p->nx * p->ny;
  const int nz = p->nz, nw = p->nw, mz = nz + 6;
  const int64_t ch = chunk_columns(c, p, true, U != nullptr, kappa != nullptr, V != nullptr, Vtop || Vbot);
  CU(c->pil.ensure((size_t)ch * nz * record_bytes(p->form)));
  for (auto &st : c->stage) {
    CU(st.rho.ensure((size_t)ch * nz * sizeof(double)));
    CU(st.T.ensure((size_t)ch * nz * sizeof(double)));
    if (U) CU(st.U.ensure((size_t)ch * mz * nw * sizeof(double)));
    if (kappa) CU(st.K.ensure((size_t)ch * nz * nw * sizeof(double)));
    if (V) CU(st.V.ensure((size_t)ch * nz * nw * sizeof(double)));
    if (Vtop) CU(st.top.ensure((size_t)ch * nw * sizeof(double)));
    if (Vbot) CU(st.bot.ensure((size_t)ch * nw * sizeof(double)));
  }
  if (c->status_pending && (rc = oco_synchronize(c))) return rc;
  if ((rc = reset_status(c, c->stream))) return rc;
  SolveArgs a{};
  a.nz = nz;
  a.nw = nw;
  a.dz = p->dz;
  a.dz1 = 1.0 / p->dz;
  a.dz2 = p->dz * p->dz;
  a.sigma_grey = p->sigma_grey;
  int k = 0;
  for (int64_t c0 = 0; c0 < ncol; c0 += ch, k ^= 1) {
    const int64_t nb = std::min(ch, ncol - c0);
    Stage &st = c->stage[k];
    /* the previous copy-back from this staging set must be done before reuse */
    CU(cudaStreamWaitEvent(c->stream, st.done, 0));
    CU(cudaMemcpyAsync(st.rho.p, rho + c0 * nz, (size_t)nb * nz * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    CU(cudaMemcpyAsync(st.T.p, T + c0 * nz, (size_t)nb * nz * sizeof(double), cudaMemcpyHostToDevice,
                       c->stream));
    fill_strides(a, p, OCO_LAYOUT_REFERENCE, nb);
    a.U = U ? st.U.as<double>() : nullptr;
    a.K = kappa ? st.K.as<double>() : nullptr;
    a.V = V ? st.V.as<double>() : nullptr;
    a.Vtop = Vtop ? st.top.as<double>() : nullptr;
    a.Vbot = Vbot ? st.bot.as<double>() : nullptr;
    a.c_off = 0;
    if ((rc = run_chunk(c, p, st.rho.as<double>(), st.T.as<double>(), nb, a, c->stream))) return rc;
    /* copy-back on the copy stream, after the kernels */
    cudaEvent_t ready;
    CU(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    CU(cudaEventRecord(ready, c->stream));
    CU(cudaStreamWaitEvent(c->copy, ready, 0));
    CU(cudaEventDestroy(ready));
    const size_t dp_u = (size_t)ncol * mz * sizeof(double), sp_u = (size_t)nb * mz * sizeof(double);
    if (U) CU(cudaMemcpy2DAsync(U + c0 * mz, dp_u, st.U.p, sp_u, sp_u, nw, cudaMemcpyDeviceToHost, c->copy));
    const size_t dp_k = (size_t)ncol * nz * sizeof(double), sp_k = (size_t)nb * nz * sizeof(double);
    if (kappa) CU(cudaMemcpy2DAsync(kappa + c0 * nz, dp_k, st.K.p, sp_k, sp_k, nw, cudaMemcpyDeviceToHost, c->copy));
    if (V) CU(cudaMemcpy2DAsync(V + c0 * nz, dp_k, st.V.p, sp_k, sp_k, nw, cudaMemcpyDeviceToHost, c->copy));
    const size_t dp_p = (size_t)ncol * sizeof(double), sp_p = (size_t)nb * sizeof(double);
    if (Vtop) CU(cudaMemcpy2DAsync(Vtop + c0, dp_p, st.top.p, sp_p, sp_p, nw, cudaMemcpyDeviceToHost, c->copy));
    if (Vbot) CU(cudaMemcpy2DAsync(Vbot + c0, dp_p, st.bot.p, sp_p, sp_p, nw, cudaMemcpyDeviceToHost, c->copy));
    CU(cudaEventRecord(st.done, c->copy));
  }
  CU(cudaStreamSynchronize(c->copy));
  return read_status(c, c->stream, p);
}

extern "C" int oco_synchronize(oco_ctx *c) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  CU(cudaSetDevice(c->device));
  if (c->status_pending) {
    oco_params p = c->status_params;
    int rc = read_status(c, c->status_stream, &p);
    if (rc) return rc;
  }
  CU(cudaStreamSynchronize(c->stream));
  CU(cudaStreamSynchronize(c->copy));
  return OCO_OK;
}

extern "C" int oco_set_mixed_repair(oco_ctx *c, double cond_max) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  if (!(cond_max >= 1.0)) return oco_set_err(c, OCO_EINVAL, "cond_max must be at least 1 (got %g)", cond_max);
  c->repair_cond = cond_max >= 3.0e38 ? INFINITY : (float)cond_max;
  return OCO_OK;
}

extern "C" int oco_mixed_repairs(oco_ctx *c, int64_t *items) {
  if (!c || !items) return oco_set_err(c, OCO_EINVAL, "NULL argument");
  CU(cudaSetDevice(c->device));
  if (c->status_pending) CU(cudaStreamSynchronize(c->status_stream));
  CU(cudaStreamSynchronize(c->stream));
  unsigned long long n = 0;
  CU(cudaMemcpy(&n, c->stats.p, sizeof n, cudaMemcpyDeviceToHost));
  CU(cudaMemset(c->stats.p, 0, sizeof n));
  *items = (int64_t)n;
  return OCO_OK;
}

static int epilogue_args(oco_ctx *c, const oco_params *p, EpilogueArgs &a) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  if (!p || p->nx < 1 || p->ny < 1 || p->nz < 2 || p->nw < 1)
    return oco_set_err(c, OCO_EINVAL, "bad block dimensions");
  if (p->layout != OCO_LAYOUT_REFERENCE && p->layout != OCO_LAYOUT_LAMBDA_FASTEST)
    return oco_set_err(c, OCO_EINVAL, "unknown layout %d", p->layout);
  a = EpilogueArgs{};
  a.ncol = (int64_t)p->nx * p->ny;
  a.nz = p->nz;
  a.nw = p->nw;
  a.layout = p->layout;
  a.dz = p->dz;
  return OCO_OK;
}

static int epilogue_blocks(oco_ctx *c, int64_t items) {
  const int64_t want = (items + 255) / 256, cap = (int64_t)c->num_sms * 8;
  return (int)std::max<int64_t>(1, std::min(want, cap));
}

extern "C" int oco_intensities_device(oco_ctx *c, const oco_params *p, const double *U, const double *V, double *Ip,
                                      double *Im, void *stream) {
  EpilogueArgs a;
  int rc = epilogue_args(c, p, a);
  if (rc) return rc;
  if (!U || !V || (!Ip && !Im)) return oco_set_err(c, OCO_EINVAL, "U, V and at least one of Ip, Im are required");
  a.U = U;
  a.V = V;
  a.Ip = Ip;
  a.Im = Im;
  CU(cudaSetDevice(c->device));
  CU(launch_intensities(a, epilogue_blocks(c, a.ncol * a.nw), (cudaStream_t)stream));
  c->launches++;
  return OCO_OK;
}

extern "C" int oco_optical_depth_device(oco_ctx *c, const oco_params *p, const double *kappa, const double *rho,
                                        double target_tau, double *tau, int32_t *photo_index, void *stream) {
  EpilogueArgs a;
  int rc = epilogue_args(c, p, a);
  if (rc) return rc;
  if (!kappa || !rho || (!tau && !photo_index))
    return oco_set_err(c, OCO_EINVAL, "kappa, rho and at least one of tau, photo_index are required");
  a.K = kappa;
  a.rho = rho;
  a.tau = tau;
  a.photo = photo_index;
  a.target = target_tau;
  CU(cudaSetDevice(c->device));
  CU(launch_optical_depth(a, epilogue_blocks(c, a.ncol * a.nw), (cudaStream_t)stream));
  c->launches++;
  return OCO_OK;
}

extern "C" int oco_integrated_flux_device(oco_ctx *c, const oco_params *p, const double *V, double *F, void *stream) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  if (!p || p->nx < 1 || p->ny < 1 || p->nw < 1) return oco_set_err(c, OCO_EINVAL, "bad block dimensions");
  if (p->nw != c->nw)
    return oco_set_err(c, OCO_EINVAL, "nw = %d but the context's wavelength grid has %d", p->nw, c->nw);
  if (!V || !F) return oco_set_err(c, OCO_EINVAL, "V and F are required");
  const int64_t ncol = (int64_t)p->nx * p->ny;
  CU(cudaSetDevice(c->device));
  CU(launch_integrated_flux(V, c->trapw.as<double>(), ncol, p->nw, ncol, F, epilogue_blocks(c, ncol),
                            (cudaStream_t)stream));
  c->launches++;
  return OCO_OK;
}

extern "C" int oco_check_bounded_wait(oco_ctx *c, int64_t spin_limit) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  if (spin_limit < 0 || spin_limit > (1ll << 30)) return oco_set_err(c, OCO_EINVAL, "spin_limit must be 0..2^30");
  CU(cudaSetDevice(c->device));
  CU(cudaStreamSynchronize(c->stream));
  c->status_pending = false;
  int rc = reset_status(c, c->stream);
  if (rc) return rc;
  CU(launch_bounded_wait_check(spin_limit, c->status.as<unsigned long long>(), c->stream));
  c->launches++;
  oco_params p{};
  p.nx = p.ny = p.nw = 1;
  return read_status(c, c->stream, &p);
}

extern "C" int64_t oco_kernel_launches(const oco_ctx *c) { return c ? c->launches : 0; }

extern "C" int oco_set_profiling(oco_ctx *c, int enable) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  c->prof = enable != 0;
  return OCO_OK;
}

extern "C" int oco_kernel_times(oco_ctx *c, double *solve_ms, double *pillars_ms, int64_t *solve_launches) {
  if (!c) return oco_set_err(nullptr, OCO_EINVAL, "NULL context");
  CU(cudaSetDevice(c->device));
  double ts = 0.0, tp = 0.0;
  int64_t n = (int64_t)c->ev_solve.size();
  for (auto *v : {&c->ev_solve, &c->ev_pil}) {
    for (auto &pr : *v) {
      CU(cudaEventSynchronize(pr.second));
      float ms = 0.f;
      CU(cudaEventElapsedTime(&ms, pr.first, pr.second));
      (v == &c->ev_solve ? ts : tp) += ms;
      c->ev_pool.push_back(pr.first);
      c->ev_pool.push_back(pr.second);
    }
    v->clear();
  }
  if (solve_ms) *solve_ms = ts;
  if (pillars_ms) *pillars_ms = tp;
  if (solve_launches) *solve_launches = n;
  return OCO_OK;
}
