/*
 * oco.h -- C ABI of the B200 engine for ocotillo's per-column, per-wavelength radiative
 * transfer (Saha ionization -> continuous H opacities -> Feautrier solve along z).
 *
 * The engine replaces the reference's xy/lambda loop, source/flux_feautrier.f90:160-228,
 * and the module state it reads (wavelength tables, gas-state and grey parameters, grid
 * spacing).  The caller keeps everything around that loop: namelist input, the synthetic
 * disk or Athena reader, and the output writers.
 *
 * Plain types only (int32_t, int64_t, double, pointers), so Fortran binds it with
 * ISO_C_BINDING, Python with ctypes.  All functions return 0 (OCO_OK) or a negative OCO_E*
 * code; oco_last_error() gives the message.  A context is used by one host thread at a
 * time (the reference is single-threaded); separate contexts may run concurrently.
 *
 * Array layouts
 *   OCO_LAYOUT_REFERENCE (Fortran column-major, exactly the reference's arrays):
 *     rho, T       (nz, ny, nx)        z fastest          flux_feautrier.f90:42 rho3d/temp3d
 *     U            (nz+6, ny, nx, nw)  ghosts included    flux_feautrier.f90:36
 *     kappa, V     (nz, ny, nx, nw)                       flux_feautrier.f90:37
 *     Vtop, Vbot   (ny, nx, nw)        V at z index nz (top) and 1 (bottom)
 *   OCO_LAYOUT_LAMBDA_FASTEST (device-native, coalesced for one thread per (column, lambda)):
 *     U [nz+6][ny*nx][nw], kappa and V [nz][ny*nx][nw] (C order, lambda fastest);
 *     rho, T, Vtop, Vbot as in the reference layout.
 *   Column index col = ix*ny + iy (y fastest), as in the reference's loops.
 */
#ifndef OCO_H
#define OCO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OCO_ABI_VERSION 1

/* Return codes.  The first group mirrors the reference's 'print ... ; stop' sites. */
#define OCO_OK 0
#define OCO_EINVAL (-1)      /* bad argument or dimension (nz < 2, nw < 1, NULL input, dz not
                                positive and finite, nx*ny*nw*(nz+6) above 2^56 elements) */
#define OCO_ENOMEM (-2)      /* allocation failed; flux_feautrier.f90:95-104 */
#define OCO_EZEROPIVOT (-3)  /* a Thomas pivot was exactly 0; auxiliary.f90:27-39 */
#define OCO_EGREY (-4)       /* grey RT with nw != 1; flux_feautrier.f90:84-87 */
#define OCO_ECUDA (-5)       /* CUDA runtime error */
#define OCO_ETIMEDOUT (-6)   /* a bounded wait ran out (serving loop) */
#define OCO_EAGAIN (-7)      /* result not ready yet (serving loop) */
#define OCO_EADMIT (-8)      /* job refused: its footprint exceeds the admission limit */
#define OCO_EIO (-9)         /* missing or truncated input file; read_athena.f90:112-116 */
#define OCO_EDIM (-10)       /* input dimensions do not match; read_athena.f90:124-137 */
#define OCO_ENOWAVES (-11)   /* oco_set_wavelengths was not called or nw mismatches */
#define OCO_ENAN (-12)       /* rho_floor not set; read_athena.f90:243-247 */
#define OCO_ECLOSED (-13)    /* serving loop is shut down */

/* Solver forms. */
#define OCO_FORM_PLAIN 0  /* the reference's FP64 arithmetic, operation for operation */
#define OCO_FORM_STABLE 1 /* FP64, difference-form Thomas pivots (no cancellation) */
#define OCO_FORM_MIXED 2  /* FP64 Saha; FP32 log-space opacities, pivots and back-substitution */

#define OCO_LAYOUT_REFERENCE 0
#define OCO_LAYOUT_LAMBDA_FASTEST 1

typedef struct oco_ctx oco_ctx;

/* Per-block parameters: the module state the reference's loop reads.
 *   nx, ny         nxloc, nyloc of resolution.in (columns of this block)
 *   nz, nw         resolution.in (run-time here)
 *   dz             grid spacing in cm (flux_feautrier.f90:151-154 derives dz1, dz2)
 *   sigma_grey     &input sigma_grey (cm^2/g), used when lgrey != 0
 *   fully_ionized_T  &gas_state_input fully_ionized_T (K), gas_state.f90:70-74
 *   lgrey          &input lgrey (grey RT; requires nw == 1)
 *   form           OCO_FORM_*
 *   layout         OCO_LAYOUT_* (device-array entry points only; host arrays always use
 *                  the reference layout) */
typedef struct oco_params {
  int32_t nx, ny, nz, nw;
  double dz;
  double sigma_grey;
  double fully_ionized_T;
  int32_t lgrey;
  int32_t form;
  int32_t layout;
  int32_t reserved; /* must be 0 */
} oco_params;

/* ABI version of the loaded library (OCO_ABI_VERSION). */
int oco_abi_version(void);

/* Creates a context on CUDA device `device` (streams, workspace, wavelength tables).
 * No reference counterpart: replaces the reference's module-level state and the static
 * allocations of flux_feautrier.f90:36-37, 94-104. */
int oco_create(oco_ctx **ctx, int device);

/* Releases the context and its device memory. */
void oco_destroy(oco_ctx *ctx);

/* Message of the last failed call on this context (or on this thread when ctx is NULL). */
const char *oco_last_error(const oco_ctx *ctx);

/* Linear wavelength grid in Angstrom: wa[i] = w0 + i*(w1-w0)/(nw-1); nw == 1 gives w0.
 * Replaces calc_wavelength, continuous_opacity.f90:37-62 (argument order as there). */
int oco_calc_wavelength(double w1, double w0, int32_t nw, double *wa);

/* Builds the wavelength tables (chi, nu, lambda^3, H- fits, bound-free Gaunt factors, ...)
 * for an arbitrary grid wa[nw] (Angstrom) and uploads them.  Replaces
 * pre_calc_opacity_quantities, continuous_opacity.f90:64-141.  Must precede a solve. */
int oco_set_wavelengths(oco_ctx *ctx, const double *wa_angstrom, int32_t nw);

/* The xy/lambda loop of one block on HOST arrays (reference layout), including the
 * host<->device copies.  Replaces flux_feautrier.f90:160-228 (and the stores at :205,
 * :215-216).  Any of U, kappa, V, Vtop, Vbot may be NULL (not stored).  Returns OCO_EZEROPIVOT
 * when some (column, wavelength) met an exactly zero pivot (all other results are
 * written; oco_last_error names the first such item). */
int oco_solve_block(oco_ctx *ctx, const oco_params *p, const double *rho, const double *T,
                    double *U, double *kappa, double *V, double *Vtop, double *Vbot);

/* Same loop on DEVICE arrays (p->layout selects the output layout), enqueued on `stream`
 * (a cudaStream_t; NULL is the CUDA default stream); returns after enqueueing.  Zero pivots are
 * reported by the next oco_synchronize.  Any output may be NULL.  The inputs must stay
 * valid and the outputs untouched until the stream reaches this work.  The context's work
 * buffers serve one call at a time: a call on another stream than a pending one waits for it
 * on the device (an event; the host does not block). */
int oco_solve_block_device(oco_ctx *ctx, const oco_params *p, const double *rho,
                           const double *T, double *U, double *kappa, double *V,
                           double *Vtop, double *Vbot, void *stream);

/* Waits for the context's work; returns OCO_EZEROPIVOT if a device-array solve since the
 * last call met a zero pivot.  oco_last_error names the first such item's (ix, iy, iw) when
 * every pending call had the same nx, ny and nw, and only the count otherwise. */
int oco_synchronize(oco_ctx *ctx);

/* Mixed form: the FP32 arithmetic resolves an emergent flux to ~1e-5 only where the flux is
 * well conditioned.  The flux is a weighted sum of the boundary differences of U, computed as
 * D_k = u_k - q_k U_{k+1} from non-negative terms, and its condition number is
 * sum |w_k| (u_k + q_k U_{k+1}) / |sum w_k D_k|.  The solve kernels compute it for every item
 * (top and bottom) and list the items whose condition number exceeds cond_max (and every item
 * of a column holding a cell with a negative neutral fraction, where the reference's Saha root
 * rounds above 1); a second kernel on the same stream re-solves the listed items in the stable
 * FP64 form (bit-identical to OCO_FORM_STABLE) over the mixed results.  Default 100 (the FP32
 * error grows as ~1e-5 + 2e-7 x condition number); cond_max >= 3e38 turns the re-solve off;
 * values below 1 are refused.  Block solves use the value current at the call; a batch uses the
 * value current when its graph is captured (oco_batch_bind, _tune, _set_tiling).  No reference
 * counterpart: the reference computes in FP64 only. */
int oco_set_mixed_repair(oco_ctx *ctx, double cond_max);

/* Waits for the context's work and returns in *items the number of (column, wavelength) items
 * the mixed form re-solved in FP64 since the previous call (or since creation) in the
 * context's block solves and batches; resets the count.  Batches replayed on other streams
 * must have been waited for (oco_batch_wait). */
int oco_mixed_repairs(oco_ctx *ctx, int64_t *items);

/* Number of kernel launches this context has issued since creation (for accounting). */
int64_t oco_kernel_launches(const oco_ctx *ctx);

/* Kernel timing: when enabled, every pillar and solve launch is bracketed by CUDA events
 * on its stream.  oco_kernel_times waits for the recorded launches, returns the summed
 * durations (ms) and the number of solve launches since the last call, and resets them. */
int oco_set_profiling(oco_ctx *ctx, int enable);
int oco_kernel_times(oco_ctx *ctx, double *solve_ms, double *pillars_ms, int64_t *solve_launches);

/* Upward and downward intensities of a block solved on the device: Ip = U + V, Im = U - V on
 * the interior z (auxiliary.f90:80-94, calc_intensity, which the reference keeps but does not
 * call).  U, V, Ip, Im are device arrays in p->layout (Ip and Im shaped like V; either may be
 * NULL); enqueued on `stream`. */
int oco_intensities_device(oco_ctx *ctx, const oco_params *p, const double *U, const double *V, double *Ip,
                           double *Im, void *stream);

/* Optical depth and photosphere of a block solved on the device, as the reference's analysis
 * tools define them (tools/ocoutils/ReadOcotillo.py:248-293): tau(z) = cumulative sum from z
 * index 1 of kappa * rho * dz (kappa as the solve wrote it, rho the block's input), and per
 * (column, wavelength) the first 0-based z index with tau >= target_tau, or -1.  kappa and
 * tau in p->layout, rho (nz, ny, nx), photo_index (ny, nx, nw) like Vtop; tau or photo_index
 * may be NULL.  Enqueued on `stream`. */
int oco_optical_depth_device(oco_ctx *ctx, const oco_params *p, const double *kappa, const double *rho,
                             double target_tau, double *tau, int32_t *photo_index, void *stream);

/* Wavelength-integrated emergent flux of a block solved on the device: for an emergent-flux
 * plane V laid out like Vtop / Vbot (ny, nx, nw), F[col] = sum over the context's wavelength
 * grid of the trapezoid rule in lambda (cm), (ny, nx) values; summed in increasing wavelength
 * index with weights from oco_set_wavelengths (a single wavelength gives 0).  p->nw must equal
 * the context's grid.  No reference counterpart (the bolometric flux of each column).
 * Enqueued on `stream`. */
int oco_integrated_flux_device(oco_ctx *ctx, const oco_params *p, const double *V, double *F, void *stream);

/* ---- Synthetic disk inputs ---------------------------------------------------------------
 * The reference's synthetic disk (source/disk.f90:42-129: calc_grid, calc_density with its
 * floor, calc_temperature with switchTemp = (1 + 2^-52)*isoTemp, the Gaussian and the floor),
 * every column the same profile, times a seeded lognormal perturbation of the density per cell
 * (10^(sigma_dex*N), N standard normal from Philox4x32-10 keyed by seed and counted by cell;
 * sigma_dex = 0: none).  The reference evaluates exp with the C library; here both builds use
 * the library's correctly rounded exp so that host and device give the same bits. */
typedef struct oco_disk_params {
  int32_t nx, ny, nz;
  int32_t reserved;  /* must be 0 */
  double z0, z1;     /* &input z0, z1 (cm): the grid of calc_grid */
  double rho0, H, rho_floor;                   /* &density_input */
  double midTemp, sigma, floorTemp, isoTemp;   /* &temperature_input */
  double sigma_dex;  /* lognormal density perturbation (dex) */
  uint64_t seed;
} oco_disk_params;

/* Fills host arrays rho, T (nz, ny, nx) and *dz (may be NULL).  No GPU needed. */
int oco_disk_inputs(const oco_disk_params *p, double *rho, double *T, double *dz);

/* Same on device arrays, enqueued on `stream`; bit-identical to oco_disk_inputs. */
int oco_disk_inputs_device(oco_ctx *ctx, const oco_disk_params *p, double *rho, double *T, void *stream);

/* Diagnostic of the failure path: runs the kernels' bounded wait (the mbarrier poll the
 * solve kernels use for their shared-memory copies) on a barrier phase that nothing
 * completes, polling spin_limit times.  Returns OCO_ETIMEDOUT when the wait ran out, as a
 * solve does, with the context still usable.  No reference counterpart. */
int oco_check_bounded_wait(oco_ctx *ctx, int64_t spin_limit);

/* ---- Solve without device allocation ----------------------------------------------------
 * No counterpart in the reference (whose loop allocates nothing on a GPU): this entry point
 * serves callers that cannot call cudaMalloc -- hosts that own the device heap, plugins not
 * allowed to allocate after start-up, drivers with a fixed GPU-memory budget.  It runs the
 * same kernels as oco_solve_block_device, on the calling thread's current device, with all
 * intermediate data (pillars, Thomas scratch, wavelength table, counters) in one static
 * device array of OCO_NOALLOC_WORKSPACE_BYTES that every GPU loading the library holds until
 * the process exits.  The caller passes the wavelengths (Angstrom), the device inputs and
 * the device outputs (layout p->layout).  No context, no cudaMalloc/cudaFree, no allocating
 * library call.  The first call on a device looks up the array's device address (do it
 * before any stream capture).  Calls on a device share its array, so calls whose GPU work
 * overlapped would race: each call holds a per-device lock until its work on `stream` is done,
 * and returns only then (also on an error after work was enqueued).  Any of U, kappa, V, Vtop,
 * Vbot may be NULL (not stored), as for oco_solve_block_device.  Limits: nz <=
 * OCO_NOALLOC_MAX_NZ together with nw <= OCO_NOALLOC_MAX_NW always fit (the library checks this
 * at compile time), forms PLAIN and STABLE; larger sizes return OCO_EINVAL.
 * Errors: oco_noalloc_last_error(). */
#define OCO_NOALLOC_WORKSPACE_BYTES (32u << 20)
#define OCO_NOALLOC_MAX_NZ 4096
#define OCO_NOALLOC_MAX_NW 4096
int oco_solve_block_noalloc(const oco_params *p, const double *wa_angstrom, const double *rho,
                            const double *T, double *U, double *kappa, double *V, double *Vtop,
                            double *Vbot, void *stream);
const char *oco_noalloc_last_error(void);

/* ---- Ragged batches ---------------------------------------------------------------------
 * No counterpart in the reference, whose loop runs one block with one nz and one wavelength
 * grid: a batch is a set of independent columns, each with its own nz, dz and wavelength
 * grid (for instance columns of several snapshots), solved by one persistent launch fed from
 * a device work queue and replayed as a CUDA graph.  Per column the arithmetic is that of
 * oco_solve_block_device with p->form set to the batch's form (plain, stable or mixed).
 *
 * Array layout (device arrays, element offsets given per column):
 *   rho, T      nz values from in_off (z fastest), read-only
 *   U           from u_off: (nz+6) x nw values, [lambda][z] (z fastest) for
 *               OCO_LAYOUT_REFERENCE, [z][lambda] for OCO_LAYOUT_LAMBDA_FASTEST
 *   kappa, V    from kv_off: nz x nw values, same order as U
 *   Vtop, Vbot  from flux_off: nw values (V at z index nz and 1)
 * Output ranges of different columns must not overlap (oco_batch_bind checks this for the
 * arrays it is given); offsets are at most 2^56. */
typedef struct oco_batch oco_batch;

typedef struct oco_batch_column {
  int64_t in_off;   /* first element (z = 1) of the column's rho and T profiles */
  int64_t u_off;    /* first element of the column's U block */
  int64_t kv_off;   /* first element of the column's kappa and V blocks */
  int64_t flux_off; /* first element of the column's Vtop and Vbot entries */
  int64_t wave_off; /* first wavelength (Angstrom) of the column's grid in `waves` */
  int32_t nz;       /* >= 2 */
  int32_t nw;       /* >= 1 */
  double dz;        /* grid spacing, cm */
} oco_batch_column;

/* Tilings (oco_batch_info.tiling). */
#define OCO_TILING_WARP_COLUMN 0 /* a warp solves 32 wavelengths of one column */
#define OCO_TILING_PACKED 1      /* a warp solves 32 consecutive items of the nz-sorted item list */

typedef struct oco_batch_info {
  int64_t ncol;          /* columns */
  int64_t npoints;       /* sum of nz * nw */
  int32_t max_nz, max_nw;
  int32_t tiling;        /* OCO_TILING_* in use */
  int32_t blocks_per_sm; /* resident 128-thread blocks per SM of the persistent launch */
  int32_t tuned;         /* 1 after oco_batch_tune */
  int32_t ncandidates;   /* tilings timed by oco_batch_tune */
  int32_t cand_tiling[16];
  int32_t cand_blocks_per_sm[16];
  double cand_ms[16];    /* one timed run of each candidate */
  int64_t graph_launches; /* oco_batch_run calls so far */
} oco_batch_info;

/* Describes a batch of ncol columns on the context's device: validates the descriptors,
 * builds one wavelength table per distinct (wave_off, nw) grid from waves[nwaves] (Angstrom,
 * host memory), sorts the work longest column first and reserves the device workspace.
 * form is OCO_FORM_PLAIN, OCO_FORM_STABLE (per item the block solve's FP64 arithmetic, so
 * the same bits) or OCO_FORM_MIXED; layout is OCO_LAYOUT_*. */
int oco_batch_create(oco_ctx *ctx, const oco_batch_column *cols, int64_t ncol, const double *waves,
                     int64_t nwaves, int32_t form, int32_t layout, double fully_ionized_T,
                     oco_batch **batch);

/* Binds the device arrays (element counts for the bounds check of every column's ranges)
 * and captures the batch's launches into a CUDA graph.  U, kappa, V, Vtop, Vbot may be NULL
 * (not stored; their count is then ignored).  OCO_EINVAL when a bound output array's
 * ranges of two columns overlap (the message names the pair).  Rebinding recaptures. */
int oco_batch_bind(oco_batch *batch, const double *rho, const double *T, int64_t n_in, double *U,
                   int64_t n_u, double *kappa, double *V, int64_t n_kv, double *Vtop, double *Vbot,
                   int64_t n_flux);

/* Autotuner: runs the bound batch once per candidate tiling (tiling x resident blocks per
 * SM), keeps the fastest and recaptures the graph with it.  Writes the outputs as a run
 * does.  Synchronous. */
int oco_batch_tune(oco_batch *batch);

/* Sets the tiling by hand (instead of oco_batch_tune): tiling OCO_TILING_*, blocks_per_sm
 * from 1 to the kernel's occupancy limit (0 = that limit).  Recaptures the graph if bound.
 * OCO_TILING_PACKED is available for the mixed form only. */
int oco_batch_set_tiling(oco_batch *batch, int32_t tiling, int32_t blocks_per_sm);

/* Replays the batch's graph on `stream` (a cudaStream_t; NULL is the CUDA default stream):
 * records, then every (column, wavelength) item.  Returns after enqueueing; the bound inputs
 * must stay valid and the outputs untouched until the stream reaches this work.  Replays share
 * the batch's work queue, so a replay on another stream than the pending one waits for it on
 * the device (an event; the host does not block). */
int oco_batch_run(oco_batch *batch, void *stream);

/* Waits for the last oco_batch_run; returns OCO_ETIMEDOUT if a bounded wait in the kernel
 * ran out (its results are then incomplete), and for the plain form OCO_EZEROPIVOT when some
 * item met an exactly zero Thomas pivot (every item is still computed, as in
 * oco_solve_block; the message names the first column and wavelength). */
int oco_batch_wait(oco_batch *batch);

int oco_batch_get_info(const oco_batch *batch, oco_batch_info *info);

/* Releases the batch (waits for its work first). */
void oco_batch_destroy(oco_batch *batch);

/* ---- Serving loop -----------------------------------------------------------------------
 * No counterpart in the reference (a batch program that solves one snapshot per run): a
 * server owns one device and a scheduler thread that takes post-processing jobs (a block of
 * columns plus its wavelength grid, as for oco_solve_block_device) as they arrive.  Jobs are
 * admitted first come first served while a job slot is free and the summed device footprint
 * of admitted jobs stays within the budget; an admitted job's inputs, results and wavelength
 * tables stay in HBM.  Continuous batching: every admitted job is cut into launches of about
 * chunk_points mesh*lambda points, and the scheduler keeps two launches in flight per job on
 * the job's own stream, each persistent grid sized to the job's share of the GPU (full grid /
 * running jobs), so the work of a job that arrives while others run starts at once and
 * overlaps theirs on the device.  Results do not depend on the mix: every (column, lambda)
 * item runs the same arithmetic whatever grid runs it.
 * Thread safety: all functions may be called from any thread. */
typedef struct oco_server oco_server;

typedef struct oco_server_config {
  int32_t device;
  int32_t max_jobs;      /* job slots (jobs running at once), >= 1 */
  int32_t max_nz;        /* workspace is sized for nz <= max_nz at creation (larger nz grows it) */
  int32_t reserved;      /* must be 0 */
  double budget_bytes;   /* admission limit on the summed footprint of admitted jobs;
                          * 0: 85% of the device memory free after the workspace */
  int64_t chunk_points;  /* mesh*lambda points per launch; 0: 2^28 */
  double reserve_bytes;  /* device memory for job arrays mapped at creation, so that the first
                          * admissions do not wait for the allocator to grow (0: none) */
} oco_server_config;

typedef struct oco_job {
  int32_t nx, ny, nz, nw;
  double dz;
  double fully_ionized_T;
  int32_t form;            /* OCO_FORM_PLAIN, _STABLE or _MIXED (non-grey) */
  int32_t want_fields;     /* 1: keep U, kappa and V as well as the emergent flux */
  const double *rho, *T;   /* (nz, ny, nx) reference layout, host or device memory (complete
                            * when submitted); must stay valid until inputs_consumed is set */
  const double *waves;     /* nw wavelengths (Angstrom), host memory, copied by submit */
} oco_job;

#define OCO_JOB_QUEUED 0
#define OCO_JOB_RUNNING 1
#define OCO_JOB_DONE 2
#define OCO_JOB_FAILED 3

typedef struct oco_job_status {
  int32_t state;           /* OCO_JOB_* */
  int32_t error;           /* OCO_E* of a failed job (or OCO_EZEROPIVOT on a done job with zero pivots) */
  int32_t inputs_consumed; /* the job no longer reads rho and T */
  int32_t reserved;
  int64_t bytes;           /* device footprint counted by admission */
  double submit_s, admit_s, done_s; /* host monotonic clock, seconds (0 until reached) */
} oco_job_status;

int oco_server_create(const oco_server_config *cfg, oco_server **server);

/* Queues a job; returns its id in *job_id.  OCO_EADMIT if its footprint can never fit the
 * budget, OCO_ECLOSED after oco_server_destroy began. */
int oco_server_submit(oco_server *server, const oco_job *job, int64_t *job_id);

int oco_server_status(oco_server *server, int64_t job_id, oco_job_status *status);

/* Waits up to timeout_s seconds for the job to finish: OCO_OK when done, OCO_EAGAIN on
 * timeout, the job's error when it failed. */
int oco_server_wait(oco_server *server, int64_t job_id, double timeout_s);

/* Copies a done job's results into host arrays (reference layout: Vtop, Vbot (ny, nx, nw);
 * U (nz+6, ny, nx, nw), kappa and V (nz, ny, nx, nw) when the job kept its fields; any may be
 * NULL), then releases the job and its device memory.  OCO_EAGAIN while the job is not done or
 * another call is fetching it; a failed copy leaves the job done and fetchable. */
int oco_server_fetch(oco_server *server, int64_t job_id, double *Vtop, double *Vbot, double *U, double *kappa,
                     double *V);

/* Stops accepting jobs, fails the queued ones with OCO_ECLOSED, finishes the running ones,
 * joins the scheduler and releases everything (results not fetched are dropped). */
void oco_server_destroy(oco_server *server);

/* Message of the last failed server call on this thread. */
const char *oco_server_last_error(void);

/* ---- Decks: the reference's driver around the loop --------------------------------------
 * A deck is a run directory of the reference: input.in (namelists &input, &temperature_input,
 * &density_input, &gas_state_input, &athena_input), resolution.in (the Fortran include of
 * integer parameters nx, ny, nz, nw, nprocx, nprocy, nprocz, nxloc, nyloc; read at run time
 * here) and, when lread_athena, the Athena snapshot under datadir.  Replaces the main program
 * flux_feautrier.f90:1-269 with the xy/lambda loop on the GPU. */
typedef struct oco_deck_info {
  int32_t nx, ny, nz, nw;
  int32_t nprocx, nprocy, nprocz;
  int32_t nxloc, nyloc;
  int32_t lgrey, lread_athena, reserved;
  double dz;               /* grid spacing of the block (0 if its inputs were not built) */
  double sigma_grey;
  double fully_ionized_T;
} oco_deck_info;

/* Builds processor block (iprocx, iprocy)'s inputs as the reference does: the synthetic disk
 * (disk.f90:42-129) or the Athena reader (read_athena.f90:64-291).  rho and T (may be NULL:
 * then only *info and wa are filled) receive (nz, nyloc, nxloc) values, wa the nw wavelengths
 * (calc_wavelength), z (may be NULL) the nz+6 grid with ghosts.  Host only, no GPU needed.
 * snapshot NULL or "" is "0000". */
int oco_deck_block_inputs(const char *deck_dir, const char *snapshot, int32_t iprocx, int32_t iprocy,
                          oco_deck_info *info, double *rho, double *T, double *wa, double *z);

/* Same block inputs delivered into DEVICE arrays rho, T (nz, nyloc, nxloc) on the context's
 * device (info, wa and z as above, host memory).  For an Athena deck the snapshot goes from disk
 * to HBM: the host streams each z-block file's raw fields through pinned memory and the device
 * reassembles the block and applies the reader's physics (read_athena.f90:101-277, calc_temperature
 * disk.f90:64-109), bit-identical to oco_deck_block_inputs; a synthetic-disk deck is built on
 * the host and copied.  Returns when the arrays are complete (uses `stream`). */
int oco_deck_block_inputs_device(oco_ctx *ctx, const char *deck_dir, const char *snapshot, int32_t iprocx,
                                 int32_t iprocy, oco_deck_info *info, double *rho, double *T, double *wa, double *z,
                                 void *stream);

/* Runs a deck: every processor block solved on CUDA device `device` in form `form`, writing
 * into out_dir (NULL or "": deck_dir/output) what the reference writes into output/:
 * diagnostics.txt (io.f90:31-46, gfortran Ew.d editing), zgrid.txt/.bin and wavegrid.txt/.bin
 * (io.f90:48-75) and, when write_binary, procx<i>_procy<j>/{mean_intensity,
 * absorption_coefficients,flux}_<snapshot>.bin as Fortran unformatted sequential records
 * (io.f90:77-101).  Returns OCO_EZEROPIVOT (after writing everything) where the reference
 * would stop at a zero pivot.  Messages: oco_deck_last_error(). */
int oco_run_deck(const char *deck_dir, const char *snapshot, const char *out_dir, int32_t form, int32_t device,
                 int32_t write_binary);

/* gfortran Ew.d editing of v into out (w characters + NUL); the `0.ddddd-ddd` form for
 * three-digit exponents, asterisks when the value does not fit. */
void oco_format_e(double v, int32_t w, int32_t d, char *out);

/* Message of the last failed deck call on this thread. */
const char *oco_deck_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* OCO_H */
