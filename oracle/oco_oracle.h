/*
 * oco_oracle.h -- CPU restatement of ocotillo's per-column, per-wavelength radiative
 * transfer (the reference's xy/lambda loop), used ONLY as the checker of the GPU path.
 *
 * TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load this code.  The product (ocotillo_b200/) never links or calls it.
 *
 * The reference (Fortran 90, all REAL promoted to double by -fdefault-real-8) cannot be
 * compiled here (no Fortran compiler), so this file restates it in C99 with the same
 * operation order, no FMA contraction (-ffp-contract=off) and the reference's lowering of
 * integer powers.  Three back-ends are built from the same source:
 *   - glibc    (no macro): exp/log/log10/pow from the C library, as the gfortran-built
 *              reference calls them;
 *   - ocomath  (OCO_ORACLE_OCOMATH): the project's correctly rounded functions, which the GPU
 *              kernels also use, for bit-for-bit comparisons;
 *   - longdouble (OCO_ORACLE_LONGDOUBLE): the per-column and per-item work in long double
 *              (x87 extended) arithmetic with glibc's long double functions, on the same double
 *              inputs, wavelength tables and constants; it measures the rounding error of the
 *              double forms (oracle_math_backend() returns 2).
 * Only calls inside the xy/lambda loop switch back-ends; the once-per-run wavelength tables
 * and the input construction (disk model, Athena reader) use glibc in both, as the product's
 * host code does.
 *
 * Pinning: the four samples/<deck>/reference.out golden files of the reference are
 * reproduced text-exactly by oco_oracle_run_deck() (tests/test_oracle_golden.py).
 */
#ifndef OCO_ORACLE_H
#define OCO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Solver forms. */
#define ORACLE_FORM_REFERENCE 0 /* the reference's Thomas recursion, auxiliary.f90:14-47 */
#define ORACLE_FORM_STABLE 1    /* same system: difference-form pivots, 1 - albedo from the absorption
                                 * terms, flux from the differences of U (no cancellation) */

/* Error codes (same values as the product's include/oco.h). */
#define ORACLE_OK 0
#define ORACLE_EINVAL (-1)
#define ORACLE_ENOMEM (-2)
#define ORACLE_EZEROPIVOT (-3)
#define ORACLE_EGREY (-4)
#define ORACLE_EIO (-9)
#define ORACLE_EDIM (-10)
#define ORACLE_ENAN (-12)

typedef struct oracle_params {
  int32_t nx, ny, nz, nw;
  double dz;
  int32_t lgrey;
  int32_t form;
  double sigma_grey;
  double fully_ionized_T;
} oracle_params;

/* 0 = glibc, 1 = ocomath, 2 = longdouble. */
int oracle_math_backend(void);

/* calc_wavelength, continuous_opacity.f90:37-62. */
void oracle_calc_wavelength(double w1, double w0, int32_t nw, double *wa);

/*
 * The xy/lambda loop, flux_feautrier.f90:160-228, for one block.
 *   rho, T : (nz, ny, nx) Fortran order (z fastest)
 *   U      : (nz+6, ny, nx, nw), kappa and V : (nz, ny, nx, nw); each may be NULL.
 * Returns ORACLE_OK, or ORACLE_EZEROPIVOT when a Thomas pivot is exactly zero (the
 * reference prints and stops there; this function records the first such (column,
 * wavelength) in *bad_item = col*nw + iw and continues).
 */
int oracle_solve_block(const oracle_params *p, const double *wa, const double *rho,
                       const double *T, double *U, double *kappa, double *V,
                       int64_t *bad_item);

/* Same loop for a contiguous range of columns [col0, col1) of the block (for sampling). */
int oracle_solve_columns(const oracle_params *p, const double *wa, const double *rho,
                         const double *T, int64_t col0, int64_t col1, double *U,
                         double *kappa, double *V, int64_t *bad_item);

/* Runs a reference sample deck (input.in, resolution.in, input_athena/) from deck_dir and
 * writes <out_dir>/diagnostics.txt exactly as io.f90:31-46 does.  Returns 0 on success. */
int oracle_run_deck(const char *deck_dir, const char *out_dir, char *msg, int msglen);

/* gfortran Ew.d editing of one value into out (w characters + NUL). */
void oracle_format_e(double v, int w, int d, char *out);

#ifdef __cplusplus
}
#endif
#endif
