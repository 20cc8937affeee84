/*
 * oco_internal.h -- device data layouts and kernel entry points shared by the runtime
 * (oco_api.cu) and the kernel translation units.
 */
#ifndef OCO_INTERNAL_H
#define OCO_INTERNAL_H

#include <cstdint>

#include <cuda_runtime.h>

namespace oco {

/* Whether a block's largest array (U, nx*ny*nw*(nz+6) elements) stays within 2^56 elements,
 * the limit the entry points accept: every element index and byte count of the host code and
 * the kernels then fits int64.  Computed in double, whose rounding only blurs the bound. */
inline bool block_elements_fit(int nx, int ny, int nz, int nw) {
  return (double)nx * (double)ny * (double)nw * ((double)nz + 6.0) <= 72057594037927936.0;
}

/* Per-(column, z) quantities written by the pillar kernel and read by the solve kernels:
 * the wavelength-independent part of the reference's per-(z, lambda) work
 * (gas_state.f90:30-110 plus every factor of continuous_opacity.f90 that depends on z
 * only).  Layout [col][z][NF] doubles. */
enum PillarField {
  F_RHO = 0,   /* rho */
  F_RHO1,      /* 1/rho */
  F_T1,        /* 1/T */
  F_DFT1,      /* damping_factor_const*T1 (source function, c_o :399) */
  F_THETA,     /* 5040/T */
  F_TH1L,      /* theta1*log10e (H free-free Gaunt factor, c_o :264) */
  F_LGT,       /* log10(theta) */
  F_LGT2,      /* log10(theta)**2 */
  F_IONF,      /* nHI/(nHI+nHII) */
  F_ESCAT,     /* Thomson cross-section per H (c_o :149) */
  F_ESCM,      /* e_scatter*mp1 (albedo numerator, c_o :195) */
  F_HMBF,      /* H- bound-free factor (c_o :161) */
  F_NEUTRAL,   /* 1 if (1 - NHII/N) > switch_ionfraction else 0 (c_o :262) */
  F_E1,        /* exp(-chi_n(n)*k1*T1), n = 1..6 (c_o :238) */
  F_E2,
  F_E3,
  F_E4,
  F_E5,
  F_E6,
  F_UNSOLD,    /* Unsold integral (c_o :242) */
  F_AFF,       /* ionf*ne*k*T (H- free-free prefactor, c_o :339) */
  F_EF,        /* H free-free energy factor (c_o :265) */
  F_TPOW,      /* (T*1e-4)**(-1.5) (bremsstrahlung Gaunt factor, c_o :290) */
  F_LZ,        /* log(ne*(nHI+nHII)) + 2*log(1) - 0.5*log(T) (c_o :292-294) */
  F_LNRHO,     /* log(rho) (mixed form) */
  F_PAD,
  NF
};
/* Grey RT re-uses the slots (continuous_opacity.f90:377-390). */
enum GreyField { G_RHO = F_RHO, G_S = F_RHO1, G_ALPHA = F_T1 };

/* Per-wavelength quantities: continuous_opacity.f90:64-141 plus every factor of the hot
 * loop that depends on lambda only.  Layout [NL][nw]. */
enum LambdaField {
  L_CHI = 0,   /* chi = 1.2398e4/wa */
  L_CHI1,      /* 1/chi */
  L_GFF,       /* gff_factor */
  L_WA3,       /* wa**3 */
  L_SCOEF,     /* H- bound-free fit s_coeff */
  L_HMON,      /* 1 if wa < 16000 (H- bound-free active) else 0 */
  L_F1, L_F2, L_F3,  /* H- free-free fit f_coeff(iw, 1..3) */
  L_GN1, L_GN2, L_GN3, L_GN4, L_GN5, L_GN6, /* g(iw,n)*n1_array(n)**3 */
  L_NU9,       /* nu*1e-9 */
  L_L3NU,      /* 3*log(nu) */
  L_HNUK,      /* h*nu*k1 */
  L_WCM1,      /* 1/wcm */
  L_SW5,       /* source_function_const*w1cm5 */
  L_LNSW5,     /* log(source_function_const*w1cm5) (mixed form) */
  NL
};

/* Arguments of the FP64 solve kernels (plain and stable forms, grey or not). */
struct SolveArgs {
  const double *pil; /* [ncol][nz][NF] pillars of this chunk */
  const double *lam; /* [NL][nw] */
  int64_t ncol;      /* columns in this chunk */
  int nz, nw;
  double dz, dz1, dz2, sigma_grey;
  /* Outputs: element (z, item) lives at base + z*zs + idx*is, where idx is the column-major
   * item index of the destination:
   *   layout REFERENCE:       idx = iw*ld_col + c_off + cl
   *   layout LAMBDA_FASTEST:  idx = (c_off + cl)*nw + iw                              */
  double *U;
  int64_t U_zs, U_is;
  double *K;
  int64_t K_zs, K_is;
  double *V;
  int64_t V_zs, V_is;
  double *Vtop, *Vbot; /* [iw*ld_col + c_off + cl] */
  int64_t ld_col, c_off;
  int layout;
  /* Scratch [warp slot][nz][32] each (slot_stride*nz values): forward-sweep gamma, u,
   * 1/kappa and (stable form) q, one contiguous block per warp. */
  double *gam, *uu, *o1, *q;
  int64_t slot_stride; /* resident threads the scratch is sized for (each warp's block is 32*nz) */
  unsigned long long *work;   /* persistent-kernel work counter (warp tasks) */
  unsigned long long *status; /* [0] zero-pivot count, [1] first bad item (min), [2] timeout flag */
};

/* Arguments of the mixed-precision solve kernels. */
struct MixedArgs {
  const float *rec; /* [ncol][nz][MIXED_ZN] mixed records of this chunk */
  const float *lam; /* [MIXED_LN][nw] */
  int64_t ncol;
  int nz, nw;
  double dz;
  float ldz2i, ldz2f; /* log2(dz^2) = integer + fraction */
  double *U;
  int64_t U_zs, U_is;
  double *K;
  int64_t K_zs, K_is;
  double *V;
  int64_t V_zs, V_is;
  double *Vtop, *Vbot;
  int64_t ld_col, c_off;
  int layout;
  float4 *s4; /* scratch [warp slot][nz][32]: |gamma| or q, 1/kappa, u mantissa, u exponent (int bits) */
  int64_t slot_stride; /* resident threads the scratch is sized for */
  unsigned long long *work;
  unsigned long long *status;
  /* Items whose emergent flux the FP32 arithmetic cannot resolve are appended to ilist
   * (chunk-local id cl*nw + iw; *icount of them) and set their bit in
   * rbits[cl * ceil(nw/32) + iw/32] (cleared by the caller); each word that receives a bit is
   * appended once to rlist (*rcount of them).  Both lists feed the FP64 re-solve (RepairArgs). */
  float repair_cond;           /* flag when the boundary-flux condition number exceeds this */
  const unsigned *colflag;     /* [ncol] columns flagged entirely (record kernel) */
  unsigned *rbits;
  int *rslot;              /* [word * 32 + bit]: the flagged item's index in ilist */
  unsigned long long *rlist, *rcount, *ilist, *icount;
};

/* One column of a ragged batch as the batch kernels see it (built from oco_batch_column). */
struct MBatchCol {
  int64_t in_off;   /* rho/T of z = 0 in the bound input arrays */
  int64_t rec_off;  /* first mixed record of the column (dense prefix of nz) */
  int64_t u_off;    /* first U element of the column */
  int64_t kv_off;   /* first kappa / V element */
  int64_t flux_off; /* first emergent-flux element */
  int64_t lam_off;  /* first element of the column's wavelength table ([MIXED_LN][nw] floats or [NL][nw] doubles) */
  int32_t nz, nw;
  float dzf;        /* dz */
  float ldz2i, ldz2f; /* log2(dz^2) = integer + fraction */
  double dz1;       /* 1/dz */
  double dz, dz2;   /* dz and dz*dz (FP64 forms, flux_feautrier.f90:151-154) */
};

/* Arguments of the ragged-batch kernels (mixed form). */
struct MixedBatchArgs {
  const float *rec;        /* [sum nz][MIXED_ZN] */
  const float *lam;        /* packed wavelength tables */
  const MBatchCol *cols;
  const uint2 *tasks;      /* warp-column tiling: (column, 32-wavelength tile), longest first */
  const int32_t *order;    /* packed tiling: columns, longest first */
  const int64_t *item_pre; /* packed tiling: prefix sums of nw over order, ncol + 1 entries */
  int64_t ncol, ntasks, nitems;
  double *U, *K, *V, *Vtop, *Vbot;
  int layout;
  float4 *s4;        /* scratch: per warp slot max_nz levels of 32 12-byte records (MScratch12) */
  int64_t slot_stride; /* resident threads the scratch is sized for */
  int max_nz;
  unsigned long long *work;
  unsigned long long *status;
  /* flagged items as in MixedArgs: item id (column << 32) | wavelength, word
   * rbits[col * rwstride + iw/32] */
  float repair_cond;
  const unsigned *colflag; /* [ncol] columns flagged entirely */
  unsigned *rbits;
  int *rslot;              /* [word * 32 + bit]: the flagged item's index in ilist */
  int rwstride;            /* ceil(max nw / 32) */
  unsigned long long *rlist, *rcount, *ilist, *icount;
};

/* The FP64 re-solve (stable form) of the items the mixed kernels flagged (kernels_repair.cu):
 * k_repair_coef computes the items' row coefficients in parallel over (listed word, chunk of
 * levels) into one slot per item, k_repair_solve runs each item's recurrences, one lane per
 * slot; a re-solved item equals the stable FP64 form bit for bit and is stored over the mixed
 * one.  block != 0: items of a block chunk (the outputs as in SolveArgs); otherwise items of a
 * ragged batch (the outputs as in FP64BatchArgs). */
struct RepairArgs {
  const unsigned long long *list, *count;   /* listed words: index col * wstride + word into bits */
  const unsigned long long *ilist, *icount; /* listed items (ids as in MixedArgs / MixedBatchArgs); index = slot */
  const unsigned *bits;
  const int *slot;                          /* [word * 32 + bit]: the item's index in ilist */
  int64_t wstride;
  int block;
  /* block chunk */
  const double *rho, *T; /* the chunk's inputs [ncol][nz] */
  int nz, nw;
  double dz, dz1, dz2;
  double *U, *K, *V, *Vtop, *Vbot;
  int64_t U_zs, U_is, K_zs, K_is, V_zs, V_is, ld_col, c_off;
  int layout;
  /* batch */
  const MBatchCol *cols;   /* lam_off indexes the mixed tables: the FP64 table starts at lam_off / MIXED_LN * NL */
  /* both */
  const double *lam64;     /* [NL][nw] (block) or packed tables (batch) */
  double fully_ionized_T;
  double *scratch;         /* the mixed solve's scratch: cap slots x 5 x max_nz doubles, then per
                              k_repair_solve warp 4 x max_nz doubles (repair_capacity) */
  int64_t cap;             /* slots: items beyond are re-solved one warp per item */
  int max_nz;
  unsigned long long *queue;   /* k_repair_coef's task counter, zero at launch */
  unsigned long long *repairs; /* += the re-solved items */
  unsigned long long *status;  /* zero-pivot words as in SolveArgs */
};
/* Threads per block of k_repair_solve. */
constexpr int REPAIR_THREADS = 64;
constexpr int REPAIR_SOLVE_BLOCKS_PER_SM = 6;
constexpr int REPAIR_COEF_BLOCKS_PER_SM = 4;
/* Slots that a scratch of scratch_bytes holds beside k_repair_solve's per-warp arrays. */
int64_t repair_capacity(size_t scratch_bytes, int max_nz, int solve_blocks);
cudaError_t launch_repair(const RepairArgs &a, int coef_blocks, int solve_blocks, cudaStream_t s);

/* Arguments of the ragged-batch kernels (plain and stable FP64 forms; warp-column tiling). */
struct FP64BatchArgs {
  const double *pil;       /* [sum nz][NF] records */
  const double *lam;       /* packed [NL][nw] wavelength tables */
  const MBatchCol *cols;
  const uint2 *tasks;      /* (column, 32-wavelength tile), longest column first */
  int64_t ntasks;
  double *U, *K, *V, *Vtop, *Vbot;
  int layout;
  double *gam, *uu, *o1, *q; /* scratch [warp slot][max_nz][32] each */
  int64_t slot_stride; /* resident threads the scratch is sized for */
  int max_nz;
  unsigned long long *work;
  unsigned long long *status; /* [0] zero pivots, [1] first (column << 32 | wavelength), [2] timeout */
};
cudaError_t launch_pillars_batch(const double *rho, const double *T, const MBatchCol *cols, const int64_t *rec_pre,
                                 int64_t ncol, int64_t nrec, double fully_ionized_T, double *pil, cudaStream_t s);
cudaError_t launch_batch_fp64(const FP64BatchArgs &a, int form, int blocks, int threads, cudaStream_t s);
int batch_fp64_max_blocks_per_sm(int form, int threads);

/* Tilings of the batch kernels. */
constexpr int BATCH_TILING_WARP_COLUMN = 0; /* a warp solves 32 wavelengths of one column, records staged */
constexpr int BATCH_TILING_PACKED = 1;      /* a warp solves 32 consecutive items of the nz-sorted list */

cudaError_t launch_pillars_mixed_batch(const double *rho, const double *T, const MBatchCol *cols,
                                       const int64_t *rec_pre, int64_t ncol, int64_t nrec, double fully_ionized_T,
                                       float *rec, unsigned *colflag, cudaStream_t s);
cudaError_t launch_batch_mixed(const MixedBatchArgs &a, int tiling, int blocks, int threads, cudaStream_t s);
int batch_mixed_max_blocks_per_sm(int tiling, int threads);

/* Arguments of the epilogue kernels (kernels_epilogue.cu) over one block's device arrays:
 * layout 0: U (nw, ncol, nz+6), z-indexed arrays (nw, ncol, nz), z fastest;
 * layout 1: U [nz+6][ncol][nw], z-indexed arrays [nz][ncol][nw];
 * rho (ncol, nz); per-item planes (nw, ncol). */
struct EpilogueArgs {
  const double *U, *V, *K, *rho;
  double *Ip, *Im, *tau;
  int32_t *photo;
  int64_t ncol;
  int nz, nw, layout;
  double dz, target;
};
cudaError_t launch_intensities(const EpilogueArgs &a, int blocks, cudaStream_t s);
cudaError_t launch_optical_depth(const EpilogueArgs &a, int blocks, cudaStream_t s);
/* F[col] = sum_iw w[iw] * V[iw * ld_col + col] for col < ncol, iw in increasing order. */
cudaError_t launch_integrated_flux(const double *V, const double *w, int64_t ncol, int nw, int64_t ld_col, double *F,
                                   int blocks, cudaStream_t s);
/* Copies a lambda-fastest chunk plane set (src[z * src_zs + col * nw + iw], rows z values)
 * into reference-layout arrays (dst[(iw * ld_col + c_off + col) * rows + z]). */
cudaError_t launch_lambda_to_reference(const double *src, int64_t src_zs, double *dst, int64_t ld_col, int64_t c_off,
                                       int64_t nb, int rows, int nw, int num_sms, cudaStream_t s);

/* One z-block file of an Athena snapshot in device memory (kernels_inputs.cu): raw = the five
 * fields [5][nzl][nyl][nxl] as stored; the block arrays rho, T are (nxl, nyl, nz), z fastest. */
struct AthenaZBlock {
  const double *raw;
  int nxl, nyl, nzl, nz, iz0, lavoid;
  double *rho, *T;
};
cudaError_t launch_athena_zblock(const AthenaZBlock &b, cudaStream_t s);
cudaError_t launch_athena_post(double *rho, double *T, int64_t n, int nz, double unit_density, double rho_floor,
                               double gamma1, double unit_T, const double *Tgauss, double switchTemp, double floorTemp,
                               cudaStream_t s);

/* Fills tab[NL*nw] (layout [field][iw]) with the wavelength table of waves[nw] (Angstrom):
 * pre_calc_opacity_quantities' arithmetic plus the hot loop's lambda-only factors
 * (defined in oco_api.cu). */
void fill_lambda_table(const double *waves, int nw, double *tab);

/* Kernel launchers (defined in kernels_fp64.cu). Return cudaGetLastError(). */
cudaError_t launch_pillars(const double *rho, const double *T, int64_t ncol, int nz,
                           double fully_ionized_T, int grey, double *pil, cudaStream_t s);
cudaError_t launch_solve_fp64(const SolveArgs &a, int form, int grey, int nslot_blocks,
                              int threads, cudaStream_t s);
int solve_fp64_max_blocks_per_sm(int form, int grey, int threads);
/* Runs the bounded-wait diagnostic kernel (one warp) on s; sets status[2] when the wait ran out. */
cudaError_t launch_bounded_wait_check(long long limit, unsigned long long *status, cudaStream_t s);

/* Mixed-precision kernels (kernels_mixed.cu). */
constexpr int MIXED_ZN = 64; /* floats per mixed record */
/* Default condition number of the mixed form's emergent flux above which an item is re-solved
 * in FP64 (stable form, k_repair): the flux is a weighted sum of boundary differences
 * D_k = u_k - q_k U_{k+1}, and its condition number is sum |w_k| (u_k + q_k U_{k+1}) / |sum w_k D_k|. */
constexpr float MIXED_REPAIR_COND = 100.0f;
constexpr int MIXED_LN = 29; /* fields of the mixed wavelength table */
/* colflag[ncol] (cleared by the caller) marks columns to re-solve in FP64 (mx::pillar). */
cudaError_t launch_pillars_mixed(const double *rho, const double *T, int64_t ncol, int nz, double fully_ionized_T,
                                 float *rec, unsigned *colflag, cudaStream_t s);
cudaError_t launch_solve_mixed(const MixedArgs &a, int blocks, int threads, cudaStream_t s);
int solve_mixed_max_blocks_per_sm(int threads, int nw); /* occupancy of the kernel used for nw */
/* Fills tab32[MIXED_LN*nw] from the FP64 table tab[NL*nw]. */
void fill_mixed_lambda_table(const double *tab, int nw, float *tab32);

}  // namespace oco

#endif
