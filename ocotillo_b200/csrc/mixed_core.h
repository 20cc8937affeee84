/*
 * mixed_core.h -- the mixed-precision form of the per-(column, wavelength) solve, shared by
 * the CUDA kernels (kernels_mixed.cu) and a host build used for accuracy studies.
 *
 * Same physics and the same linear system as the reference loop
 * (source/flux_feautrier.f90:160-228), evaluated as follows:
 *   - per (column, z), in FP64: Saha ionization and every z-only factor, as in the FP64
 *     pillar kernel, stored as a record (MixedZ) of base-2 logarithms so that nothing
 *     underflows (opacity terms per H atom span ~1e-60..1e-17);
 *   - per (z, lambda), in FP32 log2 space: every opacity term of calc_opacity_and_albedo
 *     (continuous_opacity.f90:175-201) is a sum of log2 factors; terms are added with a
 *     log-sum-exp on the SFU (ex2/lg2).  Logarithms of that size (|log2| up to ~200) would
 *     resolve only ~1e-5 as FP32 numbers, and a per-cell error of that size in kappa is what
 *     sensitive columns amplify, so every large logarithm is carried as an exact integer plus
 *     a small FP32 fraction (L2: i + f, |f| <= 1/2 when stored).  Integers add exactly in
 *     FP32, the fractions keep ~3e-8 absolute precision, and every 2^x is taken as
 *     2^int * ex2(fraction): kappa and the source function come out to a few 1e-7.  The
 *     Planck exponent x*log2(e) is a double-float product (FMA two-product of split FP32
 *     factors) for the same reason.  The H bound-free level sum
 *     sum_n g(lambda,n) n^-3 exp(-chi_n/kT) (:237-239) is factored by its first non-zero
 *     level n0(lambda): E_n0 * (g_n0 + sum_{n>n0} g_n * E_n/E_n0), with the ratios E_n/E_n0
 *     precomputed per z.  The absorption fraction 1 - omega = kappa_abs/kappa_rad is a linear
 *     ratio of the same sums (one reciprocal; no cancellation when scattering dominates).  The
 *     reference's double addition of the H free-free opacity (:267-268, :274-275) is kept:
 *     neutral cells get kappa = rho (2 kr0 + kHff/mp), kappa_rad = kr0 + kHff/mp; ionized
 *     cells kappa = rho kr0 + k_brems, kappa_rad = 2 kr0 + k_brems/rho.
 *   - the tridiagonal system of auxiliary.f90:111-201 with every row divided by kappa_i^2
 *     (a' = 1/kappa_{i-1/2}, c' = 1/kappa_{i+1/2}, diagonal excess dz^2 kappa (1-omega)) and
 *     the Thomas recursion in difference form (all terms non-negative), in FP32, with the
 *     right-hand side and u carried as extended-exponent FP32 (XF) values;
 *   - back-substitution in extended FP32 for U_j and for the differences
 *     D_j = U_j - U_{j+1} = u_j - q_j U_{j+1} (q_j = h_j/(c_j+h_j)), so the flux never
 *     subtracts two nearly equal U; ghost zones and the 6th-order flux in FP64 from the D_j;
 *     outputs U, kappa, V in FP64.
 */
#ifndef OCO_MIXED_CORE_H
#define OCO_MIXED_CORE_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "ocomath.h"
#include "oco_consts.h"

#ifdef __CUDACC__
#define MX_HD static __host__ __device__ __forceinline__
#else
#define MX_HD static inline
#endif

namespace oco {
namespace mx {

/* Per-(column, z) FP32 record: the z-only factors.  A large base-2 logarithm takes two
 * slots, its fraction and then its integer part (value = integer + fraction); the others are
 * small logarithms or linear values.  damping_factor_const/T is split into hi + lo (the Planck
 * exponent needs it to ~1e-12). */
enum MixedZ {
  MZ_TH = 0,        /* theta = 5040/T */
  MZ_PU,            /* log2(ionf * Unsold integral) [2] */
  MZ_PE = MZ_PU + 2, /* log2(ionf * exp(-chi_n/kT)), n = 1..6 [2 each] */
  MZ_LHM = MZ_PE + 12, /* log2(hm_bf_factor * ionf) [2] */
  MZ_LAFF = MZ_LHM + 2, /* log2(ionf ne k T) [2] */
  MZ_LESC = MZ_LAFF + 2, /* log2(e_scatter) [2] */
  MZ_LIONFEF = MZ_LESC + 2, /* log2(ionf * energyfactor) [2] */
  MZ_LRHO = MZ_LIONFEF + 2, /* log2(rho) [2] */
  MZ_LZ2 = MZ_LRHO + 2, /* log2(ne (nHI+nHII) T^-1/2) [2] */
  MZ_LGT = MZ_LZ2 + 2, /* log10(theta) */
  MZ_LGT2,          /* log10(theta)^2 */
  MZ_NEUTRAL,       /* 1 if (1 - NHII/N) > switch_ionfraction */
  MZ_TH1L,          /* theta1 * log10e */
  MZ_LNTPOW,        /* ln((T*1e-4)^-1.5) */
  MZ_T1,            /* 1/T */
  MZ_DFT1,          /* damping_factor_const / T, high part */
  MZ_DFT1L,         /* low part */
  MZ_R,             /* level ratios E_n/E_n0 by first level n0 = 1..6: row n0 at MZ_R + rrow(n0)
                       holds 1, E_{n0+1}/E_n0, ..., E_6/E_n0 (linear); 21 values + 5 zeros, so
                       that six consecutive values can be read from any row */
  MZ_END = MZ_R + 26,
  MZN = 64          /* 256 B */
};
/* start of row n0 (1..6) of the level-ratio table: sum over m < n0 of (7 - m) */
MX_HD int rrow(int n0) { return (n0 - 1) * 7 - ((n0 - 1) * n0) / 2; }
static_assert(MZ_END <= MZN && MZN % 4 == 0, "mixed record layout");

/* Per-wavelength FP32 record (device layout [field][nw]); [2] as in MixedZ. */
enum MixedL {
  ML_CL2 = 0,  /* chi * log2(10) */
  ML_LAW,      /* log2(AHbf * wa^3) [2] */
  ML_GS = ML_LAW + 2, /* g(lambda,n) n^-3 from the first level n0 with g > 0: n = n0..6, then 0 [6] */
  ML_ROFF = ML_GS + 6, /* MixedZ offset of row n0 of the level-ratio table (MZ_R + rrow(n0)) */
  ML_PEOFF,    /* MixedZ offset of log2(ionf E_n0) (MZ_PE + 2 (n0 - 1)); MZ_PU when no level has g > 0 */
  ML_LS,       /* log2(s_coeff) if wa < 16000 else -1000 [2] */
  ML_FC = ML_LS + 2, /* (f1 - 26) log2(10) [2] */
  ML_F2 = ML_FC + 2, /* f2 log2(10) */
  ML_F3,       /* f3 log2(10) */
  ML_LAL0W,    /* log2(alpha0 * wa^3 * mp1) [2] */
  ML_GFF = ML_LAL0W + 2,
  ML_CHI1,
  ML_LNNU9,    /* ln(nu * 1e-9) */
  ML_HNUK,     /* h nu / k */
  ML_L3NU,     /* log2(nu^3) [2] */
  ML_CH = ML_L3NU + 2, /* log2(e) / lambda_cm, high part */
  ML_CL,       /* low part */
  ML_LSI,      /* log2(2 h c^2 lambda_cm^-5) = LSI + LSF, LSI an integer */
  ML_LSF,
  MLN
};

constexpr float kNeg = -1000.0f; /* log2 of a vanishing term */
constexpr double kLog2e = 1.4426950408889634;
constexpr double kLn2 = 0.6931471805599453;
constexpr double kLog2_10 = 3.321928094887362;
constexpr float kLog2e_f = 1.44269504f;
constexpr float kLn2_f = 0.693147181f;
constexpr float kLog2_10_f = 3.32192809f;

/* ---- SFU helpers: MUFU on the device, libm on the host ---------------------------- */
MX_HD float ex2(float x) {
#ifdef __CUDA_ARCH__
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return exp2f(x);
#endif
}
MX_HD float lg2(float x) {
#ifdef __CUDA_ARCH__
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return log2f(x);
#endif
}
MX_HD float rcp(float x) {
#ifdef __CUDA_ARCH__
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
#else
  return 1.0f / x;
#endif
}

MX_HD float fmaxf_(float a, float b) { return a > b ? a : b; }
/* log2(1 - 2^-t) for t > 0 (accurate to a few 1e-7 relative of the result's argument
 * for t >= 2^-6; a two-term series below that). */
MX_HD float log2_one_minus_exp2neg(float t) {
  const float x = t * kLn2_f; /* 1 - e^-x = x (1 - x/2 + x^2/6) below 2^-6; one ex2 and one lg2 */
  const float series = x * (1.0f - x * (0.5f - x * (1.0f / 6.0f)));
  const float direct = 1.0f - ex2(-t);
  return lg2(t < 0.015625f ? series : direct);
}

MX_HD float tolog(double v) { return v > 0.0 ? (float)(oco_log(v) * kLog2e) : kNeg; }
/* hi + lo split of a double into two floats */
MX_HD void split2(double v, float &hi, float &lo) {
  hi = (float)v;
  lo = (float)(v - (double)hi);
}
/* A large log2 value as fraction o[0] and integer o[1] (nearest integer: |fraction| <= 1/2). */
MX_HD void put_l2(double v, float *o) {
  const double i = floor(v + 0.5);
  o[0] = (float)(v - i);
  o[1] = (float)i;
}

/* FP64 logarithm and exponential of the record's wavelength-independent factors, which the
 * record keeps in FP32: the math library's (an ulp or so), where the FP64 forms need ocomath's
 * correctly rounded ones for bit-parity with the oracle.  Saha's root keeps ocomath's, so that
 * the negative-neutral-fraction test below sees the FP64 forms' value. */
MX_HD double dlog(double v) { return log(v); }
MX_HD double dexp(double v) { return exp(v); }

/* ---- per-(column, z) record (gas_state.f90:30-110, c_o :143-163) ------------------------ */
/* Returns true when the cell's neutral hydrogen density is negative.  The reference's Saha root
 * 0.5*(sqrt(C^2 + 4C) - C) (gas_state.f90:63) cancels for large C and can round above 1 below
 * fully_ionized_T; nHI = n - nHII and ionf are then negative, and the reference's opacity terms
 * proportional to ionf (continuous_opacity.f90:237-244, :318-322, :337-339, :265) turn negative.
 * Logarithms cannot carry that (the record holds such terms as vanishing): a column with such a
 * cell is solved in FP64 instead. */
MX_HD bool pillar(double r, double t, double fully_ionized_T, float *o) {
  using namespace oco::k;
  const double rho1 = 1.0 / r, T1 = 1.0 / t;
  double c_ion = (mp * rho1) * (saha_const * oco_pow(t, 1.5) * oco_exp(-((T1 * hydrogen_ionization_eV) * k1_eV)));
  double x = 0.5 * (sqrt(c_ion * c_ion + 4.0 * c_ion) - c_ion);
  if (t > fully_ionized_T) x = 1.0;
  double nn = r * mp1, nHII = x * nn, nHI = nn - nHII, ne = nHII;
  double ionf = (nHI != 0.0) ? nHI / (nHI + nHII) : 0.0;
  double Pe = (ne * k_cgs) * t;
  double escat = (alpha_e * nHII) * (rho1 * mp);
  double theta = 5040.0 * T1, theta1 = 1.0 / theta;
  double lgt = log10(theta);
  double ktemp1 = k1_cgs * T1;
  double chi[7];
  for (int n = 1; n <= 6; n++) {
    double n1 = 1.0 / (double)n;
    chi[n] = RydbergEnergy * (1.0 - n1 * n1);
  }
  const double lionf = ionf > 0.0 ? dlog(ionf) * kLog2e : (double)kNeg;
  o[MZ_TH] = (float)(theta);
  /* E_n/E_n0 = exp(-(chi_n - chi_n0)/kT) as e_n / e_n0 with e_n = exp(-chi_n/kT) (chi_1 = 0; e_6 >= 5e-34
   * at the 2000 K floor) */
  double e[7];
  e[1] = 1.0;
  for (int n = 2; n <= 6; n++) e[n] = dexp(-(chi[n] * ktemp1));
  for (int n0 = 1; n0 <= 6; n0++) {
    o[MZ_R + rrow(n0)] = 1.0f;
    for (int n = n0 + 1; n <= 6; n++) o[MZ_R + rrow(n0) + (n - n0)] = (float)(e[n] / e[n0]);
  }
  for (int k2 = MZ_R + 21; k2 < MZ_END; k2++) o[k2] = 0.0f;
  /* Unsold: 0.5 kT/Ry (exp(-chi_6/kT) - exp(-Ry/kT)) = 0.5 kT/Ry e^{-chi_6/kT} (1 - e^{-(Ry-chi_6)/kT}) */
  double lu = dlog((0.5 * (k_cgs * t)) * RydbergEnergy1) - chi[6] * ktemp1 +
              dlog(1.0 - dexp(-((RydbergEnergy - chi[6]) * ktemp1)));
  put_l2(ionf > 0.0 ? lionf + lu * kLog2e : (double)kNeg, o + MZ_PU);
  for (int n = 1; n <= 6; n++)
    put_l2(ionf > 0.0 ? lionf - (chi[n] * ktemp1) * kLog2e : (double)kNeg, o + MZ_PE + 2 * (n - 1));
  /* hm_bf_factor = 4.158e-10 Pe theta^2.5 10^(0.754 theta), in logs */
  double lhm = (Pe > 0.0 && ionf > 0.0)
                   ? (dlog(4.158e-10 * Pe) + 2.5 * dlog(theta)) * kLog2e + 0.754 * theta * kLog2_10 + lionf
                   : (double)kNeg;
  put_l2(lhm, o + MZ_LHM);
  const double aff = ((ionf * ne) * k_cgs) * t;
  put_l2(aff > 0.0 ? dlog(aff) * kLog2e : (double)kNeg, o + MZ_LAFF);
  put_l2(escat > 0.0 ? dlog(escat) * kLog2e : (double)kNeg, o + MZ_LESC);
  /* energyfactor = 0.5 log10e theta1 / Iev * 10^(-theta Iev) */
  double lef = dlog(((0.5 * log10e) * theta1) * Iev1) * kLog2e - theta * Iev * kLog2_10;
  put_l2(ionf > 0.0 ? lef + lionf : (double)kNeg, o + MZ_LIONFEF);
  put_l2(dlog(r) * kLog2e, o + MZ_LRHO);
  double nprod = ne * (nHI + nHII);
  put_l2(nprod > 0.0 ? (dlog(nprod) - 0.5 * dlog(t)) * kLog2e : (double)kNeg, o + MZ_LZ2);
  o[MZ_LGT] = (float)(lgt);
  o[MZ_LGT2] = (float)((lgt * lgt));
  o[MZ_NEUTRAL] = (float)(((1.0 - x) > switch_ionfraction) ? 1.0 : 0.0);
  o[MZ_TH1L] = (float)((theta1 * log10e));
  o[MZ_LNTPOW] = (float)((-1.5 * dlog(t * 1e-4)));
  o[MZ_T1] = (float)(T1);
  split2(damping_factor_const * T1, o[MZ_DFT1], o[MZ_DFT1L]);
  for (int k2 = MZ_END; k2 < MZN; k2++) o[k2] = 0.0f;
  return nHI < 0.0;
}

/* ---- per-wavelength record from the FP64 table entries --------------------------------- */
struct LamIn {
  double chi, gff, chi1, wa3, s, hmon, f1, f2, f3, gn[6], nu9, l3nu, hnuk, wcm1, sw5;
};
MX_HD void lambda_record(const LamIn &L, float *o) {
  using namespace oco::k;
  o[ML_CL2] = (float)(L.chi * kLog2_10);
  put_l2(oco_log(AHbf * L.wa3) * kLog2e, o + ML_LAW);
  int n0 = 7;
  for (int n = 6; n >= 1; n--)
    if (L.gn[n - 1] > 0.0) n0 = n;
  for (int t = 0; t < 6; t++) o[ML_GS + t] = (n0 + t <= 6) ? (float)L.gn[n0 + t - 1] : 0.0f;
  o[ML_ROFF] = (float)(MZ_R + (n0 <= 6 ? rrow(n0) : 0));
  o[ML_PEOFF] = (float)(n0 <= 6 ? MZ_PE + 2 * (n0 - 1) : MZ_PU);
  put_l2((L.hmon != 0.0 && L.s > 0.0) ? oco_log(L.s) * kLog2e : (double)kNeg, o + ML_LS);
  put_l2((L.f1 - 26.0) * kLog2_10, o + ML_FC);
  o[ML_F2] = (float)(L.f2 * kLog2_10);
  o[ML_F3] = (float)(L.f3 * kLog2_10);
  put_l2(oco_log((alpha0 * L.wa3) * mp1) * kLog2e, o + ML_LAL0W);
  o[ML_GFF] = (float)L.gff;
  o[ML_CHI1] = (float)L.chi1;
  o[ML_LNNU9] = (float)oco_log(L.nu9);
  o[ML_HNUK] = (float)L.hnuk;
  put_l2(L.l3nu * kLog2e, o + ML_L3NU);
  split2(L.wcm1 * kLog2e, o[ML_CH], o[ML_CL]);
  const double lsw5 = oco_log(L.sw5) * kLog2e;
  const double fl = floor(lsw5);
  o[ML_LSI] = (float)fl;
  o[ML_LSF] = (float)(lsw5 - fl);
}

/* Wavelength constants held in registers by the solve; *i members are the integer parts of
 * the large logarithms (value = member + member_i). */
struct Lam32 {
  float cl2, law, lawi, gs[6], ls, lsi_, fc, fci, f2, f3, lal0w, lal0wi, gff, chi1, lnnu9, hnuk, l3nu, l3nui;
  float ch, cl;   /* log2(e)/lambda_cm = ch + cl */
  float lsi, lsf; /* log2(2 h c^2 lambda_cm^-5) = lsi + lsf, lsi an integer */
  int roff, peoff; /* MixedZ offsets of the level-ratio row and of log2(ionf E_n0) */
};
/* Lam32 from a record laid out as MixedL (field f at t[f * stride]). */
template <class Get>
MX_HD void lam32_from(Lam32 &L, Get t) {
  L.cl2 = t(ML_CL2);
  L.law = t(ML_LAW);
  L.lawi = t(ML_LAW + 1);
  for (int q = 0; q < 6; q++) L.gs[q] = t(ML_GS + q);
  L.roff = (int)t(ML_ROFF);
  L.peoff = (int)t(ML_PEOFF);
  L.ls = t(ML_LS);
  L.lsi_ = t(ML_LS + 1);
  L.fc = t(ML_FC);
  L.fci = t(ML_FC + 1);
  L.f2 = t(ML_F2);
  L.f3 = t(ML_F3);
  L.lal0w = t(ML_LAL0W);
  L.lal0wi = t(ML_LAL0W + 1);
  L.gff = t(ML_GFF);
  L.chi1 = t(ML_CHI1);
  L.lnnu9 = t(ML_LNNU9);
  L.hnuk = t(ML_HNUK);
  L.l3nu = t(ML_L3NU);
  L.l3nui = t(ML_L3NU + 1);
  L.ch = t(ML_CH);
  L.cl = t(ML_CL);
  L.lsi = t(ML_LSI);
  L.lsf = t(ML_LSF);
}

/* Opacity, absorption fraction and source function of one (z, lambda):
 * log2 kappa = lki + lkf (lki an integer), omw = 1 - omega (linear, in [2^-126, 1]) and
 * log2(S (1 - omega) / mant(omw)) = lSi + lSf (lSi an integer): the right-hand side takes the
 * binary exponent of 1 - omega in its exact integer part and the mantissa as a factor in
 * [1, 2), so that it never underflows. */
struct Opac32 {
  float lki, lkf;
  float omw;
  float lSi, lSf;
};

/* 308 log2(e) as hi + lo: the reference clamps the Planck exponent x at log_overflow_limit = 308 */
constexpr float kT2Clamp = (float)(308.0 * kLog2e);
constexpr float kT2ClampLo = (float)(308.0 * kLog2e - (double)kT2Clamp);

/* w = pow2_mant(w) * 2^pow2_expo(w) with the mantissa in [1, 2), for a normal w > 0; the
 * exponent is returned as an integer-valued float (bit operations and one exact FADD). */
MX_HD float pow2_mant(float w) {
#ifdef __CUDA_ARCH__
  return __int_as_float((__float_as_int(w) & 0x007fffff) | 0x3f800000);
#else
  uint32_t b;
  memcpy(&b, &w, 4);
  b = (b & 0x007fffffu) | 0x3f800000u;
  float r;
  memcpy(&r, &b, 4);
  return r;
#endif
}
MX_HD float pow2_expo(float w) {
#ifdef __CUDA_ARCH__
  return __int_as_float(0x4b000000 | ((__float_as_int(w) >> 23) & 0xff)) - 8388735.0f; /* 2^23 + 127 */
#else
  uint32_t b;
  memcpy(&b, &w, 4);
  b = 0x4b000000u | ((b >> 23) & 0xffu);
  float r;
  memcpy(&r, &b, 4);
  return r - 8388735.0f;
#endif
}

/* log2(1/mp) and log2(369234910.67735046) (bremsstrahlung constant) as integer + fraction */
constexpr float kLog2mp1I = 79.0f, kLog2mp1F = -0.0158371009f;
constexpr float kBremsI = 28.0f, kBremsF = 0.459963723f;

template <class Rec>
MX_HD Opac32 opacity(const Rec &Z, const Lam32 &L) {
  /* stim = 1 - 10^(-chi theta) (c_o :171) */
  const float t10 = L.cl2 * Z[MZ_TH];
  const float ls = (t10 > 40.0f) ? 0.0f : log2_one_minus_exp2neg(t10);
  /* H bound-free (c_o :233-244): AHbf wa^3 stim ionf (Unsold + E_n0 sm), sm = sum over
   * t = 0..5 of g_{n0+t} E_{n0+t}/E_n0: six FMAs down row n0 of the ratio table (levels below
   * n0 have g = 0 and drop out; past level 6 the weights are 0) */
  float ai = Z[MZ_PU + 1], af = Z[MZ_PU];
  float sm = 0.0f;
#pragma unroll
  for (int t = 0; t < 6; t++) sm = fmaf(L.gs[t], Z[L.roff + t], sm);
  {
    const float ef = Z[L.peoff], ei = Z[L.peoff + 1]; /* log2(ionf E_n0); = MZ_PU (d = 0) if no level */
    /* log2(Unsold) - log2(E_n0), both times ionf; the larger one sets the scale */
    const float d = (ai - ei) + (af - ef);
    const bool ug = d >= 0.0f;
    const float x = ex2(-fabsf(d)); /* branch-free: one ex2 and one lg2 whichever side is larger */
    const float arg = ug ? fmaf(x, sm, 1.0f) : x + sm;
    af = (ug ? af : ef) + lg2(arg);
    ai = ug ? ai : ei;
  }
  const float Ai = ai + L.lawi, Af = (L.law + ls) + af;
  /* H- bound-free (c_o :318-322) */
  const float Bi = Z[MZ_LHM + 1] + L.lsi_, Bf = (ls + Z[MZ_LHM]) + L.ls;
  /* H- free-free (c_o :337-339): log2(ionf ne k T) + (f1 + f2 lgt + f3 lgt^2 - 26) log2(10) */
  const float Ci = Z[MZ_LAFF + 1] + L.fci, Cf = (Z[MZ_LAFF] + L.fc) + (L.f2 * Z[MZ_LGT] + L.f3 * Z[MZ_LGT2]);
  const float Di = Z[MZ_LESC + 1], Df = Z[MZ_LESC];
  /* scale 2^mi, mi the largest integer part: each 2^(term - mi) = ex2((int diff, exact) + frac) */
  const float mi = fmaxf_(fmaxf_(Ai, Bi), fmaxf_(Ci, Di));
  const float eA = ex2((Ai - mi) + Af), eB = ex2((Bi - mi) + Bf), eC = ex2((Ci - mi) + Cf), eD = ex2((Di - mi) + Df);
  const float S4 = (eA + eB) + (eC + eD); /* sum per H / 2^mi */
  const float S3 = (eA + eB) + eC;        /* absorption part (no Thomson) */
  /* per-mass scale of S4 and S3: 2^(Xi + Xf) */
  const float Xi = mi + kLog2mp1I, Xf = kLog2mp1F;
  /* kappa and kappa_rad are one lg2 each of a linear combination scaled to M = max(X, extra
   * term); of the two scale factors one is exactly 1.  1 - omega = kappa_abs / kappa_rad. */
  Opac32 o;
  float Mi, Mf, es, ex, num, den, lin;
  if (Z[MZ_NEUTRAL] != 0.0f) { /* c_o :262-268: kappa = rho (2 kr0 + kHff/mp), kappa_rad = kr0 + kHff/mp */
    const float gff = 1.0f + L.gff * (Z[MZ_TH1L] * L.chi1 + 0.5f);
    const float Hi = Z[MZ_LIONFEF + 1] + L.lal0wi, Hf = ((ls + Z[MZ_LIONFEF]) + L.lal0w) + lg2(gff); /* kHff mp1 */
    const float dx = (Xi - Hi) + (Xf - Hf);
    const bool xs = dx >= 0.0f;
    const float e = ex2(-fabsf(dx));
    es = xs ? 1.0f : e;
    ex = xs ? e : 1.0f;
    Mi = xs ? Xi : Hi;
    Mf = xs ? Xf : Hf;
    lin = 2.0f * S4 * es + ex;
    num = S3 * es + ex;
    den = S4 * es + ex;
  } else { /* c_o :270-275, bremsstrahlung :281-300: kappa = rho kr0 + kb, kappa_rad = 2 kr0 + kb/rho */
    const float y = 5.960f - 0.551328895f * (L.lnnu9 + Z[MZ_LNTPOW]); /* sqrt(3)/pi */
    const float gaunt = kLn2_f * lg2(ex2(y * kLog2e_f) + 2.71828183f);
    const float xh = L.hnuk * Z[MZ_T1];
    const float lq = (xh > 30.0f) ? 0.0f : log2_one_minus_exp2neg(xh * kLog2e_f); /* log2(1 - e^-xh) */
    /* log2(kb / rho) = log2(369234910.67735046 ne n T^-1/2 nu^-3 (1 - e^-xh) gaunt / rho) */
    const float Ki = ((Z[MZ_LZ2 + 1] - L.l3nui) - Z[MZ_LRHO + 1]) + kBremsI;
    const float Kf = ((Z[MZ_LZ2] - L.l3nu) - Z[MZ_LRHO]) + ((lq + lg2(gaunt)) + kBremsF);
    const float dx = (Xi - Ki) + (Xf - Kf);
    const bool xs = dx >= 0.0f;
    const float e = ex2(-fabsf(dx));
    es = xs ? 1.0f : e;
    ex = xs ? e : 1.0f;
    Mi = xs ? Xi : Ki;
    Mf = xs ? Xf : Kf;
    lin = S4 * es + ex;
    num = (2.0f * S3 + eD) * es + ex;
    den = 2.0f * S4 * es + ex;
  }
  o.lki = Z[MZ_LRHO + 1] + Mi;
  o.lkf = (Z[MZ_LRHO] + Mf) + lg2(lin);
  const float w = num * rcp(den);
  o.omw = w > 1.0f ? 1.0f : (w < 1.17549435e-38f ? 1.17549435e-38f : w); /* [2^-126, 1] */
  /* Planck function (c_o :399-407): S = sw5 / (e^x - 1), x = dft1/lambda_cm clamped at 308.
   * t2 = x log2(e) = (dft1_hi + dft1_lo)(ch + cl) as hi + lo (FMA two-product). */
  const float dh = Z[MZ_DFT1], dl = Z[MZ_DFT1L];
  float p = dh * L.ch;
  float lo = fmaf(dh, L.ch, -p) + (dh * L.cl + dl * L.ch);
  if (p > kT2Clamp) {
    p = kT2Clamp;
    lo = kT2ClampLo;
  }
  const float ti = floorf(p);
  const float tf = (p - ti) + lo; /* t2 = ti + tf */
  const float lm = (p > 40.0f) ? 0.0f : log2_one_minus_exp2neg(p);
  o.lSi = (L.lsi - ti) + pow2_expo(o.omw);
  o.lSf = (L.lsf - tf) - lm;
  return o;
}

/* ---- extended-exponent numbers: value = m * 2^e, m FP32, e int ------------------------ */
struct XF {
  float m;
  int e;
};
MX_HD int f2bits(float f) {
#ifdef __CUDA_ARCH__
  return __float_as_int(f);
#else
  int i;
  memcpy(&i, &f, 4);
  return i;
#endif
}
MX_HD float bits2f(int i) {
#ifdef __CUDA_ARCH__
  return __int_as_float(i);
#else
  float f;
  memcpy(&f, &i, 4);
  return f;
#endif
}
/* 2^k as a float for -126 <= k <= 127; +0 below (k = -127 is the zero bit pattern). */
MX_HD float pow2f(int k) { return bits2f(((k < -127 ? -127 : k) + 127) << 23); }
/* renormalise so that |m| is in [1, 2) with bit operations: the exponent field moves into e.
 * A zero or subnormal m (exponent field 0) is kept as it is, value-exact. */
MX_HD XF xnorm(float m, int e) {
  const int b = f2bits(m);
  const int ef = (b >> 23) & 0xff;
  XF r;
  r.m = ef ? bits2f((b & (int)0x807fffff) | 0x3f800000) : m;
  r.e = ef ? e + (ef - 127) : e;
  return r;
}
/* 2^(I + F) for an integer-valued float I and a small float F */
MX_HD XF xexp2(float I, float F) {
  XF r;
  const float fl = floorf(F);
  r.e = (int)(I + fl);
  r.m = ex2(F - fl);
  return r;
}
/* x*s + y*t for FP32 factors s, t: the operand with the smaller exponent is scaled by 2^-|de|
 * (the other by exactly 1) and added with one FMA. */
MX_HD XF xaxpy(XF x, float s, XF y, float t) {
  const int d = x.e - y.e;
  const bool ge = d >= 0;
  const float a = x.m * s, b = y.m * t;
  const float big = ge ? a : b, small = ge ? b : a;
  return xnorm(fmaf(small, pow2f(ge ? -d : d), big), ge ? x.e : y.e);
}
/* The two back-substitution updates of one step, x + y*t1 and x + y*t2, sharing the alignment. */
MX_HD void xaxpy2(XF x, XF y, float t1, float t2, XF &r1, XF &r2) {
  const int d = x.e - y.e;
  const bool ge = d >= 0;
  const float p = pow2f(ge ? -d : d);
  const float b1 = y.m * t1, b2 = y.m * t2;
  const int e = ge ? x.e : y.e;
  r1 = xnorm(ge ? fmaf(b1, p, x.m) : fmaf(x.m, p, b1), e);
  r2 = xnorm(ge ? fmaf(b2, p, x.m) : fmaf(x.m, p, b2), e);
}
MX_HD double xtod(XF x) {
  if (x.m == 0.0f || x.e < -1000) return 0.0;
  return (double)x.m * oco_u2d((uint64_t)(int64_t)(x.e + 1023) << 52);
}

/* 1/kappa (> 0) and an XF u = m 2^e with m in [1, 2) in two 32-bit words: w1 = 1/kappa with
 * bit 9 of e + 512 in its sign bit, w2 = m's 23 fraction bits with bits 0-8 of e + 512 in its
 * sign and exponent field.  Returns whether the pair fits (e in [-512, 511], m normal in
 * [1, 2)); unpacking a fitting pair gives the same bits back. */
MX_HD bool pack_o1_u(float o1, float m, int e, int &w1, int &w2) {
  const int mb = f2bits(m), eb = e + 512;
  w1 = f2bits(o1) | ((eb & 0x200) << 22);
  w2 = (mb & 0x7fffff) | ((eb & 0x1ff) << 23);
  return ((unsigned)eb < 1024u) & ((mb >> 23) == 127);
}
MX_HD void unpack_o1_u(int w1, int w2, float &o1, float &m, int &e) {
  o1 = bits2f(w1 & 0x7fffffff);
  m = bits2f((w2 & 0x7fffff) | 0x3f800000);
  e = (((w2 >> 23) & 0x1ff) | ((w1 >> 22) & 0x200)) - 512;
}

/* ---- scaled tridiagonal rows (auxiliary.f90:125-201 divided by kappa_i^2) ------------- */
struct Row32 {
  float a, c, e;  /* sub, super, diagonal excess -(a+b+c) */
  float ldi, ldf; /* -d (right-hand side) = w * 2^(ldi + ldf), ldi an integer */
  float w;        /* mantissa of 1 - omega, in [1, 2) */
};
/* 2^(i + f) for an integer-valued i and a small f, the exponent clamped to the FP32 normal
 * range [-126, 127] */
MX_HD float exp2_split(float i, float f) {
  const float fl = floorf(f);
  const float L = i + fl;
  if (L < -126.0f) return pow2f(-126);
  if (L >= 127.0f) return pow2f(127);
  return ex2(f - fl) * pow2f((int)L);
}
MX_HD float kappa_lin(const Opac32 &o) { return exp2_split(o.lki, o.lkf); }
/* the right-hand side S e' as w 2^(ldi + ldf): le + log2 S with le split as i + f, and the
 * mantissa w of 1 - omega (its exponent is in o.lSi) */
MX_HD void row_rhs(Row32 &r, float lei, float lef, const Opac32 &o) {
  const float fi = floorf(lef);
  r.ldi = (lei + fi) + o.lSi;
  r.ldf = (lef - fi) + o.lSf;
  r.w = pow2_mant(o.omw);
}
/* e' = dz^2 kappa (1 - omega) as a linear product (kappa dz^2 capped at FLT_MAX) */
MX_HD float row_excess(float kj, const Opac32 &o, float dz2f) {
  const float t = kj * dz2f;
  return (t < 3.40282347e38f ? t : 3.40282347e38f) * o.omw;
}
/* centre row: a' = 1/kappa_{i-1/2} (= c' of the row below, passed in), c' = 1/kappa_{i+1/2},
 * e' = dz^2 kappa (1-omega), d' = -S e'; log2(dz^2) = ldz2i + ldz2f */
MX_HD Row32 row_center(float a, float kj, float kp, const Opac32 &o, float dz2f, float ldz2i, float ldz2f) {
  Row32 r;
  r.a = a;
  r.c = 2.0f * rcp(kp + kj);
  r.e = row_excess(kj, o, dz2f);
  row_rhs(r, ldz2i + o.lki, ldz2f + o.lkf, o);
  return r;
}
/* boundary rows: zeta = kappa dz^2 (1-omega)/4; excess dz + zeta; d' = -S zeta;
 * bottom: a' = 0, c' = 1/kappa; top: a' = 1/kappa, c' = 0 */
MX_HD Row32 row_boundary(float kj, const Opac32 &o, float dz, float dz2f, float ldz2i, float ldz2f, bool top) {
  Row32 r;
  r.a = top ? rcp(kj) : 0.0f;
  r.c = top ? 0.0f : rcp(kj);
  r.e = dz + 0.25f * row_excess(kj, o, dz2f);
  row_rhs(r, (ldz2i + o.lki) - 2.0f, ldz2f + o.lkf, o);
  return r;
}
/* log2(dz^2) as integer + fraction */
MX_HD void ldz2_split(double dz, float &i, float &f) {
  const double v = 2.0 * oco_log(dz) * kLog2e;
  const double n = floor(v + 0.5);
  i = (float)n;
  f = (float)(v - n);
}

/* 6th-order flux at interior index m (auxiliary.f90:64-109) from the differences
 * Dl[k] = f_k - f_{k+1} of the ghosted array (ghost differences mirror the interior ones). */
MX_HD double flux_from_diffs(const double *Dl, int m, double o1, double dz1) {
  const double s1 = Dl[m - 1] + Dl[m];
  const double s2 = (s1 + Dl[m - 2]) + Dl[m + 1];
  const double s3 = (s2 + Dl[m - 3]) + Dl[m + 2];
  const double df = -((1.0 / 60.0) * (((45.0 * s1) - 9.0 * s2) + s3));
  return ((-o1) * df) * dz1;
}

/* Reference implementation of the mixed solve for one (column, wavelength) item on the host
 * (accuracy studies; the CUDA kernel streams the same arithmetic).  Zat(z): record of z;
 * work: 6*nz floats; dwork: nz+6 doubles.  Outputs U[nz+6], K[nz], V[nz] in FP64. */
template <class ZAt>
MX_HD void solve_item_host(ZAt Zat, const Lam32 &L, int nz, double dz, float *work, double *dwork, double *U,
                           double *K, double *V) {
  const float dzf = (float)dz, dz2f = (float)(dz * dz);
  float ldz2i, ldz2f;
  ldz2_split(dz, ldz2i, ldz2f);
  float *g = work, *um = work + nz, *o1 = work + 2 * nz, *kap = work + 3 * nz, *qv = work + 5 * nz;
  int *ue = (int *)(work + 4 * nz);
  Opac32 cur = opacity(Zat(0), L), nxt = opacity(Zat(1), L);
  float kc = kappa_lin(cur), kn = kappa_lin(nxt);
  Row32 r = row_boundary(kc, cur, dzf, dz2f, ldz2i, ldz2f, false);
  float h = r.e, cprev = r.c;
  float an = 2.0f * rcp(kn + kc); /* a' of row 1 */
  XF u = xexp2(r.ldi, r.ldf);
  u.m *= r.w * rcp(r.c + h);
  u = xnorm(u.m, u.e);
  um[0] = u.m;
  ue[0] = u.e;
  o1[0] = rcp(kc);
  kap[0] = kc;
  for (int j = 1; j < nz; j++) {
    cur = nxt;
    kc = kn;
    if (j < nz - 1) {
      nxt = opacity(Zat(j + 1), L);
      kn = kappa_lin(nxt);
      r = row_center(an, kc, kn, cur, dz2f, ldz2i, ldz2f);
      an = r.c;
    } else {
      r = row_boundary(kc, cur, dzf, dz2f, ldz2i, ldz2f, true);
    }
    const float rr = rcp(cprev + h);
    g[j] = cprev * rr;  /* |gamma_j| = c_{j-1}/(c_{j-1}+h_{j-1}) */
    qv[j - 1] = h * rr; /* q_{j-1} = h_{j-1}/(c_{j-1}+h_{j-1}) */
    h = r.e + (r.a * rr) * h; /* a'/(c'+h) is O(1); a' h alone can overflow */
    const float rb = rcp(r.c + h); /* 1/|bet_j| */
    u = xaxpy(xexp2(r.ldi, r.ldf), r.w * rb, u, r.a * rb); /* u_j = (|d_j| + a_j u_{j-1}) / |bet_j| */
    um[j] = u.m;
    ue[j] = u.e;
    o1[j] = rcp(kc);
    kap[j] = kc;
    cprev = r.c;
  }
  /* back-substitution: U_j = u_j + |gamma_{j+1}| U_{j+1} (all terms >= 0) and the differences
   * D_j = U_j - U_{j+1} = u_j - q_j U_{j+1}, in extended FP32; flux in FP64 from the D_j */
  XF Un = u;
  const int n1 = 3, n2 = nz + 2;
  double *Dl = dwork;
  U[n1 + nz - 1] = xtod(Un);
  for (int j = nz - 2; j >= 0; j--) {
    XF uj;
    uj.m = um[j];
    uj.e = ue[j];
    XF Dj;
    xaxpy2(uj, Un, g[j + 1], -qv[j], Un, Dj);
    U[n1 + j] = xtod(Un);
    Dl[n1 + j] = xtod(Dj);
  }
  for (int i = 1; i <= 3; i++) {
    U[n1 - i] = 2.0 * U[n1] - U[n1 + i];
    U[n2 + i] = 2.0 * U[n2] - U[n2 - i];
    Dl[n2 + i - 1] = Dl[n2 - i];
    Dl[n1 - i] = Dl[n1 + i - 1];
  }
  const double dz1 = 1.0 / dz;
  for (int j = 0; j < nz; j++) {
    V[j] = flux_from_diffs(Dl, n1 + j, (double)o1[j], dz1);
    K[j] = (double)kap[j];
  }
}

}  // namespace mx
}  // namespace oco

#endif
