/*
 * oco_oracle.c -- CPU restatement of the reference hot path (TEST INFRASTRUCTURE ONLY).
 * See oco_oracle.h for the rules.  Every function cites the reference lines it follows
 * (paths relative to the ocotillo repository).
 *
 * Conventions for bit-faithfulness with gfortran -O2 -fdefault-real-8:
 *   - Fortran evaluates a*b*c left to right: ((a*b)*c); unary minus binds below '*'.
 *   - x**2, x**3, x**4, x**5 with constant integer exponents are multiplication chains
 *     (x*x, x*(x*x), (x*x)*(x*x), (x*x)*(x*(x*x))).
 *   - x**n with a variable integer exponent is right-to-left binary powering.
 *   - x**r with a real exponent is pow(x, r); 10**r is pow(10.0, r).
 *   - constant expressions folded by the compiler are given as exact hex literals.
 */
#include "oco_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* oreal: the arithmetic type of the per-column and per-(column, wavelength) work.  double in
 * the glibc and ocomath back-ends; long double (x87 extended, 64-bit significand) in the
 * longdouble back-end, which evaluates the same problem -- the same double inputs, wavelength
 * tables and constants -- with 11 more bits per operation, to measure the rounding error of
 * the double forms (the stable form in particular). */
#ifdef OCO_ORACLE_LONGDOUBLE
typedef long double oreal;
#define MEXP(x) expl(x)
#define MLOG(x) logl(x)
#define MLOG10(x) log10l(x)
#define MPOW(x, y) powl((x), (y))
#define MSQRT(x) sqrtl(x)
#define BACKEND 2
#elif defined(OCO_ORACLE_OCOMATH)
#include "ocomath.h"
typedef double oreal;
#define MEXP(x) oco_exp(x)
#define MLOG(x) oco_log(x)
#define MLOG10(x) oco_log10(x)
#define MPOW(x, y) oco_pow((x), (y))
#define MSQRT(x) sqrt(x)
#define BACKEND 1
#else
typedef double oreal;
#define MEXP(x) exp(x)
#define MLOG(x) log(x)
#define MLOG10(x) log10(x)
#define MPOW(x, y) pow((x), (y))
#define MSQRT(x) sqrt(x)
#define BACKEND 0
#endif

int oracle_math_backend(void) { return BACKEND; }

/* ---- constants, common.f90:23-81 ------------------------------------------------------ */
static const double sigma_sb = 5.6703744191844314e-05;     /* :24 */
static const double log_overflow_limit = 308.0;             /* :28 floor(log10(huge(1d0))) */
static const double mp = 1.67262192369e-24;                 /* :31 */
static const double mp1 = 1.0 / 1.67262192369e-24;          /* :32 */
static const double h_planck = 6.62607015e-27;              /* :39 */
static const double pi1 = 1.0 / 0x1.921fb54442d18p+1;       /* :43-44, pi = 4*atan(1d0) */
static const double sqrt3 = 0x1.bb67ae8584caap+0;           /* :45 sqrt(3d0) */
static const double exp1 = 0x1.5bf0a8b145769p+1;            /* :46 exp(1d0) */
static const double k_cgs = 1.380649e-16;                   /* :49 */
static const double k1_cgs = 1.0 / 1.380649e-16;            /* :51 */
static const double k1_eV = 1.0 / 8.617333262145179e-05;    /* :52 */
static const double hydrogen_ionization_eV = 13.6;          /* :55 */
static const double c_light = 2.99792458e10;                /* :57 */
static const double RydbergEnergy = 2.1798741e-11;          /* :60 */
static const double RydbergEnergy1 = 1.0 / 2.1798741e-11;   /* :61 */
static const double log10e = 0x1.bcb7b1526e50ep-2;          /* :67 log10(exp(1d0)) */
/* :68-70 Rcm = 2*pi**2*me*e**4/(h**3*c) and Iev = h*c*Rcm*6.2419d11, folded by the
 * compiler with one rounding per operation (powers correctly rounded). */
static const double Iev = 0x1.b369160866803p+3;
static const double Iev1 = 1.0 / 0x1.b369160866803p+3;
static const double bremsstrahlung_constant = 369234910.67735046; /* :71 */
static const double hcR1 = (6.62607015e-27 * 2.99792458e10) / 2.1798741e-11; /* :79 */
static const double one_third = 1.0 / 3.0;  /* :80 */
static const double two_thirds = 2.0 / 3.0; /* :81 */

/* continuous_opacity.f90:20-25, :146 */
static const double switch_ionfraction = 1e-2;
static const double AHbf = 1.0449e-26;
static const double Rangstrom = 1.0968e-3;
static const double alpha0 = 1.0443e-26;
static const double alpha_e = 0.6648e-24;
#define MDIM 6

/* Right-to-left binary powering: the operation order of the library routine gfortran
 * calls for REAL**INTEGER with a non-constant exponent. */
static double powi_var(double x, int m) {
  unsigned n = m < 0 ? -(unsigned)m : (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return m < 0 ? 1.0 / y : y;
}

/* ---- wavelength tables, continuous_opacity.f90:64-141 -------------------------------- */
typedef struct {
  int nw;
  double *wa, *wcm, *wcm1, *nu, *chi, *chi1, *wa3, *w1cm5, *gff_factor, *s_coeff;
  double *f_coeff; /* [iw*3 + i] */
  double *g;       /* [iw*6 + n] */
  double n1_array[MDIM], chi_n[MDIM], chi_m;
  double damping_factor_const, source_function_const;
} otab;

/* gaunt, continuous_opacity.f90:343-375 */
static double gaunt_bf(int n, double wave_cm) {
  double lam_n = (double)(n * n) * hcR1;
  if (wave_cm <= lam_n) {
    double t = (wave_cm / lam_n) - 1.0;
    double eps2 = t * t;
    return 1.0 - (0.17285714285714285 * (1.0 - eps2)) * pow((double)n * (1.0 + eps2), -two_thirds);
  }
  return 0.0;
}

static void otab_free(otab *t) {
  free(t->wa);
  memset(t, 0, sizeof *t);
}

static int otab_build(otab *t, const double *waves, int nw) {
  memset(t, 0, sizeof *t);
  t->nw = nw;
  double *blk = (double *)calloc((size_t)nw * (10 + 3 + 6), sizeof(double));
  if (!blk) return ORACLE_ENOMEM;
  t->wa = blk;
  t->wcm = blk + nw;
  t->wcm1 = blk + 2 * nw;
  t->nu = blk + 3 * nw;
  t->chi = blk + 4 * nw;
  t->chi1 = blk + 5 * nw;
  t->wa3 = blk + 6 * nw;
  t->w1cm5 = blk + 7 * nw;
  t->gff_factor = blk + 8 * nw;
  t->s_coeff = blk + 9 * nw;
  t->f_coeff = blk + 10 * nw;
  t->g = blk + 13 * nw;
  t->damping_factor_const = (h_planck * c_light) * k1_cgs;        /* :73 */
  t->source_function_const = (2.0 * h_planck) * (c_light * c_light); /* :74 */
  static const double a_coeff[7] = {+1.99654,     -1.18267e-6,  +2.62423e-7, -4.40524e-11,
                                    +3.23992e-15, -1.39568e-19, +2.78701e-24}; /* :98-104 */
  static const double b_coeff[3][5] = {{-2.276300, -1.685000, +0.766610, -0.053356, +0.000000},
                                       {+15.28270, -9.284600, +1.993810, -0.142631, +0.000000},
                                       {-197.789, +190.266, -67.9775, +10.6913, -0.62515}};
  for (int iw = 0; iw < nw; iw++) {
    double wa = waves[iw];
    t->wa[iw] = wa;                           /* :76 */
    t->wcm[iw] = wa * 1e-8;                   /* :78 */
    t->wcm1[iw] = 1.0 / t->wcm[iw];           /* :79 */
    t->nu[iw] = c_light * t->wcm1[iw];        /* :80 */
    t->chi[iw] = 1.2398e4 / wa;               /* :82 */
    t->chi1[iw] = 1.0 / t->chi[iw];           /* :83 */
    t->wa3[iw] = wa * (wa * wa);              /* :85 wa**3 */
    double x = t->wcm1[iw], x2 = x * x;
    t->w1cm5[iw] = x2 * (x * x2);             /* :86 wcm1**5 */
    t->gff_factor[iw] = 0.3456 * pow(wa * Rangstrom, -one_third); /* :91 */
    double s = 0.0;
    for (int i = 1; i <= 7; i++) s = s + (1e-17 * a_coeff[i - 1]) * powi_var(wa, i - 1); /* :106-109 */
    t->s_coeff[iw] = s;
  }
  for (int n = 1; n <= MDIM; n++) { /* :121-127 */
    t->n1_array[n - 1] = 1.0 / (double)n;
    double n1 = t->n1_array[n - 1];
    t->chi_n[n - 1] = RydbergEnergy * (1.0 - 1.0 * (n1 * n1));
    for (int iw = 0; iw < nw; iw++) t->g[iw * MDIM + (n - 1)] = gaunt_bf(n, t->wcm[iw]);
  }
  {
    double n1 = t->n1_array[MDIM - 1];
    t->chi_m = RydbergEnergy * (1.0 - n1 * n1); /* :129 */
  }
  for (int iw = 0; iw < nw; iw++) { /* :131-139 */
    double lg = log10(t->wa[iw]);
    for (int i = 0; i < 3; i++) {
      double f = 0.0;
      for (int j = 1; j <= 5; j++) f = f + powi_var(lg, j - 1) * b_coeff[i][j - 1];
      t->f_coeff[iw * 3 + i] = f;
    }
  }
  return ORACLE_OK;
}

/* calc_wavelength, continuous_opacity.f90:37-62 */
void oracle_calc_wavelength(double w1, double w0, int32_t nw, double *wa) {
  if (nw > 1) {
    double dw = (w1 - w0) / (double)(nw - 1);
    for (int i = 1; i <= nw; i++) wa[i - 1] = w0 + (double)(i - 1) * dw;
  } else if (nw == 1) {
    wa[0] = w0;
  }
}

/* ---- pillar_case, pillars.inc:2-8 -------------------------------------------------- */
enum {
  P_RHO, P_RHO1, P_T, P_T1, P_X, P_N, P_INVN, P_NHI, P_NHII, P_NE, P_IONF, P_PE, P_ESCAT,
  P_THETA, P_THETA1, P_LGT, P_LGT2, P_HMBF, P_STIM, P_S, P_ALB, P_OP, P_OP1, P_OP2, P_FLUX,
  P_OMA, /* 1 - albedo from the absorption terms (stable form) */
  P_NFIELDS
};
typedef struct {
  int nz;
  oreal *f[P_NFIELDS];
  oreal *mem;
} opillar;

static int pillar_alloc(opillar *p, int nz) {
  p->nz = nz;
  p->mem = (oreal *)calloc((size_t)nz * P_NFIELDS, sizeof(oreal));
  if (!p->mem) return ORACLE_ENOMEM;
  for (int k = 0; k < P_NFIELDS; k++) p->f[k] = p->mem + (size_t)k * nz;
  return ORACLE_OK;
}

/* wavelength_independent_pillars + calc_hydrogen_ion_frac + solve_gas_state +
 * get_electron_pressure (gas_state.f90:30-110) + get_electron_thomson_scattering and
 * get_hydrogen_ion_bound_free (continuous_opacity.f90:143-163). */
static void pillars(opillar *p, oreal fully_ionized_T) {
  const int nz = p->nz;
  oreal **f = p->f;
  for (int i = 0; i < nz; i++) {
    f[P_RHO1][i] = 1.0 / f[P_RHO][i]; /* gas_state :34 */
    f[P_T1][i] = 1.0 / f[P_T][i];     /* :35 */
  }
  for (int i = 0; i < nz; i++) { /* calc_hydrogen_ion_frac :57-63 */
    oreal T = f[P_T][i];
    oreal constants = 2414683039571967.0 * MPOW(T, 1.5);
    oreal exparg = (f[P_T1][i] * hydrogen_ionization_eV) * k1_eV;
    oreal niine_ni = constants * MEXP(-exparg);
    oreal c_ion = (mp * f[P_RHO1][i]) * niine_ni;
    f[P_X][i] = 0.5 * (MSQRT(c_ion * c_ion + 4.0 * c_ion) - c_ion);
  }
  for (int i = 0; i < nz; i++) /* :70-74 */
    if (f[P_T][i] > fully_ionized_T) f[P_X][i] = 1.0;
  for (int i = 0; i < nz; i++) { /* solve_gas_state :85-97 */
    f[P_N][i] = f[P_RHO][i] * mp1;
    f[P_INVN][i] = f[P_RHO1][i] * mp;
    f[P_NHII][i] = f[P_X][i] * f[P_N][i];
    f[P_NHI][i] = f[P_N][i] - f[P_NHII][i];
    f[P_NE][i] = f[P_NHII][i];
    f[P_IONF][i] = (f[P_NHI][i] != 0.0) ? f[P_NHI][i] / (f[P_NHI][i] + f[P_NHII][i]) : 0.0;
  }
  for (int i = 0; i < nz; i++) {
    f[P_PE][i] = (f[P_NE][i] * k_cgs) * f[P_T][i];                    /* :108 */
    f[P_ESCAT][i] = (alpha_e * f[P_NHII][i]) * f[P_INVN][i];          /* c_o :149 */
    f[P_THETA][i] = 5040.0 * f[P_T1][i];                               /* gas_state :40 */
    f[P_THETA1][i] = 1.0 / f[P_THETA][i];                              /* :41 */
    f[P_LGT][i] = MLOG10(f[P_THETA][i]);                               /* :42 */
    f[P_LGT2][i] = f[P_LGT][i] * f[P_LGT][i];                          /* :43 */
    f[P_HMBF][i] = ((4.158e-10 * f[P_PE][i]) * MPOW(f[P_THETA][i], 2.5)) *
                   MPOW(10.0, 0.754 * f[P_THETA][i]);                  /* c_o :161 */
  }
}

/* bremsstrahlung_absorptionCoeff, continuous_opacity.f90:281-300 (zprotons = 1.0) */
static oreal bremsstrahlung(const opillar *p, int i, oreal frequency) {
  oreal *const *f = p->f;
  const oreal zprotons = 1.0;
  oreal gaunt = MLOG(MEXP(5.960 - (sqrt3 * pi1) * MLOG((frequency * 1e-9) * MPOW(f[P_T][i] * 1e-4, -1.5))) + exp1);
  oreal ln_physQuant = (((MLOG(f[P_NE][i] * (f[P_NHI][i] + f[P_NHII][i])) + 2.0 * MLOG(zprotons)) -
                          0.5 * MLOG(f[P_T][i])) - 3.0 * MLOG(frequency)) +
                        MLOG(1.0 - MEXP(-(((h_planck * frequency) * k1_cgs) * f[P_T1][i])));
  return (bremsstrahlung_constant * MEXP(ln_physQuant)) * gaunt;
}

/* calc_opacity_and_albedo, continuous_opacity.f90:175-201, with get_kappa_H_bf (:203-246),
 * get_kappa_Hm_bf (:302-324), get_kappa_Hm_ff (:326-341), calc_kappa_H_ff (:248-279) and
 * get_source_function (:392-409).  kr is scratch of length nz. */
static void opacity_and_albedo(opillar *p, const otab *t, int iw, oreal *kr) {
  const int nz = p->nz;
  oreal **f = p->f;
  const oreal chi = t->chi[iw], wa3 = t->wa3[iw];
  for (int i = 0; i < nz; i++) f[P_STIM][i] = 1.0 - MPOW(10.0, -(chi * f[P_THETA][i])); /* :171 */
  for (int i = 0; i < nz; i++) {
    /* get_kappa_H_bf :233-244 */
    oreal sm = 0.0;
    oreal ktemp = k_cgs * f[P_T][i];
    oreal ktemp1 = k1_cgs * f[P_T1][i];
    for (int n = 0; n < MDIM; n++) {
      oreal n1 = t->n1_array[n];
      sm = sm + (t->g[iw * MDIM + n] * (n1 * (n1 * n1))) * MEXP(-(t->chi_n[n] * ktemp1));
    }
    oreal unsold = ((0.5 * ktemp) * RydbergEnergy1) *
                    (MEXP(-(t->chi_m * ktemp1)) - MEXP(-(RydbergEnergy * ktemp1)));
    oreal kHbf = (((AHbf * f[P_STIM][i]) * f[P_IONF][i]) * wa3) * (unsold + sm);
    /* get_kappa_Hm_bf :318-322 */
    oreal kHmbf = (t->wa[iw] < 16000.0)
                       ? ((f[P_HMBF][i] * f[P_STIM][i]) * f[P_IONF][i]) * t->s_coeff[iw]
                       : 0.0;
    /* get_kappa_Hm_ff :337-339 */
    oreal flam = ((t->f_coeff[iw * 3 + 0] + t->f_coeff[iw * 3 + 1] * f[P_LGT][i]) +
                   t->f_coeff[iw * 3 + 2] * f[P_LGT2][i]) - 26.0;
    oreal kHmff = (((f[P_IONF][i] * f[P_NE][i]) * k_cgs) * f[P_T][i]) * MPOW(10.0, flam);
    kr[i] = (((kHbf + kHmbf) + kHmff) + f[P_ESCAT][i]) * mp1; /* :188 */
    f[P_OMA][i] = ((kHbf + kHmbf) + kHmff) * mp1; /* absorption part of kr, stable form */
    f[P_OP][i] = kr[i] * f[P_RHO][i];                          /* :189 */
  }
  for (int i = 0; i < nz; i++) { /* calc_kappa_H_ff :261-277 */
    if ((1.0 - f[P_X][i]) > switch_ionfraction) {
      oreal g_ff = 1.0 + t->gff_factor[iw] * (((f[P_THETA1][i] * log10e) * t->chi1[iw]) + 0.5);
      oreal energyfactor = (((0.5 * log10e) * f[P_THETA1][i]) * Iev1) * MPOW(10.0, -(f[P_THETA][i] * Iev));
      oreal kHff = ((((f[P_STIM][i] * f[P_IONF][i]) * alpha0) * wa3) * g_ff) * energyfactor;
      kr[i] = kr[i] + kHff * mp1;
      f[P_OMA][i] = f[P_OMA][i] + kHff * mp1;
      f[P_OP][i] = f[P_OP][i] + kr[i] * f[P_RHO][i];
    } else {
      oreal ob = bremsstrahlung(p, i, t->nu[iw]);
      f[P_OP][i] = f[P_OP][i] + ob;
      kr[i] = kr[i] + f[P_OP][i] * f[P_RHO1][i];
      f[P_OMA][i] = f[P_OMA][i] + f[P_OP][i] * f[P_RHO1][i];
    }
  }
  for (int i = 0; i < nz; i++) {
    f[P_ALB][i] = (f[P_ESCAT][i] * mp1) / kr[i]; /* :195 */
    f[P_OMA][i] = f[P_OMA][i] / kr[i];             /* = 1 - albedo without cancellation */
    f[P_OP1][i] = 1.0 / f[P_OP][i];              /* :196 */
    f[P_OP2][i] = f[P_OP][i] * f[P_OP][i];       /* :197 */
  }
  for (int i = 0; i < nz; i++) { /* get_source_function :399-407 */
    oreal damping = (t->damping_factor_const * f[P_T1][i]) * t->wcm1[iw];
    if (damping > log_overflow_limit) damping = log_overflow_limit;
    f[P_S][i] = (t->source_function_const * t->w1cm5[iw]) / (MEXP(damping) - 1.0);
  }
}

/* grey_parameters, continuous_opacity.f90:377-390 */
static void grey_parameters(opillar *p, oreal sigma_grey) {
  oreal **f = p->f;
  for (int i = 0; i < p->nz; i++) {
    oreal T = f[P_T][i], T2 = T * T;
    f[P_S][i] = sigma_sb * (T2 * T2);
    oreal alpha_grey = (3.68e22 * MPOW(T, -3.5)) * f[P_RHO][i];
    f[P_OP][i] = (alpha_grey + sigma_grey) * f[P_RHO][i];
    f[P_ALB][i] = sigma_grey / (alpha_grey + sigma_grey);
    f[P_OMA][i] = alpha_grey / (alpha_grey + sigma_grey);
    f[P_OP1][i] = 1.0 / f[P_OP][i];
    f[P_OP2][i] = f[P_OP][i] * f[P_OP][i];
  }
}

/* get_tridag_coefficients -> fill_center_coeffs + fill_boundary_coeffs,
 * auxiliary.f90:111-201.  ex receives the diagonal excess -(a+b+c) computed directly
 * (used only by the stable form). */
static void tridag_coefficients(oreal *aa, oreal *bb, oreal *cc, oreal *dd, oreal *ex,
                                const opillar *p, oreal dz, oreal dz2, oreal *kp, int stable) {
  const int nz = p->nz;
  oreal *const *f = p->f;
  for (int iz = 0; iz < nz - 1; iz++) kp[iz] = 0.5 * (f[P_OP][iz + 1] + f[P_OP][iz]); /* :147-149 */
  for (int iz = 1; iz < nz - 1; iz++) { /* :159-165; kappa_m(iz) == kappa_p(iz-1) */
    oreal op = f[P_OP][iz];
    aa[iz] = f[P_OP2][iz] / kp[iz - 1];
    cc[iz] = f[P_OP2][iz] / kp[iz];
    oreal oma = stable ? f[P_OMA][iz] : (1.0 - f[P_ALB][iz]);
    oreal zeta = (dz2 * (op * (op * op))) * oma;
    bb[iz] = -((aa[iz] + cc[iz]) + zeta);
    dd[iz] = -(f[P_S][iz] * zeta);
    ex[iz] = zeta;
  }
  /* :187-197 */
  oreal zeta = ((f[P_OP][0] * dz2) * (stable ? f[P_OMA][0] : (1.0 - f[P_ALB][0]))) * 0.25;
  aa[0] = 0.0;
  bb[0] = -(((f[P_OP1][0] + dz) + zeta) * f[P_OP2][0]);
  cc[0] = f[P_OP][0];
  dd[0] = -((f[P_S][0] * zeta) * f[P_OP2][0]);
  ex[0] = (dz + zeta) * f[P_OP2][0];
  int n = nz - 1;
  zeta = ((f[P_OP][n] * dz2) * (stable ? f[P_OMA][n] : (1.0 - f[P_ALB][n]))) * 0.25;
  aa[n] = f[P_OP][n];
  bb[n] = -(((f[P_OP1][n] + dz) + zeta) * f[P_OP2][n]);
  cc[n] = 0.0;
  dd[n] = -((f[P_S][n] * zeta) * f[P_OP2][n]);
  ex[n] = (dz + zeta) * f[P_OP2][n];
}

/* tridag, auxiliary.f90:14-47.  Returns 0, or -1 on an exactly zero pivot (the reference
 * stops there; here the solve continues so that a status can be reported). */
static int tridag(const oreal *a, const oreal *b, const oreal *c, const oreal *r, oreal *u,
                  int n, oreal *gam) {
  int bad = 0;
  oreal bet = b[0];
  if (bet == 0.0) bad = -1;
  u[0] = r[0] / bet;
  for (int j = 1; j < n; j++) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    if (bet == 0.0) bad = -1;
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 2; j >= 0; j--) u[j] = u[j] - gam[j + 1] * u[j + 1];
  return bad;
}

/* Same system, difference-form pivots: bet_j = -(c_j + h_j) with
 * h_j = e_j + a_j h_{j-1} / (c_{j-1} + h_{j-1}), all terms non-negative.  The back-substitution
 * also returns the differences D_j = U_j - U_{j+1} = u_j - q_j U_{j+1}, q_j = h_j/(c_j + h_j):
 * in optically thin layers |gamma| = 1 - q rounds to 1 and U_j - U_{j+1} is below the
 * resolution of U itself, while u_j and q_j U_{j+1} are of the size of the difference. */
static int tridag_stable(const oreal *a, const oreal *c, const oreal *r, const oreal *e,
                         oreal *u, int n, oreal *gam, oreal *q, oreal *D) {
  int bad = 0;
  oreal h = e[0];
  oreal bet = -(c[0] + h);
  if (bet == 0.0) bad = -1;
  u[0] = r[0] / bet;
  for (int j = 1; j < n; j++) {
    oreal den = c[j - 1] + h;
    gam[j] = -(c[j - 1] / den);
    q[j - 1] = h / den;
    h = e[j] + (a[j] * h) / den;
    bet = -(c[j] + h);
    if (bet == 0.0) bad = -1;
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 2; j >= 0; j--) {
    oreal uf = u[j];
    u[j] = uf - gam[j + 1] * u[j + 1];
    D[j] = uf - q[j] * u[j + 1];
  }
  return bad;
}

/* 6th-order flux (auxiliary.f90:64-109, ghosts :49-62) written in the differences
 * Delta_m = f_m - f_{m+1}: f_{m+k} - f_{m-k} = -(Delta_{m-k} + ... + Delta_{m+k-1}), and the
 * ghost zones mirror the differences next to each boundary.  Same value as the stencil on
 * f in exact arithmetic; used by the stable form (nz >= 4), whose D_j are accurate where
 * the differences of U are not resolved. */
static void calc_flux_diff(const oreal *D, opillar *p, oreal dz1, oreal *Dl) {
  const int nz = p->nz, n1 = 3;
  oreal **pf = p->f;
  for (int m = n1; m <= nz + 1; m++) Dl[m] = D[m - n1];
  for (int i = 1; i <= 3; i++) {
    Dl[nz + 2 + i - 1] = Dl[nz + 2 - i];
    Dl[n1 - i] = Dl[n1 + i - 1];
  }
  for (int j = 0; j < nz; j++) {
    int m = n1 + j;
    oreal s1 = Dl[m - 1] + Dl[m];
    oreal s2 = (s1 + Dl[m - 2]) + Dl[m + 1];
    oreal s3 = (s2 + Dl[m - 3]) + Dl[m + 2];
    oreal df = -((1.0 / 60.0) * (((45.0 * s1) - 9.0 * s2) + s3));
    pf[P_FLUX][j] = ((-1.0 * pf[P_OP1][j]) * df) * dz1;
  }
}

/* update_ghosts, auxiliary.f90:49-62 (f has nz+6 entries, n1 = 3, n2 = nz+2 0-based) */
static void update_ghosts(oreal *f, int nz) {
  const int n1 = 3, n2 = nz + 2;
  for (int i = 1; i <= 3; i++) {
    f[n1 - i] = 2.0 * f[n1] - f[n1 + i];
    f[n2 + i] = 2.0 * f[n2] - f[n2 - i];
  }
}

/* der + calc_flux, auxiliary.f90:64-78 and :96-109 */
static void calc_flux(const oreal *f, opillar *p, oreal dz1) {
  const int n1 = 3;
  oreal **pf = p->f;
  for (int i = 0; i < p->nz; i++) {
    int c = n1 + i;
    oreal df = (1.0 / 60.0) * (((45.0 * (f[c + 1] - f[c - 1])) - 9.0 * (f[c + 2] - f[c - 2])) +
                                (f[c + 3] - f[c - 3]));
    pf[P_FLUX][i] = ((-1.0 * pf[P_OP1][i]) * df) * dz1;
  }
}

int oracle_solve_columns(const oracle_params *prm, const double *wa, const double *rho,
                         const double *T, int64_t col0, int64_t col1, double *U, double *kappa,
                         double *V, int64_t *bad_item) {
  const int nz = prm->nz, nw = prm->nw, mz = nz + 6;
  const int64_t ncol = (int64_t)prm->nx * prm->ny;
  if (bad_item) *bad_item = -1;
  if (nz < 2 || nw < 1 || prm->nx < 1 || prm->ny < 1 || col0 < 0 || col1 > ncol) return ORACLE_EINVAL;
  if (prm->lgrey && nw != 1) return ORACLE_EGREY; /* flux_feautrier.f90:84-87 */
  otab t;
  int rc = ORACLE_OK;
  if (!prm->lgrey) {
    if ((rc = otab_build(&t, wa, nw)) != ORACLE_OK) return rc;
  } else {
    memset(&t, 0, sizeof t);
  }
  opillar p;
  if (pillar_alloc(&p, nz) != ORACLE_OK) {
    otab_free(&t);
    return ORACLE_ENOMEM;
  }
  oreal *work = (oreal *)calloc((size_t)nz * 10 + 2 * mz, sizeof(oreal));
  if (!work) {
    free(p.mem);
    otab_free(&t);
    return ORACLE_ENOMEM;
  }
  oreal *a = work, *b = work + nz, *c = work + 2 * nz, *d = work + 3 * nz, *ex = work + 4 * nz;
  oreal *kr = work + 5 * nz, *gam = work + 6 * nz, *kp = work + 7 * nz, *u = work + 8 * nz;
  oreal *qv = work + 8 * nz + mz, *Dv = work + 9 * nz + mz, *Dl = work + 10 * nz + mz;
  const oreal dz = prm->dz, dz1 = (oreal)1.0 / dz, dz2 = dz * dz;
  for (int64_t col = col0; col < col1; col++) {
    for (int i = 0; i < nz; i++) {
      p.f[P_RHO][i] = rho[col * nz + i];
      p.f[P_T][i] = T[col * nz + i];
    }
    pillars(&p, prm->fully_ionized_T);
    for (int iw = 0; iw < nw; iw++) {
      if (prm->lgrey)
        grey_parameters(&p, prm->sigma_grey);
      else
        opacity_and_albedo(&p, &t, iw, kr);
      tridag_coefficients(a, b, c, d, ex, &p, dz, dz2, kp, prm->form == ORACLE_FORM_STABLE);
      const int stable = prm->form == ORACLE_FORM_STABLE;
      int bad = stable ? tridag_stable(a, c, d, ex, u + 3, nz, gam, qv, Dv) : tridag(a, b, c, d, u + 3, nz, gam);
      if (bad && rc == ORACLE_OK) {
        rc = ORACLE_EZEROPIVOT;
        if (bad_item) *bad_item = col * nw + iw;
      }
      update_ghosts(u, nz);
      if (stable && nz >= 4)
        calc_flux_diff(Dv, &p, dz1, Dl);
      else
        calc_flux(u, &p, dz1);
      size_t item = (size_t)iw * (size_t)ncol + (size_t)col;
      if (U)
        for (int i = 0; i < mz; i++) U[item * mz + i] = (double)u[i];
      if (kappa)
        for (int i = 0; i < nz; i++) kappa[item * nz + i] = (double)p.f[P_OP][i];
      if (V)
        for (int i = 0; i < nz; i++) V[item * nz + i] = (double)p.f[P_FLUX][i];
    }
  }
  free(work);
  free(p.mem);
  otab_free(&t);
  return rc;
}

int oracle_solve_block(const oracle_params *p, const double *wa, const double *rho,
                       const double *T, double *U, double *kappa, double *V, int64_t *bad_item) {
  return oracle_solve_columns(p, wa, rho, T, 0, (int64_t)p->nx * p->ny, U, kappa, V, bad_item);
}
