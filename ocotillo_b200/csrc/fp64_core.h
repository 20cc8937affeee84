/*
 * fp64_core.h -- the FP64 per-item arithmetic of the plain and stable forms, shared by the
 * FP64 kernels (kernels_fp64.cu) and the mixed kernels' FP64 re-solve of flagged items
 * (kernels_mixed.cu).
 *
 *   pillar_record  one (column, z) record: Saha ionization and every factor of the
 *                  reference's per-(z, lambda) opacity that depends on z only
 *                  (gas_state.f90:30-110, continuous_opacity.f90:143-163 and the z-only parts
 *                  of :203-300), each with the reference's operand order.
 *   opacity_at     calc_opacity_and_albedo for one (z, lambda), continuous_opacity.f90:175-201.
 *   solve_item     one (column, wavelength) item: coefficients (auxiliary.f90:111-201), the
 *                  Thomas sweep (:14-47) with its scratch, ghosts (:49-62) and flux (:64-109).
 *
 * Bit-faithfulness to the CPU oracle needs this code compiled without FMA contraction
 * (kernels_fp64.cu is built with -fmad=false); the exponentials and logarithms (ocomath) use
 * non-contracting intrinsics everywhere.
 */
#ifndef OCO_FP64_CORE_H
#define OCO_FP64_CORE_H

#include <cuda_runtime.h>

#include "ocomath.h"
#include "oco_consts.h"
#include "oco_internal.h"

namespace oco {
using namespace k;

/* ---- pillars ------------------------------------------------------------------------ */
/* The record of one (column, z) cell from its rho and T. */
__device__ __forceinline__ void pillar_record(const double r, const double t, double fully_ionized_T, int grey,
                                              double *__restrict__ o) {
  if (grey) { /* grey_parameters, continuous_opacity.f90:383-384 */
    double t2 = t * t;
    o[G_RHO] = r;
    o[G_S] = sigma_sb * (t2 * t2);
    o[G_ALPHA] = (3.68e22 * oco_pow(t, -3.5)) * r;
    return;
  }
  const double rho1 = 1.0 / r; /* gas_state.f90:34-35 */
  const double T1 = 1.0 / t;
  /* calc_hydrogen_ion_frac, gas_state.f90:57-74 */
  double constants = saha_const * oco_pow(t, 1.5);
  double exparg = (T1 * hydrogen_ionization_eV) * k1_eV;
  double niine_ni = constants * oco_exp(-exparg);
  double c_ion = (mp * rho1) * niine_ni;
  double x = 0.5 * (sqrt(c_ion * c_ion + 4.0 * c_ion) - c_ion);
  if (t > fully_ionized_T) x = 1.0;
  /* solve_gas_state, gas_state.f90:85-97 */
  double nn = r * mp1;
  double invn = rho1 * mp;
  double nHII = x * nn;
  double nHI = nn - nHII;
  double ne = nHII;
  double ionf = (nHI != 0.0) ? nHI / (nHI + nHII) : 0.0;
  double Pe = (ne * k_cgs) * t;                    /* gas_state.f90:108 */
  double escat = (alpha_e * nHII) * invn;          /* c_o :149 */
  double theta = 5040.0 * T1;                      /* gas_state.f90:40-43 */
  double theta1 = 1.0 / theta;
  double lgt = oco_log10(theta);
  double hmbf = ((4.158e-10 * Pe) * oco_pow(theta, 2.5)) * oco_pow10(0.754 * theta); /* c_o :161 */
  /* z-only factors of get_kappa_H_bf, c_o :234-242.  chi_n(n) = Ry*(1 - 1*(1/n)**2) as
   * in pre_calc_opacity_quantities :121-129; chi_m equals chi_n(6). */
  double ktemp = k_cgs * t, ktemp1 = k1_cgs * T1;
  double E[6];
#pragma unroll
  for (int nq = 1; nq <= 6; nq++) {
    double n1 = 1.0 / (double)nq;
    double chi_n = RydbergEnergy * (1.0 - 1.0 * (n1 * n1));
    E[nq - 1] = oco_exp(-(chi_n * ktemp1));
  }
  double unsold = ((0.5 * ktemp) * RydbergEnergy1) * (E[5] - oco_exp(-(RydbergEnergy * ktemp1)));
  o[F_RHO] = r;
  o[F_RHO1] = rho1;
  o[F_T1] = T1;
  o[F_DFT1] = damping_factor_const * T1;
  o[F_THETA] = theta;
  o[F_TH1L] = theta1 * log10e;
  o[F_LGT] = lgt;
  o[F_LGT2] = lgt * lgt;
  o[F_IONF] = ionf;
  o[F_ESCAT] = escat;
  o[F_ESCM] = escat * mp1;
  o[F_HMBF] = hmbf;
  o[F_NEUTRAL] = ((1.0 - x) > switch_ionfraction) ? 1.0 : 0.0;
#pragma unroll
  for (int q = 0; q < 6; q++) o[F_E1 + q] = E[q];
  o[F_UNSOLD] = unsold;
  o[F_AFF] = ((ionf * ne) * k_cgs) * t;                                             /* c_o :339 */
  o[F_EF] = (((0.5 * log10e) * theta1) * Iev1) * oco_pow10(-(theta * Iev));   /* c_o :265 */
  o[F_TPOW] = oco_pow(t * 1e-4, -1.5);                                              /* c_o :290 */
  o[F_LZ] = (oco_log(ne * (nHI + nHII)) + 2.0 * oco_log(1.0)) - 0.5 * oco_log(t);   /* c_o :292-294 */
  o[F_LNRHO] = oco_log(r);
  o[F_PAD] = 0.0;
}

/* ---- per-wavelength constants ------------------------------------------------------- */
struct Lam {
  double chi, chi1, gff, wa3, s, hmon, f1, f2, f3, gn[6], nu9, l3nu, hnuk, wcm1, sw5;
};

__device__ __forceinline__ void load_lam(Lam &L, const double *__restrict__ lam, int iw, int nw) {
#define LD(f) __ldg(lam + (int64_t)(f) * nw + iw)
  L.chi = LD(L_CHI);
  L.chi1 = LD(L_CHI1);
  L.gff = LD(L_GFF);
  L.wa3 = LD(L_WA3);
  L.s = LD(L_SCOEF);
  L.hmon = LD(L_HMON);
  L.f1 = LD(L_F1);
  L.f2 = LD(L_F2);
  L.f3 = LD(L_F3);
#pragma unroll
  for (int q = 0; q < 6; q++) L.gn[q] = LD(L_GN1 + q);
  L.nu9 = LD(L_NU9);
  L.l3nu = LD(L_L3NU);
  L.hnuk = LD(L_HNUK);
  L.wcm1 = LD(L_WCM1);
  L.sw5 = LD(L_SW5);
#undef LD
}

/* The constants as opacity_at reads them: LamR holds them in registers (loaded from the global
 * table); LamS reads them from the warp's shared-memory table [field][32], one column per lane,
 * which frees ~40 registers of the staged kernel (no spills at 128 registers; +3% plain, +5%
 * stable on the AGN grid).  Same values, so the same bits. */
enum { NLF = 20 }; /* fields of the shared table, in the order of store_lam_shared */
struct LamR {
  Lam L;
  template <class IT> __device__ __forceinline__ LamR(const IT &it, const double *, bool load = true) {
    if (load) load_lam(L, it.lam(), it.iw(), it.nw()); /* grey: no wavelength table */
  }
  __device__ __forceinline__ double chi() const { return L.chi; }
  __device__ __forceinline__ double chi1() const { return L.chi1; }
  __device__ __forceinline__ double gff() const { return L.gff; }
  __device__ __forceinline__ double wa3() const { return L.wa3; }
  __device__ __forceinline__ double s() const { return L.s; }
  __device__ __forceinline__ double hmon() const { return L.hmon; }
  __device__ __forceinline__ double f1() const { return L.f1; }
  __device__ __forceinline__ double f2() const { return L.f2; }
  __device__ __forceinline__ double f3() const { return L.f3; }
  __device__ __forceinline__ double gn(int q) const { return L.gn[q]; }
  __device__ __forceinline__ double nu9() const { return L.nu9; }
  __device__ __forceinline__ double l3nu() const { return L.l3nu; }
  __device__ __forceinline__ double hnuk() const { return L.hnuk; }
  __device__ __forceinline__ double wcm1() const { return L.wcm1; }
  __device__ __forceinline__ double sw5() const { return L.sw5; }
};
struct LamS {
  const double *p; /* &table[0][lane] */
  template <class IT> __device__ __forceinline__ LamS(const IT &, const double *col, bool = true) : p(col) {}
  __device__ __forceinline__ double f(int k) const { return p[k * 32]; }
  __device__ __forceinline__ double chi() const { return f(0); }
  __device__ __forceinline__ double chi1() const { return f(1); }
  __device__ __forceinline__ double gff() const { return f(2); }
  __device__ __forceinline__ double wa3() const { return f(3); }
  __device__ __forceinline__ double s() const { return f(4); }
  __device__ __forceinline__ double hmon() const { return f(5); }
  __device__ __forceinline__ double f1() const { return f(6); }
  __device__ __forceinline__ double f2() const { return f(7); }
  __device__ __forceinline__ double f3() const { return f(8); }
  __device__ __forceinline__ double gn(int q) const { return f(9 + q); }
  __device__ __forceinline__ double nu9() const { return f(15); }
  __device__ __forceinline__ double l3nu() const { return f(16); }
  __device__ __forceinline__ double hnuk() const { return f(17); }
  __device__ __forceinline__ double wcm1() const { return f(18); }
  __device__ __forceinline__ double sw5() const { return f(19); }
};
/* Lane's column of the warp's shared table (wavelength iw of the global table). */
__device__ __forceinline__ void store_lam_shared(double *col, const double *__restrict__ lam, int iw, int nw) {
  const int src[NLF] = {L_CHI, L_CHI1, L_GFF, L_WA3, L_SCOEF, L_HMON, L_F1, L_F2, L_F3, L_GN1, L_GN2, L_GN3,
                        L_GN4, L_GN5, L_GN6, L_NU9, L_L3NU, L_HNUK, L_WCM1, L_SW5};
#pragma unroll
  for (int k = 0; k < NLF; k++) col[k * 32] = __ldg(lam + (int64_t)src[k] * nw + iw);
}

/* One pillar record, read through the read-only cache (global) or from shared memory. */
struct GlobalRec {
  const double *p;
  __device__ __forceinline__ double operator[](int f) const { return __ldg(p + f); }
};
struct SharedRec {
  const double *p;
  __device__ __forceinline__ double operator[](int f) const { return p[f]; }
};

struct Opac {
  double op, alb, S;
  double oma; /* stable form: 1 - albedo from the absorption terms (no cancellation) */
};

/* calc_opacity_and_albedo for one (z, lambda), continuous_opacity.f90:175-201 with
 * :171, :233-244, :318-322, :337-339, :261-277, :290-298, :399-407. */
/* 10^y1, 10^y2 and e^x3 as oco_pow10, oco_pow10 and oco_exp compute them, with the three
 * fast phases side by side (branch-free, so that their dependency chains overlap) and the
 * full evaluation only where a fast phase cannot decide. */
__device__ __forceinline__ void pow10_pow10_exp(double y1, double y2, double x3, double &r1, double &r2,
                                                double &r3) {
  const double p1 = OCO_M(y1, OCO_LN10_HI), p2 = OCO_M(y2, OCO_LN10_HI);
  const double l1 = OCO_A(OCO_FMA(y1, OCO_LN10_HI, -p1), OCO_M(y1, OCO_LN10_LO));
  const double l2 = OCO_A(OCO_FMA(y2, OCO_LN10_HI, -p2), OCO_M(y2, OCO_LN10_LO));
  double f1, f2, f3;
  const int ok1 = oco_exp_fast_nb(p1, l1, &f1);
  const int ok2 = oco_exp_fast_nb(p2, l2, &f2);
  const int ok3 = oco_exp_fast_nb(x3, 0.0, &f3);
  if (!ok1) f1 = oco_exp_dd(p1, l1);
  if (!ok2) f2 = oco_exp_dd(p2, l2);
  if (!ok3) f3 = oco_exp_dd(x3, 0.0);
  r1 = OCO_M(1.0, f1);
  r2 = OCO_M(1.0, f2);
  r3 = f3;
}

template <bool STABLE, class R, class LM>
__device__ __forceinline__ Opac opacity_at(const R P, const LM &L) {
  double damping = P[F_DFT1] * L.wcm1();
  if (damping > log_overflow_limit) damping = log_overflow_limit;
  double p10_stim, p10_flam, e_planck;
  pow10_pow10_exp(-(L.chi() * P[F_THETA]), ((L.f1() + L.f2() * P[F_LGT]) + L.f3() * P[F_LGT2]) - 26.0, damping,
                  p10_stim, p10_flam, e_planck);
  /* read after the exponentials: one register fewer across them (the batch kernels spill less) */
  const double ionf = P[F_IONF];
  const double stim = 1.0 - p10_stim;
  double sm = 0.0;
#pragma unroll
  for (int q = 0; q < 6; q++) sm = sm + L.gn(q) * P[F_E1 + q];
  double kHbf = (((AHbf * stim) * ionf) * L.wa3()) * (P[F_UNSOLD] + sm);
  double kHmbf = (L.hmon() != 0.0) ? ((P[F_HMBF] * stim) * ionf) * L.s() : 0.0;
  double kHmff = P[F_AFF] * p10_flam; /* 10^(f1 + f2 lgt + f3 lgt^2 - 26) */
  double kr = (((kHbf + kHmbf) + kHmff) + P[F_ESCAT]) * mp1;
  double kabs = STABLE ? ((kHbf + kHmbf) + kHmff) * mp1 : 0.0;
  const double rho = P[F_RHO];
  double op = kr * rho;
  if (P[F_NEUTRAL] != 0.0) {
    double g_ff = 1.0 + L.gff() * ((P[F_TH1L] * L.chi1()) + 0.5);
    double kHff = ((((stim * ionf) * alpha0) * L.wa3()) * g_ff) * P[F_EF];
    kr = kr + kHff * mp1;
    op = op + kr * rho;
    if (STABLE) kabs = kabs + kHff * mp1;
  } else {
    double gaunt = oco_log(oco_exp(5.960 - (sqrt3 * pi1) * oco_log(L.nu9() * P[F_TPOW])) + exp1);
    double lnq = (P[F_LZ] - L.l3nu()) + oco_log(1.0 - oco_exp(-(L.hnuk() * P[F_T1])));
    double krho = (bremsstrahlung_constant * oco_exp(lnq)) * gaunt;
    op = op + krho;
    kr = kr + op * P[F_RHO1];
    if (STABLE) kabs = kabs + op * P[F_RHO1];
  }
  Opac o;
  o.op = op;
  o.alb = P[F_ESCM] / kr;
  o.oma = STABLE ? kabs / kr : 0.0;
  o.S = L.sw5() / (e_planck - 1.0);
  return o;
}

/* grey_parameters, continuous_opacity.f90:377-390 */
template <class R>
__device__ __forceinline__ Opac opacity_grey(const R P, double sg) {
  double alpha = P[G_ALPHA];
  Opac o;
  o.op = (alpha + sg) * P[G_RHO];
  o.alb = sg / (alpha + sg);
  o.oma = alpha / (alpha + sg);
  o.S = P[G_S];
  return o;
}

/* ---- the solve ----------------------------------------------------------------------- */
/* Solves one (column, wavelength) item.  `active` false: the lane only keeps the warp's
 * shared pipeline in step (staged path, wavelength index beyond nw) and stores nothing. */
/* The reverse sweep of one item (back-substitution, tridag :43-45; ghost zones :49-62; flux
 * :96-109) from the forward sweep's last u and its scratch (gam, uu, o1s and, stable form, qs at
 * stride it.ss()), storing U, V and the emergent fluxes through the item accessor. */
/* Issues an L2 prefetch of the line holding p. */
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(p)));
}

/* PF: the scratch was written long before (by another kernel) and few warps run, so its loads
 * are DRAM latency: 1/kappa is loaded with the other scratch arrays 8 levels ahead of the
 * serial chain and the next blocks of 8 levels are prefetched into L2 (the block solves keep
 * PF off: their scratch is recent and many warps hide its latency). */
template <int FORM, class IT, bool PF = false>
__device__ __forceinline__ void solve_reverse(const IT &it, double u, const double *__restrict__ gam,
                                              const double *__restrict__ uu, const double *__restrict__ o1s,
                                              const double *__restrict__ qs) {
  const int nz = it.nz();
  const int64_t ss = it.ss();
  double *Ub = it.U();
  double *Vb = it.V();
  const double dz1 = it.dz1();
  const int64_t uz = it.uz();
  double vtop = 0.0, vbot = 0.0;
  if (FORM == 1 && nz >= 4) {
    /* Stable form: the differences D_k = U_k - U_{k+1} = u_k - q_k U_{k+1} come out of the
     * back-substitution directly, and the flux is the 6th-order stencil written in them
     * (ghost differences mirror the interior ones); exact in the same arithmetic as the
     * stencil on U, accurate where U's differences are below its resolution. */
    const int n = nz;
    double Un = u; /* U_{n-1} */
    if (Ub) __stcs(&Ub[(3 + n - 1) * uz], Un);
    double Uk[3], Dt[3];
    for (int t = 0; t < 3; t++) {
      const int k = n - 2 - t;
      const double uf = uu[k * ss];
      Dt[t] = uf - qs[k * ss] * Un;
      Un = uf - gam[(k + 1) * ss] * Un;
      Uk[t] = Un;
      if (Ub) __stcs(&Ub[(3 + k) * uz], Un);
    }
    const double fn = u;
    if (Ub) __stcs(&Ub[(n + 3) * uz], 2.0 * fn - Uk[0]);
    if (Ub) __stcs(&Ub[(n + 4) * uz], 2.0 * fn - Uk[1]);
    if (Ub) __stcs(&Ub[(n + 5) * uz], 2.0 * fn - Uk[2]);
    double d0 = Dt[2], d1 = Dt[1], d2 = Dt[0], d3 = Dt[0], d4 = Dt[1], d5 = Dt[2];
    auto emitDo = [&](int j, double o1j) -> double {
      const double s1 = d2 + d3;
      const double s2 = (s1 + d1) + d4;
      const double s3 = (s2 + d0) + d5;
      const double df = -((1.0 / 60.0) * (((45.0 * s1) - 9.0 * s2) + s3));
      const double v = ((-1.0 * o1j) * df) * dz1;
      if (Vb) __stcs(&Vb[j * it.vz()], v);
      return v;
    };
    auto emitD = [&](int j) -> double { return emitDo(j, o1s[j * ss]); };
    vtop = emitD(n - 1);
    double U0 = Uk[2], U1 = Uk[1], U2 = Uk[0], U3 = u; /* the four lowest U seen so far */
    auto stepDo = [&](int k, double uf, double qk, double gk1, double o1k3) {
      const double Dk = uf - qk * Un;
      Un = uf - gk1 * Un;
      if (Ub) __stcs(&Ub[(3 + k) * uz], Un);
      U3 = U2; U2 = U1; U1 = U0; U0 = Un;
      d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = Dk;
      emitDo(k + 3, o1k3);
    };
    auto stepD = [&](int k, double uf, double qk, double gk1) { stepDo(k, uf, qk, gk1, o1s[(k + 3) * ss]); };
    int k = n - 5;
    for (; k >= 7; k -= 8) { /* scratch loads of 8 steps hoisted off the serial chain */
      double ub[8], qb[8], gb[8];
      if (PF) {
        double ob[8];
        for (int q = 16; q < 24 && k - q >= 0; q++) { /* the block after next */
          prefetch_l2(&uu[(k - q) * ss]);
          prefetch_l2(&qs[(k - q) * ss]);
          prefetch_l2(&gam[(k - q + 1) * ss]);
          prefetch_l2(&o1s[(k - q + 3) * ss]);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          ub[q] = uu[(k - q) * ss];
          qb[q] = qs[(k - q) * ss];
          gb[q] = gam[(k - q + 1) * ss];
          ob[q] = o1s[(k - q + 3) * ss];
        }
#pragma unroll
        for (int q = 0; q < 8; q++) stepDo(k - q, ub[q], qb[q], gb[q], ob[q]);
      } else {
#pragma unroll
        for (int q = 0; q < 8; q++) {
          ub[q] = uu[(k - q) * ss];
          qb[q] = qs[(k - q) * ss];
          gb[q] = gam[(k - q + 1) * ss];
        }
#pragma unroll
        for (int q = 0; q < 8; q++) stepD(k - q, ub[q], qb[q], gb[q]);
      }
    }
    for (; k >= 0; k--) stepD(k, uu[k * ss], qs[k * ss], gam[(k + 1) * ss]);
    if (Ub) __stcs(&Ub[2 * uz], 2.0 * U0 - U1);
    if (Ub) __stcs(&Ub[1 * uz], 2.0 * U0 - U2);
    if (Ub) __stcs(&Ub[0], 2.0 * U0 - U3);
    const double D0 = d0, D1 = d1, D2 = d2;
    d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = D0;
    emitD(2);
    d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = D1;
    emitD(1);
    d5 = d4; d4 = d3; d3 = d2; d2 = d1; d1 = d0; d0 = D2;
    vbot = emitD(0);
  } else if (nz >= 4) {
    auto emitV = [&](int j, double o1j, double w0, double w1, double w2, double w4, double w5, double w6) -> double {
      double df = (1.0 / 60.0) * (((45.0 * (w4 - w2)) - 9.0 * (w5 - w1)) + (w6 - w0));
      double v = ((-1.0 * o1j) * df) * dz1;
      if (Vb) __stcs(&Vb[j * it.vz()], v);
      return v;
    };
    const int n = nz;
    double u1 = u; /* U_{n-1} */
    double u2 = uu[(n - 2) * ss] - gam[(n - 1) * ss] * u1;
    double u3 = uu[(n - 3) * ss] - gam[(n - 2) * ss] * u2;
    double u4 = uu[(n - 4) * ss] - gam[(n - 3) * ss] * u3;
    if (Ub) __stcs(&Ub[(3 + n - 1) * uz], u1);
    if (Ub) __stcs(&Ub[(3 + n - 2) * uz], u2);
    if (Ub) __stcs(&Ub[(3 + n - 3) * uz], u3);
    if (Ub) __stcs(&Ub[(3 + n - 4) * uz], u4);
    double g1 = 2.0 * u1 - u2, g2 = 2.0 * u1 - u3, g3 = 2.0 * u1 - u4;
    if (Ub) __stcs(&Ub[(n + 3) * uz], g1);
    if (Ub) __stcs(&Ub[(n + 4) * uz], g2);
    if (Ub) __stcs(&Ub[(n + 5) * uz], g3);
    double w0 = u4, w1 = u3, w2 = u2, w3 = u1, w4 = g1, w5 = g2, w6 = g3;
    vtop = emitV(n - 1, o1s[(n - 1) * ss], w0, w1, w2, w4, w5, w6);
    int kk = n - 5;
    /* blocks of 8 steps with the scratch loads hoisted off the serial U chain */
    for (; kk >= 7; kk -= 8) {
      double ub[8], gb[8], ob[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        ub[q] = uu[(kk - q) * ss];
        gb[q] = gam[(kk - q + 1) * ss];
        ob[q] = o1s[(kk - q + 3) * ss];
      }
#pragma unroll
      for (int q = 0; q < 8; q++) {
        double Uk = ub[q] - gb[q] * w0;
        if (Ub) __stcs(&Ub[(3 + kk - q) * uz], Uk);
        w6 = w5; w5 = w4; w4 = w3; w3 = w2; w2 = w1; w1 = w0; w0 = Uk;
        emitV(kk - q + 3, ob[q], w0, w1, w2, w4, w5, w6);
      }
    }
    for (; kk >= 0; kk--) {
      double Uk = uu[kk * ss] - gam[(kk + 1) * ss] * w0;
      if (Ub) __stcs(&Ub[(3 + kk) * uz], Uk);
      w6 = w5; w5 = w4; w4 = w3; w3 = w2; w2 = w1; w1 = w0; w0 = Uk;
      emitV(kk + 3, o1s[(kk + 3) * ss], w0, w1, w2, w4, w5, w6);
    }
    double b1 = 2.0 * w0 - w1, b2 = 2.0 * w0 - w2, b3 = 2.0 * w0 - w3;
    if (Ub) __stcs(&Ub[2 * uz], b1);
    if (Ub) __stcs(&Ub[1 * uz], b2);
    if (Ub) __stcs(&Ub[0], b3);
    w6 = w5; w5 = w4; w4 = w3; w3 = w2; w2 = w1; w1 = w0; w0 = b1;
    emitV(2, o1s[2 * ss], w0, w1, w2, w4, w5, w6);
    w6 = w5; w5 = w4; w4 = w3; w3 = w2; w2 = w1; w1 = w0; w0 = b2;
    emitV(1, o1s[1 * ss], w0, w1, w2, w4, w5, w6);
    w6 = w5; w5 = w4; w4 = w3; w3 = w2; w2 = w1; w1 = w0; w0 = b3;
    vbot = emitV(0, o1s[0], w0, w1, w2, w4, w5, w6);
  } else { /* nz = 2 or 3: the reference's ghost update order matters (ghosts feed ghosts) */
    double f[9];
    const int n1 = 3, n2 = nz + 2;
    f[n1 + nz - 1] = u;
    for (int j = nz - 2; j >= 0; j--) f[n1 + j] = uu[j * ss] - gam[(j + 1) * ss] * f[n1 + j + 1];
    for (int i = 1; i <= 3; i++) {
      f[n1 - i] = 2.0 * f[n1] - f[n1 + i];
      f[n2 + i] = 2.0 * f[n2] - f[n2 - i];
    }
    if (Ub)
      for (int m = 0; m < nz + 6; m++) __stcs(&Ub[m * uz], f[m]);
    for (int j = 0; j < nz; j++) {
      int c = n1 + j;
      double df = (1.0 / 60.0) * (((45.0 * (f[c + 1] - f[c - 1])) - 9.0 * (f[c + 2] - f[c - 2])) +
                                  (f[c + 3] - f[c - 3]));
      double v = ((-1.0 * o1s[j * ss]) * df) * dz1;
      if (Vb) __stcs(&Vb[j * it.vz()], v);
      if (j == 0) vbot = v;
      if (j == nz - 1) vtop = v;
    }
  }
  if (double *p = it.vtop()) __stcs(p, vtop);
  if (double *p = it.vbot()) __stcs(p, vbot);
}

template <int FORM, bool GREY, class IT, class PA, class LMT = LamR>
__device__ __forceinline__ void solve_item(const IT &it, bool active, PA &pa, double *__restrict__ gam,
                                           double *__restrict__ uu, double *__restrict__ o1s,
                                           double *__restrict__ qs, const double *lam_col = nullptr) {
  const int nz = it.nz();
  const int64_t ss = it.ss();
  const LMT L(it, lam_col, !GREY);
  double *Kb = active ? it.K() : nullptr;
  const double dz = it.dz(), dz2 = it.dz2();
  bool bad = false;

  /* forward sweep: row 0 (fill_boundary_coeffs :187-191) */
  Opac cur = GREY ? opacity_grey(pa.at(0), it.sigma_grey()) : opacity_at<FORM == 1>(pa.at(0), L);
  Opac nxt = GREY ? opacity_grey(pa.at(1), it.sigma_grey()) : opacity_at<FORM == 1>(pa.at(1), L);
  double o1 = 1.0 / cur.op, o2 = cur.op * cur.op;
  double zeta = ((cur.op * dz2) * (FORM == 1 ? cur.oma : (1.0 - cur.alb))) * 0.25;
  double bet, h = 0.0;
  if (FORM == 0) {
    bet = -(((o1 + dz) + zeta) * o2);
  } else {
    h = (dz + zeta) * o2;
    bet = -(cur.op + h);
  }
  if (bet == 0.0) bad = true;
  double u = (-((cur.S * zeta) * o2)) / bet;
  uu[0] = u;
  o1s[0] = o1;
  if (Kb) __stcs(&Kb[0], cur.op);
  double c_prev = cur.op;
  double kh_prev = 0.5 * (nxt.op + cur.op); /* kappa_p(1) = kappa_m(2), :147-154 */
  cur = nxt;
  for (int j = 1; j < nz; j++) {
    const double op = cur.op;
    o1 = 1.0 / op;
    o2 = op * op;
    double aa, bb, cc, dd, ee;
    if (j < nz - 1) { /* fill_center_coeffs :159-165 */
      nxt = GREY ? opacity_grey(pa.at(j + 1), it.sigma_grey()) : opacity_at<FORM == 1>(pa.at(j + 1), L);
      aa = o2 / kh_prev;
      double kh = 0.5 * (nxt.op + op);
      cc = o2 / kh;
      double z3 = (dz2 * (op * (op * op))) * (FORM == 1 ? cur.oma : (1.0 - cur.alb));
      bb = -((aa + cc) + z3);
      dd = -(cur.S * z3);
      ee = z3;
      kh_prev = kh;
    } else { /* fill_boundary_coeffs :193-197 */
      aa = op;
      double zt = ((op * dz2) * (FORM == 1 ? cur.oma : (1.0 - cur.alb))) * 0.25;
      bb = -(((o1 + dz) + zt) * o2);
      cc = 0.0;
      dd = -((cur.S * zt) * o2);
      ee = (dz + zt) * o2;
    }
    double g;
    if (FORM == 0) { /* tridag :34-35 */
      g = c_prev / bet;
      bet = bb - aa * g;
    } else { /* difference form: bet = -(c + h), h = e + a*h_prev/(c_prev + h_prev) */
      double den = c_prev + h;
      g = -(c_prev / den);
      qs[(j - 1) * ss] = h / den; /* q_{j-1} = h_{j-1}/(c_{j-1} + h_{j-1}) */
      h = ee + (aa * h) / den;
      bet = -(cc + h);
      (void)bb;
    }
    if (bet == 0.0) bad = true;
    u = (dd - aa * u) / bet; /* tridag :40 */
    gam[j * ss] = g;
    uu[j * ss] = u;
    o1s[j * ss] = o1;
    if (Kb) __stcs(&Kb[j * it.kz()], op);
    c_prev = cc;
    cur = nxt;
  }
  if (!active) return;
  if (bad) {
    atomicAdd(&it.status()[0], 1ull);
    atomicMin(&it.status()[1], it.id());
  }

  solve_reverse<FORM>(it, u, gam, uu, o1s, qs);
}

}  // namespace oco

#endif
