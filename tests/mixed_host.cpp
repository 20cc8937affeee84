// Host build of the mixed form's arithmetic (mixed_core.h: records, wavelength record, opacity,
// rows and the extended-exponent Thomas solve) for the CPU tests: libm exp2f/log2f stand in for
// the GPU's ex2/lg2.approx, everything else is the same code the kernels inline.
#include <vector>

#include "mixed_core.h"
#include "oco_internal.h"

using namespace oco;

// U[(iw*ncol + c)*(nz+6) + z], K and V [(iw*ncol + c)*nz + z]; rho, T [c*nz + z]; waves in Angstrom.
extern "C" void mixed_host_solve(const double *rho, const double *T, const double *wa, int ncol, int nz, int nw,
                                 double dz, double fully_ionized_T, double *U, double *K, double *V) {
  std::vector<double> tab((size_t)NL * nw);
  fill_lambda_table(wa, nw, tab.data());
  std::vector<float> Z((size_t)nz * mx::MZN), work((size_t)8 * nz);
  std::vector<double> dwork((size_t)nz + 6);
  for (int c = 0; c < ncol; c++) {
    for (int z = 0; z < nz; z++) mx::pillar(rho[(size_t)c * nz + z], T[(size_t)c * nz + z], fully_ionized_T, &Z[(size_t)z * mx::MZN]);
    for (int iw = 0; iw < nw; iw++) {
      auto t = [&](int f) { return tab[(size_t)f * nw + iw]; };
      mx::LamIn li;
      li.chi = t(L_CHI);
      li.gff = t(L_GFF);
      li.chi1 = t(L_CHI1);
      li.wa3 = t(L_WA3);
      li.s = t(L_SCOEF);
      li.hmon = t(L_HMON);
      li.f1 = t(L_F1);
      li.f2 = t(L_F2);
      li.f3 = t(L_F3);
      for (int q = 0; q < 6; q++) li.gn[q] = t(L_GN1 + q);
      li.nu9 = t(L_NU9);
      li.l3nu = t(L_L3NU);
      li.hnuk = t(L_HNUK);
      li.wcm1 = t(L_WCM1);
      li.sw5 = t(L_SW5);
      float lr[mx::MLN];
      mx::lambda_record(li, lr);
      mx::Lam32 L;
      mx::lam32_from(L, [&](int f) { return lr[f]; });
      auto zat = [&](int z) { return &Z[(size_t)z * mx::MZN]; };
      const size_t item = (size_t)iw * ncol + c;
      mx::solve_item_host(zat, L, nz, dz, work.data(), dwork.data(), U + item * (nz + 6), K + item * nz,
                          V + item * nz);
    }
  }
}

// The 12-byte scratch record's packing of 1/kappa and u (pack_o1_u / unpack_o1_u) over n triples:
// fits[i], and the unpacked values' bits.
extern "C" void mixed_host_pack_roundtrip(const float *o1, const float *m, const int *e, int n, int *fits, float *o1r,
                                          float *mr, int *er) {
  for (int i = 0; i < n; i++) {
    int w1, w2;
    fits[i] = mx::pack_o1_u(o1[i], m[i], e[i], w1, w2) ? 1 : 0;
    mx::unpack_o1_u(w1, w2, o1r[i], mr[i], er[i]);
  }
}

// The extended exponents of the forward sweep's u over every item of the columns (after each
// item, solve_item_host leaves u's mantissas in work[nz, 2nz) and exponents in work[4nz, 5nz)):
// out[0] = min exponent, out[1] = max, out[2] = mantissas outside [1, 2).
extern "C" void mixed_host_u_exponents(const double *rho, const double *T, const double *wa, int ncol, int nz, int nw,
                                       double dz, double fully_ionized_T, int *out) {
  std::vector<double> tab((size_t)NL * nw);
  fill_lambda_table(wa, nw, tab.data());
  std::vector<float> Z((size_t)nz * mx::MZN), work((size_t)8 * nz);
  std::vector<double> dwork((size_t)nz + 6), U((size_t)nz + 6), K((size_t)nz), V((size_t)nz);
  int emin = 1 << 30, emax = -(1 << 30), bad = 0;
  for (int c = 0; c < ncol; c++) {
    for (int z = 0; z < nz; z++) mx::pillar(rho[(size_t)c * nz + z], T[(size_t)c * nz + z], fully_ionized_T, &Z[(size_t)z * mx::MZN]);
    for (int iw = 0; iw < nw; iw++) {
      auto t = [&](int f) { return tab[(size_t)f * nw + iw]; };
      mx::LamIn li;
      li.chi = t(L_CHI);
      li.gff = t(L_GFF);
      li.chi1 = t(L_CHI1);
      li.wa3 = t(L_WA3);
      li.s = t(L_SCOEF);
      li.hmon = t(L_HMON);
      li.f1 = t(L_F1);
      li.f2 = t(L_F2);
      li.f3 = t(L_F3);
      for (int q = 0; q < 6; q++) li.gn[q] = t(L_GN1 + q);
      li.nu9 = t(L_NU9);
      li.l3nu = t(L_L3NU);
      li.hnuk = t(L_HNUK);
      li.wcm1 = t(L_WCM1);
      li.sw5 = t(L_SW5);
      float lr[mx::MLN];
      mx::lambda_record(li, lr);
      mx::Lam32 L;
      mx::lam32_from(L, [&](int f) { return lr[f]; });
      auto zat = [&](int z) { return &Z[(size_t)z * mx::MZN]; };
      mx::solve_item_host(zat, L, nz, dz, work.data(), dwork.data(), U.data(), K.data(), V.data());
      const float *um = work.data() + nz;
      const int *ue = reinterpret_cast<const int *>(work.data() + 4 * nz);
      for (int j = 0; j < nz; j++) {
        emin = ue[j] < emin ? ue[j] : emin;
        emax = ue[j] > emax ? ue[j] : emax;
        if (!(um[j] >= 1.0f && um[j] < 2.0f)) bad++;
      }
    }
  }
  out[0] = emin;
  out[1] = emax;
  out[2] = bad;
}
