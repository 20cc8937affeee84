/*
 * oco_consts.h -- physical constants of the reference (source/common.f90:23-81,
 * source/continuous_opacity.f90:20-25 and :146) as compile-time doubles usable in host and
 * device code.
 *
 * The reference is compiled with -fdefault-real-8, so every literal is a double.  Values
 * that gfortran folds from constant expressions are given as exact hex literals:
 *   pi     = 4*atan(1d0)                         (common.f90:43)
 *   sqrt3  = sqrt(3d0), exp1 = exp(1d0)          (common.f90:45-46)
 *   log10e = log10(exp(1d0))                     (common.f90:67)
 *   Iev    = h*c*Rcm*6.2419d11 with Rcm = 2*pi**2*me*e**4/(h**3*c)   (common.f90:68-69),
 *            one rounding per operation, integer powers correctly rounded.
 *   log_overflow_limit = floor(log10(huge(1d0))) = 308  (common.f90:28)
 */
#ifndef OCO_CONSTS_H
#define OCO_CONSTS_H

namespace oco {
namespace k {
constexpr double sigma_sb = 5.6703744191844314e-05;
constexpr double log_overflow_limit = 308.0;
constexpr double mp = 1.67262192369e-24;
constexpr double mp1 = 1.0 / 1.67262192369e-24;
constexpr double h_planck = 6.62607015e-27;
constexpr double pi = 0x1.921fb54442d18p+1;
constexpr double pi1 = 1.0 / 0x1.921fb54442d18p+1;
constexpr double sqrt3 = 0x1.bb67ae8584caap+0;
constexpr double exp1 = 0x1.5bf0a8b145769p+1;
constexpr double k_cgs = 1.380649e-16;
constexpr double k_eV = 8.617333262145179e-05;
constexpr double k1_cgs = 1.0 / 1.380649e-16;
constexpr double k1_eV = 1.0 / 8.617333262145179e-05;
constexpr double hydrogen_ionization_eV = 13.6;
constexpr double c_light = 2.99792458e10;
constexpr double RydbergEnergy = 2.1798741e-11;
constexpr double RydbergEnergy1 = 1.0 / 2.1798741e-11;
constexpr double log10e = 0x1.bcb7b1526e50ep-2;
constexpr double Iev = 0x1.b369160866803p+3;
constexpr double Iev1 = 1.0 / 0x1.b369160866803p+3;
constexpr double bremsstrahlung_constant = 369234910.67735046;
constexpr double hcR1 = (6.62607015e-27 * 2.99792458e10) / 2.1798741e-11;
constexpr double one_third = 1.0 / 3.0;
constexpr double two_thirds = 2.0 / 3.0;
constexpr double switch_ionfraction = 1e-2;
constexpr double AHbf = 1.0449e-26;
constexpr double Rangstrom = 1.0968e-3;
constexpr double alpha0 = 1.0443e-26;
constexpr double alpha_e = 0.6648e-24;
constexpr double saha_const = 2414683039571967.0; /* gas_state.f90:57 */
constexpr double damping_factor_const = (h_planck * c_light) * k1_cgs;       /* c_o :73 */
constexpr double source_function_const = (2.0 * h_planck) * (c_light * c_light); /* c_o :74 */
}  // namespace k
}  // namespace oco

#endif
