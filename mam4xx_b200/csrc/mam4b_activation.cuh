// mam4b_activation.cuh -- aerosol activation of a cell, the per-cell part
// of the droplet-nucleation process (src/mam4xx/ndrop.hpp): the modes'
// number, volume and hygroscopicity from the interstitial mixing ratios
// (loadaer :244-331, get_aer_mmr_sum :116-155, get_aer_num :157-181), and
// the Abdul-Razzak & Ghan activated number and mass fractions for a given
// updraft (activate_modal :509-697 with maxsat :183-242), as
// get_activate_frac (:699-765) composes them. A consumer of the state the
// microphysics step produces.
#pragma once

#include "mam4b_physics.cuh"

namespace mam4b {
namespace act {

// species-type data of get_e3sm_parameters (ndrop.hpp:44-114): the type of
// species s of mode m (1-based) and each type's density and hygroscopicity
MAM4B_HD constexpr int spectype(int m, int s) {
  constexpr int t[4][7] = {{1, 4, 5, 6, 8, 7, 9}, {1, 5, 7, 9, 0, 0, 0},
                           {8, 7, 1, 6, 4, 5, 9}, {4, 6, 9, 0, 0, 0, 0}};
  return t[m][s];
}
MAM4B_HD constexpr double type_dens(int t) {
  constexpr double d[9] = {0.1770000000E+04, 0.0, 0.0, 0.1000000000E+04, 0.1000000000E+04,
                           0.1700000000E+04, 0.1900000000E+04, 0.2600000000E+04,
                           0.1601000000E+04};
  return d[t - 1];
}
MAM4B_HD constexpr double type_hygro(int t) {
  constexpr double h[9] = {0.5070000000E+00, 0.0, 0.0, 0.1000000083E-09, 0.1400000000E+00,
                           0.1000000013E-09, 0.1160000000E+01, 0.6800000000E-01,
                           0.1000000015E+00};
  return h[t - 1];
}

// mam4 physical constants (mam4_constants.hpp:33-123)
constexpr double kRGas = 6.022214076e23 * 1.380649e-23;  // J/K/mol
constexpr double kRAir = kRGas / 0.028966;
constexpr double kRH2o = kRGas / 0.018016;
constexpr double kLatvap = 2.501e6;
constexpr double kCpAir = 1.00464e3;
constexpr double kGravity = 9.80616;
constexpr double kRhoH2o = 1.0e3;
constexpr double kT0 = 273.0;
constexpr double kP0 = 1013.25e2;
constexpr double kSurften = 0.076;

// saturation vapour pressure with the water-ice transition below 0 C
// (wv_sat_svp_trans, wv_sat_methods.hpp:139-164) and the saturation
// specific humidity (ndrop::qsat, ndrop.hpp:450-471)
MAM4B_HD void qsat_trans(double t, double p, double &svp, double &qs) {
  const double ttrice = 20.0, tmelt = 273.15;
  double es = 0.0;
  if (t >= (tmelt - ttrice)) {
    const double tboil = 373.16, ten = 10, one = 1;
    es = pow(ten, -7.90298 * (tboil / t - one) + 5.02808 * log10(tboil / t) -
                      1.3816e-7 * (pow(ten, 11.344 * (one - t / tboil)) - one) +
                      8.1328e-3 * (pow(ten, -3.49149 * (tboil / t - one)) - one) +
                      log10(1013.246)) *
         ten * ten;
  }
  if (t < tmelt) {
    double weight = 1.0;
    const double h2otrip = 273.16, ten = 10, one = 1;
    const double esice = pow(ten, -9.09718 * (h2otrip / t - one) -
                                      3.56654 * log10(h2otrip / t) +
                                      0.876793 * (one - t / h2otrip) + log10(6.1071)) *
                         ten * ten;
    if ((tmelt - t) < ttrice)
      weight = (tmelt - t) / ttrice;
    es = weight * esice + (one - weight) * es;
  }
  const double epsilo = 0.018016 / 0.028966;
  const double omeps = 1.0 - epsilo;
  qs = ((p - es) <= 0.0) ? 1.0 : epsilo * es / (p - omeps * es);
  svp = dmin(es, p);
}

// maximum supersaturation of competing modes (maxsat, ndrop.hpp:183-242)
MAM4B_HD double max_supersat(double zeta, const double (&eta)[NMODE],
                             const double (&smc)[NMODE]) {
  const double small = 1e-20, mid = 1e5, big = 1.0 / small;
  double smax = 0.0;
  bool weak = true;
  for (int m = 0; m < NMODE; ++m) {
    if (zeta > mid * eta[m] || smc[m] * smc[m] > mid * eta[m]) {
      smax = small;
    } else {
      weak = false;
      break;
    }
  }
  if (weak)
    return smax;
  double sum = 0.0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    const double ls = log(K::sig(m));
    const double f1 = 0.5 * exp(2.5 * (ls * ls));
    const double f2 = 1.0 + 0.25 * log(K::sig(m));
    if (eta[m] > small) {
      const double g1 = (zeta / eta[m]) * sqrt(zeta / eta[m]);
      const double g2 = (smc[m] / sqrt(eta[m] + 3.0 * zeta)) *
                        sqrt(smc[m] / sqrt(eta[m] + 3.0 * zeta));
      sum += (f1 * g1 + f2 * g2) / (smc[m] * smc[m]);
    } else {
      sum = big;
    }
  }
  return 1.0 / sqrt(sum);
}

// One cell: ai the 25 interstitial populations (kg/kg, #/kg), air density
// [kg/m3] at the level the aerosol is loaded from and at the cell, updraft
// w [m/s], temperature. out: fn[4], fm[4], fluxn[4], fluxm[4],
// flux_fullact (all zero when there is no accumulation-mode aerosol or no
// updraft, the cases where activate_modal returns without writing; the
// return value is false then).
MAM4B_HD bool activate_cell(const StepConsts &C, const double (&ai)[NPOP], double rho_load,
                            double rho, double w, double tair, double (&out)[17]) {
#pragma unroll
  for (int k = 0; k < 17; ++k)
    out[k] = 0.0;
  // loadaer (phase 1, no cloud-borne part)
  double na[NMODE], vol[NMODE], hyg[NMODE];
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    double vs = 0.0, hs = 0.0;
#pragma unroll
    for (int s = 0; s < K::nspec(m); ++s) {
      const int t = spectype(m, s);
      const double v = dmax(ai[K::spec0(m) + s] + 0.0, 0.0) / type_dens(t);
      vs += v;
      hs += v * type_hygro(t);
    }
    if (vs > 1.0e-30) {
      hyg[m] = hs / vs;
      vol[m] = vs * rho_load;
    } else {
      hyg[m] = 0.0;
      vol[m] = 0.0;
    }
    const double nraw = (ai[K::numslot(m)] + 0.0) * rho_load;
    na[m] = bound(vol[m] * C.n2v_min[m], vol[m] * C.n2v_max[m], nraw);
  }
  // activate_modal with wmaxf = 10
  if (na[0] < 1.0e-20 || w <= 0.0)
    return false;
  const double wmaxf = 10.0;
  const double sq2 = sqrt(2.0);
  const double twothird = 2.0 / 3.0;
  const double aten = 2.0 * (0.018016 * 1e3) * kSurften / ((kRGas * 1e3) * kT0 * kRhoH2o);
  const double pres = kRAir * rho * tair;
  double svp, qs;
  qsat_trans(tair, pres, svp, qs);
  const double dqsdt = kLatvap / (kRH2o * tair * tair) * qs;
  const double alpha = kGravity * (kLatvap / (kCpAir * kRH2o * tair * tair) - 1.0 / (kRAir * tair));
  const double gamma = (1.0 + kLatvap / kCpAir * dqsdt) / (rho * qs);
  const double etafac2max = 1.0e10 / pow((alpha * wmaxf), 1.5);
  const double diff0 = 0.211e-4 * (kP0 / pres) * pow(tair / kT0, 1.94);
  const double conduct0 = (5.69 + 0.017 * (tair - kT0)) * 4.186e2 * 1.0e-5;
  const double gtherm = 1.0 / (kRhoH2o / (diff0 * rho * qs) +
                               kLatvap * kRhoH2o / (conduct0 * tair) *
                                   (kLatvap / (kRH2o * tair) - 1.0));
  const double beta = 2.0 * K::pi * kRhoH2o * gtherm * gamma;
  const double alw = alpha * w;
  const double etafac1 = alw * sqrt(alw);
  const double zeta = twothird * sqrt(alw) * aten / sqrt(gtherm);
  double smc[NMODE], lnsm[NMODE], eta[NMODE], alogsig[NMODE];
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    alogsig[m] = log(K::sig(m));
    const double exp45 = exp(4.5 * alogsig[m] * alogsig[m]);
    double ef2;
    if (vol[m] > 1.0e-39 && na[m] > 1.0e-39) {
      const double amcube = (3.0 / 4.0) * vol[m] / (K::pi * exp45 * na[m]);
      ef2 = 1.0 / (na[m] * beta * sqrt(gtherm));
      smc[m] = (hyg[m] > 1.0e-10) ? 2.0 * aten * sqrt(aten / (27.0 * hyg[m] * amcube)) : 100.0;
    } else {
      smc[m] = 1.0;
      ef2 = etafac2max;
    }
    lnsm[m] = log(smc[m]);
    eta[m] = etafac1 * ef2;
  }
  const double lnsmax = log(max_supersat(zeta, eta, smc));
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    const double an = twothird * (lnsm[m] - lnsmax) / (sq2 * alogsig[m]);
    out[m] = 0.5 * (1.0 - erf(an));
    const double am = an - 1.5 * sq2 * alogsig[m];
    out[4 + m] = 0.5 * (1.0 - erf(am));
    out[8 + m] = out[m] * w;
    out[12 + m] = out[4 + m] * w;
  }
  out[16] = w;
  return true;
}

}  // namespace act
}  // namespace mam4b
