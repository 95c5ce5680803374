// mam4b_dropmix.cuh -- droplet activation and vertical mixing of a column,
// mam4::ndrop::dropmixnuc (src/mam4xx/ndrop.hpp:1393-1714): per level the
// activation of new and of growing cloud (update_from_newcld :954-1089,
// update_from_cldn_profile :767-952), then the explicit, sub-stepped
// vertical mixing of droplets and of interstitial and cloud-borne aerosol
// (update_from_explmix :1164-1391 with explmix :1090-1162), then the
// tendencies and the CCN at six supersaturations (ccncalc :333-448). The
// per-level pieces are here; the column kernel that orders them lives with
// the other kernels. Species are held in the population order of the
// step's inputs (E3SM state_q order: per mode its species, then its
// number); the reference's own order (per mode the number first) only
// permutes storage.
#pragma once

#include "mam4b_activation.cuh"

namespace mam4b {
namespace dmx {

constexpr int kPsat = 6;  // supersaturations of the CCN diagnostic

// population of species l of mode m in the reference's per-mode order:
// l = 0 the number, l >= 1 species l - 1
MAM4B_HD constexpr int pop_of(int m, int l) { return l == 0 ? K::numslot(m) : K::spec0(m) + l - 1; }
// mode of population p (its species, then its number, mode by mode)
MAM4B_HD constexpr int mode_of(int p) {
  return p <= K::numslot(0) ? 0 : p <= K::numslot(1) ? 1 : p <= K::numslot(2) ? 2 : 3;
}

// explmix (ndrop.hpp:1090-1110): droplet number and cloud-borne aerosol
MAM4B_HD double explmix(double qkm1, double qk, double qkp1, double src, double ekp, double ekm,
                        double ovp, double ovm, double dtmix) {
  const double q = qk + dtmix * (src + ekp * (ovp * qkp1 - qk) + ekm * (ovm * qkm1 - qk));
  return dmax(q, 0.0);
}

// explmix (ndrop.hpp:1111-1162): interstitial aerosol, which gains the
// cloud-borne aerosol of neighbouring levels where the cloud does not
// overlap
MAM4B_HD double explmix_act(double qkm1, double qk, double qkp1, double src, double ekp,
                            double ekm, double ovp, double ovm, double dtmix, double qact_km1,
                            double qact_kp1) {
  const double q = qk + dtmix * (-src + ekp * (qkp1 - qk + qact_kp1 * (1.0 - ovp)) +
                                 ekm * (qkm1 - qk + qact_km1 * (1.0 - ovm)));
  return dmax(q, 0.0);
}

// CCN number [#/cm3] at 0.02, 0.05, 0.1, 0.2, 0.5 and 1 % supersaturation
// from interstitial plus cloud-borne aerosol (ccncalc, with loadaer's
// phase 3). qcb_shift[m][s] is the cloud-borne mass the reference adds to
// species s of mode m: dropmixnuc fills its array one species up
// (qcldbrn[l][m] with l the 1-based species, loadaer reads qcldbrn[s][m]
// with s 0-based), so species s gets species s - 1's cloud-borne mass and
// the first species none; kept as the reference does it.
MAM4B_HD void ccn_cell(const StepConsts &C, const double (&ai)[NPOP],
                       const double (&qcb_shift)[NMODE][7], const double (&qcb_num)[NMODE],
                       double tair, double rho, double (&ccn)[kPsat]) {
  const double super[kPsat] = {0.0002, 0.0005, 0.001, 0.002, 0.005, 0.01};
  const double sq2 = sqrt(2.0);
  const double two_over_root27 = 2.0 / sqrt(27.0);
  const double surften_coef =
      2.0 * (0.018016 * 1e3) * act::kSurften / ((act::kRGas * 1e3) * act::kRhoH2o);
  const double aparam = surften_coef / tair;
  const double ssat_coeff = two_over_root27 * aparam * sqrt(aparam);
#pragma unroll
  for (int l = 0; l < kPsat; ++l)
    ccn[l] = 0.0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    double vs = 0.0, hs = 0.0;
#pragma unroll
    for (int s = 0; s < K::nspec(m); ++s) {
      const int t = act::spectype(m, s);
      const double v = dmax(ai[K::spec0(m) + s] + qcb_shift[m][s], 0.0) / act::type_dens(t);
      vs += v;
      hs += v * act::type_hygro(t);
    }
    double hyg, vol;
    if (vs > 1.0e-30) {
      hyg = hs / vs;
      vol = vs * rho;
    } else {
      hyg = 0.0;
      vol = 0.0;
    }
    const double na = bound(vol * C.n2v_min[m], vol * C.n2v_max[m], (ai[K::numslot(m)] + qcb_num[m]) * rho);
    const double alogsig = log(K::sig(m));
    const double exp45 = exp(4.5 * alogsig * alogsig);
    double ss_crit = 1;
    if (na > 1.0e-3) {
      const double amcube = (3.0 / 4.0) / (K::pi * exp45) * vol / na;
      ss_crit = ssat_coeff / sqrt(hyg * amcube);
    }
    const double argf = (2.0 / 3.0) / (sq2 * alogsig);
#pragma unroll
    for (int l = 0; l < kPsat; ++l) {
      const double arg = argf * log(ss_crit / super[l]);
      ccn[l] += na * 0.5 * (1.0 - erf(arg));
    }
  }
#pragma unroll
  for (int l = 0; l < kPsat; ++l)
    ccn[l] *= 1.0e-6;
}

}  // namespace dmx
}  // namespace mam4b
