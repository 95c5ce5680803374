// mam4b_setsox.cuh -- aqueous-phase sulfate chemistry of a cell,
// mam4::mo_setsox::setsox_single_level (src/mam4xx/mo_setsox.hpp:944-1254):
// the pH of cloud water from the electro-neutrality equation (bisection),
// S(IV) oxidation by H2O2 and by O3 over dt, and the uptake of H2SO4 gas by
// cloud droplets; the sulfate formed is given to the cloud-borne SO4 of the
// accumulation, aitken and coarse modes in proportion to their activated
// number. State: the 31 amicphys tracers (mol/mol, #/kmol) of the gas and
// interstitial phase (qin) and of the cloud-borne phase (qcw), the tracer
// offset of the reference's host (loffset = 9) already applied.
#pragma once

#include "mam4b_physics.cuh"

namespace mam4b {
namespace sox {

constexpr int kO3 = 0, kH2o2 = 1, kH2so4 = 2, kSo2 = 3;  // gas tracers
// cloud-borne SO4 of modes 1-3 and cloud-borne numbers of modes 1-4
MAM4B_HD constexpr int so4_cw(int m) { return m == 0 ? 6 : (m == 1 ? 14 : 21); }
MAM4B_HD constexpr int num_cw(int m) { return m == 0 ? 13 : (m == 1 ? 18 : (m == 2 ? 26 : 30)); }
constexpr double kSmallLwc = 1.0e-8;
constexpr double kP0 = 101300.0;
constexpr double kRa = 8314.0 / 101325.0;
constexpr double kXkw = 1.0e-14;
constexpr double kConst0 = 1.0e3 / 6.023e23;
constexpr double kCo2g = 330.0e-6;
constexpr int kItermax = 20;

// Henry's-law parameters at t_factor = 1/T - 1/298 (mo_setsox.hpp:140-200)
MAM4B_HD void henry_so2(double tf, double &xk, double &xe, double &x2) {
  xk = 1.230 * exp(3120.0 * tf);
  xe = 1.7e-2 * exp(2090.0 * tf);
  x2 = 6.0e-8 * exp(1120.0 * tf);
}
MAM4B_HD void henry_co2(double tf, double &xk, double &xe) {
  xk = 3.1e-2 * exp(2423.0 * tf);
  xe = 4.3e-7 * exp(-913.0 * tf);
}
MAM4B_HD void henry_h2o2(double tf, double &xk, double &xe) {
  xk = 7.4e4 * exp(6621.0 * tf);
  xe = 2.2e-12 * exp(-3730.0 * tf);
}
MAM4B_HD double henry_o3(double tf) { return 1.15e-2 * exp(2560.0 * tf); }

// net positive charge at pH yph (calc_ynetpos, mo_setsox.hpp:204-236)
MAM4B_HD double net_positive(double yph, double f1, double f2, double f3, double f4,
                             double eco2, double eh2o, double eso4, double so4_fact,
                             double &xph) {
  xph = pow(10.0, -yph);
  const double eso2 = f1 / (1.0 + f2 * (1.0 + (f3 / xph) * (1.0 + f4 / xph)));
  const double hso3 = eso2 / xph;
  const double so3 = hso3 * 2.0 * f4 / xph;
  const double hco3 = eco2 / xph;
  const double oh = eh2o / xph;
  const double so4 = so4_fact * eso4;
  const double neg = oh + hco3 + hso3 + so3 + so4;
  return xph - neg;
}

// H+ concentration of cloud water (calc_ph_values, mo_setsox.hpp:238-383):
// bisection on pH in [2, 7] until the bracket is 0.005 wide
MAM4B_HD double cloud_ph(double temp, double patm, double xlwc, double tf, double xso2,
                         double xso4, double xhnm, double so4_fact) {
  double xk, xe, x2;
  henry_so2(tf, xk, xe, x2);
  const double f1 = xk * xe * patm * xso2;
  const double f2 = xk * kRa * temp * xlwc;
  const double f3 = xe, f4 = x2;
  const double eh2o = kXkw;
  henry_co2(tf, xk, xe);
  const double eco2 = xk * xe * kCo2g * patm;
  const double eso4 = xso4 * xhnm * kConst0 / xlwc;
  double xph;
  double lo = 2.00, hi = lo, yph = lo;
  net_positive(yph, f1, f2, f3, f4, eco2, eh2o, eso4, so4_fact, xph);
  hi = 7.0;
  yph = hi;
  net_positive(yph, f1, f2, f3, f4, eco2, eh2o, eso4, so4_fact, xph);
  for (int i = 3; i < kItermax; ++i) {
    yph = 0.5 * (lo + hi);
    const double y = net_positive(yph, f1, f2, f3, f4, eco2, eh2o, eso4, so4_fact, xph);
    if (y >= 0.0)
      lo = yph;
    else
      hi = yph;
    if (fabs(hi - lo) <= 0.005) {
      yph = 0.5 * (hi + lo);
      return pow(10.0, -yph);
    }
  }
  return xph;
}

// droplet uptake rate of H2SO4 (cldaero_uptakerate, mo_setsox.hpp:583-667)
MAM4B_HD double droplet_uptake_rate(double xl, double cldnum, double cfact, double cldfrc,
                                    double tfld, double press) {
  constexpr double pi_x4 = 12.56637, one_third = 0.3333333, cm3_to_l = 1.0e-3;
  double num_cd = cm3_to_l * cldnum * cfact / cldfrc;
  num_cd = dmax(num_cd, 0.0);
  const double vol34pi = (xl * 0.75) / K::pi;
  double radxnum = pow(vol34pi * (num_cd * num_cd), one_third);
  double rad;
  if (radxnum <= vol34pi * 4.0e4) {
    radxnum = vol34pi * 4.0e4;
    rad = 50.0e-4;
  } else if (radxnum >= vol34pi * 4.0e8) {
    radxnum = vol34pi * 4.0e8;
    rad = 0.5e-4;
  } else {
    rad = radxnum / num_cd;
  }
  const double gasdiffus = 0.557 * pow(tfld, 1.75) / press;
  const double gasspeed = 1.455e4 * sqrt(tfld / 98.0);
  const double knudsen = 3.0 * gasdiffus / (gasspeed * rad);
  const double fs = (0.4875 * (1.0 + knudsen)) / (knudsen * (1.184 + knudsen) + 0.4875);
  return pi_x4 * radxnum * gasdiffus * fs;
}

// One cell. qin, qcw: the 31 tracers, updated; dso4 / dh2so4 receive the
// cloud-borne SO4 tendencies from aqueous oxidation and from H2SO4 uptake
// (dqdt_aqso4 / dqdt_aqh2so4 of the reference; zero elsewhere).
MAM4B_HD void setsox_cell(double dt, double press, double tfld, double lwc, double cldfrc,
                          double cldnum, double xhnm, double (&qin)[31], double (&qcw)[31],
                          double (&dso4)[3], double (&dh2so4)[3]) {
  const double cfact = xhnm * 1.0e6 * 1.38e-23 / 287.0 * 1.0e-3;
  // sox_cldaero_create_obj (mo_setsox.hpp:87-136)
  double xlwc = 0.0;
  if (cldfrc > 0.0) {
    xlwc = lwc * cfact;
    xlwc = xlwc / cldfrc;
  }
  const double so4c = qcw[so4_cw(0)] + qcw[so4_cw(1)] + qcw[so4_cw(2)];
  const double so4_fact = 1.0;
  double xso4 = 0.0, xph;
  double xso2 = qin[kSo2], xh2o2 = qin[kH2o2];
  const double xo3 = qin[kO3], xh2so4 = qin[kH2so4];
  if (xlwc >= kSmallLwc) {
    const double tf = (1.0 / tfld) - (1.0 / 298.0);
    const double patm = press / kP0;
    if (cldfrc > 0.0)
      xso4 = so4c / cldfrc;
    xph = cloud_ph(tfld, patm, xlwc, tf, xso2, xso4, xhnm, so4_fact);
  } else {
    xph = 1.0e-7;
  }
  const double tf = (1.0 / tfld) - (1.0 / 298.0);
  const double patm = press / kP0;
  double xk, xe, x2;
  henry_h2o2(tf, xk, xe);
  const double heh2o2 = xk * (1.0 + xe / xph);
  henry_so2(tf, xk, xe, x2);
  const double heso2 = xk * (1.0 + xe / xph * (1.0 + x2 / xph));
  const double heo3 = henry_o3(tf);
  double px = heh2o2 * kRa * tfld * xlwc;
  const double h2o2g = xh2o2 / (1.0 + px);
  px = heso2 * kRa * tfld * xlwc;
  const double so2g = xso2 / (1.0 + px);
  px = heo3 * kRa * tfld * xlwc;
  const double o3g = xo3 / (1.0 + px);
  const double rah2o2 = 8.e4 * exp(-3650.0 * tf) / (0.1 + xph);
  const double rao3 = 4.39e11 * exp(-4131.0 / tfld) + 2.56e3 * exp(-996.0 / tfld) / xph;
  // calc_sox_aqueous (mo_setsox.hpp:385-521)
  double xdelso4hp = 0.0, xso4_init = 0.0;
  if (xlwc >= kSmallLwc) {
    double pso4 = rah2o2 * 7.4e4 * exp(6621.0 * tf) * h2o2g * patm * 1.23 *
                  exp(3120.0 * tf) * so2g * patm;
    pso4 = pso4 * xlwc / kConst0 / xhnm;
    double ds = dmax(pso4 * dt, 1.0e-30);
    xso4_init = xso4;
    if ((ds <= xso2) && (ds <= xh2o2)) {
      xso4 = xso4 + ds;
      xh2o2 = xh2o2 - ds;
      xso2 = xso2 - ds;
    } else if (xh2o2 > xso2) {
      xso4 = xso4 + xso2;
      xh2o2 = xh2o2 - xso2;
      xso2 = 1.0e-20;
    } else {
      xso4 = xso4 + xh2o2;
      xso2 = xso2 - xh2o2;
      xh2o2 = 1.0e-20;
    }
    xdelso4hp = xso4 - xso4_init;
    pso4 = rao3 * heo3 * o3g * patm * heso2 * so2g * patm;
    pso4 = pso4 * xlwc / kConst0 / xhnm;
    ds = dmax(pso4 * dt, 1.0e-30);
    xso4_init = xso4;
    if (ds > xso2) {
      xso4 = xso4 + xso2;
      xso2 = 1.0e-20;
    } else {
      xso4 = xso4 + ds;
      xso2 = xso2 - ds;
    }
  }
  // sox_cldaero_update (mo_setsox.hpp:688-939)
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    dso4[m] = 0.0;
    dh2so4[m] = 0.0;
  }
  if ((cldfrc >= 1.0e-5) && (xlwc >= 1.0e-8)) {
    // compute_aer_factor (mo_setsox.hpp:523-581)
    double qn[4], fgain[4], sumf = 0.0;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      qn[m] = dmax(0.0, qcw[num_cw(m)]);
      if (m == 0)
        qn[m] = dmax(1.0e-10, qn[m]);
      fgain[m] = 0.0;
      if (m < 3) {
        fgain[m] = qn[m];
        sumf += fgain[m];
      }
    }
    if (sumf > 0.0) {
#pragma unroll
      for (int m = 0; m < 4; ++m)
        fgain[m] /= sumf;
    }
    double uptk = droplet_uptake_rate(xlwc, cldnum, cfact, cldfrc, tfld, press);
    uptk = (1.0 - exp(-1.0 * dmin(100.0, dt * uptk))) / dt;
    const double dso4dt_gasuptk = xh2so4 * uptk;
    const double delso4_o3rxn = xso4 - xso4_init;
    const double dso4dt_aqrxn = (delso4_o3rxn + xdelso4hp) / dt;
    const double dso4dt_hprxn = xdelso4hp / dt;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      dso4[m] = fgain[m] * dso4dt_aqrxn * cldfrc;
      dh2so4[m] = fgain[m] * dso4dt_gasuptk * cldfrc;
      const double dq = dso4[m] + dh2so4[m];
      qcw[so4_cw(m)] += (dq + 0.0) * dt;
    }
    qin[kH2so4] = qin[kH2so4] - dso4dt_gasuptk * dt * cldfrc;
    qin[kSo2] += (-dso4dt_aqrxn * cldfrc + 0.0) * dt;
    qin[kH2o2] += (-dso4dt_hprxn * cldfrc + 0.0) * dt;
  }
#pragma unroll
  for (int m = 0; m < 3; ++m)
    qcw[so4_cw(m)] = dmax(qcw[so4_cw(m)], 1.0e-20);
  qin[kSo2] = dmax(qin[kSo2], 1.0e-20);
}

}  // namespace sox
}  // namespace mam4b
