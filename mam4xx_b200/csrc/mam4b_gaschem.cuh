// mam4b_gaschem.cuh -- gas-phase chemistry of a cell,
// mam4::microphysics::gas_phase_chemistry (src/mam4xx/gas_phase_chemistry.hpp:
// 40-117) for the mechanism of src/mam4xx/gas_chem_mechanism.hpp (31 tracers,
// 7 reactions, 30 implicit species): reaction rates, then the fully implicit
// Euler step of imp_sol (src/mam4xx/gas_chem.hpp:234-424) with its
// Newton-Raphson iteration (:73-231) and time-step control.
//
// The mechanism is linear in the tracers and nearly diagonal: implicit
// species k is tracer k+1, and only two off-diagonal couplings exist, SO2 ->
// H2SO4 (rate r3) and DMS -> SO2 (r4 + 0.5 r5 + r6). Every other species
// decays by its wet-removal rate and gains its external forcing. The system
// is therefore solved directly here -- a reciprocal per species and the two
// couplings by back substitution -- instead of through generic sparse
// matrix code. The rounding order of each sum and product is the
// reference's.
#pragma once

#include "mam4b_physics.cuh"

namespace mam4b {
namespace gch {

constexpr int kTracers = 31;   // gas_pcnst
constexpr int kImplicit = 30;  // clscnt4: implicit species k is tracer k + 1
constexpr int kExt = 9;        // extcnt
constexpr int kInv = 8;        // nfs
constexpr int kRxn = 7;        // rxntot
constexpr int kNewtonMax = 11; // itermax
constexpr int kStepsMax = 1000;
constexpr int kCutLimit = 5;
constexpr double kRelErr = 1.0e-3;
constexpr double kSmallForcing = 1.0e-40;

// external forcing feeding implicit species k (-1: none), indprd class 4
// (gas_chem_mechanism.hpp:101-140); species 0 (H2O2) gains r1 instead
MAM4B_HD constexpr int ext_of_species(int k) {
  return k == 2 ? 0 : k == 4 ? 8 : k == 5 ? 1 : k == 12 ? 5 : k == 13 ? 2 : k == 17 ? 6
       : k == 26 ? 3 : k == 27 ? 4 : k == 29 ? 7 : -1;
}

// Reaction rates of the 7 reactions (setrxt, usrrxt, adjrxt;
// gas_chem_mechanism.hpp:41-71, gas_chem.hpp:21-63): temperature and
// invariant densities inv [molecules/cm3] (0 total, 3 H2O, 4 OH, 5 NO3,
// 6 HO2), photolysis rate of H2O2 in r[0].
MAM4B_HD void reaction_rates(double temp, double photo, const double (&inv)[kInv],
                             double (&r)[kRxn]) {
  const double m = inv[0];
  r[2] = 2.9000000000e-12 * exp(-160.000000 / temp);
  r[4] = 9.6000000000e-12 * exp(-234.000000 / temp);
  r[6] = 1.9000000000e-13 * exp(520.000000 / temp);
  {  // HO2 + HO2 -> H2O2, enhanced by water vapour
    const double ko = 3.5e-13 * exp(430.0 / temp);
    const double kinf = 1.7e-33 * m * exp(1000. / temp);
    const double fc = 1.0 + 1.4e-21 * inv[3] * exp(2200. / temp);
    r[1] = (ko + kinf) * fc;
  }
  {  // DMS + OH -> 0.5 SO2
    const double ko = 1.0 + 5.5e-31 * exp(7460. / temp) * m * 0.21;
    r[5] = 1.7e-42 * exp(7810. / temp) * m * 0.21 / ko;
  }
  {  // SO2 + OH -> SO4, fall-off form
    const double fc = 3.0e-31 * pow(300. / temp, 3.3);
    const double ko = fc * m / (1.0 + fc * m / 1.5e-12);
    const double lg = log10(fc * m / 1.5e-12);
    r[3] = ko * pow(0.6, 1.0 / (1.0 + lg * lg));
  }
  r[2] *= inv[4];
  r[3] *= inv[4];
  r[4] *= inv[4];
  r[5] *= inv[4];
  r[6] *= inv[5];
  r[1] *= inv[6] * inv[6] / m;
  r[0] = photo;
}

// Coefficients of the linear system, fixed over the call.
struct System {
  double lin_diag[4];  // linmat diagonal of species 0-3 (others: -het)
  double loss[4];      // imp_prod_loss loss coefficients of species 0-3
  double c12, c23;     // couplings SO2 -> H2SO4, DMS -> SO2
};

template <class Het>
MAM4B_HD void make_system(const double (&r)[kRxn], const Het &het, System &s) {
  s.lin_diag[0] = -(+r[0] + r[2] + het(1));
  s.lin_diag[1] = -(+het(2));
  s.lin_diag[2] = -(+r[3] + het(3));
  s.lin_diag[3] = -(+r[4] + r[5] + r[6] + het(4));
  s.loss[0] = het(1) + r[0] + r[2];
  s.loss[1] = het(2);
  s.loss[2] = het(3) + r[3];
  s.loss[3] = het(4) + r[4] + r[5] + r[6];
  s.c12 = +r[3];
  s.c23 = +r[4] + 0.500000 * r[5] + r[6];
}

// One Newton-Raphson solve at step size 1/dti (newton_raphson_iter):
// y [tracers] is the iterate, inv_term = dti * y(step start) + independent
// production, het(t) the removal rate of tracer t. Returns whether every
// species met the relative tolerance (tested from the second iteration on).
// Species 4-29 are uncoupled and are finished one at a time, before species
// 0-3, which read only tracers 1-4: the same arithmetic as forming the whole
// residual first, without holding it.
template <class Het>
MAM4B_HD bool newton(const System &s, const Het &het, double dti,
                     const double (&inv_term)[kImplicit], double (&y)[kTracers]) {
  for (int it = 0; it < kNewtonMax; ++it) {
    bool all = true;
    auto finish = [&](int k, double f) {
      double v = y[k + 1] + f;
      if (v < 0.0)
        v = 0.0;
      y[k + 1] = v;
      if (fabs(f) > kSmallForcing && !(fabs(f) <= kRelErr * fabs(v)))
        all = false;
    };
#pragma unroll
    for (int k = kImplicit - 1; k >= 4; --k) {
      const double h = het(k + 1);
      double f = y[k + 1] * dti - (inv_term[k] - h * y[k + 1]);
      f *= 1.0 / (-(+h) - dti);
      finish(k, f);
    }
    double f[4];
    f[0] = y[1] * dti - (inv_term[0] - s.loss[0] * y[1]);
    f[1] = y[2] * dti - (inv_term[1] + s.c12 * y[3] - s.loss[1] * y[2]);
    f[2] = y[3] * dti - (inv_term[2] + s.c23 * y[4] - s.loss[2] * y[3]);
    f[3] = y[4] * dti - (inv_term[3] - s.loss[3] * y[4]);
    f[3] *= 1.0 / (s.lin_diag[3] - dti);
    f[2] -= s.c23 * f[3];
    f[2] *= 1.0 / (s.lin_diag[2] - dti);
    f[1] -= s.c12 * f[2];
    f[1] *= 1.0 / (s.lin_diag[1] - dti);
    f[0] *= 1.0 / (s.lin_diag[0] - dti);
#pragma unroll
    for (int k = 3; k >= 0; --k)
      finish(k, f[k]);
    if (it > 0 && all)
      return true;
  }
  return false;
}

// gas_phase_chemistry for one cell: qq [tracers, mol/mol] advanced over
// delt by the implicit Euler scheme with imp_sol's step control (halve the
// step after a failed Newton solve, the fifth time cut it to a tenth;
// double it after two converged steps; the interval counts the step as
// taken either way). extfrc [molecules/cm3/s], het(t) the removal rate of
// tracer t [1/s].
template <class Het>
MAM4B_HD void gas_chemistry_cell(double temp, double delt, double photo,
                                 const double (&extfrc)[kExt], const double (&inv)[kInv],
                                 const Het &het, double (&qq)[kTracers]) {
  double r[kRxn];
  reaction_rates(temp, photo, inv, r);
  System s;
  make_system(r, het, s);
  double ind[kImplicit];
#pragma unroll
  for (int k = 0; k < kImplicit; ++k) {
    const int e = ext_of_species(k);
    ind[k] = k == 0 ? +r[1] : (e >= 0 ? +(extfrc[e] / inv[0]) : 0.0);
  }
  double dt = delt, done = 0.0;
  int cuts = 0, good = 0;
  for (int step = 0; step < kStepsMax; ++step) {
    const double dti = 1.0 / dt;
    double inv_term[kImplicit];
#pragma unroll
    for (int k = 0; k < kImplicit; ++k)
      inv_term[k] = dti * qq[k + 1] + ind[k];
    const bool ok = newton(s, het, dti, inv_term, qq);
    if (!ok) {
      good = 0;
      if (cuts < kCutLimit) {
        ++cuts;
        dt *= cuts < kCutLimit ? 0.5 : 0.1;
      }
    }
    done += dt;
    if (fabs(delt - done) <= 0.0001)
      break;
    if (ok)
      ++good;
    if (good >= 2) {
      dt *= 2.0;
      good = 0;
    }
    dt = dmin(dt, delt - done);
  }
}

}  // namespace gch
}  // namespace mam4b
