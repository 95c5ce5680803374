// ref_step.cpp -- batched CPU driver around the mam4xx reference headers.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref/libmam4ref.so). The reference
// headers are included read-only from the mam4xx source tree and compiled
// unchanged against the host shim in oracle/shim; this file only composes
// them into the microphysics step and exposes C entry points for tests and
// for the CPU baseline timing.
//
// Step composition per cell (the host-model sequence the GPU kernel
// replaces):
//   1. pack state_q[40] / qqcw[40] (E3SM tracer order, kg/kg and #/kg,
//      src/mam4xx/utils.hpp:222-259);
//   2. modal_aero_calcsize_sub (src/mam4xx/modal_aero_calcsize.hpp:750)
//      with CalcsizeData::initialize (:142);
//   3. modal_aero_water_uptake_dr (src/mam4xx/water_uptake.hpp:481) on the
//      same state_q and the calcsize dry diameters, as in
//      src/validation/aero_model/aero_model_calcsize_water_uptake_dr.cpp:
//      75-111;
//   4. the calcsize tendencies applied for one step, q = max(0, q+tend*dt),
//      to interstitial and cloud-borne aerosol entries (the update_mmr
//      branch of the same driver, :112-118);
//   5. mmr -> vmr with the chemistry mechanism molecular weights
//      (src/mam4xx/gas_chem_mechanism.hpp:31-38; numbers x 28.966 kg/kmol);
//   6. modal_aero_amicphys_intr (src/mam4xx/mam4_amicphys.hpp:2120) with
//      q_pregaschem = q_precldchem = qq and qqcw_precldchem = qqcw;
//   7. vmr -> mmr and tendency = (after - before)/dt.

#include <mam4xx/calcsize.hpp>
#include <mam4xx/aero_rad_props.hpp>
#include <mam4xx/coagulation.hpp>
#include <mam4xx/gas_phase_chemistry.hpp>
#include <mam4xx/mam4_amicphys.hpp>
#include <mam4xx/modal_aero_calcsize.hpp>
#include <mam4xx/mo_setsox.hpp>
#include <mam4xx/ndrop.hpp>
#include <mam4xx/modal_aero_opt.hpp>
#include <mam4xx/water_uptake.hpp>

#include "../oracle_api.h"

#include <cstring>
#include <vector>
#include <omp.h>

namespace {

using mam4::Real;
using CalcsizeData = mam4::modal_aero_calcsize::CalcsizeData;

const CalcsizeData &calcsize_data() {
  static const CalcsizeData d = [] {
    CalcsizeData x;
    x.initialize();
    return x;
  }();
  return d;
}

constexpr double kMwDryAir = 28.966; // kg/kmol

bool is_number_slot(int i31) {
  return i31 == 13 || i31 == 18 || i31 == 26 || i31 == 30;
}
double to_vmr_factor(int i31) {
  return is_number_slot(i31)
             ? kMwDryAir
             : kMwDryAir / mam4::gas_chemistry::adv_mass[i31];
}
double to_mmr_factor(int i31) {
  return is_number_slot(i31)
             ? 1.0 / kMwDryAir
             : mam4::gas_chemistry::adv_mass[i31] / kMwDryAir;
}

mam4::microphysics::AmicPhysConfig amicphys_config(const mam4b_config &c) {
  mam4::microphysics::AmicPhysConfig a;
  a.do_cond = c.do_cond != 0;
  a.do_rename = c.do_rename != 0;
  a.do_newnuc = c.do_newnuc != 0;
  a.do_coag = c.do_coag != 0;
  a.gaexch_h2so4_uptake_optaa = c.gaexch_h2so4_uptake_optaa;
  a.newnuc_h2so4_conc_optaa = c.newnuc_h2so4_conc_optaa;
  return a;
}

void calcsize_cell(const Real (&state_q)[40], const Real (&qqcw)[40], Real dt,
                   Real (&dgncur_a)[4], Real (&dgncur_c)[4], Real (&ptend)[40],
                   Real (&dqqcwdt)[40]) {
  for (int i = 0; i < 40; ++i) {
    ptend[i] = 0;
    dqqcwdt[i] = 0;
  }
  Real sq[40], cw[40];
  std::memcpy(sq, state_q, sizeof(sq));
  std::memcpy(cw, qqcw, sizeof(cw));
  mam4::modal_aero_calcsize::modal_aero_calcsize_sub(
      sq, cw, dt, calcsize_data(), dgncur_a, dgncur_c, ptend, dqqcwdt);
}

void water_uptake_cell(const Real (&state_q)[40], Real temp, Real pmid,
                       Real cld, const Real (&dgncur_a)[4],
                       Real (&dgncur_awet)[4], Real (&qaerwat)[4],
                       Real (&wetdens)[4]) {
  const CalcsizeData &cd = calcsize_data();
  Real sq[40];
  std::memcpy(sq, state_q, sizeof(sq));
  Real dgn[4];
  std::memcpy(dgn, dgncur_a, sizeof(dgn));
  mam4::water_uptake::modal_aero_water_uptake_dr(
      cd.nspec_amode, cd.specdens_amode, cd.spechygro, cd.lspectype_amode, sq,
      temp, pmid, cld, dgn, dgncur_awet, qaerwat, wetdens);
}

void amicphys_cell(const mam4b_config &cfg, Real dt, Real temp, Real pmid,
                   Real zm, Real pblh, Real qv, Real cld, Real (&qq)[31],
                   Real (&qqcw)[31], const Real (&dgncur_a)[4],
                   const Real (&dgncur_awet)[4], const Real (&wetdens)[4],
                   Real *diag /* [5][31] or null */) {
  using View2D = mam4::microphysics::View2D;
  View2D d[5];
  if (diag) {
    for (int p = 0; p < 5; ++p)
      d[p] = View2D("gas_aero_exchange", 31, 1);
  }
  Real q_pregaschem[31], q_precldchem[31], qqcw_precldchem[31];
  std::memcpy(q_pregaschem, qq, sizeof(q_pregaschem));
  std::memcpy(q_precldchem, qq, sizeof(q_precldchem));
  std::memcpy(qqcw_precldchem, qqcw, sizeof(qqcw_precldchem));
  const Real pdel_unused = 0.0; // passed through, never read by amicphys
  mam4::microphysics::modal_aero_amicphys_intr(
      amicphys_config(cfg), dt, cfg.n_so4_monolayers_pcage, temp, pmid,
      pdel_unused, zm, pblh, qv, cld, qq, qqcw, 0, d[0], d[1], d[2], d[3], d[4],
      q_pregaschem, q_precldchem, qqcw_precldchem, dgncur_a, dgncur_awet,
      wetdens);
  if (diag) {
    for (int p = 0; p < 5; ++p)
      for (int i = 0; i < 31; ++i)
        diag[p * 31 + i] = d[p](i, 0);
  }
}

void step_cell(const double *in, size_t ld, size_t c, double pblh, double *out,
               size_t ldo, double *diag, size_t ldd, double dt,
               const mam4b_config &cfg) {
  auto IN = [&](int f) { return in[(size_t)f * ld + c]; };
  Real state_q[40] = {}, qqcw[40] = {};
  state_q[0] = IN(MAM4B_IN_QV);
  state_q[11] = IN(MAM4B_IN_H2SO4);
  state_q[14] = IN(MAM4B_IN_SOAG);
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    state_q[15 + p] = IN(MAM4B_IN_AER_I + p);
    qqcw[15 + p] = IN(MAM4B_IN_AER_C + p);
  }
  const Real temp = IN(MAM4B_IN_T), pmid = IN(MAM4B_IN_P);
  const Real cld = IN(MAM4B_IN_CLD);

  Real dgncur_a[4], dgncur_c[4], ptend[40], dqqcwdt[40];
  calcsize_cell(state_q, qqcw, dt, dgncur_a, dgncur_c, ptend, dqqcwdt);

  Real dgncur_awet[4], qaerwat[4], wetdens[4];
  water_uptake_cell(state_q, temp, pmid, cld, dgncur_a, dgncur_awet, qaerwat,
                    wetdens);

  for (int i = 15; i < 40; ++i) {
    state_q[i] = mam4::max(0.0, state_q[i] + ptend[i] * dt);
    qqcw[i] = mam4::max(0.0, qqcw[i] + dqqcwdt[i] * dt);
  }

  Real qq[31], qqcw31[31];
  for (int i = 0; i < 31; ++i) {
    qq[i] = state_q[9 + i] * to_vmr_factor(i);
    qqcw31[i] = qqcw[9 + i] * to_vmr_factor(i);
  }

  Real dg[5 * 31];
  amicphys_cell(cfg, dt, temp, pmid, IN(MAM4B_IN_ZM), pblh, IN(MAM4B_IN_QV),
                cld, qq, qqcw31, dgncur_a, dgncur_awet, wetdens,
                diag ? dg : nullptr);

  auto OUT = [&](int f) -> double & { return out[(size_t)f * ldo + c]; };
  OUT(MAM4B_OUT_TEND + 0) = (qq[2] * to_mmr_factor(2) - IN(MAM4B_IN_H2SO4)) / dt;
  OUT(MAM4B_OUT_TEND + 1) = (qq[5] * to_mmr_factor(5) - IN(MAM4B_IN_SOAG)) / dt;
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    const int i31 = 6 + p;
    OUT(MAM4B_OUT_TEND + 2 + p) =
        (qq[i31] * to_mmr_factor(i31) - IN(MAM4B_IN_AER_I + p)) / dt;
    OUT(MAM4B_OUT_TEND + 27 + p) =
        (qqcw31[i31] * to_mmr_factor(i31) - IN(MAM4B_IN_AER_C + p)) / dt;
  }
  for (int m = 0; m < 4; ++m) {
    OUT(MAM4B_OUT_DGN_A + m) = dgncur_a[m];
    OUT(MAM4B_OUT_DGN_AWET + m) = dgncur_awet[m];
    OUT(MAM4B_OUT_WETDENS + m) = wetdens[m];
    OUT(MAM4B_OUT_QAERWAT + m) = qaerwat[m];
  }
  if (diag) {
    for (int k = 0; k < 5 * 31; ++k)
      diag[(size_t)k * ldd + c] = dg[k];
  }
}

// The step with chemistry ahead of amicphys (the GPU's mam4b_step_chem_slab):
// steps 1-4 of step_cell; the 31 tracers in vmr with O3, H2O2, SO2, DMS from
// chem_in; microphysics::gas_phase_chemistry; mo_setsox::setsox_single_level
// (loffset 9, the total air density = invariant 0); modal_aero_amicphys_intr
// with q_pregaschem = before gas chemistry, q_precldchem / qqcw_precldchem =
// before aqueous chemistry; vmr -> mmr and tendencies as step_cell, plus the
// four chemistry gases' tendencies in chem_out.
void step_chem_cell(const double *in, size_t ld, size_t c, double pblh,
                    const double *chem, double *out, double *chem_out, double dt,
                    const mam4b_config &cfg) {
  using namespace mam4::gas_chemistry;
  auto IN = [&](int f) { return in[(size_t)f * ld + c]; };
  auto CH = [&](int f) { return chem[(size_t)f * ld + c]; };
  Real state_q[40] = {}, qqcw[40] = {};
  state_q[0] = IN(MAM4B_IN_QV);
  state_q[11] = IN(MAM4B_IN_H2SO4);
  state_q[14] = IN(MAM4B_IN_SOAG);
  const int gas_slot[4] = {9, 10, 12, 13}; // O3, H2O2, SO2, DMS in state_q
  for (int g = 0; g < 4; ++g)
    state_q[gas_slot[g]] = CH(MAM4B_CHEM_IN_O3 + g);
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    state_q[15 + p] = IN(MAM4B_IN_AER_I + p);
    qqcw[15 + p] = IN(MAM4B_IN_AER_C + p);
  }
  const Real temp = IN(MAM4B_IN_T), pmid = IN(MAM4B_IN_P);
  const Real cld = IN(MAM4B_IN_CLD);

  Real dgncur_a[4], dgncur_c[4], ptend[40], dqqcwdt[40];
  calcsize_cell(state_q, qqcw, dt, dgncur_a, dgncur_c, ptend, dqqcwdt);
  Real dgncur_awet[4], qaerwat[4], wetdens[4];
  water_uptake_cell(state_q, temp, pmid, cld, dgncur_a, dgncur_awet, qaerwat, wetdens);
  for (int i = 15; i < 40; ++i) {
    state_q[i] = mam4::max(0.0, state_q[i] + ptend[i] * dt);
    qqcw[i] = mam4::max(0.0, qqcw[i] + dqqcwdt[i] * dt);
  }
  Real qq[31], qqcw31[31];
  for (int i = 0; i < 31; ++i) {
    qq[i] = state_q[9 + i] * to_vmr_factor(i);
    qqcw31[i] = qqcw[9 + i] * to_vmr_factor(i);
  }
  Real q_pregaschem[31];
  std::memcpy(q_pregaschem, qq, sizeof(qq));

  Real ph[mam4::mo_photo::phtcnt], ex[extcnt], iv[nfs], ht[gas_pcnst];
  ph[0] = CH(MAM4B_CHEM_IN_PHOTO);
  for (int k = 0; k < extcnt; ++k)
    ex[k] = CH(MAM4B_CHEM_IN_EXTFRC + k);
  for (int k = 0; k < nfs; ++k)
    iv[k] = CH(MAM4B_CHEM_IN_INV + k);
  for (int k = 0; k < gas_pcnst; ++k)
    ht[k] = CH(MAM4B_CHEM_IN_HET + k);
  mam4::microphysics::gas_phase_chemistry(temp, dt, ph, ex, iv, ht, qq);

  Real q_precldchem[31], qqcw_precldchem[31];
  std::memcpy(q_precldchem, qq, sizeof(qq));
  std::memcpy(qqcw_precldchem, qqcw31, sizeof(qqcw31));
  {
    const mam4::mo_setsox::Config scfg;
    Real d1[31], d2[31];
    mam4::mo_setsox::setsox_single_level(9, dt, pmid, 0.0, temp, 0.0, CH(MAM4B_CHEM_IN_LWC), cld,
                                         CH(MAM4B_CHEM_IN_CLDNUM), iv[0], scfg, d1, d2, qqcw31,
                                         qq);
  }
  {
    using View2D = mam4::microphysics::View2D;
    View2D d[5];
    mam4::microphysics::modal_aero_amicphys_intr(
        amicphys_config(cfg), dt, cfg.n_so4_monolayers_pcage, temp, pmid, 0.0,
        IN(MAM4B_IN_ZM), pblh, IN(MAM4B_IN_QV), cld, qq, qqcw31, 0, d[0], d[1], d[2], d[3],
        d[4], q_pregaschem, q_precldchem, qqcw_precldchem, dgncur_a, dgncur_awet, wetdens);
  }
  auto OUT = [&](int f) -> double & { return out[(size_t)f * ld + c]; };
  OUT(MAM4B_OUT_TEND + 0) = (qq[2] * to_mmr_factor(2) - IN(MAM4B_IN_H2SO4)) / dt;
  OUT(MAM4B_OUT_TEND + 1) = (qq[5] * to_mmr_factor(5) - IN(MAM4B_IN_SOAG)) / dt;
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    const int i31 = 6 + p;
    OUT(MAM4B_OUT_TEND + 2 + p) = (qq[i31] * to_mmr_factor(i31) - IN(MAM4B_IN_AER_I + p)) / dt;
    OUT(MAM4B_OUT_TEND + 27 + p) =
        (qqcw31[i31] * to_mmr_factor(i31) - IN(MAM4B_IN_AER_C + p)) / dt;
  }
  for (int m = 0; m < 4; ++m) {
    OUT(MAM4B_OUT_DGN_A + m) = dgncur_a[m];
    OUT(MAM4B_OUT_DGN_AWET + m) = dgncur_awet[m];
    OUT(MAM4B_OUT_WETDENS + m) = wetdens[m];
    OUT(MAM4B_OUT_QAERWAT + m) = qaerwat[m];
  }
  const int gas_i31[4] = {0, 1, 3, 4};
  for (int g = 0; g < 4; ++g)
    chem_out[(size_t)(MAM4B_CHEM_OUT_TEND + g) * ld + c] =
        (qq[gas_i31[g]] * to_mmr_factor(gas_i31[g]) - CH(MAM4B_CHEM_IN_O3 + g)) / dt;
}

} // namespace

extern "C" {

int mam4ref_step(int ncell, const double *in, size_t ld_in,
                 const double *pblh_cell, double *out, size_t ld_out,
                 double *diag, size_t ld_diag, double dt,
                 const mam4b_config *cfg, int nthreads) {
  if (ncell < 0 || !in || !pblh_cell || !out || !cfg || dt <= 0)
    return MAM4B_ERR_INVALID_ARGUMENT;
  (void)calcsize_data();
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
  for (int c = 0; c < ncell; ++c)
    step_cell(in, ld_in, (size_t)c, pblh_cell[c], out, ld_out, diag, ld_diag,
              dt, *cfg);
  return MAM4B_OK;
}

int mam4ref_step_chem(int ncell, const double *in, const double *pblh_cell,
                      const double *chem_in, double *out, double *chem_out, double dt,
                      const mam4b_config *cfg, int nthreads) {
  if (ncell < 0 || !in || !pblh_cell || !chem_in || !out || !chem_out || !cfg || dt <= 0)
    return MAM4B_ERR_INVALID_ARGUMENT;
  (void)calcsize_data();
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
  for (int c = 0; c < ncell; ++c)
    step_chem_cell(in, (size_t)ncell, (size_t)c, pblh_cell[c], chem_in, out, chem_out, dt, *cfg);
  return MAM4B_OK;
}

void mam4ref_calcsize(int ncell, const double *state_q, const double *qqcw,
                      double dt, double *dgncur_a, double *dgncur_c,
                      double *ptend, double *dqqcwdt) {
  for (int c = 0; c < ncell; ++c) {
    Real sq[40], cw[40];
    std::memcpy(sq, state_q + 40 * c, sizeof(sq));
    std::memcpy(cw, qqcw + 40 * c, sizeof(cw));
    Real a[4], b[4], pt[40], dq[40];
    calcsize_cell(sq, cw, dt, a, b, pt, dq);
    std::memcpy(dgncur_a + 4 * c, a, sizeof(a));
    std::memcpy(dgncur_c + 4 * c, b, sizeof(b));
    std::memcpy(ptend + 40 * c, pt, sizeof(pt));
    std::memcpy(dqqcwdt + 40 * c, dq, sizeof(dq));
  }
}

void mam4ref_water_uptake(int ncell, const double *state_q, const double *temp,
                          const double *pmid, const double *cld,
                          const double *dgncur_a, double *dgncur_awet,
                          double *qaerwat, double *wetdens) {
  for (int c = 0; c < ncell; ++c) {
    Real sq[40], dg[4], w[4], q[4], d[4];
    std::memcpy(sq, state_q + 40 * c, sizeof(sq));
    std::memcpy(dg, dgncur_a + 4 * c, sizeof(dg));
    water_uptake_cell(sq, temp[c], pmid[c], cld[c], dg, w, q, d);
    std::memcpy(dgncur_awet + 4 * c, w, sizeof(w));
    std::memcpy(qaerwat + 4 * c, q, sizeof(q));
    std::memcpy(wetdens + 4 * c, d, sizeof(d));
  }
}

void mam4ref_amicphys(int ncell, const mam4b_config *cfg, double dt,
                      const double *temp, const double *pmid, const double *zm,
                      const double *pblh, const double *qv, const double *cld,
                      double *qq, double *qqcw, const double *dgncur_a,
                      const double *dgncur_awet, const double *wetdens,
                      double *diag) {
  for (int c = 0; c < ncell; ++c) {
    Real q[31], cw[31], a[4], w[4], d[4];
    std::memcpy(q, qq + 31 * c, sizeof(q));
    std::memcpy(cw, qqcw + 31 * c, sizeof(cw));
    std::memcpy(a, dgncur_a + 4 * c, sizeof(a));
    std::memcpy(w, dgncur_awet + 4 * c, sizeof(w));
    std::memcpy(d, wetdens + 4 * c, sizeof(d));
    amicphys_cell(*cfg, dt, temp[c], pmid[c], zm[c], pblh[c], qv[c], cld[c], q,
                  cw, a, w, d, diag ? diag + 155 * c : nullptr);
    std::memcpy(qq + 31 * c, q, sizeof(q));
    std::memcpy(qqcw + 31 * c, cw, sizeof(cw));
  }
}

void mam4ref_h2so4_update(double dt, double qgas_netprod_otrproc,
                          const double *uptkaer, double *qgas_cur,
                          double *qgas_avg, double *qaer_cur) {
  mam4::gasaerexch::mam_gasaerexch_1subarea_1gas_nonvolatile(
      dt, qgas_netprod_otrproc, uptkaer, *qgas_cur, *qgas_avg, qaer_cur);
}

double mam4ref_bm0ij(int n1, int n2a, int n2n) {
  return mam4::coagulation::bm0ij_data(n1, n2a, n2n);
}
double mam4ref_bm3i(int n1, int n2a, int n2n) {
  return mam4::coagulation::bm3i_data(n1, n2a, n2n);
}

void mam4ref_aging(unsigned n_so4_monolayers_pcage, const double *dgn_a,
                   double *qnum_cur, double *qnum_del_cond,
                   double *qnum_del_coag, double *qaer_cur,
                   double *qaer_del_cond, double *qaer_del_coag,
                   double *qaer_del_coag_in) {
  mam4::aging::mam_pcarbon_aging_1subarea(
      n_so4_monolayers_pcage, dgn_a, qnum_cur, qnum_del_cond, qnum_del_coag,
      reinterpret_cast<Real(*)[4]>(qaer_cur),
      reinterpret_cast<Real(*)[4]>(qaer_del_cond),
      reinterpret_cast<Real(*)[4]>(qaer_del_coag),
      reinterpret_cast<Real(*)[1]>(qaer_del_coag_in));
}

// Per-process entries: the reference's CalcSize and Coagulation process
// classes run column by column (OpenMP over columns) on Prognostics / Diagnostics / Tendencies
// whose ColumnViews point into the caller's field-major arrays
// (cell = col * nlev + lev):
//   prog, tend  64 fields: n_mode_i[4], n_mode_c[4], q_aero_i[4][7],
//               q_aero_c[4][7] (tend is read and written)
//   dgn         8 fields: dry diameters interstitial [4], cloud-borne [4]
namespace {
constexpr int kProgFields = 64;

void bind_prog(mam4::Prognostics &p, double *base, size_t n, size_t c0, int nlev) {
  for (int m = 0; m < 4; ++m) {
    p.n_mode_i[m] = mam4::ColumnView(base + (size_t)m * n + c0, nlev);
    p.n_mode_c[m] = mam4::ColumnView(base + (size_t)(4 + m) * n + c0, nlev);
    for (int a = 0; a < 7; ++a) {
      p.q_aero_i[m][a] = mam4::ColumnView(base + (size_t)(8 + 7 * m + a) * n + c0, nlev);
      p.q_aero_c[m][a] = mam4::ColumnView(base + (size_t)(36 + 7 * m + a) * n + c0, nlev);
    }
  }
}

mam4::Atmosphere column_atmosphere(int nlev, const double *temp, const double *pmid,
                                   std::vector<double> &zeros) {
  zeros.assign((size_t)nlev + 1, 0.0);
  mam4::ConstColumnView z(zeros.data(), nlev);
  mam4::ConstColumnView t = temp ? mam4::ConstColumnView(temp, nlev) : z;
  mam4::ConstColumnView p = pmid ? mam4::ConstColumnView(pmid, nlev) : z;
  mam4::ConstColumnView zi(zeros.data(), nlev + 1);
  return mam4::Atmosphere(nlev, t, p, z, z, z, z, z, z, z, zi, z, z, 1000.0);
}
} // namespace

void mam4ref_calcsize_process(int ncol, int nlev, int do_aitacc_transfer, int do_adjust,
                              double dt, double *prog, double *tend, double *dgn) {
  const size_t n = (size_t)ncol * nlev;
  mam4::AeroConfig aero_config;
  mam4::CalcSize::Config cfg;
  cfg.do_aitacc_transfer = do_aitacc_transfer != 0;
  cfg.do_adjust = do_adjust != 0;
  mam4::CalcSize process;
  process.init(aero_config, cfg);
  const mam4::Surface sfc{};
#pragma omp parallel for schedule(dynamic, 16)
  for (int col = 0; col < ncol; ++col) {
    std::vector<double> zeros;
    const size_t c0 = (size_t)col * nlev;
    mam4::Prognostics progs(nlev);
    mam4::Tendencies tends(nlev);
    mam4::Diagnostics diags(nlev);
    bind_prog(progs, prog, n, c0, nlev);
    bind_prog(tends, tend, n, c0, nlev);
    for (int m = 0; m < 4; ++m) {
      diags.dry_geometric_mean_diameter_i[m] = mam4::ColumnView(dgn + (size_t)m * n + c0, nlev);
      diags.dry_geometric_mean_diameter_c[m] =
          mam4::ColumnView(dgn + (size_t)(4 + m) * n + c0, nlev);
    }
    const mam4::Atmosphere atm = column_atmosphere(nlev, nullptr, nullptr, zeros);
    mam4::ThreadTeam team;
    process.compute_tendencies(aero_config, team, 0.0, dt, atm, sfc, progs, diags, tends);
  }
}

// wet: 8 fields, wet density [4] then wet diameter [4]
void mam4ref_coag_process(int ncol, int nlev, double dt, const double *temp,
                          const double *pmid, double *wet, double *prog, double *tend) {
  const size_t n = (size_t)ncol * nlev;
  mam4::AeroConfig aero_config;
  mam4::Coagulation process;
  process.init(aero_config);
  const mam4::Surface sfc{};
#pragma omp parallel for schedule(dynamic, 16)
  for (int col = 0; col < ncol; ++col) {
    std::vector<double> zeros;
    const size_t c0 = (size_t)col * nlev;
    mam4::Prognostics progs(nlev);
    mam4::Tendencies tends(nlev);
    mam4::Diagnostics diags(nlev);
    bind_prog(progs, prog, n, c0, nlev);
    bind_prog(tends, tend, n, c0, nlev);
    for (int m = 0; m < 4; ++m) {
      diags.wet_density[m] = mam4::ColumnView(wet + (size_t)m * n + c0, nlev);
      diags.wet_geometric_mean_diameter_i[m] =
          mam4::ColumnView(wet + (size_t)(4 + m) * n + c0, nlev);
    }
    const mam4::Atmosphere atm = column_atmosphere(nlev, temp + c0, pmid + c0, zeros);
    mam4::ThreadTeam team;
    process.compute_tendencies(aero_config, team, 0.0, dt, atm, sfc, progs, diags, tends);
  }
}

// mo_setsox::setsox_single_level per cell with the host offset loffset = 9
// (31-tracer arrays); qin, qcw [31][ncell] in/out, dso4, dh2so4 [31][ncell]
// out. pdel and mbar are passed as zero: the routine does not use them.
void mam4ref_setsox(int ncell, double dt, const double *press, const double *temp,
                    const double *lwc, const double *cldfrc, const double *cldnum,
                    const double *xhnm, double *qin, double *qcw, double *dso4,
                    double *dh2so4) {
  const mam4::mo_setsox::Config cfg;
  const size_t n = (size_t)ncell;
#pragma omp parallel for schedule(dynamic, 256)
  for (int c = 0; c < ncell; ++c) {
    Real qi[31], qc[31], d1[31], d2[31];
    for (int k = 0; k < 31; ++k) {
      qi[k] = qin[k * n + c];
      qc[k] = qcw[k * n + c];
    }
    mam4::mo_setsox::setsox_single_level(9, dt, press[c], 0.0, temp[c], 0.0, lwc[c], cldfrc[c],
                                         cldnum[c], xhnm[c], cfg, d1, d2, qc, qi);
    for (int k = 0; k < 31; ++k) {
      qin[k * n + c] = qi[k];
      qcw[k * n + c] = qc[k];
      dso4[k * n + c] = d1[k];
      dh2so4[k * n + c] = d2[k];
    }
  }
}

// microphysics::gas_phase_chemistry per cell: photo [ncell], extfrc
// [9][ncell], inv [8][ncell], het [31][ncell]; qq [31][ncell] in/out.
void mam4ref_gas_chemistry(int ncell, double dt, const double *temp, const double *photo,
                           const double *extfrc, const double *inv, const double *het,
                           double *qq) {
  using namespace mam4::gas_chemistry;
  const size_t n = (size_t)ncell;
#pragma omp parallel for schedule(dynamic, 256)
  for (int c = 0; c < ncell; ++c) {
    Real ph[mam4::mo_photo::phtcnt], ex[extcnt], iv[nfs], ht[gas_pcnst], q[gas_pcnst];
    ph[0] = photo[c];
    for (int k = 0; k < extcnt; ++k)
      ex[k] = extfrc[k * n + c];
    for (int k = 0; k < nfs; ++k)
      iv[k] = inv[k * n + c];
    for (int k = 0; k < gas_pcnst; ++k) {
      ht[k] = het[k * n + c];
      q[k] = qq[k * n + c];
    }
    mam4::microphysics::gas_phase_chemistry(temp[c], dt, ph, ex, iv, ht, q);
    for (int k = 0; k < gas_pcnst; ++k)
      qq[k * n + c] = q[k];
  }
}

// ndrop::get_activate_frac per cell on the interstitial populations of a
// step input slab (field-major, ld = ncell), with the E3SM parameters of
// get_e3sm_parameters and the constants of ndrop_init; the mode number
// bounds are ndrop_init's volume-to-number ratios (at the maximum and the
// minimum diameter). out [17][ncell]: fn[4], fm[4], fluxn[4], fluxm[4],
// flux_fullact (zero where activate_modal returns early).
void mam4ref_activate(int ncell, const double *in, const double *rho, const double *w,
                      double *out) {
  using namespace mam4::ndrop;
  int nspec_amode[4], lspectype[maxd_aspectype][4], lmassptr[maxd_aspectype][4], numptr[4];
  Real specdens[maxd_aspectype], spechygro[maxd_aspectype];
  int mam_idx[4][nspec_max], mam_cnst_idx[4][nspec_max];
  get_e3sm_parameters(nspec_amode, lspectype, lmassptr, numptr, specdens, spechygro, mam_idx,
                      mam_cnst_idx);
  Real exp45logsig[4], alogsig[4], aten, v2n_min[4], v2n_max[4];
  ndrop_init(exp45logsig, alogsig, aten, v2n_min, v2n_max);
  const size_t n = (size_t)ncell;
#pragma omp parallel for schedule(dynamic, 256)
  for (int c = 0; c < ncell; ++c) {
    Real state_q[mam4::aero_model::pcnst] = {};
    for (int p = 0; p < 25; ++p)
      state_q[15 + p] = in[(size_t)(MAM4B_IN_AER_I + p) * n + c];
    Real fn[4] = {}, fm[4] = {}, fluxn[4] = {}, fluxm[4] = {}, flux_fullact = 0;
    get_activate_frac(state_q, rho[c], rho[c], w[c], in[(size_t)MAM4B_IN_T * n + c], lspectype,
                      specdens, spechygro, lmassptr, v2n_min, v2n_max, numptr, nspec_amode,
                      exp45logsig, alogsig, aten, fn, fm, fluxn, fluxm, flux_fullact);
    for (int m = 0; m < 4; ++m) {
      out[(size_t)m * n + c] = fn[m];
      out[(size_t)(4 + m) * n + c] = fm[m];
      out[(size_t)(8 + m) * n + c] = fluxn[m];
      out[(size_t)(12 + m) * n + c] = fluxm[m];
    }
    out[(size_t)16 * n + c] = flux_fullact;
  }
}

// modal_aero_opt::modal_aero_lw_k per cell on a step input slab
// (field-major, ld = ncell) with the given tables (layouts of
// mam4b_optics_lw_tables); tau [16][ncell].
void mam4ref_optics_lw(int ncell, const double *in, const double *pdeldry, double dt,
                       const double *specref, const double *water, const double *refr,
                       const double *refi, const double *absp, double *tau) {
  using namespace mam4::modal_aero_opt;
  AerosolOpticsDeviceData d;
  set_aerosol_optics_data_for_modal_aero_lw_views(d);
  set_complex_views_modal_aero(d);
  ComplexView2D::host_mirror_type host("specrefndx", nlwbands, mam4::ndrop::maxd_aspectype);
  for (int b = 0; b < nlwbands; ++b)
    for (int t = 0; t < mam4::ndrop::maxd_aspectype; ++t)
      host(b, t) = Kokkos::complex<Real>(specref[2 * (b * 14 + t)], specref[2 * (b * 14 + t) + 1]);
  set_device_specrefindex(d.specrefindex_lw, "long_wave", host);
  for (int b = 0; b < nlwbands; ++b)
    d.crefwlw(b) = Kokkos::complex<Real>(water[2 * b], water[2 * b + 1]);
  for (int m = 0; m < 4; ++m)
    for (int b = 0; b < nlwbands; ++b) {
      for (int i = 0; i < prefr; ++i)
        d.refrtablw[m][b](i) = refr[(m * nlwbands + b) * prefr + i];
      for (int j = 0; j < prefi; ++j)
        d.refitablw[m][b](j) = refi[(m * nlwbands + b) * prefi + j];
      for (int c = 0; c < ncoef; ++c)
        for (int i = 0; i < prefr; ++i)
          for (int j = 0; j < prefi; ++j)
            d.absplw[m][b](c, i, j) =
                absp[(((m * nlwbands + b) * ncoef + c) * prefr + i) * prefi + j];
    }
  const CalcsizeData &cd = calcsize_data();
  const size_t n = (size_t)ncell;
#pragma omp parallel for schedule(dynamic, 64)
  for (int c = 0; c < ncell; ++c) {
    auto IN = [&](int f) { return in[(size_t)f * n + c]; };
    Real state_q[40] = {}, qqcw[40] = {};
    state_q[0] = IN(MAM4B_IN_QV);
    state_q[11] = IN(MAM4B_IN_H2SO4);
    state_q[14] = IN(MAM4B_IN_SOAG);
    for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
      state_q[15 + p] = IN(MAM4B_IN_AER_I + p);
      qqcw[15 + p] = IN(MAM4B_IN_AER_C + p);
    }
    Real cld = IN(MAM4B_IN_CLD);
    Real t[nlwbands] = {};
    modal_aero_lw_k(pdeldry[c], IN(MAM4B_IN_P), IN(MAM4B_IN_T), cld, state_q, qqcw, dt, d, cd,
                    t);
    for (int b = 0; b < nlwbands; ++b)
      tau[(size_t)b * n + c] = t[b];
  }
}

// modal_aero_opt::modal_aero_sw_wo_diagnostics_k per cell, then the mode
// sums and the visible-band column sum of modal_aero_sw (same order:
// modes 0..3; levels top down, modes within each level). out [4][14][ncell]
// (tauxar, wa, ga, fa); aod [ncol].
void mam4ref_optics_sw(int ncol, int nlev, const double *in, const double *pdeldry, double dt,
                       const double *specref, const double *water, const double *refr,
                       const double *refi, const double *extp, const double *absp,
                       const double *asmp, double *out, double *aod) {
  using namespace mam4::modal_aero_opt;
  AerosolOpticsDeviceData d;
  set_aerosol_optics_data_for_modal_aero_sw_views(d);
  set_complex_views_modal_aero(d);
  ComplexView2D::host_mirror_type host("specrefndx", nswbands, mam4::ndrop::maxd_aspectype);
  for (int b = 0; b < nswbands; ++b)
    for (int t = 0; t < mam4::ndrop::maxd_aspectype; ++t)
      host(b, t) = Kokkos::complex<Real>(specref[2 * (b * 14 + t)], specref[2 * (b * 14 + t) + 1]);
  set_device_specrefindex(d.specrefindex_sw, "short_wave", host);
  for (int b = 0; b < nswbands; ++b)
    d.crefwsw(b) = Kokkos::complex<Real>(water[2 * b], water[2 * b + 1]);
  for (int m = 0; m < 4; ++m)
    for (int b = 0; b < nswbands; ++b) {
      for (int i = 0; i < prefr; ++i)
        d.refrtabsw[m][b](i) = refr[(m * nswbands + b) * prefr + i];
      for (int j = 0; j < prefi; ++j)
        d.refitabsw[m][b](j) = refi[(m * nswbands + b) * prefi + j];
      for (int c = 0; c < ncoef; ++c)
        for (int i = 0; i < prefr; ++i)
          for (int j = 0; j < prefi; ++j) {
            const size_t k = (((size_t)(m * nswbands + b) * ncoef + c) * prefr + i) * prefi + j;
            d.extpsw[m][b](c, i, j) = extp[k];
            d.abspsw[m][b](c, i, j) = absp[k];
            d.asmpsw[m][b](c, i, j) = asmp[k];
          }
    }
  const CalcsizeData &cd = calcsize_data();
  const size_t n = (size_t)ncol * nlev;
  std::vector<double> vis(n * 4);
#pragma omp parallel for schedule(dynamic, 64)
  for (long long cc = 0; cc < (long long)n; ++cc) {
    const size_t c = (size_t)cc;
    auto IN = [&](int f) { return in[(size_t)f * n + c]; };
    Real state_q[40] = {}, qqcw[40] = {};
    state_q[0] = IN(MAM4B_IN_QV);
    state_q[11] = IN(MAM4B_IN_H2SO4);
    state_q[14] = IN(MAM4B_IN_SOAG);
    for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
      state_q[15 + p] = IN(MAM4B_IN_AER_I + p);
      qqcw[15 + p] = IN(MAM4B_IN_AER_C + p);
    }
    Real cld = IN(MAM4B_IN_CLD);
    View2D t("t", 4, nswbands), wa("wa", 4, nswbands), ga("ga", 4, nswbands),
        fa("fa", 4, nswbands);
    modal_aero_sw_wo_diagnostics_k(pdeldry[c], IN(MAM4B_IN_P), IN(MAM4B_IN_T), cld, state_q,
                                   qqcw, dt, d, cd, t, wa, ga, fa);
    const View2D *q4[4] = {&t, &wa, &ga, &fa};
    for (int q = 0; q < 4; ++q)
      for (int b = 0; b < nswbands; ++b) {
        Real sum = 0;
        for (int m = 0; m < 4; ++m)
          sum += (*q4[q])(m, b);
        out[((size_t)q * nswbands + b) * n + c] = sum;
      }
    for (int m = 0; m < 4; ++m)
      vis[c * 4 + m] = t(m, idx_sw_diag);
  }
  for (int col = 0; col < ncol; ++col) {
    Real s = 0;
    for (int k = 0; k < nlev; ++k)
      for (int m = 0; m < 4; ++m)
        s += vis[((size_t)col * nlev + k) * 4 + m];
    aod[col] = s;
  }
}

// The part of aero_rad_props_sw / aero_rad_props_lw after the modal optics:
// tropopause_or_quit and the volcanic updates, column by column, on the
// modal results (mam4ref_optics_sw's out [4][14][n] or mam4ref_optics_lw's
// tau [16][n], updated in place) in the reference's own layouts
// (tau (band, 0:nlev); odap (band, nlev); sw extinction (band, nlev), sw
// albedo and asymmetry and lw extinction (nlev, band)). pint, zi: nlev+1
// per column; ext/ssa/af: [band][n]; trop: [ncol] out.
void mam4ref_rad_props_volcanic(int sw, int ncol, int nlev, const double *in, const double *pint,
                                const double *zi, const double *ext, const double *ssa,
                                const double *af, double *out, int *trop) {
  namespace arp = mam4::aero_rad_props;
  using View2D = arp::View2D;
  const size_t n = (size_t)ncol * nlev;
  const int nb = sw ? arp::nswbands : arp::nlwbands;
#pragma omp parallel for schedule(dynamic, 16)
  for (int col = 0; col < ncol; ++col) {
    const size_t c0 = (size_t)col * nlev, i0 = (size_t)col * (nlev + 1);
    mam4::ConstColumnView pmid(in + (size_t)MAM4B_IN_P * n + c0, nlev);
    mam4::ConstColumnView temp(in + (size_t)MAM4B_IN_T * n + c0, nlev);
    mam4::ConstColumnView zm(in + (size_t)MAM4B_IN_ZM * n + c0, nlev);
    mam4::ConstColumnView pi(pint + i0, nlev + 1), z(zi + i0, nlev + 1);
    const int lev = arp::tropopause_or_quit(pmid, pi, temp, zm, z);
    trop[col] = lev;
    mam4::ThreadTeam team;
    if (sw) {
      View2D q[4] = {View2D("tau", nb, nlev + 1), View2D("tau_w", nb, nlev + 1),
                     View2D("tau_w_g", nb, nlev + 1), View2D("tau_w_f", nb, nlev + 1)};
      View2D e("ext", nb, nlev), a("ssa", nlev, nb), g("af", nlev, nb);
      for (int b = 0; b < nb; ++b)
        for (int k = 0; k < nlev; ++k) {
          e(b, k) = ext[(size_t)b * n + c0 + k];
          a(k, b) = ssa[(size_t)b * n + c0 + k];
          g(k, b) = af[(size_t)b * n + c0 + k];
          for (int j = 0; j < 4; ++j)
            q[j](b, k + 1) = out[((size_t)j * nb + b) * n + c0 + k];
        }
      arp::volcanic_cmip_sw(team, z, lev, e, a, g, q[0], q[1], q[2], q[3]);
      for (int b = 0; b < nb; ++b)
        for (int k = 0; k < nlev; ++k)
          for (int j = 0; j < 4; ++j)
            out[((size_t)j * nb + b) * n + c0 + k] = q[j](b, k + 1);
    } else {
      View2D odap("odap", nb, nlev), e("ext", nlev, nb);
      for (int b = 0; b < nb; ++b)
        for (int k = 0; k < nlev; ++k) {
          odap(b, k) = out[(size_t)b * n + c0 + k];
          e(k, b) = ext[(size_t)b * n + c0 + k];
        }
      arp::compute_odap_volcanic_at_troplayer_lw(team, lev, z, e, odap);
      arp::compute_odap_volcanic_above_troplayer_lw(team, lev, z, e, odap);
      for (int b = 0; b < nb; ++b)
        for (int k = 0; k < nlev; ++k)
          out[(size_t)b * n + c0 + k] = odap(b, k);
    }
  }
}

// ndrop::dropmixnuc column by column (OpenMP over columns) on the step's
// input layout (in [NIN][n]), mix [4][n] (pdel, cldo, ncldwtr, wsub), pint
// and kvh (nlev + 1 per column); rpdel = 1 / pdel, factnum and every work
// array start at zero. out [66][n] in the layout of MAM4B_DROPMIX_OUT_*
// (populations in the step's order; the reference's qqcw_fld is in its own
// per-mode number-first order).
void mam4ref_dropmixnuc(int ncol, int nlev, int top_lev, int vertical_mix, double dt,
                        const double *in, const double *mix, const double *pint,
                        const double *kvh, double *out) {
  namespace nd = mam4::ndrop;
  using V1 = mam4::ColumnView;
  using V2 = nd::View2D;
  using V3 = nd::View3D;
  constexpr int nm = 4, np = MAM4B_NUM_POPS;
  const size_t n = (size_t)ncol * nlev;
  int nspec_amode[nd::maxd_aspectype] = {}, numptr_amode[nm];
  int lspectype_amode[nd::maxd_aspectype][nm], lmassptr_amode[nd::maxd_aspectype][nm];
  Real specdens_amode[nd::maxd_aspectype], spechygro[nd::maxd_aspectype];
  int mam_idx[nm][nd::nspec_max], mam_cnst_idx[nm][nd::nspec_max];
  nd::get_e3sm_parameters(nspec_amode, lspectype_amode, lmassptr_amode, numptr_amode,
                          specdens_amode, spechygro, mam_idx, mam_cnst_idx);
  Real exp45logsig[nm], alogsig[nm], aten, n2v_min[nm], n2v_max[nm];
  nd::ndrop_init(exp45logsig, alogsig, aten, n2v_min, n2v_max);
#pragma omp parallel for schedule(dynamic, 4)
  for (int col = 0; col < ncol; ++col) {
    const size_t c0 = (size_t)col * nlev, i0 = (size_t)col * (nlev + 1);
    auto colv = [&](const double *base) { return mam4::ConstColumnView(base + c0, nlev); };
    std::vector<double> rpdel_v(nlev), wsub_v(nlev), cldo_v(nlev);
    for (int k = 0; k < nlev; ++k) {
      rpdel_v[k] = 1.0 / mix[0 * n + c0 + k];
      cldo_v[k] = mix[1 * n + c0 + k];
      wsub_v[k] = mix[3 * n + c0 + k];
    }
    V2 sq("state_q", nlev, mam4::aero_model::pcnst);
    V2 qqcw("qqcw", nd::ncnst_tot, nlev);
    for (int k = 0; k < nlev; ++k)
      for (int p = 0; p < np; ++p)
        sq(k, 15 + p) = in[(size_t)(MAM4B_IN_AER_I + p) * n + c0 + k];
    for (int m = 0; m < nm; ++m)
      for (int l = 0; l <= nspec_amode[m]; ++l) {
        const int mm = mam_idx[m][l] - 1, q = mam_cnst_idx[m][l] - 1 - 15;
        for (int k = 0; k < nlev; ++k)
          qqcw(mm, k) = in[(size_t)(MAM4B_IN_AER_C + q) * n + c0 + k];
      }
    V1 qcld("qcld", nlev), wsub(wsub_v.data(), nlev), cldo(cldo_v.data(), nlev);
    V2 ptend("ptend", mam4::aero_model::pcnst, nlev), factnum("factnum", nm, nlev);
    V1 tendnd("tendnd", nlev), ndropcol("ndropcol", nlev), ndropmix("ndropmix", nlev),
        nsource("nsource", nlev), wtke("wtke", nlev);
    V2 ccn("ccn", nlev, nd::psat), coltend("coltend", nd::ncnst_tot, nlev),
        coltend_cw("coltend_cw", nd::ncnst_tot, nlev);
    V3 raercol_cw("raercol_cw", nlev, 2, nd::ncnst_tot), raercol("raercol", nlev, 2, nd::ncnst_tot);
    V2 nact("nact", nlev, nm), mact("mact", nlev, nm);
    V1 w[15];
    for (auto &v : w)
      v = V1("work", nlev);
    mam4::ThreadTeam team;
    nd::dropmixnuc(team, dt, colv(in + (size_t)MAM4B_IN_T * n), colv(in + (size_t)MAM4B_IN_P * n),
                   mam4::ConstColumnView(pint + i0, nlev + 1), colv(mix + 0 * n),
                   mam4::ConstColumnView(rpdel_v.data(), nlev), colv(in + (size_t)MAM4B_IN_ZM * n),
                   sq, colv(mix + 2 * n), mam4::ConstColumnView(kvh + i0, nlev + 1),
                   colv(in + (size_t)MAM4B_IN_CLD * n), lspectype_amode, specdens_amode, spechygro,
                   lmassptr_amode, n2v_min, n2v_max, numptr_amode, nspec_amode, exp45logsig,
                   alogsig, aten, mam_idx, mam_cnst_idx, vertical_mix != 0, qcld, wsub, cldo, qqcw,
                   ptend, tendnd, factnum, ndropcol, ndropmix, nsource, wtke, ccn, coltend,
                   coltend_cw, top_lev, raercol_cw, raercol, nact, mact, w[0], w[1], w[2], w[3],
                   w[4], w[5], w[6], w[7], w[8], w[9], w[10], w[11], w[12], w[13], w[14]);
    auto O = [&](int f, int k) -> double & { return out[(size_t)f * n + c0 + k]; };
    for (int k = 0; k < nlev; ++k) {
      O(MAM4B_DROPMIX_OUT_QCLD, k) = qcld(k);
      O(MAM4B_DROPMIX_OUT_TENDND, k) = tendnd(k);
      O(MAM4B_DROPMIX_OUT_NSOURCE, k) = nsource(k);
      O(MAM4B_DROPMIX_OUT_NDROPMIX, k) = ndropmix(k);
      O(MAM4B_DROPMIX_OUT_NDROPCOL, k) = ndropcol(k);
      O(MAM4B_DROPMIX_OUT_WTKE, k) = wtke(k);
      for (int m = 0; m < nm; ++m)
        O(MAM4B_DROPMIX_OUT_FACTNUM + m, k) = factnum(m, k);
      for (int l = 0; l < nd::psat; ++l)
        O(MAM4B_DROPMIX_OUT_CCN + l, k) = ccn(k, l);
      for (int p = 0; p < np; ++p)
        O(MAM4B_DROPMIX_OUT_PTEND + p, k) = ptend(15 + p, k);
      for (int m = 0; m < nm; ++m)
        for (int l = 0; l <= nspec_amode[m]; ++l) {
          const int mm = mam_idx[m][l] - 1, q = mam_cnst_idx[m][l] - 1 - 15;
          O(MAM4B_DROPMIX_OUT_QQCW + q, k) = qqcw(mm, k);
        }
    }
  }
}

double mam4ref_maxsat(double zeta, const double *eta, const double *smc) {
  Real e[4], sm[4], smax = 0;
  for (int m = 0; m < 4; ++m) {
    e[m] = eta[m];
    sm[m] = smc[m];
  }
  mam4::ndrop::maxsat(zeta, e, 4, sm, smax);
  return smax;
}

long mam4ref_assert_failures(void) { return mam4shim::assert_failures(); }

} // extern "C"
