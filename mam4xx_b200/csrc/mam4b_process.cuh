// mam4b_process.cuh -- two mam4xx AeroProcess implementations as batched
// per-cell device functions, for hosts that call processes one by one:
//
//   CalcSize::compute_tendencies     (src/mam4xx/calcsize.hpp:963-1220)
//   Coagulation::compute_tendencies  (src/mam4xx/coagulation.hpp:1198-1209,
//                                     coagulation_rates_1box :1121-1183)
//
// They work on Prognostics-style fields: one array per (mode, index), one
// entry per cell. The second index follows each reference process: CalcSize
// reads q_aero_*[mode][species of the mode] (aero_modes.hpp:214-243 order),
// Coagulation reads q_aero_i[mode][AeroId] for all seven AeroIds of every
// mode (coagulation.hpp:1144-1146) and writes them all back.
#pragma once

#include "mam4b_physics.cuh"

namespace mam4b {

// Prognostics / Tendencies fields (device pointers, [cell])
struct ProgFields {
  double *n_i[NMODE], *n_c[NMODE];
  double *q_i[NMODE][NAER], *q_c[NMODE][NAER];
};

struct CalcSizeArgs {
  ProgFields progs, tends;
  double *dgn_i[NMODE], *dgn_c[NMODE];
  long long ncell;
  double dt;
  int do_aitacc_transfer, do_adjust;
};

struct CoagProcessArgs {
  const double *temp, *pmid;
  const double *wet_density[NMODE], *dgn_awet[NMODE];
  ProgFields progs, tends;
  long long ncell;
  double dt;
  double *cc;  // [12][ncell]: the coefficients, from the pair stage to the update
};

// CalcSize::compute_tendencies for one cell (level k of a column):
// number adjustment of the modes it adjusts (tendency assigned), dry
// diameters of both phases, then the aitken <-> accumulation exchange
// (calcsize.hpp:595-829), whose number and species transfers are added to
// the tendencies in the reference's order.
MAM4B_HD void calcsize_process_cell(const StepConsts &C, const CalcSizeArgs &a, long long c) {
  const ProgFields &P = a.progs;
  const ProgFields &T = a.tends;
  const double adj_inv = safe_denominator(dmax(86400.0, a.dt));
  double dv_i[NMODE], dv_c[NMODE], num_i[NMODE], num_c[NMODE], dgi[NMODE], dgc[NMODE];
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    dgi[m] = K::dnom(m);
    dgc[m] = K::dnom(m);
    // compute_dry_volume_k (calcsize.hpp:28-45)
    double vi = 0.0, vc = 0.0;
#pragma unroll
    for (int s = 0; s < K::nspec(m); ++s) {
      vi += dmax(0.0, P.q_i[m][s][c]) * C.inv_density[m][s];
      vc += dmax(0.0, P.q_c[m][s][c]) * C.inv_density[m][s];
    }
    dv_i[m] = vi;
    dv_c[m] = vc;
    const double init_i = P.n_i[m][c], init_c = P.n_c[m][c];
    num_i[m] = init_i < 0 ? 0.0 : init_i;
    num_c[m] = init_c < 0 ? 0.0 : init_c;
    if (a.do_adjust && !(a.do_aitacc_transfer && m <= 1)) {
      double ti, tc;
      adjust_num_sizes(vi, vc, init_i, init_c, a.dt, C.n2v_min[m], C.n2v_max[m], adj_inv,
                       num_i[m], num_c[m], ti, tc);
      T.n_i[m][c] = ti;
      T.n_c[m][c] = tc;
    }
    diameter_from_num(vi, num_i[m], C.n2v_min[m], C.n2v_max[m], K::dmin(m), K::dmax(m),
                      C.log_sig[m], dgi[m]);
    diameter_from_num(vc, num_c[m], C.n2v_min[m], C.n2v_max[m], K::dmin(m), K::dmax(m),
                      C.log_sig[m], dgc[m]);
  }
  if (a.do_aitacc_transfer) {
    const double v2n_ait = C.n2v_nom[1], v2n_acc = C.n2v_nom[0];
    const double gm = C.geomean_ait_acc;
    double xt00 = 0, xt01 = 0, xt10 = 0, xt11 = 0, xv_ait2acc = 0, xv_acc2ait = 0;
    double noxf_i = 0.0, noxf_c = 0.0;
    bool ait2acc = false, acc2ait = false;
    {  // compute_coef_ait_acc_transfer (calcsize.hpp:314-376)
      const double drv_t = dv_i[1] + dv_c[1], num_t = num_i[1] + num_c[1];
      if (drv_t > 0.0 && num_t < drv_t * gm) {
        ait2acc = true;
        double fn, fv;
        if (num_t < drv_t * v2n_acc) {
          fn = 1.0;
          fv = 1.0;
        } else {
          fv = ((num_t / drv_t) - gm) / (v2n_acc - gm);
          fn = fv * (drv_t * v2n_acc / num_t);
          if (fn <= 0.0 || fv <= 0.0) {
            fn = 0.0;
            fv = 0.0;
          } else if (fn >= 1.0 || fv >= 1.0) {
            fn = 1.0;
            fv = 1.0;
          }
        }
        const double xn = fn * adj_inv;
        xv_ait2acc = fv * adj_inv;
        xt00 = num_i[1] * xn;
        xt01 = num_c[1] * xn;
      }
    }
    {  // compute_coef_acc_ait_transfer (calcsize.hpp:381-479): accumulation
       // species without an aitken counterpart (POM, BC, DST) stay
      double drv_t = dv_i[0] + dv_c[0], num_t = num_i[0] + num_c[0], num_t0 = 0.0;
      if (drv_t > 0.0 && num_t > drv_t * gm) {
        constexpr int noxf_s[3] = {1, 3, 4};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          noxf_i += dmax(0.0, P.q_i[0][noxf_s[k]][c]) * C.inv_density[0][noxf_s[k]];
          noxf_c += dmax(0.0, P.q_c[0][noxf_s[k]][c]) * C.inv_density[0][noxf_s[k]];
        }
        const double drv_noxf = noxf_i + noxf_c;
        const double num_noxf = drv_noxf * C.n2v_min[0];
        num_t0 = num_t;
        num_t = dmax(0.0, num_t - num_noxf);
        drv_t = dmax(0.0, drv_t - drv_noxf);
      }
      if (drv_t > 0.0 && num_t > drv_t * gm) {
        acc2ait = true;
        double fn, fv;
        if (num_t > drv_t * v2n_ait) {
          fn = 1.0;
          fv = 1.0;
        } else {
          fv = ((num_t / drv_t) - gm) / (v2n_ait - gm);
          fn = fv * (drv_t * v2n_ait / num_t);
          if (fn <= 0.0 || fv <= 0.0) {
            fn = 0.0;
            fv = 0.0;
          } else if (fn >= 1.0 || fv >= 1.0) {
            fn = 1.0;
            fv = 1.0;
          }
        }
        fn = fn * num_t * safe_denominator(num_t0);
        const double xn = fn * adj_inv;
        xv_acc2ait = fv * adj_inv;
        xt10 = num_i[0] * xn;
        xt11 = num_c[0] * xn;
      }
    }
    if (ait2acc || acc2ait) {
      const double ndi = (xt00 - xt10) * a.dt;
      const double ni_ait = dmax(0.0, num_i[1] - ndi), ni_acc = dmax(0.0, num_i[0] + ndi);
      const double vdi = (dv_i[1] * xv_ait2acc - (dv_i[0] - noxf_i) * xv_acc2ait) * a.dt;
      const double vi_ait = dmax(0.0, dv_i[1] - vdi), vi_acc = dmax(0.0, dv_i[0] + vdi);
      const double ndc = (xt01 - xt11) * a.dt;
      const double nc_ait = dmax(0.0, num_c[1] - ndc), nc_acc = dmax(0.0, num_c[0] + ndc);
      const double vdc = (dv_c[1] * xv_ait2acc - (dv_c[0] - noxf_c) * xv_acc2ait) * a.dt;
      const double vc_ait = dmax(0.0, dv_c[1] - vdc), vc_acc = dmax(0.0, dv_c[0] + vdc);
      dgi[1] = size_after_transfer(vi_ait, ni_ait, C.n2v_min[1], C.n2v_max[1], K::dmax(1),
                                   K::dmin(1), K::dnom(1), C.log_sig[1]);
      dgc[1] = size_after_transfer(vc_ait, nc_ait, C.n2v_min[1], C.n2v_max[1], K::dmax(1),
                                   K::dmin(1), K::dnom(1), C.log_sig[1]);
      dgi[0] = size_after_transfer(vi_acc, ni_acc, C.n2v_min[0], C.n2v_max[0], K::dmax(0),
                                   K::dmin(0), K::dnom(0), C.log_sig[0]);
      dgc[0] = size_after_transfer(vc_acc, nc_acc, C.n2v_min[0], C.n2v_max[0], K::dmax(0),
                                   K::dmin(0), K::dnom(0), C.log_sig[0]);
      // update_tends_flx (calcsize.hpp:529-590): common species of the two
      // modes, accumulation SO4 SOA NaCl MOM <-> aitken SO4 SOA NaCl MOM
      constexpr int acc_s[4] = {0, 2, 5, 6};
      constexpr int ait_s[4] = {0, 1, 2, 3};
      double tni_ait = T.n_i[1][c], tni_acc = T.n_i[0][c];
      double tnc_ait = T.n_c[1][c], tnc_acc = T.n_c[0][c];
      double tqi_ait[4], tqi_acc[4], tqc_ait[4], tqc_acc[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        tqi_ait[k] = T.q_i[1][ait_s[k]][c];
        tqi_acc[k] = T.q_i[0][acc_s[k]][c];
        tqc_ait[k] = T.q_c[1][ait_s[k]][c];
        tqc_acc[k] = T.q_c[0][acc_s[k]][c];
      }
      if (ait2acc) {
        tni_ait -= xt00;
        tni_acc += xt00;
        tnc_ait -= xt01;
        tnc_acc += xt01;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double xi = dmax(0.0, P.q_i[1][ait_s[k]][c]) * xv_ait2acc;
          tqi_ait[k] -= xi;
          tqi_acc[k] += xi;
          const double xc = dmax(0.0, P.q_c[1][ait_s[k]][c]) * xv_ait2acc;
          tqc_ait[k] -= xc;
          tqc_acc[k] += xc;
        }
      }
      if (acc2ait) {
        tni_acc -= xt10;
        tni_ait += xt10;
        tnc_acc -= xt11;
        tnc_ait += xt11;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double xi = dmax(0.0, P.q_i[0][acc_s[k]][c]) * xv_acc2ait;
          tqi_acc[k] -= xi;
          tqi_ait[k] += xi;
          const double xc = dmax(0.0, P.q_c[0][acc_s[k]][c]) * xv_acc2ait;
          tqc_acc[k] -= xc;
          tqc_ait[k] += xc;
        }
      }
      T.n_i[1][c] = tni_ait;
      T.n_i[0][c] = tni_acc;
      T.n_c[1][c] = tnc_ait;
      T.n_c[0][c] = tnc_acc;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        T.q_i[1][ait_s[k]][c] = tqi_ait[k];
        T.q_i[0][acc_s[k]][c] = tqi_acc[k];
        T.q_c[1][ait_s[k]][c] = tqc_ait[k];
        T.q_c[0][acc_s[k]][c] = tqc_acc[k];
      }
    }
  }
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    a.dgn_i[m][c] = dgi[m];
    a.dgn_c[m][c] = dgc[m];
  }
}

// coagulation_rates_1box (coagulation.hpp:1121-1183) for one cell: the air
// molar concentration is pmid / (r_gas T) with r_gas = N_A k_B per mole
// (mam4_constants.hpp:45), as that routine computes it; the wet density is
// used as given (no lower bound); tendencies += (after - before) / dt and
// the prognostics are updated in place.
constexpr double kRGasMole = 6.022214076e23 * 1.380649e-23;

MAM4B_HD double coag_process_aircon(const CoagProcessArgs &a, long long c) {
  return a.pmid[c] / (kRGasMole * a.temp[c]);
}

// The coefficients of mode pair p (coag_pair_coefs: bij0, bij3, bii0,
// bjj0, the pair's entries of coag_all_coefs) for one cell.
MAM4B_HD void coag_process_pair(const StepConsts &C, const CoagTables &Tb,
                                const CoagProcessArgs &a, long long c, int p, double &bij0,
                                double &bij3, double &bii0, double &bjj0) {
  const int sm = coag_src(p), dm = coag_dst(p);
  coag_pair_coefs(C, Tb, p, a.temp[c], a.pmid[c], coag_process_aircon(a, c), a.dgn_awet[sm][c],
                  a.dgn_awet[dm][c], a.wet_density[sm][c], a.wet_density[dm][c], bij0, bij3,
                  bii0, bjj0);
}

// The coagulation update of one cell with its 12 coefficients cc
// (coag_all_coefs order) and the tendencies.
MAM4B_HD void coag_process_update(const CoagProcessArgs &a, long long c,
                                  const double (&cc)[12]) {
  Sub s, s0;
  s.gas[0] = s.gas[1] = 0.0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    s.num[m] = a.progs.n_i[m][c];
#pragma unroll
    for (int x = 0; x < NAER; ++x)
      s.aer[x][m] = a.progs.q_i[m][x][c];
  }
  s0 = s;
  double coag_in[NAER];
  coagulation(a.dt, cc, s, coag_in);
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      a.tends.q_i[m][x][c] += (s.aer[x][m] - s0.aer[x][m]) / a.dt;
      a.progs.q_i[m][x][c] = s.aer[x][m];
    }
    a.tends.n_i[m][c] += (s.num[m] - s0.num[m]) / a.dt;
    a.progs.n_i[m][c] = s.num[m];
  }
}

// Both parts for one cell in one thread.
MAM4B_HD void coag_process_cell(const StepConsts &C, const CoagTables &Tb,
                                const CoagProcessArgs &a, long long c) {
  double cc[12];
#pragma unroll
  for (int p = 0; p < 3; ++p)
    coag_process_pair(C, Tb, a, c, p, cc[p], cc[3 + p], cc[6 + p], cc[9 + p]);
  coag_process_update(a, c, cc);
}

}  // namespace mam4b
