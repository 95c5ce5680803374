// mam4b_physics.cuh -- per-cell device physics of the MAM4 microphysics step
// for sm_100a: calcsize, water uptake and the amicphys sequence
// (condensation, renaming, nucleation, coagulation, primary-carbon aging)
// over clear and cloudy subareas.
//
// Layout of the per-thread state. The reference keeps 31-entry tracer
// arrays per subarea and per time level (qsub1..4, qqcwsub2..4,
// src/mam4xx/mam4_amicphys.hpp:2256-2307); here a cell carries only what
// the step reads: the 2 condensing gases, 4 mode numbers and 21 species
// masses per phase, in amicphys units, held in registers through fully
// unrolled loops with compile-time indices.
//
// The arithmetic follows the reference routine cited at each function,
// including its order of operations and its quirks (listed where they
// occur), so FP64 results agree with the reference CPU build to rounding.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mam4b {

constexpr int NMODE = 4;
constexpr int NAER = 7;
constexpr int NPOP = 25;
constexpr int NQTEND = 4;

// ------------------------------------------------------------- constants
// Mode parameters (src/mam4xx/aero_modes.hpp:76-123): accumulation, aitken,
// coarse, primary carbon, and the tables of the step, as constexpr accessors
// that fold to immediates once the per-mode loops are unrolled.
#define MAM4B_HD __host__ __device__ __forceinline__
// read-only table load: through the non-coherent cache on the device
#ifdef __CUDA_ARCH__
#define MAM4B_LDG(p) __ldg(p)
#else
#define MAM4B_LDG(p) (*(p))
#endif
namespace K {
constexpr double pi = 3.14159265358979323846264;
constexpr double pi_sixth = 3.14159265358979323846264 / 6;
constexpr double eps = 2.220446049250313080847e-16;
constexpr double rh_cryst = 0.35, rh_deliq = 0.8;
constexpr double mw_dry_air = 28.966;
MAM4B_HD constexpr double dmin(int m) {
  constexpr double t[NMODE] = {5.35e-8, 8.7e-9, 1e-6, 1e-8};
  return t[m];
}
MAM4B_HD constexpr double dnom(int m) {
  constexpr double t[NMODE] = {1.1e-7, 2.6e-8, 2e-6, 5e-8};
  return t[m];
}
MAM4B_HD constexpr double dmax(int m) {
  constexpr double t[NMODE] = {4.4e-7, 5.2e-8, 4e-6, 1e-7};
  return t[m];
}
MAM4B_HD constexpr double sig(int m) {
  constexpr double t[NMODE] = {1.8, 1.6, 1.8, 1.60000002384186};
  return t[m];
}
MAM4B_HD constexpr int nspec(int m) {
  constexpr int t[NMODE] = {7, 4, 7, 3};
  return t[m];
}
// population slot (0..24) of the first species and of the number of each
// mode, E3SM state_q order (src/mam4xx/utils.hpp:222-259)
MAM4B_HD constexpr int spec0(int m) {
  constexpr int t[NMODE] = {0, 8, 13, 21};
  return t[m];
}
MAM4B_HD constexpr int numslot(int m) {
  constexpr int t[NMODE] = {7, 12, 20, 24};
  return t[m];
}
// AeroId of species s of mode m (aero_modes.hpp:214-243);
// SOA 0, SO4 1, POM 2, BC 3, NaCl 4, DST 5, MOM 6
MAM4B_HD constexpr int mode_spec(int m, int s) {
  constexpr int t[NMODE][7] = {{1, 2, 0, 3, 5, 4, 6},
                               {1, 0, 4, 6, -1, -1, -1},
                               {5, 4, 1, 3, 2, 0, 6},
                               {2, 3, 6, -1, -1, -1, -1}};
  return t[m][s];
}
// population slot holding AeroId a in mode m, -1 if absent
// (mam4_amicphys.hpp:111-118, lmap_aer minus 6)
MAM4B_HD constexpr int aer_slot(int a, int m) {
  constexpr int t[NAER][NMODE] = {{2, 9, 18, -1},  {0, 8, 15, -1}, {1, -1, 17, 21},
                                  {3, -1, 16, 22}, {5, 10, 14, -1}, {4, -1, 13, -1},
                                  {6, 11, 19, 23}};
  return t[a][m];
}
MAM4B_HD constexpr double aero_dens(int a) {
  constexpr double t[NAER] = {1000.0, 1770.0, 1000.0, 1700.0, 1900.0, 2600.0, 1601.0};
  return t[a];
}
// water-uptake species types (ndrop.hpp:59-80): density / hygroscopicity
// of the species of each of the 21 mass populations
MAM4B_HD constexpr double wu_dens(int w) {
  constexpr double t[21] = {1770.0, 1000.0, 1000.0, 1700.0, 2600.0, 1900.0, 1601.0,
                            1770.0, 1000.0, 1900.0, 1601.0,
                            2600.0, 1900.0, 1770.0, 1700.0, 1000.0, 1000.0, 1601.0,
                            1000.0, 1700.0, 1601.0};
  return t[w];
}
MAM4B_HD constexpr double wu_hygro(int w) {
  constexpr double t[21] = {
      0.5070000000E+00, 0.1000000083E-09, 0.1400000000E+00, 0.1000000013E-09,
      0.6800000000E-01, 0.1160000000E+01, 0.1000000015E+00,
      0.5070000000E+00, 0.1400000000E+00, 0.1160000000E+01, 0.1000000015E+00,
      0.6800000000E-01, 0.1160000000E+01, 0.5070000000E+00, 0.1000000013E-09,
      0.1000000083E-09, 0.1400000000E+00, 0.1000000015E+00,
      0.1000000083E-09, 0.1000000013E-09, 0.1000000015E+00};
  return t[w];
}
// amicphys unit factors (mam4_amicphys.hpp:121-153)
MAM4B_HD constexpr double fcvt_aer(int a) {
  constexpr double t[NAER] = {8.000000000000000E-002, 1, 8.000000000000000E-002, 1, 1, 1, 1};
  return t[a];
}
MAM4B_HD constexpr double mass_2_vol(int a) {
  constexpr double t[NAER] = {0.15,
                              6.4971751412429377e-002,
                              0.15,
                              7.0588235294117650e-003,
                              3.0789473684210526e-002,
                              5.1923076923076926e-002,
                              156.20986883198000};
  return t[a];
}
// chemistry-mechanism molecular weights of the 31 tracers
// (gas_chem_mechanism.hpp:31-38)
MAM4B_HD constexpr double adv_mass(int i) {
  constexpr double t[31] = {
      47.998200,     34.013600,  98.078400,     64.064800, 62.132400,
      12.011000,     115.107340, 12.011000,     12.011000, 12.011000,
      135.064039,    58.442468,  250092.672000, 1.007400,  115.107340,
      12.011000,     58.442468,  250092.672000, 1.007400,  135.064039,
      58.442468,     115.107340, 12.011000,     12.011000, 12.011000,
      250092.672000, 1.007400,   12.011000,     12.011000, 250092.672000,
      1.007400};
  return t[i];
}
}  // namespace K

// Runtime-derived constants computed once on the host (exactly the
// expressions the reference evaluates) and placed in constant memory.
struct StepConsts {
  double n2v_nom[NMODE], n2v_min[NMODE], n2v_max[NMODE];
  double inv_density[NMODE][7];
  double to_vmr[NPOP + 2];  // H2SO4, SOAG, then 25 populations
  double to_mmr[NPOP + 2];
  double fcvt_soag;         // 12.011/150
  double log_sig[NMODE];
  double rn_fac, rn_v2n_lo_rlx, rn_v2n_hi_rlx, rn_ln_tail_fac, rn_ln_cutoff, rn_threshold;
  double nuc_dplom, nuc_mass1p_lo, nuc_mass1p_hi;
  double so4_vol, soa_fac_eqvhyg, aging_fac_volsfc;
  double geomean_ait_acc;
  double hystfac;
  double kohler_aa;
};

// Device copies of the coagulation correction tables (Whitby/CMAQ data,
// src/mam4xx/coagulation.hpp:81-591), read through the L1 cache.
struct CoagTables {
  const double *bm0ij;  // [n1][n2a][n2n], 1000
  const double *bm3i;   // 1000
  const double *bm0;    // 10
};

MAM4B_HD double dmax(double a, double b) { return (a < b) ? b : a; }
MAM4B_HD double dmin(double a, double b) { return (b < a) ? b : a; }
MAM4B_HD double sq(double x) { return x * x; }
MAM4B_HD double cube(double x) { return x * x * x; }
MAM4B_HD double bound(double lo, double hi, double x) { return dmax(lo, dmin(hi, x)); }
MAM4B_HD double safe_denominator(double x) {
  return x / (x * x + K::eps * K::eps);
}
MAM4B_HD double diam_from_vol(double v, double log_sig) {
  // conversions.hpp:299-304
  return cbrt(v / K::pi_sixth) * exp(-1.5 * sq(log_sig));
}

// ================================================================ calcsize
// modal_aero_calcsize.hpp:750-932 with calcsize.hpp:56-310, 314-376, 481-515.
// ai/ac: 25 populations (mmr). Writes dgn_i and the calcsize tendencies of
// the populations (pt_i, pt_c, zero where calcsize leaves them).
MAM4B_HD void adjust_num_sizes(double drv_i, double drv_c, double init_i,
                                                 double init_c, double dt, double v2nmin,
                                                 double v2nmax, double adj_inv, double &num_i,
                                                 double &num_c, double &dqdt, double &dqqcwdt) {
  const double frac = dmax(0.0, dmin(1.0, dt * adj_inv));
  const double dtinv = safe_denominator(dt);
  const double minrl = v2nmin / 27.0, maxrl = v2nmax * 27.0;
  if (drv_i <= 0.0 && drv_c <= 0.0) {
    num_i = 0.0;
    num_c = 0.0;
  } else if (drv_c <= 0.0) {
    num_c = 0.0;
    const double nb = bound(drv_i * v2nmin, drv_i * v2nmax, num_i);
    num_i = num_i + (nb - num_i) * frac;
  } else if (drv_i <= 0.0) {
    const double nb = bound(drv_c * v2nmin, drv_c * v2nmax, num_c);
    num_c = num_c + (nb - num_c) * frac;
    num_i = 0.0;
  } else {
    const double ni1 = num_i, nc1 = num_c;
    double nb = bound(drv_i * minrl, drv_i * maxrl, ni1);
    const double dni2 = (nb - ni1) * frac;
    double ni2 = ni1 + dni2;
    nb = bound(drv_c * minrl, drv_c * maxrl, nc1);
    const double dnc2 = (nb - nc1) * frac;
    double nc2 = nc1 + dnc2;
    if (dni2 == 0.0 && dnc2 != 0.0)
      ni2 = bound(drv_i * minrl, drv_i * maxrl, ni1 - dnc2);
    else if (dni2 != 0.0 && dnc2 == 0.0)
      nc2 = bound(drv_c * minrl, drv_c * maxrl, nc1 - dni2);
    const double tdrv = drv_i + drv_c, tnum = ni2 + nc2;
    double dni3 = 0.0, dnc3 = 0.0;
    const double minb = tdrv * v2nmin, maxb = tdrv * v2nmax;
    if (tnum < minb) {
      const double d3 = (minb - tnum) * frac;
      if ((ni2 < drv_i * v2nmin) && (nc2 < drv_c * v2nmin)) {
        dni3 = d3 * (ni2 / tnum);
        dnc3 = d3 * (nc2 / tnum);
      } else if (nc2 < drv_c * v2nmin) {
        dnc3 = d3;
      } else if (ni2 < drv_i * v2nmin) {
        dni3 = d3;
      }
    } else if (tnum > maxb) {
      const double d3 = (maxb - tnum) * frac;
      if ((ni2 > drv_i * v2nmax) && (nc2 > drv_c * v2nmax)) {
        dni3 = d3 * (ni2 / tnum);
        dnc3 = d3 * (nc2 / tnum);
      } else if (nc2 > drv_c * v2nmax) {
        dnc3 = d3;
      } else if (ni2 > drv_i * v2nmax) {
        dni3 = d3;
      }
    }
    num_i = ni2 + dni3;
    num_c = nc2 + dnc3;
  }
  dqdt = (num_i - init_i) * dtinv;
  dqqcwdt = (num_c - init_c) * dtinv;
}

MAM4B_HD void diameter_from_num(double drv, double num, double v2nmin,
                                                  double v2nmax, double dgnmin, double dgnmax,
                                                  double log_sig, double &dgn) {
  // calcsize.hpp:56-78 (leaves dgn untouched when drv <= 0)
  if (!(drv > 0.0))
    return;
  if (num <= drv * v2nmin)
    dgn = dgnmax;
  else if (num >= drv * v2nmax)
    dgn = dgnmin;
  else
    dgn = diam_from_vol(1.0 / (num / drv), log_sig);
}

MAM4B_HD double size_after_transfer(double drv, double num, double v2n_hi,
                                                      double v2n_lo, double dgn_hi,
                                                      double dgn_lo, double dgn_nom,
                                                      double log_sig) {
  // calcsize.hpp:481-515
  if (drv > 0.0) {
    if (num <= drv * v2n_hi)
      return dgn_hi;
    if (num >= drv * v2n_lo)
      return dgn_lo;
    return diam_from_vol(1.0 / (num / drv), log_sig);
  }
  return dgn_nom;
}

MAM4B_HD void calcsize(const StepConsts &C, const double (&ai)[NPOP],
                                         const double (&ac)[NPOP], double dt,
                                         double (&dgn_i)[NMODE], double (&pt_i)[NPOP],
                                         double (&pt_c)[NPOP]) {
  const double adj_inv = safe_denominator(dmax(86400.0, dt));
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    pt_i[p] = 0.0;
    pt_c[p] = 0.0;
  }
  double dv_i_acc = 0, dv_c_acc = 0, dv_i_ait = 0, dv_c_ait = 0;
  double n_i_acc = 0, n_c_acc = 0, n_i_ait = 0, n_c_ait = 0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    dgn_i[m] = K::dnom(m);
    double dv_i = 0.0, dv_c = 0.0;
#pragma unroll
    for (int s = 0; s < K::nspec(m); ++s) {
      dv_i += dmax(0.0, ai[K::spec0(m) + s]) * C.inv_density[m][s];
      dv_c += dmax(0.0, ac[K::spec0(m) + s]) * C.inv_density[m][s];
    }
    const double init_i = ai[K::numslot(m)], init_c = ac[K::numslot(m)];
    double num_i = init_i < 0 ? 0.0 : init_i;
    double num_c = init_c < 0 ? 0.0 : init_c;
    if (m >= 2)
      adjust_num_sizes(dv_i, dv_c, init_i, init_c, dt, C.n2v_min[m], C.n2v_max[m], adj_inv,
                       num_i, num_c, pt_i[K::numslot(m)], pt_c[K::numslot(m)]);
    double v2nmin = C.n2v_min[m], v2nmax = C.n2v_max[m];
    if (m == 1)
      v2nmin /= 1.0e6;
    if (m == 0)
      v2nmax *= 1.0e6;
    diameter_from_num(dv_i, num_i, v2nmin, v2nmax, K::dmin(m), K::dmax(m), C.log_sig[m],
                      dgn_i[m]);
    if (m == 1) {
      dv_i_ait = dv_i;
      n_i_ait = num_i;
      dv_c_ait = dv_c;
      n_c_ait = num_c;
    } else if (m == 0) {
      dv_i_acc = dv_i;
      n_i_acc = num_i;
      dv_c_acc = dv_c;
      n_c_acc = num_c;
    }
  }
  // aitken <-> accumulation exchange (modal_aero_calcsize.hpp:499-747)
  const double v2n_ait = C.n2v_nom[1], v2n_acc = C.n2v_nom[0];
  const double gm = C.geomean_ait_acc;
  double xt00 = 0, xt01 = 0, xt10 = 0, xt11 = 0;
  bool ait2acc = false, acc2ait = false;
  double xv_ait2acc = 0, xv_acc2ait = 0, noxf_i = 0, noxf_c = 0;
  {
    const double drv_t = dv_i_ait + dv_c_ait, num_t = n_i_ait + n_c_ait;
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
      xt00 = n_i_ait * xn;
      xt01 = n_c_ait * xn;
    }
  }
  {
    double drv_t = dv_i_acc + dv_c_acc, num_t = n_i_acc + n_c_acc, num_t0 = 0.0;
    if (drv_t > 0.0 && num_t > drv_t * gm) {
      // accumulation species without an aitken counterpart: POM, BC, DST
      noxf_i = dmax(0.0, ai[1]) * C.inv_density[0][1];
      noxf_c = dmax(0.0, ac[1]) * C.inv_density[0][1];
      noxf_i += dmax(0.0, ai[3]) * C.inv_density[0][3];
      noxf_c += dmax(0.0, ac[3]) * C.inv_density[0][3];
      noxf_i += dmax(0.0, ai[4]) * C.inv_density[0][4];
      noxf_c += dmax(0.0, ac[4]) * C.inv_density[0][4];
      const double drv_noxf = noxf_i + noxf_c;
      const double num_noxf = drv_noxf * C.n2v_max[0];
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
      xt10 = n_i_acc * xn;
      xt11 = n_c_acc * xn;
    }
  }
  if (ait2acc || acc2ait) {
    const double ndi = (xt00 - xt10) * dt;
    const double num_i = dmax(0.0, n_i_ait - ndi);
    const double num_i_acc = dmax(0.0, n_i_acc + ndi);
    const double vdi = (dv_i_ait * xv_ait2acc - (dv_i_acc - noxf_i) * xv_acc2ait) * dt;
    const double drv_i = dmax(0.0, dv_i_ait - vdi);
    const double drv_i_acc = dmax(0.0, dv_i_acc + vdi);
    dgn_i[1] = size_after_transfer(drv_i, num_i, C.n2v_min[1], C.n2v_max[1], K::dmax(1),
                                   K::dmin(1), K::dnom(1), C.log_sig[1]);
    dgn_i[0] = size_after_transfer(drv_i_acc, num_i_acc, C.n2v_min[0], C.n2v_max[0], K::dmax(0),
                                   K::dmin(0), K::dnom(0), C.log_sig[0]);
    // common species slots: acc SO4 0, SOA 2, NaCl 5, MOM 6 <-> ait 8..11
    constexpr int acc_s[4] = {0, 2, 5, 6};
    constexpr int ait_s[4] = {8, 9, 10, 11};
    if (ait2acc) {
      pt_i[12] -= xt00;
      pt_i[7] += xt00;
      pt_c[12] -= xt01;
      pt_c[7] += xt01;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double xi = dmax(0.0, ai[ait_s[k]]) * xv_ait2acc;
        pt_i[ait_s[k]] -= xi;
        pt_i[acc_s[k]] += xi;
        const double xc = dmax(0.0, ac[ait_s[k]]) * xv_ait2acc;
        pt_c[ait_s[k]] -= xc;
        pt_c[acc_s[k]] += xc;
      }
    }
    if (acc2ait) {
      pt_i[7] -= xt10;
      pt_i[12] += xt10;
      pt_c[7] -= xt11;
      pt_c[12] += xt11;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double xi = dmax(0.0, ai[acc_s[k]]) * xv_acc2ait;
        pt_i[acc_s[k]] -= xi;
        pt_i[ait_s[k]] += xi;
        const double xc = dmax(0.0, ac[acc_s[k]]) * xv_acc2ait;
        pt_c[acc_s[k]] -= xc;
        pt_c[ait_s[k]] += xc;
      }
    }
  }
}

// ============================================================ water uptake
// water_uptake.hpp:73-480 and wv_sat_methods.hpp:14-131.
// Complex arithmetic follows Kokkos::complex (textbook product, quotient
// scaled by the divisor's 1-norm, abs = hypot, half-angle sqrt,
// pow = polar(pow(|z|,y), y*atan2)).
struct cplx {
  double re, im;
};
MAM4B_HD cplx cmk(double r, double i) { return cplx{r, i}; }
MAM4B_HD cplx cadd(cplx a, cplx b) { return cmk(a.re + b.re, a.im + b.im); }
MAM4B_HD cplx csub(cplx a, cplx b) { return cmk(a.re - b.re, a.im - b.im); }
MAM4B_HD cplx cneg(cplx a) { return cmk(-a.re, -a.im); }
MAM4B_HD cplx cmul(cplx a, cplx b) {
  return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
MAM4B_HD cplx cscale(double s, cplx a) { return cmk(s * a.re, s * a.im); }
MAM4B_HD cplx cdiv(cplx x, cplx y) {
  const double s = fabs(y.re) + fabs(y.im);
  if (s == 0.0)
    return cmk(x.re / s, x.im / s);
  const cplx xs = cmk(x.re / s, x.im / s);
  const cplx ycs = cmk(y.re / s, -y.im / s);
  const double yabs2 = ycs.re * ycs.re + ycs.im * ycs.im;
  const cplx r = cmul(xs, ycs);
  return cmk(r.re / yabs2, r.im / yabs2);
}
MAM4B_HD cplx csqrt_k(cplx x) {
  const double r = x.re, i = x.im;
  if (r == 0.0) {
    const double t = sqrt(fabs(i) / 2);
    return cmk(t, i < 0.0 ? -t : t);
  }
  const double t = sqrt(2 * (hypot(r, i) + fabs(r)));
  const double u = t / 2;
  return r > 0.0 ? cmk(u, i / t) : cmk(fabs(i) / t, i < 0.0 ? -u : u);
}
MAM4B_HD cplx cpow_k(cplx x, double y) {
  const double r = hypot(x.re, x.im);
  const double th = atan2(x.im, x.re);
  const double rho = pow(r, y), ang = y * th;
  return cmk(rho * cos(ang), rho * sin(ang));
}

// Smallest real root >= rdry of x^4 + p3 x^3 + p1 x + p0 (p2 = 0),
// makoh_quartic + find_real_solution (water_uptake.hpp:101-171).
MAM4B_HD double kohler_quartic_root(double rdry, double p3, double p1,
                                                      double p0) {
  const double p2 = 0.0;
  const double qq = -p2 * p2 / 36.0 + (p3 * p1 - 4.0 * p0) / 12.0;
  const double rr = -cube(p2 / 6.0) + p2 * (p3 * p1 - 4.0 * p0) / 48.0 +
                    (4.0 * p0 * p2 - p0 * p3 * p3 - p1 * p1) / 16.0;
  cplx crad = csqrt_k(cmk(rr * rr + qq * qq * qq, 0.0));
  cplx cb = csub(cmk(rr, 0.0), crad);
  cplx cx[4];
  if (cb.re == 0.0 && cb.im == 0.0) {
    const double r = cbrt(-p1);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      cx[i] = cmk(r, 0.0);
  } else {
    cb = cpow_k(cb, 1.0 / 3.0);
    const cplx cy = cadd(cadd(cneg(cb), cdiv(cmk(qq, 0.0), cb)), cmk(p2 / 6.0, 0.0));
    const cplx cb0 = csqrt_k(csub(cmul(cy, cy), cmk(p0, 0.0)));
    const cplx cb1 = cdiv(csub(cscale(p3, cy), cmk(p1, 0.0)), cscale(2.0, cb0));
    cb = cadd(cmk(p3 / 2.0, 0.0), cb1);
    crad = csqrt_k(csub(cmul(cb, cb), cscale(4.0, cadd(cy, cb0))));
    cx[0] = cmk((-cb.re + crad.re) / 2.0, (-cb.im + crad.im) / 2.0);
    cx[1] = cmk((-cb.re - crad.re) / 2.0, (-cb.im - crad.im) / 2.0);
    cb = csub(cmk(p3 / 2.0, 0.0), cb1);
    crad = csqrt_k(csub(cmul(cb, cb), cscale(4.0, csub(cy, cb0))));
    cx[2] = cmk((-cb.re + crad.re) / 2.0, (-cb.im + crad.im) / 2.0);
    cx[3] = cmk((-cb.re - crad.re) / 2.0, (-cb.im - crad.im) / 2.0);
  }
  const double eps = 1e-4;
  double rwet = 1000.0 * rdry;
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    const double xr = cx[n].re, xi = cx[n].im;
    if (fabs(xi) > fabs(xr) * eps)
      continue;
    if (xr > rwet)
      continue;
    if (xr < rdry * (1.0 - eps))
      continue;
    if (isnan(xr))
      continue;
    rwet = xr;
  }
  return rwet;
}

// modal_aero_kohler (water_uptake.hpp:180-230); rdry in m, returns m
MAM4B_HD double kohler(const StepConsts &C, double rdry_in, double hygro,
                                         double rh) {
  const double eps = 1e-4;
  const double aa = C.kohler_aa;
  const double rdry = rdry_in * 1.e6;
  const double vol = cube(rdry);
  const double bb = vol * hygro;
  const double ss = bound(1.e-10, 1.0 - eps, rh);
  const double slog = log(ss);
  const double p43 = -aa / slog;
  const double p41 = bb / slog - vol;
  const double p40 = aa * vol / slog;
  const double pp = fabs(-bb / aa) / (rdry * rdry);
  double rwet;
  if (pp < eps)
    rwet = rdry * (1.0 + pp * (1.0 / 3.0) / (1.0 - slog * rdry / aa));
  else
    rwet = kohler_quartic_root(rdry, p43, p41, p40);
  rwet = dmin(rwet, 30.0);
  return rwet * 1.e-6;
}

MAM4B_HD double qsat_water(double t, double p) {
  // GoffGratch_svp_water + wv_sat_svp_to_qsat (wv_sat_methods.hpp:14-46, 94-115)
  const double tboil = 373.16, ten = 10, one = 1;
  const double es = pow(ten, -7.90298 * (tboil / t - one) + 5.02808 * log10(tboil / t) -
                                 1.3816e-7 * (pow(ten, 11.344 * (one - t / tboil)) - one) +
                                 8.1328e-3 * (pow(ten, -3.49149 * (tboil / t - one)) - one) +
                                 log10(1013.246)) *
                    ten * ten;
  const double epsilo = 0.018016 / 0.028966;
  const double omeps = 1 - epsilo;
  if ((p - es) <= 0)
    return 1;
  return epsilo * es / (p - omeps * es);
}

// modal_aero_water_uptake_dr with wet density (water_uptake.hpp:362-480);
// uses the state before the calcsize update, like the reference driver.
// Relative humidity of the clear part of the cell:
MAM4B_HD double water_uptake_rh(double qv, double temp, double pmid,
                                                  double cldn) {
  const double qs = qsat_water(temp, pmid);
  const double rh_max = 0.98;
  double rh = (qs > qv) ? qv / qs : rh_max;
  rh = bound(0.0, rh_max, rh);
  if (cldn < 1.0)
    rh = (rh - cldn) / (1.0 - cldn);
  return dmax(rh, 0.0);
}

// One mode: sp holds its species masses in mode order (sp[0..nspec(m)-1]).
template <int M>
MAM4B_HD void water_uptake_mode(const StepConsts &C, const double (&sp)[7],
                                                  double rh, double dgn_a, double &dgn_awet,
                                                  double &qaerwat, double &wetdens) {
  double hygro = 0.0, dryvolmr = 0.0, maer = 0.0;
#pragma unroll
  for (int s = 0; s < K::nspec(M); ++s) {
    const int w = K::spec0(M) + s - M;  // species index among the 21 masses
    const double raer = sp[s];
    const double vol_tmp = raer / K::wu_dens(w);
    maer = maer + raer;
    dryvolmr += vol_tmp;
    hygro += vol_tmp * K::wu_hygro(w);
  }
  const int w0 = K::spec0(M) - M;
  if (dryvolmr > 1e-30)
    hygro = hygro / dryvolmr;
  else
    hygro = K::wu_hygro(w0);
  const double v2ncur_a = 1.0 / ((K::pi / 6.0) * cube(dgn_a) * exp(4.5 * sq(C.log_sig[M])));
  const double naer = dryvolmr * v2ncur_a;
  const double drydens = (maer > 1e-31) ? maer / dryvolmr : 1.0;
  const double dryvol = 1.0 / v2ncur_a;
  const double drymass = drydens * dryvol;
  const double dryrad = cbrt(dryvol / (K::pi * 4.0 / 3.0));
  double wetrad, wetvol, wtrvol;
  if (rh < K::rh_cryst) {
    // the reference computes the Kohler radius and then discards it below
    // the crystallisation humidity: the values are those it keeps
    wetrad = dryrad;
    wetvol = dryvol;
    wtrvol = 0.0;
  } else {
    wetrad = kohler(C, dryrad, hygro, rh);
    wetrad = dmax(wetrad, dryrad);
    wetvol = (K::pi * 4.0 / 3.0) * cube(wetrad);
    wetvol = dmax(wetvol, dryvol);
    wtrvol = wetvol - dryvol;
    wtrvol = dmax(wtrvol, 0.0);
    if (rh < K::rh_deliq) {
      wtrvol = wtrvol * C.hystfac * (rh - K::rh_cryst);
      wtrvol = dmax(wtrvol, 0.0);
      wetvol = dryvol + wtrvol;
      wetrad = cbrt(wetvol / (4.0 / 3.0 * K::pi));
    }
  }
  dgn_awet = dgn_a * (wetrad / dryrad);
  qaerwat = 1.0e3 * naer * wtrvol;
  wetdens = (wetvol > 1.0e-30) ? (drymass + 1.0e3 * wtrvol) / wetvol : K::wu_dens(w0);
}

template <int M>
MAM4B_HD void mode_species(const double (&ai)[NPOP], double (&sp)[7]) {
#pragma unroll
  for (int s = 0; s < 7; ++s)
    sp[s] = (s < K::nspec(M)) ? ai[K::spec0(M) + (s < K::nspec(M) ? s : 0)] : 0.0;
}

MAM4B_HD void water_uptake(const StepConsts &C, const double (&ai)[NPOP],
                                             double qv, double temp, double pmid, double cldn,
                                             const double (&dgn_a)[NMODE],
                                             double (&dgn_awet)[NMODE],
                                             double (&qaerwat)[NMODE],
                                             double (&wetdens)[NMODE]) {
  const double rh = water_uptake_rh(qv, temp, pmid, cldn);
  double sp[7];
  mode_species<0>(ai, sp);
  water_uptake_mode<0>(C, sp, rh, dgn_a[0], dgn_awet[0], qaerwat[0], wetdens[0]);
  mode_species<1>(ai, sp);
  water_uptake_mode<1>(C, sp, rh, dgn_a[1], dgn_awet[1], qaerwat[1], wetdens[1]);
  mode_species<2>(ai, sp);
  water_uptake_mode<2>(C, sp, rh, dgn_a[2], dgn_awet[2], qaerwat[2], wetdens[2]);
  mode_species<3>(ai, sp);
  water_uptake_mode<3>(C, sp, rh, dgn_a[3], dgn_awet[3], qaerwat[3], wetdens[3]);
}

// ============================================================== amicphys
// Per-subarea state in amicphys internal units (mol/mol with fcvt_aer,
// #/kmol): gas[0]=SOAG, gas[1]=H2SO4; aer[AeroId][mode]; num[mode].
struct Sub {
  double gas[2];
  double num[NMODE];
  double aer[NAER][NMODE];
};

// State of the clear subarea between the start of condensation and the SOA
// loop (everything the rest of mam_amicphys_1subarea needs from before it).
struct ClearMid {
  double netprod1;
  double uptk1[NMODE];
  double sv_so4_ait, sv_soa_ait;
  // DIAG only: values before condensation
  double gas_sv[2];
  double sv_all[NAER][NMODE];
};

// population slot <-> Sub (mass slots in fcvt units, numbers as is)
MAM4B_HD void sub_to_pop(const Sub &s, double (&p)[NPOP]) {
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    p[K::numslot(m)] = s.num[m];
#pragma unroll
    for (int x = 0; x < NAER; ++x)
      if (K::aer_slot(x, m) >= 0)
        p[K::aer_slot(x, m)] = s.aer[x][m];
  }
}
MAM4B_HD void pop_to_sub(const double (&p)[NPOP], Sub &s) {
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    s.num[m] = p[K::numslot(m)];
#pragma unroll
    for (int x = 0; x < NAER; ++x)
      s.aer[x][m] = (K::aer_slot(x, m) >= 0) ? p[K::aer_slot(x, m)] : 0.0;
  }
}

// Sub-area fields of a Sub from populations with per-mode factors
// (number, mass), as the subarea set-up does (mam4_amicphys.hpp:460-560).
MAM4B_HD void load_sub(Sub &s, const double (&q)[NPOP],
                                         const double (&fac_num)[NMODE],
                                         const double (&fac_mass)[NMODE]) {
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    s.num[m] = (q[K::numslot(m)] * fac_num[m]) * 1;
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      const int slot = K::aer_slot(x, m);
      s.aer[x][m] = (slot >= 0) ? (q[slot] * fac_mass[m]) * K::fcvt_aer(x) : 0.0;
    }
  }
}
MAM4B_HD void load_sub_plain(Sub &s, const double (&q)[NPOP]) {
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    s.num[m] = q[K::numslot(m)] * 1;
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      const int slot = K::aer_slot(x, m);
      s.aer[x][m] = (slot >= 0) ? q[slot] * K::fcvt_aer(x) : 0.0;
    }
  }
}

// gasaerexch.hpp:255-353: uptake rate per unit number of mode n for a gas
// with the given diffusivity and mean free path (accommodation 0.65)
MAM4B_HD double uptake_rate_mode(const StepConsts &C, int n, double gasdiffus,
                                                   double freepath, double dgn_awet) {
  const double tworootpi = 2 * sqrt(K::pi);
  const double root2 = sqrt(2.0);
  const double xg = 7.071067690849304E-01;
  const double wg = 8.862269520759583E-01;
  const double a283 = 0.65 * 0.283, a75 = 0.65 * 0.75;
  const double lnsg = C.log_sig[n];
  const double lndpgn = log(dgn_awet);
  const double kn = 2.0 * freepath / dgn_awet;
  const double tmpa =
      1.0 / (1.0 + kn) - (2.0 * kn + 1.0 + a283) / (kn * (kn + 1.0 + a283) + a75);
  double beta = 1.0 - kn * tmpa;
  beta = dmax(1.0, dmin(2.0, beta));
  const double constant = tworootpi * exp(beta * lndpgn + 0.5 * pow(beta * lnsg, 2.0));
  double sum = 0.0;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const double lndp = lndpgn + beta * lnsg * lnsg + root2 * lnsg * (q == 0 ? xg : -xg);
    const double dp = exp(lndp);
    const double knq = 2.0 * freepath / dp;
    const double hh = (a75 * (1.0 + knq)) / (knq * (knq + 1.0 + a283) + a75);
    sum += wg * dp * hh / pow(dp, beta);
  }
  return constant * gasdiffus * sum;
}

MAM4B_HD void uptake_rates(const StepConsts &C, double gasdiffus,
                                             double freepath, const double (&dgn_awet)[NMODE],
                                             double (&uptk)[NMODE]) {
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    uptk[n] = uptake_rate_mode(C, n, gasdiffus, freepath, dgn_awet[n]);
}

// H2SO4 gas diffusivity and mean free path (gasaerexch.hpp:223-253,
// 402-417)
MAM4B_HD void h2so4_diffusivity(double temp, double pmid, double &gas_diffus,
                                                  double &freepath) {
  const double p_in_atm = pmid / 1.013e5;
  const double dgas = (1.0e-3 * pow(temp, 1.75) * sqrt(1. / 9.807840000000000E+01 + 0.035)) /
                      (p_in_atm * pow((pow(4.288000000000000E+01, 1.0 / 3.0) + 2.7189), 2.0));
  gas_diffus = dgas * 1.0e-4;
  const double speed = 145.5 * sqrt(temp / 9.807840000000000E+01);
  freepath = 3.0 * gas_diffus / speed;
}

// SOA gas-particle exchange: mam_soaexch_1subarea (gasaerexch_soaexch.hpp:
// 80-341), semi-implicit with adaptive sub-steps dt = 0.05 / sum(k |phi|),
// bounded by the reference's own cap of 1000 sub-steps. Split into the
// loop state, its set-up and one sub-step so that the same arithmetic runs
// inline or in the work-stealing solver kernel.
struct SoaState {
  double g;              // SOA gas (internal units)
  double a[NMODE];       // particle SOA per mode
  double opoa[NMODE];    // oxygenated POA per mode (0.1 x POM; 0 for pca)
  double uptk[NMODE];    // SOAG uptake rate per mode [1/s]
  double g0;             // equilibrium SOA gas without solute effect
  double tcur, dtfull;
  int niter;
};

MAM4B_HD void soa_init(SoaState &st, double dtfull, double temp, double pmid,
                                         const Sub &s, const double (&uptk)[NMODE]) {
  const double p0_soa = 1.0e-10 * exp(-(156.0e3 / 8.3144) * ((1.0 / temp) - (1.0 / 298.0)));
  st.g0 = 1.01325e5 * p0_soa / pmid;
  constexpr double opoa_frac[NMODE] = {0.1, 0.1, 0.1, 0.0};
  st.g = s.gas[0];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    st.a[n] = s.aer[0][n];
    st.uptk[n] = uptk[n];
    st.opoa[n] = 0.0 + opoa_frac[n] * dmax(s.aer[2][n], 0.0);
  }
  st.tcur = 0.0;
  st.dtfull = dtfull;
  st.niter = 0;
}

// sum(uptake * |phi|) of the loop's first pass (the first sub-step is
// 0.05 / this): a cheap predictor of how many passes the loop will take.
MAM4B_HD double soa_first_rate(const SoaState &st) {
  const double g = dmax(st.g, 0.0);
  double r = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (!(st.uptk[n] > 1.0e-15))
      continue;
    const double a = dmax(st.a[n], 0.0);
    const double gs = (st.g0 / dmax(st.opoa[n] + a, 1.0e-20)) * a;
    r += st.uptk[n] * fabs((g - gs) / dmax(g, dmax(gs, 1.0e-20)));
  }
  return r;
}

// One pass of the reference's while loop; false once the loop has ended.
MAM4B_HD bool soa_step(SoaState &st) {
  if (!(st.tcur < st.dtfull - 1.0e-3))
    return false;
  st.niter++;
  if (st.niter > 1000)
    return false;
  const double qgas_prv = st.g;
  double g_soa = dmax(qgas_prv, 0.0);
  double tot_soa = g_soa;
  double a_soa[NMODE], sat[NMODE], g_star[NMODE], beta[NMODE];
  bool skip[NMODE];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    skip[n] = !(st.uptk[n] > 1.0e-15);
    a_soa[n] = 0.0;
    if (skip[n])
      continue;
    a_soa[n] = dmax(st.a[n], 0.0);
    tot_soa += a_soa[n];
  }
  double tmpb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    const double a_ooa = st.opoa[n] + a_soa[n];
    sat[n] = st.g0 / dmax(a_ooa, 1.0e-20);
    g_star[n] = sat[n] * a_soa[n];
    const double phi = (g_soa - g_star[n]) / dmax(g_soa, dmax(g_star[n], 1.0e-20));
    tmpb += st.uptk[n] * fabs(phi);
  }
  const double tmpa = dmax(0.0, tmpb);
  double dtcur;
  const double dtmax = st.dtfull - st.tcur;
  if (dtmax * tmpa <= 0.05) {
    dtcur = dtmax;
    st.tcur = st.dtfull;
  } else {
    dtcur = 0.05 / tmpa;
    st.tcur += dtcur;
  }
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    double a_tmp = a_soa[n];
    beta[n] = dtcur * st.uptk[n];
    const double del_g = g_soa - g_star[n];
    if (del_g > 0.0) {
      a_tmp += beta[n] * del_g;
      const double a_ooa = st.opoa[n] + a_tmp;
      sat[n] = st.g0 / dmax(a_ooa, 1.0e-20);
    }
  }
  double ta = 0.0, tb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    ta += a_soa[n] / (1.0 + beta[n] * sat[n]);
    tb += beta[n] / (1.0 + beta[n] * sat[n]);
  }
  g_soa = (tot_soa - ta) / (1.0 + tb);
  g_soa = dmax(0.0, g_soa);
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    a_soa[n] = (a_soa[n] + beta[n] * g_soa) / (1.0 + beta[n] * sat[n]);
  }
  st.g = g_soa;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    st.a[n] = a_soa[n];
  return true;
}

// Inline form: runs the whole loop for one subarea; returns the sub-step
// count (1001 when the cap was reached).
MAM4B_HD int soa_exchange(double dtfull, double temp, double pmid, Sub &s,
                                            const double (&uptk)[NMODE]) {
  SoaState st;
  soa_init(st, dtfull, temp, pmid, s, uptk);
  while (soa_step(st)) {
  }
  s.gas[0] = st.g;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    s.aer[0][n] = st.a[n];
  return st.niter;
}

// H2SO4 quasi-analytic update (gasaerexch.hpp:486-537)
MAM4B_HD void h2so4_update(double dt, double netprod, Sub &s,
                                             const double (&uptk)[NMODE], double &qavg) {
  const double q1 = s.gas[1];
  double tmpa = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    tmpa += uptk[n];
  const double kxt = tmpa * dt, pxt = netprod * dt;
  if (kxt >= 1.0e-20) {
    double q3, q4;
    if (kxt > 0.001) {
      const double pok = pxt / kxt;
      const double e = exp(-kxt);
      q3 = (q1 - pok) * e + pok;
      q4 = (q1 - pok) * (1.0 - e) / kxt + pok;
    } else {
      const double kxt2 = kxt * kxt;
      q3 = q1 * (1.0 - kxt + kxt2 * 0.5) + pxt * (1.0 - kxt * 0.5 + kxt2 / 6.0);
      q4 = q1 * (1.0 - kxt * 0.5 + kxt2 / 6.0) + pxt * (0.5 - kxt / 6.0 + kxt2 / 24.0);
    }
    s.gas[1] = q3;
    const double qdel = (q1 + pxt) - q3;
    qavg = q4;
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      if (uptk[n] > 0.0)
        s.aer[1][n] = s.aer[1][n] + qdel * (uptk[n] / tmpa);
  } else {
    s.gas[1] = q1 + pxt;
    qavg = q1 + pxt * 0.5;
  }
}

// Aitken->accumulation renaming of one subarea (rename.hpp:23-390 with
// the pair constants of find_renaming_pairs :393-476). grow_i/grow_c are
// the growth increments of the aitken species (AeroId order).
template <bool CLOUDY>
MAM4B_HD void rename_subarea(const StepConsts &C, Sub &si, Sub &sc,
                                               const double (&grow_i)[NAER],
                                               const double (&grow_c)[NAER]) {
  const int src = 1, dst = 0;
  double dv_i, ddv_i, dv_c = 0.0, ddv_c = 0.0;
  {
    double t = 0.0, td = 0.0;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      t += si.aer[a][src] * K::mass_2_vol(a);
      td += grow_i[a] * K::mass_2_vol(a);
    }
    dv_i = t - td;
    ddv_i = td;
  }
  if (CLOUDY) {
    double t = 0.0, td = 0.0;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      t += sc.aer[a][src] * K::mass_2_vol(a);
      td += grow_c[a] * K::mass_2_vol(a);
    }
    dv_c = t - td;
    ddv_c = td;
  }
  double b4_dv = dv_i;
  if (CLOUDY)
    b4_dv = b4_dv + dv_c;
  const double b4_dv_b = dmax(b4_dv, 1.0e-25);
  double b4_n = si.num[src];
  if (CLOUDY)
    b4_n = b4_n + sc.num[src];
  b4_n = dmax(0.0, b4_n);
  const double b4_n_b = bound(b4_dv_b * C.rn_v2n_hi_rlx, b4_dv_b * C.rn_v2n_lo_rlx, b4_n);
  double del = ddv_i;
  if (CLOUDY)
    del = del + ddv_c;
  const double aft_dv = b4_dv + del;
  if (aft_dv <= 1.0e-25)
    return;
  double b4_d = diam_from_vol(b4_dv_b / b4_n_b, C.log_sig[src]);
  if (b4_d > C.rn_threshold) {
    b4_dv = b4_dv * cube(C.rn_threshold / b4_d);
    b4_d = C.rn_threshold;
  }
  if ((aft_dv - b4_dv) <= 1.0e-6 * b4_dv_b)
    return;
  const double aft_d = diam_from_vol(aft_dv / b4_n_b, C.log_sig[src]);
  if (aft_d <= K::dnom(src))
    return;
  const double lb4 = log(b4_d), laft = log(aft_d);
  const double b4_tn = 0.5 * erfc((C.rn_ln_cutoff - lb4) * C.rn_fac);
  const double b4_tv = 0.5 * erfc((C.rn_ln_cutoff - (lb4 + C.rn_ln_tail_fac)) * C.rn_fac);
  const double aft_tn = 0.5 * erfc((C.rn_ln_cutoff - laft) * C.rn_fac);
  const double aft_tv = 0.5 * erfc((C.rn_ln_cutoff - (laft + C.rn_ln_tail_fac)) * C.rn_fac);
  const double vfrac = aft_tv * aft_dv - b4_tv * b4_dv;
  if (vfrac <= 0.0)
    return;
  double xv = dmin(vfrac, aft_dv) / aft_dv;
  xv = dmin(xv, 1.0 - 10.0 * K::eps);
  double xn = aft_tn - b4_tn;
  xn = dmax(0.0, dmin(xn, xv));
  {
    const double nt = si.num[src] * xn;
    si.num[src] -= nt;
    si.num[dst] += nt;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      const double vt = si.aer[a][src] * xv;
      si.aer[a][src] -= vt;
      si.aer[a][dst] += vt;
    }
  }
  if (CLOUDY) {
    const double nt = sc.num[src] * xn;
    sc.num[src] -= nt;
    sc.num[dst] += nt;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      const double vt = sc.aer[a][src] * xv;
      sc.aer[a][src] -= vt;
      sc.aer[a][dst] += vt;
    }
  }
}

// ------------------------------------------------------------ nucleation
// Vehkamaki et al. (2002) fits (vehkamaki2002.hpp:54-190)
MAM4B_HD double veh02_x_crit(double lna, double t, double lrh) {
  return 0.740997 - 0.00266379 * t - 0.00349998 * lna + 0.0000504022 * t * lna +
         0.00201048 * lrh - 0.000183289 * t * lrh + 0.00157407 * sq(lrh) -
         0.0000179059 * t * sq(lrh) + 0.000184403 * cube(lrh) - 1.50345e-6 * t * cube(lrh);
}
MAM4B_HD double veh02_log_rate(double lna, double t, double lrh, double x) {
  const double a = 0.14309 + 2.21956 * t - 0.0273911 * sq(t) + 0.0000722811 * cube(t) + 5.91822 / x;
  const double b = 0.117489 + 0.462532 * t - 0.0118059 * sq(t) + 0.0000404196 * cube(t) + 15.7963 / x;
  const double c = -0.215554 - 0.0810269 * t + 0.00143581 * sq(t) - 4.7758e-6 * cube(t) - 2.91297 / x;
  const double d = -3.58856 + 0.049508 * t - 0.00021382 * sq(t) + 3.10801e-7 * cube(t) - 0.0293333 / x;
  const double e = 1.14598 - 0.600796 * t + 0.00864245 * sq(t) - 0.0000228947 * cube(t) - 8.44985 / x;
  const double f = 2.15855 + 0.0808121 * t - 0.000407382 * sq(t) - 4.01957e-7 * cube(t) + 0.721326 / x;
  const double g = 1.6241 - 0.0160106 * t + 0.0000377124 * sq(t) + 3.21794e-8 * cube(t) - 0.0113255 / x;
  const double h = 9.71682 - 0.115048 * t + 0.000157098 * sq(t) + 4.00914e-7 * cube(t) + 0.71186 / x;
  const double i = -1.05611 + 0.00903378 * t - 0.0000198417 * sq(t) + 2.46048e-8 * cube(t) - 0.0579087 / x;
  const double j = -0.148712 + 0.00283508 * t - 9.24619e-6 * sq(t) + 5.00427e-9 * cube(t) - 0.0127081 / x;
  return a + b * lrh + c * sq(lrh) + d * cube(lrh) + e * lna + f * lrh * lna + g * sq(lrh) * lna +
         h * sq(lna) + i * lrh * sq(lna) + j * cube(lna);
}
MAM4B_HD double veh02_ntot(double lna, double t, double lrh, double x) {
  const double A = -0.00295413 - 0.0976834 * t + 0.00102485 * sq(t) - 2.18646e-6 * cube(t) - 0.101717 / x;
  const double B = -0.00205064 - 0.00758504 * t + 0.000192654 * sq(t) - 6.7043e-7 * cube(t) - 0.255774 / x;
  const double Cc = +0.00322308 + 0.000852637 * t - 0.0000154757 * sq(t) + 5.66661e-8 * cube(t) + 0.0338444 / x;
  const double D = +0.0474323 - 0.000625104 * t + 2.65066e-6 * sq(t) - 3.67471e-9 * cube(t) - 0.000267251 / x;
  const double E = -0.0125211 + 0.00580655 * t - 0.000101674 * sq(t) + 2.88195e-7 * cube(t) + 0.0942243 / x;
  const double F = -0.038546 - 0.000672316 * t + 2.60288e-6 * sq(t) + 1.19416e-8 * cube(t) - 0.00851515 / x;
  const double G = -0.0183749 + 0.000172072 * t - 3.71766e-7 * sq(t) - 5.14875e-10 * cube(t) + 0.00026866 / x;
  const double H = -0.0619974 + 0.000906958 * t - 9.11728e-7 * sq(t) - 5.36796e-9 * cube(t) - 0.00774234 / x;
  const double I = +0.0121827 - 0.00010665 * t + 2.5346e-7 * sq(t) - 3.63519e-10 * cube(t) + 0.000610065 / x;
  const double J = +0.000320184 - 0.0000174762 * t + 6.06504e-8 * sq(t) - 1.4177e-11 * cube(t) + 0.000135751 / x;
  return exp(A + B * lrh + Cc * sq(lrh) + D * cube(lrh) + E * lna + F * lrh * lna +
             G * sq(lrh) * lna + H * sq(lna) + I * lrh * sq(lna) + J * cube(lna));
}

// mam_newnuc_1subarea (mam4_amicphys.hpp:917-1094) with
// mer07_veh02_nuc_mosaic_1box (nucleation.hpp:347-860) for method 11, one
// size bin, no NH3. Quirk kept: a critical cluster that falls between the
// bin bounds produces nothing (nucleation.hpp:620-631).
MAM4B_HD void nucleation(const StepConsts &C, double deltat, double temp,
                                           double pmid, double zmid, double pblh, double relhum,
                                           double uptkrate_h2so4, double qgas_avg1, Sub &s) {
  const double qh2so4_cur = s.gas[1];
  const double qh2so4_avg = qgas_avg1;
  if (qh2so4_avg <= 4.0e-16)
    return;
  const double rh_in = dmax(0.01, dmin(0.99, relhum));
  const double rgas = 8.31446759100000, avogad = 6.022140000000000E+023;
  const double mw_so4a = 96.0, mw_so4a_host = 115.0, dens = 1770.0;
  const double cair = pmid / (temp * rgas);
  const double so4vol = qh2so4_avg * cair * avogad * 1.0e-6;
  double rateloge = log(1.0e-38);
  double cnum_h2so4 = 0.0, radius_cluster = 0.0;
  if (so4vol >= 1.0e4) {
    const double t = dmax(230.15, dmin(305.15, temp));
    const double rh = dmax(1.0e-4, dmin(1.0, rh_in));
    const double na = dmax(1.0e4, dmin(1.0e11, so4vol));
    const double lna = log(na), lrh = log(rh);
    const double x_crit = veh02_x_crit(lna, t, lrh);
    rateloge = veh02_log_rate(lna, t, lrh, x_crit);
    const double cnum_tot = veh02_ntot(lna, t, lrh, x_crit);
    cnum_h2so4 = cnum_tot * x_crit;
    radius_cluster = exp(-1.6524245 + 0.42316402 * x_crit + 0.3346648 * log(cnum_tot));
  }
  rateloge = rateloge + 0.0;  // + log(adjust factor 1)
  if (zmid <= dmax(pblh, 100.0)) {
    // first-order boundary-layer rate, Wang & Penner (2008)
    const double tmp_rate = 1e-6 * so4vol;
    const double tmp_loge = log(dmax(1.0e-38, tmp_rate));
    if (!(tmp_loge <= rateloge)) {
      rateloge = tmp_loge;
      radius_cluster = 0.5;
      const double tmp_diam = radius_cluster * 2.0e-7;
      const double tmp_volu = cube(tmp_diam) * (K::pi / 6.0);
      const double tmp_mass = tmp_volu * 1.8;
      cnum_h2so4 = (tmp_mass / 98.0) * 6.023e23;
    }
  }
  if (rateloge <= -13.82)
    return;
  const double ratenuclt_bb = exp(rateloge) * 1.0e6;
  const double wetvol_dryvol = 1.0 - 0.56 / log(dmax(0.10, dmin(0.95, rh_in)));
  double voldry_clus = (dmax(cnum_h2so4, 1.0) * mw_so4a + 0.0 * 18.0) / (1.0e3 * dens * avogad);
  voldry_clus = voldry_clus * (mw_so4a_host / mw_so4a);
  const double dpdry_clus = pow(voldry_clus * 6.0 / K::pi, 1.0 / 3.0);
  const double dp_lo = C.nuc_dplom, dp_hi = K::dmax(1);
  bool igrow;
  double dpdry_part;
  if (dpdry_clus <= dp_lo) {
    igrow = true;
    dpdry_part = dp_lo;
  } else if (dpdry_clus >= dp_hi) {
    igrow = false;
    dpdry_part = dp_hi;
  } else {
    return;
  }
  const double voldry_part = (K::pi / 6.0) * pow(dpdry_part, 3.0);
  // composition of the grown particles with no NH3 (nucleation.hpp:660-690):
  // sulfuric acid, except the reference's ammonium branch taken when the
  // remaining H2SO4 is exactly zero
  double n1 = 0.0, n2 = 0.0, n3 = 0.0;
  if (!igrow) {
    n3 = 1.0;
  } else if (0.0 >= qh2so4_cur) {
    n1 = (0.0 / qh2so4_cur) - 1.0;
    n1 = dmax(0.0, dmin(1.0, n1));
    n2 = 1.0 - n1;
  } else {
    n2 = (0.0 / qh2so4_cur);
    n2 = dmax(0.0, dmin(1.0, n2));
    n3 = 1.0 - n2;
  }
  const double m1 = n1 * 132.0, m2 = n2 * 114.0, m3 = n3 * 96.0;
  const double dens_part = (m1 + m2 + m3) / ((m1 / dens) + (m2 / dens) + (m3 / dens));
  const double mass_part = voldry_part * dens_part;
  const double mole_nh4 = 2.0 * n1 + n2;
  double kgaero = 1.0e-3 * (m1 + m2 + m3);
  kgaero = kgaero * (mw_so4a_host / mw_so4a);
  const double wet_volfrac_so4a = 1.0 / (wetvol_dryvol * (1.0 + mole_nh4 * 17.0 / 98.0));
  double factor_kk = 1.0;
  if (igrow) {
    const double tmp_spd = 14.7 * sqrt(temp);
    const double gr_kk = 3.0e-9 * tmp_spd * 96.0 * so4vol / (dens_part * wet_volfrac_so4a);
    const double dfin_kk = 1.0e9 * dpdry_part * pow(wetvol_dryvol, 1.0 / 3.0);
    const double dnuc_kk = dmax(2.0 * radius_cluster, 1.0);
    const double gamma_kk = 0.23 * pow(dnuc_kk, 0.2) * pow(dfin_kk / 3.0, 0.075) *
                            pow(dens_part * 1.0e-3, -0.33) * pow(temp / 293.0, -0.75);
    const double tmpa = dmax(uptkrate_h2so4 * 3600.0, 0.0);
    const double tmpb = (6.7037e-6 * pow(temp, 0.75) / cair) * 3600.0;
    const double cs_prime_kk = tmpa / (4.0 * K::pi * tmpb * 0.65);
    const double nu_kk = gamma_kk * cs_prime_kk / gr_kk;
    factor_kk = exp((nu_kk / dfin_kk) - (nu_kk / dnuc_kk));
  }
  const double ratenuclt_kk = ratenuclt_bb * factor_kk;
  const double qmolso4a_del_max = dmax(0.0, (ratenuclt_kk * deltat * mass_part)) / (kgaero * cair);
  double freducea = 1.0, freduceb = 1.0;
  if (qmolso4a_del_max > qh2so4_cur)
    freducea = qh2so4_cur / qmolso4a_del_max;
  if (mole_nh4 >= 1.0e-10) {
    if (qmolso4a_del_max * mole_nh4 > 0.0)
      freduceb = 0.0 / (qmolso4a_del_max * mole_nh4);
  }
  const double freduce = dmin(freducea, freduceb);
  if ((freduce * ratenuclt_kk) <= 1.0e-12)
    return;
  const double qh2so4_del = dmin(0.9999 * qh2so4_cur, freduce * qmolso4a_del_max);
  const double qnh3_del = dmin(0.9999 * 0.0, qh2so4_del * mole_nh4);
  const double qso4a_del = qh2so4_del;
  const double qnuma_del = 1.0e-3 * (qso4a_del * mw_so4a + qnh3_del * 18.0) / mass_part;
  // back in mam_newnuc_1subarea
  double dndt = (qnuma_del * 1.0e3) / deltat;
  double dmdt = dmax(0.0, ((qso4a_del * mw_so4a_host) / deltat));
  if (dndt < 1.0e2) {
    dndt = 0.0;
    dmdt = 0.0;
  } else {
    const double mass1p = dmdt / dndt;
    if (mass1p < C.nuc_mass1p_lo)
      dndt = dmdt / C.nuc_mass1p_lo;
    else if (mass1p > C.nuc_mass1p_hi)
      dmdt = dndt * C.nuc_mass1p_hi;
  }
  s.num[1] = s.num[1] + dndt * deltat;
  const double dso4dt = dmdt * 1.0 / mw_so4a_host;
  if (dso4dt > 0.0) {
    double tq = dso4dt * deltat;
    s.aer[1][1] = s.aer[1][1] + tq;
    tq = dmin(tq, s.gas[1]);
    s.gas[1] = s.gas[1] - tq;
  }
}

// ----------------------------------------------------------- coagulation
// getcoags_wrapper_f + getcoags (coagulation.hpp:651-817) for one mode pair
MAM4B_HD void coag_coefs(const CoagTables &T, double airtemp, double airprs,
                                           double dgatk, double dgacc, double sgatk,
                                           double sgacc, double xxlsgat, double xxlsgac,
                                           double pdensat, double pdensac, double &bij0,
                                           double &bij3, double &bii0, double &bjj0) {
  const double t0 = 273.15 + 15.0;
  const double sqrt_temp = sqrt(airtemp);
  const double lamda = 6.6328e-8 * 101325.0 * airtemp / (t0 * airprs);
  const double amu = 1.458e-6 * airtemp * sqrt_temp / (airtemp + 110.4);
  const double boltzmann = 1.3806500000000000e-023;
  const double knc = (2.0 / 3.0) * boltzmann * airtemp / amu;
  const double kfmat = sqrt(3.0 * boltzmann * airtemp / pdensat);
  const double kfmac = sqrt(3.0 * boltzmann * airtemp / pdensac);
  const double kfmatac = sqrt(6.0 * boltzmann * airtemp / (pdensat + pdensac));
  const double a = 1.246;
  const double esat01 = exp(0.125 * xxlsgat * xxlsgat);
  const double esac01 = exp(0.125 * xxlsgac * xxlsgac);
  const double dlgsqt2 = 1.0 / log(sqrt(2.0));
  const double esat04 = pow(esat01, 4.0), esac04 = pow(esac01, 4.0);
  const double esat05 = esat04 * esat01, esac05 = esac04 * esac01;
  const double esat08 = esat04 * esat04, esac08 = esac04 * esac04;
  const double esat09 = esat08 * esat01, esac09 = esac08 * esac01;
  const double esat16 = esat08 * esat08, esac16 = esac08 * esac08;
  const double esat20 = esat16 * esat04, esac20 = esac16 * esac04;
  const double esat24 = esat20 * esat04;
  const double esat25 = esat20 * esat05, esac25 = esac20 * esac05;
  const double esat36 = esat20 * esat16;
  const double esat49 = esat24 * esat25;
  const double esat64 = esat20 * esat20 * esat24;
  const double esat100 = esat64 * esat36;
  const double dgat3 = dgatk * dgatk * dgatk;
  const double sqdgat = sqrt(dgatk), sqdgac = sqrt(dgacc);
  const double sqdgat7 = dgat3 * sqdgat;
  const double r1 = sqdgac / sqdgat;
  const double r2 = r1 * r1;
  const double rx4 = r2 * r2;
  const double ri1 = 1.0 / r1;
  const double ri2 = 1.0 / (r1 * r1);
  const double ri3 = 1.0 / (r1 * r1 * r1);
  const double kngat = 2.0 * lamda / dgatk;
  const double kngac = 2.0 * lamda / dgacc;
  const double rat = dgacc / dgatk;
  const int n2n = (int)dmax(1.0, dmin(10.0, round(4.0 * (sgatk - 0.75)))) - 1;
  const int n2a = (int)dmax(1.0, dmin(10.0, round(4.0 * (sgacc - 0.75)))) - 1;
  const int n1 = (int)dmax(1.0, dmin(10.0, 1.0 + round(dlgsqt2 * log(rat)))) - 1;
  // the reference passes (n1, n2n, n2a) into bm*_data(n1, n2a, n2n)
  // (coagulation.hpp:309, 558), i.e. it reads table[n1][n2n][n2a]
  const int tix = n1 * 100 + n2n * 10 + n2a;
  const double bm0ij = MAM4B_LDG(T.bm0ij + tix);
  const double bm3i = MAM4B_LDG(T.bm3i + tix);
  const double coagnc0 = knc * (2.0 + a * (kngat * (esat04 + r2 * esat16 * esac04) +
                                           kngac * (esac04 + ri2 * esac16 * esat04)) +
                                (r2 + ri2) * esat04 * esac04);
  const double coagfm0 = kfmatac * sqdgat * bm0ij *
                         (esat01 + r1 * esac01 + 2.0 * r2 * esat01 * esac04 +
                          rx4 * esat09 * esac16 + ri3 * esat16 * esac09 + 2.0 * ri1 * esat04 +
                          esac01);
  const double qn12 = coagnc0 * coagfm0 / (coagnc0 + coagfm0);
  const double coagnc3 =
      knc * dgat3 *
      (2.0 * esat36 + a * kngat * (esat16 + r2 * esat04 * esac04) +
       a * kngac * (esat36 * esac04 + ri2 * esat64 * esac16) + r2 * esat16 * esac04 +
       ri2 * esat64 * esac04);
  const double coagfm3 = kfmatac * sqdgat7 * bm3i *
                         (esat49 + r1 * esat36 * esac01 + 2.0 * r2 * esat25 * esac04 +
                          rx4 * esat09 * esac16 + ri3 * esat100 * esac09 +
                          2.0 * ri1 * esat64 * esac01);
  const double qv12 = coagnc3 * coagfm3 / (coagnc3 + coagfm3);
  const double cnc11 = knc * (1.0 + esat08 + a * kngat * (esat20 + esat04));
  const double cfm11 = kfmat * sqdgat * MAM4B_LDG(T.bm0 + n2n) * (esat01 + esat25 + 2.0 * esat05);
  const double qn11 = cfm11 * cnc11 / (cfm11 + cnc11);
  const double cnc22 = knc * (1.0 + esac08 + a * kngac * (esac20 + esac04));
  const double cfm22 = kfmac * sqdgac * MAM4B_LDG(T.bm0 + n2a) * (esac01 + esac25 + 2.0 * esac05);
  const double qn22 = cfm22 * cnc22 / (cfm22 + cnc22);
  bii0 = dmax(0.0, qn11);
  bjj0 = dmax(0.0, qn22);
  bij0 = dmax(0.0, qn12);
  const double dumatk3 = (cube(dgatk) * exp(4.5 * xxlsgat * xxlsgat));
  bij3 = dmax(0.0, qv12 / dumatk3);
}

MAM4B_HD double qnum_intra_inter(double bijdtqnumj, double biidt,
                                                   double qnumi_bgn) {
  // coagulation.hpp:938-952
  if (bijdtqnumj < 1.0e-5)
    return qnumi_bgn / (1.0 + (bijdtqnumj + biidt * qnumi_bgn) * (1.0 + 0.5 * bijdtqnumj));
  const double e = exp(-bijdtqnumj);
  return qnumi_bgn * e / (1.0 + (biidt * qnumi_bgn / bijdtqnumj) * (1.0 - e));
}

// Coagulation coefficients of the three mode pairs (aitken->accumulation,
// pcarbon->accumulation, aitken->pcarbon) in the order mam_coag_1subarea
// uses them (coagulation.hpp:1060-1085), times the air molar concentration:
// cc[0..2] bij0, cc[3..5] bij3, cc[6..8] bii0, cc[9..11] bjj0.
MAM4B_HD constexpr int coag_src(int p) { return p == 1 ? 3 : 1; }
MAM4B_HD constexpr int coag_dst(int p) { return p == 2 ? 3 : 0; }
MAM4B_HD void coag_pair_coefs(const StepConsts &C, const CoagTables &T, int p,
                                                double temp, double pmid, double aircon,
                                                double dgn_src, double dgn_dst, double dens_src,
                                                double dens_dst, double &bij0, double &bij3,
                                                double &bii0, double &bjj0) {
  const int sm = coag_src(p), dm = coag_dst(p);
  coag_coefs(T, temp, pmid, dgn_src, dgn_dst, K::sig(sm), K::sig(dm), C.log_sig[sm],
             C.log_sig[dm], dens_src, dens_dst, bij0, bij3, bii0, bjj0);
  bij0 *= aircon;
  bij3 *= aircon;
  bii0 *= aircon;
  bjj0 *= aircon;
}

MAM4B_HD void coag_all_coefs(const StepConsts &C, const CoagTables &T,
                                               double temp, double pmid, double aircon,
                                               const double (&dgn_awet)[NMODE],
                                               const double (&wetdens)[NMODE], double (&cc)[12]) {
#pragma unroll
  for (int p = 0; p < 3; ++p)
    coag_pair_coefs(C, T, p, temp, pmid, aircon, dgn_awet[coag_src(p)], dgn_awet[coag_dst(p)],
                    wetdens[coag_src(p)], wetdens[coag_dst(p)], cc[p], cc[3 + p], cc[6 + p],
                    cc[9 + p]);
}

// mam_coag_1subarea (coagulation.hpp:1038-1119) with the coefficients cc of
// coag_all_coefs; coag_in receives the mass moved into the primary-carbon
// mode (AeroId order)
MAM4B_HD void coagulation(double deltat, const double (&cc)[12], Sub &s,
                                            double (&coag_in)[NAER]) {
  double bgn[NAER][NMODE], nbgn[NMODE];
#pragma unroll
  for (int a = 0; a < NAER; ++a)
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      s.aer[a][m] = dmax(0.0, s.aer[a][m]);
      bgn[a][m] = s.aer[a][m];
    }
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    s.num[m] = dmax(0.0, s.num[m]);
    nbgn[m] = s.num[m];
  }
  const double bij0[3] = {cc[0], cc[1], cc[2]}, bij3[3] = {cc[3], cc[4], cc[5]};
  const double bii0[3] = {cc[6], cc[7], cc[8]}, bjj0[3] = {cc[9], cc[10], cc[11]};
  // mam_coag_num_update (:982-1027): accumulation, then pcarbon, then aitken
  double tavg[NMODE];
  s.num[0] = nbgn[0] / (1.0 + bjj0[0] * deltat * nbgn[0]);
  tavg[0] = (nbgn[0] + s.num[0]) * 0.5;
  s.num[3] = qnum_intra_inter(dmax(0.0, deltat * bij0[1] * tavg[0]), dmax(0.0, deltat * bii0[1]),
                              nbgn[3]);
  tavg[3] = (nbgn[3] + s.num[3]) * 0.5;
  {
    double bq = bij0[0] * tavg[0];
    bq = bq + bij0[2] * tavg[3];
    s.num[1] = qnum_intra_inter(dmax(0.0, deltat * bq), dmax(0.0, deltat * bii0[0]), nbgn[1]);
  }
  // mam_coag_aer_update (:850-930)
#pragma unroll
  for (int a = 0; a < NAER; ++a)
    coag_in[a] = 0.0;
  const double bq1 = dmax(0.0, bij3[0] * tavg[0]);
  const double bq2 = dmax(0.0, bij3[2] * tavg[3]);
  double decay_const = bq1 + bq2;
  double decay_factor = deltat * decay_const;
  if (decay_factor > K::eps * 2.0) {
    const double prtn2 = bq2 / decay_const;
    const double prtn1 = 1.0 - prtn2;
    const double xf = 1.0 - exp(-decay_factor);
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      const double dq = xf * bgn[a][1];
      s.aer[a][1] -= dq;
      s.aer[a][0] += dq * prtn1;
      s.aer[a][3] += dq * prtn2;
      coag_in[a] += dq * prtn2;
    }
  }
  decay_const = dmax(0.0, bij3[1] * tavg[0]);
  decay_factor = deltat * decay_const;
  if (decay_factor > K::eps * 2.0) {
    const double xf = 1.0 - exp(-decay_factor);
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      const double dq = xf * bgn[a][3];
      s.aer[a][3] -= dq;
      s.aer[a][0] += dq;
    }
  }
}

// ------------------------------------------------------------------ aging
// mam_pcarbon_aging_1subarea (aging.hpp:70-361)
MAM4B_HD void aging(const StepConsts &C, unsigned nmono, double dgn_a_pc, Sub &s,
                                      double (&dnum_cond)[NMODE], double (&dnum_coag)[NMODE],
                                      double (&daer_cond)[NAER][NMODE],
                                      double (&daer_coag)[NAER][NMODE],
                                      const double (&coag_in)[NAER]) {
  const int pc = 3, acc = 0;
  const double vol_shell = s.aer[1][pc] * C.so4_vol + s.aer[0][pc] * C.soa_fac_eqvhyg;
  double dcond = daer_cond[1][pc] * C.so4_vol + daer_cond[0][pc] * C.soa_fac_eqvhyg;
  const double dcoag = coag_in[1] * C.so4_vol + coag_in[0] * C.soa_fac_eqvhyg;
  dcond = dmax(dcond, 1e-35);
  const double frac_cond = dcond / (dcond + dmax(dcoag, 0.0));
  const double frac_coag = 1.0 - frac_cond;
  double vol_core = 0.0;
  vol_core += s.aer[2][pc] * K::mass_2_vol(2);
  vol_core += s.aer[3][pc] * K::mass_2_vol(3);
  vol_core += s.aer[6][pc] * K::mass_2_vol(6);
  const double xmax = 1.0 - 10.0 * K::eps;
  const double tmp1 = vol_shell * dgn_a_pc * C.aging_fac_volsfc;
  const double dr = nmono * 4.76e-10;
  const double tmp2 = dmax(6.0 * dr * vol_core, 0.0);
  const double xfer = (tmp1 >= tmp2) ? xmax : dmin(tmp1 / tmp2, xmax);
  constexpr int to_acc[3] = {2, 3, 6};
  constexpr int all_to_acc[4] = {0, 1, 4, 5};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = to_acc[k];
    const double q = s.aer[a][pc] * xfer;
    s.aer[a][pc] -= q;
    s.aer[a][acc] += q;
    daer_cond[a][pc] -= q * frac_cond;
    daer_cond[a][acc] += q * frac_cond;
    daer_coag[a][pc] -= q * frac_coag;
    daer_coag[a][acc] += q * frac_coag;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int a = all_to_acc[k];
    s.aer[a][acc] += s.aer[a][pc];
    daer_cond[a][acc] += daer_cond[a][pc];
    daer_coag[a][acc] += daer_coag[a][pc];
    s.aer[a][pc] = 0.0;
    daer_cond[a][pc] = 0.0;
    daer_coag[a][pc] = 0.0;
  }
  const double q = s.num[pc] * xfer;
  s.num[pc] -= q;
  s.num[acc] += q;
  dnum_cond[pc] -= q * frac_cond;
  dnum_cond[acc] += q * frac_cond;
  dnum_coag[pc] -= q * frac_coag;
  dnum_coag[acc] += q * frac_coag;
}

}  // namespace mam4b
