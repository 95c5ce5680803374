// mam4b_optics.cuh -- longwave aerosol optics of a cell,
// mam4::modal_aero_opt::modal_aero_lw_k (src/mam4xx/modal_aero_opt.hpp:
// 879-989): dry and wet mode sizes (calcsize and water uptake, as the
// microphysics step computes them), then for every mode and longwave band
// the volume-mixed complex refractive index of the species and water
// (calc_refin_complex :329-410), a bilinear interpolation of the
// Chebyshev coefficients of specific absorption over the refractive-index
// table (binterp / compute_factors :412-508), their evaluation at the
// mode's surface radius (modal_size_parameters / calc_parameterized
// :192-258) and the layer's absorption optical depth.
#pragma once

#include "mam4b_activation.cuh"
#include "mam4b_physics.cuh"

namespace mam4b {
namespace opt {

constexpr int kLwBands = 16, kNcoef = 5, kPrefr = 7, kPrefi = 10;
// device table layout (doubles): per-mode species refractive indices
// (mapped from the per-type table by species type), water, the
// refractive-index grids and the absorption coefficient tables
constexpr int kSpecRe = 0;                                    // [4][7][16]
constexpr int kSpecIm = kSpecRe + 4 * 7 * kLwBands;           // [4][7][16]
constexpr int kWaterRe = kSpecIm + 4 * 7 * kLwBands;          // [16]
constexpr int kWaterIm = kWaterRe + kLwBands;                 // [16]
constexpr int kRefr = kWaterIm + kLwBands;                    // [4][16][7]
constexpr int kRefi = kRefr + 4 * kLwBands * kPrefr;          // [4][16][10]
constexpr int kAbsp = kRefi + 4 * kLwBands * kPrefi;          // [4][16][5][7][10]
constexpr int kTableDoubles = kAbsp + 4 * kLwBands * kNcoef * kPrefr * kPrefi;

// Where the tables of one band sit. LwTables / SwTables: the whole device
// table (the layouts here, read through the read-only data cache). LwBand /
// SwBand: one band's values staged in shared memory by the band kernels
// (species and water indices, the two refractive-index grids and the
// coefficient tables of the four modes, band index dropped). The functions
// below read the same values in the same order through either, so their
// results do not depend on where the tables are.
struct LwTables {
  static constexpr bool kShared = false;
  MAM4B_HD static int spec_re(int m, int s, int b) { return kSpecRe + (m * 7 + s) * kLwBands + b; }
  MAM4B_HD static int spec_im(int m, int s, int b) { return kSpecIm + (m * 7 + s) * kLwBands + b; }
  MAM4B_HD static int water_re(int b) { return kWaterRe + b; }
  MAM4B_HD static int water_im(int b) { return kWaterIm + b; }
  MAM4B_HD static int refr(int m, int b) { return kRefr + (m * kLwBands + b) * kPrefr; }
  MAM4B_HD static int refi(int m, int b) { return kRefi + (m * kLwBands + b) * kPrefi; }
  MAM4B_HD static int absp(int m, int b) {
    return kAbsp + (m * kLwBands + b) * kNcoef * kPrefr * kPrefi;
  }
};

struct LwBand {
  static constexpr bool kShared = true;
  MAM4B_HD static int spec_re(int m, int s, int) { return m * 7 + s; }
  MAM4B_HD static int spec_im(int m, int s, int) { return 28 + m * 7 + s; }
  MAM4B_HD static int water_re(int) { return 56; }
  MAM4B_HD static int water_im(int) { return 57; }
  MAM4B_HD static int refr(int m, int) { return 58 + m * kPrefr; }
  MAM4B_HD static int refi(int m, int) { return 86 + m * kPrefi; }
  MAM4B_HD static int absp(int m, int) { return 126 + m * kNcoef * kPrefr * kPrefi; }
};
constexpr int kLwBandDoubles = 126 + 4 * kNcoef * kPrefr * kPrefi;

template <class L>
MAM4B_HD double tld(const double *p) {
  if constexpr (L::kShared)
    return *p;
  else
    return MAM4B_LDG(p);
}

// position of ref in a table: index of the bracket and the fraction
// (compute_factors)
template <class L>
MAM4B_HD void table_factors(int n, double ref, const double *tab, int &ix, double &tt) {
  ix = 1;
  tt = 0.0;
  if (n > 1) {
    int ii = 0;
    for (ii = 0; ii < n; ++ii)
      if (ref < tld<L>(tab + ii))
        break;
    ix = (ii - 1 > 0) ? ii - 1 : 0;
    const int ip1 = (ix + 1 < n - 1) ? ix + 1 : n - 1;
    const double dx = tld<L>(tab + ip1) - tld<L>(tab + ix);
    if (fabs(dx) > 1.e-20)
      tt = (ref - tld<L>(tab + ix)) / dx;
  }
}

// Chebyshev polynomials at the surface-mode radius of a mode with wet
// diameter dgn_w (modal_size_parameters, method 2)
MAM4B_HD void mode_cheb(int m, double dgn_w, double (&cheb)[kNcoef]) {
  const double xrmin = log(0.01e-6), xrmax = log(25.e-6);
  const double alnsg = log(K::sig(m));
  const double logradsurf = log(0.5 * dgn_w) + 2.0 * alnsg * alnsg;
  double xrad = bound(xrmin, xrmax, logradsurf);
  xrad = (2.0 * xrad - xrmax - xrmin) / (xrmax - xrmin);
  cheb[0] = 1.0;
  cheb[1] = xrad;
#pragma unroll
  for (int nc = 2; nc < kNcoef; ++nc)
    cheb[nc] = 2.0 * xrad * cheb[nc - 1] - cheb[nc - 2];
}

// Absorption optical depth of mode m in band b for one cell: specvol the
// mode's species volumes, qaerwat the mode's water, cheb its Chebyshev
// polynomials, mass the layer's dry mass per area (calc_refin_complex,
// binterp, calc_parameterized and the product of modal_aero_lw_k)
// species volumes of mode m (specmmr / specdens, no clipping)
MAM4B_HD void mode_specvol(int m, const double (&ai)[NPOP], double (&specvol)[7]) {
  for (int s = 0; s < K::nspec(m); ++s)
    specvol[s] = ai[K::spec0(m) + s] / act::type_dens(act::spectype(m, s));
}

template <class L = LwTables>
MAM4B_HD double mode_band_tau(const double *tables, int m, int b, const double (&specvol)[7],
                              double qaerwat, const double (&cheb)[kNcoef], double mass) {
  const int nspec = K::nspec(m);
  double dryvol = 0.0, cre = 0.0, cim = 0.0;
  for (int s = 0; s < nspec; ++s) {
    dryvol += specvol[s];
    cre += specvol[s] * tld<L>(tables + L::spec_re(m, s, b));
    cim += specvol[s] * tld<L>(tables + L::spec_im(m, s, b));
  }
  double watervol = qaerwat / 1.0e3;
  double wetvol = watervol + dryvol;
  if (watervol < 0.0) {
    watervol = 0.0;
    wetvol = dryvol;
  }
  cre += watervol * tld<L>(tables + L::water_re(b));
  cim += watervol * tld<L>(tables + L::water_im(b));
  if (wetvol > 1.e-40) {
    cre /= wetvol;
    cim /= wetvol;
  }
  const double refr = cre, refi = fabs(cim);
  const double *rt = tables + L::refr(m, b);
  const double *it = tables + L::refi(m, b);
  int itab, jtab;
  double ttab, utab;
  table_factors<L>(kPrefr, refr, rt, itab, ttab);
  table_factors<L>(kPrefi, refi, it, jtab, utab);
  const double tu = ttab * utab;
  const double tuc = ttab - tu;
  const double tcuc = 1.0 - tuc - utab;
  const double tcu = utab - tu;
  const int jp1 = (jtab + 1 < kPrefi - 1) ? jtab + 1 : kPrefi - 1;
  const int ip1 = (itab + 1 < kPrefr - 1) ? itab + 1 : kPrefr - 1;
  const double *tb = tables + L::absp(m, b);
  double pabs = 0.0;
#pragma unroll
  for (int c = 0; c < kNcoef; ++c) {
    const double *tc = tb + c * kPrefr * kPrefi;
    const double coef = tcuc * tld<L>(tc + itab * kPrefi + jtab) +
                        tuc * tld<L>(tc + ip1 * kPrefi + jtab) +
                        tu * tld<L>(tc + ip1 * kPrefi + jp1) +
                        tcu * tld<L>(tc + itab * kPrefi + jp1);
    pabs = (c == 0) ? 0.5 * coef : pabs + cheb[c] * coef;
  }
  pabs *= wetvol * 1.0e3;
  pabs = dmax(0.0, pabs);
  return pabs * mass;
}

}  // namespace opt
}  // namespace mam4b

namespace mam4b {
namespace opt {

// ---------------------------------------------------------------- shortwave
// modal_aero_sw_wo_diagnostics_k (modal_aero_opt.hpp:536-747) and the mode
// sums of modal_aero_sw (:749-878). Device table layout (doubles):
constexpr int kSwBands = 14;
constexpr int kSwSpecRe = 0;                                     // [4][7][14]
constexpr int kSwSpecIm = kSwSpecRe + 4 * 7 * kSwBands;          // [4][7][14]
constexpr int kSwWaterRe = kSwSpecIm + 4 * 7 * kSwBands;         // [14]
constexpr int kSwWaterIm = kSwWaterRe + kSwBands;                // [14]
constexpr int kSwRefr = kSwWaterIm + kSwBands;                   // [4][14][7]
constexpr int kSwRefi = kSwRefr + 4 * kSwBands * kPrefr;         // [4][14][10]
constexpr int kSwTab = kNcoef * kPrefr * kPrefi;                 // one coefficient table
constexpr int kSwExt = kSwRefi + 4 * kSwBands * kPrefi;          // [4][14][5][7][10]
constexpr int kSwAbs = kSwExt + 4 * kSwBands * kSwTab;
constexpr int kSwAsm = kSwAbs + 4 * kSwBands * kSwTab;
constexpr int kSwTableDoubles = kSwAsm + 4 * kSwBands * kSwTab;
constexpr int kSwDiagBand = 9;  // visible band of the optical-depth diagnostic

// the shortwave tables of one band: in the device table, or staged in
// shared memory
struct SwTables {
  static constexpr bool kShared = false;
  MAM4B_HD static int spec_re(int m, int s, int b) { return kSwSpecRe + (m * 7 + s) * kSwBands + b; }
  MAM4B_HD static int spec_im(int m, int s, int b) { return kSwSpecIm + (m * 7 + s) * kSwBands + b; }
  MAM4B_HD static int water_re(int b) { return kSwWaterRe + b; }
  MAM4B_HD static int water_im(int b) { return kSwWaterIm + b; }
  MAM4B_HD static int refr(int m, int b) { return kSwRefr + (m * kSwBands + b) * kPrefr; }
  MAM4B_HD static int refi(int m, int b) { return kSwRefi + (m * kSwBands + b) * kPrefi; }
  MAM4B_HD static int ext(int m, int b) { return kSwExt + (m * kSwBands + b) * kSwTab; }
  MAM4B_HD static int abs_(int m, int b) { return kSwAbs + (m * kSwBands + b) * kSwTab; }
  MAM4B_HD static int asm_(int m, int b) { return kSwAsm + (m * kSwBands + b) * kSwTab; }
};
struct SwBand {
  static constexpr bool kShared = true;
  MAM4B_HD static int spec_re(int m, int s, int) { return m * 7 + s; }
  MAM4B_HD static int spec_im(int m, int s, int) { return 28 + m * 7 + s; }
  MAM4B_HD static int water_re(int) { return 56; }
  MAM4B_HD static int water_im(int) { return 57; }
  MAM4B_HD static int refr(int m, int) { return 58 + m * kPrefr; }
  MAM4B_HD static int refi(int m, int) { return 86 + m * kPrefi; }
  MAM4B_HD static int ext(int m, int) { return 126 + m * kSwTab; }
  MAM4B_HD static int abs_(int m, int) { return 126 + (4 + m) * kSwTab; }
  MAM4B_HD static int asm_(int m, int) { return 126 + (8 + m) * kSwTab; }
};
constexpr int kSwBandDoubles = 126 + 12 * kSwTab;  // 4,326

// surface-mode radius, its log (method 1: log of the radius) and the
// Chebyshev polynomials (modal_size_parameters)
MAM4B_HD void mode_cheb_sw(int m, double dgn_w, double &radsurf, double &logradsurf,
                           double (&cheb)[kNcoef]) {
  const double xrmin = log(0.01e-6), xrmax = log(25.e-6);
  const double alnsg = log(K::sig(m));
  const double explnsigma = exp(2.0 * alnsg * alnsg);
  radsurf = 0.5 * dgn_w * explnsigma;
  logradsurf = log(radsurf);
  double xrad = bound(xrmin, xrmax, logradsurf);
  xrad = (2.0 * xrad - xrmax - xrmin) / (xrmax - xrmin);
  cheb[0] = 1.0;
  cheb[1] = xrad;
#pragma unroll
  for (int nc = 2; nc < kNcoef; ++nc)
    cheb[nc] = 2.0 * xrad * cheb[nc - 1] - cheb[nc - 2];
}

// bilinear weights of the three coefficient tables of (m, b)
template <class L = SwTables>
MAM4B_HD void sw_coefs(const double *tables, int m, int b, double refr, double refi,
                       double (&cext)[kNcoef], double (&cabs)[kNcoef],
                       double (&casm)[kNcoef]) {
  const double *rt = tables + L::refr(m, b);
  const double *it = tables + L::refi(m, b);
  int itab, jtab;
  double ttab, utab;
  table_factors<L>(kPrefr, refr, rt, itab, ttab);
  table_factors<L>(kPrefi, refi, it, jtab, utab);
  const double tu = ttab * utab;
  const double tuc = ttab - tu;
  const double tcuc = 1.0 - tuc - utab;
  const double tcu = utab - tu;
  const int jp1 = (jtab + 1 < kPrefi - 1) ? jtab + 1 : kPrefi - 1;
  const int ip1 = (itab + 1 < kPrefr - 1) ? itab + 1 : kPrefr - 1;
#pragma unroll
  for (int c = 0; c < kNcoef; ++c) {
    const int o = c * kPrefr * kPrefi;
    const double *e = tables + L::ext(m, b) + o, *a = tables + L::abs_(m, b) + o,
                 *s = tables + L::asm_(m, b) + o;
    cext[c] = tcuc * tld<L>(e + itab * kPrefi + jtab) + tuc * tld<L>(e + ip1 * kPrefi + jtab) +
              tu * tld<L>(e + ip1 * kPrefi + jp1) + tcu * tld<L>(e + itab * kPrefi + jp1);
    cabs[c] = tcuc * tld<L>(a + itab * kPrefi + jtab) + tuc * tld<L>(a + ip1 * kPrefi + jtab) +
              tu * tld<L>(a + ip1 * kPrefi + jp1) + tcu * tld<L>(a + itab * kPrefi + jp1);
    casm[c] = tcuc * tld<L>(s + itab * kPrefi + jtab) + tuc * tld<L>(s + ip1 * kPrefi + jtab) +
              tu * tld<L>(s + ip1 * kPrefi + jp1) + tcu * tld<L>(s + itab * kPrefi + jp1);
  }
}

MAM4B_HD double cheb_eval(const double (&coef)[kNcoef], const double (&cheb)[kNcoef]) {
  double p = 0.5 * coef[0];
#pragma unroll
  for (int nc = 1; nc < kNcoef; ++nc)
    p += cheb[nc] * coef[nc];
  return p;
}

// optical depth, single-scattering and asymmetry products of mode m in
// band b for one cell: out = {tauxar, wa, ga, fa}
template <class L = SwTables>
MAM4B_HD void mode_band_sw(const double *tables, int m, int b, const double (&specvol)[7],
                           double qaerwat, const double (&cheb)[kNcoef], double radsurf,
                           double logradsurf, double mass, double (&out)[4]) {
  const int nspec = K::nspec(m);
  double dryvol = 0.0;
  for (int s = 0; s < nspec; ++s)
    dryvol += specvol[s];
  if (dryvol < 0.0 && dryvol > -1.e-16) {
    out[0] = out[1] = out[2] = out[3] = 0.0;
    return;
  }
  // calc_refin_complex (shortwave)
  double dv = 0.0, cre = 0.0, cim = 0.0;
  for (int s = 0; s < nspec; ++s) {
    dv += specvol[s];
    cre += specvol[s] * tld<L>(tables + L::spec_re(m, s, b));
    cim += specvol[s] * tld<L>(tables + L::spec_im(m, s, b));
  }
  double watervol = qaerwat / 1.0e3;
  double wetvol = watervol + dv;
  if (watervol < 0.0) {
    watervol = 0.0;
    wetvol = dv;
  }
  cre += watervol * tld<L>(tables + L::water_re(b));
  cim += watervol * tld<L>(tables + L::water_im(b));
  const double den = dmax(wetvol, 1.e-40);
  cre /= den;
  cim /= den;
  double cext[kNcoef], cabs[kNcoef], casm[kNcoef];
  sw_coefs<L>(tables, m, b, cre, fabs(cim), cext, cabs, casm);
  double pext = cheb_eval(cext, cheb);
  double pabs = cheb_eval(cabs, cheb);
  const double pasm = cheb_eval(casm, cheb);
  const double xrmax = log(25.e-6);
  if (logradsurf <= xrmax)
    pext = exp(pext);
  else
    pext = 1.5 / (radsurf * 1.0e3);
  pext *= wetvol * 1.0e3;
  pabs *= wetvol * 1.0e3;
  pabs = bound(0.0, pext, pabs);
  const double palb = 1.0 - pabs / dmax(pext, 1.e-40);
  const double dopaer = pext * mass;
  out[0] = dopaer;
  out[1] = dopaer * palb;
  out[2] = dopaer * palb * pasm;
  out[3] = dopaer * palb * pasm * pasm;
}

#ifdef __CUDACC__
// Band b's values of the refractive-index mixing and the tables of the
// four modes, copied from the device table (layout G) into the block's
// shared slice s (layout S) by all threads of the block; the caller
// synchronises the block before reading s.
template <class G, class S>
__device__ void stage_band_common(const double *g, int b, double *s) {
  const int t = threadIdx.x, nt = blockDim.x;
  for (int i = t; i < 28; i += nt) {
    const int m = i / 7, k = i % 7;
    s[S::spec_re(m, k, b)] = __ldg(g + G::spec_re(m, k, b));
    s[S::spec_im(m, k, b)] = __ldg(g + G::spec_im(m, k, b));
  }
  if (t == 0) {
    s[S::water_re(b)] = __ldg(g + G::water_re(b));
    s[S::water_im(b)] = __ldg(g + G::water_im(b));
  }
  for (int i = t; i < 4 * kPrefr; i += nt)
    s[S::refr(i / kPrefr, b) + i % kPrefr] = __ldg(g + G::refr(i / kPrefr, b) + i % kPrefr);
  for (int i = t; i < 4 * kPrefi; i += nt)
    s[S::refi(i / kPrefi, b) + i % kPrefi] = __ldg(g + G::refi(i / kPrefi, b) + i % kPrefi);
}

__device__ void stage_lw_band(const double *g, int b, double *s) {
  stage_band_common<LwTables, LwBand>(g, b, s);
  constexpr int kT = kNcoef * kPrefr * kPrefi;
  for (int i = threadIdx.x; i < 4 * kT; i += blockDim.x)
    s[LwBand::absp(i / kT, b) + i % kT] = __ldg(g + LwTables::absp(i / kT, b) + i % kT);
}

__device__ void stage_sw_band(const double *g, int b, double *s) {
  stage_band_common<SwTables, SwBand>(g, b, s);
  for (int i = threadIdx.x; i < 4 * kSwTab; i += blockDim.x) {
    const int m = i / kSwTab, k = i % kSwTab;
    s[SwBand::ext(m, b) + k] = __ldg(g + SwTables::ext(m, b) + k);
    s[SwBand::abs_(m, b) + k] = __ldg(g + SwTables::abs_(m, b) + k);
    s[SwBand::asm_(m, b) + k] = __ldg(g + SwTables::asm_(m, b) + k);
  }
}
#endif

}  // namespace opt
}  // namespace mam4b

// ---- radiation-facing optics: the tropopause and the volcanic (CMIP6)
// stratospheric aerosol, aero_rad_props (src/mam4xx/aero_rad_props.hpp).
namespace mam4b {
namespace rad {

// R/cp of dry air and -g/R_dry (tropopause.hpp:17-30, mam4_constants.hpp)
constexpr double kRgas = 6.022214076e23 * 1.380649e-23;
constexpr double kKap = ((kRgas * 1e3) / (0.028966 * 1e3)) / 1.00464e3;
constexpr double kFaktor = -9.80616 / (kRgas / 0.028966);
constexpr double kKa1 = kKap - 1.0;

// lapse rate and mean temperature between two levels in p^kappa
// (get_dtdz, tropopause.hpp:34-55)
MAM4B_HD void lapse_rate(double pm, double pmk, double p_up, double p_down, double t_up,
                         double t_down, double &dtdz, double &tm) {
  const double a1 = (t_up - t_down) / (pow(p_up, kKap) - pow(p_down, kKap));
  const double b1 = t_down - a1 * pow(p_down, kKap);
  tm = a1 * pmk + b1;
  const double dtdp = a1 * kKap * (pow(pm, kKa1));
  dtdz = kFaktor * dtdp * pm / tm;
}

// The lapse-rate quantities of the layer between levels k - 1 and k
// (k >= 1): mean p^kappa, mean pressure, dT/dz and mean temperature, as
// twmo computes them for its scan (tropopause.hpp:114-119, 124-129,
// 171-188); the same values wherever the scan asks for them.
struct LapsePair {
  double pmk, pm, dtdz, tm;
};
template <class ColT, class ColP>
MAM4B_HD LapsePair lapse_pair(const ColT &temp, const ColP &pmid, int k) {
  LapsePair q;
  q.pmk = 0.5 * (pow(pmid(k - 1), kKap) + pow(pmid(k), kKap));
  q.pm = pow(q.pmk, (1.0 / kKap));
  lapse_rate(q.pm, q.pmk, pmid(k - 1), pmid(k), temp(k - 1), temp(k), q.dtdz, q.tm);
  return q;
}

// WMO lapse-rate tropopause of a column (twmo, Reichler et al. 2003;
// tropopause.hpp:81-204) from its layers' lapse-rate quantities pair(k),
// k = 1 .. nlev-1: scanning up from the surface, the first layer where the
// lapse rate falls below 2 K/km, between 75 and 450 hPa, and stays below
// it on average over the 2 km above. Returns its pressure, or -99 when
// there is none.
template <class Pairs>
MAM4B_HD double twmo_from_pairs(const Pairs &pair, int nlev) {
  const double gam = -0.002, plimu = 45000, pliml = 7500, deltaz = 2000.0;
  LapsePair cur = pair(nlev - 1);
  for (int k = nlev - 2; k >= 1; --k) {
    const double pmk0 = cur.pmk, dtdz0 = cur.dtdz;
    cur = pair(k);
    const double pmk = cur.pmk, pm = cur.pm, dtdz = cur.dtdz, tm = cur.tm;
    if (dtdz <= gam || pm > plimu)
      continue;
    double ptph;
    if (dtdz0 < gam) {
      const double ag = (dtdz - dtdz0) / (pmk - pmk0);
      const double bg = dtdz0 - (ag * pmk0);
      ptph = exp(log((gam - bg) / ag) / kKap);
    } else {
      ptph = pm;
    }
    if (ptph < pliml || ptph > plimu)
      continue;
    const double p2km = ptph + deltaz * (pm / tm) * kFaktor;
    double asum = 0.0;
    int icount = 0;
    for (int j = k; j >= 1; --j) {
      const LapsePair up = pair(j);
      if (up.pm > ptph)
        continue;
      if (up.pm < p2km)
        return ptph;  // the layer above stays stable: tropopause found
      asum += up.dtdz;
      icount++;
      const double aquer = asum / double(icount);
      if (aquer <= gam)
        break;  // not stable enough above: try the next level up
    }
  }
  return -99.0;
}

// tropopause_twmo's level search (tropopause.hpp:222-231) for tropopause
// pressure tp: the level k in [2, nlev-1], scanning up, whose upper
// interface pressure pint(k) lies at or below tp; 0 when tp is not
// positive or no level qualifies.
template <class ColI>
MAM4B_HD int tropopause_level_at(double tp, const ColI &pint, int nlev) {
  if (tp > 0) {
    for (int k = nlev - 1; k > 1; --k)
      if (tp >= pint(k))
        return k;
  }
  return 0;
}

// tropopause_twmo (tropopause.hpp:210-233) of one column, serially.
template <class ColT, class ColP, class ColI>
MAM4B_HD int tropopause_level(const ColT &temp, const ColP &pmid, const ColI &pint, int nlev) {
  auto pair = [&](int k) { return lapse_pair(temp, pmid, k); };
  return tropopause_level_at(twmo_from_pairs(pair, nlev), pint, nlev);
}

}  // namespace rad
}  // namespace mam4b
