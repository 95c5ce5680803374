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

// position of ref in a table: index of the bracket and the fraction
// (compute_factors)
MAM4B_HD void table_factors(int n, double ref, const double *tab, int &ix, double &tt) {
  ix = 1;
  tt = 0.0;
  if (n > 1) {
    int ii = 0;
    for (ii = 0; ii < n; ++ii)
      if (ref < MAM4B_LDG(tab + ii))
        break;
    ix = (ii - 1 > 0) ? ii - 1 : 0;
    const int ip1 = (ix + 1 < n - 1) ? ix + 1 : n - 1;
    const double dx = MAM4B_LDG(tab + ip1) - MAM4B_LDG(tab + ix);
    if (fabs(dx) > 1.e-20)
      tt = (ref - MAM4B_LDG(tab + ix)) / dx;
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

MAM4B_HD double mode_band_tau(const double *tables, int m, int b, const double (&specvol)[7],
                              double qaerwat, const double (&cheb)[kNcoef], double mass) {
  const int nspec = K::nspec(m);
  double dryvol = 0.0, cre = 0.0, cim = 0.0;
  for (int s = 0; s < nspec; ++s) {
    dryvol += specvol[s];
    cre += specvol[s] * MAM4B_LDG(tables + kSpecRe + (m * 7 + s) * kLwBands + b);
    cim += specvol[s] * MAM4B_LDG(tables + kSpecIm + (m * 7 + s) * kLwBands + b);
  }
  double watervol = qaerwat / 1.0e3;
  double wetvol = watervol + dryvol;
  if (watervol < 0.0) {
    watervol = 0.0;
    wetvol = dryvol;
  }
  cre += watervol * MAM4B_LDG(tables + kWaterRe + b);
  cim += watervol * MAM4B_LDG(tables + kWaterIm + b);
  if (wetvol > 1.e-40) {
    cre /= wetvol;
    cim /= wetvol;
  }
  const double refr = cre, refi = fabs(cim);
  const double *rt = tables + kRefr + (m * kLwBands + b) * kPrefr;
  const double *it = tables + kRefi + (m * kLwBands + b) * kPrefi;
  int itab, jtab;
  double ttab, utab;
  table_factors(kPrefr, refr, rt, itab, ttab);
  table_factors(kPrefi, refi, it, jtab, utab);
  const double tu = ttab * utab;
  const double tuc = ttab - tu;
  const double tcuc = 1.0 - tuc - utab;
  const double tcu = utab - tu;
  const int jp1 = (jtab + 1 < kPrefi - 1) ? jtab + 1 : kPrefi - 1;
  const int ip1 = (itab + 1 < kPrefr - 1) ? itab + 1 : kPrefr - 1;
  const double *tb = tables + kAbsp + (m * kLwBands + b) * kNcoef * kPrefr * kPrefi;
  double pabs = 0.0;
#pragma unroll
  for (int c = 0; c < kNcoef; ++c) {
    const double *tc = tb + c * kPrefr * kPrefi;
    const double coef = tcuc * MAM4B_LDG(tc + itab * kPrefi + jtab) +
                        tuc * MAM4B_LDG(tc + ip1 * kPrefi + jtab) +
                        tu * MAM4B_LDG(tc + ip1 * kPrefi + jp1) +
                        tcu * MAM4B_LDG(tc + itab * kPrefi + jp1);
    pabs = (c == 0) ? 0.5 * coef : pabs + cheb[c] * coef;
  }
  pabs *= wetvol * 1.0e3;
  pabs = dmax(0.0, pabs);
  return pabs * mass;
}

}  // namespace opt
}  // namespace mam4b
