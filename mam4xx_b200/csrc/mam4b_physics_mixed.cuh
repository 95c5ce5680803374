// mam4b_physics_mixed.cuh -- FP32 forms of the bulk of the microphysics
// step for the mixed-precision path (MAM4B_MIXED).
//
// In FP32: water uptake (dry/wet size, Kohler equilibrium), the per-particle
// H2SO4 uptake coefficients, the Brownian coagulation coefficients and the
// SOA gas-particle sub-stepping. In FP64 (the double-precision functions of
// mam4b_physics.cuh): calcsize, the H2SO4 implicit exponential update, the
// renaming transfer fractions, the nucleation rate fits (their polynomials
// in T cancel to a few digits), aging and every state update and sum that
// carries species mass.
//
// The formulas are those of the reference routines cited with each
// function; where FP32 would underflow or lose the root, the same quantity
// is computed from rescaled variables (stated at the function).
#pragma once

#include "mam4b_physics.cuh"

namespace mam4b {
namespace f32 {

__device__ __forceinline__ float fmx(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float fmn(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float fbound(float lo, float hi, float x) { return fmx(lo, fmn(hi, x)); }
__device__ __forceinline__ float fcube(float x) { return x * x * x; }

// ------------------------------------------------------------ water uptake
// The Kohler wet radius (makoh_quartic / find_real_solution,
// water_uptake.hpp:101-171: the smallest real root x >= r_dry of
// x^4 + p43 x^3 + p41 x + p40, p43 = -aa/ln S, p41 = r^3 (hygro/ln S - 1),
// p40 = aa r^3/ln S) in the variable z = x / r_dry - 1:
//   g(z) = z^4 + (4 + a) z^3 + (6 + 3a) z^2 + (3 + 3a + h) z + h,
//   a = aa / (-ln S r_dry) > 0,  h = hygro / ln S < 0,
// so g(0) = h < 0 and g'' > 0 for z > -1: g has exactly one root above 0,
// the reference's root. Newton's method from an upper bound zhi with
// g(zhi) > 0 decreases monotonically to it. Solving for z rather than for
// x / r_dry keeps the water volume r^3 ((1 + z)^3 - 1) accurate when the
// particle barely grows (hygroscopicity ~1e-10 for BC/POM), and avoids the
// closed-form quartic, whose cancellations leave single precision without
// a real root in some cells. At most 6 steps on the workloads.
__device__ __forceinline__ float kohler_growth(float a, float h) {
  const float c3 = 4.0f + a, c2 = 6.0f + 3.0f * a, c1 = 3.0f + 3.0f * a + h;
  // (1 + zhi)^3 >= |h - 1| + a and 1 + zhi >= 1 bound the root from above
  float z = fmx(1.0f, cbrtf(fabsf(h - 1.0f) + a)) * 1.0001f + 1.0e-3f - 1.0f;
  if (z > 999.0f) {
    // the reference keeps 1000 r_dry when no root lies below it
    const float y = 999.0f;
    if ((((y + c3) * y + c2) * y + c1) * y + h <= 0.0f)
      return y;
  }
  for (int it = 0; it < 40; ++it) {
    const float gz = (((z + c3) * z + c2) * z + c1) * z + h;
    const float dg = ((4.0f * z + 3.0f * c3) * z + 2.0f * c2) * z + c1;
    const float d = gz / dg;
    z -= d;
    if (fabsf(d) <= 1.0e-6f * z)
      break;
  }
  return z;
}

// modal_aero_kohler (water_uptake.hpp:180-230) as growth z = r_wet/r_dry - 1
// (r_wet capped at 30 um as in the reference); rdry in m.
__device__ __forceinline__ float kohler_z(float aa, float rdry_in, float hygro, float rh) {
  const float eps = 1e-4f;
  const float rdry = rdry_in * 1.e6f;
  const float ss = fbound(1.e-10f, 1.0f - eps, rh);
  const float slog = logf(ss);
  const float pp = fabsf(rdry * hygro / aa);
  float z;
  if (pp < eps)
    z = pp * (1.0f / 3.0f) / (1.0f - slog * rdry / aa);
  else
    z = kohler_growth(-aa / (slog * rdry), hygro / slog);
  return fmn(z, 30.0f / rdry - 1.0f);
}

// Water uptake of one mode (water_uptake.hpp:73-480), as
// water_uptake_mode<M> of the double-precision path.
template <int M>
__device__ __forceinline__ void water_uptake_mode(const StepConsts &C, const float (&sp)[7],
                                                  double rh64, float dgn_a, float &dgn_awet,
                                                  float &qaerwat, float &wetdens) {
  const float pi = (float)K::pi;
  const float rh = (float)rh64;
  float hygro = 0.0f, dryvolmr = 0.0f, maer = 0.0f;
#pragma unroll
  for (int s = 0; s < K::nspec(M); ++s) {
    const int w = K::spec0(M) + s - M;
    const float raer = sp[s];
    const float vol_tmp = raer / (float)K::wu_dens(w);
    maer += raer;
    dryvolmr += vol_tmp;
    hygro += vol_tmp * (float)K::wu_hygro(w);
  }
  const int w0 = K::spec0(M) - M;
  hygro = (dryvolmr > 1e-30f) ? hygro / dryvolmr : (float)K::wu_hygro(w0);
  const float ls = (float)C.log_sig[M];
  // dry volume of one particle; its inverse is the number per dry volume
  const float dryvol = (pi / 6.0f) * fcube(dgn_a) * expf(4.5f * ls * ls);
  const float naer = dryvolmr / dryvol;
  const float drydens = (maer > 1e-31f) ? maer / dryvolmr : 1.0f;
  const float drymass = drydens * dryvol;
  const float dryrad = 0.5f * dgn_a * expf(1.5f * ls * ls);
  // growth z >= 0: wet radius dryrad (1 + z), water dryvol ((1 + z)^3 - 1)
  float z = fmx(kohler_z((float)C.kohler_aa, dryrad, hygro, rh), 0.0f);
  float wtrvol = dryvol * (z * (3.0f + z * (3.0f + z)));
  // the hysteresis thresholds compare the double-precision humidity
  if (rh64 < K::rh_cryst) {
    z = 0.0f;
    wtrvol = 0.0f;
  } else if (rh64 < K::rh_deliq) {
    wtrvol = fmx(wtrvol * (float)(C.hystfac * (rh64 - K::rh_cryst)), 0.0f);
    z = cbrtf(1.0f + wtrvol / dryvol) - 1.0f;
  }
  const float wetvol = dryvol + wtrvol;
  dgn_awet = dgn_a * (1.0f + z);
  qaerwat = 1.0e3f * naer * wtrvol;
  wetdens = (wetvol > 1.0e-30f) ? (drymass + 1.0e3f * wtrvol) / wetvol : (float)K::wu_dens(w0);
}

// Per-particle H2SO4 uptake rate of mode n (gasaerexch.hpp:255-353)
__device__ __forceinline__ float uptake_rate_mode(const StepConsts &C, int n, float gasdiffus,
                                                  float freepath, float dgn_awet) {
  const float tworootpi = 2.0f * sqrtf((float)K::pi);
  const float root2 = 1.41421356f;
  const float xg = 0.70710677f, wg = 0.88622695f;
  const float a283 = 0.65f * 0.283f, a75 = 0.65f * 0.75f;
  const float lnsg = (float)C.log_sig[n];
  const float lndpgn = logf(dgn_awet);
  const float kn = 2.0f * freepath / dgn_awet;
  const float tmpa = 1.0f / (1.0f + kn) - (2.0f * kn + 1.0f + a283) / (kn * (kn + 1.0f + a283) + a75);
  const float beta = fmx(1.0f, fmn(2.0f, 1.0f - kn * tmpa));
  const float bl = beta * lnsg;
  const float constant = tworootpi * expf(beta * lndpgn + 0.5f * bl * bl);
  float sum = 0.0f;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const float lndp = lndpgn + beta * lnsg * lnsg + root2 * lnsg * (q == 0 ? xg : -xg);
    const float dp = expf(lndp);
    const float knq = 2.0f * freepath / dp;
    const float hh = (a75 * (1.0f + knq)) / (knq * (knq + 1.0f + a283) + a75);
    // dp / dp^beta = exp((1 - beta) ln dp)
    sum += wg * hh * expf((1.0f - beta) * lndp);
  }
  return constant * gasdiffus * sum;
}

// ------------------------------------------------------------ coagulation
// getcoags (coagulation.hpp:651-817) for one mode pair, times aircon.
// The third-moment rates are formed without the factor dg_src^3, which
// cancels in bij3 = qv12 / (dg_src^3 exp(4.5 ln^2 sg_src)) and would take
// the intermediate products below the single-precision range.
__device__ __forceinline__ void coag_pair_coefs(const StepConsts &C, const CoagTables &T, int p,
                                                float airtemp, float airprs, float aircon,
                                                float dgatk, float dgacc, float pdensat,
                                                float pdensac, float &bij0, float &bij3,
                                                float &bii0, float &bjj0) {
  const int sm = coag_src(p), dm = coag_dst(p);
  const float sgatk = (float)K::sig(sm), sgacc = (float)K::sig(dm);
  const float xxlsgat = (float)C.log_sig[sm], xxlsgac = (float)C.log_sig[dm];
  const float t0 = 273.15f + 15.0f;
  const float sqrt_temp = sqrtf(airtemp);
  const float lamda = 6.6328e-8f * 101325.0f * airtemp / (t0 * airprs);
  const float amu = 1.458e-6f * airtemp * sqrt_temp / (airtemp + 110.4f);
  const float boltzmann = 1.38065e-23f;
  const float knc = (2.0f / 3.0f) * boltzmann * airtemp / amu;
  const float kfmat = sqrtf(3.0f * boltzmann * airtemp / pdensat);
  const float kfmac = sqrtf(3.0f * boltzmann * airtemp / pdensac);
  const float kfmatac = sqrtf(6.0f * boltzmann * airtemp / (pdensat + pdensac));
  const float a = 1.246f;
  const float esat01 = expf(0.125f * xxlsgat * xxlsgat);
  const float esac01 = expf(0.125f * xxlsgac * xxlsgac);
  const float esat04 = (esat01 * esat01) * (esat01 * esat01);
  const float esac04 = (esac01 * esac01) * (esac01 * esac01);
  const float esat05 = esat04 * esat01, esac05 = esac04 * esac01;
  const float esat08 = esat04 * esat04, esac08 = esac04 * esac04;
  const float esat09 = esat08 * esat01, esac09 = esac08 * esac01;
  const float esat16 = esat08 * esat08, esac16 = esac08 * esac08;
  const float esat20 = esat16 * esat04, esac20 = esac16 * esac04;
  const float esat24 = esat20 * esat04;
  const float esat25 = esat20 * esat05, esac25 = esac20 * esac05;
  const float esat36 = esat20 * esat16;
  const float esat49 = esat24 * esat25;
  const float esat64 = esat20 * esat20 * esat24;
  const float esat100 = esat64 * esat36;
  const float sqdgat = sqrtf(dgatk), sqdgac = sqrtf(dgacc);
  const float r1 = sqdgac / sqdgat;
  const float r2 = r1 * r1;
  const float rx4 = r2 * r2;
  const float ri1 = 1.0f / r1;
  const float ri2 = 1.0f / (r1 * r1);
  const float ri3 = 1.0f / (r1 * r1 * r1);
  const float kngat = 2.0f * lamda / dgatk;
  const float kngac = 2.0f * lamda / dgacc;
  const float rat = dgacc / dgatk;
  const float dlgsqt2 = 1.0f / logf(sqrtf(2.0f));
  const int n2n = (int)fmx(1.0f, fmn(10.0f, roundf(4.0f * (sgatk - 0.75f)))) - 1;
  const int n2a = (int)fmx(1.0f, fmn(10.0f, roundf(4.0f * (sgacc - 0.75f)))) - 1;
  const int n1 = (int)fmx(1.0f, fmn(10.0f, 1.0f + roundf(dlgsqt2 * logf(rat)))) - 1;
  const int tix = n1 * 100 + n2n * 10 + n2a;
  const float bm0ij = (float)__ldg(T.bm0ij + tix);
  const float bm3i = (float)__ldg(T.bm3i + tix);
  const float coagnc0 = knc * (2.0f + a * (kngat * (esat04 + r2 * esat16 * esac04) +
                                           kngac * (esac04 + ri2 * esac16 * esat04)) +
                               (r2 + ri2) * esat04 * esac04);
  const float coagfm0 = kfmatac * sqdgat * bm0ij *
                        (esat01 + r1 * esac01 + 2.0f * r2 * esat01 * esac04 +
                         rx4 * esat09 * esac16 + ri3 * esat16 * esac09 + 2.0f * ri1 * esat04 +
                         esac01);
  const float qn12 = coagnc0 * coagfm0 / (coagnc0 + coagfm0);
  // coagnc3 / dg^3 and coagfm3 / dg^3
  const float nc3 = knc * (2.0f * esat36 + a * kngat * (esat16 + r2 * esat04 * esac04) +
                           a * kngac * (esat36 * esac04 + ri2 * esat64 * esac16) +
                           r2 * esat16 * esac04 + ri2 * esat64 * esac04);
  const float fm3 = kfmatac * sqdgat * bm3i *
                    (esat49 + r1 * esat36 * esac01 + 2.0f * r2 * esat25 * esac04 +
                     rx4 * esat09 * esac16 + ri3 * esat100 * esac09 + 2.0f * ri1 * esat64 * esac01);
  const float qv12_dg3 = nc3 * fm3 / (nc3 + fm3);
  const float cnc11 = knc * (1.0f + esat08 + a * kngat * (esat20 + esat04));
  const float cfm11 = kfmat * sqdgat * (float)__ldg(T.bm0 + n2n) * (esat01 + esat25 + 2.0f * esat05);
  const float qn11 = cfm11 * cnc11 / (cfm11 + cnc11);
  const float cnc22 = knc * (1.0f + esac08 + a * kngac * (esac20 + esac04));
  const float cfm22 = kfmac * sqdgac * (float)__ldg(T.bm0 + n2a) * (esac01 + esac25 + 2.0f * esac05);
  const float qn22 = cfm22 * cnc22 / (cfm22 + cnc22);
  bii0 = fmx(0.0f, qn11) * aircon;
  bjj0 = fmx(0.0f, qn22) * aircon;
  bij0 = fmx(0.0f, qn12) * aircon;
  bij3 = fmx(0.0f, qv12_dg3 / expf(4.5f * xxlsgat * xxlsgat)) * aircon;
}

// ------------------------------------------------- SOA sub-stepping, mixed
// mam_soaexch_1subarea (gasaerexch_soaexch.hpp:80-341) for MAM4B_MIXED:
// every value in double precision (state, saturation ratios, departures
// phi, step control, the semi-implicit update), as in the FP64 loop, but
// without IEEE divisions and with fused multiply-adds:
//  * each quotient x / d is x * rcp(d), rcp the hardware's approximate
//    double reciprocal refined by two Newton-Raphson steps (mx::rcp), one
//    reciprocal shared by the three quotients over 1 + beta sat;
//  * the products that feed a sum are fused with it (__fma_rn).
// The results differ from the FP64 loop's by rounding only (a few ulps per
// pass), so the loop takes the FP64 loop's sub-steps except where a step
// decision sits within rounding of its threshold. No value changes type:
// conversions between double and float issue at a quarter of the FP64 rate
// on this GPU, so a loop that mixes the two types is no faster.
// Conservation: the update conserves g + sum a for any values of r, as the
// same r enter the sums and the particle update.
namespace mx {
// 1 / d for a positive, normal d without a division: the special-function
// unit's approximate reciprocal (PTX rcp.approx.ftz.f64) and two steps of
// Newton's iteration for 1/d, r <- r + r (1 - d r), each of which squares
// the relative error; the result is within a few ulps of 1 / d.
__device__ __forceinline__ double rcp(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = __fma_rn(-d, r, 1.0);
  r = __fma_rn(r, e, r);
  e = __fma_rn(-d, r, 1.0);
  return __fma_rn(r, e, r);
}
}  // namespace mx

__device__ __forceinline__ bool soa_step_mx(SoaState &st) {
  if (!(st.tcur < st.dtfull - 1.0e-3))
    return false;
  st.niter++;
  if (st.niter > 1000)
    return false;
  double g_soa = dmax(st.g, 0.0);
  double tot_soa = g_soa;
  double a_soa[NMODE], sat[NMODE], g_star[NMODE];
  bool skip[NMODE];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    skip[n] = !(st.uptk[n] > 1.0e-15);
    a_soa[n] = skip[n] ? 0.0 : dmax(st.a[n], 0.0);
    tot_soa += a_soa[n];
  }
  double tmpb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    // both denominators are at least 1e-20: normal numbers
    sat[n] = st.g0 * mx::rcp(dmax(st.opoa[n] + a_soa[n], 1.0e-20));
    g_star[n] = sat[n] * a_soa[n];
    const double phi = (g_soa - g_star[n]) * mx::rcp(dmax(g_soa, dmax(g_star[n], 1.0e-20)));
    tmpb = __fma_rn(st.uptk[n], fabs(phi), tmpb);
  }
  const double tmpa = dmax(0.0, tmpb);
  double dtcur;
  const double dtmax = st.dtfull - st.tcur;
  if (dtmax * tmpa <= 0.05) {
    dtcur = dtmax;
    st.tcur = st.dtfull;
  } else {
    // tmpa > 0.05 / dtmax here
    dtcur = 0.05 * mx::rcp(tmpa);
    st.tcur += dtcur;
  }
  double beta[NMODE], r[NMODE], ta = 0.0, tb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    beta[n] = dtcur * st.uptk[n];
    const double del_g = g_soa - g_star[n];
    if (del_g > 0.0)
      sat[n] = st.g0 * mx::rcp(dmax(st.opoa[n] + __fma_rn(beta[n], del_g, a_soa[n]), 1.0e-20));
    // 1 + beta sat >= 1
    r[n] = mx::rcp(__fma_rn(beta[n], sat[n], 1.0));
    ta = __fma_rn(a_soa[n], r[n], ta);
    tb = __fma_rn(beta[n], r[n], tb);
  }
  g_soa = dmax(0.0, (tot_soa - ta) * mx::rcp(1.0 + tb));
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    st.a[n] = skip[n] ? 0.0 : __fma_rn(beta[n], g_soa, a_soa[n]) * r[n];
  st.g = g_soa;
  return true;
}

// ------------------------------------------------------- SOA sub-stepping
// mam_soaexch_1subarea (gasaerexch_soaexch.hpp:80-341) in single
// precision with approximate division (__fdividef, 2 ulp) and one
// reciprocal per mode for the three quotients sharing 1 + beta*sat; the time
// bookkeeping (elapsed time, step count) stays double so that the loop
// ends where the double-precision loop would.
struct SoaStateF {
  float g, a[NMODE], opoa[NMODE], uptk[NMODE], g0;
  double tcur, dtfull;
  int niter;
};

__device__ __forceinline__ bool soa_step(SoaStateF &st) {
  if (!(st.tcur < st.dtfull - 1.0e-3))
    return false;
  st.niter++;
  if (st.niter > 1000)
    return false;
  float g_soa = fmx(st.g, 0.0f);
  float tot_soa = g_soa;
  float a_soa[NMODE], sat[NMODE], g_star[NMODE], beta[NMODE];
  bool skip[NMODE];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    skip[n] = !(st.uptk[n] > 1.0e-15f);
    a_soa[n] = skip[n] ? 0.0f : fmx(st.a[n], 0.0f);
    tot_soa += a_soa[n];
  }
  float tmpb = 0.0f;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    sat[n] = __fdividef(st.g0, fmx(st.opoa[n] + a_soa[n], 1.0e-20f));
    g_star[n] = sat[n] * a_soa[n];
    const float phi = __fdividef(g_soa - g_star[n], fmx(g_soa, fmx(g_star[n], 1.0e-20f)));
    tmpb += st.uptk[n] * fabsf(phi);
  }
  const double dtmax = st.dtfull - st.tcur;
  float dtcur;
  if (dtmax * (double)tmpb <= 0.05) {
    dtcur = (float)dtmax;
    st.tcur = st.dtfull;
  } else {
    dtcur = __fdividef(0.05f, tmpb);
    st.tcur += (double)dtcur;
  }
  float ta = 0.0f, tb = 0.0f, den[NMODE];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    beta[n] = dtcur * st.uptk[n];
    const float del_g = g_soa - g_star[n];
    if (del_g > 0.0f)
      sat[n] = __fdividef(st.g0, fmx(st.opoa[n] + (a_soa[n] + beta[n] * del_g), 1.0e-20f));
    den[n] = __fdividef(1.0f, 1.0f + beta[n] * sat[n]);
    ta += a_soa[n] * den[n];
    tb += beta[n] * den[n];
  }
  g_soa = fmx(0.0f, __fdividef(tot_soa - ta, 1.0f + tb));
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    st.a[n] = skip[n] ? 0.0f : (a_soa[n] + beta[n] * g_soa) * den[n];
  st.g = g_soa;
  return true;
}

}  // namespace f32
}  // namespace mam4b
