/*
 * mam4_oracle.c -- CPU restatement of the mam4xx microphysics step.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA path is compared
 * with (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline leg). It is
 * never linked into, loaded by or called from the product library.
 *
 * Plain C99, double precision, glibc libm; compiled with -ffp-contract=off
 * so that every expression rounds in the order written. Each function
 * restates one mam4xx routine (file:line relative to the mam4xx tree) and
 * keeps its order of operations, so the restatement can be checked bit for
 * bit against the reference headers compiled in oracle/_ref.
 *
 * Parity is pinned by: the 30 H2SO4 known-answer vectors of
 * src/tests/mam4_gasaerexch_unit_tests.cpp, the coagulation table values of
 * src/tests/mam4_coagulation_unit_tests.cpp, the aging transfer tests of
 * src/tests/mam4_aging_unit_tests.cpp, and stage-by-stage comparison with
 * the reference headers compiled unchanged (oracle/_ref).
 *
 * Complex arithmetic in the water-uptake quartic follows Kokkos::complex
 * (Kokkos 4.x Kokkos_Complex.hpp): textbook product, quotient scaled by the
 * 1-norm of the divisor, abs = hypot, sqrt by the half-angle formula and
 * pow(z, y) = polar(pow(|z|, y), y*atan2(im, re)).
 */
#include <float.h>
#include <math.h>
#include <string.h>

#include "oracle_api.h"

#ifdef _OPENMP
#include <omp.h>
#endif

/* The same source compiles for the host (gcc) and, as the libm-matched
 * diagnostic oracle, for the GPU (oracle/mam4_oracle_gpu.cu, nvcc): there
 * every function is device code and every table lives in device memory. */
#ifdef ORACLE_GPU
#define ORC_FN static __device__
#define ORC_TABLE static __device__ const
#else
#define ORC_FN static
#define ORC_TABLE static const
#endif

#ifdef ORACLE_ULP_NOISE
/* Rounding-sensitivity build (libmam4oracle_ulp.so): every libm result is
 * moved by one ulp up or down, the direction drawn from a xorshift stream
 * seeded per cell, so the run is deterministic under any thread schedule.
 * The spread of such runs around the canonical build measures how much the
 * reference algorithm itself amplifies last-bit differences of its math
 * library; the CUDA kernel is held to that spread on rounding-sensitive
 * cells and to 1e-12 everywhere else. */
#include <stdint.h>
static uint64_t g_noise_seed = 0;
static __thread uint64_t t_noise;
static void noise_seed_cell(size_t c) {
  uint64_t z = (uint64_t)c + 0x9E3779B97F4A7C15ull * (g_noise_seed + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  t_noise = (z ^ (z >> 31)) | 1ull;
}
static double nudge(double v, int k) {
  for (int i = 0; i < k; ++i)
    v = nextafter(v, INFINITY);
  for (int i = 0; i > k; --i)
    v = nextafter(v, -INFINITY);
  return v;
}
/* moves v by a nonzero number of ulps in [-maxulp, maxulp] */
static double noisy_k(double v, int maxulp) {
  if (g_noise_seed == 0 || !isfinite(v) || v == 0.0)
    return v;
  t_noise ^= t_noise << 13;
  t_noise ^= t_noise >> 7;
  t_noise ^= t_noise << 17;
  const int k = 1 + (int)((t_noise >> 1) % (uint64_t)maxulp);
  return nudge(v, (t_noise & 1) ? k : -k);
}
/* ulp bounds of the GPU math library for these functions: 2 ulp, erfc 5 */
static double noisy(double v) { return noisy_k(v, 2); }
static double n_exp(double x) { return noisy(exp(x)); }
static double n_log(double x) { return noisy(log(x)); }
static double n_pow(double x, double y) { return noisy(pow(x, y)); }
static double n_cbrt(double x) { return noisy(cbrt(x)); }
static double n_erfc(double x) { return noisy_k(erfc(x), 5); }
static double n_log10(double x) { return noisy(log10(x)); }
static double n_atan2(double y, double x) { return noisy(atan2(y, x)); }
static double n_hypot(double x, double y) { return noisy(hypot(x, y)); }
static double n_sin(double x) { return noisy(sin(x)); }
static double n_cos(double x) { return noisy(cos(x)); }
#define exp n_exp
#define log n_log
#define pow n_pow
#define cbrt n_cbrt
#define erfc n_erfc
#define log10 n_log10
#define atan2 n_atan2
#define hypot n_hypot
#define sin n_sin
#define cos n_cos
void mam4orc_set_ulp_noise(unsigned long long seed) { g_noise_seed = seed; }
#define NOISE_SEED_CELL(c) noise_seed_cell(c)
#else
#define NOISE_SEED_CELL(c) ((void)0)
#endif

#ifndef ORACLE_REAL
typedef double real;
#else
typedef ORACLE_REAL real;
#endif

#define NMODE 4
#define NAER 7
#define NGAS 2
#define PCNST 31
#define NSUB 3
#define NQTEND 4

ORC_TABLE real PI = 3.14159265358979323846264;
#define PI_SIXTH (3.14159265358979323846264 / 6)
#define EPS DBL_EPSILON

ORC_FN real rmax(real a, real b) { return (a < b) ? b : a; }
ORC_FN real rmin(real a, real b) { return (b < a) ? b : a; }
ORC_FN real square(real x) { return x * x; }
ORC_FN real cube(real x) { return x * x * x; }
/* utils.hpp:24 */
ORC_FN real min_max_bound(real lo, real hi, real x) { return rmax(lo, rmin(hi, x)); }
/* floating_point.hpp:79 */
ORC_FN real safe_denominator(real x) { return x / (x * x + EPS * EPS); }

/* ------------------------------------------------------------ constants */
/* aero_modes.hpp:76-123 (accumulation, aitken, coarse, primary carbon) */
ORC_TABLE real MODE_DMIN[NMODE] = {5.35e-8, 8.7e-9, 1e-6, 1e-8};
ORC_TABLE real MODE_DNOM[NMODE] = {1.1e-7, 2.6e-8, 2e-6, 5e-8};
ORC_TABLE real MODE_DMAX[NMODE] = {4.4e-7, 5.2e-8, 4e-6, 1e-7};
ORC_TABLE real MODE_SIG[NMODE] = {1.8, 1.6, 1.8, 1.60000002384186};
ORC_TABLE real RH_CRYST = 0.35, RH_DELIQ = 0.8;
/* aero_modes.hpp:214-243; AeroId: SOA 0 SO4 1 POM 2 BC 3 NaCl 4 DST 5 MOM 6 */
ORC_TABLE int NSPEC[NMODE] = {7, 4, 7, 3};
ORC_TABLE int MODE_SPEC[NMODE][7] = {{1, 2, 0, 3, 5, 4, 6},
                                        {1, 0, 4, 6, -1, -1, -1},
                                        {5, 4, 1, 3, 2, 0, 6},
                                        {2, 3, 6, -1, -1, -1, -1}};
/* aero_modes.hpp:140-150 densities by AeroId */
ORC_TABLE real AERO_DENS[NAER] = {1000.0, 1770.0, 1000.0, 1700.0, 1900.0, 2600.0, 1601.0};
/* state_q indices (0-based): number of each mode (utils.hpp:205-218) and the
 * first species slot of each mode (ndrop.hpp:77-80, minus one) */
ORC_TABLE int NUM_IDX[NMODE] = {22, 27, 35, 39};
ORC_TABLE int SPEC0_IDX[NMODE] = {15, 23, 28, 36};
/* water uptake species types (water_uptake.hpp:314-344 /
 * ndrop.hpp:59-80): density and hygroscopicity by type 1..9 */
ORC_TABLE real SPECDENS[14] = {0.1770000000E+04, 0.1797693135 + 309, 0.1797693135 + 309,
                                  0.1000000000E+04, 0.1000000000E+04, 0.1700000000E+04,
                                  0.1900000000E+04, 0.2600000000E+04, 0.1601000000E+04,
                                  0, 0, 0, 0, 0};
ORC_TABLE real SPECHYGRO[14] = {0.5070000000E+00, 0.1797693135 + 309, 0.1797693135 + 309,
                                   0.1000000083E-09, 0.1400000000E+00, 0.1000000013E-09,
                                   0.1160000000E+01, 0.6800000000E-01, 0.1000000015E+00,
                                   0, 0, 0, 0, 0};
ORC_TABLE int LSPECTYPE[NMODE][7] = {{1, 4, 5, 6, 8, 7, 9},
                                        {1, 5, 7, 9, 0, 0, 0},
                                        {8, 7, 1, 6, 4, 5, 9},
                                        {4, 6, 9, 0, 0, 0, 0}};
/* chemistry mechanism molecular weights (gas_chem_mechanism.hpp:31-38) */
ORC_TABLE real ADV_MASS[PCNST] = {
    47.998200, 34.013600, 98.078400, 64.064800, 62.132400, 12.011000, 115.107340, 12.011000,
    12.011000, 12.011000, 135.064039, 58.442468, 250092.672000, 1.007400, 115.107340,
    12.011000, 58.442468, 250092.672000, 1.007400, 135.064039, 58.442468, 115.107340,
    12.011000, 12.011000, 12.011000, 250092.672000, 1.007400, 12.011000, 12.011000,
    250092.672000, 1.007400};
/* mam4_amicphys.hpp:35-154 index maps and unit factors */
ORC_TABLE int NUMPTR31[NMODE] = {13, 18, 26, 30};
ORC_TABLE int LMASSPTR31[NAER][NMODE] = {{6, 14, 19, 27},  {7, 15, 20, 28},
                                            {8, 16, 21, 29},  {9, 17, 22, -6},
                                            {10, -6, 23, -6}, {11, -6, 24, -6},
                                            {12, -6, 25, -6}};
ORC_TABLE int LMAPCC_ALL[PCNST] = {0, 0, 1, 0, 0, 1, 2, 2, 2, 2, 2, 2, 2, 3, 2, 2,
                                      2, 2, 3, 2, 2, 2, 2, 2, 2, 2, 3, 2, 2, 2, 3};
ORC_TABLE int LMAP_GAS[NGAS] = {5, 2};
ORC_TABLE int LMAP_AER[NAER][NMODE] = {{8, 15, 24, -1},  {6, 14, 21, -1}, {7, -1, 23, 27},
                                          {9, -1, 22, 28},  {11, 16, 20, -1},
                                          {10, -1, 19, -1}, {12, 17, 25, 29}};
ORC_TABLE real FCVT_AER[NAER] = {8.000000000000000E-002, 1, 8.000000000000000E-002, 1, 1, 1, 1};
/* rename / aging mass-to-volume factors (mam4_amicphys.hpp:1495-1502) */
ORC_TABLE real MASS_2_VOL[NAER] = {0.15, 6.4971751412429377e-002, 0.15,
                                      7.0588235294117650e-003, 3.0789473684210526e-002,
                                      5.1923076923076926e-002, 156.20986883198000};

/* coagulation correction tables (coagulation.hpp:81, :330, :588) */
#define COAG_TABLE_QUALIFIER ORC_TABLE
#include "../mam4xx_b200/csrc/coag_tables.inc"

ORC_FN real fcvt_gas(int igas) { /* mam4_amicphys.hpp:137-153 */
  const real mw_gas = ADV_MASS[LMAP_GAS[igas]];
  real denom = mw_gas;
  if (igas < 1)
    denom = 150;
  return mw_gas / denom;
}
/* fcvt_wtr (mam4_amicphys.hpp:97) is not needed: amicphys zeroes the aerosol
 * water of the subareas (:2248-2250), so every water entry stays zero. */

/* conversions.hpp:299-315 */
ORC_FN real mean_particle_diameter_from_volume(real v, real sig) {
  return cbrt(v / PI_SIXTH) * exp(-1.5 * square(log(sig)));
}
ORC_FN real mean_particle_volume_from_diameter(real d, real sig) {
  return cube(d) * exp(4.5 * square(log(sig))) * PI_SIXTH;
}

/* ================================================================ calcsize
 * modal_aero_calcsize.hpp, calcsize.hpp */
typedef struct {
  real inv_density[NMODE][NAER];
  real n2v_min[NMODE], n2v_max[NMODE], n2v_nom[NMODE];
} calcsize_data;

ORC_FN void calcsize_init(calcsize_data *d) { /* modal_aero_calcsize.hpp:22-108 */
  for (int m = 0; m < NMODE; ++m) {
    d->n2v_nom[m] = 1.0 / mean_particle_volume_from_diameter(MODE_DNOM[m], MODE_SIG[m]);
    d->n2v_min[m] = 1.0 / mean_particle_volume_from_diameter(MODE_DMAX[m], MODE_SIG[m]);
    d->n2v_max[m] = 1.0 / mean_particle_volume_from_diameter(MODE_DMIN[m], MODE_SIG[m]);
    for (int i = 0; i < NSPEC[m]; ++i)
      d->inv_density[m][i] = 1.0 / AERO_DENS[MODE_SPEC[m][i]];
  }
}

/* calcsize.hpp:56-78 */
ORC_FN void update_diameter_and_vol2num(real drv, real num, real v2nmin, real v2nmax,
                                        real dgnmin, real dgnmax, real sig, real *dgncur,
                                        real *v2ncur) {
  if (!(drv > 0.0))
    return;
  if (num <= drv * v2nmin) {
    *dgncur = dgnmax;
    *v2ncur = v2nmin;
  } else if (num >= drv * v2nmax) {
    *dgncur = dgnmin;
    *v2ncur = v2nmax;
  } else {
    *v2ncur = num / drv;
    *dgncur = mean_particle_diameter_from_volume(1.0 / *v2ncur, sig);
  }
}

/* calcsize.hpp:95-310 */
ORC_FN void adjust_num_sizes(real drv_i, real drv_c, real init_num_i, real init_num_c, real dt,
                             real v2nmin, real v2nmax, real adj_tscale_inv, real *num_i,
                             real *num_c, real *dqdt, real *dqqcwdt) {
  const real frac = rmax(0.0, rmin(1.0, dt * adj_tscale_inv));
  const real dtinv = safe_denominator(dt);
  const real relax = 27.0;
  const real minrl = v2nmin / relax, maxrl = v2nmax * relax;
  if (drv_i <= 0.0 && drv_c <= 0.0) {
    *num_i = 0.0;
    *num_c = 0.0;
    *dqdt = (*num_i - init_num_i) * dtinv;
    *dqqcwdt = (*num_c - init_num_c) * dtinv;
    return; /* the reference recomputes the same values below */
  } else if (drv_c <= 0.0) {
    *num_c = 0.0;
    const real numbnd = min_max_bound(drv_i * v2nmin, drv_i * v2nmax, *num_i);
    *num_i = *num_i + (numbnd - *num_i) * frac;
  } else if (drv_i <= 0.0) {
    const real numbnd = min_max_bound(drv_c * v2nmin, drv_c * v2nmax, *num_c);
    *num_c = *num_c + (numbnd - *num_c) * frac;
    *num_i = 0.0;
  } else {
    const real ni1 = *num_i, nc1 = *num_c;
    real numbnd = min_max_bound(drv_i * minrl, drv_i * maxrl, ni1);
    const real dni2 = (numbnd - ni1) * frac;
    real ni2 = ni1 + dni2;
    numbnd = min_max_bound(drv_c * minrl, drv_c * maxrl, nc1);
    const real dnc2 = (numbnd - nc1) * frac;
    real nc2 = nc1 + dnc2;
    if (dni2 == 0.0 && dnc2 != 0.0)
      ni2 = min_max_bound(drv_i * minrl, drv_i * maxrl, ni1 - dnc2);
    else if (dni2 != 0.0 && dnc2 == 0.0)
      nc2 = min_max_bound(drv_c * minrl, drv_c * maxrl, nc1 - dni2);
    const real total_drv = drv_i + drv_c;
    const real total_num = ni2 + nc2;
    real dni3 = 0.0, dnc3 = 0.0;
    const real minb = total_drv * v2nmin, maxb = total_drv * v2nmax;
    if (total_num < minb) {
      const real dt3 = (minb - total_num) * frac;
      if ((ni2 < drv_i * v2nmin) && (nc2 < drv_c * v2nmin)) {
        dni3 = dt3 * (ni2 / total_num);
        dnc3 = dt3 * (nc2 / total_num);
      } else if (nc2 < drv_c * v2nmin) {
        dnc3 = dt3;
      } else if (ni2 < drv_i * v2nmin) {
        dni3 = dt3;
      }
    } else if (total_num > maxb) {
      const real dt3 = (maxb - total_num) * frac;
      if ((ni2 > drv_i * v2nmax) && (nc2 > drv_c * v2nmax)) {
        dni3 = dt3 * (ni2 / total_num);
        dnc3 = dt3 * (nc2 / total_num);
      } else if (nc2 > drv_c * v2nmax) {
        dnc3 = dt3;
      } else if (ni2 > drv_i * v2nmax) {
        dni3 = dt3;
      }
    }
    *num_i = ni2 + dni3;
    *num_c = nc2 + dnc3;
  }
  *dqdt = (*num_i - init_num_i) * dtinv;
  *dqqcwdt = (*num_c - init_num_c) * dtinv;
}

/* calcsize.hpp:481-515 */
ORC_FN void compute_new_sz_after_transfer(real drv, real num, real v2n_hi, real v2n_lo, real v2n,
                                          real dgn_hi, real dgn_lo, real dgn_nom, real sig,
                                          real *dgncur, real *v2ncur) {
  if (drv > 0.0) {
    if (num <= drv * v2n_hi) {
      *dgncur = dgn_hi;
      *v2ncur = v2n_hi;
    } else if (num >= drv * v2n_lo) {
      *dgncur = dgn_lo;
      *v2ncur = v2n_lo;
    } else {
      *v2ncur = num / drv;
      *dgncur = mean_particle_diameter_from_volume(1.0 / *v2ncur, sig);
    }
  } else {
    *dgncur = dgn_nom;
    *v2ncur = v2n;
  }
}

/* modal_aero_calcsize.hpp:448-497 (update_tends_flx) */
ORC_FN void update_tends_flx(int jmode, int src, int dest, const int *src_idx,
                             const int *dest_idx, const real xfertend_num[2][2], real xfercoef,
                             const real *state_q, const real *qqcw, real *ptend, real *dqqcwdt) {
  ptend[src] -= xfertend_num[jmode][0];
  ptend[dest] += xfertend_num[jmode][0];
  dqqcwdt[src] -= xfertend_num[jmode][1];
  dqqcwdt[dest] += xfertend_num[jmode][1];
  for (int i = 0; i < 4; ++i) {
    const real xi = rmax(0.0, state_q[src_idx[i]]) * xfercoef;
    ptend[src_idx[i]] -= xi;
    ptend[dest_idx[i]] += xi;
    const real xc = rmax(0.0, qqcw[src_idx[i]]) * xfercoef;
    dqqcwdt[src_idx[i]] -= xc;
    dqqcwdt[dest_idx[i]] += xc;
  }
}

/* modal_aero_calcsize.hpp:750-932 (modal_aero_calcsize_sub with
 * size_adjustment :263, compute_dry_volume :421, aitken_accum_exchange :499,
 * compute_coef_acc_ait_transfer :162, calcsize.hpp:314) */
ORC_FN void calcsize_sub(const calcsize_data *cd, const real *state_q, const real *qqcw, real dt,
                         real dgncur_i[NMODE], real dgncur_c[NMODE], real ptend[40],
                         real dqqcwdt[40]) {
  const int ait = 1, acc = 0;
  const real adj_tscale = rmax(86400.0, dt);
  const real adj_tscale_inv = safe_denominator(adj_tscale);
  real dv_i_accsv = 0, dv_c_accsv = 0, dv_i_aitsv = 0, dv_c_aitsv = 0;
  real n_i_accsv = 0, n_c_accsv = 0, n_i_aitsv = 0, n_c_aitsv = 0;
  for (int m = 0; m < NMODE; ++m) {
    dgncur_i[m] = MODE_DNOM[m];
    real v2n_i = cd->n2v_nom[m];
    dgncur_c[m] = MODE_DNOM[m];
    real v2n_c = cd->n2v_nom[m];
    real dv_i = 0.0, dv_c = 0.0;
    for (int s = 0; s < NSPEC[m]; ++s) {
      const int idx = SPEC0_IDX[m] + s;
      dv_i += rmax(0.0, state_q[idx]) * cd->inv_density[m][s];
      dv_c += rmax(0.0, qqcw[idx]) * cd->inv_density[m][s];
    }
    const real init_num_i = state_q[NUM_IDX[m]];
    const real init_num_c = qqcw[NUM_IDX[m]];
    real num_i = init_num_i < 0 ? 0.0 : init_num_i;
    real num_c = init_num_c < 0 ? 0.0 : init_num_c;
    const int ait_or_acc = (m == acc || m == ait);
    if (!ait_or_acc)
      adjust_num_sizes(dv_i, dv_c, init_num_i, init_num_c, dt, cd->n2v_min[m], cd->n2v_max[m],
                       adj_tscale_inv, &num_i, &num_c, &ptend[NUM_IDX[m]],
                       &dqqcwdt[NUM_IDX[m]]);
    real v2nmin = cd->n2v_min[m], v2nmax = cd->n2v_max[m];
    if (m == ait)
      v2nmin /= 1.0e6;
    if (m == acc)
      v2nmax *= 1.0e6;
    update_diameter_and_vol2num(dv_i, num_i, v2nmin, v2nmax, MODE_DMIN[m], MODE_DMAX[m],
                                MODE_SIG[m], &dgncur_i[m], &v2n_i);
    update_diameter_and_vol2num(dv_c, num_c, v2nmin, v2nmax, MODE_DMIN[m], MODE_DMAX[m],
                                MODE_SIG[m], &dgncur_c[m], &v2n_c);
    if (m == ait) {
      dv_i_aitsv = dv_i;
      n_i_aitsv = num_i;
      dv_c_aitsv = dv_c;
      n_c_aitsv = num_c;
    } else if (m == acc) {
      dv_i_accsv = dv_i;
      n_i_accsv = num_i;
      dv_c_accsv = dv_c;
      n_c_accsv = num_c;
    }
  }

  /* aitken_accum_exchange (modal_aero_calcsize.hpp:499-747) */
  const real v2n_ait = cd->n2v_nom[ait], v2n_acc = cd->n2v_nom[acc];
  const real geomean = sqrt(v2n_ait) * sqrt(v2n_acc);
  real xfertend_num[2][2] = {{0, 0}, {0, 0}};
  /* compute_coef_ait_acc_transfer (calcsize.hpp:314-376) */
  int ait2acc = 0;
  real xfc_num_ait2acc = 0, xfc_vol_ait2acc = 0;
  {
    const real drv_t = dv_i_aitsv + dv_c_aitsv;
    const real num_t = n_i_aitsv + n_c_aitsv;
    real fn = 0, fv = 0;
    if (drv_t > 0.0 && num_t < drv_t * geomean) {
      ait2acc = 1;
      if (num_t < drv_t * v2n_acc) {
        fn = 1.0;
        fv = 1.0;
      } else {
        fv = ((num_t / drv_t) - geomean) / (v2n_acc - geomean);
        fn = fv * (drv_t * v2n_acc / num_t);
        if (fn <= 0.0 || fv <= 0.0) {
          fn = 0.0;
          fv = 0.0;
        } else if (fn >= 1.0 || fv >= 1.0) {
          fn = 1.0;
          fv = 1.0;
        }
      }
      xfc_num_ait2acc = fn * adj_tscale_inv;
      xfc_vol_ait2acc = fv * adj_tscale_inv;
      xfertend_num[0][0] = n_i_aitsv * xfc_num_ait2acc;
      xfertend_num[0][1] = n_c_aitsv * xfc_num_ait2acc;
    }
  }
  /* compute_coef_acc_ait_transfer (modal_aero_calcsize.hpp:162-259) */
  int acc2ait = 0;
  real xfc_num_acc2ait = 0, xfc_vol_acc2ait = 0, drv_i_noxf = 0, drv_c_noxf = 0;
  {
    const int noxf[7] = {0, 1, 0, 1, 1, 0, 0};
    real drv_t = dv_i_accsv + dv_c_accsv;
    real num_t = n_i_accsv + n_c_accsv;
    real num_t0 = 0;
    if (drv_t > 0.0 && num_t > drv_t * geomean) {
      for (int s = 0; s < NSPEC[acc]; ++s) {
        if (noxf[s]) {
          const int idx = SPEC0_IDX[acc] + s;
          drv_i_noxf += rmax(0.0, state_q[idx]) * cd->inv_density[acc][s];
          drv_c_noxf += rmax(0.0, qqcw[idx]) * cd->inv_density[acc][s];
        }
      }
      const real drv_t_noxf = drv_i_noxf + drv_c_noxf;
      const real num_t_noxf = drv_t_noxf * cd->n2v_max[acc];
      num_t0 = num_t;
      num_t = rmax(0.0, num_t - num_t_noxf);
      drv_t = rmax(0.0, drv_t - drv_t_noxf);
    }
    if (drv_t > 0.0 && num_t > drv_t * geomean) {
      real fn, fv;
      acc2ait = 1;
      if (num_t > drv_t * v2n_ait) {
        fn = 1.0;
        fv = 1.0;
      } else {
        fv = ((num_t / drv_t) - geomean) / (v2n_ait - geomean);
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
      xfc_num_acc2ait = fn * adj_tscale_inv;
      xfc_vol_acc2ait = fv * adj_tscale_inv;
      xfertend_num[1][0] = n_i_accsv * xfc_num_acc2ait;
      xfertend_num[1][1] = n_c_accsv * xfc_num_acc2ait;
    }
  }
  if (ait2acc + acc2ait > 0) {
    real tmp;
    const real num_diff_i = (xfertend_num[0][0] - xfertend_num[1][0]) * dt;
    const real num_i = rmax(0.0, n_i_aitsv - num_diff_i);
    const real num_i_acc = rmax(0.0, n_i_accsv + num_diff_i);
    const real vol_diff_i =
        (dv_i_aitsv * xfc_vol_ait2acc - (dv_i_accsv - drv_i_noxf) * xfc_vol_acc2ait) * dt;
    const real drv_i = rmax(0.0, dv_i_aitsv - vol_diff_i);
    const real drv_i_acc = rmax(0.0, dv_i_accsv + vol_diff_i);
    const real num_diff_c = (xfertend_num[0][1] - xfertend_num[1][1]) * dt;
    const real num_c = rmax(0.0, n_c_aitsv - num_diff_c);
    const real num_c_acc = rmax(0.0, n_c_accsv + num_diff_c);
    const real vol_diff_c =
        (dv_c_aitsv * xfc_vol_ait2acc - (dv_c_accsv - drv_c_noxf) * xfc_vol_acc2ait) * dt;
    const real drv_c = rmax(0.0, dv_c_aitsv - vol_diff_c);
    const real drv_c_acc = rmax(0.0, dv_c_accsv + vol_diff_c);
    compute_new_sz_after_transfer(drv_i, num_i, cd->n2v_min[ait], cd->n2v_max[ait],
                                  cd->n2v_nom[ait], MODE_DMAX[ait], MODE_DMIN[ait],
                                  MODE_DNOM[ait], MODE_SIG[ait], &dgncur_i[ait], &tmp);
    compute_new_sz_after_transfer(drv_c, num_c, cd->n2v_min[ait], cd->n2v_max[ait],
                                  cd->n2v_nom[ait], MODE_DMAX[ait], MODE_DMIN[ait],
                                  MODE_DNOM[ait], MODE_SIG[ait], &dgncur_c[ait], &tmp);
    compute_new_sz_after_transfer(drv_i_acc, num_i_acc, cd->n2v_min[acc], cd->n2v_max[acc],
                                  cd->n2v_nom[acc], MODE_DMAX[acc], MODE_DMIN[acc],
                                  MODE_DNOM[acc], MODE_SIG[acc], &dgncur_i[acc], &tmp);
    compute_new_sz_after_transfer(drv_c_acc, num_c_acc, cd->n2v_min[acc], cd->n2v_max[acc],
                                  cd->n2v_nom[acc], MODE_DMAX[acc], MODE_DMIN[acc],
                                  MODE_DNOM[acc], MODE_SIG[acc], &dgncur_c[acc], &tmp);
    /* common species: accumulation slots SO4, SOA, NaCl, MOM and their
     * aitken counterparts (modal_aero_calcsize.hpp:46-70) */
    const int acc_in_ait[4] = {15, 17, 20, 21};
    const int ait_in_acc[4] = {23, 24, 25, 26};
    if (ait2acc > 0)
      update_tends_flx(0, 27, 22, ait_in_acc, acc_in_ait, xfertend_num, xfc_vol_ait2acc,
                       state_q, qqcw, ptend, dqqcwdt);
    if (acc2ait > 0)
      update_tends_flx(1, 22, 27, acc_in_ait, ait_in_acc, xfertend_num, xfc_vol_acc2ait,
                       state_q, qqcw, ptend, dqqcwdt);
  }
}

/* ============================================================ water uptake
 * water_uptake.hpp, wv_sat_methods.hpp */
typedef struct {
  real re, im;
} cplx;
ORC_FN cplx cmk(real r, real i) {
  cplx z = {r, i};
  return z;
}
ORC_FN cplx cadd(cplx a, cplx b) { return cmk(a.re + b.re, a.im + b.im); }
ORC_FN cplx csub(cplx a, cplx b) { return cmk(a.re - b.re, a.im - b.im); }
ORC_FN cplx cmul(cplx a, cplx b) {
  return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
ORC_FN cplx cscale(real s, cplx a) { return cmk(s * a.re, s * a.im); }
ORC_FN cplx cdivr(cplx a, real s) { return cmk(a.re / s, a.im / s); }
ORC_FN cplx cdiv(cplx x, cplx y) {
  const real s = fabs(y.re) + fabs(y.im);
  if (s == 0.0)
    return cmk(x.re / s, x.im / s);
  const cplx xs = cmk(x.re / s, x.im / s);
  const cplx ycs = cmk(y.re / s, -y.im / s);
  const real yabs2 = ycs.re * ycs.re + ycs.im * ycs.im;
  const cplx r = cmul(xs, ycs);
  return cmk(r.re / yabs2, r.im / yabs2);
}
ORC_FN cplx csqrt_k(cplx x) {
  const real r = x.re, i = x.im;
  if (r == 0.0) {
    const real t = sqrt(fabs(i) / 2);
    return cmk(t, i < 0.0 ? -t : t);
  }
  const real t = sqrt(2 * (hypot(r, i) + fabs(r)));
  const real u = t / 2;
  return r > 0.0 ? cmk(u, i / t) : cmk(fabs(i) / t, i < 0.0 ? -u : u);
}
ORC_FN cplx cpow_k(cplx x, real y) {
  const real r = hypot(x.re, x.im);
  const real th = atan2(x.im, x.re);
  const real rho = pow(r, y), ang = y * th;
  return cmk(rho * cos(ang), rho * sin(ang));
}

/* water_uptake.hpp:131-171 */
ORC_FN void makoh_quartic(cplx cx[4], real p3, real p2, real p1, real p0) {
  const real qq = -p2 * p2 / 36.0 + (p3 * p1 - 4.0 * p0) / 12.0;
  const real rr = -cube(p2 / 6.0) + p2 * (p3 * p1 - 4.0 * p0) / 48.0 +
                  (4.0 * p0 * p2 - p0 * p3 * p3 - p1 * p1) / 16.0;
  const cplx sq_crad = cmk(rr * rr + qq * qq * qq, 0.0);
  cplx crad = csqrt_k(sq_crad);
  cplx cb = csub(cmk(rr, 0.0), crad);
  if (cb.re == 0.0 && cb.im == 0.0) {
    const real r = cbrt(-p1);
    for (int i = 0; i < 4; ++i)
      cx[i] = cmk(r, 0.0);
    return;
  }
  cb = cpow_k(cb, 1.0 / 3.0);
  const cplx cy = cadd(cadd(cmk(-cb.re, -cb.im), cdiv(cmk(qq, 0.0), cb)), cmk(p2 / 6.0, 0.0));
  const cplx cb0 = csqrt_k(csub(cmul(cy, cy), cmk(p0, 0.0)));
  const cplx cb1 = cdiv(csub(cscale(p3, cy), cmk(p1, 0.0)), cscale(2.0, cb0));
  cb = cadd(cmk(p3 / 2.0, 0.0), cb1);
  crad = csqrt_k(csub(cmul(cb, cb), cscale(4.0, cadd(cy, cb0))));
  cx[0] = cdivr(cadd(cmk(-cb.re, -cb.im), crad), 2.0);
  cx[1] = cdivr(csub(cmk(-cb.re, -cb.im), crad), 2.0);
  cb = csub(cmk(p3 / 2.0, 0.0), cb1);
  crad = csqrt_k(csub(cmul(cb, cb), cscale(4.0, csub(cy, cb0))));
  cx[2] = cdivr(cadd(cmk(-cb.re, -cb.im), crad), 2.0);
  cx[3] = cdivr(csub(cmk(-cb.re, -cb.im), crad), 2.0);
}

/* water_uptake.hpp:101-125 */
ORC_FN real find_real_solution(real rdry, const cplx cx[4]) {
  const real eps = 1e-4;
  real rwet = 1000.0 * rdry;
  for (int n = 0; n < 4; ++n) {
    const real xr = cx[n].re, xi = cx[n].im;
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

/* water_uptake.hpp:180-230 */
ORC_FN real kohler(real rdry_in, real hygro, real rh) {
  const real rhow = 1.0, surften = 76.0, mw = 18.0, tair = 273.0, ugascon = 8.3e7;
  const real eps = 1e-4;
  const real aa = 2.0e4 * mw * surften / (ugascon * tair * rhow);
  const real rdry = rdry_in * 1.e6;
  const real vol = cube(rdry);
  const real bb = vol * hygro;
  const real ss = min_max_bound(1.e-10, 1.0 - eps, rh);
  const real slog = log(ss);
  const real p43 = -aa / slog;
  const real p42 = 0.0;
  const real p41 = bb / slog - vol;
  const real p40 = aa * vol / slog;
  const real pp = fabs(-bb / aa) / (rdry * rdry);
  real rwet;
  if (pp < eps) {
    rwet = rdry * (1.0 + pp * (1.0 / 3.0) / (1.0 - slog * rdry / aa));
  } else {
    cplx cx[4];
    makoh_quartic(cx, p43, p42, p41, p40);
    rwet = find_real_solution(rdry, cx);
  }
  rwet = rmin(rwet, 30.0);
  return rwet * 1.e-6;
}

/* wv_sat_methods.hpp:14-46, 94-131 */
ORC_FN real goffgratch_svp_water(real t) {
  const real tboil = 373.16, ten = 10, one = 1;
  return pow(ten, -7.90298 * (tboil / t - one) + 5.02808 * log10(tboil / t) -
                      1.3816e-7 * (pow(ten, 11.344 * (one - t / tboil)) - one) +
                      8.1328e-3 * (pow(ten, -3.49149 * (tboil / t - one)) - one) +
                      log10(1013.246)) *
         ten * ten;
}
ORC_FN real qsat_water(real t, real p) {
  const real es = goffgratch_svp_water(t);
  const real epsilo = 0.018016 / 0.028966;
  const real omeps = 1 - epsilo;
  if ((p - es) <= 0)
    return 1;
  return epsilo * es / (p - omeps * es);
}

/* water_uptake.hpp:362-480 (dryaer, rh_clearair, wetaer, wetdens) */
ORC_FN void water_uptake_dr(const real *state_q, real temp, real pmid, real cldn,
                            const real dgncur_a[NMODE], real dgncur_awet[NMODE],
                            real qaerwat[NMODE], real wetdens[NMODE]) {
  real hygro[NMODE], naer[NMODE], dryrad[NMODE], dryvol[NMODE], drymass[NMODE];
  real specdens_1[NMODE];
  for (int m = 0; m < NMODE; ++m) {
    hygro[m] = 0.0;
    real dryvolmr = 0.0, maer = 0.0;
    const real sigmag = MODE_SIG[m];
    int t = LSPECTYPE[m][0] - 1;
    specdens_1[m] = SPECDENS[t];
    const real spechygro_1 = SPECHYGRO[t];
    const real alnsg = log(sigmag);
    for (int s = 0; s < NSPEC[m]; ++s) {
      t = LSPECTYPE[m][s] - 1;
      const real raer = state_q[SPEC0_IDX[m] + s];
      const real vol_tmp = raer / SPECDENS[t];
      maer = maer + raer;
      dryvolmr += vol_tmp;
      hygro[m] += vol_tmp * SPECHYGRO[t];
    }
    if (dryvolmr > 1e-30)
      hygro[m] = hygro[m] / dryvolmr;
    else
      hygro[m] = spechygro_1;
    const real v2ncur_a = 1.0 / ((PI / 6.0) * cube(dgncur_a[m]) * exp(4.5 * square(alnsg)));
    naer[m] = dryvolmr * v2ncur_a;
    const real drydens = (maer > 1e-31) ? maer / dryvolmr : 1.0;
    dryvol[m] = 1.0 / v2ncur_a;
    drymass[m] = drydens * dryvol[m];
    dryrad[m] = cbrt(dryvol[m] / (PI * 4.0 / 3.0));
  }
  /* rh_clearair */
  real rh;
  {
    const real qs = qsat_water(temp, pmid);
    const real h2ommr = state_q[0];
    const real rh_max = 0.98;
    rh = (qs > h2ommr) ? h2ommr / qs : rh_max;
    rh = min_max_bound(0.0, rh_max, rh);
    if (cldn < 1.0)
      rh = (rh - cldn) / (1.0 - cldn);
    rh = rmax(rh, 0.0);
  }
  /* wetaer + wetdens */
  for (int m = 0; m < NMODE; ++m) {
    const real hystfac = 1.0 / rmax(1.0e-5, (RH_DELIQ - RH_CRYST));
    real wetrad = kohler(dryrad[m], hygro[m], rh);
    wetrad = rmax(wetrad, dryrad[m]);
    real wetvol = (PI * 4.0 / 3.0) * cube(wetrad);
    wetvol = rmax(wetvol, dryvol[m]);
    real wtrvol = wetvol - dryvol[m];
    wtrvol = rmax(wtrvol, 0.0);
    if (rh < RH_CRYST) {
      wetrad = dryrad[m];
      wetvol = dryvol[m];
      wtrvol = 0.0;
    } else if (rh < RH_DELIQ) {
      wtrvol = wtrvol * hystfac * (rh - RH_CRYST);
      wtrvol = rmax(wtrvol, 0.0);
      wetvol = dryvol[m] + wtrvol;
      wetrad = cbrt(wetvol / (4.0 / 3.0 * PI));
    }
    dgncur_awet[m] = dgncur_a[m] * (wetrad / dryrad[m]);
    qaerwat[m] = 1.0e3 * naer[m] * wtrvol;
    if (wetvol > 1.0e-30)
      wetdens[m] = (drymass[m] + 1.0e3 * wtrvol) / wetvol;
    else
      wetdens[m] = specdens_1[m];
  }
}

/* ================================================================ amicphys
 * gasaerexch.hpp, gasaerexch_soaexch.hpp */

/* gasaerexch.hpp:255-268 */
ORC_FN real fuchs_sutugin(real d_p, real freepath, real a283, real a75) {
  const real kn = 2.0 * freepath / d_p;
  return (a75 * (1.0 + kn)) / (kn * (kn + 1.0 + a283) + a75);
}

/* gasaerexch.hpp:270-353 */
ORC_FN void gas_aer_uptkrates_1box1gas(real accom, real gasdiffus, real freepath,
                                       const real dgn_awet[NMODE], const real lnsg[NMODE],
                                       real uptk[NMODE]) {
  const real tworootpi = 2 * sqrt(PI);
  const real root2 = sqrt(2.0);
  const real xghq[2] = {7.071067690849304E-01, -7.071067690849304E-01};
  const real wghq[2] = {8.862269520759583E-01, 8.862269520759583E-01};
  const real a283 = accom * 0.283, a75 = accom * 0.75;
  for (int n = 0; n < NMODE; ++n) {
    const real lndpgn = log(dgn_awet[n]);
    const real d_p = dgn_awet[n];
    const real kn = 2.0 * freepath / d_p;
    const real tmpa = 1.0 / (1.0 + kn) - (2.0 * kn + 1.0 + a283) / (kn * (kn + 1.0 + a283) + a75);
    real beta = 1.0 - kn * tmpa;
    beta = rmax(1.0, rmin(2.0, beta));
    const real constant = tworootpi * exp(beta * lndpgn + 0.5 * pow(beta * lnsg[n], 2.0));
    real sum = 0.0;
    for (int q = 0; q < 2; ++q) {
      const real lndp = lndpgn + beta * lnsg[n] * lnsg[n] + root2 * lnsg[n] * xghq[q];
      const real dp = exp(lndp);
      const real hh = fuchs_sutugin(dp, freepath, a283, a75);
      sum += wghq[q] * dp * hh / pow(dp, beta);
    }
    uptk[n] = constant * gasdiffus * sum;
  }
}

/* gasaerexch_soaexch.hpp:80-341 (the 9-argument variant called by
 * mam_gasaerexch_1subarea); returns the number of sub-steps */
ORC_FN int soaexch_1subarea(real dtsubstep, real temp, real pmid, real qgas_cur[NGAS],
                            real qgas_avg[NGAS], real qaer_cur[NAER][NMODE],
                            const real uptkaer[NGAS][NMODE]) {
  const int niter_max = 1000;
  int niter = 0;
  const real dtfull = dtsubstep;
  real tcur = 0.0, dtcur = 0.0, dtsum_qgas_avg = 0.0;
  real qgas_prv = 0.0;
  real qaer_prv[NAER][NMODE];
  real uptk_tmp[NMODE] = {0};
  real a_ooa_sum_tmp[NMODE] = {0};
  real a_opoa[NMODE] = {0};
  real a_soa[NMODE] = {0}, a_soa_tmp[NMODE] = {0}, beta[NMODE] = {0};
  real g_star[NMODE] = {0}, phi[NMODE] = {0}, sat[NMODE] = {0};
  real del_g_soa_tmp = 0.0, g_soa = 0.0, tot_soa = 0.0;
  int skip[NMODE];
  const real opoa_frac[NMODE] = {0.1, 0.1, 0.1, 0.0};
  const real delh_vap_soa = 156.0e3, p0_soa_298 = 1.0e-10, rgas = 8.3144;
  const real alpha_astem = 0.05, a_min1 = 1.0e-20, g_min1 = 1.0e-20;
  const real p0_soa = p0_soa_298 * exp(-(delh_vap_soa / rgas) * ((1.0 / temp) - (1.0 / 298.0)));
  const real g0_soa = 1.01325e5 * p0_soa / pmid;
  qgas_avg[0] = 0.0;
  dtsum_qgas_avg = 0.0;
  while (tcur < dtfull - 1.0e-3) {
    niter++;
    if (niter > niter_max)
      break;
    qgas_prv = qgas_cur[0];
    for (int a = 0; a < NAER; ++a)
      for (int n = 0; n < NMODE; ++n)
        qaer_prv[a][n] = qaer_cur[a][n];
    for (int n = 0; n < NMODE; ++n) {
      skip[n] = 1;
      if (uptkaer[0][n] > 1.0e-15) {
        uptk_tmp[n] = uptkaer[0][n];
        skip[n] = 0;
      } else {
        uptk_tmp[n] = 0.0;
      }
    }
    g_soa = rmax(qgas_prv, 0.0);
    tot_soa = g_soa;
    for (int n = 0; n < NMODE; ++n) {
      if (skip[n])
        continue;
      a_soa[n] = rmax(qaer_prv[0][n], 0.0);
      tot_soa += a_soa[n];
    }
    for (int n = 0; n < NMODE; ++n) {
      if (skip[n])
        continue;
      a_opoa[n] = 0.0;
      a_opoa[n] += opoa_frac[n] * rmax(qaer_prv[2][n], 0.0); /* iaer_pom = 2 */
    }
    real tmpa = 0.0;
    for (int n = 0; n < NMODE; ++n) {
      if (skip[n])
        continue;
      a_ooa_sum_tmp[n] = a_opoa[n];
      a_ooa_sum_tmp[n] += a_soa[n];
    }
    {
      real tmpb = 0.0;
      for (int n = 0; n < NMODE; ++n) {
        if (skip[n])
          continue;
        sat[n] = g0_soa / rmax(a_ooa_sum_tmp[n], a_min1);
        g_star[n] = sat[n] * a_soa[n];
        phi[n] = (g_soa - g_star[n]) / rmax(g_soa, rmax(g_star[n], g_min1));
        tmpb += uptk_tmp[n] * fabs(phi[n]);
      }
      tmpa = rmax(tmpa, tmpb);
    }
    {
      const real dtmax = dtfull - tcur;
      if (dtmax * tmpa <= alpha_astem) {
        dtcur = dtmax;
        tcur = dtfull;
      } else {
        dtcur = alpha_astem / tmpa;
        tcur += dtcur;
      }
    }
    for (int n = 0; n < NMODE; ++n) {
      if (skip[n])
        continue;
      a_soa_tmp[n] = a_soa[n];
      beta[n] = dtcur * uptk_tmp[n];
      del_g_soa_tmp = g_soa - g_star[n];
      if (del_g_soa_tmp > 0.0)
        a_soa_tmp[n] += beta[n] * del_g_soa_tmp;
      a_ooa_sum_tmp[n] = a_opoa[n];
      a_ooa_sum_tmp[n] += a_soa_tmp[n];
      if (del_g_soa_tmp > 0.0) {
        sat[n] = g0_soa / rmax(a_ooa_sum_tmp[n], a_min1);
        g_star[n] = sat[n] * a_soa_tmp[n];
      }
    }
    {
      real ta = 0.0, tb = 0.0;
      for (int n = 0; n < NMODE; ++n) {
        if (skip[n])
          continue;
        ta += a_soa[n] / (1.0 + beta[n] * sat[n]);
        tb += beta[n] / (1.0 + beta[n] * sat[n]);
      }
      g_soa = (tot_soa - ta) / (1.0 + tb);
      g_soa = rmax(0.0, g_soa);
      for (int n = 0; n < NMODE; ++n) {
        if (skip[n])
          continue;
        a_soa[n] = (a_soa[n] + beta[n] * g_soa) / (1.0 + beta[n] * sat[n]);
      }
    }
    qgas_cur[0] = g_soa;
    {
      const real tmpc = qgas_cur[0] - qgas_prv;
      qgas_avg[0] += dtcur * (qgas_prv + 0.5 * tmpc);
    }
    for (int n = 0; n < NMODE; ++n)
      qaer_cur[0][n] = a_soa[n];
    dtsum_qgas_avg += dtcur;
  }
  qgas_avg[0] = rmax(0.0, qgas_avg[0] / dtsum_qgas_avg);
  return niter;
}

/* gasaerexch.hpp:355-557; returns SOA sub-step count */
ORC_FN int gasaerexch_1subarea(real dtsubstep, real temp, real pmid, real aircon,
                               real qgas_cur[NGAS], real qgas_avg[NGAS],
                               const real qgas_netprod[NGAS], real qaer_cur[NAER][NMODE],
                               const real qnum_cur[NMODE], const real dgn_awet[NMODE],
                               real uptkaer[NGAS][NMODE], real *uptkrate_h2so4) {
  real alnsg[NMODE];
  for (int m = 0; m < NMODE; ++m)
    alnsg[m] = log(MODE_SIG[m]);
  const real mw_gas[NGAS] = {1.500000000000000E+02, 9.807840000000000E+01};
  const real vol_molar_gas[NGAS] = {6.563265306122449E+01, 4.288000000000000E+01};
  const real accom_coef_gas[NGAS] = {6.5000E-01, 6.5000E-01};
  qgas_avg[0] = 0.0;
  qgas_avg[1] = 0.0;
  {
    const real p_in_atm = pmid / 1.013e5;
    for (int g = 0; g < NGAS; ++g) {
      /* gas_diffusivity :223-240, mean_molecular_speed :242-253 */
      const real onethird = 1.0 / 3.0;
      const real dgas = (1.0e-3 * pow(temp, 1.75) * sqrt(1. / mw_gas[g] + 0.035)) /
                        (p_in_atm * pow((pow(vol_molar_gas[g], onethird) + 2.7189), 2.0));
      const real gas_diffus = dgas * 1.0e-4;
      const real speed = 145.5 * sqrt(temp / mw_gas[g]);
      const real freepath = 3.0 * gas_diffus / speed;
      real uptk[NMODE];
      gas_aer_uptkrates_1box1gas(accom_coef_gas[g], gas_diffus, freepath, dgn_awet, alnsg, uptk);
      for (int n = 0; n < NMODE; ++n)
        uptkaer[g][n] = uptk[n] * (qnum_cur[n] * aircon); /* all modes condense */
    }
    for (int n = 0; n < NMODE; ++n)
      uptkaer[0][n] = uptkaer[1][n] * 0.81;
    for (int n = 0; n < NMODE; ++n)
      *uptkrate_h2so4 += uptkaer[1][n];
  }
  const int niter = soaexch_1subarea(dtsubstep, temp, pmid, qgas_cur, qgas_avg, qaer_cur,
                                     (const real(*)[NMODE])uptkaer);
  /* H2SO4: quasi-analytic update (gasaerexch.hpp:486-537) */
  {
    const real qgas_prv = qgas_cur[1];
    real qaer_prv[NMODE];
    for (int n = 0; n < NMODE; ++n)
      qaer_prv[n] = qaer_cur[1][n];
    real tmpa = 0.0;
    for (int n = 0; n < NMODE; ++n)
      tmpa += uptkaer[1][n];
    const real kxt = tmpa * dtsubstep;
    const real pxt = qgas_netprod[1] * dtsubstep;
    const real q1 = qgas_prv;
    if (kxt >= 1.0e-20) {
      real q3, q4;
      if (kxt > 0.001) {
        const real pok = pxt / kxt;
        q3 = (q1 - pok) * exp(-kxt) + pok;
        q4 = (q1 - pok) * (1.0 - exp(-kxt)) / kxt + pok;
      } else {
        const real kxt2 = kxt * kxt;
        q3 = q1 * (1.0 - kxt + kxt2 * 0.5) + pxt * (1.0 - kxt * 0.5 + kxt2 / 6.0);
        q4 = q1 * (1.0 - kxt * 0.5 + kxt2 / 6.0) + pxt * (0.5 - kxt / 6.0 + kxt2 / 24.0);
      }
      qgas_cur[1] = q3;
      const real qdel = (q1 + pxt) - q3;
      qgas_avg[1] = q4;
      for (int n = 0; n < NMODE; ++n) {
        if (uptkaer[1][n] <= 0.0)
          continue;
        qaer_cur[1][n] = qaer_prv[n] + qdel * (uptkaer[1][n] / tmpa);
      }
    } else {
      qgas_cur[1] = q1 + pxt;
      qgas_avg[1] = q1 + pxt * 0.5;
    }
  }
  return niter;
}

/* gasaerexch.hpp:140-221 (the unit-tested single-gas form) */
ORC_FN void h2so4_nonvolatile(real dt, real netprod, const real uptk[NMODE], real *qgas_cur,
                              real *qgas_avg, real qaer_cur[NMODE]) {
  real qaer_prev[NMODE];
  for (int i = 0; i < NMODE; ++i)
    qaer_prev[i] = qaer_cur[i];
  real total = 0;
  for (int i = 0; i < NMODE; ++i)
    total += uptk[i];
  const real kxt = total * dt, pxt = netprod * dt, q0 = *qgas_cur;
  if (kxt < 1.0e-20) {
    *qgas_cur = q0 + pxt;
    *qgas_avg = q0 + pxt * 0.5;
    return;
  }
  real qend, qavg;
  if (kxt > 0.001) {
    const real qeq = pxt / kxt;
    qend = (q0 - qeq) * exp(-kxt) + qeq;
    qavg = (q0 - qeq) * (1.0 - exp(-kxt)) / kxt + qeq;
  } else {
    const real kxt2 = kxt * kxt;
    qend = q0 * (1.0 - kxt + kxt2 * 0.5) + pxt * (1.0 - kxt * 0.5 + kxt2 / 6.0);
    qavg = q0 * (1.0 - kxt * 0.5 + kxt2 / 6.0) + pxt * (0.5 - kxt / 6.0 + kxt2 / 24.0);
  }
  *qgas_cur = qend;
  *qgas_avg = qavg;
  const real qdel = (q0 + pxt) - qend;
  for (int n = 0; n < NMODE; ++n)
    if (0 < uptk[n])
      qaer_cur[n] = qaer_prev[n] + qdel * (uptk[n] / total);
}

/* ---------------------------------------------------------------- rename
 * rename.hpp:138-170, 225-390, 711-790 */
ORC_FN real tail_fraction(real diameter, real ln_cutoff, real fac, real ln_tail_fac, int use_tail) {
  const real ld = use_tail ? log(diameter) + ln_tail_fac : log(diameter);
  const real tail = (ln_cutoff - ld) * fac;
  return 0.5 * erfc(tail);
}

ORC_FN void rename_1subarea(int is_cloudy, real qnum_i[NMODE], real qaer_i[NAER][NMODE],
                            const real qdel_i[NAER][NMODE], real qnum_c[NMODE],
                            real qaer_c[NAER][NMODE], const real qdel_c[NAER][NMODE]) {
  /* find_renaming_pairs (rename.hpp:393-476) for the only pair aitken->acc */
  const int src = 1, dest = 0;
  const real sqrt_half = sqrt(0.5), frelax = 27.0;
  const real alnsg = log(MODE_SIG[src]);
  const real fmode_dist_tail_fac = sqrt_half / alnsg;
  const real v2n_lo_rlx =
      1.0 / mean_particle_volume_from_diameter(MODE_DMIN[src], MODE_SIG[src]) * frelax;
  const real v2n_hi_rlx =
      1.0 / mean_particle_volume_from_diameter(MODE_DMAX[src], MODE_SIG[src]) / frelax;
  const real ln_tail_fac = 3.0 * square(alnsg);
  const real alnsg_dest = log(MODE_SIG[dest]);
  const real cutoff = sqrt(MODE_DNOM[src] * exp(1.5 * square(alnsg)) * MODE_DNOM[dest] *
                           exp(1.5 * square(alnsg_dest)));
  const real ln_cutoff = log(cutoff);
  const real threshold = 0.99 * cutoff;
  const real smallest = 1.0e-25;
  /* compute_dryvol_change_in_src_mode (rename.hpp:23-62) */
  real dv_i = 0.0, ddv_i = 0.0, dv_c = 0.0, ddv_c = 0.0;
  {
    real t = 0.0, td = 0.0;
    for (int s = 0; s < NAER; ++s) {
      t += qaer_i[s][src] * MASS_2_VOL[s];
      td += qdel_i[s][src] * MASS_2_VOL[s];
    }
    dv_i = t - td;
    ddv_i = td;
  }
  if (is_cloudy) {
    real t = 0.0, td = 0.0;
    for (int s = 0; s < NAER; ++s) {
      t += qaer_c[s][src] * MASS_2_VOL[s];
      td += qdel_c[s][src] * MASS_2_VOL[s];
    }
    dv_c = t - td;
    ddv_c = td;
  }
  /* do_inter_mode_transfer (rename.hpp:225-390) */
  real b4_dv = dv_i;
  if (is_cloudy)
    b4_dv = b4_dv + dv_c;
  const real b4_dv_b = rmax(b4_dv, smallest);
  real b4_n = qnum_i[src];
  if (is_cloudy)
    b4_n = b4_n + qnum_c[src];
  b4_n = rmax(0.0, b4_n);
  const real b4_n_b = min_max_bound(b4_dv_b * v2n_hi_rlx, b4_dv_b * v2n_lo_rlx, b4_n);
  real del = ddv_i;
  if (is_cloudy)
    del = del + ddv_c;
  const real aft_dv = b4_dv + del;
  if (aft_dv <= smallest)
    return;
  real b4_d = mean_particle_diameter_from_volume(b4_dv_b / b4_n_b, MODE_SIG[src]);
  if (b4_d > threshold) {
    b4_dv = b4_dv * cube(threshold / b4_d);
    b4_d = threshold;
  }
  if ((aft_dv - b4_dv) <= 1.0e-6 * b4_dv_b)
    return;
  const real aft_d = mean_particle_diameter_from_volume(aft_dv / b4_n_b, MODE_SIG[src]);
  if (aft_d <= MODE_DNOM[src])
    return;
  const real b4_tn = tail_fraction(b4_d, ln_cutoff, fmode_dist_tail_fac, 0, 0);
  const real b4_tv = tail_fraction(b4_d, ln_cutoff, fmode_dist_tail_fac, ln_tail_fac, 1);
  const real aft_tn = tail_fraction(aft_d, ln_cutoff, fmode_dist_tail_fac, 0, 0);
  const real aft_tv = tail_fraction(aft_d, ln_cutoff, fmode_dist_tail_fac, ln_tail_fac, 1);
  /* compute_xfer_fractions (rename.hpp:164-202) */
  const real xferfrac_max = 1.0 - 10.0 * EPS;
  const real vfrac = aft_tv * aft_dv - b4_tv * b4_dv;
  if (vfrac <= 0.0)
    return;
  real xv = rmin(vfrac, aft_dv) / aft_dv;
  xv = rmin(xv, xferfrac_max);
  real xn = aft_tn - b4_tn;
  xn = rmax(0.0, rmin(xn, xv));
  /* do_num_and_mass_transfer (rename.hpp:204-223) */
  {
    const real nt = qnum_i[src] * xn;
    qnum_i[src] -= nt;
    qnum_i[dest] += nt;
    for (int s = 0; s < NAER; ++s) {
      const real vt = qaer_i[s][src] * xv;
      qaer_i[s][src] -= vt;
      qaer_i[s][dest] += vt;
    }
  }
  if (is_cloudy) {
    const real nt = qnum_c[src] * xn;
    qnum_c[src] -= nt;
    qnum_c[dest] += nt;
    for (int s = 0; s < NAER; ++s) {
      const real vt = qaer_c[s][src] * xv;
      qaer_c[s][src] -= vt;
      qaer_c[s][dest] += vt;
    }
  }
}

/* ------------------------------------------------------------ nucleation
 * nucleation.hpp:38-118 (pbl_nuc_wang2008), :128-160 (binary), :347-860
 * (mer07_veh02_nuc_mosaic_1box), vehkamaki2002.hpp:54-190 */
ORC_FN real veh02_x_crit(real n_a, real t, real rh) {
  return 0.740997 - 0.00266379 * t - 0.00349998 * log(n_a) + 0.0000504022 * t * log(n_a) +
         0.00201048 * log(rh) - 0.000183289 * t * log(rh) + 0.00157407 * square(log(rh)) -
         0.0000179059 * t * square(log(rh)) + 0.000184403 * cube(log(rh)) -
         1.50345e-6 * t * cube(log(rh));
}
ORC_FN real veh02_log_rate(real n_a, real t, real rh, real x) {
  const real a = 0.14309 + 2.21956 * t - 0.0273911 * square(t) + 0.0000722811 * cube(t) + 5.91822 / x;
  const real b = 0.117489 + 0.462532 * t - 0.0118059 * square(t) + 0.0000404196 * cube(t) + 15.7963 / x;
  const real c = -0.215554 - 0.0810269 * t + 0.00143581 * square(t) - 4.7758e-6 * cube(t) - 2.91297 / x;
  const real d = -3.58856 + 0.049508 * t - 0.00021382 * square(t) + 3.10801e-7 * cube(t) - 0.0293333 / x;
  const real e = 1.14598 - 0.600796 * t + 0.00864245 * square(t) - 0.0000228947 * cube(t) - 8.44985 / x;
  const real f = 2.15855 + 0.0808121 * t - 0.000407382 * square(t) - 4.01957e-7 * cube(t) + 0.721326 / x;
  const real g = 1.6241 - 0.0160106 * t + 0.0000377124 * square(t) + 3.21794e-8 * cube(t) - 0.0113255 / x;
  const real h = 9.71682 - 0.115048 * t + 0.000157098 * square(t) + 4.00914e-7 * cube(t) + 0.71186 / x;
  const real i = -1.05611 + 0.00903378 * t - 0.0000198417 * square(t) + 2.46048e-8 * cube(t) - 0.0579087 / x;
  const real j = -0.148712 + 0.00283508 * t - 9.24619e-6 * square(t) + 5.00427e-9 * cube(t) - 0.0127081 / x;
  return a + b * log(rh) + c * square(log(rh)) + d * cube(log(rh)) + e * log(n_a) +
         f * log(rh) * log(n_a) + g * square(log(rh)) * (log(n_a)) + h * square(log(n_a)) +
         i * log(rh) * square(log(n_a)) + j * cube(log(n_a));
}
ORC_FN real veh02_ntot(real n_a, real t, real rh, real x) {
  const real A = -0.00295413 - 0.0976834 * t + 0.00102485 * square(t) - 2.18646e-6 * cube(t) - 0.101717 / x;
  const real B = -0.00205064 - 0.00758504 * t + 0.000192654 * square(t) - 6.7043e-7 * cube(t) - 0.255774 / x;
  const real C = +0.00322308 + 0.000852637 * t - 0.0000154757 * square(t) + 5.66661e-8 * cube(t) + 0.0338444 / x;
  const real D = +0.0474323 - 0.000625104 * t + 2.65066e-6 * square(t) - 3.67471e-9 * cube(t) - 0.000267251 / x;
  const real E = -0.0125211 + 0.00580655 * t - 0.000101674 * square(t) + 2.88195e-7 * cube(t) + 0.0942243 / x;
  const real F = -0.038546 - 0.000672316 * t + 2.60288e-6 * square(t) + 1.19416e-8 * cube(t) - 0.00851515 / x;
  const real G = -0.0183749 + 0.000172072 * t - 3.71766e-7 * square(t) - 5.14875e-10 * cube(t) + 0.00026866 / x;
  const real H = -0.0619974 + 0.000906958 * t - 9.11728e-7 * square(t) - 5.36796e-9 * cube(t) - 0.00774234 / x;
  const real I = +0.0121827 - 0.00010665 * t + 2.5346e-7 * square(t) - 3.63519e-10 * cube(t) + 0.000610065 / x;
  const real J = +0.000320184 - 0.0000174762 * t + 6.06504e-8 * square(t) - 1.4177e-11 * cube(t) + 0.000135751 / x;
  return exp(A + B * log(rh) + C * square(log(rh)) + D * cube(log(rh)) + E * log(n_a) +
             F * log(rh) * log(n_a) + G * square(log(rh)) * log(n_a) + H * square(log(n_a)) +
             I * log(rh) * square(log(n_a)) + J * cube(log(n_a)));
}
ORC_FN real veh02_radius(real x, real ntot) {
  return exp(-1.6524245 + 0.42316402 * x + 0.3346648 * log(ntot));
}

/* mer07_veh02_nuc_mosaic_1box with newnuc_method_flagaa = 11, nsize = 1,
 * no NH3 (mam4_amicphys.hpp:965-995); outputs qnuma_del, qso4a_del */
ORC_FN void nuc_mosaic_1box(real dtnuc, real temp_in, real rh_in, real press_in, real zm_in,
                            real pblh_in, real qh2so4_cur, real qh2so4_avg,
                            real h2so4_uptkrate, real mw_so4a_host, real dp_lo, real dp_hi,
                            real rgas, real avogad, real mw_nh4a, real mw_so4a,
                            real *qnuma_del, real *qso4a_del) {
  const real onethird = 1.0 / 3.0, accom_coef_h2so4 = 0.65;
  const real dens_ammsulf = 1770.0, dens_ammbisulf = 1770.0, dens_sulfacid = 1770.0;
  const real mw_ammsulf = 132.0, mw_ammbisulf = 114.0, mw_sulfacid = 96.0;
  const real qnh3_cur = 0.0;
  *qnuma_del = 0.0;
  *qso4a_del = 0.0;
  const real cair = press_in / (temp_in * rgas);
  const real so4vol_in = qh2so4_avg * cair * avogad * 1.0e-6;
  real ratenuclt = 1.0e-38;
  real rateloge = log(ratenuclt);
  real cnum_h2so4 = 0.0, cnum_tot = 0.0, radius_cluster = 0.0, cnum_nh3 = 0.0;
  if (so4vol_in >= 1.0e4) {
    const real temp_bb = rmax(230.15, rmin(305.15, temp_in));
    const real rh_bb = rmax(1.0e-4, rmin(1.0, rh_in));
    const real so4vol_bb = rmax(1.0e4, rmin(1.0e11, so4vol_in));
    const real x_crit = veh02_x_crit(so4vol_bb, temp_bb, rh_bb);
    rateloge = veh02_log_rate(so4vol_bb, temp_bb, rh_bb, x_crit);
    ratenuclt = exp(rmin(rateloge, log(1e38)));
    cnum_tot = veh02_ntot(so4vol_bb, temp_bb, rh_bb, x_crit);
    cnum_h2so4 = cnum_tot * x_crit;
    radius_cluster = veh02_radius(x_crit, cnum_tot);
  }
  cnum_nh3 = 0.0;
  rateloge = rateloge + log(rmax(1.0e-38, 1.0));
  if (zm_in <= rmax(pblh_in, 100.0)) {
    /* pbl_nuc_wang2008 first order (wang2008.hpp:23) */
    real tmp_ratenucl = 1e-6 * so4vol_in;
    tmp_ratenucl = tmp_ratenucl * 1.0;
    const real tmp_rateloge = log(rmax(1.0e-38, tmp_ratenucl));
    if (!(tmp_rateloge <= rateloge)) {
      rateloge = tmp_rateloge;
      ratenuclt = tmp_ratenucl;
      radius_cluster = 0.5;
      const real tmp_diam = radius_cluster * 2.0e-7;
      const real tmp_volu = cube(tmp_diam) * (PI / 6.0);
      const real tmp_mass = tmp_volu * 1.8;
      cnum_h2so4 = (tmp_mass / 98.0) * 6.023e23;
      cnum_nh3 = 0.0;
      cnum_tot = cnum_h2so4;
    }
  }
  if (rateloge <= -13.82)
    return;
  ratenuclt = exp(rateloge);
  const real ratenuclt_bb = ratenuclt * 1.0e6;
  real tmpa = rmax(0.10, rmin(0.95, rh_in));
  const real wetvol_dryvol = 1.0 - 0.56 / log(tmpa);
  real voldry_clus = (rmax(cnum_h2so4, 1.0) * mw_so4a + cnum_nh3 * mw_nh4a) /
                     (1.0e3 * dens_sulfacid * avogad);
  voldry_clus = voldry_clus * (mw_so4a_host / mw_so4a);
  const real dpdry_clus = pow(voldry_clus * 6.0 / PI, onethird);
  int igrow;
  real dpdry_part = dp_lo;
  if (dpdry_clus <= dp_lo) {
    igrow = 1;
  } else if (dpdry_clus >= dp_hi) {
    igrow = 0;
    dpdry_part = dp_hi;
  } else {
    return; /* cluster between the bin bounds: nucleation.hpp:620-631 */
  }
  const real voldry_part = (PI / 6.0) * pow(dpdry_part, 3);
  real n1 = 0.0, n2 = 0.0, n3 = 0.0;
  if (igrow <= 0) {
    n3 = 1.0;
  } else if (qnh3_cur >= qh2so4_cur) {
    n1 = (qnh3_cur / qh2so4_cur) - 1.0;
    n1 = rmax(0.0, rmin(1.0, n1));
    n2 = 1.0 - n1;
  } else {
    n2 = (qnh3_cur / qh2so4_cur);
    n2 = rmax(0.0, rmin(1.0, n2));
    n3 = 1.0 - n2;
  }
  const real m1 = n1 * mw_ammsulf, m2 = n2 * mw_ammbisulf, m3 = n3 * mw_sulfacid;
  const real dens_part =
      (m1 + m2 + m3) / ((m1 / dens_ammsulf) + (m2 / dens_ammbisulf) + (m3 / dens_sulfacid));
  const real mass_part = voldry_part * dens_part;
  const real molenh4a_per_moleso4a = 2.0 * n1 + n2;
  real kgaero_per_moleso4a = 1.0e-3 * (m1 + m2 + m3);
  kgaero_per_moleso4a = kgaero_per_moleso4a * (mw_so4a_host / mw_so4a);
  real tmpb = 1.0 + molenh4a_per_moleso4a * 17.0 / 98.0;
  const real wet_volfrac_so4a = 1.0 / (wetvol_dryvol * tmpb);
  real factor_kk;
  if (igrow <= 0) {
    factor_kk = 1.0;
  } else {
    const real tmp_spd = 14.7 * sqrt(temp_in);
    const real gr_kk =
        3.0e-9 * tmp_spd * mw_sulfacid * so4vol_in / (dens_part * wet_volfrac_so4a);
    const real dfin_kk = 1.0e9 * dpdry_part * pow(wetvol_dryvol, onethird);
    real dnuc_kk = 2.0 * radius_cluster;
    dnuc_kk = rmax(dnuc_kk, 1.0);
    const real gamma_kk = 0.23 * pow(dnuc_kk, 0.2) * pow(dfin_kk / 3.0, 0.075) *
                          pow(dens_part * 1.0e-3, -0.33) * pow(temp_in / 293.0, -0.75);
    tmpa = h2so4_uptkrate * 3600.0;
    tmpa = rmax(tmpa, 0.0);
    tmpb = 6.7037e-6 * pow(temp_in, 0.75) / cair;
    tmpb = tmpb * 3600.0;
    const real cs_prime_kk = tmpa / (4.0 * PI * tmpb * accom_coef_h2so4);
    const real nu_kk = gamma_kk * cs_prime_kk / gr_kk;
    factor_kk = exp((nu_kk / dfin_kk) - (nu_kk / dnuc_kk));
  }
  const real ratenuclt_kk = ratenuclt_bb * factor_kk;
  tmpa = rmax(0.0, (ratenuclt_kk * dtnuc * mass_part));
  const real qmolso4a_del_max = tmpa / (kgaero_per_moleso4a * cair);
  real freducea = 1.0;
  if (qmolso4a_del_max > qh2so4_cur)
    freducea = qh2so4_cur / qmolso4a_del_max;
  real freduceb = 1.0;
  if (molenh4a_per_moleso4a >= 1.0e-10) {
    const real qmolnh4a_del_max = qmolso4a_del_max * molenh4a_per_moleso4a;
    if (qmolnh4a_del_max > qnh3_cur)
      freduceb = qnh3_cur / qmolnh4a_del_max;
  }
  const real freduce = rmin(freducea, freduceb);
  if ((freduce * ratenuclt_kk) <= 1.0e-12)
    return;
  tmpa = 0.9999;
  real qh2so4_del = rmin(tmpa * qh2so4_cur, freduce * qmolso4a_del_max);
  real qnh3_del = rmin(tmpa * qnh3_cur, qh2so4_del * molenh4a_per_moleso4a);
  qh2so4_del = -qh2so4_del;
  qnh3_del = -qnh3_del;
  *qso4a_del = -qh2so4_del;
  const real qnh4a_del = -qnh3_del;
  *qnuma_del = 1.0e-3 * (*qso4a_del * mw_so4a + qnh4a_del * mw_nh4a) / mass_part;
}

/* mam4_amicphys.hpp:917-1094 */
ORC_FN void newnuc_1subarea(real deltat, real temp, real pmid, real zmid, real pblh,
                            real relhum, real uptkrate_h2so4, real qgas_cur[NGAS],
                            const real qgas_avg[NGAS], real qnum_cur[NMODE],
                            real qaer_cur[NAER][NMODE]) {
  const real qh2so4_cutoff = 4.0e-16;
  const real qh2so4_cur = qgas_cur[1];
  const real qh2so4_avg = qgas_avg[1];
  if (qh2so4_avg <= qh2so4_cutoff)
    return;
  const int nait = 1;
  const real dplom = exp(0.67 * log(MODE_DMIN[nait]) + 0.33 * log(MODE_DNOM[nait]));
  const real dphim = MODE_DMAX[nait];
  real tmpa = 1770.0 * PI / 6.0;
  const real mass1p_aitlo = tmpa * (pow(dplom, 3.0));
  const real mass1p_aithi = tmpa * (pow(dphim, 3.0));
  const real relhumnn = rmax(0.01, rmin(0.99, relhum));
  const real mw_so4a_host = 115, mwnh4 = 18, mwso4 = 96;
  const real rgas = 8.31446759100000, avogadro = 6.022140000000000E+023;
  real qnuma_del, qso4a_del;
  nuc_mosaic_1box(deltat, temp, relhumnn, pmid, zmid, pblh, qh2so4_cur, qh2so4_avg,
                  uptkrate_h2so4, mw_so4a_host, dplom, dphim, rgas, avogadro, mwnh4, mwso4,
                  &qnuma_del, &qso4a_del);
  qnuma_del = qnuma_del * 1.0e3;
  real dndt_ait = qnuma_del / deltat;
  tmpa = qso4a_del * mw_so4a_host;
  const real tmpb = tmpa;
  const real tmp_frso4 = 1.0;
  real dmdt_ait = rmax(0.0, (tmpb / deltat));
  if (dndt_ait < 1.0e2) {
    dndt_ait = 0.0;
    dmdt_ait = 0.0;
  } else {
    const real mass1p = dmdt_ait / dndt_ait;
    if (mass1p < mass1p_aitlo)
      dndt_ait = dmdt_ait / mass1p_aitlo;
    else if (mass1p > mass1p_aithi)
      dmdt_ait = dndt_ait * mass1p_aithi;
  }
  dndt_ait = dndt_ait * 1;
  dmdt_ait = dmdt_ait * 1;
  real tmp_q_del = dndt_ait * deltat;
  qnum_cur[nait] = qnum_cur[nait] + tmp_q_del;
  const real dso4dt_ait = dmdt_ait * tmp_frso4 / mw_so4a_host;
  if (dso4dt_ait > 0.0) {
    tmp_q_del = dso4dt_ait * deltat;
    qaer_cur[1][nait] = qaer_cur[1][nait] + tmp_q_del;
    tmp_q_del = rmin(tmp_q_del, qgas_cur[1]);
    qgas_cur[1] = qgas_cur[1] - tmp_q_del;
  }
}

/* ---------------------------------------------------------- coagulation
 * coagulation.hpp:298-817, 850-1119 */
ORC_FN void getcoags_wrapper(real airtemp, real airprs, real dgatk, real dgacc, real sgatk,
                             real sgacc, real xxlsgat, real xxlsgac, real pdensat,
                             real pdensac, real *betaij0, real *betaij3, real *betaii0,
                             real *betajj0) {
  const real t0 = 273.15 + 15.0;
  const real sqrt_temp = sqrt(airtemp);
  const real lamda = 6.6328e-8 * 101325.0 * airtemp / (t0 * airprs);
  const real amu = 1.458e-6 * airtemp * sqrt_temp / (airtemp + 110.4);
  const real boltzmann = 1.3806500000000000e-023;
  const real knc = (2.0 / 3.0) * boltzmann * airtemp / amu;
  const real kfmat = sqrt(3.0 * boltzmann * airtemp / pdensat);
  const real kfmac = sqrt(3.0 * boltzmann * airtemp / pdensac);
  const real kfmatac = sqrt(6.0 * boltzmann * airtemp / (pdensat + pdensac));
  /* getcoags (coagulation.hpp:651-748) */
  const real a = 1.246;
  const real esat01 = exp(0.125 * xxlsgat * xxlsgat);
  const real esac01 = exp(0.125 * xxlsgac * xxlsgac);
  const real sqrttwo = sqrt(2.0);
  const real dlgsqt2 = 1.0 / log(sqrttwo);
  const real esat04 = pow(esat01, 4.0), esac04 = pow(esac01, 4.0);
  const real esat05 = esat04 * esat01, esac05 = esac04 * esac01;
  const real esat08 = esat04 * esat04, esac08 = esac04 * esac04;
  const real esat09 = esat08 * esat01, esac09 = esac08 * esac01;
  const real esat16 = esat08 * esat08, esac16 = esac08 * esac08;
  const real esat20 = esat16 * esat04, esac20 = esac16 * esac04;
  const real esat24 = esat20 * esat04;
  const real esat25 = esat20 * esat05, esac25 = esac20 * esac05;
  const real esat36 = esat20 * esat16;
  const real esat49 = esat24 * esat25;
  const real esat64 = esat20 * esat20 * esat24;
  const real esat100 = esat64 * esat36;
  const real dgat3 = dgatk * dgatk * dgatk;
  const real sqdgat = sqrt(dgatk), sqdgac = sqrt(dgacc);
  const real sqdgat7 = dgat3 * sqdgat;
  const real r1 = sqdgac / sqdgat;
  const real r2 = r1 * r1;
  const real rx4 = r2 * r2;
  const real ri1 = 1.0 / r1;
  const real ri2 = 1.0 / (r1 * r1);
  const real ri3 = 1.0 / (r1 * r1 * r1);
  const real kngat = 2.0 * lamda / dgatk;
  const real kngac = 2.0 * lamda / dgacc;
  const real rat = dgacc / dgatk;
  const int n2n = (int)rmax(1, rmin(10, round(4.0 * (sgatk - 0.75)))) - 1;
  const int n2a = (int)rmax(1, rmin(10, round(4.0 * (sgacc - 0.75)))) - 1;
  const int n1 = (int)rmax(1, rmin(10, 1 + round(dlgsqt2 * log(rat)))) - 1;
  /* table lookups take (n1, n2n, n2a) into [n1][n2a'][n2n'] (the call
   * passes n2n in the n2a slot, coagulation.hpp:309, 558) */
  const real bm0ij = kCoagBm0ij[n1 * 100 + n2n * 10 + n2a];
  const real bm3i = kCoagBm3i[n1 * 100 + n2n * 10 + n2a];
  /* intermodal 0th moment :298-327 */
  const real coagnc0 = knc * (2.0 + a * (kngat * (esat04 + r2 * esat16 * esac04) +
                                         kngac * (esac04 + ri2 * esac16 * esat04)) +
                              (r2 + ri2) * esat04 * esac04);
  const real coagfm0 = kfmatac * sqdgat * bm0ij *
                       (esat01 + r1 * esac01 + 2.0 * r2 * esat01 * esac04 +
                        rx4 * esat09 * esac16 + ri3 * esat16 * esac09 + 2.0 * ri1 * esat04 +
                        esac01);
  const real qn12 = coagnc0 * coagfm0 / (coagnc0 + coagfm0);
  /* intermodal 3rd moment :549-579 */
  const real coagnc3 =
      knc * dgat3 *
      (2.0 * esat36 + a * kngat * (esat16 + r2 * esat04 * esac04) +
       a * kngac * (esat36 * esac04 + ri2 * esat64 * esac16) + r2 * esat16 * esac04 +
       ri2 * esat64 * esac04);
  const real coagfm3 = kfmatac * sqdgat7 * bm3i *
                       (esat49 + r1 * esat36 * esac01 + 2.0 * r2 * esat25 * esac04 +
                        rx4 * esat09 * esac16 + ri3 * esat100 * esac09 +
                        2.0 * ri1 * esat64 * esac01);
  const real qv12 = coagnc3 * coagfm3 / (coagnc3 + coagfm3);
  /* intramodal 0th moment :582-610 */
  const real cnc11 = knc * (1.0 + esat08 + a * kngat * (esat20 + esat04));
  const real cfm11 = kfmat * sqdgat * kCoagBm0[n2n] * (esat01 + esat25 + 2.0 * esat05);
  const real qn11 = cfm11 * cnc11 / (cfm11 + cnc11);
  const real cnc22 = knc * (1.0 + esac08 + a * kngac * (esac20 + esac04));
  const real cfm22 = kfmac * sqdgac * kCoagBm0[n2a] * (esac01 + esac25 + 2.0 * esac05);
  const real qn22 = cfm22 * cnc22 / (cfm22 + cnc22);
  *betaii0 = rmax(0.0, qn11);
  *betajj0 = rmax(0.0, qn22);
  *betaij0 = rmax(0.0, qn12);
  const real dumatk3 = (cube(dgatk) * exp(4.5 * xxlsgat * xxlsgat));
  *betaij3 = rmax(0.0, qv12 / dumatk3);
}

ORC_FN void qnum_intra_inter(real bijdtqnumj, real biidt, real qnumi_bgn, real *qnumi_end) {
  if (bijdtqnumj < 1.0e-5) {
    *qnumi_end = qnumi_bgn / (1.0 + (bijdtqnumj + biidt * qnumi_bgn) * (1.0 + 0.5 * bijdtqnumj));
  } else {
    const real tmp_exp = exp(-bijdtqnumj);
    *qnumi_end =
        qnumi_bgn * tmp_exp / (1.0 + (biidt * qnumi_bgn / bijdtqnumj) * (1.0 - tmp_exp));
  }
}

ORC_FN void coag_1subarea(real deltat, real temp, real pmid, real aircon,
                          const real dgn_awet[NMODE], const real wetdens[NMODE],
                          real qnum_cur[NMODE], real qaer_cur[NAER][NMODE],
                          real qaer_del_coag_out[NAER]) {
  const int nacc = 0, nait = 1, npca = 3;
  real qaer_bgn[NAER][NMODE], qnum_bgn[NMODE];
  for (int s = 0; s < NAER; ++s)
    for (int m = 0; m < NMODE; ++m) {
      qaer_cur[s][m] = rmax(0.0, qaer_cur[s][m]);
      qaer_bgn[s][m] = qaer_cur[s][m];
    }
  for (int m = 0; m < NMODE; ++m) {
    qnum_cur[m] = rmax(0.0, qnum_cur[m]);
    qnum_bgn[m] = qnum_cur[m];
  }
  const int srcm[3] = {nait, npca, nait}, dstm[3] = {nacc, nacc, npca};
  real bij0[3], bij3[3], bii0[3], bjj0[3];
  for (int p = 0; p < 3; ++p) {
    const real ss = MODE_SIG[srcm[p]], sd = MODE_SIG[dstm[p]];
    getcoags_wrapper(temp, pmid, dgn_awet[srcm[p]], dgn_awet[dstm[p]], ss, sd, log(ss), log(sd),
                     wetdens[srcm[p]], wetdens[dstm[p]], &bij0[p], &bij3[p], &bii0[p],
                     &bjj0[p]);
  }
  for (int p = 0; p < 3; ++p) {
    bij0[p] *= aircon;
    bij3[p] *= aircon;
    bii0[p] *= aircon;
    bjj0[p] *= aircon;
  }
  /* mam_coag_num_update :982-1027 */
  real qnum_tavg[NMODE];
  qnum_cur[nacc] = qnum_bgn[nacc] / (1.0 + bjj0[0] * deltat * qnum_bgn[nacc]);
  qnum_tavg[nacc] = (qnum_bgn[nacc] + qnum_cur[nacc]) * 0.5;
  {
    const real bijdtqnumj = rmax(0.0, deltat * bij0[1] * qnum_tavg[nacc]);
    const real biidt = rmax(0.0, deltat * bii0[1]);
    qnum_intra_inter(bijdtqnumj, biidt, qnum_bgn[npca], &qnum_cur[npca]);
    qnum_tavg[npca] = (qnum_bgn[npca] + qnum_cur[npca]) * 0.5;
  }
  {
    real bijqnumj = bij0[0] * qnum_tavg[nacc];
    bijqnumj = bijqnumj + bij0[2] * qnum_tavg[npca];
    const real bijdtqnumj = rmax(0.0, deltat * bijqnumj);
    const real biidt = rmax(0.0, deltat * bii0[0]);
    qnum_intra_inter(bijdtqnumj, biidt, qnum_bgn[nait], &qnum_cur[nait]);
    qnum_tavg[nait] = (qnum_bgn[nait] + qnum_cur[nait]) * 0.5;
  }
  /* mam_coag_aer_update :850-930 */
  for (int s = 0; s < NAER; ++s)
    qaer_del_coag_out[s] = 0.0;
  const real bq1 = rmax(0.0, bij3[0] * qnum_tavg[nacc]);
  const real bq2 = rmax(0.0, bij3[2] * qnum_tavg[npca]);
  real decay_const = bq1 + bq2;
  const real eps2 = EPS * 2.0;
  real decay_factor = deltat * decay_const;
  if (decay_factor > eps2) {
    const real prtn2 = bq2 / decay_const;
    const real prtn1 = 1.0 - prtn2;
    const real xf = 1.0 - exp(-decay_factor);
    for (int s = 0; s < NAER; ++s) {
      const real dq = xf * qaer_bgn[s][nait];
      qaer_cur[s][nait] -= dq;
      qaer_cur[s][nacc] += dq * prtn1;
      qaer_cur[s][npca] += dq * prtn2;
      qaer_del_coag_out[s] += dq * prtn2;
    }
  }
  decay_const = rmax(0.0, bij3[1] * qnum_tavg[nacc]);
  decay_factor = deltat * decay_const;
  if (decay_factor > eps2) {
    const real xf = 1.0 - exp(-decay_factor);
    for (int s = 0; s < NAER; ++s) {
      const real dq = xf * qaer_bgn[s][npca];
      qaer_cur[s][npca] -= dq;
      qaer_cur[s][nacc] += dq;
    }
  }
}

/* ------------------------------------------------------------------ aging
 * aging.hpp:70-361 */
ORC_FN void pcarbon_aging_1subarea(unsigned n_so4_monolayers, const real dgn_a[NMODE],
                                   real qnum_cur[NMODE], real qnum_del_cond[NMODE],
                                   real qnum_del_coag[NMODE], real qaer_cur[NAER][NMODE],
                                   real qaer_del_cond[NAER][NMODE],
                                   real qaer_del_coag[NAER][NMODE],
                                   const real qaer_del_coag_in[NAER]) {
  const int pc = 3, acc = 0, so4 = 1, soa = 0;
  const real mw_soa = 150 / 1000.0, mw_so4 = 115 / 1000.0;
  const real so4_vol = mw_so4 * 1000.0 / AERO_DENS[so4];
  const real soa_vol = mw_soa * 1000.0 / AERO_DENS[soa];
  const real hygro_soa = 0.14000000000000001, hygro_so4 = 0.50700000000000001;
  const real fac = soa_vol * hygro_soa / hygro_so4;
  const real vol_shell = qaer_cur[so4][pc] * so4_vol + qaer_cur[soa][pc] * fac;
  real dcond = qaer_del_cond[so4][pc] * so4_vol + qaer_del_cond[soa][pc] * fac;
  const real dcoag = qaer_del_coag_in[so4] * so4_vol + qaer_del_coag_in[soa] * fac;
  dcond = rmax(dcond, 1e-35);
  const real frac_cond = dcond / (dcond + rmax(dcoag, 0.0));
  const real frac_coag = 1.0 - frac_cond;
  real vol_core = 0.0;
  for (int s = 0; s < NAER; ++s)
    if (LMAP_AER[s][pc] > 0)
      vol_core += qaer_cur[s][pc] * MASS_2_VOL[s];
  const real fac_volsfc = exp(2.5 * square(log(MODE_SIG[pc])));
  const real xferfrac_max = 1.0 - 10.0 * EPS;
  const real tmp1 = vol_shell * dgn_a[pc] * fac_volsfc;
  const real dr = n_so4_monolayers * 4.76e-10;
  const real tmp2 = rmax(6.0 * dr * vol_core, 0.0);
  real xferfrac;
  if (tmp1 >= tmp2)
    xferfrac = xferfrac_max;
  else
    xferfrac = rmin(tmp1 / tmp2, xferfrac_max);
  const int to_acc[3] = {2, 3, 6};     /* POM, BC, MOM */
  const int all_to_acc[4] = {0, 1, 4, 5}; /* SOA, SO4, NaCl, DST */
  for (int k = 0; k < 3; ++k) {
    const int s = to_acc[k];
    const real q = qaer_cur[s][pc] * xferfrac;
    qaer_cur[s][pc] -= q;
    qaer_cur[s][acc] += q;
    qaer_del_cond[s][pc] -= q * frac_cond;
    qaer_del_cond[s][acc] += q * frac_cond;
    qaer_del_coag[s][pc] -= q * frac_coag;
    qaer_del_coag[s][acc] += q * frac_coag;
  }
  for (int k = 0; k < 4; ++k) {
    const int s = all_to_acc[k];
    qaer_cur[s][acc] += qaer_cur[s][pc];
    qaer_del_cond[s][acc] += qaer_del_cond[s][pc];
    qaer_del_coag[s][acc] += qaer_del_coag[s][pc];
    qaer_cur[s][pc] = 0.0;
    qaer_del_cond[s][pc] = 0.0;
    qaer_del_coag[s][pc] = 0.0;
  }
  {
    const real q = qnum_cur[pc] * xferfrac;
    qnum_cur[pc] -= q;
    qnum_cur[acc] += q;
    qnum_del_cond[pc] -= q * frac_cond;
    qnum_del_cond[acc] += q * frac_cond;
    qnum_del_coag[pc] -= q * frac_coag;
    qnum_del_coag[acc] += q * frac_coag;
  }
}

/* ----------------------------------------------------- one subarea
 * mam4_amicphys.hpp:1127-1697 */
typedef struct {
  int do_cond, do_rename, do_newnuc, do_coag, optaa;
} sub_flags;

ORC_FN int amicphys_1subarea(const sub_flags *f, real deltat, int iscldy, unsigned nmono,
                             real temp, real pmid, real zmid, real pblh, real relhum,
                             const real dgn_a[NMODE], const real dgn_awet[NMODE],
                             const real wetdens[NMODE], const real qgas1[NGAS],
                             const real qgas3[NGAS], real qgas_cur[NGAS],
                             real qgas_delaa[NGAS][NQTEND], const real qnum3[NMODE],
                             real qnum_cur[NMODE], real qnum_delaa[NMODE][NQTEND],
                             const real qaer2[NAER][NMODE], const real qaer3[NAER][NMODE],
                             real qaer_cur[NAER][NMODE], real qaer_delaa[NAER][NMODE][NQTEND],
                             const real qnumcw3[NMODE], real qnumcw_cur[NMODE],
                             real qnumcw_delaa[NMODE], const real qaercw2[NAER][NMODE],
                             const real qaercw3[NAER][NMODE], real qaercw_cur[NAER][NMODE],
                             real qaercw_delaa[NAER][NMODE]) {
  const real r_universal = 8314.46759100000;
  const real aircon = pmid / (r_universal * temp);
  int niter = 0;
  for (int g = 0; g < NGAS; ++g)
    qgas_cur[g] = qgas3[g];
  for (int s = 0; s < NAER; ++s)
    for (int m = 0; m < NMODE; ++m)
      qaer_cur[s][m] = qaer3[s][m];
  for (int m = 0; m < NMODE; ++m)
    qnum_cur[m] = qnum3[m];
  if (iscldy) {
    for (int m = 0; m < NMODE; ++m)
      qnumcw_cur[m] = qnumcw3[m];
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaercw_cur[s][m] = qaercw3[s][m];
  }
  real qgas_netprod[NGAS] = {0.0, 0.0};
  if (f->do_cond && f->optaa == 2) {
    /* only H2SO4 (igas 1); igas_nh3 = -1 */
    qgas_netprod[1] = (qgas3[1] - qgas1[1]) / deltat;
    qgas_cur[1] = (qgas_netprod[1] >= 0) ? qgas1[1] : 0;
  }
  const int dtsubstep_i = (int)(deltat / 1);
  const real dtsub = (real)dtsubstep_i;
  memset(qgas_delaa, 0, sizeof(real) * NGAS * NQTEND);
  memset(qnum_delaa, 0, sizeof(real) * NMODE * NQTEND);
  memset(qaer_delaa, 0, sizeof(real) * NAER * NMODE * NQTEND);
  memset(qnumcw_delaa, 0, sizeof(real) * NMODE);
  memset(qaercw_delaa, 0, sizeof(real) * NAER * NMODE);

  real qgas_sv1[NGAS], qnum_sv1[NMODE], qaer_sv1[NAER][NMODE];
  real del_h2so4_aeruptk;
  real qgas_avg[NGAS] = {0.0, 0.0};
  real qnum_delsub_cond[NMODE] = {0}, qnum_delsub_coag[NMODE] = {0};
  real qaer_delsub_cond[NAER][NMODE] = {{0}}, qaer_delsub_coag[NAER][NMODE] = {{0}};
  real qaer_delsub_grow4rnam[NAER][NMODE] = {{0}}, qaercw_delsub_grow4rnam[NAER][NMODE] = {{0}};
  real qaer_delsub_coag_in[NAER];
  real uptkrate_h2so4 = 0;
  (void)del_h2so4_aeruptk;

  if (f->do_cond) {
    memcpy(qgas_sv1, qgas_cur, sizeof(qgas_sv1));
    memcpy(qnum_sv1, qnum_cur, sizeof(qnum_sv1));
    memcpy(qaer_sv1, qaer_cur, sizeof(qaer_sv1));
    real uptkaer[NGAS][NMODE];
    niter = gasaerexch_1subarea(dtsub, temp, pmid, aircon, qgas_cur, qgas_avg, qgas_netprod,
                                qaer_cur, qnum_cur, dgn_awet, uptkaer, &uptkrate_h2so4);
    for (int g = 0; g < NGAS; ++g)
      qgas_delaa[g][0] = qgas_delaa[g][0] + (qgas_cur[g] - (qgas_sv1[g] + qgas_netprod[g] * dtsub));
    for (int m = 0; m < NMODE; ++m)
      qnum_delsub_cond[m] = qnum_cur[m] - qnum_sv1[m];
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaer_delsub_cond[s][m] = qaer_cur[s][m] - qaer_sv1[s][m];
    del_h2so4_aeruptk = qgas_cur[1] - (qgas_sv1[1] + qgas_netprod[1] * dtsub);
  } else {
    memcpy(qgas_avg, qgas_cur, sizeof(qgas_avg));
    del_h2so4_aeruptk = 0;
  }

  if (f->do_rename) {
    memcpy(qaer_delsub_grow4rnam, qaer_delsub_cond, sizeof(qaer_delsub_grow4rnam));
    if (iscldy) {
      for (int s = 0; s < NAER; ++s)
        for (int m = 0; m < NMODE; ++m) {
          qaer_delsub_grow4rnam[s][m] = (qaer3[s][m] - qaer2[s][m]) / 1 + qaer_delsub_grow4rnam[s][m];
          qaercw_delsub_grow4rnam[s][m] = (qaercw3[s][m] - qaercw2[s][m]) / 1;
        }
    }
    memcpy(qnum_sv1, qnum_cur, sizeof(qnum_sv1));
    memcpy(qaer_sv1, qaer_cur, sizeof(qaer_sv1));
    real qnumcw_sv1[NMODE], qaercw_sv1[NAER][NMODE];
    memcpy(qnumcw_sv1, qnumcw_cur, sizeof(qnumcw_sv1));
    memcpy(qaercw_sv1, qaercw_cur, sizeof(qaercw_sv1));
    rename_1subarea(iscldy, qnum_cur, qaer_cur, (const real(*)[NMODE])qaer_delsub_grow4rnam,
                    qnumcw_cur, qaercw_cur, (const real(*)[NMODE])qaercw_delsub_grow4rnam);
    for (int m = 0; m < NMODE; ++m)
      qnum_delaa[m][1] = qnum_delaa[m][1] + (qnum_cur[m] - qnum_sv1[m]);
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaer_delaa[s][m][1] = qaer_delaa[s][m][1] + (qaer_cur[s][m] - qaer_sv1[s][m]);
    if (iscldy)
      for (int m = 0; m < NMODE; ++m)
        qnumcw_delaa[m] = qnumcw_delaa[m] + (qnumcw_cur[m] - qnumcw_sv1[m]);
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaercw_delaa[s][m] = qaercw_delaa[s][m] + (qaercw_cur[s][m] - qaercw_sv1[s][m]);
  }

  if (f->do_newnuc) {
    memcpy(qgas_sv1, qgas_cur, sizeof(qgas_sv1));
    memcpy(qnum_sv1, qnum_cur, sizeof(qnum_sv1));
    memcpy(qaer_sv1, qaer_cur, sizeof(qaer_sv1));
    newnuc_1subarea(dtsub, temp, pmid, zmid, pblh, relhum, uptkrate_h2so4, qgas_cur, qgas_avg,
                    qnum_cur, qaer_cur);
    for (int g = 0; g < NGAS; ++g)
      qgas_delaa[g][2] += (qgas_cur[g] - qgas_sv1[g]);
    for (int m = 0; m < NMODE; ++m)
      qnum_delaa[m][2] += (qnum_cur[m] - qnum_sv1[m]);
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaer_delaa[s][m][2] += (qaer_cur[s][m] - qaer_sv1[s][m]);
  }

  if (f->do_coag) {
    memcpy(qnum_sv1, qnum_cur, sizeof(qnum_sv1));
    memcpy(qaer_sv1, qaer_cur, sizeof(qaer_sv1));
    coag_1subarea(dtsub, temp, pmid, aircon, dgn_awet, wetdens, qnum_cur, qaer_cur,
                  qaer_delsub_coag_in);
    for (int m = 0; m < NMODE; ++m)
      qnum_delsub_coag[m] = qnum_cur[m] - qnum_sv1[m];
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaer_delsub_coag[s][m] = qaer_cur[s][m] - qaer_sv1[s][m];
    for (int m = 0; m < NMODE; ++m)
      qnum_delaa[m][3] += qnum_delsub_coag[m];
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaer_delaa[s][m][3] += qaer_delsub_coag[s][m];
  } else {
    for (int s = 0; s < NAER; ++s)
      qaer_delsub_coag_in[s] = 0.0;
    memset(qaer_delsub_coag, 0, sizeof(qaer_delsub_coag));
    memset(qnum_delsub_coag, 0, sizeof(qnum_delsub_coag));
  }

  if ((!iscldy) || (iscldy && f->do_cond))
    pcarbon_aging_1subarea(nmono, dgn_a, qnum_cur, qnum_delsub_cond, qnum_delsub_coag, qaer_cur,
                           qaer_delsub_cond, qaer_delsub_coag, qaer_delsub_coag_in);

  if (f->do_cond) {
    for (int m = 0; m < NMODE; ++m)
      qnum_delaa[m][0] = qnum_delaa[m][0] + qnum_delsub_cond[m];
    for (int s = 0; s < NAER; ++s)
      for (int m = 0; m < NMODE; ++m)
        qaer_delaa[s][m][0] = qaer_delaa[s][m][0] + qaer_delsub_cond[s][m];
  }
  return niter;
}

/* ------------------------------------------------------ subarea set-up
 * mam4_amicphys.hpp:242-911 */
ORC_FN void get_partition_factors(real q_i, real q_c, real fcldy, real fclea, real *fac_clea,
                                  real *fac_cldy) {
  const real cldbrn_cldy = q_c / fcldy;
  const real intrst_cldy = rmax(0, ((q_i + q_c) - cldbrn_cldy));
  const real intrst_clea = (q_i - fcldy * intrst_cldy) / fclea;
  const real eps = 1.e-35;
  real r = rmax(eps, intrst_clea * fclea) / rmax(eps, q_i);
  r = rmax(0, rmin(1, r));
  *fac_clea = r / fclea;
  *fac_cldy = (1 - r) / fcldy;
}

typedef real qsub_t[PCNST][NSUB];

ORC_FN void set_subarea_intrst(int jclea, int jcldy, real fclea, real fcldy, const real *qgcm,
                               const real *qqcwgcm, const real *qgcmx, qsub_t qsubx) {
  for (int m = 0; m < NMODE; ++m) {
    real fc, fy;
    const int ic = NUMPTR31[m];
    get_partition_factors(qgcm[ic], qqcwgcm[ic], fcldy, fclea, &fc, &fy);
    qsubx[ic][jclea] = qgcmx[ic] * fc;
    qsubx[ic][jcldy] = qgcmx[ic] * fy;
  }
  for (int m = 0; m < NMODE; ++m) {
    real qi = 0, qc = 0;
    for (int s = 0; s < NSPEC[m]; ++s) {
      qi = qi + qgcm[LMASSPTR31[s][m]];
      qc = qc + qqcwgcm[LMASSPTR31[s][m]];
    }
    real fc, fy;
    get_partition_factors(qi, qc, fcldy, fclea, &fc, &fy);
    for (int s = 0; s < NSPEC[m]; ++s) {
      const int ic = LMASSPTR31[s][m];
      qsubx[ic][jclea] = qgcmx[ic] * fc;
      qsubx[ic][jcldy] = qgcmx[ic] * fy;
    }
  }
}

ORC_FN void set_subarea_cldbrn(int jclea, int jcldy, real fcldy, const real *qqcwgcm,
                               qsub_t qqcwsub) {
  for (int m = 0; m < NMODE; ++m) {
    const int ic = NUMPTR31[m];
    qqcwsub[ic][jclea] = 0;
    qqcwsub[ic][jcldy] = qqcwgcm[ic] / fcldy;
  }
  for (int m = 0; m < NMODE; ++m)
    for (int s = 0; s < NSPEC[m]; ++s) {
      const int ic = LMASSPTR31[s][m];
      qqcwsub[ic][jclea] = 0;
      qqcwsub[ic][jcldy] = qqcwgcm[ic] / fcldy;
    }
}

/* modal_aero_amicphys_intr (mam4_amicphys.hpp:2120-2376) for one cell */
ORC_FN int amicphys_intr(const mam4b_config *cfg, real deltat, real temp, real pmid, real zm,
                         real pblh, real qv, real cld, real qq[PCNST], real qqcw[PCNST],
                         const real q_pregaschem[PCNST], const real q_precldchem[PCNST],
                         const real qqcw_precldchem[PCNST], const real dgncur_a[NMODE],
                         const real dgncur_awet[NMODE], const real wetdens_host[NMODE],
                         real *diag /* [5][31] or NULL */) {
  const real epsqs = 0.018016 / 0.028966;
  /* vapor_saturation_pressure_magnus (conversions.hpp:148-180) */
  const real tc = temp - 273.15;
  const real ew = 610.94 * exp(17.625 * tc / (234.04 + tc));
  const real ev_sat = 1.00071 * exp(4.5e-8 * pmid) * ew;
  const real qv_sat = epsqs * ev_sat / (pmid - (1 - epsqs) * ev_sat);
  /* setup_subareas (:242-321) */
  int nsubarea, ncldy, jclea, jcldy;
  real fcldy, fclea;
  if (cld < 1.0e-5) {
    fcldy = 0;
    nsubarea = 1;
    ncldy = 0;
    jclea = 1;
    jcldy = 0;
  } else if (cld > 0.999) {
    fcldy = 1;
    nsubarea = 1;
    ncldy = 1;
    jclea = 0;
    jcldy = 1;
  } else {
    fcldy = cld;
    nsubarea = 2;
    ncldy = 1;
    jclea = 1;
    jcldy = 2;
  }
  fclea = 1.0 - fcldy;
  int iscldy[NSUB] = {0, 0, 0};
  real afracsub[NSUB] = {0, 0, 0};
  if (jcldy > 0)
    iscldy[jcldy] = 1;
  if (jclea > 0)
    afracsub[jclea] = fclea;
  if (jcldy > 0)
    afracsub[jcldy] = fcldy;
  const real relhumgcm = rmax(0.0, rmin(1.0, qv / qv_sat));
  /* set_subarea_rh (:323-361) */
  real relhumsub[NSUB];
  if (ncldy <= 0) {
    for (int j = 0; j < NSUB; ++j)
      relhumsub[j] = relhumgcm;
  } else {
    relhumsub[0] = relhumsub[1] = relhumsub[2] = 0; /* unset in the reference */
    relhumsub[jcldy] = 1;
    if (jclea > 0) {
      const real t = (relhumgcm - afracsub[jcldy]) / afracsub[jclea];
      relhumsub[jclea] = min_max_bound(0, 1, t);
    }
  }
  real qgcm1[PCNST], qgcm2[PCNST], qgcm3[PCNST], qqcwgcm2[PCNST], qqcwgcm3[PCNST];
  for (int i = 0; i < PCNST; ++i) {
    qgcm1[i] = rmax(0, q_pregaschem[i]);
    qgcm2[i] = rmax(0, q_precldchem[i]);
    qgcm3[i] = rmax(0, qq[i]);
    qqcwgcm2[i] = rmax(0, qqcw_precldchem[i]);
    qqcwgcm3[i] = rmax(0, qqcw[i]);
  }
  /* set_subarea_gases_and_aerosols (:679-911) */
  qsub_t qsub1, qsub2, qsub3, qqcwsub2, qqcwsub3;
  memset(qsub1, 0, sizeof(qsub_t));
  memset(qsub2, 0, sizeof(qsub_t));
  memset(qsub3, 0, sizeof(qsub_t));
  memset(qqcwsub2, 0, sizeof(qsub_t));
  memset(qqcwsub3, 0, sizeof(qsub_t));
  if (nsubarea == 1) {
    for (int i = 0; i < PCNST; ++i)
      if (LMAPCC_ALL[i] > 0) {
        qsub1[i][1] = qgcm1[i];
        qsub2[i][1] = qgcm2[i];
        qsub3[i][1] = qgcm3[i];
        qqcwsub2[i][1] = qqcwgcm2[i];
        qqcwsub3[i][1] = qqcwgcm3[i];
      }
  } else {
    for (int i = 0; i < PCNST; ++i)
      if (LMAPCC_ALL[i] == 1) {
        for (int j = 1; j <= nsubarea; ++j) {
          qsub1[i][j] = qgcm1[i];
          qsub2[i][j] = qgcm2[i];
        }
        qsub3[i][jclea] = qsub2[i][jclea];
      }
    /* compute_qsub_from_gcm_and_qsub_of_other_subarea (:367-410) */
    for (int i = 0; i < PCNST; ++i)
      if (LMAPCC_ALL[i] == 1) {
        qsub3[i][jcldy] = (qgcm3[i] - fclea * qsub3[i][jclea]) / fcldy;
        if (qsub3[i][jcldy] < 0) {
          qsub3[i][jcldy] = 0;
          qsub3[i][jclea] = qgcm3[i] / fclea;
        }
      }
    set_subarea_cldbrn(jclea, jcldy, fcldy, qqcwgcm2, qqcwsub2);
    set_subarea_cldbrn(jclea, jcldy, fcldy, qqcwgcm3, qqcwsub3);
    set_subarea_intrst(jclea, jcldy, fclea, fcldy, qgcm2, qqcwgcm2, qgcm2, qsub2);
    set_subarea_intrst(jclea, jcldy, fclea, fcldy, qgcm2, qqcwgcm2, qgcm3, qsub3);
  }
  qsub_t qsub4, qqcwsub4;
  memset(qsub4, 0, sizeof(qsub_t));
  memset(qqcwsub4, 0, sizeof(qsub_t));
  real qsub_tendaa[PCNST][NQTEND][NSUB], qqcwsub_tendaa[PCNST][NSUB];
  memset(qsub_tendaa, 0, sizeof(qsub_tendaa));
  memset(qqcwsub_tendaa, 0, sizeof(qqcwsub_tendaa));
  real dgn_a[NMODE], dgn_awet[NMODE], wetdens[NMODE];
  for (int m = 0; m < NMODE; ++m) {
    dgn_a[m] = dgncur_a[m];
    dgn_awet[m] = dgncur_awet[m];
    wetdens[m] = rmax(1000.0, wetdens_host[m]);
  }
  /* mam_amicphys_1gridcell (:1700-1995) */
  int niter_clear = 0;
  for (int i = 0; i < 6; ++i)
    for (int j = 1; j < NSUB; ++j) {
      qsub4[i][j] = qsub3[i][j];
      qqcwsub4[i][j] = qqcwsub3[i][j];
    }
  for (int jsub = 1; jsub <= nsubarea; ++jsub) {
    sub_flags fl;
    fl.optaa = cfg->gaexch_h2so4_uptake_optaa;
    if (iscldy[jsub]) {
      fl.do_cond = 0; /* mdo_gaexch_cldy_subarea = 0 */
      fl.do_rename = cfg->do_rename;
      fl.do_newnuc = 0;
      fl.do_coag = 0;
    } else {
      fl.do_cond = cfg->do_cond;
      fl.do_rename = cfg->do_rename;
      fl.do_newnuc = cfg->do_newnuc;
      fl.do_coag = cfg->do_coag;
    }
    const int do_map_gas = fl.do_cond || fl.do_newnuc;
    real qgas1[NGAS] = {0}, qgas3[NGAS] = {0}, qgas4[NGAS] = {0};
    if (do_map_gas)
      for (int g = 0; g < NGAS; ++g) {
        const int l = LMAP_GAS[g];
        qgas1[g] = qsub1[l][jsub] * fcvt_gas(g);
        qgas3[g] = qsub3[l][jsub] * fcvt_gas(g);
        qgas4[g] = qgas3[g];
      }
    real qaer2[NAER][NMODE] = {{0}}, qaer3[NAER][NMODE] = {{0}}, qaer4[NAER][NMODE] = {{0}};
    real qnum3[NMODE] = {0}, qnum4[NMODE] = {0};
    for (int m = 0; m < NMODE; ++m) {
      const int ln = NUMPTR31[m];
      qnum3[m] = qsub3[ln][jsub] * 1;
      qnum4[m] = qnum3[m];
      for (int a = 0; a < NAER; ++a) {
        const int la = LMAP_AER[a][m];
        if (la > 0) {
          qaer2[a][m] = qsub2[la][jsub] * FCVT_AER[a];
          qaer3[a][m] = qsub3[la][jsub] * FCVT_AER[a];
          qaer4[a][m] = qaer3[a][m];
        }
      }
    }
    real qaercw2[NAER][NMODE] = {{0}}, qaercw3[NAER][NMODE] = {{0}}, qaercw4[NAER][NMODE] = {{0}};
    real qnumcw3[NMODE] = {0}, qnumcw4[NMODE] = {0};
    if (iscldy[jsub]) {
      for (int m = 0; m < NMODE; ++m) {
        const int ln = NUMPTR31[m];
        qnumcw3[m] = qqcwsub3[ln][jsub] * 1;
        qnumcw4[m] = qnumcw3[m];
      }
      for (int a = 0; a < NAER; ++a)
        for (int m = 0; m < NMODE; ++m) {
          const int la = LMAP_AER[a][m];
          if (la > 0) {
            qaercw2[a][m] = qqcwsub2[la][jsub] * FCVT_AER[a];
            qaercw3[a][m] = qqcwsub3[la][jsub] * FCVT_AER[a];
            qaercw4[a][m] = qaercw3[a][m];
          }
        }
    }
    real qgas_delaa[NGAS][NQTEND], qnum_delaa[NMODE][NQTEND], qnumcw_delaa[NMODE];
    real qaer_delaa[NAER][NMODE][NQTEND], qaercw_delaa[NAER][NMODE];
    const int nit = amicphys_1subarea(
        &fl, deltat, iscldy[jsub], cfg->n_so4_monolayers_pcage, temp, pmid, zm, pblh,
        relhumsub[jsub], dgn_a, dgn_awet, wetdens, qgas1, qgas3, qgas4, qgas_delaa, qnum3, qnum4,
        qnum_delaa, (const real(*)[NMODE])qaer2, (const real(*)[NMODE])qaer3, qaer4, qaer_delaa,
        qnumcw3, qnumcw4, qnumcw_delaa, (const real(*)[NMODE])qaercw2,
        (const real(*)[NMODE])qaercw3, qaercw4, qaercw_delaa);
    if (!iscldy[jsub])
      niter_clear = nit;
    if (do_map_gas)
      for (int g = 0; g < NGAS; ++g) {
        const int l = LMAP_GAS[g];
        qsub4[l][jsub] = qgas4[g] / fcvt_gas(g);
        for (int k = 0; k < NQTEND; ++k)
          qsub_tendaa[l][k][jsub] = qgas_delaa[g][k] / (fcvt_gas(g) * deltat);
      }
    for (int m = 0; m < NMODE; ++m) {
      const int l = NUMPTR31[m];
      qsub4[l][jsub] = qnum4[m] / (1.0);
      for (int k = 0; k < NQTEND; ++k)
        qsub_tendaa[l][k][jsub] = qnum_delaa[m][k] / (1.0 * deltat);
      for (int a = 0; a < NAER; ++a) {
        const int la = LMAP_AER[a][m];
        if (la > 0) {
          qsub4[la][jsub] = qaer4[a][m] / FCVT_AER[a];
          for (int k = 0; k < NQTEND; ++k)
            qsub_tendaa[la][k][jsub] = qaer_delaa[a][m][k] / (FCVT_AER[a] * deltat);
        }
      }
      if (iscldy[jsub]) {
        qqcwsub4[l][jsub] = qnumcw4[m] / 1.0;
        qqcwsub_tendaa[l][jsub] = qnumcw_delaa[m] / (1.0 * deltat);
        for (int a = 0; a < NAER; ++a) {
          const int la = LMAP_AER[a][m];
          if (la > 0) {
            qqcwsub4[la][jsub] = qaercw4[a][m] / FCVT_AER[a];
            qqcwsub_tendaa[la][jsub] = qaercw_delaa[a][m] / (FCVT_AER[a] * deltat);
          }
        }
      }
    }
  }
  /* form_gcm_of_gases_and_aerosols_from_subareas (:1997-2068) */
  real qgcm4[PCNST], qqcwgcm4[PCNST];
  for (int i = 0; i < PCNST; ++i) {
    qgcm4[i] = 0;
    for (int j = 1; j <= nsubarea; ++j)
      qgcm4[i] += qsub4[i][j] * afracsub[j];
    qgcm4[i] = rmax(0, qgcm4[i]);
  }
  if (ncldy <= 0) {
    for (int i = 0; i < PCNST; ++i)
      qqcwgcm4[i] = qqcwgcm3[i];
  } else {
    for (int i = 0; i < PCNST; ++i) {
      qqcwgcm4[i] = 0;
      for (int j = 1; j <= nsubarea; ++j)
        qqcwgcm4[i] += qqcwsub4[i][j] * afracsub[j];
    }
  }
  for (int i = 0; i < PCNST; ++i) {
    if (LMAPCC_ALL[i] > 0)
      qq[i] = qgcm4[i];
    if (LMAPCC_ALL[i] >= 2)
      qqcw[i] = qqcwgcm4[i];
  }
  if (diag) {
    /* get_gcm_tend_diags_from_subareas (:2070-2113) */
    for (int k = 0; k < NQTEND; ++k)
      for (int i = 0; i < PCNST; ++i) {
        real t = 0;
        for (int j = 1; j <= nsubarea; ++j)
          t += qsub_tendaa[i][k][j] * afracsub[j];
        diag[k * PCNST + i] = t;
      }
    for (int i = 0; i < PCNST; ++i) {
      real t = 0;
      if (ncldy > 0)
        for (int j = 1; j <= nsubarea; ++j)
          t += qqcwsub_tendaa[i][j] * afracsub[j];
      diag[4 * PCNST + i] = t;
    }
  }
  return niter_clear;
}

/* ============================================================ full step */
#ifndef ORACLE_GPU
static const calcsize_data *cdata(void) {
  static calcsize_data d;
  static int init = 0;
  if (!init) {
    calcsize_init(&d);
    init = 1;
  }
  return &d;
}
#endif

ORC_FN real to_vmr(int i31) {
  const int num = (i31 == 13 || i31 == 18 || i31 == 26 || i31 == 30);
  return num ? 28.966 : 28.966 / ADV_MASS[i31];
}
ORC_FN real to_mmr(int i31) {
  const int num = (i31 == 13 || i31 == 18 || i31 == 26 || i31 == 30);
  return num ? 1.0 / 28.966 : ADV_MASS[i31] / 28.966;
}

ORC_FN int step_cell(const calcsize_data *cd, const double *in, size_t ld, size_t c, double pblh,
                     double *out, size_t ldo, double *diag, size_t ldd, double dt,
                     const mam4b_config *cfg) {
#define IN(f) in[(size_t)(f) * ld + c]
  NOISE_SEED_CELL(c);
  real state_q[40] = {0}, qqcw[40] = {0};
  state_q[0] = IN(MAM4B_IN_QV);
  state_q[11] = IN(MAM4B_IN_H2SO4);
  state_q[14] = IN(MAM4B_IN_SOAG);
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    state_q[15 + p] = IN(MAM4B_IN_AER_I + p);
    qqcw[15 + p] = IN(MAM4B_IN_AER_C + p);
  }
  const real temp = IN(MAM4B_IN_T), pmid = IN(MAM4B_IN_P), cld = IN(MAM4B_IN_CLD);
  real dgncur_a[NMODE], dgncur_c[NMODE], ptend[40] = {0}, dqqcwdt[40] = {0};
  calcsize_sub(cd, state_q, qqcw, dt, dgncur_a, dgncur_c, ptend, dqqcwdt);
  real dgncur_awet[NMODE], qaerwat[NMODE], wetdens[NMODE];
  water_uptake_dr(state_q, temp, pmid, cld, dgncur_a, dgncur_awet, qaerwat, wetdens);
  for (int i = 15; i < 40; ++i) {
    state_q[i] = rmax(0.0, state_q[i] + ptend[i] * dt);
    qqcw[i] = rmax(0.0, qqcw[i] + dqqcwdt[i] * dt);
  }
  real qq[PCNST], qqcw31[PCNST], qpre[PCNST], qcwpre[PCNST];
  for (int i = 0; i < PCNST; ++i) {
    qq[i] = state_q[9 + i] * to_vmr(i);
    qqcw31[i] = qqcw[9 + i] * to_vmr(i);
    qpre[i] = qq[i];
    qcwpre[i] = qqcw31[i];
  }
  real dg[5 * PCNST];
  const int niter = amicphys_intr(cfg, dt, temp, pmid, IN(MAM4B_IN_ZM), pblh, IN(MAM4B_IN_QV),
                                  cld, qq, qqcw31, qpre, qpre, qcwpre, dgncur_a, dgncur_awet,
                                  wetdens, diag ? dg : NULL);
  if (out) {
#define OUT(f) out[(size_t)(f) * ldo + c]
    /* (double) casts: no-ops here, conversions in the op-counting build */
    OUT(MAM4B_OUT_TEND + 0) = (double)((qq[2] * to_mmr(2) - IN(MAM4B_IN_H2SO4)) / dt);
    OUT(MAM4B_OUT_TEND + 1) = (double)((qq[5] * to_mmr(5) - IN(MAM4B_IN_SOAG)) / dt);
    for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
      const int i31 = 6 + p;
      OUT(MAM4B_OUT_TEND + 2 + p) =
          (double)((qq[i31] * to_mmr(i31) - IN(MAM4B_IN_AER_I + p)) / dt);
      OUT(MAM4B_OUT_TEND + 27 + p) =
          (double)((qqcw31[i31] * to_mmr(i31) - IN(MAM4B_IN_AER_C + p)) / dt);
    }
    for (int m = 0; m < NMODE; ++m) {
      OUT(MAM4B_OUT_DGN_A + m) = (double)dgncur_a[m];
      OUT(MAM4B_OUT_DGN_AWET + m) = (double)dgncur_awet[m];
      OUT(MAM4B_OUT_WETDENS + m) = (double)wetdens[m];
      OUT(MAM4B_OUT_QAERWAT + m) = (double)qaerwat[m];
    }
#undef OUT
  }
  if (diag)
    for (int k = 0; k < 5 * PCNST; ++k)
      diag[(size_t)k * ldd + c] = (double)dg[k];
#undef IN
  return niter;
}

/* ============================================================== C entries */
#ifndef ORACLE_GPU
int mam4orc_step(int ncell, const double *in, size_t ld_in, const double *pblh_cell,
                 double *out, size_t ld_out, double *diag, size_t ld_diag, double dt,
                 const mam4b_config *cfg, int nthreads) {
  if (ncell < 0 || !in || !pblh_cell || !out || !cfg || !(dt > 0))
    return MAM4B_ERR_INVALID_ARGUMENT;
  (void)cdata();
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
#else
  (void)nthreads;
#endif
  for (int c = 0; c < ncell; ++c)
    step_cell(cdata(), in, ld_in, (size_t)c, pblh_cell[c], out, ld_out, diag, ld_diag, dt, cfg);
  return MAM4B_OK;
}

void mam4orc_soa_niter(int ncell, const double *in, size_t ld_in, const double *pblh_cell,
                       double dt, const mam4b_config *cfg, int *niter, int nthreads) {
  (void)cdata();
#ifdef _OPENMP
  const int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
#else
  (void)nthreads;
#endif
  for (int c = 0; c < ncell; ++c)
    niter[c] = step_cell(cdata(), in, ld_in, (size_t)c, pblh_cell[c], NULL, 0, NULL, 0, dt, cfg);
}

/* stage-level entries: plain-double builds only (the op-counting build of
 * oracle/opcount.cpp counts the whole step) */
#ifndef ORACLE_REAL
void mam4orc_calcsize(int ncell, const double *state_q, const double *qqcw, double dt,
                      double *dgncur_a, double *dgncur_c, double *ptend, double *dqqcwdt) {
  for (int c = 0; c < ncell; ++c) {
    real pt[40] = {0}, dq[40] = {0};
    calcsize_sub(cdata(), state_q + 40 * c, qqcw + 40 * c, dt, dgncur_a + 4 * c,
                 dgncur_c + 4 * c, pt, dq);
    memcpy(ptend + 40 * c, pt, sizeof(pt));
    memcpy(dqqcwdt + 40 * c, dq, sizeof(dq));
  }
}

void mam4orc_water_uptake(int ncell, const double *state_q, const double *temp,
                          const double *pmid, const double *cld, const double *dgncur_a,
                          double *dgncur_awet, double *qaerwat, double *wetdens) {
  for (int c = 0; c < ncell; ++c)
    water_uptake_dr(state_q + 40 * c, temp[c], pmid[c], cld[c], dgncur_a + 4 * c,
                    dgncur_awet + 4 * c, qaerwat + 4 * c, wetdens + 4 * c);
}

void mam4orc_amicphys(int ncell, const mam4b_config *cfg, double dt, const double *temp,
                      const double *pmid, const double *zm, const double *pblh, const double *qv,
                      const double *cld, double *qq, double *qqcw, const double *dgncur_a,
                      const double *dgncur_awet, const double *wetdens, double *diag) {
  for (int c = 0; c < ncell; ++c) {
    real qpre[PCNST], qcwpre[PCNST];
    memcpy(qpre, qq + PCNST * c, sizeof(qpre));
    memcpy(qcwpre, qqcw + PCNST * c, sizeof(qcwpre));
    amicphys_intr(cfg, dt, temp[c], pmid[c], zm[c], pblh[c], qv[c], cld[c], qq + PCNST * c,
                  qqcw + PCNST * c, qpre, qpre, qcwpre, dgncur_a + 4 * c, dgncur_awet + 4 * c,
                  wetdens + 4 * c, diag ? diag + 5 * PCNST * c : NULL);
  }
}

void mam4orc_h2so4_update(double dt, double qgas_netprod_otrproc, const double *uptkaer,
                          double *qgas_cur, double *qgas_avg, double *qaer_cur) {
  h2so4_nonvolatile(dt, qgas_netprod_otrproc, uptkaer, qgas_cur, qgas_avg, qaer_cur);
}

double mam4orc_bm0ij(int n1, int n2a, int n2n) { return kCoagBm0ij[n1 * 100 + n2a * 10 + n2n]; }
double mam4orc_bm3i(int n1, int n2a, int n2n) { return kCoagBm3i[n1 * 100 + n2a * 10 + n2n]; }

void mam4orc_aging(unsigned n_so4_monolayers_pcage, const double *dgn_a, double *qnum_cur,
                   double *qnum_del_cond, double *qnum_del_coag, double *qaer_cur,
                   double *qaer_del_cond, double *qaer_del_coag, double *qaer_del_coag_in) {
  pcarbon_aging_1subarea(n_so4_monolayers_pcage, dgn_a, qnum_cur, qnum_del_cond, qnum_del_coag,
                         (real(*)[NMODE])qaer_cur, (real(*)[NMODE])qaer_del_cond,
                         (real(*)[NMODE])qaer_del_coag, qaer_del_coag_in);
}
#endif /* !ORACLE_REAL */
#endif /* !ORACLE_GPU */
