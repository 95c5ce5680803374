// mam4b_adjoint.cuh -- hand-written reverse-mode adjoint of the FP64
// microphysics step (calcsize -> water uptake -> amicphys).
//
// Every forward function f of mam4b_physics.cuh that the step calls has a
// reverse function f_rev here. f_rev takes f's inputs and the cotangents of
// its outputs, recomputes f's internals (nothing is taped inside a
// function) and ADDS the cotangents of f's inputs to the *_bar arguments
// (x_bar += (df/dx)^T y_bar). Branches follow the forward path taken at the
// given inputs; max/min pass the cotangent to the selected argument; the
// Kohler root is differentiated implicitly from its quartic.
//
// Differentiated inputs: temperature, water vapour, H2SO4, SOAG and the 50
// aerosol populations. Pressure, height, cloud fraction and the
// boundary-layer height are parameters of the step here (their cotangents
// are not formed).
#pragma once

#include "mam4b_physics.cuh"
#include "mam4b_physics_mixed.cuh"

namespace mam4b {
namespace adj {

// ------------------------------------------------------------ primitives
// r = dmax(a, b): the cotangent goes to the argument dmax returned
MAM4B_HD void max_rev(double a, double b, double rb, double &ab, double &bb) {
  if (a < b)
    bb += rb;
  else
    ab += rb;
}
MAM4B_HD void min_rev(double a, double b, double rb, double &ab, double &bb) {
  if (b < a)
    bb += rb;
  else
    ab += rb;
}
// r = dmax(0, x) / dmax(c, x) with constant c: cotangent to x when selected
MAM4B_HD double maxc_rev(double c, double x, double rb) { return (c < x) ? rb : 0.0; }
MAM4B_HD double minc_rev(double c, double x, double rb) { return (x < c) ? rb : 0.0; }
// bound(lo, hi, x) = dmax(lo, dmin(hi, x)) with constant bounds
MAM4B_HD double boundc_rev(double lo, double hi, double x, double rb) {
  const double m = dmin(hi, x);
  if (lo < m)
    return (x < hi) ? rb : 0.0;
  return 0.0;
}

// diam_from_vol(v, ls) = cbrt(v / pi6) exp(-1.5 ls^2); d/dv = d / (3 v)
MAM4B_HD double diam_from_vol_rev(double v, double log_sig, double db) {
  const double d = diam_from_vol(v, log_sig);
  return db * d / (3.0 * v);
}

// ================================================================ calcsize
// adjust_num_sizes (calcsize.hpp:95-310): inputs drv_i, drv_c, init_i,
// init_c, num_i0, num_c0 (the clipped numbers); outputs num_i, num_c,
// dqdt, dqqcwdt.
struct AdjNumOut {
  double num_i, num_c, dqdt, dqqcwdt;
};

MAM4B_HD void adjust_num_sizes_rev(double drv_i, double drv_c, double init_i, double init_c,
                                   double num_i0, double num_c0, double dt, double v2nmin,
                                   double v2nmax, double adj_inv, double num_ib, double num_cb,
                                   double dqdtb, double dqqcwdtb, double &drv_ib,
                                   double &drv_cb, double &init_ib, double &init_cb,
                                   double &num_i0b, double &num_c0b) {
  const double frac = dmax(0.0, dmin(1.0, dt * adj_inv));
  const double dtinv = safe_denominator(dt);
  const double minrl = v2nmin / 27.0, maxrl = v2nmax * 27.0;
  // dqdt = (num_i - init_i) * dtinv
  num_ib += dqdtb * dtinv;
  init_ib -= dqdtb * dtinv;
  num_cb += dqqcwdtb * dtinv;
  init_cb -= dqqcwdtb * dtinv;
  if (drv_i <= 0.0 && drv_c <= 0.0)
    return;
  if (drv_c <= 0.0) {
    // num_i = num_i0 + (nb - num_i0) * frac, nb = bound(drv_i*v2nmin, drv_i*v2nmax, num_i0)
    const double lo = drv_i * v2nmin, hi = drv_i * v2nmax;
    const double nbb = num_ib * frac;
    num_i0b += num_ib * (1.0 - frac);
    // nb = dmax(lo, dmin(hi, num_i0))
    const double m = dmin(hi, num_i0);
    if (lo < m) {
      if (num_i0 < hi)
        num_i0b += nbb;
      else
        drv_ib += nbb * v2nmax;
    } else {
      drv_ib += nbb * v2nmin;
    }
    return;
  }
  if (drv_i <= 0.0) {
    const double lo = drv_c * v2nmin, hi = drv_c * v2nmax;
    const double nbb = num_cb * frac;
    num_c0b += num_cb * (1.0 - frac);
    const double m = dmin(hi, num_c0);
    if (lo < m) {
      if (num_c0 < hi)
        num_c0b += nbb;
      else
        drv_cb += nbb * v2nmax;
    } else {
      drv_cb += nbb * v2nmin;
    }
    return;
  }
  // both phases: recompute the forward
  const double ni1 = num_i0, nc1 = num_c0;
  auto bnd = [](double lo, double hi, double x) { return dmax(lo, dmin(hi, x)); };
  const double nbi = bnd(drv_i * minrl, drv_i * maxrl, ni1);
  const double dni2 = (nbi - ni1) * frac;
  double ni2 = ni1 + dni2;
  const double nbc = bnd(drv_c * minrl, drv_c * maxrl, nc1);
  const double dnc2 = (nbc - nc1) * frac;
  double nc2 = nc1 + dnc2;
  int which2 = 0;  // 1: ni2 rebounded with nc's step, 2: nc2 rebounded with ni's step
  if (dni2 == 0.0 && dnc2 != 0.0) {
    ni2 = bnd(drv_i * minrl, drv_i * maxrl, ni1 - dnc2);
    which2 = 1;
  } else if (dni2 != 0.0 && dnc2 == 0.0) {
    nc2 = bnd(drv_c * minrl, drv_c * maxrl, nc1 - dni2);
    which2 = 2;
  }
  const double tdrv = drv_i + drv_c, tnum = ni2 + nc2;
  const double minb = tdrv * v2nmin, maxb = tdrv * v2nmax;
  // num_i = ni2 + dni3, num_c = nc2 + dnc3
  double ni2b = num_ib, nc2b = num_cb, tdrvb = 0.0, tnumb = 0.0;
  double dni3b = num_ib, dnc3b = num_cb;
  if (tnum < minb || tnum > maxb) {
    const bool low = tnum < minb;
    const double bndv = low ? minb : maxb;
    const double vv = low ? v2nmin : v2nmax;
    const double d3 = (bndv - tnum) * frac;
    double d3b = 0.0;
    const bool ci = low ? (ni2 < drv_i * v2nmin) : (ni2 > drv_i * v2nmax);
    const bool cc = low ? (nc2 < drv_c * v2nmin) : (nc2 > drv_c * v2nmax);
    if (ci && cc) {
      // dni3 = d3 * (ni2 / tnum), dnc3 = d3 * (nc2 / tnum)
      d3b += dni3b * (ni2 / tnum) + dnc3b * (nc2 / tnum);
      ni2b += dni3b * d3 / tnum;
      nc2b += dnc3b * d3 / tnum;
      tnumb -= (dni3b * d3 * ni2 + dnc3b * d3 * nc2) / (tnum * tnum);
    } else if (cc) {
      d3b += dnc3b;
    } else if (ci) {
      d3b += dni3b;
    }
    // d3 = (bndv - tnum) * frac, bndv = tdrv * vv
    tdrvb += d3b * frac * vv;
    tnumb -= d3b * frac;
  }
  // tnum = ni2 + nc2, tdrv = drv_i + drv_c
  ni2b += tnumb;
  nc2b += tnumb;
  drv_ib += tdrvb;
  drv_cb += tdrvb;
  // bound(lo, hi, x) cotangent distribution helper
  auto bnd_rev = [&](double d, double x, double rb, double &db, double &xb) {
    const double lo = d * minrl, hi = d * maxrl;
    const double m = dmin(hi, x);
    if (lo < m) {
      if (x < hi)
        xb += rb;
      else
        db += rb * maxrl;
    } else {
      db += rb * minrl;
    }
  };
  double ni1b = 0.0, nc1b = 0.0, dni2b = 0.0, dnc2b = 0.0;
  if (which2 == 1) {
    // ni2 = bnd(drv_i.., ni1 - dnc2)
    double xb = 0.0;
    bnd_rev(drv_i, ni1 - dnc2, ni2b, drv_ib, xb);
    ni1b += xb;
    dnc2b -= xb;
  } else {
    // ni2 = ni1 + dni2
    ni1b += ni2b;
    dni2b += ni2b;
  }
  if (which2 == 2) {
    double xb = 0.0;
    bnd_rev(drv_c, nc1 - dni2, nc2b, drv_cb, xb);
    nc1b += xb;
    dni2b -= xb;
  } else {
    nc1b += nc2b;
    dnc2b += nc2b;
  }
  // dnc2 = (nbc - nc1) * frac
  {
    const double nbb = dnc2b * frac;
    nc1b -= dnc2b * frac;
    bnd_rev(drv_c, nc1, nbb, drv_cb, nc1b);
  }
  // dni2 = (nbi - ni1) * frac
  {
    const double nbb = dni2b * frac;
    ni1b -= dni2b * frac;
    bnd_rev(drv_i, ni1, nbb, drv_ib, ni1b);
  }
  num_i0b += ni1b;
  num_c0b += nc1b;
}

// diameter_from_num (calcsize.hpp:56-78): dgn depends on drv, num only in
// the interior branch
MAM4B_HD void diameter_from_num_rev(double drv, double num, double v2nmin, double v2nmax,
                                    double log_sig, double dgnb, double &drvb, double &numb) {
  if (!(drv > 0.0))
    return;
  if (num <= drv * v2nmin || num >= drv * v2nmax)
    return;
  // dgn = diam_from_vol(1 / (num / drv)); v = drv / num (as 1/(num/drv))
  const double u = num / drv;
  const double v = 1.0 / u;
  const double vb = diam_from_vol_rev(v, log_sig, dgnb);
  const double ub = -vb / (u * u);
  numb += ub / drv;
  drvb -= ub * num / (drv * drv);
}

MAM4B_HD void size_after_transfer_rev(double drv, double num, double v2n_hi, double v2n_lo,
                                      double log_sig, double dgnb, double &drvb, double &numb) {
  if (!(drv > 0.0))
    return;
  if (num <= drv * v2n_hi || num >= drv * v2n_lo)
    return;
  const double u = num / drv;
  const double v = 1.0 / u;
  const double vb = diam_from_vol_rev(v, log_sig, dgnb);
  const double ub = -vb / (u * u);
  numb += ub / drv;
  drvb -= ub * num / (drv * drv);
}

// calcsize: inputs ai[25], ac[25]; outputs dgn_i[4], pt_i[25], pt_c[25].
MAM4B_HD void calcsize_rev(const StepConsts &C, const double (&ai)[NPOP], const double (&ac)[NPOP],
                           double dt, const double (&dgnb)[NMODE], const double (&pt_ib)[NPOP],
                           const double (&pt_cb)[NPOP], double (&aib)[NPOP],
                           double (&acb)[NPOP]) {
  const double adj_inv = safe_denominator(dmax(86400.0, dt));
  // ---- forward recomputation of the per-mode quantities
  double dv_i[NMODE], dv_c[NMODE], num_i0[NMODE], num_c0[NMODE], num_i[NMODE], num_c[NMODE];
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    dv_i[m] = 0.0;
    dv_c[m] = 0.0;
#pragma unroll
    for (int s = 0; s < K::nspec(m); ++s) {
      dv_i[m] += dmax(0.0, ai[K::spec0(m) + s]) * C.inv_density[m][s];
      dv_c[m] += dmax(0.0, ac[K::spec0(m) + s]) * C.inv_density[m][s];
    }
    const double init_i = ai[K::numslot(m)], init_c = ac[K::numslot(m)];
    num_i0[m] = init_i < 0 ? 0.0 : init_i;
    num_c0[m] = init_c < 0 ? 0.0 : init_c;
    num_i[m] = num_i0[m];
    num_c[m] = num_c0[m];
    if (m >= 2) {
      double d1, d2;
      adjust_num_sizes(dv_i[m], dv_c[m], init_i, init_c, dt, C.n2v_min[m], C.n2v_max[m], adj_inv,
                       num_i[m], num_c[m], d1, d2);
    }
  }
  // exchange quantities (modal_aero_calcsize.hpp:499-747)
  const double v2n_ait = C.n2v_nom[1], v2n_acc = C.n2v_nom[0];
  const double gm = C.geomean_ait_acc;
  const double dv_i_ait = dv_i[1], dv_c_ait = dv_c[1], n_i_ait = num_i[1], n_c_ait = num_c[1];
  const double dv_i_acc = dv_i[0], dv_c_acc = dv_c[0], n_i_acc = num_i[0], n_c_acc = num_c[0];
  bool ait2acc = false, acc2ait = false;
  double xt00 = 0, xt01 = 0, xt10 = 0, xt11 = 0;
  double xv_ait2acc = 0, xv_acc2ait = 0, noxf_i = 0, noxf_c = 0;
  // ait -> acc
  const double a_drv_t = dv_i_ait + dv_c_ait, a_num_t = n_i_ait + n_c_ait;
  int a_case = 0;  // 0: fn=fv=1 (num below acc), 1: interior, 2: clipped 0, 3: clipped 1
  double a_fn = 0, a_fv = 0;
  if (a_drv_t > 0.0 && a_num_t < a_drv_t * gm) {
    ait2acc = true;
    if (a_num_t < a_drv_t * v2n_acc) {
      a_fn = 1.0;
      a_fv = 1.0;
      a_case = 0;
    } else {
      a_fv = ((a_num_t / a_drv_t) - gm) / (v2n_acc - gm);
      a_fn = a_fv * (a_drv_t * v2n_acc / a_num_t);
      a_case = 1;
      if (a_fn <= 0.0 || a_fv <= 0.0) {
        a_fn = 0.0;
        a_fv = 0.0;
        a_case = 2;
      } else if (a_fn >= 1.0 || a_fv >= 1.0) {
        a_fn = 1.0;
        a_fv = 1.0;
        a_case = 3;
      }
    }
    xv_ait2acc = a_fv * adj_inv;
    xt00 = n_i_ait * (a_fn * adj_inv);
    xt01 = n_c_ait * (a_fn * adj_inv);
  }
  // acc -> ait
  double b_drv_t = dv_i_acc + dv_c_acc, b_num_t = n_i_acc + n_c_acc, b_num_t0 = 0.0;
  const double b_drv_t_in = b_drv_t, b_num_t_in = b_num_t;
  bool b_noxf = false;
  if (b_drv_t > 0.0 && b_num_t > b_drv_t * gm) {
    b_noxf = true;
    noxf_i = dmax(0.0, ai[1]) * C.inv_density[0][1];
    noxf_c = dmax(0.0, ac[1]) * C.inv_density[0][1];
    noxf_i += dmax(0.0, ai[3]) * C.inv_density[0][3];
    noxf_c += dmax(0.0, ac[3]) * C.inv_density[0][3];
    noxf_i += dmax(0.0, ai[4]) * C.inv_density[0][4];
    noxf_c += dmax(0.0, ac[4]) * C.inv_density[0][4];
    const double drv_noxf = noxf_i + noxf_c;
    const double num_noxf = drv_noxf * C.n2v_max[0];
    b_num_t0 = b_num_t;
    b_num_t = dmax(0.0, b_num_t - num_noxf);
    b_drv_t = dmax(0.0, b_drv_t - drv_noxf);
  }
  int b_case = 0;
  double b_fn0 = 0, b_fv = 0, b_fn = 0;
  if (b_drv_t > 0.0 && b_num_t > b_drv_t * gm) {
    acc2ait = true;
    if (b_num_t > b_drv_t * v2n_ait) {
      b_fn0 = 1.0;
      b_fv = 1.0;
      b_case = 0;
    } else {
      b_fv = ((b_num_t / b_drv_t) - gm) / (v2n_ait - gm);
      b_fn0 = b_fv * (b_drv_t * v2n_ait / b_num_t);
      b_case = 1;
      if (b_fn0 <= 0.0 || b_fv <= 0.0) {
        b_fn0 = 0.0;
        b_fv = 0.0;
        b_case = 2;
      } else if (b_fn0 >= 1.0 || b_fv >= 1.0) {
        b_fn0 = 1.0;
        b_fv = 1.0;
        b_case = 3;
      }
    }
    b_fn = b_fn0 * b_num_t * safe_denominator(b_num_t0);
    xv_acc2ait = b_fv * adj_inv;
    xt10 = n_i_acc * (b_fn * adj_inv);
    xt11 = n_c_acc * (b_fn * adj_inv);
  }

  // ---- reverse
  double dv_ib[NMODE] = {0, 0, 0, 0}, dv_cb[NMODE] = {0, 0, 0, 0};
  double num_ib[NMODE] = {0, 0, 0, 0}, num_cb[NMODE] = {0, 0, 0, 0};
  double xt00b = 0, xt01b = 0, xt10b = 0, xt11b = 0, xv_a2b = 0, xv_b2b = 0, noxf_ib = 0;
  constexpr int acc_s[4] = {0, 2, 5, 6};
  constexpr int ait_s[4] = {8, 9, 10, 11};
  double dgn0b = dgnb[0], dgn1b = dgnb[1];
  if (ait2acc || acc2ait) {
    // species transfers
    if (acc2ait) {
      xt10b += pt_ib[12] - pt_ib[7];
      xt11b += pt_cb[12] - pt_cb[7];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        // xi = max(0, ai[acc]) * xv_acc2ait: pt_i[acc] -= xi, pt_i[ait] += xi
        const double xib = pt_ib[ait_s[k]] - pt_ib[acc_s[k]];
        const double xcb = pt_cb[ait_s[k]] - pt_cb[acc_s[k]];
        aib[acc_s[k]] += maxc_rev(0.0, ai[acc_s[k]], xib * xv_acc2ait);
        acb[acc_s[k]] += maxc_rev(0.0, ac[acc_s[k]], xcb * xv_acc2ait);
        xv_b2b += xib * dmax(0.0, ai[acc_s[k]]) + xcb * dmax(0.0, ac[acc_s[k]]);
      }
    }
    if (ait2acc) {
      xt00b += pt_ib[7] - pt_ib[12];
      xt01b += pt_cb[7] - pt_cb[12];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const double xib = pt_ib[acc_s[k]] - pt_ib[ait_s[k]];
        const double xcb = pt_cb[acc_s[k]] - pt_cb[ait_s[k]];
        aib[ait_s[k]] += maxc_rev(0.0, ai[ait_s[k]], xib * xv_ait2acc);
        acb[ait_s[k]] += maxc_rev(0.0, ac[ait_s[k]], xcb * xv_ait2acc);
        xv_a2b += xib * dmax(0.0, ai[ait_s[k]]) + xcb * dmax(0.0, ac[ait_s[k]]);
      }
    }
    // diameters after the transfer
    const double ndi = (xt00 - xt10) * dt;
    const double num_i1 = dmax(0.0, n_i_ait - ndi);
    const double num_i_acc = dmax(0.0, n_i_acc + ndi);
    const double vdi = (dv_i_ait * xv_ait2acc - (dv_i_acc - noxf_i) * xv_acc2ait) * dt;
    const double drv_i1 = dmax(0.0, dv_i_ait - vdi);
    const double drv_i_acc = dmax(0.0, dv_i_acc + vdi);
    double drv_i1b = 0, num_i1b = 0, drv_i_accb = 0, num_i_accb = 0;
    size_after_transfer_rev(drv_i1, num_i1, C.n2v_min[1], C.n2v_max[1], C.log_sig[1], dgn1b,
                            drv_i1b, num_i1b);
    size_after_transfer_rev(drv_i_acc, num_i_acc, C.n2v_min[0], C.n2v_max[0], C.log_sig[0],
                            dgn0b, drv_i_accb, num_i_accb);
    dgn0b = 0.0;
    dgn1b = 0.0;
    double vdib = 0.0, ndib = 0.0;
    {
      const double t = maxc_rev(0.0, dv_i_ait - vdi, drv_i1b);
      dv_ib[1] += t;
      vdib -= t;
      const double u = maxc_rev(0.0, dv_i_acc + vdi, drv_i_accb);
      dv_ib[0] += u;
      vdib += u;
    }
    // vdi = (dv_i_ait*xv_a2 - (dv_i_acc - noxf_i)*xv_b2) * dt
    dv_ib[1] += vdib * dt * xv_ait2acc;
    xv_a2b += vdib * dt * dv_i_ait;
    dv_ib[0] -= vdib * dt * xv_acc2ait;
    noxf_ib += vdib * dt * xv_acc2ait;
    xv_b2b -= vdib * dt * (dv_i_acc - noxf_i);
    {
      const double t = maxc_rev(0.0, n_i_ait - ndi, num_i1b);
      num_ib[1] += t;
      ndib -= t;
      const double u = maxc_rev(0.0, n_i_acc + ndi, num_i_accb);
      num_ib[0] += u;
      ndib += u;
    }
    xt00b += ndib * dt;
    xt10b -= ndib * dt;
  }
  // acc -> ait fractions
  if (acc2ait) {
    // xt10 = n_i_acc * (fn * adj_inv), xt11 = n_c_acc * (fn * adj_inv), xv = fv * adj_inv
    double fnb = (xt10b * n_i_acc + xt11b * n_c_acc) * adj_inv;
    num_ib[0] += xt10b * b_fn * adj_inv;
    num_cb[0] += xt11b * b_fn * adj_inv;
    double fvb = xv_b2b * adj_inv;
    // fn = fn0 * num_t * sd(num_t0)
    const double sd = safe_denominator(b_num_t0);
    double fn0b = fnb * b_num_t * sd;
    double num_tb = fnb * b_fn0 * sd;
    // sd(x) = x / (x^2 + e^2): d/dx = (e^2 - x^2) / (x^2 + e^2)^2
    const double e2 = K::eps * K::eps;
    const double den = b_num_t0 * b_num_t0 + e2;
    double num_t0b = fnb * b_fn0 * b_num_t * (e2 - b_num_t0 * b_num_t0) / (den * den);
    double drv_tb = 0.0;
    if (b_case == 1) {
      // fn0 = fv * (drv_t * v2n / num_t); fv = (num_t/drv_t - gm) / (v2n - gm)
      const double g = b_drv_t * v2n_ait / b_num_t;
      fvb += fn0b * g;
      drv_tb += fn0b * b_fv * v2n_ait / b_num_t;
      num_tb -= fn0b * b_fv * b_drv_t * v2n_ait / (b_num_t * b_num_t);
      const double rb = fvb / (v2n_ait - gm);
      num_tb += rb / b_drv_t;
      drv_tb -= rb * b_num_t / (b_drv_t * b_drv_t);
    }
    // num_t, drv_t after the no-transfer species correction (acc2ait
    // implies it was applied: the same test on the same values)
    const double drv_noxf = noxf_i + noxf_c;
    const double num_noxf = drv_noxf * C.n2v_max[0];
    const double ntb = maxc_rev(0.0, b_num_t_in - num_noxf, num_tb);
    const double dtb = maxc_rev(0.0, b_drv_t_in - drv_noxf, drv_tb);
    const double num_t_inb = ntb + num_t0b;  // num_t0 = num_t_in
    const double drv_noxfb = -dtb - ntb * C.n2v_max[0];
    noxf_ib += drv_noxfb;
    const double noxf_cb = drv_noxfb;
    num_ib[0] += num_t_inb;
    num_cb[0] += num_t_inb;
    dv_ib[0] += dtb;
    dv_cb[0] += dtb;
    // noxf_* = sum max(0, a[k]) * inv_density[0][k], k = 1, 3, 4
    const int ks[3] = {1, 3, 4};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      aib[ks[j]] += maxc_rev(0.0, ai[ks[j]], noxf_ib * C.inv_density[0][ks[j]]);
      acb[ks[j]] += maxc_rev(0.0, ac[ks[j]], noxf_cb * C.inv_density[0][ks[j]]);
    }
    (void)b_noxf;
  }
  // ait -> acc fractions
  if (ait2acc) {
    double fnb = (xt00b * n_i_ait + xt01b * n_c_ait) * adj_inv;
    num_ib[1] += xt00b * a_fn * adj_inv;
    num_cb[1] += xt01b * a_fn * adj_inv;
    double fvb = xv_a2b * adj_inv;
    double num_tb = 0.0, drv_tb = 0.0;
    if (a_case == 1) {
      const double g = a_drv_t * v2n_acc / a_num_t;
      fvb += fnb * g;
      drv_tb += fnb * a_fv * v2n_acc / a_num_t;
      num_tb -= fnb * a_fv * a_drv_t * v2n_acc / (a_num_t * a_num_t);
      const double rb = fvb / (v2n_acc - gm);
      num_tb += rb / a_drv_t;
      drv_tb -= rb * a_num_t / (a_drv_t * a_drv_t);
    }
    num_ib[1] += num_tb;
    num_cb[1] += num_tb;
    dv_ib[1] += drv_tb;
    dv_cb[1] += drv_tb;
  }
  // per-mode diameters and number adjustment
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    double v2nmin = C.n2v_min[m], v2nmax = C.n2v_max[m];
    if (m == 1)
      v2nmin /= 1.0e6;
    if (m == 0)
      v2nmax *= 1.0e6;
    const double db = (m == 0) ? dgn0b : (m == 1) ? dgn1b : dgnb[m];
    diameter_from_num_rev(dv_i[m], num_i[m], v2nmin, v2nmax, C.log_sig[m], db, dv_ib[m], num_ib[m]);
    const double init_i = ai[K::numslot(m)], init_c = ac[K::numslot(m)];
    double num_i0b = 0.0, num_c0b = 0.0;
    if (m >= 2) {
      adjust_num_sizes_rev(dv_i[m], dv_c[m], init_i, init_c, num_i0[m], num_c0[m], dt, C.n2v_min[m],
                           C.n2v_max[m], adj_inv, num_ib[m], num_cb[m], pt_ib[K::numslot(m)],
                           pt_cb[K::numslot(m)], dv_ib[m], dv_cb[m], aib[K::numslot(m)],
                           acb[K::numslot(m)], num_i0b, num_c0b);
    } else {
      num_i0b = num_ib[m];
      num_c0b = num_cb[m];
    }
    if (!(init_i < 0))
      aib[K::numslot(m)] += num_i0b;
    if (!(init_c < 0))
      acb[K::numslot(m)] += num_c0b;
#pragma unroll
    for (int s = 0; s < K::nspec(m); ++s) {
      aib[K::spec0(m) + s] += maxc_rev(0.0, ai[K::spec0(m) + s], dv_ib[m] * C.inv_density[m][s]);
      acb[K::spec0(m) + s] += maxc_rev(0.0, ac[K::spec0(m) + s], dv_cb[m] * C.inv_density[m][s]);
    }
  }
}


// ============================================================ water uptake
// qsat_water (Goff-Gratch, wv_sat_methods.hpp:14-46, 94-115): d qs / d T
MAM4B_HD double qsat_water_dT(double t, double p) {
  const double tboil = 373.16, ten = 10, one = 1;
  const double ln10 = 2.302585092994045684;
  const double a = 11.344 * (one - t / tboil), b = -3.49149 * (tboil / t - one);
  const double e = -7.90298 * (tboil / t - one) + 5.02808 * log10(tboil / t) -
                   1.3816e-7 * (pow(ten, a) - one) + 8.1328e-3 * (pow(ten, b) - one) +
                   log10(1013.246);
  const double es = pow(ten, e) * ten * ten;
  if ((p - es) <= 0)
    return 0.0;
  const double de = 7.90298 * tboil / (t * t) - 5.02808 / (t * ln10) +
                    1.3816e-7 * pow(ten, a) * ln10 * (11.344 / tboil) +
                    8.1328e-3 * pow(ten, b) * ln10 * (3.49149 * tboil / (t * t));
  const double des = es * ln10 * de;
  const double epsilo = 0.018016 / 0.028966;
  const double omeps = 1 - epsilo;
  const double d = p - omeps * es;
  return des * epsilo * p / (d * d);
}

// water_uptake_rh: rh from qv, T (P, cloud fraction fixed)
MAM4B_HD void water_uptake_rh_rev(double qv, double temp, double pmid, double cldn, double rhb,
                                  double &qvb, double &tb) {
  const double qs = qsat_water(temp, pmid);
  const double rh_max = 0.98;
  const double rh0 = (qs > qv) ? qv / qs : rh_max;
  const double rh1 = bound(0.0, rh_max, rh0);
  double rh2 = rh1;
  if (cldn < 1.0)
    rh2 = (rh1 - cldn) / (1.0 - cldn);
  double b = maxc_rev(0.0, rh2, rhb);  // rh = dmax(rh2, 0)
  if (cldn < 1.0)
    b /= (1.0 - cldn);
  b = boundc_rev(0.0, rh_max, rh0, b);
  if (qs > qv) {
    qvb += b / qs;
    tb -= b * qv / (qs * qs) * qsat_water_dT(temp, pmid);
  }
}

// kohler (water_uptake.hpp:180-230); returns the wet radius in m
MAM4B_HD void kohler_rev(const StepConsts &C, double rdry_in, double hygro, double rh,
                         double rwb_out, double &rdry_inb, double &hygrob, double &rhb) {
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
  // rwet = dmin(rwet, 30) then * 1e-6
  const double rwetb = minc_rev(30.0, rwet, rwb_out * 1.e-6);
  double rdryb = 0.0, slogb = 0.0, volb = 0.0, bbb = 0.0;
  if (pp < eps) {
    const double D = 1.0 - slog * rdry / aa;
    rdryb += rwetb * (1.0 + pp * (1.0 / 3.0) / D);
    const double ppb = rwetb * rdry * (1.0 / 3.0) / D;
    const double Db = -rwetb * rdry * pp * (1.0 / 3.0) / (D * D);
    slogb -= Db * rdry / aa;
    rdryb -= Db * slog / aa;
    // pp = |bb| / (aa rdry^2)
    const double sg = (-bb / aa) < 0 ? 1.0 : -1.0;  // d|(-bb/aa)|/dbb = -sign(-bb/aa)/aa
    bbb += ppb * sg / aa / (rdry * rdry);
    rdryb -= ppb * 2.0 * pp / rdry;
  } else if (rwet == 1000.0 * rdry) {
    rdryb += rwetb * 1000.0;
  } else {
    // implicit: P(x) = x^4 + p43 x^3 + p41 x + p40 = 0
    const double x = rwet;
    const double dP = 4.0 * x * x * x + 3.0 * p43 * x * x + p41;
    const double p43b = -rwetb * x * x * x / dP;
    const double p41b = -rwetb * x / dP;
    const double p40b = -rwetb / dP;
    slogb += p43b * aa / (slog * slog);
    bbb += p41b / slog;
    slogb -= p41b * bb / (slog * slog);
    volb -= p41b;
    volb += p40b * aa / slog;
    slogb -= p40b * aa * vol / (slog * slog);
  }
  volb += bbb * hygro;
  hygrob += bbb * vol;
  rdryb += volb * 3.0 * rdry * rdry;
  rhb += boundc_rev(1.e-10, 1.0 - eps, rh, slogb / ss);
  rdry_inb += rdryb * 1.e6;
}

// water_uptake_mode<M>: inputs species masses sp[], rh, dgn_a; outputs
// dgn_awet, qaerwat, wetdens (cotangents dwb, qwb, wdb)
template <int M>
MAM4B_HD void water_uptake_mode_rev(const StepConsts &C, const double (&sp)[7], double rh,
                                    double dgn_a, double dwb, double qwb, double wdb,
                                    double (&spb)[7], double &rhb, double &dgn_ab) {
  // ---- forward
  double hygro0 = 0.0, dryvolmr = 0.0, maer = 0.0;
#pragma unroll
  for (int s = 0; s < K::nspec(M); ++s) {
    const int w = K::spec0(M) + s - M;
    const double vol_tmp = sp[s] / K::wu_dens(w);
    maer = maer + sp[s];
    dryvolmr += vol_tmp;
    hygro0 += vol_tmp * K::wu_hygro(w);
  }
  const int w0 = K::spec0(M) - M;
  const bool hy = dryvolmr > 1e-30;
  const double hygro = hy ? hygro0 / dryvolmr : K::wu_hygro(w0);
  const double e45 = exp(4.5 * sq(C.log_sig[M]));
  const double v2ncur_a = 1.0 / ((K::pi / 6.0) * cube(dgn_a) * e45);
  const double naer = dryvolmr * v2ncur_a;
  const bool dd = maer > 1e-31;
  const double drydens = dd ? maer / dryvolmr : 1.0;
  const double dryvol = 1.0 / v2ncur_a;
  const double drymass = drydens * dryvol;
  const double dryrad = cbrt(dryvol / (K::pi * 4.0 / 3.0));
  // below the crystallisation humidity the Kohler radius is discarded (the
  // forward skips it): nothing of it enters the outputs or their cotangents
  const bool dry = rh < K::rh_cryst;
  double wr0 = dryrad, wr1 = dryrad, wv0 = dryvol, wv1 = dryvol, wt0 = 0.0;
  if (!dry) {
    wr0 = kohler(C, dryrad, hygro, rh);
    wr1 = dmax(wr0, dryrad);
    wv0 = (K::pi * 4.0 / 3.0) * cube(wr1);
    wv1 = dmax(wv0, dryvol);
    wt0 = dmax(wv1 - dryvol, 0.0);
  }
  int hbranch = 0;
  double wetrad = wr1, wetvol = wv1, wtrvol = wt0, wt1 = 0.0;
  if (rh < K::rh_cryst) {
    hbranch = 1;
    wetrad = dryrad;
    wetvol = dryvol;
    wtrvol = 0.0;
  } else if (rh < K::rh_deliq) {
    hbranch = 2;
    wt1 = wt0 * C.hystfac * (rh - K::rh_cryst);
    wtrvol = dmax(wt1, 0.0);
    wetvol = dryvol + wtrvol;
    wetrad = cbrt(wetvol / (4.0 / 3.0 * K::pi));
  }
  // ---- reverse
  double naerb = 0.0, wtrvolb = 0.0, wetvolb = 0.0, drymassb = 0.0, wetradb = 0.0;
  double dryradb = 0.0, dryvolb = 0.0, hygrob = 0.0;
  // dgn_awet = dgn_a * (wetrad / dryrad)
  dgn_ab += dwb * (wetrad / dryrad);
  wetradb += dwb * dgn_a / dryrad;
  dryradb -= dwb * dgn_a * wetrad / (dryrad * dryrad);
  // qaerwat = 1e3 naer wtrvol
  naerb += qwb * 1.0e3 * wtrvol;
  wtrvolb += qwb * 1.0e3 * naer;
  // wetdens
  if (wetvol > 1.0e-30) {
    drymassb += wdb / wetvol;
    wtrvolb += wdb * 1.0e3 / wetvol;
    wetvolb -= wdb * (drymass + 1.0e3 * wtrvol) / (wetvol * wetvol);
  }
  double wt0b = 0.0, wv1b = 0.0, wr1b = 0.0;
  if (hbranch == 1) {
    dryradb += wetradb;
    dryvolb += wetvolb;
  } else if (hbranch == 2) {
    // wetrad = cbrt(wetvol / (4/3 pi)) -> d/dwetvol = wetrad / (3 wetvol)
    wetvolb += wetradb * wetrad / (3.0 * wetvol);
    dryvolb += wetvolb;
    wtrvolb += wetvolb;
    const double wt1b = maxc_rev(0.0, wt1, wtrvolb);
    wt0b += wt1b * C.hystfac * (rh - K::rh_cryst);
    rhb += wt1b * wt0 * C.hystfac;
  } else {
    wt0b += wtrvolb;
    wv1b += wetvolb;
    wr1b += wetradb;
  }
  if (!dry) {
    // wt0 = dmax(wv1 - dryvol, 0)
    {
      const double t = maxc_rev(0.0, wv1 - dryvol, wt0b);
      wv1b += t;
      dryvolb -= t;
    }
    // wv1 = dmax(wv0, dryvol)
    double wv0b = 0.0;
    max_rev(wv0, dryvol, wv1b, wv0b, dryvolb);
    wr1b += wv0b * (K::pi * 4.0 / 3.0) * 3.0 * wr1 * wr1;
    // wr1 = dmax(wr0, dryrad)
    double wr0b = 0.0;
    max_rev(wr0, dryrad, wr1b, wr0b, dryradb);
    kohler_rev(C, dryrad, hygro, rh, wr0b, dryradb, hygrob, rhb);
  }
  // dryrad = cbrt(dryvol / (4/3 pi))
  dryvolb += dryradb * dryrad / (3.0 * dryvol);
  // drymass = drydens * dryvol
  double drydensb = drymassb * dryvol;
  dryvolb += drymassb * drydens;
  // dryvol = 1 / v2ncur_a, naer = dryvolmr * v2ncur_a
  double v2nb = -dryvolb / (v2ncur_a * v2ncur_a) + naerb * dryvolmr;
  double dryvolmrb = naerb * v2ncur_a;
  // v2ncur_a = 1 / ((pi/6) dgn^3 e45): d/d dgn = -3 v2n / dgn
  dgn_ab += v2nb * (-3.0 * v2ncur_a / dgn_a);
  double maerb = 0.0;
  if (dd) {
    maerb += drydensb / dryvolmr;
    dryvolmrb -= drydensb * maer / (dryvolmr * dryvolmr);
  }
  double hygro0b = 0.0;
  if (hy) {
    hygro0b += hygrob / dryvolmr;
    dryvolmrb -= hygrob * hygro0 / (dryvolmr * dryvolmr);
  }
#pragma unroll
  for (int s = 0; s < K::nspec(M); ++s) {
    const int w = K::spec0(M) + s - M;
    const double vtb = dryvolmrb + hygro0b * K::wu_hygro(w);
    spb[s] += maerb + vtb / K::wu_dens(w);
  }
}

// relative humidity of amicphys (Magnus, mam4_amicphys.hpp:2202-2235):
// relhumgcm = clamp(qv / qv_sat(T, p), 0, 1)
MAM4B_HD void relhum_gcm_rev(double qv, double temp, double pmid, double rb, double &qvb,
                             double &tb) {
  const double epsqs = 0.018016 / 0.028966;
  const double tc = temp - 273.15;
  const double ew = 610.94 * exp(17.625 * tc / (234.04 + tc));
  const double ev_sat = 1.00071 * exp(4.5e-8 * pmid) * ew;
  const double den = pmid - (1 - epsqs) * ev_sat;
  const double qv_sat = epsqs * ev_sat / den;
  const double r0 = qv / qv_sat;
  // dmax(0, dmin(1, r0))
  const double m = dmin(1.0, r0);
  double r0b = 0.0;
  if (0.0 < m && r0 < 1.0)
    r0b = rb;
  qvb += r0b / qv_sat;
  const double qsb = -r0b * qv / (qv_sat * qv_sat);
  const double evb = qsb * epsqs * pmid / (den * den);
  const double ewb = evb * 1.00071 * exp(4.5e-8 * pmid);
  tb += ewb * ew * 17.625 * 234.04 / ((234.04 + tc) * (234.04 + tc));
}

// h2so4_diffusivity: gas_diffus, freepath as functions of T (p fixed)
MAM4B_HD void h2so4_diffusivity_rev(double temp, double pmid, double gdb, double fpb,
                                    double &tb) {
  double gd, fp;
  h2so4_diffusivity(temp, pmid, gd, fp);
  const double speed = 145.5 * sqrt(temp / 9.807840000000000E+01);
  // fp = 3 gd / speed; gd ~ T^1.75; speed ~ T^0.5
  gdb += fpb * 3.0 / speed;
  const double speedb = -fpb * 3.0 * gd / (speed * speed);
  tb += gdb * gd * 1.75 / temp + speedb * speed / (2.0 * temp);
}

// ====================================================== forward-mode duals
// Value and N tangents; used for the scalar functions with a handful of
// inputs and many terms (uptake rates, coagulation coefficients,
// nucleation rates), evaluated from templated copies of their formulas.
template <int N>
struct Dual {
  double v;
  double d[N];
};
template <int N>
MAM4B_HD Dual<N> dconst(double v) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = 0.0;
  return r;
}
template <int N>
MAM4B_HD Dual<N> dvar(double v, int i) {
  Dual<N> r = dconst<N>(v);
  r.d[i] = 1.0;
  return r;
}
template <int N>
MAM4B_HD Dual<N> dchain(double v, const Dual<N> &a, double g) {
  Dual<N> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = g * a.d[i];
  return r;
}
template <int N>
MAM4B_HD Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
MAM4B_HD Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
MAM4B_HD Dual<N> operator-(const Dual<N> &a) {
  return dchain(-a.v, a, -1.0);
}
template <int N>
MAM4B_HD Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
MAM4B_HD Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
  Dual<N> r;
  r.v = a.v / b.v;
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
  return r;
}
template <int N> MAM4B_HD Dual<N> operator+(const Dual<N> &a, double b) { return dchain(a.v + b, a, 1.0); }
template <int N> MAM4B_HD Dual<N> operator+(double a, const Dual<N> &b) { return dchain(a + b.v, b, 1.0); }
template <int N> MAM4B_HD Dual<N> operator-(const Dual<N> &a, double b) { return dchain(a.v - b, a, 1.0); }
template <int N> MAM4B_HD Dual<N> operator-(double a, const Dual<N> &b) { return dchain(a - b.v, b, -1.0); }
template <int N> MAM4B_HD Dual<N> operator*(const Dual<N> &a, double b) { return dchain(a.v * b, a, b); }
template <int N> MAM4B_HD Dual<N> operator*(double a, const Dual<N> &b) { return dchain(a * b.v, b, a); }
template <int N> MAM4B_HD Dual<N> operator/(const Dual<N> &a, double b) { return dchain(a.v / b, a, 1.0 / b); }
template <int N> MAM4B_HD Dual<N> operator/(double a, const Dual<N> &b) {
  const double v = a / b.v;
  return dchain(v, b, -v / b.v);
}
template <int N> MAM4B_HD bool operator<(const Dual<N> &a, const Dual<N> &b) { return a.v < b.v; }
template <int N> MAM4B_HD bool operator<(const Dual<N> &a, double b) { return a.v < b; }
template <int N> MAM4B_HD bool operator<(double a, const Dual<N> &b) { return a < b.v; }
template <int N> MAM4B_HD bool operator>(const Dual<N> &a, double b) { return a.v > b; }
template <int N> MAM4B_HD bool operator<=(const Dual<N> &a, double b) { return a.v <= b; }
template <int N> MAM4B_HD bool operator>=(const Dual<N> &a, double b) { return a.v >= b; }
template <int N> MAM4B_HD bool operator<=(const Dual<N> &a, const Dual<N> &b) { return a.v <= b.v; }
template <int N> MAM4B_HD bool operator>=(const Dual<N> &a, const Dual<N> &b) { return a.v >= b.v; }
template <int N> MAM4B_HD bool operator>(const Dual<N> &a, const Dual<N> &b) { return a.v > b.v; }
template <int N> MAM4B_HD Dual<N> exp(const Dual<N> &a) {
  const double v = ::exp(a.v);
  return dchain(v, a, v);
}
template <int N> MAM4B_HD Dual<N> log(const Dual<N> &a) { return dchain(::log(a.v), a, 1.0 / a.v); }
template <int N> MAM4B_HD Dual<N> sqrt(const Dual<N> &a) {
  const double v = ::sqrt(a.v);
  return dchain(v, a, 0.5 / v);
}
template <int N> MAM4B_HD Dual<N> cbrt(const Dual<N> &a) {
  const double v = ::cbrt(a.v);
  return dchain(v, a, v / (3.0 * a.v));
}
template <int N> MAM4B_HD Dual<N> pow(const Dual<N> &a, double y) {
  const double v = ::pow(a.v, y);
  return dchain(v, a, y * ::pow(a.v, y - 1.0));
}
template <int N> MAM4B_HD Dual<N> pow(const Dual<N> &a, const Dual<N> &y) {
  const double v = ::pow(a.v, y.v);
  Dual<N> r;
  r.v = v;
  const double ga = y.v * ::pow(a.v, y.v - 1.0), gy = v * ::log(a.v);
#pragma unroll
  for (int i = 0; i < N; ++i)
    r.d[i] = ga * a.d[i] + gy * y.d[i];
  return r;
}
template <int N> MAM4B_HD Dual<N> dmax(const Dual<N> &a, const Dual<N> &b) { return (a.v < b.v) ? b : a; }
template <int N> MAM4B_HD Dual<N> dmin(const Dual<N> &a, const Dual<N> &b) { return (b.v < a.v) ? b : a; }
template <int N> MAM4B_HD Dual<N> dmax(double a, const Dual<N> &b) { return (a < b.v) ? b : dconst<N>(a); }
template <int N> MAM4B_HD Dual<N> dmax(const Dual<N> &a, double b) { return (a.v < b) ? dconst<N>(b) : a; }
template <int N> MAM4B_HD Dual<N> dmin(double a, const Dual<N> &b) { return (b.v < a) ? b : dconst<N>(a); }
template <int N> MAM4B_HD Dual<N> dmin(const Dual<N> &a, double b) { return (b < a.v) ? dconst<N>(b) : a; }
// the double-precision functions stay visible next to the Dual overloads
using ::cbrt;
using ::exp;
using ::log;
using ::pow;
using ::sqrt;
using mam4b::dmax;
using mam4b::dmin;
template <int N> MAM4B_HD double val(const Dual<N> &a) { return a.v; }
MAM4B_HD double val(double a) { return a; }

// uptake_rate_mode as a template over the number type (same formula)
template <class R>
MAM4B_HD R uptake_rate_mode_t(const StepConsts &C, int n, const R &gasdiffus, const R &freepath,
                              const R &dgn_awet) {
  const double tworootpi = 2 * ::sqrt(K::pi);
  const double root2 = ::sqrt(2.0);
  const double xg = 7.071067690849304E-01;
  const double wg = 8.862269520759583E-01;
  const double a283 = 0.65 * 0.283, a75 = 0.65 * 0.75;
  const double lnsg = C.log_sig[n];
  const R lndpgn = log(dgn_awet);
  const R kn = 2.0 * freepath / dgn_awet;
  const R tmpa = 1.0 / (1.0 + kn) - (2.0 * kn + 1.0 + a283) / (kn * (kn + 1.0 + a283) + a75);
  R beta = 1.0 - kn * tmpa;
  beta = dmax(1.0, dmin(2.0, beta));
  const R constant = tworootpi * exp(beta * lndpgn + 0.5 * pow(beta * lnsg, 2.0));
  R sum = 0.0 * kn;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const R lndp = lndpgn + beta * lnsg * lnsg + root2 * lnsg * (q == 0 ? xg : -xg);
    const R dp = exp(lndp);
    const R knq = 2.0 * freepath / dp;
    const R hh = (a75 * (1.0 + knq)) / (knq * (knq + 1.0 + a283) + a75);
    sum = sum + wg * dp * hh / pow(dp, beta);
  }
  return constant * gasdiffus * sum;
}

MAM4B_HD void uptake_rate_mode_rev(const StepConsts &C, int n, double gasdiffus, double freepath,
                                   double dgn_awet, double rb, double &gdb, double &fpb,
                                   double &dgb) {
  const Dual<3> r = uptake_rate_mode_t<Dual<3>>(C, n, dvar<3>(gasdiffus, 0), dvar<3>(freepath, 1),
                                                dvar<3>(dgn_awet, 2));
  gdb += rb * r.d[0];
  fpb += rb * r.d[1];
  dgb += rb * r.d[2];
}


// ============================================================ coagulation
// getcoags for one pair (coag_coefs) as a template over the number type
template <class R>
MAM4B_HD void coag_coefs_t(const CoagTables &T, const R &airtemp, double airprs, const R &dgatk,
                           const R &dgacc, double sgatk, double sgacc, double xxlsgat,
                           double xxlsgac, const R &pdensat, const R &pdensac, R &bij0, R &bij3,
                           R &bii0, R &bjj0) {
  const double t0 = 273.15 + 15.0;
  const R sqrt_temp = sqrt(airtemp);
  const R lamda = 6.6328e-8 * 101325.0 * airtemp / (t0 * airprs);
  const R amu = 1.458e-6 * airtemp * sqrt_temp / (airtemp + 110.4);
  const double boltzmann = 1.3806500000000000e-023;
  const R knc = (2.0 / 3.0) * boltzmann * airtemp / amu;
  const R kfmat = sqrt(3.0 * boltzmann * airtemp / pdensat);
  const R kfmac = sqrt(3.0 * boltzmann * airtemp / pdensac);
  const R kfmatac = sqrt(6.0 * boltzmann * airtemp / (pdensat + pdensac));
  const double a = 1.246;
  const double esat01 = ::exp(0.125 * xxlsgat * xxlsgat);
  const double esac01 = ::exp(0.125 * xxlsgac * xxlsgac);
  const double dlgsqt2 = 1.0 / ::log(::sqrt(2.0));
  const double esat04 = ::pow(esat01, 4.0), esac04 = ::pow(esac01, 4.0);
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
  const R dgat3 = dgatk * dgatk * dgatk;
  const R sqdgat = sqrt(dgatk), sqdgac = sqrt(dgacc);
  const R sqdgat7 = dgat3 * sqdgat;
  const R r1 = sqdgac / sqdgat;
  const R r2 = r1 * r1;
  const R rx4 = r2 * r2;
  const R ri1 = 1.0 / r1;
  const R ri2 = 1.0 / (r1 * r1);
  const R ri3 = 1.0 / (r1 * r1 * r1);
  const R kngat = 2.0 * lamda / dgatk;
  const R kngac = 2.0 * lamda / dgacc;
  const double rat = val(dgacc) / val(dgatk);
  const int n2n = (int)mam4b::dmax(1.0, mam4b::dmin(10.0, ::round(4.0 * (sgatk - 0.75)))) - 1;
  const int n2a = (int)mam4b::dmax(1.0, mam4b::dmin(10.0, ::round(4.0 * (sgacc - 0.75)))) - 1;
  const int n1 = (int)mam4b::dmax(1.0, mam4b::dmin(10.0, 1.0 + ::round(dlgsqt2 * ::log(rat)))) - 1;
  const int tix = n1 * 100 + n2n * 10 + n2a;
  const double bm0ij = MAM4B_LDG(T.bm0ij + tix);
  const double bm3i = MAM4B_LDG(T.bm3i + tix);
  const R coagnc0 = knc * (2.0 + a * (kngat * (esat04 + r2 * esat16 * esac04) +
                                      kngac * (esac04 + ri2 * esac16 * esat04)) +
                           (r2 + ri2) * esat04 * esac04);
  const R coagfm0 = kfmatac * sqdgat * bm0ij *
                    (esat01 + r1 * esac01 + 2.0 * r2 * esat01 * esac04 + rx4 * esat09 * esac16 +
                     ri3 * esat16 * esac09 + 2.0 * ri1 * esat04 + esac01);
  const R qn12 = coagnc0 * coagfm0 / (coagnc0 + coagfm0);
  const R coagnc3 = knc * dgat3 *
                    (2.0 * esat36 + a * kngat * (esat16 + r2 * esat04 * esac04) +
                     a * kngac * (esat36 * esac04 + ri2 * esat64 * esac16) + r2 * esat16 * esac04 +
                     ri2 * esat64 * esac04);
  const R coagfm3 = kfmatac * sqdgat7 * bm3i *
                    (esat49 + r1 * esat36 * esac01 + 2.0 * r2 * esat25 * esac04 +
                     rx4 * esat09 * esac16 + ri3 * esat100 * esac09 + 2.0 * ri1 * esat64 * esac01);
  const R qv12 = coagnc3 * coagfm3 / (coagnc3 + coagfm3);
  const R cnc11 = knc * (1.0 + esat08 + a * kngat * (esat20 + esat04));
  const R cfm11 = kfmat * sqdgat * MAM4B_LDG(T.bm0 + n2n) * (esat01 + esat25 + 2.0 * esat05);
  const R qn11 = cfm11 * cnc11 / (cfm11 + cnc11);
  const R cnc22 = knc * (1.0 + esac08 + a * kngac * (esac20 + esac04));
  const R cfm22 = kfmac * sqdgac * MAM4B_LDG(T.bm0 + n2a) * (esac01 + esac25 + 2.0 * esac05);
  const R qn22 = cfm22 * cnc22 / (cfm22 + cnc22);
  bii0 = dmax(0.0, qn11);
  bjj0 = dmax(0.0, qn22);
  bij0 = dmax(0.0, qn12);
  const R dumatk3 = (dgatk * dgatk * dgatk) * ::exp(4.5 * xxlsgat * xxlsgat);
  bij3 = dmax(0.0, qv12 / dumatk3);
}

// coag_pair_coefs (x aircon = p / (R T)): cotangents of the 4 coefficients
// to T, the two wet diameters and the two wet densities
MAM4B_HD void coag_pair_coefs_rev(const StepConsts &C, const CoagTables &T, int p, double temp,
                                  double pmid, double dgn_src, double dgn_dst, double dens_src,
                                  double dens_dst, const double (&cb)[4], double &tb,
                                  double &dsb, double &ddb, double &rsb, double &rdb) {
  typedef Dual<5> D5;
  const int sm = coag_src(p), dm = coag_dst(p);
  const D5 t = dvar<5>(temp, 0);
  D5 b0, b3, bi, bj;
  coag_coefs_t<D5>(T, t, pmid, dvar<5>(dgn_src, 1), dvar<5>(dgn_dst, 2), K::sig(sm), K::sig(dm),
                   C.log_sig[sm], C.log_sig[dm], dvar<5>(dens_src, 3), dvar<5>(dens_dst, 4), b0, b3,
                   bi, bj);
  const D5 aircon = pmid / (8314.46759100000 * t);
  const D5 r[4] = {b0 * aircon, b3 * aircon, bi * aircon, bj * aircon};
  double g[5] = {0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int i = 0; i < 5; ++i)
      g[i] += cb[k] * r[k].d[i];
  tb += g[0];
  dsb += g[1];
  ddb += g[2];
  rsb += g[3];
  rdb += g[4];
}

// qnum_intra_inter (coagulation.hpp:938-952): cotangents to its 3 inputs
MAM4B_HD void qnum_intra_inter_rev(double bq, double biidt, double q0, double rb, double &bqb,
                                   double &biidtb, double &q0b) {
  if (bq < 1.0e-5) {
    // r = q0 / D, D = 1 + (bq + biidt q0) (1 + 0.5 bq)
    const double A = bq + biidt * q0, B = 1.0 + 0.5 * bq;
    const double D = 1.0 + A * B;
    const double r = q0 / D;
    q0b += rb / D;
    const double Db = -rb * r / D;
    const double Ab = Db * B, Bb = Db * A;
    bqb += Ab + 0.5 * Bb;
    biidtb += Ab * q0;
    q0b += Ab * biidt;
    return;
  }
  // r = q0 e / D, e = exp(-bq), D = 1 + (biidt q0 / bq)(1 - e)
  const double e = ::exp(-bq);
  const double F = biidt * q0 / bq;
  const double D = 1.0 + F * (1.0 - e);
  const double r = q0 * e / D;
  q0b += rb * e / D;
  double eb = rb * q0 / D;
  const double Db = -rb * r / D;
  const double Fb = Db * (1.0 - e);
  eb -= Db * F;
  bqb += -eb * e;
  biidtb += Fb * q0 / bq;
  q0b += Fb * biidt / bq;
  bqb -= Fb * F / bq;
}

// coagulation (mam_coag_1subarea with coefficients cc): state s in, s out
// (in place in the forward); sb holds the cotangent of s after on entry and
// of s before on return; ccb receives the coefficients' cotangents.
MAM4B_HD void coagulation_rev(double deltat, const double (&cc)[12], const Sub &s_in, Sub &sb,
                              double (&ccb)[12], const double (&coag_inb)[NAER]) {
  // ---- forward recomputation
  double bgn[NAER][NMODE], nbgn[NMODE];
#pragma unroll
  for (int a = 0; a < NAER; ++a)
#pragma unroll
    for (int m = 0; m < NMODE; ++m)
      bgn[a][m] = dmax(0.0, s_in.aer[a][m]);
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    nbgn[m] = dmax(0.0, s_in.num[m]);
  const double bij0[3] = {cc[0], cc[1], cc[2]}, bij3[3] = {cc[3], cc[4], cc[5]};
  const double bii0[3] = {cc[6], cc[7], cc[8]}, bjj0[3] = {cc[9], cc[10], cc[11]};
  double bij0b[3] = {0, 0, 0}, bij3b[3] = {0, 0, 0}, bii0b[3] = {0, 0, 0}, bjj0b[3] = {0, 0, 0};
  const double n0 = nbgn[0] / (1.0 + bjj0[0] * deltat * nbgn[0]);
  const double tavg0 = (nbgn[0] + n0) * 0.5;
  const double x3a = dmax(0.0, deltat * bij0[1] * tavg0), x3b = dmax(0.0, deltat * bii0[1]);
  const double n3 = qnum_intra_inter(x3a, x3b, nbgn[3]);
  const double tavg3 = (nbgn[3] + n3) * 0.5;
  const double bq = bij0[0] * tavg0 + bij0[2] * tavg3;
  const double x1a = dmax(0.0, deltat * bq), x1b = dmax(0.0, deltat * bii0[0]);
  const double bq1 = dmax(0.0, bij3[0] * tavg0);
  const double bq2 = dmax(0.0, bij3[2] * tavg3);
  const double dc1 = bq1 + bq2, df1 = deltat * dc1;
  const bool t1 = df1 > K::eps * 2.0;
  const double dc2 = dmax(0.0, bij3[1] * tavg0), df2 = deltat * dc2;
  const bool t2 = df2 > K::eps * 2.0;
  // ---- reverse: mass updates (second block, then first)
  double bgnb[NAER][NMODE], nbgnb[NMODE] = {0, 0, 0, 0};
#pragma unroll
  for (int a = 0; a < NAER; ++a)
#pragma unroll
    for (int m = 0; m < NMODE; ++m)
      bgnb[a][m] = sb.aer[a][m];  // s.aer starts as bgn (clipped copy)
  double tavg0b = 0.0, tavg3b = 0.0;
  if (t2) {
    const double xf = 1.0 - ::exp(-df2);
    double xfb = 0.0;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      // dq = xf * bgn[a][3]; aer[a][3] -= dq; aer[a][0] += dq
      const double dqb = sb.aer[a][0] - sb.aer[a][3];
      xfb += dqb * bgn[a][3];
      bgnb[a][3] += dqb * xf;
    }
    const double df2b = xfb * ::exp(-df2);
    const double dc2b = df2b * deltat;
    const double pb = maxc_rev(0.0, bij3[1] * tavg0, dc2b);
    bij3b[1] += pb * tavg0;
    tavg0b += pb * bij3[1];
  }
  if (t1) {
    const double prtn2 = bq2 / dc1, prtn1 = 1.0 - prtn2;
    const double xf = 1.0 - ::exp(-df1);
    double xfb = 0.0, prtn1b = 0.0, prtn2b = 0.0;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      // dq = xf bgn[a][1]; aer[a][1] -= dq; aer[a][0] += dq prtn1;
      // aer[a][3] += dq prtn2; coag_in[a] += dq prtn2
      const double dq = xf * bgn[a][1];
      const double dqb = -sb.aer[a][1] + (sb.aer[a][0]) * prtn1 +
                         (sb.aer[a][3] + coag_inb[a]) * prtn2;
      prtn1b += sb.aer[a][0] * dq;
      prtn2b += (sb.aer[a][3] + coag_inb[a]) * dq;
      xfb += dqb * bgn[a][1];
      bgnb[a][1] += dqb * xf;
    }
    prtn2b -= prtn1b;
    double bq2b = prtn2b / dc1;
    double dc1b = -prtn2b * bq2 / (dc1 * dc1);
    const double df1b = xfb * ::exp(-df1);
    dc1b += df1b * deltat;
    double bq1b = dc1b;
    bq2b += dc1b;
    const double p1 = maxc_rev(0.0, bij3[0] * tavg0, bq1b);
    bij3b[0] += p1 * tavg0;
    tavg0b += p1 * bij3[0];
    const double p2 = maxc_rev(0.0, bij3[2] * tavg3, bq2b);
    bij3b[2] += p2 * tavg3;
    tavg3b += p2 * bij3[2];
  }
  // number updates: s.num[1] = qnum(x1a, x1b, nbgn[1]); s.num[3] = n3; s.num[0] = n0
  {
    double x1ab = 0, x1bb = 0;
    qnum_intra_inter_rev(x1a, x1b, nbgn[1], sb.num[1], x1ab, x1bb, nbgnb[1]);
    const double bqb = maxc_rev(0.0, deltat * bq, x1ab) * deltat;
    bii0b[0] += maxc_rev(0.0, deltat * bii0[0], x1bb) * deltat;
    bij0b[0] += bqb * tavg0;
    tavg0b += bqb * bij0[0];
    bij0b[2] += bqb * tavg3;
    tavg3b += bqb * bij0[2];
  }
  {
    double n3b = sb.num[3] + tavg3b * 0.5;
    nbgnb[3] += tavg3b * 0.5;
    double x3ab = 0, x3bb = 0;
    qnum_intra_inter_rev(x3a, x3b, nbgn[3], n3b, x3ab, x3bb, nbgnb[3]);
    const double pa = maxc_rev(0.0, deltat * bij0[1] * tavg0, x3ab) * deltat;
    bij0b[1] += pa * tavg0;
    tavg0b += pa * bij0[1];
    bii0b[1] += maxc_rev(0.0, deltat * bii0[1], x3bb) * deltat;
  }
  {
    const double n0b = sb.num[0] + tavg0b * 0.5;
    nbgnb[0] += tavg0b * 0.5;
    // n0 = nb0 / (1 + bjj0 dt nb0)
    const double D = 1.0 + bjj0[0] * deltat * nbgn[0];
    nbgnb[0] += n0b / D;
    const double Db = -n0b * n0 / D;
    bjj0b[0] += Db * deltat * nbgn[0];
    nbgnb[0] += Db * bjj0[0] * deltat;
  }
  nbgnb[2] += sb.num[2];
  // clipping of the incoming state
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    sb.num[m] = maxc_rev(0.0, s_in.num[m], nbgnb[m]);
#pragma unroll
  for (int a = 0; a < NAER; ++a)
#pragma unroll
    for (int m = 0; m < NMODE; ++m)
      sb.aer[a][m] = maxc_rev(0.0, s_in.aer[a][m], bgnb[a][m]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    ccb[k] += bij0b[k];
    ccb[3 + k] += bij3b[k];
    ccb[6 + k] += bii0b[k];
    ccb[9 + k] += bjj0b[k];
  }
}


// r = dmax(x, c) with constant c (returns x unless x < c)
MAM4B_HD double maxxc_rev(double x, double c, double rb) { return (x < c) ? 0.0 : rb; }

// ======================================================= H2SO4 condensation
// h2so4_update (gasaerexch.hpp:486-537): inputs q1 = s.gas[1], netprod,
// uptk[4], s.aer[1][n]; outputs s.gas[1], s.aer[1][n], qavg.
MAM4B_HD void h2so4_update_rev(double dt, double netprod, double q1, const double (&uptk)[NMODE],
                               double g1b, double qavgb, double (&a1b)[NMODE], double &q1b,
                               double &netprodb, double (&uptkb)[NMODE]) {
  double tmpa = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    tmpa += uptk[n];
  const double kxt = tmpa * dt, pxt = netprod * dt;
  double kxtb = 0.0, pxtb = 0.0, tmpab = 0.0;
  if (kxt >= 1.0e-20) {
    double q3, q4, q3b = g1b, q4b = qavgb;
    // aerosol: a1[n] += qdel * (uptk[n] / tmpa), qdel = (q1 + pxt) - q3
    double qdelb = 0.0;
    double qdel;
    if (kxt > 0.001) {
      const double pok = pxt / kxt;
      const double e = ::exp(-kxt);
      q3 = (q1 - pok) * e + pok;
      q4 = (q1 - pok) * (1.0 - e) / kxt + pok;
    } else {
      const double kxt2 = kxt * kxt;
      q3 = q1 * (1.0 - kxt + kxt2 * 0.5) + pxt * (1.0 - kxt * 0.5 + kxt2 / 6.0);
      q4 = q1 * (1.0 - kxt * 0.5 + kxt2 / 6.0) + pxt * (0.5 - kxt / 6.0 + kxt2 / 24.0);
    }
    qdel = (q1 + pxt) - q3;
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      if (uptk[n] > 0.0) {
        qdelb += a1b[n] * (uptk[n] / tmpa);
        uptkb[n] += a1b[n] * qdel / tmpa;
        tmpab -= a1b[n] * qdel * uptk[n] / (tmpa * tmpa);
      }
    q1b += qdelb;
    pxtb += qdelb;
    q3b -= qdelb;
    if (kxt > 0.001) {
      const double pok = pxt / kxt;
      const double e = ::exp(-kxt);
      // q3 = (q1 - pok) e + pok ; q4 = (q1 - pok)(1 - e)/kxt + pok
      double pokb = q3b * (1.0 - e) + q4b * (1.0 - (1.0 - e) / kxt);
      q1b += q3b * e + q4b * (1.0 - e) / kxt;
      double eb = q3b * (q1 - pok) - q4b * (q1 - pok) / kxt;
      kxtb -= q4b * (q1 - pok) * (1.0 - e) / (kxt * kxt);
      kxtb -= eb * e;
      pxtb += pokb / kxt;
      kxtb -= pokb * pok / kxt;
    } else {
      const double kxt2 = kxt * kxt;
      q1b += q3b * (1.0 - kxt + kxt2 * 0.5) + q4b * (1.0 - kxt * 0.5 + kxt2 / 6.0);
      pxtb += q3b * (1.0 - kxt * 0.5 + kxt2 / 6.0) + q4b * (0.5 - kxt / 6.0 + kxt2 / 24.0);
      kxtb += q3b * (q1 * (-1.0 + kxt) + pxt * (-0.5 + kxt / 3.0)) +
              q4b * (q1 * (-0.5 + kxt / 3.0) + pxt * (-1.0 / 6.0 + kxt / 12.0));
    }
  } else {
    q1b += g1b + qavgb;
    pxtb += g1b + qavgb * 0.5;
  }
  netprodb += pxtb * dt;
  tmpab += kxtb * dt;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    uptkb[n] += tmpab;
}

// ======================================================== SOA sub-stepping
// One pass of soa_step. State (g, a[4], tcur) before the pass in st; the
// cotangents of the state after the pass in gb, ab, tcb on entry, of the
// state before on return; the loop parameters' cotangents (opoa, uptk, g0)
// are accumulated.
struct SoaBar {
  double g, a[NMODE], tcur;
  double opoa[NMODE], uptk[NMODE], g0;
};

// x / d (FP64 arithmetic of the step), or x * mx::rcp(d) with FAST (the
// mixed-precision loop's arithmetic, f32::soa_step_mx); on the host always
// x / d.
template <bool FAST>
MAM4B_HD double qdiv(double x, double d) {
#ifdef __CUDA_ARCH__
  if constexpr (FAST)
    return x * f32::mx::rcp(d);
#endif
  return x / d;
}
// x * y + z, rounded once with FAST, twice (as the FP64 step) without
template <bool FAST>
MAM4B_HD double fmadd(double x, double y, double z) {
  if constexpr (FAST)
    return fma(x, y, z);
  return z + x * y;
}

// The forward values of the pass are recomputed with the arithmetic of the
// loop being reversed, so that every branch (skip, last sub-step, del > 0,
// the clips) is the forward's: FAST = false the FP64 loop's (soa_step),
// FAST = true f32::soa_step_mx's, the mixed-precision step's loop (every
// quotient x / d as x * mx::rcp(d), the sums fused; the mixed-precision
// adjoint). The cotangent sweep takes each reciprocal once, as
// mx::rcp(d), in both: cotangents need not round as the forward does.
template <bool FAST>
MAM4B_HD void soa_step_rev_t(const SoaState &st, SoaBar &b) {
  const double g_prev = st.g;
  const double g = dmax(g_prev, 0.0);
  double tot = g;
  double a[NMODE], aoa[NMODE], sat[NMODE], gs[NMODE], M1[NMODE], phi[NMODE];
  bool skip[NMODE];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    skip[n] = !(st.uptk[n] > 1.0e-15);
    a[n] = 0.0;
    if (skip[n])
      continue;
    a[n] = dmax(st.a[n], 0.0);
    tot += a[n];
  }
  double tmpb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    aoa[n] = st.opoa[n] + a[n];
    sat[n] = qdiv<FAST>(st.g0, dmax(aoa[n], 1.0e-20));
    gs[n] = sat[n] * a[n];
    M1[n] = dmax(g, dmax(gs[n], 1.0e-20));
    phi[n] = qdiv<FAST>(g - gs[n], M1[n]);
    tmpb = fmadd<FAST>(st.uptk[n], fabs(phi[n]), tmpb);
  }
  const double tmpa = dmax(0.0, tmpb);
  const double dtmax = st.dtfull - st.tcur;
  const bool last = dtmax * tmpa <= 0.05;
  const double dtcur = last ? dtmax : qdiv<FAST>(0.05, tmpa);
  double beta[NMODE], del[NMODE], sat2[NMODE], den[NMODE];
  double ta = 0.0, tbs = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    beta[n] = dtcur * st.uptk[n];
    del[n] = g - gs[n];
    sat2[n] = sat[n];
    if (del[n] > 0.0) {
      const double a_tmp = fmadd<FAST>(beta[n], del[n], a[n]);
      sat2[n] = qdiv<FAST>(st.g0, dmax(st.opoa[n] + a_tmp, 1.0e-20));
    }
    den[n] = fmadd<FAST>(beta[n], sat2[n], 1.0);
    if constexpr (FAST) {
      const double rd = qdiv<FAST>(1.0, den[n]);
      ta = fmadd<FAST>(a[n], rd, ta);
      tbs = fmadd<FAST>(beta[n], rd, tbs);
    } else {
      ta += a[n] / den[n];
      tbs += beta[n] / den[n];
    }
  }
  const double q = qdiv<FAST>(tot - ta, 1.0 + tbs);
  const double gn = dmax(0.0, q);
  // ---- reverse (reciprocals taken once: the cotangents need not round as
  // the forward does)
  double rden[NMODE];
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    rden[n] = skip[n] ? 0.0 : qdiv<true>(1.0, den[n]);
  const double r1 = qdiv<true>(1.0, 1.0 + tbs);
  double gnb = b.g, ab_[NMODE], betab[NMODE], denb[NMODE], sat2b[NMODE], satb[NMODE], gsb[NMODE];
  double gb = 0.0, totb = 0.0, tab = 0.0, tbb = 0.0, dtcurb = 0.0, tcurb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    ab_[n] = 0.0;
    betab[n] = 0.0;
    denb[n] = 0.0;
    sat2b[n] = 0.0;
    satb[n] = 0.0;
    gsb[n] = 0.0;
  }
  // time: tcur' = last ? dtfull : tcur + dtcur
  if (!last) {
    tcurb += b.tcur;
    dtcurb += b.tcur;
  }
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;  // a'[n] = 0
    const double an = fmadd<FAST>(beta[n], gn, a[n]) * rden[n];
    const double numb = b.a[n] * rden[n];
    denb[n] -= numb * an;
    ab_[n] += numb;
    betab[n] += numb * gn;
    gnb += numb * beta[n];
  }
  const double qb = maxc_rev(0.0, q, gnb);
  const double qr = qb * r1;
  totb += qr;
  tab -= qr;
  tbb -= qr * q;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    ab_[n] += tab * rden[n];
    betab[n] += tbb * rden[n];
    denb[n] -= (tab * a[n] + tbb * beta[n]) * (rden[n] * rden[n]);
    betab[n] += denb[n] * sat2[n];
    sat2b[n] += denb[n] * beta[n];
    if (del[n] > 0.0) {
      const double a_tmp = fmadd<FAST>(beta[n], del[n], a[n]);
      const double aoa2 = st.opoa[n] + a_tmp;
      const double rM2 = qdiv<true>(1.0, dmax(aoa2, 1.0e-20));
      b.g0 += sat2b[n] * rM2;
      const double M2b = -sat2b[n] * sat2[n] * rM2;
      const double aoa2b = maxxc_rev(aoa2, 1.0e-20, M2b);
      b.opoa[n] += aoa2b;
      ab_[n] += aoa2b;
      betab[n] += aoa2b * del[n];
      const double delb = aoa2b * beta[n];
      gb += delb;
      gsb[n] -= delb;
    } else {
      satb[n] += sat2b[n];
    }
    dtcurb += betab[n] * st.uptk[n];
    b.uptk[n] += betab[n] * dtcur;
  }
  // dtcur
  double tmpab = 0.0;
  if (last)
    tcurb -= dtcurb;  // dtcur = dtfull - tcur
  else
    tmpab -= qdiv<true>(dtcurb * dtcur, tmpa);
  const double tmpbb = maxc_rev(0.0, tmpb, tmpab);
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n])
      continue;
    b.uptk[n] += tmpbb * fabs(phi[n]);
    const double phib = tmpbb * st.uptk[n] * (phi[n] < 0.0 ? -1.0 : 1.0);
    const double rM1 = qdiv<true>(1.0, M1[n]);
    gb += phib * rM1;
    gsb[n] -= phib * rM1;
    const double M1b = -phib * phi[n] * rM1;
    // M1 = dmax(g, m2), m2 = dmax(gs, 1e-20)
    const double m2 = dmax(gs[n], 1.0e-20);
    if (g < m2) {
      gsb[n] += maxxc_rev(gs[n], 1.0e-20, M1b);
    } else {
      gb += M1b;
    }
    // gs = sat a
    satb[n] += gsb[n] * a[n];
    ab_[n] += gsb[n] * sat[n];
    // sat = g0 / dmax(aoa, 1e-20)
    const double rM = qdiv<true>(1.0, dmax(aoa[n], 1.0e-20));
    b.g0 += satb[n] * rM;
    const double Mb = -satb[n] * sat[n] * rM;
    const double aoab = maxxc_rev(aoa[n], 1.0e-20, Mb);
    b.opoa[n] += aoab;
    ab_[n] += aoab;
  }
  // tot = g + sum a
  gb += totb;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    if (skip[n]) {
      b.a[n] = 0.0;
      continue;
    }
    ab_[n] += totb;
    b.a[n] = maxxc_rev(st.a[n], 0.0, ab_[n]);
  }
  b.g = maxxc_rev(g_prev, 0.0, gb);
  b.tcur = tcurb;
}

MAM4B_HD void soa_step_rev(const SoaState &st, SoaBar &b) { soa_step_rev_t<false>(st, b); }

// soa_init (gasaerexch_soaexch.hpp:155-170): g0 from T (p fixed); opoa
// from POM; initial g, a from the subarea
MAM4B_HD double soa_g0_dT(double temp, double pmid) {
  const double c = 156.0e3 / 8.3144;
  const double p0_soa = 1.0e-10 * ::exp(-c * ((1.0 / temp) - (1.0 / 298.0)));
  const double g0 = 1.01325e5 * p0_soa / pmid;
  return g0 * c / (temp * temp);
}


// ================================================================ renaming
// rename_subarea<CLOUDY> (rename.hpp:23-390): si (and sc when CLOUDY) in
// place; grow_i, grow_c the growth increments. sib/scb: cotangents of the
// subareas after on entry, before on return; growb_i/growb_c accumulated.
template <bool CLOUDY>
MAM4B_HD void rename_subarea_rev(const StepConsts &C, const Sub &si, const Sub &sc,
                                 const double (&grow_i)[NAER], const double (&grow_c)[NAER],
                                 Sub &sib, Sub &scb, double (&growb_i)[NAER],
                                 double (&growb_c)[NAER]) {
  const int src = 1, dst = 0;
  double t_i = 0.0, td_i = 0.0, t_c = 0.0, td_c = 0.0;
#pragma unroll
  for (int a = 0; a < NAER; ++a) {
    t_i += si.aer[a][src] * K::mass_2_vol(a);
    td_i += grow_i[a] * K::mass_2_vol(a);
  }
  const double dv_i = t_i - td_i, ddv_i = td_i;
  double dv_c = 0.0, ddv_c = 0.0;
  if (CLOUDY) {
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      t_c += sc.aer[a][src] * K::mass_2_vol(a);
      td_c += grow_c[a] * K::mass_2_vol(a);
    }
    dv_c = t_c - td_c;
    ddv_c = td_c;
  }
  const double b4_dv0 = CLOUDY ? dv_i + dv_c : dv_i;
  const double b4_dv_b = dmax(b4_dv0, 1.0e-25);
  const double b4_n0 = CLOUDY ? si.num[src] + sc.num[src] : si.num[src];
  const double b4_n1 = dmax(0.0, b4_n0);
  const double lo = b4_dv_b * C.rn_v2n_hi_rlx, hi = b4_dv_b * C.rn_v2n_lo_rlx;
  const double b4_n_b = bound(lo, hi, b4_n1);
  const double del = CLOUDY ? ddv_i + ddv_c : ddv_i;
  const double aft_dv = b4_dv0 + del;
  if (aft_dv <= 1.0e-25)
    return;  // nothing moves: identity
  const double b4_d0 = diam_from_vol(b4_dv_b / b4_n_b, C.log_sig[src]);
  const bool capped = b4_d0 > C.rn_threshold;
  const double b4_dv = capped ? b4_dv0 * cube(C.rn_threshold / b4_d0) : b4_dv0;
  const double b4_d = capped ? C.rn_threshold : b4_d0;
  if ((aft_dv - b4_dv) <= 1.0e-6 * b4_dv_b)
    return;
  const double aft_d = diam_from_vol(aft_dv / b4_n_b, C.log_sig[src]);
  if (aft_d <= K::dnom(src))
    return;
  const double lb4 = ::log(b4_d), laft = ::log(aft_d);
  const double zb4n = (C.rn_ln_cutoff - lb4) * C.rn_fac;
  const double zb4v = (C.rn_ln_cutoff - (lb4 + C.rn_ln_tail_fac)) * C.rn_fac;
  const double zafn = (C.rn_ln_cutoff - laft) * C.rn_fac;
  const double zafv = (C.rn_ln_cutoff - (laft + C.rn_ln_tail_fac)) * C.rn_fac;
  const double b4_tn = 0.5 * erfc(zb4n), b4_tv = 0.5 * erfc(zb4v);
  const double aft_tn = 0.5 * erfc(zafn), aft_tv = 0.5 * erfc(zafv);
  const double vfrac = aft_tv * aft_dv - b4_tv * b4_dv;
  if (vfrac <= 0.0)
    return;
  const double xv0 = dmin(vfrac, aft_dv) / aft_dv;
  const double xv = dmin(xv0, 1.0 - 10.0 * K::eps);
  const double xn0 = aft_tn - b4_tn;
  const double xn1 = dmin(xn0, xv);
  const double xn = dmax(0.0, xn1);
  // ---- reverse of the transfers
  double xvb = 0.0, xnb = 0.0;
  {
    // num[src]' = num[src](1 - xn); num[dst]' = num[dst] + num[src] xn
    const double ns = si.num[src];
    xnb += ns * (sib.num[dst] - sib.num[src]);
    sib.num[src] = sib.num[src] * (1.0 - xn) + sib.num[dst] * xn;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      const double v = si.aer[a][src];
      xvb += v * (sib.aer[a][dst] - sib.aer[a][src]);
      sib.aer[a][src] = sib.aer[a][src] * (1.0 - xv) + sib.aer[a][dst] * xv;
    }
  }
  if (CLOUDY) {
    const double ns = sc.num[src];
    xnb += ns * (scb.num[dst] - scb.num[src]);
    scb.num[src] = scb.num[src] * (1.0 - xn) + scb.num[dst] * xn;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      const double v = sc.aer[a][src];
      xvb += v * (scb.aer[a][dst] - scb.aer[a][src]);
      scb.aer[a][src] = scb.aer[a][src] * (1.0 - xv) + scb.aer[a][dst] * xv;
    }
  }
  // xn = dmax(0, dmin(xn0, xv))
  const double xn1b = maxc_rev(0.0, xn1, xnb);
  double xn0b = 0.0;
  min_rev(xn0, xv, xn1b, xn0b, xvb);
  double aft_tnb = xn0b, b4_tnb = -xn0b;
  // xv = dmin(xv0, 1 - 10 eps); xv0 = dmin(vfrac, aft_dv) / aft_dv
  const double xv0b = minc_rev(1.0 - 10.0 * K::eps, xv0, xvb);
  double aft_dvb = -xv0b * xv0 / aft_dv;
  double vfracb = 0.0;
  min_rev(vfrac, aft_dv, xv0b / aft_dv, vfracb, aft_dvb);
  // vfrac = aft_tv aft_dv - b4_tv b4_dv
  double aft_tvb = vfracb * aft_dv, b4_tvb = -vfracb * b4_dv;
  aft_dvb += vfracb * aft_tv;
  double b4_dvb = -vfracb * b4_tv;
  // tail fractions: t = 0.5 erfc(z); dt/dz = -exp(-z^2)/sqrt(pi)
  const double isp = 0.56418958354775628695;  // 1/sqrt(pi)
  const double zb4nb = -b4_tnb * isp * ::exp(-zb4n * zb4n);
  const double zb4vb = -b4_tvb * isp * ::exp(-zb4v * zb4v);
  const double zafnb = -aft_tnb * isp * ::exp(-zafn * zafn);
  const double zafvb = -aft_tvb * isp * ::exp(-zafv * zafv);
  const double lb4b = -(zb4nb + zb4vb) * C.rn_fac;
  const double laftb = -(zafnb + zafvb) * C.rn_fac;
  double b4_db = lb4b / b4_d;
  const double aft_db = laftb / aft_d;
  // aft_d = diam_from_vol(aft_dv / b4_n_b)
  const double va = aft_dv / b4_n_b;
  const double vab = diam_from_vol_rev(va, C.log_sig[src], aft_db);
  aft_dvb += vab / b4_n_b;
  double b4_n_bb = -vab * va / b4_n_b;
  double b4_dv0b = 0.0, b4_dv_bb = 0.0;
  if (capped) {
    // b4_dv = b4_dv0 (thr / b4_d0)^3, b4_d = thr
    b4_dv0b += b4_dvb * cube(C.rn_threshold / b4_d0);
    const double b4_d0b = -b4_dvb * 3.0 * b4_dv / b4_d0;
    const double v0 = b4_dv_b / b4_n_b;
    const double v0b = diam_from_vol_rev(v0, C.log_sig[src], b4_d0b);
    b4_dv_bb += v0b / b4_n_b;
    b4_n_bb -= v0b * v0 / b4_n_b;
  } else {
    b4_dv0b += b4_dvb;
    const double v0 = b4_dv_b / b4_n_b;
    const double v0b = diam_from_vol_rev(v0, C.log_sig[src], b4_db);
    b4_dv_bb += v0b / b4_n_b;
    b4_n_bb -= v0b * v0 / b4_n_b;
  }
  // aft_dv = b4_dv0 + del
  b4_dv0b += aft_dvb;
  const double delb = aft_dvb;
  // b4_n_b = bound(lo, hi, b4_n1), lo/hi ~ b4_dv_b
  {
    const double m = dmin(hi, b4_n1);
    double b4_n1b = 0.0;
    if (lo < m) {
      if (b4_n1 < hi)
        b4_n1b += b4_n_bb;
      else
        b4_dv_bb += b4_n_bb * C.rn_v2n_lo_rlx;
    } else {
      b4_dv_bb += b4_n_bb * C.rn_v2n_hi_rlx;
    }
    const double b4_n0b = maxc_rev(0.0, b4_n0, b4_n1b);
    sib.num[src] += b4_n0b;
    if (CLOUDY)
      scb.num[src] += b4_n0b;
  }
  b4_dv0b += maxxc_rev(b4_dv0, 1.0e-25, b4_dv_bb);
  // b4_dv0 = dv_i (+ dv_c), dv = t - td, ddv = td, del = ddv_i (+ ddv_c)
  const double dv_ib = b4_dv0b, ddv_ib = delb;
  const double t_ib = dv_ib, td_ib = -dv_ib + ddv_ib;
#pragma unroll
  for (int a = 0; a < NAER; ++a) {
    sib.aer[a][src] += t_ib * K::mass_2_vol(a);
    growb_i[a] += td_ib * K::mass_2_vol(a);
  }
  if (CLOUDY) {
    const double dv_cb = b4_dv0b, ddv_cb = delb;
    const double t_cb = dv_cb, td_cb = -dv_cb + ddv_cb;
#pragma unroll
    for (int a = 0; a < NAER; ++a) {
      scb.aer[a][src] += t_cb * K::mass_2_vol(a);
      growb_c[a] += td_cb * K::mass_2_vol(a);
    }
  }
}

// =============================================================== aging
// aging (aging.hpp:70-361) as it acts on the subarea state: s in place;
// sb the cotangent after on entry, before on return; dgn_a_pcb accumulated.
MAM4B_HD void aging_rev(const StepConsts &C, unsigned nmono, double dgn_a_pc, const Sub &s,
                        Sub &sb, double &dgn_a_pcb) {
  const int pc = 3, acc = 0;
  const double vol_shell = s.aer[1][pc] * C.so4_vol + s.aer[0][pc] * C.soa_fac_eqvhyg;
  double vol_core = 0.0;
  vol_core += s.aer[2][pc] * K::mass_2_vol(2);
  vol_core += s.aer[3][pc] * K::mass_2_vol(3);
  vol_core += s.aer[6][pc] * K::mass_2_vol(6);
  const double xmax = 1.0 - 10.0 * K::eps;
  const double tmp1 = vol_shell * dgn_a_pc * C.aging_fac_volsfc;
  const double dr = nmono * 4.76e-10;
  const double tmp2a = 6.0 * dr * vol_core;
  const double tmp2 = dmax(tmp2a, 0.0);
  const bool full = tmp1 >= tmp2;
  const double r = full ? 0.0 : tmp1 / tmp2;
  const double xfer = full ? xmax : dmin(r, xmax);
  double xferb = 0.0;
  // number
  {
    xferb += s.num[pc] * (sb.num[acc] - sb.num[pc]);
    sb.num[pc] = sb.num[pc] * (1.0 - xfer) + sb.num[acc] * xfer;
  }
  // SO4, SOA, NaCl, DST moved whole: aer[acc]' = aer[acc] + aer[pc]; aer[pc]' = 0
  constexpr int all_to_acc[4] = {0, 1, 4, 5};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int a = all_to_acc[k];
    sb.aer[a][pc] = sb.aer[a][acc];
  }
  constexpr int to_acc[3] = {2, 3, 6};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = to_acc[k];
    xferb += s.aer[a][pc] * (sb.aer[a][acc] - sb.aer[a][pc]);
    sb.aer[a][pc] = sb.aer[a][pc] * (1.0 - xfer) + sb.aer[a][acc] * xfer;
  }
  if (!full) {
    const double rb = minc_rev(xmax, r, xferb);
    const double tmp1b = rb / tmp2;
    const double tmp2b = -rb * r / tmp2;
    const double tmp2ab = maxxc_rev(tmp2a, 0.0, tmp2b);
    const double vcb = tmp2ab * 6.0 * dr;
    sb.aer[2][pc] += vcb * K::mass_2_vol(2);
    sb.aer[3][pc] += vcb * K::mass_2_vol(3);
    sb.aer[6][pc] += vcb * K::mass_2_vol(6);
    const double vsb = tmp1b * dgn_a_pc * C.aging_fac_volsfc;
    dgn_a_pcb += tmp1b * vol_shell * C.aging_fac_volsfc;
    sb.aer[1][pc] += vsb * C.so4_vol;
    sb.aer[0][pc] += vsb * C.soa_fac_eqvhyg;
  }
}

// =============================================================== nucleation
template <class R>
MAM4B_HD R veh02_x_crit_t(const R &lna, const R &t, const R &lrh) {
  return 0.740997 - 0.00266379 * t - 0.00349998 * lna + 0.0000504022 * t * lna +
         0.00201048 * lrh - 0.000183289 * t * lrh + 0.00157407 * (lrh * lrh) -
         0.0000179059 * t * (lrh * lrh) + 0.000184403 * (lrh * lrh * lrh) -
         1.50345e-6 * t * (lrh * lrh * lrh);
}
template <class R>
MAM4B_HD R veh02_log_rate_t(const R &lna, const R &t, const R &lrh, const R &x) {
  const R t2 = t * t, t3 = t * t * t, l2 = lrh * lrh, l3 = lrh * lrh * lrh, n2 = lna * lna,
          n3 = lna * lna * lna;
  const R a = 0.14309 + 2.21956 * t - 0.0273911 * t2 + 0.0000722811 * t3 + 5.91822 / x;
  const R b = 0.117489 + 0.462532 * t - 0.0118059 * t2 + 0.0000404196 * t3 + 15.7963 / x;
  const R c = -0.215554 - 0.0810269 * t + 0.00143581 * t2 - 4.7758e-6 * t3 - 2.91297 / x;
  const R d = -3.58856 + 0.049508 * t - 0.00021382 * t2 + 3.10801e-7 * t3 - 0.0293333 / x;
  const R e = 1.14598 - 0.600796 * t + 0.00864245 * t2 - 0.0000228947 * t3 - 8.44985 / x;
  const R f = 2.15855 + 0.0808121 * t - 0.000407382 * t2 - 4.01957e-7 * t3 + 0.721326 / x;
  const R g = 1.6241 - 0.0160106 * t + 0.0000377124 * t2 + 3.21794e-8 * t3 - 0.0113255 / x;
  const R h = 9.71682 - 0.115048 * t + 0.000157098 * t2 + 4.00914e-7 * t3 + 0.71186 / x;
  const R i = -1.05611 + 0.00903378 * t - 0.0000198417 * t2 + 2.46048e-8 * t3 - 0.0579087 / x;
  const R j = -0.148712 + 0.00283508 * t - 9.24619e-6 * t2 + 5.00427e-9 * t3 - 0.0127081 / x;
  return a + b * lrh + c * l2 + d * l3 + e * lna + f * lrh * lna + g * l2 * lna + h * n2 +
         i * lrh * n2 + j * n3;
}
template <class R>
MAM4B_HD R veh02_ntot_t(const R &lna, const R &t, const R &lrh, const R &x) {
  const R t2 = t * t, t3 = t * t * t, l2 = lrh * lrh, l3 = lrh * lrh * lrh, n2 = lna * lna,
          n3 = lna * lna * lna;
  const R A = -0.00295413 - 0.0976834 * t + 0.00102485 * t2 - 2.18646e-6 * t3 - 0.101717 / x;
  const R B = -0.00205064 - 0.00758504 * t + 0.000192654 * t2 - 6.7043e-7 * t3 - 0.255774 / x;
  const R Cc = +0.00322308 + 0.000852637 * t - 0.0000154757 * t2 + 5.66661e-8 * t3 + 0.0338444 / x;
  const R D = +0.0474323 - 0.000625104 * t + 2.65066e-6 * t2 - 3.67471e-9 * t3 - 0.000267251 / x;
  const R E = -0.0125211 + 0.00580655 * t - 0.000101674 * t2 + 2.88195e-7 * t3 + 0.0942243 / x;
  const R F = -0.038546 - 0.000672316 * t + 2.60288e-6 * t2 + 1.19416e-8 * t3 - 0.00851515 / x;
  const R G = -0.0183749 + 0.000172072 * t - 3.71766e-7 * t2 - 5.14875e-10 * t3 + 0.00026866 / x;
  const R H = -0.0619974 + 0.000906958 * t - 9.11728e-7 * t2 - 5.36796e-9 * t3 - 0.00774234 / x;
  const R I = +0.0121827 - 0.00010665 * t + 2.5346e-7 * t2 - 3.63519e-10 * t3 + 0.000610065 / x;
  const R J = +0.000320184 - 0.0000174762 * t + 6.06504e-8 * t2 - 1.4177e-11 * t3 + 0.000135751 / x;
  return exp(A + B * lrh + Cc * l2 + D * l3 + E * lna + F * lrh * lna + G * l2 * lna + H * n2 +
             I * lrh * n2 + J * n3);
}

// nucleation (mam_newnuc_1subarea + mer07_veh02_nuc_mosaic_1box) as a
// template over the number type; the state entries it changes are
// num1 = s.num[1], aer11 = s.aer[1][1], gas1 = s.gas[1].
template <class R>
MAM4B_HD void nucleation_t(const StepConsts &C, double deltat, const R &temp, double pmid,
                           double zmid, double pblh, const R &relhum, const R &uptkrate_h2so4,
                           const R &qgas_avg1, R &gas1, R &num1, R &aer11) {
  const R qh2so4_cur = gas1;
  const R qh2so4_avg = qgas_avg1;
  if (qh2so4_avg <= 4.0e-16)
    return;
  const R rh_in = dmax(0.01, dmin(0.99, relhum));
  const double rgas = 8.31446759100000, avogad = 6.022140000000000E+023;
  const double mw_so4a = 96.0, mw_so4a_host = 115.0, dens = 1770.0;
  const R cair = pmid / (temp * rgas);
  const R so4vol = qh2so4_avg * cair * avogad * 1.0e-6;
  R rateloge = 0.0 * temp + ::log(1.0e-38);
  R cnum_h2so4 = 0.0 * temp, radius_cluster = 0.0 * temp;
  if (so4vol >= 1.0e4) {
    const R t = dmax(230.15, dmin(305.15, temp));
    const R rh = dmax(1.0e-4, dmin(1.0, rh_in));
    const R na = dmax(1.0e4, dmin(1.0e11, so4vol));
    const R lna = log(na), lrh = log(rh);
    const R x_crit = veh02_x_crit_t(lna, t, lrh);
    rateloge = veh02_log_rate_t(lna, t, lrh, x_crit);
    const R cnum_tot = veh02_ntot_t(lna, t, lrh, x_crit);
    cnum_h2so4 = cnum_tot * x_crit;
    radius_cluster = exp(-1.6524245 + 0.42316402 * x_crit + 0.3346648 * log(cnum_tot));
  }
  rateloge = rateloge + 0.0;
  if (zmid <= mam4b::dmax(pblh, 100.0)) {
    const R tmp_rate = 1e-6 * so4vol;
    const R tmp_loge = log(dmax(1.0e-38, tmp_rate));
    if (!(tmp_loge <= rateloge)) {
      rateloge = tmp_loge;
      radius_cluster = 0.5 + 0.0 * temp;
      const double tmp_diam = 0.5 * 2.0e-7;
      const double tmp_volu = (tmp_diam * tmp_diam * tmp_diam) * (K::pi / 6.0);
      const double tmp_mass = tmp_volu * 1.8;
      cnum_h2so4 = 0.0 * temp + (tmp_mass / 98.0) * 6.023e23;
    }
  }
  if (rateloge <= -13.82)
    return;
  const R ratenuclt_bb = exp(rateloge) * 1.0e6;
  const R wetvol_dryvol = 1.0 - 0.56 / log(dmax(0.10, dmin(0.95, rh_in)));
  R voldry_clus = (dmax(cnum_h2so4, 1.0) * mw_so4a + 0.0 * 18.0) / (1.0e3 * dens * avogad);
  voldry_clus = voldry_clus * (mw_so4a_host / mw_so4a);
  const R dpdry_clus = pow(voldry_clus * 6.0 / K::pi, 1.0 / 3.0);
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
  const double voldry_part = (K::pi / 6.0) * ::pow(dpdry_part, 3.0);
  // composition: sulfuric acid, except the ammonium branch at zero H2SO4
  double n1 = 0.0, n2 = 0.0, n3 = 0.0;
  if (!igrow) {
    n3 = 1.0;
  } else if (0.0 >= val(qh2so4_cur)) {
    n1 = (0.0 / val(qh2so4_cur)) - 1.0;
    n1 = mam4b::dmax(0.0, mam4b::dmin(1.0, n1));
    n2 = 1.0 - n1;
  } else {
    n2 = (0.0 / val(qh2so4_cur));
    n2 = mam4b::dmax(0.0, mam4b::dmin(1.0, n2));
    n3 = 1.0 - n2;
  }
  const double m1 = n1 * 132.0, m2 = n2 * 114.0, m3 = n3 * 96.0;
  const double dens_part = (m1 + m2 + m3) / ((m1 / dens) + (m2 / dens) + (m3 / dens));
  const double mass_part = voldry_part * dens_part;
  const double mole_nh4 = 2.0 * n1 + n2;
  double kgaero = 1.0e-3 * (m1 + m2 + m3);
  kgaero = kgaero * (mw_so4a_host / mw_so4a);
  const R wet_volfrac_so4a = 1.0 / (wetvol_dryvol * (1.0 + mole_nh4 * 17.0 / 98.0));
  R factor_kk = 1.0 + 0.0 * temp;
  if (igrow) {
    const R tmp_spd = 14.7 * sqrt(temp);
    const R gr_kk = 3.0e-9 * tmp_spd * 96.0 * so4vol / (dens_part * wet_volfrac_so4a);
    const R dfin_kk = 1.0e9 * dpdry_part * pow(wetvol_dryvol, 1.0 / 3.0);
    const R dnuc_kk = dmax(2.0 * radius_cluster, 1.0);
    const R gamma_kk = 0.23 * pow(dnuc_kk, 0.2) * pow(dfin_kk / 3.0, 0.075) *
                       ::pow(dens_part * 1.0e-3, -0.33) * pow(temp / 293.0, -0.75);
    const R tmpa = dmax(uptkrate_h2so4 * 3600.0, 0.0);
    const R tmpb = (6.7037e-6 * pow(temp, 0.75) / cair) * 3600.0;
    const R cs_prime_kk = tmpa / (4.0 * K::pi * tmpb * 0.65);
    const R nu_kk = gamma_kk * cs_prime_kk / gr_kk;
    factor_kk = exp((nu_kk / dfin_kk) - (nu_kk / dnuc_kk));
  }
  const R ratenuclt_kk = ratenuclt_bb * factor_kk;
  const R qmolso4a_del_max = dmax(0.0, (ratenuclt_kk * deltat * mass_part)) / (kgaero * cair);
  R freducea = 1.0 + 0.0 * temp;
  double freduceb = 1.0;
  if (qmolso4a_del_max > qh2so4_cur)
    freducea = qh2so4_cur / qmolso4a_del_max;
  if (mole_nh4 >= 1.0e-10) {
    if (val(qmolso4a_del_max) * mole_nh4 > 0.0)
      freduceb = 0.0 / (val(qmolso4a_del_max) * mole_nh4);
  }
  const R freduce = dmin(freducea, freduceb);
  if ((freduce * ratenuclt_kk) <= 1.0e-12)
    return;
  const R qh2so4_del = dmin(0.9999 * qh2so4_cur, freduce * qmolso4a_del_max);
  const R qnh3_del = 0.0 * qh2so4_del;  // dmin(0.9999 * 0, ...) with mole_nh4 = 0 rows
  const R qso4a_del = qh2so4_del;
  const R qnuma_del = 1.0e-3 * (qso4a_del * mw_so4a + qnh3_del * 18.0) / mass_part;
  R dndt = (qnuma_del * 1.0e3) / deltat;
  R dmdt = dmax(0.0, ((qso4a_del * mw_so4a_host) / deltat));
  if (dndt < 1.0e2) {
    dndt = 0.0 * dndt;
    dmdt = 0.0 * dmdt;
  } else {
    const R mass1p = dmdt / dndt;
    if (mass1p < C.nuc_mass1p_lo)
      dndt = dmdt / C.nuc_mass1p_lo;
    else if (mass1p > C.nuc_mass1p_hi)
      dmdt = dndt * C.nuc_mass1p_hi;
  }
  num1 = num1 + dndt * deltat;
  const R dso4dt = dmdt * 1.0 / mw_so4a_host;
  if (dso4dt > 0.0) {
    R tq = dso4dt * deltat;
    aer11 = aer11 + tq;
    tq = dmin(tq, gas1);
    gas1 = gas1 - tq;
  }
}

// nucleation_rev: cotangents of (gas1, num1, aer11) after on entry, before
// on return; temp, relhum, uptkrate, qavg accumulated.
MAM4B_HD void nucleation_rev(const StepConsts &C, double deltat, double temp, double pmid,
                             double zmid, double pblh, double relhum, double uptkrate,
                             double qavg, double gas1, double num1, double aer11, double &gas1b,
                             double &num1b, double &aer11b, double &tb, double &rhb,
                             double &ukb, double &qab) {
  typedef Dual<7> D7;
  D7 g = dvar<7>(gas1, 4), n = dvar<7>(num1, 5), a = dvar<7>(aer11, 6);
  nucleation_t<D7>(C, deltat, dvar<7>(temp, 0), pmid, zmid, pblh, dvar<7>(relhum, 1),
                   dvar<7>(uptkrate, 2), dvar<7>(qavg, 3), g, n, a);
  double in_b[7];
#pragma unroll
  for (int i = 0; i < 7; ++i)
    in_b[i] = gas1b * g.d[i] + num1b * n.d[i] + aer11b * a.d[i];
  tb += in_b[0];
  rhb += in_b[1];
  ukb += in_b[2];
  qab += in_b[3];
  gas1b = in_b[4];
  num1b = in_b[5];
  aer11b = in_b[6];
}


// ======================================================= one grid cell
struct AdjCfg {
  int do_cond, do_rename, do_newnuc, do_coag, optaa;
  unsigned nmono;
};

// interstitial partition factors (get_partition_factors,
// mam4_amicphys.hpp:414-449) and their reverse
MAM4B_HD void part_factors(double fcldy, double q_i, double q_c, double &fc, double &fy) {
  const double fclea = 1.0 - fcldy;
  const double cldbrn_cldy = q_c / fcldy;
  const double intrst_cldy = dmax(0.0, ((q_i + q_c) - cldbrn_cldy));
  const double intrst_clea = (q_i - fcldy * intrst_cldy) / fclea;
  double r = dmax(1.e-35, intrst_clea * fclea) / dmax(1.e-35, q_i);
  r = dmax(0.0, dmin(1.0, r));
  fc = r / fclea;
  fy = (1 - r) / fcldy;
}
MAM4B_HD void part_factors_rev(double fcldy, double q_i, double q_c, double fcb, double fyb,
                               double &q_ib, double &q_cb) {
  const double fclea = 1.0 - fcldy;
  const double cldbrn_cldy = q_c / fcldy;
  const double ic0 = (q_i + q_c) - cldbrn_cldy;
  const double intrst_cldy = dmax(0.0, ic0);
  const double intrst_clea = (q_i - fcldy * intrst_cldy) / fclea;
  const double nu = dmax(1.e-35, intrst_clea * fclea), de = dmax(1.e-35, q_i);
  const double r0 = nu / de;
  const double rb = fcb / fclea - fyb / fcldy;
  // r = dmax(0, dmin(1, r0))
  const double m = dmin(1.0, r0);
  const double r0b = (0.0 < m && r0 < 1.0) ? rb : 0.0;
  const double nub = r0b / de, deb = -r0b * r0 / de;
  q_ib += maxc_rev(1.e-35, q_i, deb);
  const double icb = maxc_rev(1.e-35, intrst_clea * fclea, nub) * fclea;
  q_ib += icb / fclea;
  const double iyb = -icb * fcldy / fclea;
  const double i0b = maxc_rev(0.0, ic0, iyb);
  q_ib += i0b;
  q_cb += i0b * (1.0 - 1.0 / fcldy);
}

// SOA loop with checkpoints of (g, a[4], tcur) every kSoaCheck passes
constexpr int kSoaCheck = 4;
constexpr int kSoaCkMax = 1001 / kSoaCheck + 2;
// checkpoint e, component j (g, a[0..3], tcur) at ck[(6 e + j) * cks]
MAM4B_HD int soa_forward_ck(SoaState &st, double *ck, size_t cks) {
  int k = 0;
  while (true) {
    if (k % kSoaCheck == 0) {
      double *e = ck + (size_t)6 * (k / kSoaCheck) * cks;
      e[0] = st.g;
#pragma unroll
      for (int n = 0; n < NMODE; ++n)
        e[(1 + n) * cks] = st.a[n];
      e[5 * cks] = st.tcur;
    }
    if (!soa_step(st))
      break;
    ++k;
  }
  return k;  // passes taken (the reference's niter, minus the failed test)
}

// one block of the loop's reverse: passes [base, base + kSoaCheck) from the
// checkpoint at base (tmpl supplies the loop parameters opoa, uptk, g0,
// dtfull, which the passes do not change)
MAM4B_HD void soa_block_rev(const SoaState &tmpl, int base, int passes, const double *ck,
                            size_t cks, SoaBar &b) {
  SoaState blk[kSoaCheck];
  const double *e = ck + (size_t)6 * (base / kSoaCheck) * cks;
  SoaState st = tmpl;
  st.g = e[0];
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    st.a[n] = e[(1 + n) * cks];
  st.tcur = e[5 * cks];
  st.niter = base;
  const int cnt = (passes - base < kSoaCheck) ? passes - base : kSoaCheck;
  for (int i = 0; i < cnt; ++i) {
    blk[i] = st;
    soa_step(st);
  }
  for (int i = cnt - 1; i >= 0; --i)
    soa_step_rev(blk[i], b);
}

// reverse of the loop: b holds the cotangents of the final (g, a, tcur) on
// entry, of the initial state on return (parameters accumulated)
MAM4B_HD void soa_loop_rev(const SoaState &init, int passes, const double *ck, size_t cks,
                          SoaBar &b) {
  for (int base = ((passes - 1) / kSoaCheck) * kSoaCheck; base >= 0 && passes > 0;
       base -= kSoaCheck)
    soa_block_rev(init, base, passes, ck, cks, b);
}

MAM4B_HD void sub_zero(Sub &b) {
  b.gas[0] = b.gas[1] = 0.0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    b.num[m] = 0.0;
#pragma unroll
    for (int a = 0; a < NAER; ++a)
      b.aer[a][m] = 0.0;
  }
}

// load_sub / load_sub_plain reverses (number and mass factors per mode)
MAM4B_HD void load_sub_rev(const Sub &sb, const double (&q)[NPOP], const double (&fn)[NMODE],
                           const double (&fm)[NMODE], double (&qb)[NPOP], double (&fnb)[NMODE],
                           double (&fmb)[NMODE]) {
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    qb[K::numslot(m)] += sb.num[m] * fn[m];
    fnb[m] += sb.num[m] * q[K::numslot(m)];
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      const int sl = K::aer_slot(x, m);
      if (sl >= 0) {
        qb[sl] += sb.aer[x][m] * K::fcvt_aer(x) * fm[m];
        fmb[m] += sb.aer[x][m] * K::fcvt_aer(x) * q[sl];
      }
    }
  }
}
MAM4B_HD void load_sub_plain_rev(const Sub &sb, double (&qb)[NPOP]) {
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    qb[K::numslot(m)] += sb.num[m];
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      const int sl = K::aer_slot(x, m);
      if (sl >= 0)
        qb[sl] += sb.aer[x][m] * K::fcvt_aer(x);
    }
  }
}


// ---- front: calcsize, water uptake, subareas, clear-subarea prefix
// State of the forward sweep up to the SOA loop of the clear subarea (the
// whole cell for a cloudy one).
struct FrontTape {
  int cat;  // 0 clear, 1 cloudy, 2 partly cloudy
  double dgn_a[NMODE], dgn_awet[NMODE], wetdens_wu[NMODE], wetdens[NMODE], rh_wu;
  double qi[NPOP], qc[NPOP], g_h2so4, g_soag, relhumgcm;
  double fn_c[NMODE], fn_y[NMODE], fm_c[NMODE], fm_y[NMODE], gcl[2], gcy[2], rhc;
  bool gcy_clip[2];
  Sub cy_si, cy_sc;     // cloudy (sub)area before renaming
  Sub s_entry;          // clear subarea at entry
  Sub s_pre_soa;        // clear subarea at the SOA loop
  double qgas1[2], rh_sub, gd, fp, rate[NMODE];
  ClearMid cm;
  SoaState soa0;
  double ci[NPOP], cg[2], oc[NPOP];  // cloudy-subarea contributions, cloud-borne means
};

// Forward sweep to the SOA loop (cell_step<false> arithmetic). Writes the
// 16 size outputs into y, and for a cloudy cell all 68.
// Front values that the forward pipeline has computed already (water
// uptake of each mode, H2SO4 diffusivity, mean free path and per-particle
// uptake rates): with KNOWN, front_forward takes them from kn instead of
// recomputing them.
struct FrontKnown {
  double dgn_awet[NMODE], wetdens_wu[NMODE], qaerwat[NMODE], rh_wu, gd, fp, rate[NMODE];
};

template <bool KNOWN>
MAM4B_HD void front_forward(const StepConsts &C, const AdjCfg &cf, const double (&x)[MAM4B_NIN],
                            double dt, FrontTape &ft, double (&y)[MAM4B_NOUT],
                            const FrontKnown *kn = nullptr) {
  const double temp = x[MAM4B_IN_T], pmid = x[MAM4B_IN_P];
  const double qv = x[MAM4B_IN_QV], cld = x[MAM4B_IN_CLD];
  double ai[NPOP], ac[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ai[p] = x[MAM4B_IN_AER_I + p];
    ac[p] = x[MAM4B_IN_AER_C + p];
  }
  double pt_i[NPOP], pt_c[NPOP], qaerwat[NMODE];
  calcsize(C, ai, ac, dt, ft.dgn_a, pt_i, pt_c);
  if constexpr (KNOWN) {
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      ft.dgn_awet[m] = kn->dgn_awet[m];
      ft.wetdens_wu[m] = kn->wetdens_wu[m];
      qaerwat[m] = kn->qaerwat[m];
    }
    ft.rh_wu = kn->rh_wu;
  } else {
    water_uptake(C, ai, qv, temp, pmid, cld, ft.dgn_a, ft.dgn_awet, qaerwat, ft.wetdens_wu);
    ft.rh_wu = water_uptake_rh(qv, temp, pmid, cld);
  }
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    y[MAM4B_OUT_DGN_A + m] = ft.dgn_a[m];
    y[MAM4B_OUT_DGN_AWET + m] = ft.dgn_awet[m];
    y[MAM4B_OUT_WETDENS + m] = ft.wetdens_wu[m];
    y[MAM4B_OUT_QAERWAT + m] = qaerwat[m];
    ft.wetdens[m] = dmax(1000.0, ft.wetdens_wu[m]);
  }
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ft.qi[p] = dmax(0.0, dmax(0.0, ai[p] + pt_i[p] * dt) * C.to_vmr[2 + p]);
    ft.qc[p] = dmax(0.0, dmax(0.0, ac[p] + pt_c[p] * dt) * C.to_vmr[2 + p]);
  }
  ft.g_h2so4 = dmax(0.0, x[MAM4B_IN_H2SO4] * C.to_vmr[0]);
  ft.g_soag = dmax(0.0, x[MAM4B_IN_SOAG] * C.to_vmr[1]);
  {
    const double epsqs = 0.018016 / 0.028966;
    const double tc = temp - 273.15;
    const double ew = 610.94 * ::exp(17.625 * tc / (234.04 + tc));
    const double ev_sat = 1.00071 * ::exp(4.5e-8 * pmid) * ew;
    const double qv_sat = epsqs * ev_sat / (pmid - (1 - epsqs) * ev_sat);
    ft.relhumgcm = dmax(0.0, dmin(1.0, qv / qv_sat));
  }
  const double fsoag = C.fcvt_soag;
  if (cld > 0.999) {
    ft.cat = 1;
    Sub si, sc;
    load_sub_plain(si, ft.qi);
    load_sub_plain(sc, ft.qc);
    si.gas[0] = si.gas[1] = sc.gas[0] = sc.gas[1] = 0.0;
    ft.cy_si = si;
    ft.cy_sc = sc;
    if (cf.do_rename) {
      const double z7[NAER] = {0, 0, 0, 0, 0, 0, 0};
      rename_subarea<true>(C, si, sc, z7, z7);
    }
    const double o_soag = dmax(0.0, 0.0 + ft.g_soag * 1.0);
    const double o_h2so4 = dmax(0.0, 0.0 + ft.g_h2so4 * 1.0);
    double oi[NPOP];
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] = dmax(0.0, 0.0 + (si.num[m] / 1.0) * 1.0);
      ft.oc[K::numslot(m)] = 0.0 + (sc.num[m] / 1.0) * 1.0;
#pragma unroll
      for (int xx = 0; xx < NAER; ++xx) {
        const int sl = K::aer_slot(xx, m);
        if (sl >= 0) {
          oi[sl] = dmax(0.0, 0.0 + (si.aer[xx][m] / K::fcvt_aer(xx)) * 1.0);
          ft.oc[sl] = 0.0 + (sc.aer[xx][m] / K::fcvt_aer(xx)) * 1.0;
        }
      }
    }
    y[MAM4B_OUT_TEND + 0] = (o_h2so4 * C.to_mmr[0] - x[MAM4B_IN_H2SO4]) / dt;
    y[MAM4B_OUT_TEND + 1] = (o_soag * C.to_mmr[1] - x[MAM4B_IN_SOAG]) / dt;
#pragma unroll
    for (int p = 0; p < NPOP; ++p) {
      y[MAM4B_OUT_TEND + 2 + p] = (oi[p] * C.to_mmr[2 + p] - ai[p]) / dt;
      y[MAM4B_OUT_TEND + 27 + p] = (ft.oc[p] * C.to_mmr[2 + p] - ac[p]) / dt;
    }
    return;
  }
  const bool partly = !(cld < 1.0e-5);
  ft.cat = partly ? 2 : 0;
  const double fcldy = cld, fclea = 1.0 - fcldy;
  Sub s;
  if (!partly) {
    load_sub_plain(s, ft.qi);
    s.gas[0] = ft.g_soag * fsoag;
    s.gas[1] = ft.g_h2so4 * 1.0;
    ft.rh_sub = ft.relhumgcm;
#pragma unroll
    for (int p = 0; p < NPOP; ++p) {
      ft.oc[p] = ft.qc[p];
      ft.ci[p] = 0.0;
    }
    ft.cg[0] = ft.cg[1] = 0.0;
  } else {
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      part_factors(fcldy, ft.qi[K::numslot(m)], ft.qc[K::numslot(m)], ft.fn_c[m], ft.fn_y[m]);
      double si_ = 0.0, sc_ = 0.0;
#pragma unroll
      for (int k = 0; k < K::nspec(m); ++k) {
        si_ = si_ + ft.qi[K::spec0(m) + k];
        sc_ = sc_ + ft.qc[K::spec0(m) + k];
      }
      part_factors(fcldy, si_, sc_, ft.fm_c[m], ft.fm_y[m]);
    }
    ft.gcl[0] = ft.g_soag;
    ft.gcl[1] = ft.g_h2so4;
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      ft.gcy[g] = (ft.gcl[g] - fclea * ft.gcl[g]) / fcldy;
      ft.gcy_clip[g] = ft.gcy[g] < 0;
      if (ft.gcy_clip[g]) {
        ft.gcy[g] = 0;
        ft.gcl[g] = ft.gcl[g] / fclea;
      }
    }
    ft.rhc = bound(0.0, 1.0, (ft.relhumgcm - fcldy) / fclea);
    Sub si, sc;
    load_sub(si, ft.qi, ft.fn_y, ft.fm_y);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      sc.num[m] = (ft.qc[K::numslot(m)] / fcldy) * 1;
#pragma unroll
      for (int xx = 0; xx < NAER; ++xx) {
        const int sl = K::aer_slot(xx, m);
        sc.aer[xx][m] = (sl >= 0) ? (ft.qc[sl] / fcldy) * K::fcvt_aer(xx) : 0.0;
      }
    }
    si.gas[0] = si.gas[1] = sc.gas[0] = sc.gas[1] = 0.0;
    ft.cy_si = si;
    ft.cy_sc = sc;
    if (cf.do_rename) {
      const double z7[NAER] = {0, 0, 0, 0, 0, 0, 0};
      rename_subarea<true>(C, si, sc, z7, z7);
    }
    ft.cg[0] = ft.gcy[0] * fcldy;
    ft.cg[1] = ft.gcy[1] * fcldy;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      ft.ci[K::numslot(m)] = (si.num[m] / 1.0) * fcldy;
      ft.oc[K::numslot(m)] = (0.0 + 0.0 * fclea) + (sc.num[m] / 1.0) * fcldy;
#pragma unroll
      for (int xx = 0; xx < NAER; ++xx) {
        const int sl = K::aer_slot(xx, m);
        if (sl >= 0) {
          ft.ci[sl] = (si.aer[xx][m] / K::fcvt_aer(xx)) * fcldy;
          ft.oc[sl] = (0.0 + 0.0 * fclea) + (sc.aer[xx][m] / K::fcvt_aer(xx)) * fcldy;
        }
      }
    }
    load_sub(s, ft.qi, ft.fn_c, ft.fm_c);
    s.gas[0] = ft.gcl[0] * fsoag;
    s.gas[1] = ft.gcl[1] * 1.0;
    ft.rh_sub = ft.rhc;
  }
  ft.qgas1[0] = ft.g_soag * fsoag;
  ft.qgas1[1] = ft.g_h2so4 * 1.0;
  ft.s_entry = s;
  const double aircon = pmid / (8314.46759100000 * temp);
  ClearMid &cm = ft.cm;
  cm.netprod1 = 0.0;
  if (cf.do_cond && cf.optaa == 2) {
    cm.netprod1 = (s.gas[1] - ft.qgas1[1]) / dt;
    s.gas[1] = (cm.netprod1 >= 0) ? ft.qgas1[1] : 0;
  }
  double uptk0[NMODE] = {0, 0, 0, 0};
  if constexpr (KNOWN) {
    ft.gd = kn->gd;
    ft.fp = kn->fp;
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      ft.rate[n] = kn->rate[n];
  } else {
    h2so4_diffusivity(temp, pmid, ft.gd, ft.fp);
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      ft.rate[n] = uptake_rate_mode(C, n, ft.gd, ft.fp, ft.dgn_awet[n]);
  }
  cm.sv_so4_ait = s.aer[1][1];
  cm.sv_soa_ait = s.aer[0][1];
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    cm.uptk1[n] = cf.do_cond ? ft.rate[n] * (s.num[n] * aircon) : 0.0;
    uptk0[n] = cm.uptk1[n] * 0.81;
  }
  ft.s_pre_soa = s;
  soa_init(ft.soa0, (double)(int)(dt / 1), temp, pmid, s, uptk0);
}

// ---- suffix: H2SO4 update, renaming, nucleation, coagulation, aging and
// the recombination with the cloudy subarea, from the state after the SOA
// loop (s_soa) to the 52 tendencies
struct SuffixIn {
  Sub s_soa;
  ClearMid cm;  // netprod1, uptk1, sv_so4_ait, sv_soa_ait
  double dgn_pc, rh_sub, cc[12];
  bool partly;
  double fclea, ci[NPOP], cg[2];
};

struct SuffixStates {
  Sub s_h2so4, s_ren, s_nuc, s_coag, s_fin;
  double qavg, grow[NAER], uptkrate;
};

MAM4B_HD void suffix_states(const StepConsts &C, const AdjCfg &cf, double temp, double pmid,
                            double zm, double pblh, double dt, const SuffixIn &in,
                            SuffixStates &st) {
  const double dtsub = (double)(int)(dt / 1);
  Sub s = in.s_soa;
  double qgas_avg1 = s.gas[1];
  st.uptkrate = 0.0;
#pragma unroll
  for (int k = 0; k < NAER; ++k)
    st.grow[k] = 0.0;
  if (cf.do_cond) {
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      st.uptkrate += in.cm.uptk1[n];
    h2so4_update(dtsub, in.cm.netprod1, s, in.cm.uptk1, qgas_avg1);
    st.grow[1] = s.aer[1][1] - in.cm.sv_so4_ait;
    st.grow[0] = s.aer[0][1] - in.cm.sv_soa_ait;
  }
  st.qavg = qgas_avg1;
  st.s_h2so4 = s;
  if (cf.do_rename) {
    const double z7[NAER] = {0, 0, 0, 0, 0, 0, 0};
    rename_subarea<false>(C, s, s, st.grow, z7);
  }
  st.s_ren = s;
  if (cf.do_newnuc)
    nucleation(C, dtsub, temp, pmid, zm, pblh, in.rh_sub, st.uptkrate, qgas_avg1, s);
  st.s_nuc = s;
  double coag_in[NAER] = {0, 0, 0, 0, 0, 0, 0};
  if (cf.do_coag)
    coagulation(dtsub, in.cc, s, coag_in);
  st.s_coag = s;
  double dn_c[NMODE] = {0, 0, 0, 0}, dn_g[NMODE] = {0, 0, 0, 0};
  double dc[NAER][NMODE], dq[NAER][NMODE];
#pragma unroll
  for (int a = 0; a < NAER; ++a)
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      dc[a][m] = 0.0;
      dq[a][m] = 0.0;
    }
  aging(C, cf.nmono, in.dgn_pc, s, dn_c, dn_g, dc, dq, coag_in);
  st.s_fin = s;
}

// the 52 tendencies of a cell with a clear subarea (condensation on, so the
// gases always come from the subarea states)
MAM4B_HD void suffix_outputs(const StepConsts &C, const SuffixIn &in, const SuffixStates &st,
                             const double (&x)[MAM4B_NIN], const double (&oc)[NPOP], double dt,
                             double (&y)[MAM4B_NOUT]) {
  const double fsoag = C.fcvt_soag;
  const Sub &s = st.s_fin;
  const double w = in.partly ? in.fclea : 1.0 - 0.0;
  const double o_soag = dmax(0.0, (0.0 + (s.gas[0] / fsoag) * w) + (in.partly ? in.cg[0] : 0.0));
  const double o_h2so4 = dmax(0.0, (0.0 + (s.gas[1] / 1.0) * w) + (in.partly ? in.cg[1] : 0.0));
  y[MAM4B_OUT_TEND + 0] = (o_h2so4 * C.to_mmr[0] - x[MAM4B_IN_H2SO4]) / dt;
  y[MAM4B_OUT_TEND + 1] = (o_soag * C.to_mmr[1] - x[MAM4B_IN_SOAG]) / dt;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    const int ns = K::numslot(m);
    const double oin = dmax(0.0, (0.0 + (s.num[m] / 1.0) * w) + (in.partly ? in.ci[ns] : 0.0));
    y[MAM4B_OUT_TEND + 2 + ns] = (oin * C.to_mmr[2 + ns] - x[MAM4B_IN_AER_I + ns]) / dt;
#pragma unroll
    for (int xx = 0; xx < NAER; ++xx) {
      const int sl = K::aer_slot(xx, m);
      if (sl >= 0) {
        const double o = dmax(0.0, (0.0 + (s.aer[xx][m] / K::fcvt_aer(xx)) * w) +
                                       (in.partly ? in.ci[sl] : 0.0));
        y[MAM4B_OUT_TEND + 2 + sl] = (o * C.to_mmr[2 + sl] - x[MAM4B_IN_AER_I + sl]) / dt;
      }
    }
  }
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    y[MAM4B_OUT_TEND + 27 + p] = (oc[p] * C.to_mmr[2 + p] - x[MAM4B_IN_AER_C + p]) / dt;
}

struct SuffixBar {
  Sub sb;  // cotangent of the subarea state after the SOA loop
  double netprodb, uptk1b[NMODE], sv_so4b, sv_soab, dgn_pcb, rh_subb, tb;
  double ccb[12], cib[NPOP], cgb[2];
};

// Reverse of recombination and suffix; yb: cotangents of the 52
// tendencies (the interstitial and gas rows are used here).
MAM4B_HD void suffix_rev(const StepConsts &C, const AdjCfg &cf, double temp, double pmid, double zm,
                         double pblh, double dt, const SuffixIn &in, const SuffixStates &st,
                         const double (&ybt)[MAM4B_NUM_PROG], SuffixBar &out) {
  const double fsoag = C.fcvt_soag;
  const double dtsub = (double)(int)(dt / 1);
  const double z7[NAER] = {0, 0, 0, 0, 0, 0, 0};
  Sub &sb = out.sb;
  sub_zero(sb);
  out.netprodb = out.sv_so4b = out.sv_soab = out.dgn_pcb = out.rh_subb = out.tb = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    out.uptk1b[n] = 0.0;
#pragma unroll
  for (int k = 0; k < 12; ++k)
    out.ccb[k] = 0.0;
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    out.cib[p] = 0.0;
  out.cgb[0] = out.cgb[1] = 0.0;
  // recombination
  const Sub &s = st.s_fin;
  const double w = in.partly ? in.fclea : 1.0 - 0.0;
  {
    const double o_soagb = ybt[1] * C.to_mmr[1] / dt;
    const double o_h2so4b = ybt[0] * C.to_mmr[0] / dt;
    const double b0 = maxc_rev(0.0, (0.0 + (s.gas[0] / fsoag) * w) + (in.partly ? in.cg[0] : 0.0), o_soagb);
    const double b1 = maxc_rev(0.0, (0.0 + (s.gas[1] / 1.0) * w) + (in.partly ? in.cg[1] : 0.0), o_h2so4b);
    if (in.partly) {
      out.cgb[0] += b0;
      out.cgb[1] += b1;
    }
    sb.gas[0] += b0 * w / fsoag;
    sb.gas[1] += b1 * w;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      const int ns = K::numslot(m);
      const double oib = ybt[2 + ns] * C.to_mmr[2 + ns] / dt;
      const double bn = maxc_rev(0.0, (0.0 + (s.num[m] / 1.0) * w) + (in.partly ? in.ci[ns] : 0.0), oib);
      sb.num[m] += bn * w;
      if (in.partly)
        out.cib[ns] += bn;
#pragma unroll
      for (int xx = 0; xx < NAER; ++xx) {
        const int sl = K::aer_slot(xx, m);
        if (sl >= 0) {
          const double ob = ybt[2 + sl] * C.to_mmr[2 + sl] / dt;
          const double ba = maxc_rev(0.0, (0.0 + (s.aer[xx][m] / K::fcvt_aer(xx)) * w) +
                                              (in.partly ? in.ci[sl] : 0.0), ob);
          sb.aer[xx][m] += ba * w / K::fcvt_aer(xx);
          if (in.partly)
            out.cib[sl] += ba;
        }
      }
    }
  }
  aging_rev(C, cf.nmono, in.dgn_pc, st.s_coag, sb, out.dgn_pcb);
  if (cf.do_coag) {
    const double cinb[NAER] = {0, 0, 0, 0, 0, 0, 0};
    coagulation_rev(dtsub, in.cc, st.s_nuc, sb, out.ccb, cinb);
  }
  double uptkrateb = 0.0, qavgb = 0.0;
  if (cf.do_newnuc)
    nucleation_rev(C, dtsub, temp, pmid, zm, pblh, in.rh_sub, st.uptkrate, st.qavg,
                   st.s_ren.gas[1], st.s_ren.num[1], st.s_ren.aer[1][1], sb.gas[1], sb.num[1],
                   sb.aer[1][1], out.tb, out.rh_subb, uptkrateb, qavgb);
  double growb[NAER] = {0, 0, 0, 0, 0, 0, 0};
  if (cf.do_rename) {
    Sub dummy;
    sub_zero(dummy);
    double gcb2[NAER] = {0, 0, 0, 0, 0, 0, 0};
    rename_subarea_rev<false>(C, st.s_h2so4, st.s_h2so4, st.grow, z7, sb, dummy, growb, gcb2);
  }
  if (cf.do_cond) {
    sb.aer[1][1] += growb[1];
    out.sv_so4b -= growb[1];
    sb.aer[0][1] += growb[0];
    out.sv_soab -= growb[0];
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      out.uptk1b[n] += uptkrateb;
    double a1b[NMODE];
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      a1b[n] = sb.aer[1][n];
    double q1b = 0.0;
    h2so4_update_rev(dtsub, in.cm.netprod1, in.s_soa.gas[1], in.cm.uptk1, sb.gas[1], qavgb, a1b,
                     q1b, out.netprodb, out.uptk1b);
    sb.gas[1] = q1b;
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      sb.aer[1][n] = a1b[n];
  } else {
    sb.gas[1] += qavgb;
  }
}

// coagulation coefficients reverse: ccb to T, the wet diameters and the
// wet densities (dmax(1000, .) applied)
MAM4B_HD void coef_rev(const StepConsts &C, const CoagTables &T, double temp, double pmid,
                       const double (&dgn_awet)[NMODE], const double (&wetdens)[NMODE],
                       const double (&ccb)[12], double &tb, double (&dgn_awetb)[NMODE],
                       double (&wetdensb)[NMODE]) {
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    const int sm = coag_src(p), dm = coag_dst(p);
    const double cb4[4] = {ccb[p], ccb[3 + p], ccb[6 + p], ccb[9 + p]};
    coag_pair_coefs_rev(C, T, p, temp, pmid, dgn_awet[sm], dgn_awet[dm], wetdens[sm], wetdens[dm],
                        cb4, tb, dgn_awetb[sm], dgn_awetb[dm], wetdensb[sm], wetdensb[dm]);
  }
}

// ---- reverse of the front, in three parts:
// front_rev_head: the clear-subarea prefix (from the suffix's cotangents
//   and the SOA loop's initial-state cotangents lb), the subarea set-up,
//   the cloudy (sub)area and the clipping after calcsize; xb receives the
//   partial cotangents of the inputs, tl those of the water uptake's
//   outputs and of calcsize's (diameters, tendencies);
// front_rev_mode<M>: water uptake of mode M (adds to xb's species rows of
//   the mode and to tl.dgn_ab[M]; returns the cotangent of the RH);
// front_rev_tail: RH of water uptake and calcsize, into xb.
// Extra cotangents of the front values: dgn_awetb, wetdensb (coagulation
// coefficients), tb_extra (T).
struct FrontTail {
  double pt_ib[NPOP], pt_cb[NPOP];  // calcsize tendencies
  double dgn_ab[NMODE];             // dry diameters
  double dgn_awetb[NMODE], qaerwatb[NMODE], wetdens_wub[NMODE];  // water-uptake outputs
};

MAM4B_HD void front_rev_head(const StepConsts &C, const AdjCfg &cf, const double (&x)[MAM4B_NIN],
                             double dt, const FrontTape &ft, const SuffixBar *sbar,
                             const SoaBar *lb, const double (&yb)[MAM4B_NOUT],
                             const double (&dgn_awetb_in)[NMODE],
                             const double (&wetdensb_in)[NMODE], double tb_extra,
                             double (&xb)[MAM4B_NIN], FrontTail &tl) {
  const double temp = x[MAM4B_IN_T], pmid = x[MAM4B_IN_P];
  const double qv = x[MAM4B_IN_QV], cld = x[MAM4B_IN_CLD];
  double ai[NPOP], ac[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ai[p] = x[MAM4B_IN_AER_I + p];
    ac[p] = x[MAM4B_IN_AER_C + p];
  }
#pragma unroll
  for (int f = 0; f < MAM4B_NIN; ++f)
    xb[f] = 0.0;
  double aib[NPOP], acb[NPOP], qib[NPOP], qcb[NPOP], ocb[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ocb[p] = yb[MAM4B_OUT_TEND + 27 + p] * C.to_mmr[2 + p] / dt;
    aib[p] = -yb[MAM4B_OUT_TEND + 2 + p] / dt;
    acb[p] = -yb[MAM4B_OUT_TEND + 27 + p] / dt;
    qib[p] = 0.0;
    qcb[p] = 0.0;
  }
  xb[MAM4B_IN_H2SO4] -= yb[MAM4B_OUT_TEND + 0] / dt;
  xb[MAM4B_IN_SOAG] -= yb[MAM4B_OUT_TEND + 1] / dt;
  double dgn_ab[NMODE], dgn_awetb[NMODE], wetdens_wub[NMODE], qaerwatb[NMODE], wetdensb[NMODE];
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    dgn_ab[m] = yb[MAM4B_OUT_DGN_A + m];
    dgn_awetb[m] = yb[MAM4B_OUT_DGN_AWET + m] + dgn_awetb_in[m];
    wetdens_wub[m] = yb[MAM4B_OUT_WETDENS + m];
    qaerwatb[m] = yb[MAM4B_OUT_QAERWAT + m];
    wetdensb[m] = wetdensb_in[m];
  }
  double g_h2so4b = 0.0, g_soagb = 0.0, relhumb = 0.0, tb = tb_extra, qvb = 0.0;
  const double fsoag = C.fcvt_soag;
  const double z7[NAER] = {0, 0, 0, 0, 0, 0, 0};
  if (ft.cat == 1) {
    Sub si = ft.cy_si, sc = ft.cy_sc;
    if (cf.do_rename)
      rename_subarea<true>(C, si, sc, z7, z7);
    Sub sib, scb;
    sub_zero(sib);
    sub_zero(scb);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      const int ns = K::numslot(m);
      sib.num[m] += maxc_rev(0.0, 0.0 + si.num[m], yb[MAM4B_OUT_TEND + 2 + ns] * C.to_mmr[2 + ns] / dt);
      scb.num[m] += ocb[ns];
#pragma unroll
      for (int xx = 0; xx < NAER; ++xx) {
        const int sl = K::aer_slot(xx, m);
        if (sl >= 0) {
          const double oib = yb[MAM4B_OUT_TEND + 2 + sl] * C.to_mmr[2 + sl] / dt;
          sib.aer[xx][m] += maxc_rev(0.0, 0.0 + si.aer[xx][m] / K::fcvt_aer(xx), oib) / K::fcvt_aer(xx);
          scb.aer[xx][m] += ocb[sl] / K::fcvt_aer(xx);
        }
      }
    }
    g_soagb += maxc_rev(0.0, 0.0 + ft.g_soag, yb[MAM4B_OUT_TEND + 1] * C.to_mmr[1] / dt);
    g_h2so4b += maxc_rev(0.0, 0.0 + ft.g_h2so4, yb[MAM4B_OUT_TEND + 0] * C.to_mmr[0] / dt);
    if (cf.do_rename) {
      double gb1[NAER] = {0, 0, 0, 0, 0, 0, 0}, gb2[NAER] = {0, 0, 0, 0, 0, 0, 0};
      rename_subarea_rev<true>(C, ft.cy_si, ft.cy_sc, z7, z7, sib, scb, gb1, gb2);
    }
    load_sub_plain_rev(sib, qib);
    load_sub_plain_rev(scb, qcb);
  } else {
    const bool partly = ft.cat == 2;
    const double fcldy = cld, fclea = 1.0 - fcldy;
    const double aircon = pmid / (8314.46759100000 * temp);
    Sub sb = sbar->sb;  // state after the SOA loop == before it, except SOA
    // SOA loop initial state and parameters
    if (cf.do_cond) {
      sb.gas[0] = lb->g;
      constexpr double opoa_frac[NMODE] = {0.1, 0.1, 0.1, 0.0};
#pragma unroll
      for (int n = 0; n < NMODE; ++n)
        sb.aer[0][n] = lb->a[n];
#pragma unroll
      for (int n = 0; n < NMODE; ++n)
        sb.aer[2][n] += maxxc_rev(ft.s_pre_soa.aer[2][n], 0.0, lb->opoa[n] * opoa_frac[n]);
      tb += lb->g0 * soa_g0_dT(temp, pmid);
    }
    double uptk1b[NMODE];
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      uptk1b[n] = sbar->uptk1b[n] + (cf.do_cond ? lb->uptk[n] * 0.81 : 0.0);
    tb += sbar->tb;
    dgn_ab[3] += sbar->dgn_pcb;
    // sv = state at the prefix
    sb.aer[1][1] += sbar->sv_so4b;
    sb.aer[0][1] += sbar->sv_soab;
    if (cf.do_cond) {
      double aircb = 0.0, rateb[NMODE];
#pragma unroll
      for (int n = 0; n < NMODE; ++n) {
        rateb[n] = uptk1b[n] * (ft.s_pre_soa.num[n] * aircon);
        sb.num[n] += uptk1b[n] * ft.rate[n] * aircon;
        aircb += uptk1b[n] * ft.rate[n] * ft.s_pre_soa.num[n];
      }
      tb -= aircb * aircon / temp;
      double gdb = 0.0, fpb = 0.0;
#pragma unroll
      for (int n = 0; n < NMODE; ++n)
        uptake_rate_mode_rev(C, n, ft.gd, ft.fp, ft.dgn_awet[n], rateb[n], gdb, fpb, dgn_awetb[n]);
      h2so4_diffusivity_rev(temp, pmid, gdb, fpb, tb);
    }
    // optaa-2 production split
    double qgas1b[2] = {0, 0};
    if (cf.do_cond && cf.optaa == 2) {
      if (ft.cm.netprod1 >= 0)
        qgas1b[1] += sb.gas[1];
      sb.gas[1] = sbar->netprodb / dt;
      qgas1b[1] -= sbar->netprodb / dt;
    }
    g_soagb += qgas1b[0] * fsoag;
    g_h2so4b += qgas1b[1];
    if (!partly) {
      load_sub_plain_rev(sb, qib);
      g_soagb += sb.gas[0] * fsoag;
      g_h2so4b += sb.gas[1];
      relhumb += sbar->rh_subb;
#pragma unroll
      for (int p = 0; p < NPOP; ++p)
        qcb[p] += ocb[p];
    } else {
      double fn_cb[NMODE] = {0, 0, 0, 0}, fm_cb[NMODE] = {0, 0, 0, 0};
      double fn_yb[NMODE] = {0, 0, 0, 0}, fm_yb[NMODE] = {0, 0, 0, 0};
      load_sub_rev(sb, ft.qi, ft.fn_c, ft.fm_c, qib, fn_cb, fm_cb);
      double gclb[2] = {sb.gas[0] * fsoag, sb.gas[1]};
      relhumb += boundc_rev(0.0, 1.0, (ft.relhumgcm - fcldy) / fclea, sbar->rh_subb) / fclea;
      Sub sib, scb;
      sub_zero(sib);
      sub_zero(scb);
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        sib.num[m] += sbar->cib[K::numslot(m)] * fcldy;
        scb.num[m] += ocb[K::numslot(m)] * fcldy;
#pragma unroll
        for (int xx = 0; xx < NAER; ++xx) {
          const int sl = K::aer_slot(xx, m);
          if (sl >= 0) {
            sib.aer[xx][m] += sbar->cib[sl] * fcldy / K::fcvt_aer(xx);
            scb.aer[xx][m] += ocb[sl] * fcldy / K::fcvt_aer(xx);
          }
        }
      }
      const double gcyb[2] = {sbar->cgb[0] * fcldy, sbar->cgb[1] * fcldy};
      if (cf.do_rename) {
        double gb1[NAER] = {0, 0, 0, 0, 0, 0, 0}, gb2[NAER] = {0, 0, 0, 0, 0, 0, 0};
        rename_subarea_rev<true>(C, ft.cy_si, ft.cy_sc, z7, z7, sib, scb, gb1, gb2);
      }
      load_sub_rev(sib, ft.qi, ft.fn_y, ft.fm_y, qib, fn_yb, fm_yb);
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        qcb[K::numslot(m)] += scb.num[m] / fcldy;
#pragma unroll
        for (int xx = 0; xx < NAER; ++xx) {
          const int sl = K::aer_slot(xx, m);
          if (sl >= 0)
            qcb[sl] += scb.aer[xx][m] * K::fcvt_aer(xx) / fcldy;
        }
      }
      double g0b[2];
#pragma unroll
      for (int g = 0; g < 2; ++g)
        g0b[g] = ft.gcy_clip[g] ? gclb[g] / fclea : gclb[g] + gcyb[g] * (1.0 - fclea) / fcldy;
      g_soagb += g0b[0];
      g_h2so4b += g0b[1];
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        part_factors_rev(fcldy, ft.qi[K::numslot(m)], ft.qc[K::numslot(m)], fn_cb[m], fn_yb[m],
                         qib[K::numslot(m)], qcb[K::numslot(m)]);
        double si_ = 0.0, sc_ = 0.0;
#pragma unroll
        for (int k = 0; k < K::nspec(m); ++k) {
          si_ = si_ + ft.qi[K::spec0(m) + k];
          sc_ = sc_ + ft.qc[K::spec0(m) + k];
        }
        double sib_ = 0.0, scb_ = 0.0;
        part_factors_rev(fcldy, si_, sc_, fm_cb[m], fm_yb[m], sib_, scb_);
#pragma unroll
        for (int k = 0; k < K::nspec(m); ++k) {
          qib[K::spec0(m) + k] += sib_;
          qcb[K::spec0(m) + k] += scb_;
        }
      }
    }
  }
  // front
  xb[MAM4B_IN_H2SO4] += maxc_rev(0.0, x[MAM4B_IN_H2SO4] * C.to_vmr[0], g_h2so4b) * C.to_vmr[0];
  xb[MAM4B_IN_SOAG] += maxc_rev(0.0, x[MAM4B_IN_SOAG] * C.to_vmr[1], g_soagb) * C.to_vmr[1];
  relhum_gcm_rev(qv, temp, pmid, relhumb, qvb, tb);
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    wetdens_wub[m] += maxc_rev(1000.0, ft.wetdens_wu[m], wetdensb[m]);
  {
    double dgn_tmp[NMODE], pt_i[NPOP], pt_c[NPOP];
    calcsize(C, ai, ac, dt, dgn_tmp, pt_i, pt_c);
#pragma unroll
    for (int p = 0; p < NPOP; ++p) {
      const double ui = ai[p] + pt_i[p] * dt, uc = ac[p] + pt_c[p] * dt;
      const double vi = dmax(0.0, ui) * C.to_vmr[2 + p], vc = dmax(0.0, uc) * C.to_vmr[2 + p];
      const double ubi = maxc_rev(0.0, ui, maxc_rev(0.0, vi, qib[p]) * C.to_vmr[2 + p]);
      const double ubc = maxc_rev(0.0, uc, maxc_rev(0.0, vc, qcb[p]) * C.to_vmr[2 + p]);
      aib[p] += ubi;
      acb[p] += ubc;
      tl.pt_ib[p] = ubi * dt;
      tl.pt_cb[p] = ubc * dt;
    }
  }
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    tl.dgn_ab[m] = dgn_ab[m];
    tl.dgn_awetb[m] = dgn_awetb[m];
    tl.qaerwatb[m] = qaerwatb[m];
    tl.wetdens_wub[m] = wetdens_wub[m];
  }
  xb[MAM4B_IN_T] += tb;
  xb[MAM4B_IN_QV] += qvb;
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    xb[MAM4B_IN_AER_I + p] += aib[p];
    xb[MAM4B_IN_AER_C + p] += acb[p];
  }
}

// water uptake of mode M: sp the mode's species (mode_species<M>), rh_wu
// and dgn_a the forward's values; spb receives the species' cotangents
template <int M>
MAM4B_HD double front_rev_mode(const StepConsts &C, const double (&sp)[7], double rh_wu,
                               double dgn_a, double dgn_awetb, double qaerwatb,
                               double wetdens_wub, double (&spb)[7], double &dgn_ab) {
#pragma unroll
  for (int k = 0; k < 7; ++k)
    spb[k] = 0.0;
  double rh_wub = 0.0;
  water_uptake_mode_rev<M>(C, sp, rh_wu, dgn_a, dgn_awetb, qaerwatb, wetdens_wub, spb, rh_wub,
                           dgn_ab);
  return rh_wub;
}

// rh_wub: the sum of the modes' RH cotangents; aib, acb, tb, qvb hold the
// partial cotangents of the populations, T and qv (the species complete
// with the water uptake's) and receive the rest
MAM4B_HD void front_rev_tail(const StepConsts &C, const double (&ai)[NPOP],
                             const double (&ac)[NPOP], double qv, double temp, double pmid,
                             double cld, double dt, const FrontTail &tl, double rh_wub,
                             double (&aib)[NPOP], double (&acb)[NPOP], double &tb, double &qvb) {
  water_uptake_rh_rev(qv, temp, pmid, cld, rh_wub, qvb, tb);
  calcsize_rev(C, ai, ac, dt, tl.dgn_ab, tl.pt_ib, tl.pt_cb, aib, acb);
}

// the whole reverse of the front in one thread
MAM4B_HD void front_rev(const StepConsts &C, const AdjCfg &cf, const double (&x)[MAM4B_NIN],
                        double dt, const FrontTape &ft, const SuffixBar *sbar, const SoaBar *lb,
                        const double (&yb)[MAM4B_NOUT], const double (&dgn_awetb_in)[NMODE],
                        const double (&wetdensb_in)[NMODE], double tb_extra,
                        double (&xb)[MAM4B_NIN]) {
  FrontTail tl;
  front_rev_head(C, cf, x, dt, ft, sbar, lb, yb, dgn_awetb_in, wetdensb_in, tb_extra, xb, tl);
  double ai[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    ai[p] = x[MAM4B_IN_AER_I + p];
  double rh_wub = 0.0;
  double sp[7], spb[7];
#define MAM4B_WU_REV(M)                                                                     \
  {                                                                                         \
    mode_species<M>(ai, sp);                                                                \
    const double r = front_rev_mode<M>(C, sp, ft.rh_wu, ft.dgn_a[M], tl.dgn_awetb[M],       \
                                       tl.qaerwatb[M], tl.wetdens_wub[M], spb, tl.dgn_ab[M]); \
    rh_wub += r;                                                                            \
    for (int k = 0; k < K::nspec(M); ++k)                                                   \
      xb[MAM4B_IN_AER_I + K::spec0(M) + k] += spb[k];                                       \
  }
  MAM4B_WU_REV(0)
  MAM4B_WU_REV(1)
  MAM4B_WU_REV(2)
  MAM4B_WU_REV(3)
#undef MAM4B_WU_REV
  double ac[NPOP], aib[NPOP], acb[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ac[p] = x[MAM4B_IN_AER_C + p];
    aib[p] = xb[MAM4B_IN_AER_I + p];
    acb[p] = xb[MAM4B_IN_AER_C + p];
  }
  front_rev_tail(C, ai, ac, x[MAM4B_IN_QV], x[MAM4B_IN_T], x[MAM4B_IN_P], x[MAM4B_IN_CLD], dt, tl,
                 rh_wub, aib, acb, xb[MAM4B_IN_T], xb[MAM4B_IN_QV]);
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    xb[MAM4B_IN_AER_I + p] = aib[p];
    xb[MAM4B_IN_AER_C + p] = acb[p];
  }
}

// suffix inputs of a cell from its front tape and the SOA loop result
MAM4B_HD void suffix_in_from_front(const FrontTape &ft, const SoaState &soa_end, double cld,
                                   const double (&cc)[12], SuffixIn &in) {
  in.s_soa = ft.s_pre_soa;
  in.s_soa.gas[0] = soa_end.g;
#pragma unroll
  for (int n = 0; n < NMODE; ++n)
    in.s_soa.aer[0][n] = soa_end.a[n];
  in.cm = ft.cm;
  in.dgn_pc = ft.dgn_a[3];
  in.rh_sub = ft.rh_sub;
#pragma unroll
  for (int k = 0; k < 12; ++k)
    in.cc[k] = cc[k];
  in.partly = ft.cat == 2;
  in.fclea = 1.0 - cld;
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    in.ci[p] = ft.ci[p];
  in.cg[0] = ft.cg[0];
  in.cg[1] = ft.cg[1];
}

// ---- whole cell in one thread (forward then reverse); the SOA
// checkpoints go to ck (stride cks). y gets the 68 outputs.
MAM4B_HD void cell_adjoint(const StepConsts &C, const CoagTables &T, const AdjCfg &cf,
                           const double (&x)[MAM4B_NIN], double pblh, double dt, double *ck,
                           size_t cks, const double (&yb)[MAM4B_NOUT], double (&y)[MAM4B_NOUT],
                           double (&xb)[MAM4B_NIN], int &niter) {
  FrontTape ft;
  front_forward<false>(C, cf, x, dt, ft, y);
  const double zero4[NMODE] = {0, 0, 0, 0};
  niter = 0;
  if (ft.cat == 1) {
    front_rev(C, cf, x, dt, ft, nullptr, nullptr, yb, zero4, zero4, 0.0, xb);
    return;
  }
  const double temp = x[MAM4B_IN_T], pmid = x[MAM4B_IN_P], zm = x[MAM4B_IN_ZM];
  SoaState se = ft.soa0;
  if (cf.do_cond)
    niter = soa_forward_ck(se, ck, cks);
  double cc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (cf.do_coag) {
    const double aircon = pmid / (8314.46759100000 * temp);
    coag_all_coefs(C, T, temp, pmid, aircon, ft.dgn_awet, ft.wetdens, cc);
  }
  SuffixIn in;
  if (cf.do_cond) {
    suffix_in_from_front(ft, se, x[MAM4B_IN_CLD], cc, in);
  } else {
    SoaState none = ft.soa0;
    none.g = ft.s_pre_soa.gas[0];
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      none.a[n] = ft.s_pre_soa.aer[0][n];
    suffix_in_from_front(ft, none, x[MAM4B_IN_CLD], cc, in);
  }
  SuffixStates st;
  suffix_states(C, cf, temp, pmid, zm, pblh, dt, in, st);
  suffix_outputs(C, in, st, x, ft.oc, dt, y);
  double ybt[MAM4B_NUM_PROG];
#pragma unroll
  for (int k = 0; k < MAM4B_NUM_PROG; ++k)
    ybt[k] = yb[MAM4B_OUT_TEND + k];
  SuffixBar sbar;
  suffix_rev(C, cf, temp, pmid, zm, pblh, dt, in, st, ybt, sbar);
  double dgn_awetb[NMODE] = {0, 0, 0, 0}, wetdensb[NMODE] = {0, 0, 0, 0}, tb = 0.0;
  if (cf.do_coag)
    coef_rev(C, T, temp, pmid, ft.dgn_awet, ft.wetdens, sbar.ccb, tb, dgn_awetb, wetdensb);
  SoaBar lb;
  lb.g = sbar.sb.gas[0];
  lb.tcur = 0.0;
  lb.g0 = 0.0;
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    lb.a[n] = sbar.sb.aer[0][n];
    lb.opoa[n] = 0.0;
    lb.uptk[n] = 0.0;
  }
  if (cf.do_cond)
    soa_loop_rev(ft.soa0, niter, ck, cks, lb);
  front_rev(C, cf, x, dt, ft, &sbar, &lb, yb, dgn_awetb, wetdensb, tb, xb);
}

}  // namespace adj
}  // namespace mam4b
