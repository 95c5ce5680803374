// mam4b_step.cu -- sm_100a kernels and the C ABI (include/mam4b.h) of the
// B200-native MAM4 microphysics step.
//
// One thread owns one grid cell for the whole step (calcsize -> water
// uptake -> amicphys); inputs and outputs are structure-of-arrays fields,
// so each load/store instruction of a warp touches 32 consecutive doubles.
// Cells are independent: there is no inter-thread communication and no
// shared memory; the coagulation correction tables are read through L1.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <new>
#include <type_traits>
#include <vector>

#include "../../include/mam4b.h"
#include "mam4b_physics.cuh"
#include "mam4b_physics_mixed.cuh"
#include "mam4b_adjoint.cuh"
#include "mam4b_process.cuh"
#include "mam4b_setsox.cuh"
#include "mam4b_gaschem.cuh"
#include "mam4b_activation.cuh"
#include "mam4b_dropmix.cuh"
#include "mam4b_optics.cuh"

namespace mam4b {

// ------------------------------------------------------- device constants
__constant__ StepConsts c_k;

#define COAG_TABLE_QUALIFIER __device__ const
#include "coag_tables.inc"
#undef COAG_TABLE_QUALIFIER

struct StepArgs {
  const double *in[MAM4B_NIN];
  const double *pblh;
  double *out[MAM4B_NOUT];
  double *diag[MAM4B_NDIAG];
  unsigned *flags;
  long long ncell;
  int nlev;
  double dt;
  int do_cond, do_rename, do_newnuc, do_coag, optaa;
  unsigned nmono;
  // SOA solver hand-off (see soa_kernel): per-cell loop state, the list of
  // queued cells, the solver's order and counters (CNT_*)
  double *soa;       // [SOA_FIELDS][ncell], indexed by queue slot
  double *hand;      // [H_FIELDS][ncell], indexed by queue slot
  int *task;         // [ncell]: cell of each queue slot
  int *order;        // [ncell]: slots in solver order, long loops from the
                     // front, short ones from the back
  double *aux;       // [AUX_FIELDS][ncell], indexed by cell (size/mode kernels)
  unsigned *counters;
  int *npass;        // [ncell] or null: passes of each slot's loop (adjoint only)
  int mixed;         // the mode/pair stages ran in FP32 (MAM4B_MIXED, _FAST)
  double inline_scale;  // pre_kernel<.., FUSE>: cells whose first SOA sub-step
                        // is at least 1/inline_scale of the step finish in pre
};

// The step runs as a pipeline of six kernels when condensation is on and
// no diagnostics are asked for: size_kernel, mode_kernel and pair_kernel
// compute calcsize, water uptake, uptake rates and coagulation coefficients
// into `aux` and the size outputs; pre_kernel runs each cell up to the SOA
// condensation loop of its clear subarea, writes the loop's initial state
// and the rest of the cell's state at that point to slot-indexed scratch
// and queues the cell (cloudy cells finish there); soa_kernel runs the
// queued loops with per-lane work stealing; post_kernel finishes the queued
// cells from the hand-off and the loop result. Otherwise full_kernel runs
// each cell start to end in one thread.
enum { SOA_G = 0, SOA_A = 1, SOA_OPOA = 5, SOA_UPTK = 9, SOA_G0 = 13, SOA_FIELDS = 14 };
// per-cell values from size_kernel and mode_kernel for the pre kernel:
// relative humidity for water uptake, H2SO4 diffusivity and mean free path,
// per-particle H2SO4 uptake rate of each mode
// and the 12 coagulation coefficients (coag_all_coefs order)
enum { AUX_RH = 0, AUX_GDIFF = 1, AUX_FPATH = 2, AUX_RATE = 3, AUX_COAG = 7, AUX_FIELDS = 19 };
// queue counters: queued slots, slots handed to the solver, long and short
// loops in the order list
enum { CNT_QUEUED = 0, CNT_TAKEN = 1, CNT_LONG = 2, CNT_SHORT = 3, CNT_TAKEN_ADJ = 4,
       CNT_WORDS = 8 };
// A loop is started early when its first sub-step is shorter than
// dt / kLongLoopSteps, i.e. when it is expected to take at least about that
// many sub-steps (the SOA loop's step is 0.05 / sum(uptake * |phi|)).
constexpr double kLongLoopSteps = 300.0;

// ----------------------------------------------------- per-cell amicphys
struct Diag {
  // amicphys process tendencies for the grid cell, in the 31-tracer
  // order: [process 0..3][tracer], cloud-borne renaming [tracer]
  double t[NQTEND][31];
  double cw[31];
};

__device__ __forceinline__ int pop_to_i31(int p) { return 6 + p; }
// amicphys tracer index of the number of mode m (mam4_amicphys.hpp:36)
__device__ __forceinline__ int num_i31(int m) { return m == 0 ? 13 : m == 1 ? 18 : m == 2 ? 26 : 30; }

// Hand-off of a queued cell from the pre to the post kernel: one double per
// field and queue slot ([field][slot], coalesced in both kernels).
enum {
  H_GAS1 = 0,      // H2SO4 of the clear subarea at the loop
  H_POP = 1,       // 25 numbers/masses of the clear subarea at the loop
  H_UPTK = 26,     // 4 H2SO4 uptake rates
  H_NETPROD = 30,  // H2SO4 net production of other processes
  H_SV_SO4 = 31,   // aitken SO4 and SOA before condensation
  H_SV_SOA = 32,
  H_DGN_PC = 33,   // dry diameter of the primary-carbon mode
  H_RELHUM = 34,   // relative humidity of the clear subarea
  H_CI = 35,       // 25 interstitial contributions of the cloudy subarea
  H_CG = 60,       // 2 gas contributions of the cloudy subarea (SOAG, H2SO4)
  H_SOAG0 = 62,    // SOA gas at the start of the loop (read by the adjoint)
  H_FIELDS = 63
};
// (The outgoing cloud-borne grid means are final once pre has set up the
// subareas: the clear subarea does not change them. pre writes their
// tendencies itself, store_cloudborne, so they are not handed off.)

// Clear subarea, mam_amicphys_1subarea (mam4_amicphys.hpp:1127-1697), part 1:
// optaa-2 production split and H2SO4 uptake rates from the per-particle
// rates `rate` (uptake_rates). Returns the SOAG uptake rates for the SOA
// loop.
template <bool DIAG>
__device__ __forceinline__ void clear_prefix(const StepArgs &a, double deltat, double temp,
                                             double pmid, const double (&rate)[NMODE],
                                             const double (&qgas1)[2], Sub &s, ClearMid &cm,
                                             double (&uptk0)[NMODE]) {
  const double aircon = pmid / (8314.46759100000 * temp);
  cm.netprod1 = 0.0;
  if (a.do_cond && a.optaa == 2) {
    cm.netprod1 = (s.gas[1] - qgas1[1]) / deltat;
    s.gas[1] = (cm.netprod1 >= 0) ? qgas1[1] : 0;
  }
  if (!a.do_cond)
    return;
  cm.gas_sv[0] = s.gas[0];
  cm.gas_sv[1] = s.gas[1];
  cm.sv_so4_ait = s.aer[1][1];
  cm.sv_soa_ait = s.aer[0][1];
  if (DIAG) {
#pragma unroll
    for (int x = 0; x < NAER; ++x)
#pragma unroll
      for (int m = 0; m < NMODE; ++m)
        cm.sv_all[x][m] = s.aer[x][m];
  }
#pragma unroll
  for (int n = 0; n < NMODE; ++n) {
    cm.uptk1[n] = rate[n] * (s.num[n] * aircon);
    uptk0[n] = cm.uptk1[n] * 0.81;
  }
}

// Part 2, after the SOA loop: H2SO4 update, renaming, nucleation,
// coagulation, aging. With DIAG the per-process increments are added to dg
// scaled by afrac/(fcvt*deltat). With PRECOAG, cc_pre (stride cc_stride)
// holds the 12 coagulation coefficients of the cell (coag_all_coefs) and
// dgn_awet/wetdens are not read.
template <bool DIAG, bool PRECOAG>
__device__ __forceinline__ void clear_suffix(const StepArgs &a, double deltat, double temp,
                                             double pmid, double zmid, double pblh,
                                             double relhum, double dgn_a_pc,
                                             const double (&dgn_awet)[NMODE],
                                             const double (&wetdens)[NMODE], const ClearMid &cm,
                                             Sub &s, Diag *dg, double afrac,
                                             const double *cc_pre, size_t cc_stride) {
  const StepConsts &C = c_k;
  const double aircon = pmid / (8314.46759100000 * temp);
  const double dtsub = (double)(int)(deltat / 1);
  double qgas_avg1 = s.gas[1];
  double uptkrate_h2so4 = 0.0;
  // the primary-carbon mode holds no SO4/SOA before condensation, so its
  // condensation gains are its values after it
  double cond_so4_pc = 0.0, cond_soa_pc = 0.0;
  double dcond[NAER][NMODE], dcoag[NAER][NMODE], dncond[NMODE], dncoag[NMODE];
  if (DIAG) {
#pragma unroll
    for (int x = 0; x < NAER; ++x)
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        dcond[x][m] = 0.0;
        dcoag[x][m] = 0.0;
      }
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      dncond[m] = 0.0;
      dncoag[m] = 0.0;
    }
  }
  double grow[NAER];
#pragma unroll
  for (int x = 0; x < NAER; ++x)
    grow[x] = 0.0;

  if (a.do_cond) {
#pragma unroll
    for (int n = 0; n < NMODE; ++n)
      uptkrate_h2so4 += cm.uptk1[n];
    h2so4_update(dtsub, cm.netprod1, s, cm.uptk1, qgas_avg1);
    // growth of the aitken mode by condensation: only SO4 and SOA change
    grow[1] = s.aer[1][1] - cm.sv_so4_ait;
    grow[0] = s.aer[0][1] - cm.sv_soa_ait;
    cond_so4_pc = s.aer[1][3] - 0.0;
    cond_soa_pc = s.aer[0][3] - 0.0;
    if (DIAG) {
#pragma unroll
      for (int x = 0; x < NAER; ++x)
#pragma unroll
        for (int m = 0; m < NMODE; ++m)
          dcond[x][m] = s.aer[x][m] - cm.sv_all[x][m];
      // gas increment of condensation (mam4_amicphys.hpp:1434-1438)
      dg->t[0][5] += ((0.0 + (s.gas[0] - (cm.gas_sv[0] + 0.0 * dtsub))) / (C.fcvt_soag * deltat)) * afrac;
      dg->t[0][2] += ((0.0 + (s.gas[1] - (cm.gas_sv[1] + cm.netprod1 * dtsub))) / (1.0 * deltat)) * afrac;
    }
  }

  // -------------------------------------------------------- renaming
  if (a.do_rename) {
    double nsv[NMODE], asv[NAER][NMODE];
    if (DIAG) {
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        nsv[m] = s.num[m];
#pragma unroll
        for (int x = 0; x < NAER; ++x)
          asv[x][m] = s.aer[x][m];
      }
    }
    const double zero7[NAER] = {0, 0, 0, 0, 0, 0, 0};
    rename_subarea<false>(C, s, s, grow, zero7);
    if (DIAG) {
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        dg->t[1][num_i31(m)] += ((0.0 + (s.num[m] - nsv[m])) / (1.0 * deltat)) * afrac;
#pragma unroll
        for (int x = 0; x < NAER; ++x) {
          const int slot = K::aer_slot(x, m);
          if (slot >= 0)
            dg->t[1][pop_to_i31(slot)] +=
                ((0.0 + (s.aer[x][m] - asv[x][m])) / (K::fcvt_aer(x) * deltat)) * afrac;
        }
      }
    }
  }

  // ------------------------------------------------------ nucleation
  if (a.do_newnuc) {
    const double g1 = s.gas[1], n1 = s.num[1], a1 = s.aer[1][1];
    nucleation(C, dtsub, temp, pmid, zmid, pblh, relhum, uptkrate_h2so4, qgas_avg1, s);
    if (DIAG) {
      dg->t[2][2] += ((0.0 + (s.gas[1] - g1)) / (1.0 * deltat)) * afrac;
      dg->t[2][18] += ((0.0 + (s.num[1] - n1)) / (1.0 * deltat)) * afrac;
      dg->t[2][14] += ((0.0 + (s.aer[1][1] - a1)) / (1.0 * deltat)) * afrac;
    }
  }

  // ----------------------------------------------------- coagulation
  double coag_in[NAER];
  if (a.do_coag) {
    double nsv[NMODE], asv[NAER][NMODE];
    if (DIAG) {
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        nsv[m] = s.num[m];
#pragma unroll
        for (int x = 0; x < NAER; ++x)
          asv[x][m] = s.aer[x][m];
      }
    }
    double cc[12];
    if (PRECOAG) {
      // coefficients from pair_kernel
#pragma unroll
      for (int k = 0; k < 12; ++k)
        cc[k] = cc_pre[k * cc_stride];
    } else {
      const CoagTables T = {kCoagBm0ij, kCoagBm3i, kCoagBm0};
      coag_all_coefs(C, T, temp, pmid, aircon, dgn_awet, wetdens, cc);
    }
    coagulation(dtsub, cc, s, coag_in);
    if (DIAG) {
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        dncoag[m] = s.num[m] - nsv[m];
#pragma unroll
        for (int x = 0; x < NAER; ++x)
          dcoag[x][m] = s.aer[x][m] - asv[x][m];
      }
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        dg->t[3][num_i31(m)] += ((0.0 + dncoag[m]) / (1.0 * deltat)) * afrac;
#pragma unroll
        for (int x = 0; x < NAER; ++x) {
          const int slot = K::aer_slot(x, m);
          if (slot >= 0)
            dg->t[3][pop_to_i31(slot)] += ((0.0 + dcoag[x][m]) / (K::fcvt_aer(x) * deltat)) * afrac;
        }
      }
    }
  } else {
#pragma unroll
    for (int x = 0; x < NAER; ++x)
      coag_in[x] = 0.0;
  }

  // ----------------------------------------------------------- aging
  if (DIAG) {
    aging(C, a.nmono, dgn_a_pc, s, dncond, dncoag, dcond, dcoag, coag_in);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      if (a.do_cond)
        dg->t[0][num_i31(m)] += ((0.0 + dncond[m]) / (1.0 * deltat)) * afrac;
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0 && a.do_cond)
          dg->t[0][pop_to_i31(slot)] += ((0.0 + dcond[x][m]) / (K::fcvt_aer(x) * deltat)) * afrac;
      }
    }
  } else {
    // Only the primary-carbon condensation gains of SO4/SOA enter the aging
    // fraction; the other increments are bookkeeping for diagnostics.
    double dn_c[NMODE] = {0, 0, 0, 0}, dn_g[NMODE] = {0, 0, 0, 0};
    double dc[NAER][NMODE], dq[NAER][NMODE];
#pragma unroll
    for (int x = 0; x < NAER; ++x)
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        dc[x][m] = 0.0;
        dq[x][m] = 0.0;
      }
    dc[1][3] = cond_so4_pc;
    dc[0][3] = cond_soa_pc;
    aging(C, a.nmono, dgn_a_pc, s, dn_c, dn_g, dc, dq, coag_in);
  }
}

// Whole clear subarea in one thread: part 1, the SOA loop inline, part 2.
// Returns the SOA sub-step count.
template <bool DIAG>
__device__ __forceinline__ int clear_subarea(const StepArgs &a, double deltat, double temp,
                                             double pmid, double zmid, double pblh,
                                             double relhum, const double (&dgn_a)[NMODE],
                                             const double (&dgn_awet)[NMODE],
                                             const double (&wetdens)[NMODE],
                                             const double (&qgas1)[2], Sub &s, Diag *dg,
                                             double afrac) {
  ClearMid cm;
  double uptk0[NMODE], rate[NMODE] = {0, 0, 0, 0};
  if (a.do_cond) {
    double gas_diffus, freepath;
    h2so4_diffusivity(temp, pmid, gas_diffus, freepath);
    uptake_rates(c_k, gas_diffus, freepath, dgn_awet, rate);
  }
  clear_prefix<DIAG>(a, deltat, temp, pmid, rate, qgas1, s, cm, uptk0);
  int niter = 0;
  if (a.do_cond)
    niter = soa_exchange((double)(int)(deltat / 1), temp, pmid, s, uptk0);
  clear_suffix<DIAG, false>(a, deltat, temp, pmid, zmid, pblh, relhum, dgn_a[3], dgn_awet, wetdens, cm, s,
                     dg, afrac, nullptr, 0);
  return niter;
}

// Tendencies of the 25 cloud-borne populations from their outgoing grid
// means oc (vmr) and incoming values ac (mmr).
__device__ __forceinline__ void store_cloudborne(const StepArgs &a, long long c,
                                                 const double (&oc)[NPOP],
                                                 const double (&ac)[NPOP]) {
  const StepConsts &C = c_k;
  const double dt = a.dt;
  double *const *out = a.out;
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    out[MAM4B_OUT_TEND + 27 + p][c] = (oc[p] * C.to_mmr[2 + p] - ac[p]) / dt;
}

// Tendencies of the gases and the 25 interstitial populations.
__device__ __forceinline__ void store_interstitial(const StepArgs &a, long long c, double o_h2so4,
                                                   double o_soag, const double (&oi)[NPOP],
                                                   double h2so4, double soag,
                                                   const double (&ai)[NPOP]) {
  const StepConsts &C = c_k;
  const double dt = a.dt;
  double *const *out = a.out;
  out[MAM4B_OUT_TEND + 0][c] = (o_h2so4 * C.to_mmr[0] - h2so4) / dt;
  out[MAM4B_OUT_TEND + 1][c] = (o_soag * C.to_mmr[1] - soag) / dt;
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    out[MAM4B_OUT_TEND + 2 + p][c] = (oi[p] * C.to_mmr[2 + p] - ai[p]) / dt;
}

__device__ __forceinline__ void store_outputs(const StepArgs &a, long long c, double o_h2so4,
                                              double o_soag, const double (&oi)[NPOP],
                                              const double (&oc)[NPOP], double h2so4, double soag,
                                              const double (&ai)[NPOP], const double (&ac)[NPOP]) {
  store_interstitial(a, c, o_h2so4, o_soag, oi, h2so4, soag, ai);
  store_cloudborne(a, c, oc, ac);
}

// Per-cell state after calcsize and water uptake (modal_aero_calcsize_sub,
// modal_aero_water_uptake_dr), in amicphys units where amicphys reads it.
struct Front {
  double temp, pmid, zm, qv, cld, h2so4, soag, pblh;
  double ai[NPOP], ac[NPOP];          // populations as passed in (mmr)
  double dgn_a[NMODE], dgn_awet[NMODE], wetdens[NMODE];
  double qi[NPOP], qc[NPOP];          // after the calcsize update (vmr)
  double g_h2so4, g_soag;             // gases (vmr)
  double relhumgcm;
};

// Loads the cell, checks it, runs calcsize and water uptake, writes the
// size outputs and prepares the amicphys inputs: the part of
// modal_aero_amicphys_intr (mam4_amicphys.hpp:2120-2260) before the
// subarea loop, with q_pregaschem = q_precldchem = qq and
// qqcw_precldchem = qqcw. Without WU the wet sizes are read back from the
// outputs, written by size_kernel and mode_kernel.
template <bool WU>
__device__ __forceinline__ void cell_front(const StepArgs &a, const long long c, Front &f) {
  const StepConsts &C = c_k;
  f.temp = __ldg(a.in[MAM4B_IN_T] + c);
  f.pmid = __ldg(a.in[MAM4B_IN_P] + c);
  f.zm = __ldg(a.in[MAM4B_IN_ZM] + c);
  f.qv = __ldg(a.in[MAM4B_IN_QV] + c);
  f.cld = __ldg(a.in[MAM4B_IN_CLD] + c);
  f.h2so4 = __ldg(a.in[MAM4B_IN_H2SO4] + c);
  f.soag = __ldg(a.in[MAM4B_IN_SOAG] + c);
  f.pblh = __ldg(a.pblh + c / a.nlev);
  const double dt = a.dt;
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    f.ai[p] = __ldg(a.in[MAM4B_IN_AER_I + p] + c);
    f.ac[p] = __ldg(a.in[MAM4B_IN_AER_C + p] + c);
  }
  {
    double chk = f.temp + f.pmid + f.zm + f.qv + f.cld + f.h2so4 + f.soag + f.pblh;
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      chk += f.ai[p] + f.ac[p];
    if (!isfinite(chk))
      atomicOr(a.flags, MAM4B_FLAG_NONFINITE_INPUT);
  }
  double pt_i[NPOP], pt_c[NPOP];
  calcsize(C, f.ai, f.ac, dt, f.dgn_a, pt_i, pt_c);
  double wetdens_wu[NMODE];
  if (WU) {
    double qaerwat[NMODE];
    water_uptake(C, f.ai, f.qv, f.temp, f.pmid, f.cld, f.dgn_a, f.dgn_awet, qaerwat, wetdens_wu);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      a.out[MAM4B_OUT_DGN_A + m][c] = f.dgn_a[m];
      a.out[MAM4B_OUT_DGN_AWET + m][c] = f.dgn_awet[m];
      a.out[MAM4B_OUT_WETDENS + m][c] = wetdens_wu[m];
      a.out[MAM4B_OUT_QAERWAT + m][c] = qaerwat[m];
    }
  } else {
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      f.dgn_awet[m] = a.out[MAM4B_OUT_DGN_AWET + m][c];
      wetdens_wu[m] = a.out[MAM4B_OUT_WETDENS + m][c];
    }
  }
  // calcsize tendencies applied for one step, then amicphys units
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    f.qi[p] = dmax(0.0, dmax(0.0, f.ai[p] + pt_i[p] * dt) * C.to_vmr[2 + p]);
    f.qc[p] = dmax(0.0, dmax(0.0, f.ac[p] + pt_c[p] * dt) * C.to_vmr[2 + p]);
  }
  f.g_h2so4 = dmax(0.0, f.h2so4 * C.to_vmr[0]);
  f.g_soag = dmax(0.0, f.soag * C.to_vmr[1]);
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    f.wetdens[m] = dmax(1000.0, wetdens_wu[m]);
  const double epsqs = 0.018016 / 0.028966;
  const double tc = f.temp - 273.15;
  const double ew = 610.94 * exp(17.625 * tc / (234.04 + tc));
  const double ev_sat = 1.00071 * exp(4.5e-8 * f.pmid) * ew;
  const double qv_sat = epsqs * ev_sat / (f.pmid - (1 - epsqs) * ev_sat);
  f.relhumgcm = dmax(0.0, dmin(1.0, f.qv / qv_sat));
}

// Renaming of a cloudy (sub)area, interstitial si and cloud-borne sc,
// weighted by f; adds the renaming diagnostics when DIAG.
template <bool DIAG>
__device__ __forceinline__ void cloudy_rename(const StepArgs &a, Sub &si, Sub &sc, double f,
                                              Diag *dg) {
  const StepConsts &C = c_k;
  si.gas[0] = si.gas[1] = sc.gas[0] = sc.gas[1] = 0.0;
  double nsv_i[NMODE], nsv_c[NMODE], asv_i[NAER][NMODE], asv_c[NAER][NMODE];
  if (DIAG) {
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      nsv_i[m] = si.num[m];
      nsv_c[m] = sc.num[m];
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        asv_i[x][m] = si.aer[x][m];
        asv_c[x][m] = sc.aer[x][m];
      }
    }
  }
  if (a.do_rename) {
    const double zero7[NAER] = {0, 0, 0, 0, 0, 0, 0};
    rename_subarea<true>(C, si, sc, zero7, zero7);
  }
  if (DIAG && a.do_rename) {
    const double dt = a.dt;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      const int ln = num_i31(m);
      dg->t[1][ln] += ((0.0 + (si.num[m] - nsv_i[m])) / (1.0 * dt)) * f;
      dg->cw[ln] += ((0.0 + (sc.num[m] - nsv_c[m])) / (1.0 * dt)) * f;
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0) {
          dg->t[1][pop_to_i31(slot)] +=
              ((0.0 + (si.aer[x][m] - asv_i[x][m])) / (K::fcvt_aer(x) * dt)) * f;
          dg->cw[pop_to_i31(slot)] +=
              ((0.0 + (sc.aer[x][m] - asv_c[x][m])) / (K::fcvt_aer(x) * dt)) * f;
        }
      }
    }
  }
}

// Cloudy grid cell (cloud fraction > 0.999): renaming only.
template <bool DIAG>
__device__ __forceinline__ void cloudy_cell(const StepArgs &a, const Front &f, double &o_h2so4,
                                            double &o_soag, double (&oi)[NPOP],
                                            double (&oc)[NPOP], Diag *dg) {
  Sub si, sc;
  load_sub_plain(si, f.qi);
  load_sub_plain(sc, f.qc);
  const double w = 1.0;
  cloudy_rename<DIAG>(a, si, sc, w, dg);
  o_soag = dmax(0.0, 0.0 + f.g_soag * w);
  o_h2so4 = dmax(0.0, 0.0 + f.g_h2so4 * w);
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    oi[K::numslot(m)] = dmax(0.0, 0.0 + (si.num[m] / 1.0) * w);
    oc[K::numslot(m)] = 0.0 + (sc.num[m] / 1.0) * w;
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      const int slot = K::aer_slot(x, m);
      if (slot >= 0) {
        oi[slot] = dmax(0.0, 0.0 + (si.aer[x][m] / K::fcvt_aer(x)) * w);
        oc[slot] = 0.0 + (sc.aer[x][m] / K::fcvt_aer(x)) * w;
      }
    }
  }
}

// Partly cloudy grid cell, set-up of both subareas and the cloudy one
// (jsub 2, renaming only): the clear subarea's incoming state s, its gases
// and relative humidity, and the cloudy subarea's contributions to the
// grid means (ci interstitial, cg gases SOAG/H2SO4, oc cloud-borne).
// Partition factors: get_partition_factors (mam4_amicphys.hpp:414-449).
template <bool DIAG>
__device__ __forceinline__ void partly_cloudy_setup(const StepArgs &a, const Front &f, Sub &s,
                                                    double (&gcl)[2], double &rhc,
                                                    double (&ci)[NPOP], double (&cg)[2],
                                                    double (&oc)[NPOP], Diag *dg) {
  const StepConsts &C = c_k;
  const double fcldy = f.cld, fclea = 1.0 - fcldy;
  double fn_c[NMODE], fn_y[NMODE], fm_c[NMODE], fm_y[NMODE];
  auto part = [&](double q_i, double q_c, double &fc, double &fy) {
    const double cldbrn_cldy = q_c / fcldy;
    const double intrst_cldy = dmax(0.0, ((q_i + q_c) - cldbrn_cldy));
    const double intrst_clea = (q_i - fcldy * intrst_cldy) / fclea;
    double r = dmax(1.e-35, intrst_clea * fclea) / dmax(1.e-35, q_i);
    r = dmax(0.0, dmin(1.0, r));
    fc = r / fclea;
    fy = (1 - r) / fcldy;
  };
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    part(f.qi[K::numslot(m)], f.qc[K::numslot(m)], fn_c[m], fn_y[m]);
    double si_ = 0.0, sc_ = 0.0;
#pragma unroll
    for (int k = 0; k < K::nspec(m); ++k) {
      si_ = si_ + f.qi[K::spec0(m) + k];
      sc_ = sc_ + f.qc[K::spec0(m) + k];
    }
    part(si_, sc_, fm_c[m], fm_y[m]);
  }
  // gases: clear keeps the grid mean, cloudy gets the remainder
  double gcy[2];
  gcl[0] = f.g_soag;
  gcl[1] = f.g_h2so4;
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    gcy[g] = (gcl[g] - fclea * gcl[g]) / fcldy;
    if (gcy[g] < 0) {
      gcy[g] = 0;
      gcl[g] = gcl[g] / fclea;
    }
  }
  rhc = bound(0.0, 1.0, (f.relhumgcm - fcldy) / fclea);
  {
    Sub si, sc;
    load_sub(si, f.qi, fn_y, fm_y);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      sc.num[m] = (f.qc[K::numslot(m)] / fcldy) * 1;
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        sc.aer[x][m] = (slot >= 0) ? (f.qc[slot] / fcldy) * K::fcvt_aer(x) : 0.0;
      }
    }
    cloudy_rename<DIAG>(a, si, sc, fcldy, dg);
    cg[0] = gcy[0] * fcldy;
    cg[1] = gcy[1] * fcldy;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      ci[K::numslot(m)] = (si.num[m] / 1.0) * fcldy;
      oc[K::numslot(m)] = (0.0 + 0.0 * fclea) + (sc.num[m] / 1.0) * fcldy;
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0) {
          ci[slot] = (si.aer[x][m] / K::fcvt_aer(x)) * fcldy;
          oc[slot] = (0.0 + 0.0 * fclea) + (sc.aer[x][m] / K::fcvt_aer(x)) * fcldy;
        }
      }
    }
  }
  load_sub(s, f.qi, fn_c, fm_c);
  s.gas[0] = gcl[0] * C.fcvt_soag;
  s.gas[1] = gcl[1] * 1.0;
}

// One grid cell start to end in one thread (modal_aero_amicphys_intr,
// mam4_amicphys.hpp:2120-2376): the diagnostics path, and the whole step
// when condensation is off (no SOA loop to pipeline).
template <bool DIAG>
__device__ __forceinline__ void cell_step(const StepArgs &a, const long long c) {
  const StepConsts &C = c_k;
  Front f;
  cell_front<true>(a, c, f);
  const double dt = a.dt;
  Diag dgv;
  Diag *dg = DIAG ? &dgv : nullptr;
  if (DIAG) {
#pragma unroll
    for (int k = 0; k < NQTEND; ++k)
#pragma unroll
      for (int i = 0; i < 31; ++i)
        dgv.t[k][i] = 0.0;
#pragma unroll
    for (int i = 0; i < 31; ++i)
      dgv.cw[i] = 0.0;
  }
  // outgoing grid-cell means (amicphys units): gases, interstitial, cloud
  double o_h2so4, o_soag, oi[NPOP], oc[NPOP];
  const double fsoag = C.fcvt_soag;
  const bool map_gas = a.do_cond || a.do_newnuc;
  const double qgas1[2] = {f.g_soag * fsoag, f.g_h2so4 * 1.0};

  if (f.cld > 0.999) {
    cloudy_cell<DIAG>(a, f, o_h2so4, o_soag, oi, oc, dg);
  } else if (f.cld < 1.0e-5) {
    // clear grid cell: the subarea is the grid mean
    Sub s;
    load_sub_plain(s, f.qi);
    s.gas[0] = f.g_soag * fsoag;
    s.gas[1] = f.g_h2so4 * 1.0;
    const int niter = clear_subarea<DIAG>(a, dt, f.temp, f.pmid, f.zm, f.pblh, f.relhumgcm,
                                                f.dgn_a, f.dgn_awet, f.wetdens, qgas1, s, dg, 1.0);
    if (niter > 1000)
      atomicOr(a.flags, MAM4B_FLAG_SOA_NITER_LIMIT);
    const double w = 1.0 - 0.0;
    o_soag = dmax(0.0, 0.0 + (map_gas ? s.gas[0] / fsoag : f.g_soag) * w);
    o_h2so4 = dmax(0.0, 0.0 + (map_gas ? s.gas[1] / 1.0 : f.g_h2so4) * w);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] = dmax(0.0, 0.0 + (s.num[m] / 1.0) * w);
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0)
          oi[slot] = dmax(0.0, 0.0 + (s.aer[x][m] / K::fcvt_aer(x)) * w);
      }
    }
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      oc[p] = f.qc[p];
  } else {
    // partly cloudy grid cell: cloudy subarea first (its contributions are
    // added after the clear subarea's, as in the reference's jsub order)
    const double fclea = 1.0 - f.cld;
    Sub s;
    double gcl[2], rhc, ci[NPOP], cg[2];
    partly_cloudy_setup<DIAG>(a, f, s, gcl, rhc, ci, cg, oc, dg);
    Diag dclear;
    Diag *dcp = DIAG ? &dclear : nullptr;
    if (DIAG) {
#pragma unroll
      for (int k = 0; k < NQTEND; ++k)
#pragma unroll
        for (int i = 0; i < 31; ++i)
          dclear.t[k][i] = 0.0;
    }
    const int niter = clear_subarea<DIAG>(a, dt, f.temp, f.pmid, f.zm, f.pblh, rhc, f.dgn_a,
                                                f.dgn_awet, f.wetdens, qgas1, s, dcp, fclea);
    if (niter > 1000)
      atomicOr(a.flags, MAM4B_FLAG_SOA_NITER_LIMIT);
    if (DIAG) {
      // jsub 1 then jsub 2: t = (0 + clear) + cloudy
#pragma unroll
      for (int k = 0; k < NQTEND; ++k)
#pragma unroll
        for (int i = 0; i < 31; ++i)
          dgv.t[k][i] = dclear.t[k][i] + dgv.t[k][i];
    }
    o_soag = dmax(0.0, (0.0 + (map_gas ? s.gas[0] / fsoag : gcl[0]) * fclea) + cg[0]);
    o_h2so4 = dmax(0.0, (0.0 + (map_gas ? s.gas[1] / 1.0 : gcl[1]) * fclea) + cg[1]);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] = dmax(0.0, (0.0 + (s.num[m] / 1.0) * fclea) + ci[K::numslot(m)]);
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0)
          oi[slot] = dmax(0.0, (0.0 + (s.aer[x][m] / K::fcvt_aer(x)) * fclea) + ci[slot]);
      }
    }
  }

  store_outputs(a, c, o_h2so4, o_soag, oi, oc, f.h2so4, f.soag, f.ai, f.ac);
  if (DIAG) {
#pragma unroll
    for (int k = 0; k < NQTEND; ++k)
#pragma unroll
      for (int i = 0; i < 31; ++i)
        if (a.diag[k * 31 + i])
          a.diag[k * 31 + i][c] = dgv.t[k][i];
#pragma unroll
    for (int i = 0; i < 31; ++i)
      if (a.diag[4 * 31 + i])
        a.diag[4 * 31 + i][c] = dgv.cw[i];
  }
}

// ---- the step with the chemistry that precedes amicphys, one thread per
// cell: calcsize and water uptake, the calcsize update, then gas-phase
// chemistry (gas_phase_chemistry.hpp:40) and aqueous chemistry
// (mo_setsox.hpp:944) on the cell's 31 tracers, then amicphys with the three
// states the chemistry leaves: before gas chemistry (q_pregaschem), before
// cloud chemistry (q_precldchem, qqcw_precldchem) and after it (qq, qqcw).
struct ChemArgs {
  const double *in;  // [MAM4B_CHEM_NIN][ld]
  double *out;       // [MAM4B_CHEM_NOUT][ld]
  size_t ld;
};

// amicphys-unit states before the chemistry, clipped at zero as amicphys
// clips its inputs (mam4_amicphys.hpp:2258-2267)
struct ChemPre {
  double g1[2];               // SOAG, H2SO4 before gas chemistry
  double g2[2];               // SOAG, H2SO4 before cloud chemistry
  double qi2[NPOP], qc2[NPOP];  // populations before cloud chemistry
};

// Renaming in a cloudy (sub)area whose populations grew by cloud chemistry:
// the growth increments of the aitken mode are the change from the
// before-cloud-chemistry state (mam4_amicphys.hpp:1440-1455; no
// condensation in a cloudy subarea).
__device__ __forceinline__ void cloudy_rename_grown(const StepArgs &a, Sub &si, Sub &sc,
                                                    const Sub &si2, const Sub &sc2) {
  const StepConsts &C = c_k;
  si.gas[0] = si.gas[1] = sc.gas[0] = sc.gas[1] = 0.0;
  if (!a.do_rename)
    return;
  double gi[NAER], gc[NAER];
#pragma unroll
  for (int x = 0; x < NAER; ++x) {
    gi[x] = (si.aer[x][1] - si2.aer[x][1]) / 1 + 0.0;
    gc[x] = (sc.aer[x][1] - sc2.aer[x][1]) / 1;
  }
  rename_subarea<true>(C, si, sc, gi, gc);
}

// Cloudy grid cell (cloud fraction > 0.999) after chemistry.
__device__ __forceinline__ void cloudy_cell_chem(const StepArgs &a, const Front &f,
                                                 const ChemPre &cp, double &o_h2so4,
                                                 double &o_soag, double (&oi)[NPOP],
                                                 double (&oc)[NPOP]) {
  Sub si, sc;
  load_sub_plain(si, f.qi);
  load_sub_plain(sc, f.qc);
  {
    Sub si2, sc2;
    load_sub_plain(si2, cp.qi2);
    load_sub_plain(sc2, cp.qc2);
    cloudy_rename_grown(a, si, sc, si2, sc2);
  }
  const double w = 1.0;
  o_soag = dmax(0.0, 0.0 + f.g_soag * w);
  o_h2so4 = dmax(0.0, 0.0 + f.g_h2so4 * w);
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    oi[K::numslot(m)] = dmax(0.0, 0.0 + (si.num[m] / 1.0) * w);
    oc[K::numslot(m)] = 0.0 + (sc.num[m] / 1.0) * w;
#pragma unroll
    for (int x = 0; x < NAER; ++x) {
      const int slot = K::aer_slot(x, m);
      if (slot >= 0) {
        oi[slot] = dmax(0.0, 0.0 + (si.aer[x][m] / K::fcvt_aer(x)) * w);
        oc[slot] = 0.0 + (sc.aer[x][m] / K::fcvt_aer(x)) * w;
      }
    }
  }
}

// Partly cloudy grid cell after chemistry (set_subarea_gases_and_aerosols,
// mam4_amicphys.hpp:679-911): the interstitial partition factors come from
// the before-cloud-chemistry state and split both it and the current one;
// gases keep their before-cloud-chemistry value in the clear subarea and
// the cloudy subarea takes the remainder of the current grid mean
// (compute_qsub_from_gcm_and_qsub_of_other_subarea, :367-408).
__device__ __forceinline__ void partly_cloudy_setup_chem(const StepArgs &a, const Front &f,
                                                         const ChemPre &cp, Sub &s,
                                                         double (&gcl)[2], double &rhc,
                                                         double (&ci)[NPOP], double (&cg)[2],
                                                         double (&oc)[NPOP]) {
  const StepConsts &C = c_k;
  const double fcldy = f.cld, fclea = 1.0 - fcldy;
  double fn_c[NMODE], fn_y[NMODE], fm_c[NMODE], fm_y[NMODE];
  auto part = [&](double q_i, double q_c, double &fc, double &fy) {
    const double cldbrn_cldy = q_c / fcldy;
    const double intrst_cldy = dmax(0.0, ((q_i + q_c) - cldbrn_cldy));
    const double intrst_clea = (q_i - fcldy * intrst_cldy) / fclea;
    double r = dmax(1.e-35, intrst_clea * fclea) / dmax(1.e-35, q_i);
    r = dmax(0.0, dmin(1.0, r));
    fc = r / fclea;
    fy = (1 - r) / fcldy;
  };
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    part(cp.qi2[K::numslot(m)], cp.qc2[K::numslot(m)], fn_c[m], fn_y[m]);
    double si_ = 0.0, sc_ = 0.0;
#pragma unroll
    for (int k = 0; k < K::nspec(m); ++k) {
      si_ = si_ + cp.qi2[K::spec0(m) + k];
      sc_ = sc_ + cp.qc2[K::spec0(m) + k];
    }
    part(si_, sc_, fm_c[m], fm_y[m]);
  }
  const double g3[2] = {f.g_soag, f.g_h2so4};
  double gcy[2];
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    gcl[g] = cp.g2[g];
    gcy[g] = (g3[g] - fclea * gcl[g]) / fcldy;
    if (gcy[g] < 0) {
      gcy[g] = 0;
      gcl[g] = g3[g] / fclea;
    }
  }
  rhc = bound(0.0, 1.0, (f.relhumgcm - fcldy) / fclea);
  {
    Sub si, sc, si2, sc2;
    load_sub(si, f.qi, fn_y, fm_y);
    load_sub(si2, cp.qi2, fn_y, fm_y);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      sc.num[m] = (f.qc[K::numslot(m)] / fcldy) * 1;
      sc2.num[m] = (cp.qc2[K::numslot(m)] / fcldy) * 1;
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        sc.aer[x][m] = (slot >= 0) ? (f.qc[slot] / fcldy) * K::fcvt_aer(x) : 0.0;
        sc2.aer[x][m] = (slot >= 0) ? (cp.qc2[slot] / fcldy) * K::fcvt_aer(x) : 0.0;
      }
    }
    cloudy_rename_grown(a, si, sc, si2, sc2);
    cg[0] = gcy[0] * fcldy;
    cg[1] = gcy[1] * fcldy;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      ci[K::numslot(m)] = (si.num[m] / 1.0) * fcldy;
      oc[K::numslot(m)] = (0.0 + 0.0 * fclea) + (sc.num[m] / 1.0) * fcldy;
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0) {
          ci[slot] = (si.aer[x][m] / K::fcvt_aer(x)) * fcldy;
          oc[slot] = (0.0 + 0.0 * fclea) + (sc.aer[x][m] / K::fcvt_aer(x)) * fcldy;
        }
      }
    }
  }
  load_sub(s, f.qi, fn_c, fm_c);
  s.gas[0] = gcl[0] * C.fcvt_soag;
  s.gas[1] = gcl[1] * 1.0;
}

// amicphys tracer index of the gas-chemistry gases O3, H2O2, SO2, DMS
__device__ __forceinline__ constexpr int chem_gas_i31(int g) { return g < 2 ? g : g + 1; }

// The chemistry of a cell between its front (calcsize, water uptake, the
// calcsize update) and amicphys: gas-phase chemistry, then aqueous
// chemistry, on the cell's 31 tracers in vmr; cp receives the states before
// each, f the state after both (clipped, as amicphys reads it), and the
// four chemistry gases' tendencies are written.
__device__ __forceinline__ void run_chemistry(const StepArgs &a, const ChemArgs &ch,
                                              const long long c, Front &f, ChemPre &cp) {
  const StepConsts &C = c_k;
  const double dt = a.dt;
  auto CIN = [&](int k) { return __ldg(ch.in + (size_t)k * ch.ld + c); };
  double qq[31], qqcw[31];
  double gas_in[4];
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const int i = chem_gas_i31(g);
    gas_in[g] = CIN(MAM4B_CHEM_IN_O3 + g);
    qq[i] = gas_in[g] * (K::mw_dry_air / K::adv_mass(i));
    qqcw[i] = 0.0;
  }
  qq[2] = f.h2so4 * C.to_vmr[0];
  qq[5] = f.soag * C.to_vmr[1];
  qqcw[2] = qqcw[5] = 0.0;
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    qq[6 + p] = f.qi[p];
    qqcw[6 + p] = f.qc[p];
  }
  cp.g1[0] = dmax(0.0, qq[5]);
  cp.g1[1] = dmax(0.0, qq[2]);
  {  // gas-phase chemistry
    double ext[gch::kExt], inv[gch::kInv];
#pragma unroll
    for (int e = 0; e < gch::kExt; ++e)
      ext[e] = CIN(MAM4B_CHEM_IN_EXTFRC + e);
#pragma unroll
    for (int i = 0; i < gch::kInv; ++i)
      inv[i] = CIN(MAM4B_CHEM_IN_INV + i);
    const double *het_c = ch.in + (size_t)MAM4B_CHEM_IN_HET * ch.ld + c;
    const size_t ld = ch.ld;
    auto het = [het_c, ld](int t) { return __ldg(het_c + (size_t)t * ld); };
    gch::gas_chemistry_cell(f.temp, dt, CIN(MAM4B_CHEM_IN_PHOTO), ext, inv, het, qq);
  }
  cp.g2[0] = dmax(0.0, qq[5]);
  cp.g2[1] = dmax(0.0, qq[2]);
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    cp.qi2[p] = dmax(0.0, qq[6 + p]);
    cp.qc2[p] = dmax(0.0, qqcw[6 + p]);
  }
  {  // cloud chemistry; the total air density is the invariant density of air
    double dso4[3], dh2so4[3];
    sox::setsox_cell(dt, f.pmid, f.temp, CIN(MAM4B_CHEM_IN_LWC), f.cld,
                     CIN(MAM4B_CHEM_IN_CLDNUM), CIN(MAM4B_CHEM_IN_INV + 0), qq, qqcw, dso4,
                     dh2so4);
  }
  f.g_soag = dmax(0.0, qq[5]);
  f.g_h2so4 = dmax(0.0, qq[2]);
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    f.qi[p] = dmax(0.0, qq[6 + p]);
    f.qc[p] = dmax(0.0, qqcw[6 + p]);
  }
  // the gases amicphys does not map keep the chemistry's result
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    const int i = chem_gas_i31(g);
    ch.out[(size_t)(MAM4B_CHEM_OUT_TEND + g) * ch.ld + c] =
        (qq[i] * (K::adv_mass(i) / K::mw_dry_air) - gas_in[g]) / dt;
  }
}

// First half of the pipelined step (condensation on, no diagnostics): the
// cell's front; cloudy cells finish here; every other cell sets up its
// clear subarea (and, when partly cloudy, runs the cloudy one), runs the
// clear subarea up to the SOA loop and hands the state at that point to the
// solver and the post kernel. The clear-subarea part runs converged for
// clear and partly cloudy cells alike.
// With CHEM the cell's chemistry runs between its front and amicphys
// (run_chemistry), and the subarea set-up takes the pre-chemistry states;
// the post kernel needs nothing else, as everything it reads of the cell's
// state comes through the hand-off.
// The per-particle H2SO4 uptake rate of mode M of cell c as the FP64 step
// computes it: FP64 water uptake of the mode from the cell's inputs, the
// calcsize dry diameter and the relative humidity of the size stage, then
// uptake_rate_mode. The mixed step (FP32 rates from the mode stage) uses
// it where a decision of the SOA loop sits at its threshold, so that the
// decision is the FP64 step's.
template <int M>
__device__ double rate_fp64_mode(const StepArgs &a, const long long c) {
  const StepConsts &C = c_k;
  const size_t n = (size_t)a.ncell;
  double sp[7];
#pragma unroll
  for (int s = 0; s < 7; ++s)
    sp[s] = (s < K::nspec(M)) ? __ldg(a.in[MAM4B_IN_AER_I + K::spec0(M) + (s < K::nspec(M) ? s : 0)] + c) : 0.0;
  double dgn_awet, qaerwat, wetdens;
  water_uptake_mode<M>(C, sp, a.aux[AUX_RH * n + c], a.out[MAM4B_OUT_DGN_A + M][c], dgn_awet,
                       qaerwat, wetdens);
  return uptake_rate_mode(C, M, a.aux[AUX_GDIFF * n + c], a.aux[AUX_FPATH * n + c], dgn_awet);
}
__device__ __noinline__ double rate_fp64(const StepArgs &a, const long long c, int m) {
  switch (m) {
  case 0: return rate_fp64_mode<0>(a, c);
  case 1: return rate_fp64_mode<1>(a, c);
  case 2: return rate_fp64_mode<2>(a, c);
  default: return rate_fp64_mode<3>(a, c);
  }
}

// The SOA loop skips a mode, and zeroes its SOA, when its uptake rate is
// not above 1e-15 (gasaerexch_soaexch.hpp:189-193). With FP32 rates
// (relative error well below 1e-5) a rate within 1e-4 of that threshold may
// fall on the other side of it than the FP64 step's, so such modes take
// the FP64 rate instead (a few cells in 10^4).
__device__ __forceinline__ void guard_soa_threshold(const StepArgs &a, const long long c,
                                                    double temp, double pmid, const Sub &s,
                                                    double (&rate)[NMODE], ClearMid &cm,
                                                    double (&uptk0)[NMODE]) {
  const double aircon = pmid / (8314.46759100000 * temp);
#pragma unroll
  for (int k = 0; k < NMODE; ++k) {
    if (fabs(uptk0[k] - 1.0e-15) <= 1.0e-4 * 1.0e-15) {
      rate[k] = rate_fp64(a, c, k);
      cm.uptk1[k] = rate[k] * (s.num[k] * aircon);
      uptk0[k] = cm.uptk1[k] * 0.81;
    }
  }
}

template <class Src>
__device__ __forceinline__ void cell_finish(const StepArgs &a, const long long c, double temp,
                                            double pmid, double zm, double cld, double pblh,
                                            double relhum, double dgn_pc, Sub &s, ClearMid &cm,
                                            const Src &src);
// cell_finish's late inputs held in registers (the fused path of pre)
struct FinishRegs {
  const double (&ci_)[NPOP];
  const double (&cg_)[2];
  const double (&ai_)[NPOP];
  double h2so4_, soag_;
  __device__ double ci(int p) const { return ci_[p]; }
  __device__ double cg(int g) const { return cg_[g]; }
  __device__ double ai(int p) const { return ai_[p]; }
  __device__ double h2so4() const { return h2so4_; }
  __device__ double soag() const { return soag_; }
};
template <int SOA, class State>
__device__ __forceinline__ bool soa_pass(State &st);

template <bool CHEM, bool MIXED = false, bool FUSE = false>
__device__ __forceinline__ void cell_pre(const StepArgs &a, const ChemArgs &ch,
                                         const long long c) {
  const StepConsts &C = c_k;
  Front f;
  cell_front<false>(a, c, f);
  ChemPre cp;
  if constexpr (CHEM)
    run_chemistry(a, ch, c, f, cp);
  const double dt = a.dt;
  const double fsoag = C.fcvt_soag;
  if (f.cld > 0.999) {
    double o_h2so4, o_soag, oi[NPOP], oc[NPOP];
    if constexpr (CHEM)
      cloudy_cell_chem(a, f, cp, o_h2so4, o_soag, oi, oc);
    else
      cloudy_cell<false>(a, f, o_h2so4, o_soag, oi, oc, nullptr);
    store_outputs(a, c, o_h2so4, o_soag, oi, oc, f.h2so4, f.soag, f.ai, f.ac);
    return;
  }
  const bool partly = !(f.cld < 1.0e-5);
  Sub s;
  double rh, oc[NPOP], ci[NPOP], cg[2] = {0.0, 0.0};
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    ci[p] = 0.0;
  if (!partly) {
    load_sub_plain(s, f.qi);
    s.gas[0] = f.g_soag * fsoag;
    s.gas[1] = f.g_h2so4 * 1.0;
    rh = f.relhumgcm;
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      oc[p] = f.qc[p];
  } else {
    double gcl[2];
    if constexpr (CHEM)
      partly_cloudy_setup_chem(a, f, cp, s, gcl, rh, ci, cg, oc);
    else
      partly_cloudy_setup<false>(a, f, s, gcl, rh, ci, cg, oc, nullptr);
  }
  double qgas1[2] = {f.g_soag * fsoag, f.g_h2so4 * 1.0};
  if constexpr (CHEM) {
    qgas1[0] = cp.g1[0] * fsoag;
    qgas1[1] = cp.g1[1] * 1.0;
  }
  ClearMid cm;
  double uptk0[NMODE], rate[NMODE];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    rate[k] = a.aux[(AUX_RATE + k) * (size_t)a.ncell + c];
  clear_prefix<false>(a, dt, f.temp, f.pmid, rate, qgas1, s, cm, uptk0);
  if constexpr (MIXED) {
    if (a.do_cond)
      guard_soa_threshold(a, c, f.temp, f.pmid, s, rate, cm, uptk0);
  }

  // queue the cell: solver state and hand-off at the start of the SOA loop
  SoaState st;
  soa_init(st, (double)(int)(dt / 1), f.temp, f.pmid, s, uptk0);
  const double first_rate = soa_first_rate(st) * st.dtfull;
  if constexpr (FUSE) {
    // a short loop (first sub-step at least 1/inline_scale of the step)
    // runs here and the cell finishes without the hand-off, with the same
    // arithmetic as the solver and post kernels
    if (first_rate <= 0.05 * a.inline_scale) {
      while (soa_pass<MIXED ? 1 : 0>(st)) {
      }
      if (st.niter > 1000)
        atomicOr(a.flags, MAM4B_FLAG_SOA_NITER_LIMIT);
      s.gas[0] = st.g;
#pragma unroll
      for (int k = 0; k < NMODE; ++k)
        s.aer[0][k] = st.a[k];
      store_cloudborne(a, c, oc, f.ac);
      const FinishRegs src{ci, cg, f.ai, f.h2so4, f.soag};
      cell_finish(a, c, f.temp, f.pmid, f.zm, f.cld, f.pblh, rh, f.dgn_a[3], s, cm, src);
      return;
    }
  }
  const bool long_loop = first_rate > 0.05 * kLongLoopSteps;
  // warp-aggregated appends: the slot (in discovery order, which keeps the
  // post kernel's cell accesses coalesced) and the solver order entry
  const unsigned m = __activemask();
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(m) - 1;
  const unsigned m_long = __ballot_sync(m, long_loop), m_short = m & ~m_long;
  unsigned base = 0, b_long = 0, b_short = 0;
  if (lane == leader) {
    base = atomicAdd(&a.counters[CNT_QUEUED], (unsigned)__popc(m));
    if (m_long)
      b_long = atomicAdd(&a.counters[CNT_LONG], (unsigned)__popc(m_long));
    if (m_short)
      b_short = atomicAdd(&a.counters[CNT_SHORT], (unsigned)__popc(m_short));
  }
  base = __shfl_sync(m, base, leader);
  b_long = __shfl_sync(m, b_long, leader);
  b_short = __shfl_sync(m, b_short, leader);
  const unsigned below = (1u << lane) - 1;
  const unsigned slot = base + __popc(m & below);
  a.task[slot] = (int)c;
  if (long_loop)
    a.order[b_long + __popc(m_long & below)] = (int)slot;
  else
    a.order[a.ncell - 1 - (b_short + __popc(m_short & below))] = (int)slot;
  const size_t n = (size_t)a.ncell;
  double *q = a.soa + slot;
  q[SOA_G * n] = st.g;
#pragma unroll
  for (int k = 0; k < NMODE; ++k) {
    q[(SOA_A + k) * n] = st.a[k];
    q[(SOA_OPOA + k) * n] = st.opoa[k];
    q[(SOA_UPTK + k) * n] = st.uptk[k];
  }
  q[SOA_G0 * n] = st.g0;
  double *h = a.hand + slot;
  h[H_GAS1 * n] = s.gas[1];
  double pop[NPOP];
  sub_to_pop(s, pop);
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    h[(H_POP + p) * n] = pop[p];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    h[(H_UPTK + k) * n] = cm.uptk1[k];
  h[H_NETPROD * n] = cm.netprod1;
  h[H_SV_SO4 * n] = cm.sv_so4_ait;
  h[H_SV_SOA * n] = cm.sv_soa_ait;
  h[H_DGN_PC * n] = f.dgn_a[3];
  h[H_RELHUM * n] = rh;
  h[H_SOAG0 * n] = s.gas[0];
  store_cloudborne(a, c, oc, f.ac);
  if (partly) {
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      h[(H_CI + p) * n] = ci[p];
    h[H_CG * n] = cg[0];
    h[(H_CG + 1) * n] = cg[1];
  }
}

// Second half of a cell after its SOA loop: the rest of the clear subarea
// (H2SO4 update, renaming, nucleation, coagulation with the coefficients of
// pair_kernel, aging), recombination with the cloudy subarea's
// contributions (ci, cg; partly cloudy cells), tendencies of the gases and
// interstitial populations (the cloud-borne ones are written by the pre
// stage). s holds the clear subarea with the loop's result, cm the values
// saved before condensation.
// src supplies the values read late (src.ci(p), cg(g), ai(p), h2so4(),
// soag()): from registers in pre's fused path, from the hand-off and the
// inputs in post_kernel, where reading them only when needed keeps them out
// of registers during the suffix.
template <class Src>
__device__ __forceinline__ void cell_finish(const StepArgs &a, const long long c, double temp,
                                            double pmid, double zm, double cld, double pblh,
                                            double relhum, double dgn_pc, Sub &s, ClearMid &cm,
                                            const Src &src) {
  const StepConsts &C = c_k;
  const size_t n = (size_t)a.ncell;
  const double dt = a.dt;
  // wet sizes enter the suffix only through the coagulation coefficients,
  // which pair_kernel computed
  const double unused[NMODE] = {0, 0, 0, 0};
  clear_suffix<false, true>(a, dt, temp, pmid, zm, pblh, relhum, dgn_pc, unused, unused, cm, s,
                            nullptr, 0.0, a.aux + AUX_COAG * n + c, n);
  // recombination (form_gcm_of_gases_and_aerosols_from_subareas)
  const double fsoag = C.fcvt_soag;
  double o_h2so4, o_soag, oi[NPOP];
  double po[NPOP];
  sub_to_pop(s, po);
  if (cld < 1.0e-5) {
    const double f = 1.0 - 0.0;
    o_soag = dmax(0.0, 0.0 + (s.gas[0] / fsoag) * f);
    o_h2so4 = dmax(0.0, 0.0 + (s.gas[1] / 1.0) * f);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] = dmax(0.0, 0.0 + (po[K::numslot(m)] / 1.0) * f);
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int sl = K::aer_slot(x, m);
        if (sl >= 0)
          oi[sl] = dmax(0.0, 0.0 + (po[sl] / K::fcvt_aer(x)) * f);
      }
    }
  } else {
    const double fclea = 1.0 - cld;
    o_soag = dmax(0.0, (0.0 + (s.gas[0] / fsoag) * fclea) + src.cg(0));
    o_h2so4 = dmax(0.0, (0.0 + (s.gas[1] / 1.0) * fclea) + src.cg(1));
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] =
          dmax(0.0, (0.0 + (po[K::numslot(m)] / 1.0) * fclea) + src.ci(K::numslot(m)));
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int sl = K::aer_slot(x, m);
        if (sl >= 0)
          oi[sl] = dmax(0.0, (0.0 + (po[sl] / K::fcvt_aer(x)) * fclea) + src.ci(sl));
      }
    }
  }
  double ai[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    ai[p] = src.ai(p);
  store_interstitial(a, c, o_h2so4, o_soag, oi, src.h2so4(), src.soag(), ai);
}

// cell_finish's late inputs read from the hand-off of queue slot `slot`
// and the cell's inputs (post_kernel)
struct FinishLoads {
  const StepArgs &a;
  long long c;
  const double *h;
  size_t n;
  __device__ double ci(int p) const { return h[(H_CI + p) * n]; }
  __device__ double cg(int g) const { return h[(H_CG + g) * n]; }
  __device__ double ai(int p) const { return __ldg(a.in[MAM4B_IN_AER_I + p] + c); }
  __device__ double h2so4() const { return __ldg(a.in[MAM4B_IN_H2SO4] + c); }
  __device__ double soag() const { return __ldg(a.in[MAM4B_IN_SOAG] + c); }
};

// Second half of a queued cell: the state at the SOA loop (hand-off), the
// loop's result (solver), then cell_finish.
__device__ __forceinline__ void cell_post(const StepArgs &a, unsigned slot) {
  const size_t n = (size_t)a.ncell;
  const long long c = a.task[slot];
  const double temp = __ldg(a.in[MAM4B_IN_T] + c);
  const double pmid = __ldg(a.in[MAM4B_IN_P] + c);
  const double zm = __ldg(a.in[MAM4B_IN_ZM] + c);
  const double cld = __ldg(a.in[MAM4B_IN_CLD] + c);
  const double pblh = __ldg(a.pblh + c / a.nlev);
  const double *h = a.hand + slot;
  const double *q = a.soa + slot;
  Sub s;
  {
    double pop[NPOP];
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      pop[p] = h[(H_POP + p) * n];
    pop_to_sub(pop, s);
  }
  s.gas[0] = q[SOA_G * n];
  s.gas[1] = h[H_GAS1 * n];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    s.aer[0][k] = q[(SOA_A + k) * n];
  ClearMid cm;
  cm.netprod1 = h[H_NETPROD * n];
  cm.sv_so4_ait = h[H_SV_SO4 * n];
  cm.sv_soa_ait = h[H_SV_SOA * n];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    cm.uptk1[k] = h[(H_UPTK + k) * n];
  const FinishLoads src{a, c, h, n};
  cell_finish(a, c, temp, pmid, zm, cld, pblh, h[H_RELHUM * n], h[H_DGN_PC * n], s, cm, src);
}

template <bool DIAG>
__global__ void __launch_bounds__(128) full_kernel(const __grid_constant__ StepArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.ncell)
    cell_step<DIAG>(a, c);
}

// The step with chemistry start to end in one thread (process switches
// without condensation: no SOA loop to pipeline).
__device__ __forceinline__ void cell_step_chem(const StepArgs &a, const ChemArgs &ch,
                                               const long long c) {
  const StepConsts &C = c_k;
  Front f;
  cell_front<true>(a, c, f);
  const double dt = a.dt;
  ChemPre cp;
  run_chemistry(a, ch, c, f, cp);
  double o_h2so4, o_soag, oi[NPOP], oc[NPOP];
  const double fsoag = C.fcvt_soag;
  const bool map_gas = a.do_cond || a.do_newnuc;
  const double qgas1[2] = {cp.g1[0] * fsoag, cp.g1[1] * 1.0};
  if (f.cld > 0.999) {
    cloudy_cell_chem(a, f, cp, o_h2so4, o_soag, oi, oc);
  } else if (f.cld < 1.0e-5) {
    Sub s;
    load_sub_plain(s, f.qi);
    s.gas[0] = f.g_soag * fsoag;
    s.gas[1] = f.g_h2so4 * 1.0;
    const int niter = clear_subarea<false>(a, dt, f.temp, f.pmid, f.zm, f.pblh, f.relhumgcm,
                                           f.dgn_a, f.dgn_awet, f.wetdens, qgas1, s, nullptr,
                                           1.0);
    if (niter > 1000)
      atomicOr(a.flags, MAM4B_FLAG_SOA_NITER_LIMIT);
    const double w = 1.0 - 0.0;
    o_soag = dmax(0.0, 0.0 + (map_gas ? s.gas[0] / fsoag : f.g_soag) * w);
    o_h2so4 = dmax(0.0, 0.0 + (map_gas ? s.gas[1] / 1.0 : f.g_h2so4) * w);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] = dmax(0.0, 0.0 + (s.num[m] / 1.0) * w);
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0)
          oi[slot] = dmax(0.0, 0.0 + (s.aer[x][m] / K::fcvt_aer(x)) * w);
      }
    }
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      oc[p] = f.qc[p];
  } else {
    const double fclea = 1.0 - f.cld;
    Sub s;
    double gcl[2], rhc, ci[NPOP], cg[2];
    partly_cloudy_setup_chem(a, f, cp, s, gcl, rhc, ci, cg, oc);
    const int niter = clear_subarea<false>(a, dt, f.temp, f.pmid, f.zm, f.pblh, rhc, f.dgn_a,
                                           f.dgn_awet, f.wetdens, qgas1, s, nullptr, fclea);
    if (niter > 1000)
      atomicOr(a.flags, MAM4B_FLAG_SOA_NITER_LIMIT);
    o_soag = dmax(0.0, (0.0 + (map_gas ? s.gas[0] / fsoag : gcl[0]) * fclea) + cg[0]);
    o_h2so4 = dmax(0.0, (0.0 + (map_gas ? s.gas[1] / 1.0 : gcl[1]) * fclea) + cg[1]);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      oi[K::numslot(m)] = dmax(0.0, (0.0 + (s.num[m] / 1.0) * fclea) + ci[K::numslot(m)]);
#pragma unroll
      for (int x = 0; x < NAER; ++x) {
        const int slot = K::aer_slot(x, m);
        if (slot >= 0)
          oi[slot] = dmax(0.0, (0.0 + (s.aer[x][m] / K::fcvt_aer(x)) * fclea) + ci[slot]);
      }
    }
  }
  store_outputs(a, c, o_h2so4, o_soag, oi, oc, f.h2so4, f.soag, f.ai, f.ac);
}

__global__ void __launch_bounds__(128) chem_step_kernel(const __grid_constant__ StepArgs a,
                                                        const __grid_constant__ ChemArgs ch) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.ncell)
    cell_step_chem(a, ch, c);
}

// Launch shapes of the pipeline kernels. Each whole-cell kernel is compiled
// once per register cap (__maxnreg__; a lower cap lets more warps reside on
// an SM, at the price of spills) and takes its block size and the number
// of cells each thread steps (a grid-stride loop) at launch; the values are
// chosen per device by mam4b_autotune (include/mam4b.h). The arithmetic is
// the same in every variant, so their results are bit for bit equal.
// Register caps compiled:
//   size_kernel 255, 128, 96; pre_kernel and post_kernel 255, 168, 128;
//   soa_kernel 64, 96, 128.

// Stage 1 of the pipelined step, one thread per cell: calcsize for the dry
// diameters (an output), the relative humidity of water uptake and the
// H2SO4 diffusivity and mean free path.
__device__ __forceinline__ void size_cell(const StepArgs &a, const long long c) {
  const StepConsts &C = c_k;
  double ai[NPOP], ac[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ai[p] = __ldg(a.in[MAM4B_IN_AER_I + p] + c);
    ac[p] = __ldg(a.in[MAM4B_IN_AER_C + p] + c);
  }
  double dgn_a[NMODE], pt_i[NPOP], pt_c[NPOP];
  calcsize(C, ai, ac, a.dt, dgn_a, pt_i, pt_c);
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    a.out[MAM4B_OUT_DGN_A + m][c] = dgn_a[m];
  const double temp = __ldg(a.in[MAM4B_IN_T] + c);
  const double pmid = __ldg(a.in[MAM4B_IN_P] + c);
  const size_t n = (size_t)a.ncell;
  a.aux[AUX_RH * n + c] =
      water_uptake_rh(__ldg(a.in[MAM4B_IN_QV] + c), temp, pmid, __ldg(a.in[MAM4B_IN_CLD] + c));
  double gd, fp;
  h2so4_diffusivity(temp, pmid, gd, fp);
  a.aux[AUX_GDIFF * n + c] = gd;
  a.aux[AUX_FPATH * n + c] = fp;
}

// LOOP: grid-stride loop over cells (cells_per_thread > 1); without it one
// cell per thread, which leaves the register allocation of the body as is.
template <int R, bool LOOP>
__global__ void __maxnreg__(R) size_kernel(const __grid_constant__ StepArgs a) {
  const long long c0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (LOOP) {
    const long long stride = (long long)gridDim.x * blockDim.x;
#pragma unroll 1
    for (long long c = c0; c < a.ncell; c += stride)
      size_cell(a, c);
  } else if (c0 < a.ncell) {
    size_cell(a, c0);
  }
}

// Stage 2, one thread per (cell, mode): water uptake of the mode (Kohler
// equilibrium, wet size, water, wet density; outputs) and its per-particle
// H2SO4 uptake rate. The modes are independent here, and a thread holds
// one mode's state only, so many more warps are resident than in a
// whole-cell thread.
// With MIXED the mode's arithmetic is single precision (mam4b::f32).
template <int M, bool MIXED>
__device__ __forceinline__ void mode_work(const StepArgs &a, const long long c) {
  const StepConsts &C = c_k;
  const size_t n = (size_t)a.ncell;
  if constexpr (MIXED) {
    float sp[7];
#pragma unroll
    for (int s = 0; s < 7; ++s)
      sp[s] = (s < K::nspec(M)) ? (float)__ldg(a.in[MAM4B_IN_AER_I + K::spec0(M) + (s < K::nspec(M) ? s : 0)] + c) : 0.0f;
    float dgn_awet, qaerwat, wetdens;
    f32::water_uptake_mode<M>(C, sp, a.aux[AUX_RH * n + c],
                              (float)a.out[MAM4B_OUT_DGN_A + M][c], dgn_awet, qaerwat, wetdens);
    a.out[MAM4B_OUT_DGN_AWET + M][c] = dgn_awet;
    a.out[MAM4B_OUT_WETDENS + M][c] = wetdens;
    a.out[MAM4B_OUT_QAERWAT + M][c] = qaerwat;
    a.aux[(AUX_RATE + M) * n + c] = f32::uptake_rate_mode(
        C, M, (float)a.aux[AUX_GDIFF * n + c], (float)a.aux[AUX_FPATH * n + c], dgn_awet);
    return;
  }
  double sp[7];
#pragma unroll
  for (int s = 0; s < 7; ++s)
    sp[s] = (s < K::nspec(M)) ? __ldg(a.in[MAM4B_IN_AER_I + K::spec0(M) + (s < K::nspec(M) ? s : 0)] + c) : 0.0;
  const double dgn_a = a.out[MAM4B_OUT_DGN_A + M][c];
  double dgn_awet, qaerwat, wetdens;
  water_uptake_mode<M>(C, sp, a.aux[AUX_RH * n + c], dgn_a, dgn_awet, qaerwat, wetdens);
  a.out[MAM4B_OUT_DGN_AWET + M][c] = dgn_awet;
  a.out[MAM4B_OUT_WETDENS + M][c] = wetdens;
  a.out[MAM4B_OUT_QAERWAT + M][c] = qaerwat;
  a.aux[(AUX_RATE + M) * n + c] =
      uptake_rate_mode(C, M, a.aux[AUX_GDIFF * n + c], a.aux[AUX_FPATH * n + c], dgn_awet);
}

// FP64: the block's cells are regrouped so that the cells below the
// crystallisation humidity, whose water uptake needs no Kohler solve, fill
// warps of their own (cell order kept within each group; blocks of at most
// 256 threads, the launch shapes allowed).
template <bool MIXED>
__global__ void mode_kernel(const __grid_constant__ StepArgs a) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (!MIXED) {
    __shared__ int s_perm[256];
    __shared__ unsigned s_cnt[8][2];
    const long long c0 = (long long)blockIdx.x * blockDim.x;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
    const bool valid = c < a.ncell;
    const bool dry = valid && a.aux[AUX_RH * (size_t)a.ncell + c] < K::rh_cryst;
    const unsigned bd = __ballot_sync(0xffffffffu, dry);
    const unsigned bo = __ballot_sync(0xffffffffu, valid && !dry);
    if (lane == 0) {
      s_cnt[w][0] = __popc(bd);
      s_cnt[w][1] = __popc(bo);
    }
    __syncthreads();
    unsigned before_d = 0, before_o = 0, total_d = 0, total = 0;
    for (int k = 0; k < nw; ++k) {
      if (k < w) {
        before_d += s_cnt[k][0];
        before_o += s_cnt[k][1];
      }
      total_d += s_cnt[k][0];
      total += s_cnt[k][0] + s_cnt[k][1];
    }
    if (valid) {
      const unsigned below = (1u << lane) - 1u;
      s_perm[dry ? before_d + __popc(bd & below) : total_d + before_o + __popc(bo & below)] = t;
    }
    __syncthreads();
    if ((unsigned)t >= total)
      return;
    c = c0 + s_perm[t];
  }
  if (c >= a.ncell)
    return;
  switch (blockIdx.y) {
  case 0: mode_work<0, MIXED>(a, c); break;
  case 1: mode_work<1, MIXED>(a, c); break;
  case 2: mode_work<2, MIXED>(a, c); break;
  default: mode_work<3, MIXED>(a, c); break;
  }
}

// Stage 3, one thread per (cell, mode pair): the Brownian coagulation
// coefficients of the pair (getcoags, coagulation.hpp:651-817) from the wet
// sizes and densities of stage 2; they do not depend on what condensation
// changes, so the post kernel only applies them.
template <bool MIXED>
__global__ void pair_kernel(const __grid_constant__ StepArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  const StepConsts &C = c_k;
  const int p = blockIdx.y;
  const int sm = coag_src(p), dm = coag_dst(p);
  const double temp = __ldg(a.in[MAM4B_IN_T] + c);
  const double pmid = __ldg(a.in[MAM4B_IN_P] + c);
  const double aircon = pmid / (8314.46759100000 * temp);
  const double dens_s = dmax(1000.0, a.out[MAM4B_OUT_WETDENS + sm][c]);
  const double dens_d = dmax(1000.0, a.out[MAM4B_OUT_WETDENS + dm][c]);
  const CoagTables T = {kCoagBm0ij, kCoagBm3i, kCoagBm0};
  double bij0, bij3, bii0, bjj0;
  // the FP32 coefficients unless the correction-table index (round() of
  // 2 ln(dg_dst / dg_src) / ln 2, coagulation.hpp:715-717) sits within 1e-3
  // of a rounding boundary, where FP32 might round the other way
  bool fp32 = MIXED;
  if constexpr (MIXED) {
    const double r = a.out[MAM4B_OUT_DGN_AWET + dm][c] / a.out[MAM4B_OUT_DGN_AWET + sm][c];
    const double xr = log(r) / log(sqrt(2.0));
    fp32 = fabs(xr - floor(xr) - 0.5) > 1.0e-3;
  }
  if (fp32) {
    float f0, f3, fi, fj;
    f32::coag_pair_coefs(C, T, p, (float)temp, (float)pmid, (float)aircon,
                         (float)a.out[MAM4B_OUT_DGN_AWET + sm][c],
                         (float)a.out[MAM4B_OUT_DGN_AWET + dm][c], (float)dens_s, (float)dens_d,
                         f0, f3, fi, fj);
    bij0 = f0;
    bij3 = f3;
    bii0 = fi;
    bjj0 = fj;
  } else {
    coag_pair_coefs(C, T, p, temp, pmid, aircon, a.out[MAM4B_OUT_DGN_AWET + sm][c],
                    a.out[MAM4B_OUT_DGN_AWET + dm][c], dens_s, dens_d, bij0, bij3, bii0, bjj0);
  }
  const size_t n = (size_t)a.ncell;
  double *cc = a.aux + AUX_COAG * n + c;
  cc[p * n] = bij0;
  cc[(3 + p) * n] = bij3;
  cc[(6 + p) * n] = bii0;
  cc[(9 + p) * n] = bjj0;
}

// FUSE: cells with short SOA loops finish here (StepArgs::inline_scale)
template <int R, bool MIXED, bool FUSE>
__global__ void __maxnreg__(R) pre_kernel(const __grid_constant__ StepArgs a) {
  const ChemArgs none = {nullptr, nullptr, 0};
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.ncell)
    cell_pre<false, MIXED, FUSE>(a, none, c);
}

// The pre stage of the step with chemistry (mam4b_step_chem_slab).
__global__ void __launch_bounds__(128) pre_chem_kernel(const __grid_constant__ StepArgs a,
                                                       const __grid_constant__ ChemArgs ch) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.ncell)
    cell_pre<true>(a, ch, c);
}

// (the 128-register cap, 4 blocks of 128 per SM with a few hundred bytes
// spilled to L1, was 2 % faster than the unconstrained 231-register build)
template <int R, bool LOOP>
__global__ void __maxnreg__(R) post_kernel(const __grid_constant__ StepArgs a) {
  const long long nq = (long long)a.counters[CNT_QUEUED];
  const long long i0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (LOOP) {
    const long long stride = (long long)gridDim.x * blockDim.x;
#pragma unroll 1
    for (long long i = i0; i < nq; i += stride)
      cell_post(a, (unsigned)i);
  } else if (i0 < nq) {
    cell_post(a, (unsigned)i0);
  }
}

// SOA sub-stepping of the queued cells. Persistent warps; every lane owns
// one cell's loop and, as soon as that loop ends, takes the next queued
// cell (one atomic per warp for all lanes that need work), so a warp never
// idles behind one cell that needs hundreds of sub-steps. Cells are taken
// long loops first, so that the last ones handed out are short. The loop
// is bound by FP64 division latency: 4 blocks of 256 per SM (64 registers)
// hide more of it than the unconstrained 93-register build.
// With MIXED the loop runs in single precision (f32::soa_step).
// Launched with any block size that is a multiple of 32 and one grid of
// persistent blocks (SMs x blocks per SM).
constexpr int kSoaBlock = 256;
template <int SOA, class State>
__device__ __forceinline__ bool soa_pass(State &st) {
  if constexpr (SOA == 1)
    return f32::soa_step_mx(st);
  else
    return soa_step(st);
}

// SOA: 0 the FP64 loop (soa_step), 1 FP64 state with FP32 step control
// (f32::soa_step_mx, MAM4B_MIXED), 2 the FP32 loop (f32::soa_step,
// MAM4B_MIXED_FAST).
template <int SOA, int R>
__global__ void __maxnreg__(R) soa_kernel(const __grid_constant__ StepArgs a) {
  constexpr bool F32 = SOA == 2;
  using State = typename std::conditional<F32, f32::SoaStateF, SoaState>::type;
  const unsigned ntask = a.counters[CNT_QUEUED];
  const unsigned nlong = a.counters[CNT_LONG];
  const int lane = threadIdx.x & 31;
  const size_t n = (size_t)a.ncell;
  State st;
  unsigned slot = 0;
  bool active = false, want = true;
  while (true) {
    const unsigned need = __ballot_sync(0xffffffffu, want);
    if (need) {
      const int leader = __ffs(need) - 1;
      unsigned base = 0;
      if (lane == leader)
        base = atomicAdd(&a.counters[CNT_TAKEN], (unsigned)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (want) {
        const unsigned t = base + __popc(need & ((1u << lane) - 1));
        want = false;
        if (t < ntask) {
          slot = (unsigned)(t < nlong ? a.order[t] : a.order[a.ncell - 1 - (t - nlong)]);
          const double *q = a.soa + slot;
          st.g = q[SOA_G * n];
#pragma unroll
          for (int k = 0; k < NMODE; ++k) {
            st.a[k] = q[(SOA_A + k) * n];
            st.opoa[k] = q[(SOA_OPOA + k) * n];
            st.uptk[k] = q[(SOA_UPTK + k) * n];
          }
          st.g0 = q[SOA_G0 * n];
          st.tcur = 0.0;
          st.dtfull = (double)(int)(a.dt / 1);
          st.niter = 0;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active))
      break;
    if (active && !soa_pass<SOA>(st)) {
      double *q = a.soa + slot;
      q[SOA_G * n] = st.g;
#pragma unroll
      for (int k = 0; k < NMODE; ++k)
        q[(SOA_A + k) * n] = st.a[k];
      if (st.niter > 1000)
        atomicOr(a.flags, MAM4B_FLAG_SOA_NITER_LIMIT);
      if (a.npass)
        a.npass[slot] = st.niter > 1000 ? 1000 : st.niter;
      active = false;
      want = true;
    }
  }
}

// ============================================================ adjoint
// Reverse-mode adjoint of the FP64 step: in_bar = (d out / d in)^T out_bar
// per cell. Persistent threads; each runs one cell's forward sweep (state
// at process boundaries in local memory, the SOA loop's state every
// adj::kSoaCheck passes in its own slice of `ck`, laid out
// [checkpoint][component][thread] so a warp's accesses are coalesced) and
// then its reverse sweep.
struct AdjArgs {
  const double *in;    // [MAM4B_NIN][ld]
  const double *pblh;  // [ncol]
  const double *ybar;  // [MAM4B_NOUT][ld]
  double *xbar;        // [MAM4B_NIN][ld]
  size_t ld;
  long long ncell;
  int nlev;
  double dt;
  adj::AdjCfg cfg;
  double *ck;          // [6 * kSoaCkMax][nthreads]
};

__global__ void __launch_bounds__(128) adjoint_kernel(const __grid_constant__ AdjArgs a) {
  const size_t nthreads = (size_t)gridDim.x * blockDim.x;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const CoagTables T = {kCoagBm0ij, kCoagBm3i, kCoagBm0};
  double *ck = a.ck + tid;
  for (long long c = (long long)tid; c < a.ncell; c += (long long)nthreads) {
    double x[MAM4B_NIN], yb[MAM4B_NOUT], y[MAM4B_NOUT], xb[MAM4B_NIN];
#pragma unroll
    for (int f = 0; f < MAM4B_NIN; ++f)
      x[f] = __ldg(a.in + (size_t)f * a.ld + c);
#pragma unroll
    for (int f = 0; f < MAM4B_NOUT; ++f)
      yb[f] = __ldg(a.ybar + (size_t)f * a.ld + c);
    const double pblh = __ldg(a.pblh + c / a.nlev);
    int niter;
    adj::cell_adjoint(c_k, T, a.cfg, x, pblh, a.dt, ck, nthreads, yb, y, xb, niter);
#pragma unroll
    for (int f = 0; f < MAM4B_NIN; ++f)
      a.xbar[(size_t)f * a.ld + c] = xb[f];
  }
}

// ---- pipelined adjoint (condensation on): after the forward pipeline,
// adj_post_kernel reverses each queued cell's suffix (H2SO4 update,
// renaming, nucleation, coagulation, aging, recombination) from the
// hand-off, adj_soa_kernel reverses the SOA loops with the same work
// stealing as the forward solver, and adj_pre_kernel recomputes each cell's
// front and reverses it. Cotangents pass through cell-indexed scratch.
enum {
  AB_SB = 0,        // 29: subarea state after the loop: num[4], aer[1..6][4], gas[1]
  AB_NETPROD = 29,
  AB_UPTK1 = 30,    // 4
  AB_SV_SO4 = 34,
  AB_SV_SOA = 35,
  AB_DGN_PC = 36,
  AB_RH_SUB = 37,
  AB_T = 38,
  AB_DGN_AWET = 39,  // 4
  AB_WETDENS = 43,   // 4
  AB_CI = 47,        // 25
  AB_CG = 72,        // 2
  AB_FIELDS = 74
};
enum { LB_G = 0, LB_A = 1, LB_OPOA = 5, LB_UPTK = 9, LB_G0 = 13, LB_FIELDS = 14 };

struct AdjPipeArgs {
  StepArgs s;           // the forward pipeline's arguments and scratch
  const double *ybar;   // [MAM4B_NOUT][ld]
  double *xbar;         // [MAM4B_NIN][ld]
  size_t ld;
  double *abar;         // [AB_FIELDS][ncell]
  double *lbar;         // [LB_FIELDS][ncell]
  double *ck;           // SOA states [6 adj_soa_slots(CK)][nthreads of adj_soa_kernel]
  unsigned *bins;       // [2 kPassBins]: loops per pass count, start offsets
  adj::AdjCfg cfg;
};

// sb slot j (0..28) <-> Sub components other than the SOA ones
MAM4B_HD double &sb_ref(Sub &b, int j) {
  if (j < 4)
    return b.num[j];
  if (j < 28)
    return b.aer[1 + (j - 4) / 4][(j - 4) % 4];
  return b.gas[1];
}

__global__ void __launch_bounds__(128, 4) adj_post_kernel(const __grid_constant__ AdjPipeArgs p) {
  const StepArgs &a = p.s;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)a.counters[CNT_QUEUED])
    return;
  const StepConsts &C = c_k;
  const CoagTables T = {kCoagBm0ij, kCoagBm3i, kCoagBm0};
  const size_t n = (size_t)a.ncell;
  const long long c = a.task[i];
  const double temp = __ldg(a.in[MAM4B_IN_T] + c);
  const double pmid = __ldg(a.in[MAM4B_IN_P] + c);
  const double zm = __ldg(a.in[MAM4B_IN_ZM] + c);
  const double cld = __ldg(a.in[MAM4B_IN_CLD] + c);
  const double pblh = __ldg(a.pblh + c / a.nlev);
  const double *h = a.hand + i;
  double *q = a.soa + i;
  adj::SuffixIn in;
  {
    double pop[NPOP];
#pragma unroll
    for (int k = 0; k < NPOP; ++k)
      pop[k] = h[(H_POP + k) * n];
    pop_to_sub(pop, in.s_soa);
  }
  in.s_soa.gas[0] = q[SOA_G * n];
  in.s_soa.gas[1] = h[H_GAS1 * n];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    in.s_soa.aer[0][k] = q[(SOA_A + k) * n];
  in.cm.netprod1 = h[H_NETPROD * n];
  in.cm.sv_so4_ait = h[H_SV_SO4 * n];
  in.cm.sv_soa_ait = h[H_SV_SOA * n];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    in.cm.uptk1[k] = h[(H_UPTK + k) * n];
  in.dgn_pc = h[H_DGN_PC * n];
  in.rh_sub = h[H_RELHUM * n];
#pragma unroll
  for (int k = 0; k < 12; ++k)
    in.cc[k] = a.aux[(AUX_COAG + k) * n + c];
  in.partly = !(cld < 1.0e-5);
  in.fclea = 1.0 - cld;
#pragma unroll
  for (int k = 0; k < NPOP; ++k)
    in.ci[k] = in.partly ? h[(H_CI + k) * n] : 0.0;
  in.cg[0] = in.partly ? h[H_CG * n] : 0.0;
  in.cg[1] = in.partly ? h[(H_CG + 1) * n] : 0.0;
  adj::SuffixStates st;
  adj::suffix_states(C, p.cfg, temp, pmid, zm, pblh, a.dt, in, st);
  double ybt[MAM4B_NUM_PROG];
#pragma unroll
  for (int k = 0; k < MAM4B_NUM_PROG; ++k)
    ybt[k] = __ldg(p.ybar + (size_t)(MAM4B_OUT_TEND + k) * p.ld + c);
  adj::SuffixBar sb;
  adj::suffix_rev(C, p.cfg, temp, pmid, zm, pblh, a.dt, in, st, ybt, sb);
  double dgn_awet[NMODE], wetdens[NMODE], dgn_awetb[NMODE] = {0, 0, 0, 0},
                                           wetdensb[NMODE] = {0, 0, 0, 0};
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    dgn_awet[m] = a.out[MAM4B_OUT_DGN_AWET + m][c];
    wetdens[m] = dmax(1000.0, a.out[MAM4B_OUT_WETDENS + m][c]);
  }
  double tb = sb.tb;
  if (p.cfg.do_coag)
    adj::coef_rev(C, T, temp, pmid, dgn_awet, wetdens, sb.ccb, tb, dgn_awetb, wetdensb);
  // loop-end cotangents for the solver's reverse (slot-indexed)
  q[SOA_G * n] = sb.sb.gas[0];
#pragma unroll
  for (int k = 0; k < NMODE; ++k)
    q[(SOA_A + k) * n] = sb.sb.aer[0][k];
  double *ab = p.abar + c;
#pragma unroll
  for (int j = 0; j < 29; ++j)
    ab[(AB_SB + j) * n] = sb_ref(sb.sb, j);
  ab[AB_NETPROD * n] = sb.netprodb;
#pragma unroll
  for (int k = 0; k < NMODE; ++k) {
    ab[(AB_UPTK1 + k) * n] = sb.uptk1b[k];
    ab[(AB_DGN_AWET + k) * n] = dgn_awetb[k];
    ab[(AB_WETDENS + k) * n] = wetdensb[k];
  }
  ab[AB_SV_SO4 * n] = sb.sv_so4b;
  ab[AB_SV_SOA * n] = sb.sv_soab;
  ab[AB_DGN_PC * n] = sb.dgn_pcb;
  ab[AB_RH_SUB * n] = sb.rh_subb;
  ab[AB_T * n] = tb;
#pragma unroll
  for (int k = 0; k < NPOP; ++k)
    ab[(AB_CI + k) * n] = sb.cib[k];
  ab[AB_CG * n] = sb.cgb[0];
  ab[(AB_CG + 1) * n] = sb.cgb[1];
}

// The SOA loops are reversed in order of decreasing pass count, so that the
// 32 loops of a warp take the same number of passes and run in step:
// adj_hist_kernel counts the loops per pass count (npass, written by
// soa_kernel), adj_scan_kernel turns the counts into start offsets (most
// passes first) and adj_sort_kernel writes the slots in that order over the
// forward solver's order list, which is free once soa_kernel has run.
constexpr int kPassBins = 1001;  // pass counts 0..1000

__global__ void __launch_bounds__(256) adj_hist_kernel(const __grid_constant__ AdjPipeArgs p) {
  __shared__ unsigned h[kPassBins];
  for (int i = threadIdx.x; i < kPassBins; i += blockDim.x)
    h[i] = 0;
  __syncthreads();
  const unsigned ntask = p.s.counters[CNT_QUEUED];
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < ntask; t += gridDim.x * blockDim.x)
    atomicAdd(&h[1000 - p.s.npass[t]], 1u);
  __syncthreads();
  for (int i = threadIdx.x; i < kPassBins; i += blockDim.x)
    if (h[i])
      atomicAdd(&p.bins[i], h[i]);
}

__global__ void __launch_bounds__(1024) adj_scan_kernel(const __grid_constant__ AdjPipeArgs p) {
  // exclusive scan of kPassBins counts, one block: each thread sums its
  // run of bins, the runs' totals are scanned in shared memory
  __shared__ unsigned tot[1024];
  constexpr int per = (kPassBins + 1023) / 1024;
  const int i0 = threadIdx.x * per;
  unsigned sum = 0;
  for (int i = i0; i < i0 + per && i < kPassBins; ++i)
    sum += p.bins[i];
  tot[threadIdx.x] = sum;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const unsigned v = threadIdx.x >= (unsigned)d ? tot[threadIdx.x - d] : 0u;
    __syncthreads();
    tot[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned off = tot[threadIdx.x] - sum;
  for (int i = i0; i < i0 + per && i < kPassBins; ++i) {
    const unsigned c = p.bins[i];
    p.bins[kPassBins + i] = off;
    off += c;
  }
}

__global__ void __launch_bounds__(256) adj_sort_kernel(const __grid_constant__ AdjPipeArgs p) {
  const unsigned ntask = p.s.counters[CNT_QUEUED];
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < ntask; t += gridDim.x * blockDim.x)
    p.s.order[atomicAdd(&p.bins[kPassBins + 1000 - p.s.npass[t]], 1u)] = (int)t;
}

// Reverse of the SOA loops. Warps take 32 loops at a time from the sorted
// order list (one atomic per warp); every lane runs its loop forward,
// keeping the state (g, a[4], tcur) before passes in its own column of
// p.ck ([6 * index + component][thread]: the lanes of a warp are at the
// same pass, so a warp's stores and loads are coalesced), then the reverse
// passes, last to first, starting from the loop-end cotangents left by
// adj_post_kernel. CK = 1 stores the state before every pass (1,001 states
// per thread). CK > 1 keeps a checkpoint every CK passes (the states
// before passes 0, CK, 2 CK, ...: ceil(1001 / CK) per thread) and reverses
// the loop block by block: it recomputes the block's states from its
// checkpoint into a CK-state slice of the thread's column, then reverses
// the block's passes from them. Both give the same gradient bit for bit
// (the recomputed passes are the forward's arithmetic on the same state);
// CK > 1 needs about 1/CK of the memory and recomputes up to CK - 1 passes
// per block. The forward loop is the step's: soa_step (FP64), or with FAST
// f32::soa_step_mx (the mixed-precision adjoint). The reverse of each pass
// linearises it at the stored state with the division-free arithmetic of
// f32::soa_step_mx (adj::soa_step_rev_t<true>): the trajectory is the
// forward's exactly, its local derivative is computed to rounding (a
// branch that sits within rounding of its threshold may be taken the other
// way, like a finite difference across it). 2 blocks per SM (128
// registers, some spilled to L1): the extra warps hide more FP64 latency
// than the unconstrained 255-register build (10 % faster).
constexpr int kAdjSoaStates = 1001;  // states before passes 0..1000 (passes <= 1000)
// states kept per solver thread: checkpoints plus, with CK > 1, one block
__host__ __device__ constexpr int adj_soa_slots(int ck) {
  return ck == 1 ? kAdjSoaStates : (kAdjSoaStates + ck - 1) / ck + ck;
}

template <bool FAST>
__device__ __forceinline__ bool adj_soa_pass(SoaState &st) {
  if constexpr (FAST)
    return f32::soa_step_mx(st);
  else
    return soa_step(st);
}

template <int CK, bool FAST>
__global__ void __launch_bounds__(kSoaBlock, 2) adj_soa_kernel(const __grid_constant__ AdjPipeArgs p) {
  const StepArgs &a = p.s;
  const unsigned ntask = a.counters[CNT_QUEUED];
  const int lane = threadIdx.x & 31;
  const size_t n = (size_t)a.ncell;
  const size_t nthreads = (size_t)gridDim.x * blockDim.x;
  double *ck = p.ck + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  auto put = [&](int idx, const SoaState &x) {
    double *e = ck + (size_t)6 * idx * nthreads;
    e[0] = x.g;
#pragma unroll
    for (int j = 0; j < NMODE; ++j)
      e[(1 + j) * nthreads] = x.a[j];
    e[5 * nthreads] = x.tcur;
  };
  auto get = [&](int idx, SoaState &x) {
    const double *e = ck + (size_t)6 * idx * nthreads;
    x.g = e[0];
#pragma unroll
    for (int j = 0; j < NMODE; ++j)
      x.a[j] = e[(1 + j) * nthreads];
    x.tcur = e[5 * nthreads];
  };
  while (true) {
    unsigned base = 0;
    if (lane == 0)
      base = atomicAdd(&a.counters[CNT_TAKEN_ADJ], 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= ntask)
      break;
    const unsigned t = base + lane;
    if (t >= ntask)
      continue;
    const unsigned slot = (unsigned)a.order[t];
    const double *h = a.hand + slot;
    const double *q = a.soa + slot;
    SoaState st;
    st.g = h[H_SOAG0 * n];
    {
      double pop[NPOP];
#pragma unroll
      for (int j = 0; j < NPOP; ++j)
        pop[j] = h[(H_POP + j) * n];
      Sub s0;
      pop_to_sub(pop, s0);
#pragma unroll
      for (int j = 0; j < NMODE; ++j)
        st.a[j] = s0.aer[0][j];
    }
#pragma unroll
    for (int j = 0; j < NMODE; ++j) {
      st.opoa[j] = q[(SOA_OPOA + j) * n];
      st.uptk[j] = q[(SOA_UPTK + j) * n];
    }
    st.g0 = q[SOA_G0 * n];
    st.tcur = 0.0;
    st.dtfull = (double)(int)(a.dt / 1);
    st.niter = 0;
    // forward: k passes (the states before passes 0..k-1 are reversed)
    int k = 0;
    while (true) {
      if (CK == 1 || k % CK == 0)
        put(k / CK, st);
      if (!adj_soa_pass<FAST>(st))
        break;
      ++k;
    }
    adj::SoaBar b;
    b.g = q[SOA_G * n];
#pragma unroll
    for (int j = 0; j < NMODE; ++j) {
      b.a[j] = q[(SOA_A + j) * n];
      b.opoa[j] = 0.0;
      b.uptk[j] = 0.0;
    }
    b.tcur = 0.0;
    b.g0 = 0.0;
    if constexpr (CK == 1) {
      while (k > 0) {
        --k;
        get(k, st);
        adj::soa_step_rev_t<true>(st, b);
      }
    } else {
      constexpr int kBlock = (kAdjSoaStates + CK - 1) / CK;  // first state of the block slice
      for (int b0 = k > 0 ? ((k - 1) / CK) * CK : -1; b0 >= 0; b0 -= CK) {
        const int nb = min(CK, k - b0);  // passes b0 .. b0 + nb - 1
        get(b0 / CK, st);
        // these passes all continued in the forward (niter only caps it)
        st.niter = 0;
        put(kBlock, st);
        for (int j = 1; j < nb; ++j) {
          adj_soa_pass<FAST>(st);
          put(kBlock + j, st);
        }
        for (int j = nb - 1; j >= 0; --j) {
          get(kBlock + j, st);
          adj::soa_step_rev_t<true>(st, b);
        }
      }
    }
    const long long c = a.task[slot];
    double *lb = p.lbar + c;
    lb[LB_G * n] = b.g;
#pragma unroll
    for (int j = 0; j < NMODE; ++j) {
      lb[(LB_A + j) * n] = b.a[j];
      lb[(LB_OPOA + j) * n] = b.opoa[j];
      lb[(LB_UPTK + j) * n] = b.uptk[j];
    }
    lb[LB_G0 * n] = b.g0;
  }
}

// The whole-cell reverse kernels (adj_post, adj_pre, adj_fin) run 4 blocks
// of 128 per SM (128 registers, their tapes in L1-cached local memory):
// 2.8 ms faster in total than unconstrained at 255 registers.
//
// Reverse of each cell's front (and of cloudy cells entirely), up to the
// water uptake: the front's forward sweep takes water uptake, diffusivity
// and uptake rates from the forward pipeline (out rows, aux), the
// reverse leaves the partial input cotangents in xbar and the cotangents
// of the water uptake's and calcsize's outputs in abar (FT_* fields, over
// the suffix cotangents it has read).
enum { FT_PT_IB = 0, FT_PT_CB = 25, FT_DGN_AB = 50, FT_DGN_AWETB = 54, FT_QAERWATB = 58,
       FT_WETDENS_WUB = 62, FT_RHB = 66, FT_FIELDS = 70 };
static_assert(FT_FIELDS <= AB_FIELDS, "front hand-off must fit in abar");

__global__ void __launch_bounds__(128, 4) adj_pre_kernel(const __grid_constant__ AdjPipeArgs p) {
  const StepArgs &a = p.s;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  const size_t n = (size_t)a.ncell;
  double x[MAM4B_NIN], yb[MAM4B_NOUT], y[MAM4B_NOUT], xb[MAM4B_NIN];
#pragma unroll
  for (int f = 0; f < MAM4B_NIN; ++f)
    x[f] = __ldg(a.in[f] + c);
#pragma unroll
  for (int f = 0; f < MAM4B_NOUT; ++f)
    yb[f] = __ldg(p.ybar + (size_t)f * p.ld + c);
  adj::FrontKnown kn;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    kn.dgn_awet[m] = a.out[MAM4B_OUT_DGN_AWET + m][c];
    kn.wetdens_wu[m] = a.out[MAM4B_OUT_WETDENS + m][c];
    kn.qaerwat[m] = a.out[MAM4B_OUT_QAERWAT + m][c];
    kn.rate[m] = a.aux[(AUX_RATE + m) * n + c];
  }
  kn.rh_wu = a.aux[AUX_RH * n + c];
  kn.gd = a.aux[AUX_GDIFF * n + c];
  kn.fp = a.aux[AUX_FPATH * n + c];
  adj::FrontTape ft;
  adj::front_forward<true>(c_k, p.cfg, x, a.dt, ft, y, &kn);
  const double zero4[NMODE] = {0, 0, 0, 0};
  adj::FrontTail tl;
  if (ft.cat == 1) {
    adj::front_rev_head(c_k, p.cfg, x, a.dt, ft, nullptr, nullptr, yb, zero4, zero4, 0.0, xb, tl);
  } else {
    const double *ab = p.abar + c;
    const double *lbp = p.lbar + c;
    adj::SuffixBar sb;
    adj::sub_zero(sb.sb);
#pragma unroll
    for (int j = 0; j < 29; ++j)
      sb_ref(sb.sb, j) = ab[(AB_SB + j) * n];
    sb.netprodb = ab[AB_NETPROD * n];
    double dgn_awetb[NMODE], wetdensb[NMODE];
#pragma unroll
    for (int k = 0; k < NMODE; ++k) {
      sb.uptk1b[k] = ab[(AB_UPTK1 + k) * n];
      dgn_awetb[k] = ab[(AB_DGN_AWET + k) * n];
      wetdensb[k] = ab[(AB_WETDENS + k) * n];
    }
    sb.sv_so4b = ab[AB_SV_SO4 * n];
    sb.sv_soab = ab[AB_SV_SOA * n];
    sb.dgn_pcb = ab[AB_DGN_PC * n];
    sb.rh_subb = ab[AB_RH_SUB * n];
    sb.tb = 0.0;
#pragma unroll
    for (int k = 0; k < NPOP; ++k)
      sb.cib[k] = ab[(AB_CI + k) * n];
    sb.cgb[0] = ab[AB_CG * n];
    sb.cgb[1] = ab[(AB_CG + 1) * n];
    adj::SoaBar lb;
    lb.g = lbp[LB_G * n];
#pragma unroll
    for (int k = 0; k < NMODE; ++k) {
      lb.a[k] = lbp[(LB_A + k) * n];
      lb.opoa[k] = lbp[(LB_OPOA + k) * n];
      lb.uptk[k] = lbp[(LB_UPTK + k) * n];
    }
    lb.g0 = lbp[LB_G0 * n];
    lb.tcur = 0.0;
    adj::front_rev_head(c_k, p.cfg, x, a.dt, ft, &sb, &lb, yb, dgn_awetb, wetdensb,
                        ab[AB_T * n], xb, tl);
  }
#pragma unroll
  for (int f = 0; f < MAM4B_NIN; ++f)
    p.xbar[(size_t)f * p.ld + c] = xb[f];
  double *ft_out = p.abar + c;
#pragma unroll
  for (int k = 0; k < NPOP; ++k) {
    ft_out[(FT_PT_IB + k) * n] = tl.pt_ib[k];
    ft_out[(FT_PT_CB + k) * n] = tl.pt_cb[k];
  }
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    ft_out[(FT_DGN_AB + m) * n] = tl.dgn_ab[m];
    ft_out[(FT_DGN_AWETB + m) * n] = tl.dgn_awetb[m];
    ft_out[(FT_QAERWATB + m) * n] = tl.qaerwatb[m];
    ft_out[(FT_WETDENS_WUB + m) * n] = tl.wetdens_wub[m];
  }
}

// Reverse of the water uptake, one thread per (cell, mode) as in the
// forward's mode_kernel: adds the species' cotangents to xbar, updates the
// mode's dry-diameter cotangent and leaves the RH cotangent in abar.
template <int M>
__device__ __forceinline__ void adj_mode_work(const AdjPipeArgs &p, long long c) {
  const StepArgs &a = p.s;
  const size_t n = (size_t)a.ncell;
  double sp[7], spb[7];
#pragma unroll
  for (int s = 0; s < 7; ++s)
    sp[s] = (s < K::nspec(M)) ? __ldg(a.in[MAM4B_IN_AER_I + K::spec0(M) + (s < K::nspec(M) ? s : 0)] + c) : 0.0;
  double *ft = p.abar + c;
  double dgn_ab = ft[(FT_DGN_AB + M) * n];
  const double r = adj::front_rev_mode<M>(
      c_k, sp, a.aux[AUX_RH * n + c], a.out[MAM4B_OUT_DGN_A + M][c], ft[(FT_DGN_AWETB + M) * n],
      ft[(FT_QAERWATB + M) * n], ft[(FT_WETDENS_WUB + M) * n], spb, dgn_ab);
  ft[(FT_DGN_AB + M) * n] = dgn_ab;
  ft[(FT_RHB + M) * n] = r;
#pragma unroll
  for (int s = 0; s < K::nspec(M); ++s)
    p.xbar[(size_t)(MAM4B_IN_AER_I + K::spec0(M) + s) * p.ld + c] += spb[s];
}

// Cells regrouped within the block as in mode_kernel: those below the
// crystallisation humidity (no Kohler reverse) fill warps of their own.
// Launched with 128 threads per block.
__global__ void __launch_bounds__(128) adj_mode_kernel(const __grid_constant__ AdjPipeArgs p) {
  __shared__ int s_perm[128];
  __shared__ unsigned s_cnt[4][2];
  const StepArgs &a = p.s;
  const long long c0 = (long long)blockIdx.x * blockDim.x;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
  long long c = c0 + t;
  const bool valid = c < a.ncell;
  const bool dry = valid && a.aux[AUX_RH * (size_t)a.ncell + c] < K::rh_cryst;
  const unsigned bd = __ballot_sync(0xffffffffu, dry);
  const unsigned bo = __ballot_sync(0xffffffffu, valid && !dry);
  if (lane == 0) {
    s_cnt[w][0] = __popc(bd);
    s_cnt[w][1] = __popc(bo);
  }
  __syncthreads();
  unsigned before_d = 0, before_o = 0, total_d = 0, total = 0;
  for (int k = 0; k < nw; ++k) {
    if (k < w) {
      before_d += s_cnt[k][0];
      before_o += s_cnt[k][1];
    }
    total_d += s_cnt[k][0];
    total += s_cnt[k][0] + s_cnt[k][1];
  }
  if (valid) {
    const unsigned below = (1u << lane) - 1u;
    s_perm[dry ? before_d + __popc(bd & below) : total_d + before_o + __popc(bo & below)] = t;
  }
  __syncthreads();
  if ((unsigned)t >= total)
    return;
  c = c0 + s_perm[t];
  switch (blockIdx.y) {
  case 0: adj_mode_work<0>(p, c); break;
  case 1: adj_mode_work<1>(p, c); break;
  case 2: adj_mode_work<2>(p, c); break;
  default: adj_mode_work<3>(p, c); break;
  }
}

// Last part of the reverse, per cell: RH of water uptake and calcsize.
__global__ void __launch_bounds__(128, 4) adj_fin_kernel(const __grid_constant__ AdjPipeArgs p) {
  const StepArgs &a = p.s;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  const size_t n = (size_t)a.ncell;
  double ai[NPOP], ac[NPOP], aib[NPOP], acb[NPOP];
  double *xbc = p.xbar + c;
#pragma unroll
  for (int k = 0; k < NPOP; ++k) {
    ai[k] = __ldg(a.in[MAM4B_IN_AER_I + k] + c);
    ac[k] = __ldg(a.in[MAM4B_IN_AER_C + k] + c);
    aib[k] = xbc[(size_t)(MAM4B_IN_AER_I + k) * p.ld];
    acb[k] = xbc[(size_t)(MAM4B_IN_AER_C + k) * p.ld];
  }
  double tb = xbc[(size_t)MAM4B_IN_T * p.ld], qvb = xbc[(size_t)MAM4B_IN_QV * p.ld];
  const double *ft = p.abar + c;
  adj::FrontTail tl;
#pragma unroll
  for (int k = 0; k < NPOP; ++k) {
    tl.pt_ib[k] = ft[(FT_PT_IB + k) * n];
    tl.pt_cb[k] = ft[(FT_PT_CB + k) * n];
  }
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    tl.dgn_ab[m] = ft[(FT_DGN_AB + m) * n];
  double rh_wub = 0.0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    rh_wub += ft[(FT_RHB + m) * n];
  adj::front_rev_tail(c_k, ai, ac, __ldg(a.in[MAM4B_IN_QV] + c), __ldg(a.in[MAM4B_IN_T] + c),
                      __ldg(a.in[MAM4B_IN_P] + c), __ldg(a.in[MAM4B_IN_CLD] + c), a.dt, tl, rh_wub,
                      aib, acb, tb, qvb);
  xbc[(size_t)MAM4B_IN_T * p.ld] = tb;
  xbc[(size_t)MAM4B_IN_QV * p.ld] = qvb;
#pragma unroll
  for (int k = 0; k < NPOP; ++k) {
    xbc[(size_t)(MAM4B_IN_AER_I + k) * p.ld] = aib[k];
    xbc[(size_t)(MAM4B_IN_AER_C + k) * p.ld] = acb[k];
  }
}

// ====================================================== derived constants
// Evaluated once per device by a one-thread kernel, with the same
// expressions the reference evaluates inline (and the same math library the
// kernel uses), then copied into constant memory.
__host__ __device__ static double h_vol_from_diam(double d, double sig) {
  return (d * d * d) * exp(4.5 * (log(sig) * log(sig))) * K::pi_sixth;
}

__host__ __device__ static StepConsts make_consts() {
  StepConsts C = {};
  for (int m = 0; m < NMODE; ++m) {
    C.n2v_nom[m] = 1.0 / h_vol_from_diam(K::dnom(m), K::sig(m));
    C.n2v_min[m] = 1.0 / h_vol_from_diam(K::dmax(m), K::sig(m));
    C.n2v_max[m] = 1.0 / h_vol_from_diam(K::dmin(m), K::sig(m));
    for (int s = 0; s < K::nspec(m); ++s)
      C.inv_density[m][s] = 1.0 / K::aero_dens(K::mode_spec(m, s));
    C.log_sig[m] = log(K::sig(m));
  }
  // unit factors: H2SO4 (tracer 2), SOAG (tracer 5), populations 6..30
  auto is_num = [](int i31) { return i31 == 13 || i31 == 18 || i31 == 26 || i31 == 30; };
  const int tr[2] = {2, 5};
  for (int k = 0; k < NPOP + 2; ++k) {
    const int i31 = k < 2 ? tr[k] : 6 + (k - 2);
    C.to_vmr[k] = is_num(i31) ? K::mw_dry_air : K::mw_dry_air / K::adv_mass(i31);
    C.to_mmr[k] = is_num(i31) ? 1.0 / K::mw_dry_air : K::adv_mass(i31) / K::mw_dry_air;
  }
  C.fcvt_soag = K::adv_mass(5) / 150;
  // renaming pair aitken -> accumulation (rename.hpp:393-476)
  {
    const double alnsg = log(K::sig(1));
    C.rn_fac = sqrt(0.5) / alnsg;
    C.rn_v2n_lo_rlx = 1.0 / h_vol_from_diam(K::dmin(1), K::sig(1)) * 27.0;
    C.rn_v2n_hi_rlx = 1.0 / h_vol_from_diam(K::dmax(1), K::sig(1)) / 27.0;
    C.rn_ln_tail_fac = 3.0 * (alnsg * alnsg);
    const double alnsg_d = log(K::sig(0));
    const double cutoff = sqrt(K::dnom(1) * exp(1.5 * (alnsg * alnsg)) * K::dnom(0) *
                               exp(1.5 * (alnsg_d * alnsg_d)));
    C.rn_ln_cutoff = log(cutoff);
    C.rn_threshold = 0.99 * cutoff;
  }
  // nucleation size bounds (mam4_amicphys.hpp:990-1008)
  C.nuc_dplom = exp(0.67 * log(K::dmin(1)) + 0.33 * log(K::dnom(1)));
  {
    const double tmpa = 1770.0 * K::pi / 6.0;
    C.nuc_mass1p_lo = tmpa * (pow(C.nuc_dplom, 3.0));
    C.nuc_mass1p_hi = tmpa * (pow(K::dmax(1), 3.0));
  }
  // aging (aging.hpp:82-150)
  {
    const double mw_soa = 150 / 1000.0, mw_so4 = 115 / 1000.0;
    C.so4_vol = mw_so4 * 1000.0 / 1770.0;
    const double soa_vol = mw_soa * 1000.0 / 1000.0;
    C.soa_fac_eqvhyg = soa_vol * 0.14000000000000001 / 0.50700000000000001;
    const double l = log(K::sig(3));
    C.aging_fac_volsfc = exp(2.5 * (l * l));
  }
  C.geomean_ait_acc = sqrt(C.n2v_nom[1]) * sqrt(C.n2v_nom[0]);
  C.hystfac = 1.0 / dmax(1.0e-5, (K::rh_deliq - K::rh_cryst));
  C.kohler_aa = 2.0e4 * 18.0 * 76.0 / (8.3e7 * 273.0 * 1.0);
  return C;
}

__global__ void init_consts_kernel(StepConsts *out) { *out = make_consts(); }

// ============================================ scratch of the no-alloc step
// mam4b_step_slab_noalloc keeps the pipeline's working memory in this one
// array instead of context allocations: SOA loop state [SOA_FIELDS][ncell],
// hand-off [H_FIELDS][ncell], queue and solver order ([ncell] ints each),
// per-cell values of the size and mode kernels [AUX_FIELDS][ncell], and a
// 256-byte tail with the queue counters and a spare flag word. Host code must not pass the
// name g_noalloc_scratch to a kernel (on the host it is a stand-in, not a
// device address); it uses the address from cudaGetSymbolAddress.
constexpr size_t kNoAllocCells = MAM4B_NOALLOC_MAX_CELLS;
constexpr size_t kNoAllocSoa = 0;
constexpr size_t kNoAllocHand = kNoAllocSoa + (size_t)SOA_FIELDS * kNoAllocCells;
constexpr size_t kNoAllocTask = kNoAllocHand + (size_t)H_FIELDS * kNoAllocCells;
constexpr size_t kNoAllocOrder = kNoAllocTask + kNoAllocCells / 2;
constexpr size_t kNoAllocAux = kNoAllocOrder + kNoAllocCells / 2;
constexpr size_t kNoAllocTail = kNoAllocAux + (size_t)AUX_FIELDS * kNoAllocCells;
constexpr size_t kNoAllocDoubles = kNoAllocTail + 32;
static_assert(kNoAllocCells % 64 == 0, "scratch regions stay 256-byte aligned");
static_assert(sizeof(StepConsts) <= (size_t)SOA_FIELDS * kNoAllocCells * sizeof(double),
              "constants staging fits in the SOA region");
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

// ---- per-process entries (CalcSize, Coagulation): one thread per cell
__global__ void __launch_bounds__(128) calcsize_process_kernel(const __grid_constant__ CalcSizeArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < a.ncell)
    calcsize_process_cell(c_k, a, c);
}

// In two stages, as the step's pair_kernel and post_kernel: one thread per
// (cell, mode pair) for the coefficients (the FP64 exp/pow/sqrt chains,
// with many warps resident), then one thread per cell for the update.
__global__ void __launch_bounds__(128) coag_pair_process_kernel(const __grid_constant__ CoagProcessArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  const CoagTables T = {kCoagBm0ij, kCoagBm3i, kCoagBm0};
  const int p = blockIdx.y;
  const size_t n = (size_t)a.ncell;
  double bij0, bij3, bii0, bjj0;
  coag_process_pair(c_k, T, a, c, p, bij0, bij3, bii0, bjj0);
  a.cc[p * n + c] = bij0;
  a.cc[(3 + p) * n + c] = bij3;
  a.cc[(6 + p) * n + c] = bii0;
  a.cc[(9 + p) * n + c] = bjj0;
}

__global__ void __launch_bounds__(128) coag_process_kernel(const __grid_constant__ CoagProcessArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  const size_t n = (size_t)a.ncell;
  double cc[12];
#pragma unroll
  for (int k = 0; k < 12; ++k)
    cc[k] = a.cc[k * n + c];
  coag_process_update(a, c, cc);
}

// ---- aqueous sulfate chemistry (setsox), one thread per cell
struct SetsoxArgs {
  const double *press, *temp, *lwc, *cldfrc, *cldnum, *xhnm;
  double *qin, *qcw;  // [31][ld]
  double *dso4, *dh2so4;  // [3][ld] or null
  size_t ld;
  long long ncell;
  double dt;
};

__global__ void __launch_bounds__(128) setsox_kernel(const __grid_constant__ SetsoxArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  constexpr int kIn[4] = {0, 1, 2, 3};
  constexpr int kCw[7] = {6, 13, 14, 18, 21, 26, 30};
  double qin[31], qcw[31];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    qin[kIn[k]] = a.qin[(size_t)kIn[k] * a.ld + c];
#pragma unroll
  for (int k = 0; k < 7; ++k)
    qcw[kCw[k]] = a.qcw[(size_t)kCw[k] * a.ld + c];
  double dso4[3], dh2so4[3];
  sox::setsox_cell(a.dt, a.press[c], a.temp[c], a.lwc[c], a.cldfrc[c], a.cldnum[c], a.xhnm[c],
                   qin, qcw, dso4, dh2so4);
#pragma unroll
  for (int k = 1; k < 4; ++k)
    a.qin[(size_t)k * a.ld + c] = qin[k];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    a.qcw[(size_t)sox::so4_cw(m) * a.ld + c] = qcw[sox::so4_cw(m)];
    if (a.dso4)
      a.dso4[(size_t)m * a.ld + c] = dso4[m];
    if (a.dh2so4)
      a.dh2so4[(size_t)m * a.ld + c] = dh2so4[m];
  }
}

// ---- gas-phase chemistry (gas_phase_chemistry), one thread per cell
struct GasChemArgs {
  const double *temp, *photo;
  const double *extfrc, *inv, *het;  // [9][ld], [8][ld], [31][ld]
  double *qq;                        // [31][ld]
  size_t ld;
  long long ncell;
  double dt;
};

// 4 blocks of 128 per SM (128 registers, the solver's spills in L1): 2.0 ms
// on 65,536 x 72 cells against 3.0 ms unconstrained at 247 registers.
__global__ void __launch_bounds__(128, 4) gaschem_kernel(const __grid_constant__ GasChemArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  double ext[gch::kExt], inv[gch::kInv], qq[gch::kTracers];
#pragma unroll
  for (int e = 0; e < gch::kExt; ++e)
    ext[e] = __ldg(a.extfrc + (size_t)e * a.ld + c);
#pragma unroll
  for (int i = 0; i < gch::kInv; ++i)
    inv[i] = __ldg(a.inv + (size_t)i * a.ld + c);
#pragma unroll
  for (int k = 1; k < gch::kTracers; ++k)
    qq[k] = a.qq[(size_t)k * a.ld + c];
  qq[0] = 0.0;  // O3 is neither read nor changed
  // removal rates are read where used (each Newton iteration): after the
  // first read they come from L1, and the solver's registers stay free
  const double *het_c = a.het + c;
  const size_t ld = a.ld;
  auto het = [het_c, ld](int t) { return __ldg(het_c + (size_t)t * ld); };
  gch::gas_chemistry_cell(__ldg(a.temp + c), a.dt, __ldg(a.photo + c), ext, inv, het, qq);
#pragma unroll
  for (int k = 1; k < gch::kTracers; ++k)
    a.qq[(size_t)k * a.ld + c] = qq[k];
}

// ---- aerosol activation (ndrop get_activate_frac), one thread per cell
struct ActivateArgs {
  const double *temp, *aer[NPOP], *rho, *w;
  double *out;  // [17][ld]
  size_t ld;
  long long ncell;
};

__global__ void __launch_bounds__(128) activate_kernel(const __grid_constant__ ActivateArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  double ai[NPOP], out[17];
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    ai[p] = __ldg(a.aer[p] + c);
  const double rho = __ldg(a.rho + c);
  act::activate_cell(c_k, ai, rho, rho, __ldg(a.w + c), __ldg(a.temp + c), out);
#pragma unroll
  for (int k = 0; k < 17; ++k)
    a.out[(size_t)k * a.ld + c] = out[k];
}

// ---- longwave aerosol optics (modal_aero_lw_k) in three launches, as the
// step is split: mode sizes per cell (calcsize, RH), water uptake and the
// Chebyshev polynomials per (cell, mode), then the optical depth per
// (cell, band) summed over the modes in order (one band per block row,
// so a warp's table reads share a band). Scratch rows (per cell):
// dry diameter [4], RH, aerosol water [4], Chebyshev polynomials [4][5].
enum { OS_DGN = 0, OS_RH = 4, OS_QW = 5, OS_CHEB = 9, OS_FIELDS = 29 };
struct OpticsLwArgs {
  const double *in[MAM4B_NIN];
  const double *pdeldry;
  const double *tables;
  double *tau;  // [16][ld]
  double *scr;  // [OS_FIELDS][ncell]
  size_t ld;
  long long ncell;
  double dt;
};

__global__ void __launch_bounds__(128) optics_size_kernel(const __grid_constant__ OpticsLwArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  double ai[NPOP], ac[NPOP], dgn_a[NMODE], pt_i[NPOP], pt_c[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p) {
    ai[p] = __ldg(a.in[MAM4B_IN_AER_I + p] + c);
    ac[p] = __ldg(a.in[MAM4B_IN_AER_C + p] + c);
  }
  calcsize(c_k, ai, ac, a.dt, dgn_a, pt_i, pt_c);
  const size_t n = (size_t)a.ncell;
#pragma unroll
  for (int m = 0; m < NMODE; ++m)
    a.scr[(OS_DGN + m) * n + c] = dgn_a[m];
  a.scr[OS_RH * n + c] = water_uptake_rh(__ldg(a.in[MAM4B_IN_QV] + c), __ldg(a.in[MAM4B_IN_T] + c),
                                         __ldg(a.in[MAM4B_IN_P] + c), __ldg(a.in[MAM4B_IN_CLD] + c));
}

template <int M>
__device__ __forceinline__ void optics_mode_work(const OpticsLwArgs &a, long long c) {
  const size_t n = (size_t)a.ncell;
  double sp[7];
#pragma unroll
  for (int s = 0; s < 7; ++s)
    sp[s] = (s < K::nspec(M)) ? __ldg(a.in[MAM4B_IN_AER_I + K::spec0(M) + (s < K::nspec(M) ? s : 0)] + c) : 0.0;
  double dgn_w, qw, wd;
  water_uptake_mode<M>(c_k, sp, a.scr[OS_RH * n + c], a.scr[(OS_DGN + M) * n + c], dgn_w, qw,
                       wd);
  double cheb[opt::kNcoef];
  opt::mode_cheb(M, dgn_w, cheb);
  a.scr[(OS_QW + M) * n + c] = qw;
#pragma unroll
  for (int k = 0; k < opt::kNcoef; ++k)
    a.scr[(OS_CHEB + opt::kNcoef * M + k) * n + c] = cheb[k];
}

__global__ void __launch_bounds__(128) optics_mode_kernel(const __grid_constant__ OpticsLwArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    return;
  switch (blockIdx.y) {
  case 0: optics_mode_work<0>(a, c); break;
  case 1: optics_mode_work<1>(a, c); break;
  case 2: optics_mode_work<2>(a, c); break;
  default: optics_mode_work<3>(a, c); break;
  }
}

// The band is the grid's fastest index: the blocks of one group of cells
// run back to back for every band, so each cell's inputs come from DRAM
// once and from L2 for the other bands.
// The block's band tables (12 KB) are staged in shared memory first and
// serve every group of cells the block steps (at most 1,024 blocks per
// band): 11.0 -> 10.2 ms per call on 65,536 x 72 cells. (With one group of
// cells per block the staging cost more than it saved: 12.2 ms.)
__global__ void __launch_bounds__(128) optics_band_kernel(const __grid_constant__ OpticsLwArgs a) {
  const int b = blockIdx.x;
  const size_t n = (size_t)a.ncell;
  __shared__ double s_tab[opt::kLwBandDoubles];
  opt::stage_lw_band(a.tables, b, s_tab);
  __syncthreads();
  for (long long cb = blockIdx.y; cb * blockDim.x < a.ncell; cb += gridDim.y) {
  const long long c = cb * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    break;
  double ai[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    ai[p] = (K::numslot(0) == p || K::numslot(1) == p || K::numslot(2) == p || K::numslot(3) == p)
                ? 0.0
                : __ldg(a.in[MAM4B_IN_AER_I + p] + c);
  const double mass = __ldg(a.pdeldry + c) * (1.0 / 9.80616);
  double tau = 0.0;
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    double cheb[opt::kNcoef], specvol[7];
#pragma unroll
    for (int k = 0; k < opt::kNcoef; ++k)
      cheb[k] = a.scr[(OS_CHEB + opt::kNcoef * m + k) * n + c];
    opt::mode_specvol(m, ai, specvol);
    tau += opt::mode_band_tau<opt::LwBand>(s_tab, m, b, specvol, a.scr[(OS_QW + m) * n + c],
                                           cheb, mass);
  }
  a.tau[(size_t)b * a.ld + c] = tau;
  }
}

// ---- shortwave aerosol optics (modal_aero_sw): optics_size_kernel, then
// per (cell, mode) water uptake and the method-1 size parameters, per
// (cell, band) the four mode-summed products, and per column the visible
// optical depth. Scratch rows beyond the longwave ones: Chebyshev
// polynomials [4][5], surface radius [4], its log [4], visible-band
// optical depth of each mode [4].
enum { SS_CHEB = 9, SS_RAD = 29, SS_LOGRAD = 33, SS_AOD = 37, SS_FIELDS = 41 };
struct OpticsSwArgs {
  OpticsLwArgs base;  // inputs, tables, scratch, ld, ncell, dt (base.tau unused)
  double *out;        // [4][14][ld]: tauxar, wa, ga, fa
  double *aodvis;     // [ncol] or null
  int ncol, nlev;
};

template <int M>
__device__ __forceinline__ void optics_sw_mode_work(const OpticsSwArgs &w, long long c) {
  const OpticsLwArgs &a = w.base;
  const size_t n = (size_t)a.ncell;
  double sp[7];
#pragma unroll
  for (int s = 0; s < 7; ++s)
    sp[s] = (s < K::nspec(M)) ? __ldg(a.in[MAM4B_IN_AER_I + K::spec0(M) + (s < K::nspec(M) ? s : 0)] + c) : 0.0;
  double dgn_w, qw, wd;
  water_uptake_mode<M>(c_k, sp, a.scr[OS_RH * n + c], a.scr[(OS_DGN + M) * n + c], dgn_w, qw,
                       wd);
  double cheb[opt::kNcoef], rad, lrad;
  opt::mode_cheb_sw(M, dgn_w, rad, lrad, cheb);
  a.scr[(OS_QW + M) * n + c] = qw;
#pragma unroll
  for (int k = 0; k < opt::kNcoef; ++k)
    a.scr[(SS_CHEB + opt::kNcoef * M + k) * n + c] = cheb[k];
  a.scr[(SS_RAD + M) * n + c] = rad;
  a.scr[(SS_LOGRAD + M) * n + c] = lrad;
}

__global__ void __launch_bounds__(128) optics_sw_mode_kernel(const __grid_constant__ OpticsSwArgs w) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= w.base.ncell)
    return;
  switch (blockIdx.y) {
  case 0: optics_sw_mode_work<0>(w, c); break;
  case 1: optics_sw_mode_work<1>(w, c); break;
  case 2: optics_sw_mode_work<2>(w, c); break;
  default: optics_sw_mode_work<3>(w, c); break;
  }
}

// band-fastest grid, as optics_band_kernel. The block's band tables are
// staged in shared memory first (35 KB: three coefficient tables per mode):
// the table reads of every (cell, band) thread are gathers that would
// otherwise wait on L1/L2 (with at most 1,024 blocks of cells per band:
// 17.1 -> 13.7 ms per call on 65,536 x 72 cells).
__global__ void __launch_bounds__(128) optics_sw_band_kernel(const __grid_constant__ OpticsSwArgs w) {
  const OpticsLwArgs &a = w.base;
  const int b = blockIdx.x;
  const size_t n = (size_t)a.ncell;
  __shared__ double s_tab[opt::kSwBandDoubles];
  opt::stage_sw_band(a.tables, b, s_tab);
  __syncthreads();
  for (long long cb = blockIdx.y; cb * blockDim.x < a.ncell; cb += gridDim.y) {
  const long long c = cb * blockDim.x + threadIdx.x;
  if (c >= a.ncell)
    break;
  double ai[NPOP];
#pragma unroll
  for (int p = 0; p < NPOP; ++p)
    ai[p] = (K::numslot(0) == p || K::numslot(1) == p || K::numslot(2) == p || K::numslot(3) == p)
                ? 0.0
                : __ldg(a.in[MAM4B_IN_AER_I + p] + c);
  const double mass = __ldg(a.pdeldry + c) * (1.0 / 9.80616);
  double sum[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int m = 0; m < NMODE; ++m) {
    double cheb[opt::kNcoef], specvol[7], o[4];
#pragma unroll
    for (int k = 0; k < opt::kNcoef; ++k)
      cheb[k] = a.scr[(SS_CHEB + opt::kNcoef * m + k) * n + c];
    opt::mode_specvol(m, ai, specvol);
    opt::mode_band_sw<opt::SwBand>(s_tab, m, b, specvol, a.scr[(OS_QW + m) * n + c], cheb,
                      a.scr[(SS_RAD + m) * n + c], a.scr[(SS_LOGRAD + m) * n + c], mass, o);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      sum[q] += o[q];
    if (b == opt::kSwDiagBand)
      a.scr[(SS_AOD + m) * n + c] = o[0];
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
    w.out[((size_t)q * opt::kSwBands + b) * a.ld + c] = sum[q];
  }
}

// visible optical depth of each column: its levels' mode optical depths
// summed level by level, mode by mode (the reduction of modal_aero_sw)
__global__ void __launch_bounds__(128) optics_sw_aod_kernel(const __grid_constant__ OpticsSwArgs w) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= w.ncol)
    return;
  const size_t n = (size_t)w.base.ncell;
  double s = 0.0;
  for (int k = 0; k < w.nlev; ++k) {
    const size_t c = (size_t)col * w.nlev + k;
#pragma unroll
    for (int m = 0; m < NMODE; ++m)
      s += w.base.scr[(SS_AOD + m) * n + c];
  }
  w.aodvis[col] = s;
}

// ---- aero_rad_props: tropopause per column, then the volcanic (CMIP6)
// extinction over the modal optics at and above it
struct RadArgs {
  const double *temp, *pmid;     // step input fields (cell = col * nlev + k)
  const double *pint, *zi;       // [col * (nlev + 1) + k]: interface pressure, height
  const double *ext, *ssa, *af;  // [band][ld]: extinction [1/m], albedo, asymmetry
  double *out;                   // shortwave [4][14][ld], longwave [16][ld]
  int *trop;                     // [ncol]
  size_t ld;
  int ncol, nlev;
};

// one warp per column: the lanes compute every layer's lapse-rate
// quantities (the pow-heavy part) into shared memory, then one lane runs
// the scan on them
__global__ void __launch_bounds__(128) tropopause_kernel(const __grid_constant__ RadArgs r) {
  extern __shared__ double tsm[];  // [warps][4][nlev]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nlev = r.nlev;
  const int col = blockIdx.x * (blockDim.x >> 5) + warp;
  if (col >= r.ncol)
    return;  // the whole warp: col is the same on every lane
  double *s = tsm + (size_t)warp * 4 * nlev;
  const size_t c0 = (size_t)col * nlev, i0 = (size_t)col * (nlev + 1);
  auto T = [&](int k) { return __ldg(r.temp + c0 + k); };
  auto P = [&](int k) { return __ldg(r.pmid + c0 + k); };
  for (int k = 1 + lane; k < nlev; k += 32) {
    const rad::LapsePair q = rad::lapse_pair(T, P, k);
    s[k] = q.pmk;
    s[nlev + k] = q.pm;
    s[2 * nlev + k] = q.dtdz;
    s[3 * nlev + k] = q.tm;
  }
  __syncwarp();
  if (lane == 0) {
    auto pair = [&](int k) {
      rad::LapsePair q;
      q.pmk = s[k];
      q.pm = s[nlev + k];
      q.dtdz = s[2 * nlev + k];
      q.tm = s[3 * nlev + k];
      return q;
    };
    auto PI = [&](int k) { return __ldg(r.pint + i0 + k); };
    r.trop[col] = rad::tropopause_level_at(rad::twmo_from_pairs(pair, nlev), PI, nlev);
  }
}

// volcanic_cmip_sw (aero_rad_props.hpp:38-119): at the tropopause level the
// four layer products are averaged with the volcanic ones, above it they
// are replaced (the file's values hold all stratospheric aerosol there)
__global__ void __launch_bounds__(128) volcanic_sw_kernel(const __grid_constant__ RadArgs r) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (long long)r.ncol * r.nlev)
    return;
  const int col = (int)(c / r.nlev), k = (int)(c % r.nlev);
  const int lev = __ldg(r.trop + col);
  if (k > lev)
    return;
  const size_t i0 = (size_t)col * (r.nlev + 1);
  const double thk = __ldg(r.zi + i0 + k) - __ldg(r.zi + i0 + k + 1);
  const size_t ld = r.ld, nb = opt::kSwBands;
  for (int b = 0; b < opt::kSwBands; ++b) {
    const double ext = thk * __ldg(r.ext + b * ld + c);
    const double asym = __ldg(r.af + b * ld + c);
    const double ext_ssa = ext * __ldg(r.ssa + b * ld + c);
    const double ext_ssa_asym = ext_ssa * asym;
    const double v[4] = {ext, ext_ssa, ext_ssa_asym, ext_ssa_asym * asym};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      double *o = r.out + (q * nb + b) * ld + c;
      *o = k == lev ? 0.5 * (*o + v[q]) : v[q];
    }
  }
}

// compute_odap_volcanic_at_troplayer_lw / _above_troplayer_lw
// (aero_rad_props.hpp:121-208): the absorption optical depth, averaged at
// the tropopause level, replaced above it
__global__ void __launch_bounds__(128) volcanic_lw_kernel(const __grid_constant__ RadArgs r) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (long long)r.ncol * r.nlev)
    return;
  const int col = (int)(c / r.nlev), k = (int)(c % r.nlev);
  const int lev = __ldg(r.trop + col);
  if (k > lev)
    return;
  const size_t i0 = (size_t)col * (r.nlev + 1);
  const double thk = __ldg(r.zi + i0 + k) - __ldg(r.zi + i0 + k + 1);
  const size_t ld = r.ld;
  for (int b = 0; b < opt::kLwBands; ++b) {
    double *o = r.out + b * ld + c;
    const double v = thk * __ldg(r.ext + b * ld + c);
    *o = k == lev ? 0.5 * (*o + v) : v;
  }
}

// ---- droplet activation and vertical mixing (ndrop dropmixnuc), one
// block per column; the levels are spread over the block's threads and
// every phase that reads a neighbouring level is separated by a barrier.
struct DropmixArgs {
  const double *in[MAM4B_NIN];  // step input fields: T, p, z, cloud fraction, populations
  const double *mix;            // [MAM4B_DROPMIX_NIN][ld]
  const double *pint, *kvh;     // [col * (nlev + 1) + k]
  double *out;                  // [MAM4B_DROPMIX_NOUT][ld]
  double *act;                  // [DA_FIELDS][ncol * nlev]: activation results
  unsigned *flags;
  size_t ld;
  int ncol, nlev, top_lev, vertical_mix;
  double dt;
};
// activation results of a level, computed ahead by dropmix_act_kernel:
// growing cloud (computed flag, fn, fm) and cloud base (flag, fn, fluxn,
// fluxm)
enum { DA_NEW_OK = 0, DA_NEW_FN = 1, DA_NEW_FM = 5, DA_BASE_OK = 9, DA_BASE_FN = 10,
       DA_BASE_FLUXN = 14, DA_BASE_FLUXM = 18, DA_FIELDS = 22 };

// shared-memory layout of one column (doubles)
enum { DM_CS = 0, DM_DZ, DM_ZN, DM_ZS, DM_EDDY, DM_CSBOT, DM_CSBOT_CSCEN, DM_WTKE, DM_QCLD,
       DM_QNCLD, DM_NSOURCE, DM_EKP, DM_EKM, DM_OVP, DM_OVM, DM_LEVEL_FIELDS };
constexpr int kDmMaxSub = 100000;  // bound on the mixing sub-steps

// The activation and CCN code is called from several phases; kept out of
// line so that the kernel's code stays small enough for the instruction
// cache (inlined copies made instruction fetch the first stall).
__device__ __noinline__ bool dm_activate(const double (&ai)[NPOP], double rho_load, double rho,
                                         double w, double tair, double (&o)[17]) {
  return act::activate_cell(c_k, ai, rho_load, rho, w, tair, o);
}
__device__ __noinline__ void dm_ccn(const double (&ai)[NPOP], const double (&qcb_shift)[NMODE][7],
                                    const double (&qcb_num)[NMODE], double tair, double rho,
                                    double (&ccn)[dmx::kPsat]) {
  dmx::ccn_cell(c_k, ai, qcb_shift, qcb_num, tair, rho, ccn);
}

// The activations of every level (they read only the inputs), one thread
// per cell, ahead of the column kernel: growing cloud activates the
// level's own aerosol, a cloud base the aerosol of the level below.
__global__ void __launch_bounds__(128) dropmix_act_kernel(const __grid_constant__ DropmixArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)a.ncol * a.nlev;
  if (c >= n)
    return;
  const int k = (int)(c % a.nlev);
  double *act = a.act + c;
  act[(size_t)DA_NEW_OK * n] = 0.0;
  act[(size_t)DA_BASE_OK * n] = 0.0;
  if (k < a.top_lev)
    return;
  const double rair = act::kRAir;
  auto IN = [&](int f, long long cc) { return __ldg(a.in[f] + cc); };
  const double temp = IN(MAM4B_IN_T, c), cs = IN(MAM4B_IN_P, c) / (rair * temp);
  const double wtke = dmax(__ldg(a.mix + (size_t)MAM4B_DROPMIX_IN_WSUB * a.ld + c), 0.1);
  const double cldn = IN(MAM4B_IN_CLD, c);
  double ai[NPOP], o[17];
  if (cldn - __ldg(a.mix + (size_t)MAM4B_DROPMIX_IN_CLDO * a.ld + c) > 0.01) {
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      ai[p] = IN(MAM4B_IN_AER_I + p, c);
    const bool ok = dm_activate(ai, cs, cs, wtke, temp, o);
    act[(size_t)DA_NEW_OK * n] = ok ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      act[(size_t)(DA_NEW_FN + m) * n] = o[m];
      act[(size_t)(DA_NEW_FM + m) * n] = o[4 + m];
    }
  }
  if (k < a.nlev - 1 && cldn > 0.01 && cldn - IN(MAM4B_IN_CLD, c + 1) > 0.01) {
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      ai[p] = IN(MAM4B_IN_AER_I + p, c + 1);
    const double cs1 = IN(MAM4B_IN_P, c + 1) / (rair * IN(MAM4B_IN_T, c + 1));
    const bool ok = dm_activate(ai, cs1, cs, wtke, temp, o);
    act[(size_t)DA_BASE_OK * n] = ok ? 1.0 : 0.0;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      act[(size_t)(DA_BASE_FN + m) * n] = o[m];
      act[(size_t)(DA_BASE_FLUXN + m) * n] = o[8 + m];
      act[(size_t)(DA_BASE_FLUXM + m) * n] = o[12 + m];
    }
  }
}

__global__ void __launch_bounds__(128) dropmix_kernel(const __grid_constant__ DropmixArgs a) {
  extern __shared__ double sm[];
  const int col = blockIdx.x, nlev = a.nlev, top = a.top_lev;
  const size_t c0 = (size_t)col * nlev, i0 = (size_t)col * (nlev + 1), ld = a.ld;
  double *lev = sm;                                       // [DM_LEVEL_FIELDS][nlev]
  double *nact = sm + (size_t)DM_LEVEL_FIELDS * nlev;     // [nlev][NMODE]
  double *mact = nact + (size_t)NMODE * nlev;             // [nlev][NMODE]
  double *fnum = mact + (size_t)NMODE * nlev;             // [nlev][NMODE]
  double *raer = fnum + (size_t)NMODE * nlev;             // [2][nlev][NPOP]
  double *rcw = raer + (size_t)2 * NPOP * nlev;           // [2][nlev][NPOP]
  auto L = [&](int f, int k) -> double & { return lev[(size_t)f * nlev + k]; };
  auto R = [&](int b, int k, int p) -> double & { return raer[((size_t)b * nlev + k) * NPOP + p]; };
  auto W = [&](int b, int k, int p) -> double & { return rcw[((size_t)b * nlev + k) * NPOP + p]; };
  auto IN = [&](int f, int k) { return __ldg(a.in[f] + c0 + k); };
  auto MIX = [&](int f, int k) { return __ldg(a.mix + (size_t)f * ld + c0 + k); };
  const size_t ncell = (size_t)a.ncol * nlev;
  auto ACT = [&](int f, int k) { return a.act[(size_t)f * ncell + c0 + k]; };
  auto load_ai = [&](int k, double (&ai)[NPOP]) {
#pragma unroll
    for (int p = 0; p < NPOP; ++p)
      ai[p] = IN(MAM4B_IN_AER_I + p, k);
  };
  const double dt = a.dt, dtinv = 1.0 / dt;
  const double gravity = act::kGravity, rair = act::kRAir;

  // per-level quantities (dropmixnuc :1440-1490)
  for (int k = threadIdx.x; k < nlev; k += blockDim.x) {
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      nact[k * NMODE + m] = 0.0;
      mact[k * NMODE + m] = 0.0;
      fnum[k * NMODE + m] = 0.0;  // factnum starts at zero
    }
    const double cs = IN(MAM4B_IN_P, k) / (rair * IN(MAM4B_IN_T, k));
    const double rpdel = 1.0 / MIX(MAM4B_DROPMIX_IN_PDEL, k);
    L(DM_CS, k) = cs;
    L(DM_DZ, k) = 1.0 / (cs * gravity * rpdel);
    L(DM_ZN, k) = gravity * rpdel;
    L(DM_WTKE, k) = dmax(MIX(MAM4B_DROPMIX_IN_WSUB, k), 0.1);
    L(DM_QCLD, k) = MIX(MAM4B_DROPMIX_IN_NCLDWTR, k);
    L(DM_NSOURCE, k) = 0.0;
    // levels above top_lev keep zero, as the reference's work arrays
    L(DM_ZS, k) = 0.0;
    L(DM_EDDY, k) = 0.0;
    L(DM_CSBOT, k) = 0.0;
    L(DM_CSBOT_CSCEN, k) = 0.0;
    for (int p = 0; p < NPOP; ++p) {
      R(0, k, p) = IN(MAM4B_IN_AER_I + p, k);
      W(0, k, p) = IN(MAM4B_IN_AER_C + p, k);
      R(1, k, p) = 0.0;
      W(1, k, p) = 0.0;
    }
  }
  __syncthreads();
  for (int k = top + threadIdx.x; k < nlev; k += blockDim.x) {
    if (k < nlev - 1) {
      L(DM_ZS, k) = 1.0 / (IN(MAM4B_IN_ZM, k) - IN(MAM4B_IN_ZM, k + 1));
      L(DM_EDDY, k) = bound(0.01, 100.0, __ldg(a.kvh + i0 + k + 1));
      L(DM_CSBOT, k) =
          2.0 * __ldg(a.pint + i0 + k + 1) / (rair * (IN(MAM4B_IN_T, k) + IN(MAM4B_IN_T, k + 1)));
      L(DM_CSBOT_CSCEN, k) = L(DM_CSBOT, k) / L(DM_CS, k);
    } else {
      L(DM_ZS, k) = 1.0 / (IN(MAM4B_IN_ZM, k - 1) - IN(MAM4B_IN_ZM, k));
      L(DM_EDDY, k) = 0.0;
      L(DM_CSBOT, k) = IN(MAM4B_IN_P, k) / (rair * IN(MAM4B_IN_T, k));
      L(DM_CSBOT_CSCEN, k) = 1.0;
    }
  }
  __syncthreads();

  // new cloud (update_from_newcld): shrinking cloud releases, growing cloud
  // activates the level's own aerosol
  for (int k = top + threadIdx.x; k < nlev; k += blockDim.x) {
    const double cldn = IN(MAM4B_IN_CLD, k), cldo = MIX(MAM4B_DROPMIX_IN_CLDO, k);
    const double delt_cld = cldn - cldo;
    double &qcld = L(DM_QCLD, k), &nsource = L(DM_NSOURCE, k);
    if (cldn < cldo) {
      nsource += qcld * (cldn - cldo) / cldo * dtinv;
      qcld *= (1.0 + (cldn - cldo) / cldo);
      const double frac = (cldn - cldo) / cldo;
#pragma unroll
      for (int m = 0; m < NMODE; ++m)
        for (int l = 0; l <= K::nspec(m); ++l) {
          const int p = dmx::pop_of(m, l);
          const double dact = W(0, k, p) * frac;
          W(0, k, p) += dact;
          R(0, k, p) -= dact;
        }
    }
    if (cldn - cldo > 0.01) {
      double ai[NPOP], fm[NMODE];
      load_ai(k, ai);
      const bool ok = ACT(DA_NEW_OK, k) != 0.0;
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        if (ok)
          fnum[k * NMODE + m] = ACT(DA_NEW_FN + m, k);
        fm[m] = ok ? ACT(DA_NEW_FM + m, k) : 0.0;  // else factnum as it was
      }
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        const int pn = K::numslot(m);
        const double dact = delt_cld * fnum[k * NMODE + m] * ai[pn];
        qcld += dact;
        nsource += dact * dtinv;
        W(0, k, pn) += dact;
        R(0, k, pn) -= dact;
        const double fm_delt = delt_cld * fm[m];
        for (int l = 1; l <= K::nspec(m); ++l) {
          const int p = dmx::pop_of(m, l);
          const double d = fm_delt * ai[p];
          W(0, k, p) += d;
          R(0, k, p) -= d;
        }
      }
    }
  }
  __syncthreads();

  // cloud-base activation (update_from_cldn_profile). A level reads the
  // number of the level below it before that level clears its cloud, as
  // in the reference's ascending order: reads and activation first, the
  // clearing after a barrier.
  for (int k = top + threadIdx.x; k < nlev - 1; k += blockDim.x) {
    const double cldn = IN(MAM4B_IN_CLD, k), cldn1 = IN(MAM4B_IN_CLD, k + 1);
    if (cldn > 0.01 && cldn - cldn1 > 0.01) {
      L(DM_EDDY, k) = L(DM_WTKE, k) / L(DM_ZS, k);
      const double cs = L(DM_CS, k);
      const bool ok = ACT(DA_BASE_OK, k) != 0.0;
      const double delz_cld = cldn - cldn1;
      double fluxntot = 0.0;
      const double crdz = L(DM_CSBOT_CSCEN, k) / L(DM_DZ, k);
#pragma unroll
      for (int m = 0; m < NMODE; ++m) {
        if (ok)
          fnum[k * NMODE + m] = ACT(DA_BASE_FN + m, k);
        const double fluxn = ok ? ACT(DA_BASE_FLUXN + m, k) : 0.0;
        const double fluxm = ok ? ACT(DA_BASE_FLUXM + m, k) : 0.0;
        nact[k * NMODE + m] += fluxn * crdz * delz_cld;
        mact[k * NMODE + m] += fluxm * crdz * delz_cld;
        fluxntot += fluxn * delz_cld * R(0, k + 1, K::numslot(m)) * cs;
      }
      L(DM_NSOURCE, k) += fluxntot / (cs * L(DM_DZ, k));
    }
  }
  __syncthreads();
  for (int k = top + threadIdx.x; k < nlev - 1; k += blockDim.x) {
    if (!(IN(MAM4B_IN_CLD, k) > 0.01)) {
      L(DM_NSOURCE, k) -= L(DM_QCLD, k) * dtinv;
      L(DM_QCLD, k) = 0.0;
      for (int p = 0; p < NPOP; ++p) {
        R(0, k, p) += W(0, k, p);
        W(0, k, p) = 0.0;
      }
    }
  }
  __syncthreads();

  // mixing set-up (update_from_explmix :1192-1225); the time-step bound is
  // a minimum over levels, the same in any order
  double dtmin = 1.79769313486231570e+308;
  for (int k = top + threadIdx.x; k < nlev; k += blockDim.x) {
    const int kp1 = k + 1 < nlev ? k + 1 : nlev - 1, km1 = k - 1 > top ? k - 1 : top;
    const double cld = IN(MAM4B_IN_CLD, k), cldp = IN(MAM4B_IN_CLD, kp1), cldm = IN(MAM4B_IN_CLD, km1);
    L(DM_OVP, k) = cldp > 1e-10 ? dmin(cld / cldp, 1.0) : 1.0;
    L(DM_OVM, k) = cldm > 1e-10 ? dmin(cld / cldm, 1.0) : 1.0;
    const double ekp = L(DM_ZN, k) * L(DM_EDDY, k) * L(DM_CSBOT, k) * L(DM_ZS, k);
    // top_lev >= 1: level k - 1 exists (above top_lev its terms are zero)
    const double ekm = L(DM_ZN, k) * L(DM_EDDY, k - 1) * L(DM_CSBOT, k - 1) * L(DM_ZS, km1);
    L(DM_EKP, k) = ekp;
    L(DM_EKM, k) = ekm;
    const double tinv = ekp + ekm;
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
      nact[k * NMODE + m] = dmin(nact[k * NMODE + m], ekp);
      mact[k * NMODE + m] = dmin(mact[k * NMODE + m], ekp);
    }
    if (tinv > 1e-6)
      dtmin = dmin(dtmin, 1.0 / tinv);
  }
  // block-wide minimum: warp shuffles, then one value per warp in shared memory
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1)
    dtmin = dmin(dtmin, __shfl_down_sync(0xffffffffu, dtmin, o));
  if ((threadIdx.x & 31) == 0)
    red[threadIdx.x >> 5] = dtmin;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      v = dmin(v, red[w]);
    red[0] = v;
  }
  __syncthreads();
  dtmin = red[0];
  double dtmix = 0.9 * dtmin;
  const double nsub_d = dt / dtmix + 1;
  int nsubmix = nsub_d < (double)kDmMaxSub ? (int)nsub_d : kDmMaxSub;
  if (!(nsub_d < (double)kDmMaxSub) && threadIdx.x == 0)
    atomicOr(a.flags, MAM4B_FLAG_NONFINITE_OUTPUT);
  dtmix = dt / nsubmix;

  // sub-steps: one work item per (level, population) plus one per level for
  // the droplet number, spread over the block; populations and droplet
  // number double-buffered (nsav read, nnew written), one barrier per step
  int nsav = 0, nnew = 1;
  auto Q = [&](int b, int k) -> double & { return L(b ? DM_QNCLD : DM_QCLD, k); };
  const int nitem = (nlev - top) * (NPOP + 1);
  for (int isub = 0; isub < nsubmix; ++isub) {
    if (isub > 0) {
      const int t = nsav;
      nsav = nnew;
      nnew = t;
    }
    for (int t = threadIdx.x; t < nitem; t += blockDim.x) {
      const int k = top + t / (NPOP + 1), j = t % (NPOP + 1);
      const int kp1 = k + 1 < nlev ? k + 1 : nlev - 1, km1 = k - 1 > top ? k - 1 : top;
      const double ekp = L(DM_EKP, k), ekm = L(DM_EKM, k), ovp = L(DM_OVP, k), ovm = L(DM_OVM, k);
      if (j == NPOP) {
        double srcn = 0.0;
#pragma unroll
        for (int m = 0; m < NMODE; ++m) {
          const int pn = K::numslot(m);
          srcn += nact[k * NMODE + m] * R(nsav, kp1, pn);
          if (k == nlev - 1) {
            const double tmpa = R(nsav, k, pn) * nact[k * NMODE + m] + W(nsav, k, pn) * nact[k * NMODE + m];
            srcn += dmax(0.0, tmpa);
          }
        }
        Q(nnew, k) = a.vertical_mix ? dmx::explmix(Q(nsav, km1), Q(nsav, k), Q(nsav, kp1), srcn,
                                                   ekp, ekm, ovp, ovm, dtmix)
                                    : Q(nsav, k);
      } else {
        const int p = j, m = dmx::mode_of(p);
        double source;
        if (k < nlev - 1) {
          const double act = p == K::numslot(m) ? nact[k * NMODE + m] : mact[k * NMODE + m];
          source = act * R(nsav, kp1, p);
        } else {
          const double tmpa = R(nsav, k, p) * nact[k * NMODE + m] + W(nsav, k, p) * nact[k * NMODE + m];
          source = dmax(0.0, tmpa);
        }
        W(nnew, k, p) = dmx::explmix(W(nsav, km1, p), W(nsav, k, p), W(nsav, kp1, p), source, ekp,
                                     ekm, ovp, ovm, dtmix);
        if (a.vertical_mix)
          R(nnew, k, p) = dmx::explmix_act(R(nsav, km1, p), R(nsav, k, p), R(nsav, kp1, p), source,
                                           ekp, ekm, ovp, ovm, dtmix, W(nsav, km1, p),
                                           W(nsav, kp1, p));
      }
    }
    __syncthreads();
  }

  // clear-sky levels give their cloud-borne aerosol back; outputs
  for (int k = threadIdx.x; k < nlev; k += blockDim.x) {
    const size_t c = c0 + k;
    double *o = a.out + c;
    o[(size_t)MAM4B_DROPMIX_OUT_WTKE * ld] = L(DM_WTKE, k);
    if (k < top) {
      o[(size_t)MAM4B_DROPMIX_OUT_QCLD * ld] = L(DM_QCLD, k);
      for (int f = MAM4B_DROPMIX_OUT_TENDND; f < MAM4B_DROPMIX_NOUT; ++f)
        if (f != MAM4B_DROPMIX_OUT_WTKE)
          o[(size_t)f * ld] = 0.0;
      continue;
    }
    const double ncldwtr = MIX(MAM4B_DROPMIX_IN_NCLDWTR, k);
    if (IN(MAM4B_IN_CLD, k) == 0.0) {
      Q(nnew, k) = 0.0;
      for (int p = 0; p < NPOP; ++p) {
        R(nnew, k, p) += W(nnew, k, p);
        W(nnew, k, p) = 0.0;
      }
    }
    const double qcld = Q(nnew, k);
    o[(size_t)MAM4B_DROPMIX_OUT_QCLD * ld] = qcld;
    o[(size_t)MAM4B_DROPMIX_OUT_NDROPMIX * ld] = (qcld - ncldwtr) * dtinv - L(DM_NSOURCE, k);
    o[(size_t)MAM4B_DROPMIX_OUT_TENDND * ld] = (dmax(qcld, 1.e-6) - ncldwtr) * dtinv;
    o[(size_t)MAM4B_DROPMIX_OUT_NDROPCOL * ld] = ncldwtr * MIX(MAM4B_DROPMIX_IN_PDEL, k) / gravity;
    o[(size_t)MAM4B_DROPMIX_OUT_NSOURCE * ld] = L(DM_NSOURCE, k);
#pragma unroll
    for (int m = 0; m < NMODE; ++m)
      o[(size_t)(MAM4B_DROPMIX_OUT_FACTNUM + m) * ld] = fnum[k * NMODE + m];
    double ai[NPOP], qcb_shift[NMODE][7], qcb_num[NMODE];
    load_ai(k, ai);
#pragma unroll
    for (int m = 0; m < NMODE; ++m) {
#pragma unroll
      for (int s = 0; s < 7; ++s)
        qcb_shift[m][s] = 0.0;
      for (int l = 0; l <= K::nspec(m); ++l) {
        const int p = dmx::pop_of(m, l);
        const double q = dmax(W(nnew, k, p), 0.0);
        o[(size_t)(MAM4B_DROPMIX_OUT_QQCW + p) * ld] = q;
        o[(size_t)(MAM4B_DROPMIX_OUT_PTEND + p) * ld] = (R(nnew, k, p) - ai[p]) * dtinv;
        if (l == 0)
          qcb_num[m] = q;
        else if (l < K::nspec(m))
          qcb_shift[m][l] = q;  // species l - 1's mass, read as species l
      }
    }
    double ccn[dmx::kPsat];
    dm_ccn(ai, qcb_shift, qcb_num, IN(MAM4B_IN_T, k), L(DM_CS, k), ccn);
#pragma unroll
    for (int l = 0; l < dmx::kPsat; ++l)
      o[(size_t)(MAM4B_DROPMIX_OUT_CCN + l) * ld] = ccn[l];
  }
}

}  // namespace mam4b

// =============================================================== C ABI
namespace mam4b {
// Column gather/scatter of mam4b_step_columns: tab[f * ncol + col] points
// at column col of field f (nlev doubles); slab is [nfield][ncol * nlev].
__global__ void __launch_bounds__(128) gather_columns_kernel(const double *const *tab, double *slab,
                                                             int ncol, int nlev) {
  const long long ncell = (long long)ncol * nlev;
  const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncell)
    return;
  const int f = blockIdx.y;
  const int col = (int)(cell / nlev), lev = (int)(cell - (long long)col * nlev);
  slab[(size_t)f * ncell + cell] = tab[(size_t)f * ncol + col][lev];
}
// first nadd fields added to their columns, the rest written; null columns skipped
__global__ void __launch_bounds__(128) scatter_columns_kernel(double *const *tab,
                                                              const double *slab, int ncol,
                                                              int nlev, int nadd) {
  const long long ncell = (long long)ncol * nlev;
  const long long cell = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= ncell)
    return;
  const int f = blockIdx.y;
  const int col = (int)(cell / nlev), lev = (int)(cell - (long long)col * nlev);
  double *p = tab[(size_t)f * ncol + col];
  if (!p)
    return;
  const double v = slab[(size_t)f * ncell + cell];
  p[lev] = (f < nadd) ? p[lev] + v : v;
}
}  // namespace mam4b

using namespace mam4b;

// Host-buffer path: columns are processed in chunks of about kHostChunkCells
// cells on one stream per stage: all host->device copies back to back on
// the copy-in stream, each chunk's kernels on one of kComputeStreams
// streams once its inputs have arrived, each chunk's device->host copy on
// the copy-out stream once its kernels are done. Both copy engines stay
// busy from the first chunk to the last (the copies, not the kernels,
// bound this path); the chunks' kernels overlap, which hides the tail of
// each chunk's SOA solver (its longest loop).
constexpr int kComputeStreams = 4;
constexpr int kHostStreams = 2 + kComputeStreams;  // in, compute..., out
constexpr long long kHostChunkCells = 1LL << 18;
constexpr int kMaxChunks = 64;

struct mam4b_ctx {
  mam4b_config cfg;
  int device;
  unsigned *d_flags;
  cudaStream_t last_stream;
  char err[256];
  std::atomic<unsigned long long> launches;
  // host-path scratch (device slabs), grown on demand
  double *d_in, *d_out, *d_pblh;
  size_t cap_in, cap_out, cap_pblh;
  // pipeline scratch: SOA loop state, hand-off, queued cells, counters
  // (grown on demand)
  double *d_soa;
  double *d_hand;
  int *d_task, *d_order;
  double *d_aux;
  unsigned *d_counters;  // CNT_WORDS per chunk of the host path
  size_t cap_cells;
  int sms;              // SMs of the device (persistent solver grid = sms x blocks per SM)
  mam4b_tuning tune;    // launch shape of the forward pipeline
  // graph mode (mam4b_set_graph_mode): the pipeline of the last call,
  // captured once and replayed while the call's arguments stay the same
  bool use_graph;
  cudaStream_t cap_stream;
  cudaGraph_t graph;
  cudaGraphExec_t graph_exec;
  StepArgs graph_args;
  int graph_precision;
  mam4b_tuning graph_tune;
  // adjoint: SOA checkpoints of the persistent threads (allocated on first
  // use) and the cotangent scratch of the pipelined adjoint (grown)
  double *d_ck;
  int adj_grid;
  double *d_ck2, *d_abar, *d_lbar;
  int adj_ck;           // SOA checkpoint interval of the pipelined adjoint (0 = 1)
  int ck2_slots;        // SOA states per solver thread d_ck2 holds
  int *d_npass;         // [cap_adj]: passes of each SOA loop
  double *d_optics_lw;  // longwave optics tables (opt::kTableDoubles), set by the host
  double *d_optics_sw;  // shortwave optics tables (opt::kSwTableDoubles), set by the host
  double *d_optics_scr; // optics per-cell sizes (SS_FIELDS per cell), grown
  size_t cap_optics_scr;
  int *d_trop;          // [cap_trop]: tropopause level per column (aero_rad_props)
  size_t cap_trop;
  double *d_dmx;        // dropmixnuc activation results (DA_FIELDS per cell), grown
  double *d_coag_cc;    // coagulation process: 12 coefficients per cell, grown
  size_t cap_coag_cc;
  size_t cap_dmx;
  unsigned *d_bins;     // [2 kPassBins]: loops per pass count, start offsets
  // mam4b_step_columns: device pointer tables of the columns (grown) and
  // their host staging
  void **d_coltab;
  size_t cap_coltab;
  std::vector<void *> h_coltab;
  int adj_soa_grid;
  size_t cap_adj;
  // host path: copy/compute streams and their events (created on first use)
  cudaStream_t hs[kHostStreams];
  cudaEvent_t ev_start, ev_done[kHostStreams];
  cudaEvent_t ev_in[kMaxChunks], ev_comp[kMaxChunks];  // per chunk: inputs in, kernels done
  bool host_streams;
};

namespace {
std::mutex g_init_mu;
bool g_consts_ready[64];

mam4b_status set_err(mam4b_ctx *ctx, mam4b_status st, const char *what, cudaError_t e) {
  if (ctx)
    snprintf(ctx->err, sizeof(ctx->err), "%s: %s", what,
             e == cudaSuccess ? "invalid argument" : cudaGetErrorString(e));
  return st;
}

cudaError_t ensure_consts(int dev) {
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (dev < 0 || dev >= 64)
    return cudaErrorInvalidDevice;
  if (g_consts_ready[dev])
    return cudaSuccess;
  StepConsts *d_tmp = nullptr;
  cudaError_t e = cudaMalloc(&d_tmp, sizeof(StepConsts));
  if (e == cudaSuccess) {
    init_consts_kernel<<<1, 1>>>(d_tmp);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaDeviceSynchronize();
  if (e == cudaSuccess)
    e = cudaMemcpyToSymbol(c_k, d_tmp, sizeof(StepConsts), 0, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess)
    e = cudaDeviceSynchronize();
  cudaFree(d_tmp);
  if (e == cudaSuccess)
    g_consts_ready[dev] = true;
  return e;
}

bool valid_config(const mam4b_config *c) {
  return c && (c->gaexch_h2so4_uptake_optaa == 1 || c->gaexch_h2so4_uptake_optaa == 2);
}

cudaError_t ensure_solver_scratch(mam4b_ctx *ctx, size_t ncell) {
  cudaError_t e = cudaSuccess;
  if (!ctx->d_counters)
    e = cudaMalloc(&ctx->d_counters, (size_t)CNT_WORDS * kMaxChunks * sizeof(unsigned));
  if (e != cudaSuccess || ctx->cap_cells >= ncell)
    return e;
  cudaFree(ctx->d_soa);
  cudaFree(ctx->d_hand);
  cudaFree(ctx->d_task);
  cudaFree(ctx->d_order);
  cudaFree(ctx->d_aux);
  ctx->d_aux = nullptr;
  ctx->d_soa = nullptr;
  ctx->d_hand = nullptr;
  ctx->d_task = nullptr;
  ctx->d_order = nullptr;
  ctx->cap_cells = 0;
  e = cudaMalloc(&ctx->d_soa, (size_t)SOA_FIELDS * ncell * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMalloc(&ctx->d_hand, (size_t)H_FIELDS * ncell * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMalloc(&ctx->d_task, ncell * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMalloc(&ctx->d_order, ncell * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMalloc(&ctx->d_aux, (size_t)AUX_FIELDS * ncell * sizeof(double));
  if (e == cudaSuccess)
    ctx->cap_cells = ncell;
  return e;
}

void set_step_config(const mam4b_ctx *ctx, StepArgs &a, long long ncell, int nlev, double dt) {
  a.flags = ctx->d_flags;
  a.ncell = ncell;
  a.nlev = nlev;
  a.dt = dt;
  a.do_cond = ctx->cfg.do_cond;
  a.do_rename = ctx->cfg.do_rename;
  a.do_newnuc = ctx->cfg.do_newnuc;
  a.do_coag = ctx->cfg.do_coag;
  a.optaa = ctx->cfg.gaexch_h2so4_uptake_optaa;
  a.nmono = ctx->cfg.n_so4_monolayers_pcage;
}

// Pipeline scratch of the cells [c0, c0 + a.ncell) of a batch (one host
// chunk; c0 = 0 for a whole batch); chunk selects its counters.
void set_step_scratch(const mam4b_ctx *ctx, StepArgs &a, size_t c0, int chunk) {
  a.soa = ctx->d_soa + (size_t)SOA_FIELDS * c0;
  a.hand = ctx->d_hand + (size_t)H_FIELDS * c0;
  a.task = ctx->d_task + c0;
  a.order = ctx->d_order + c0;
  a.aux = ctx->d_aux + (size_t)AUX_FIELDS * c0;
  a.counters = ctx->d_counters + (size_t)CNT_WORDS * chunk;
}

// ----------------------------------------------------- launch shapes
// The forward pipeline's launch shape (mam4b_tuning): block sizes, register
// caps (compiled variants of the whole-cell kernels) and cells per thread.
// Every shape runs the same arithmetic, so results are bit for bit equal.
bool valid_block(int b, int regs) {
  return (b == 64 || b == 128 || b == 256) && (long long)b * regs <= 65536;
}
bool valid_tuning(const mam4b_tuning &t) {
  return (t.size_regs == 255 || t.size_regs == 128 || t.size_regs == 96) &&
         valid_block(t.size_block, t.size_regs) &&
         valid_block(t.mode_block, 64) && valid_block(t.pair_block, 128) &&
         (t.pre_regs == 255 || t.pre_regs == 168 || t.pre_regs == 128) &&
         valid_block(t.pre_block, t.pre_regs) &&
         (t.post_regs == 255 || t.post_regs == 168 || t.post_regs == 128) &&
         valid_block(t.post_block, t.post_regs) &&
         (t.soa_regs == 64 || t.soa_regs == 96 || t.soa_regs == 128) &&
         (t.soa_block == 128 || t.soa_block == 256) &&
         (long long)t.soa_block * t.soa_regs <= 65536 && t.soa_blocks_per_sm >= 1 &&
         t.soa_blocks_per_sm <= 16 &&
         (t.cells_per_thread == 1 || t.cells_per_thread == 2 || t.cells_per_thread == 4) &&
         (t.inline_scale == 0 || t.inline_scale == 1 || t.inline_scale == 4 ||
          t.inline_scale == 16 || t.inline_scale == 64);
}

unsigned grid_for(long long n, int block, int cpt) {
  const long long per = (long long)block * cpt;
  const long long g = (n + per - 1) / per;
  return (unsigned)(g > 0 ? g : 1);
}

// Stage launchers. Stage order: 0 size, 1 mode, 2 pair, 3 pre, 4 soa, 5 post.
template <bool LOOP>
void launch_size_t(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s) {
  const unsigned g = grid_for(a.ncell, t.size_block, t.cells_per_thread);
  if (t.size_regs == 96)
    size_kernel<96, LOOP><<<g, t.size_block, 0, s>>>(a);
  else if (t.size_regs == 128)
    size_kernel<128, LOOP><<<g, t.size_block, 0, s>>>(a);
  else
    size_kernel<255, LOOP><<<g, t.size_block, 0, s>>>(a);
}
void launch_size(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s) {
  if (t.cells_per_thread > 1)
    launch_size_t<true>(t, a, s);
  else
    launch_size_t<false>(t, a, s);
}
void launch_mode(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s, bool mixed) {
  const dim3 g(grid_for(a.ncell, t.mode_block, 1), NMODE);
  if (mixed)
    mode_kernel<true><<<g, t.mode_block, 0, s>>>(a);
  else
    mode_kernel<false><<<g, t.mode_block, 0, s>>>(a);
}
void launch_pair(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s, bool mixed) {
  const dim3 g(grid_for(a.ncell, t.pair_block, 1), 3);
  if (mixed)
    pair_kernel<true><<<g, t.pair_block, 0, s>>>(a);
  else
    pair_kernel<false><<<g, t.pair_block, 0, s>>>(a);
}
template <bool MIXED, bool FUSE>
void launch_pre_t(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s) {
  const unsigned g = grid_for(a.ncell, t.pre_block, 1);
  if (t.pre_regs == 128)
    pre_kernel<128, MIXED, FUSE><<<g, t.pre_block, 0, s>>>(a);
  else if (t.pre_regs == 168)
    pre_kernel<168, MIXED, FUSE><<<g, t.pre_block, 0, s>>>(a);
  else
    pre_kernel<255, MIXED, FUSE><<<g, t.pre_block, 0, s>>>(a);
}
// fuse: cells with short SOA loops finish in pre (a.inline_scale > 0)
void launch_pre(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s, bool mixed = false,
                bool fuse = false) {
  if (mixed)
    fuse ? launch_pre_t<true, true>(t, a, s) : launch_pre_t<true, false>(t, a, s);
  else
    fuse ? launch_pre_t<false, true>(t, a, s) : launch_pre_t<false, false>(t, a, s);
}
template <int SOA>
void launch_soa_t(const mam4b_tuning &t, int sms, const StepArgs &a, cudaStream_t s) {
  const unsigned g = (unsigned)(sms * t.soa_blocks_per_sm);
  if (t.soa_regs == 128)
    soa_kernel<SOA, 128><<<g, t.soa_block, 0, s>>>(a);
  else if (t.soa_regs == 96)
    soa_kernel<SOA, 96><<<g, t.soa_block, 0, s>>>(a);
  else
    soa_kernel<SOA, 64><<<g, t.soa_block, 0, s>>>(a);
}
// the SOA loop of each precision (mam4b_precision)
void launch_soa(const mam4b_tuning &t, int sms, const StepArgs &a, cudaStream_t s,
                int precision) {
  if (precision == MAM4B_MIXED_FAST)
    launch_soa_t<2>(t, sms, a, s);
  else if (precision == MAM4B_MIXED)
    launch_soa_t<1>(t, sms, a, s);
  else
    launch_soa_t<0>(t, sms, a, s);
}
template <bool LOOP>
void launch_post_t(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s) {
  // one thread per queued slot at most; the kernel reads the queue length
  const unsigned g = grid_for(a.ncell, t.post_block, t.cells_per_thread);
  if (t.post_regs == 255)
    post_kernel<255, LOOP><<<g, t.post_block, 0, s>>>(a);
  else if (t.post_regs == 168)
    post_kernel<168, LOOP><<<g, t.post_block, 0, s>>>(a);
  else
    post_kernel<128, LOOP><<<g, t.post_block, 0, s>>>(a);
}
void launch_post(const mam4b_tuning &t, const StepArgs &a, cudaStream_t s) {
  if (t.cells_per_thread > 1)
    launch_post_t<true>(t, a, s);
  else
    launch_post_t<false>(t, a, s);
}

// Clears the counters and queues the pipeline kernels on s in the
// arithmetic of `precision` (mam4b_precision) with launch shape t on a
// device of `sms` SMs. With ch (FP64 only) the cells' chemistry runs in
// the pre stage. With ev (7 events), ev[k] is recorded before stage k and
// ev[6] after the last: the per-stage times of mam4b_autotune.
cudaError_t launch_pipeline_t(const mam4b_tuning &t, int sms, const StepArgs &a_in,
                              cudaStream_t s, int precision, const ChemArgs *ch, cudaEvent_t *ev,
                              std::atomic<unsigned long long> *launches) {
  StepArgs a = a_in;
  a.mixed = precision != MAM4B_FP64;
  // short SOA loops finish in pre unless the adjoint needs every loop's
  // pass count (npass) or the loop runs in FP32 (MIXED_FAST)
  const bool fuse = t.inline_scale > 0 && !a.npass && precision != MAM4B_MIXED_FAST;
  a.inline_scale = fuse ? (double)t.inline_scale : 0.0;
  cudaError_t e = cudaMemsetAsync(a.counters, 0, CNT_WORDS * sizeof(unsigned), s);
  if (e != cudaSuccess)
    return e;
  if (!a.do_cond) {
    // no SOA loop to pipeline
    const int block = 128;
    const unsigned grid = (unsigned)((a.ncell + block - 1) / block);
    if (ch)
      chem_step_kernel<<<grid, block, 0, s>>>(a, *ch);
    else
      full_kernel<false><<<grid, block, 0, s>>>(a);
    e = cudaGetLastError();
    if (e == cudaSuccess && launches)
      *launches += 1;
    return e;
  }
  const bool mixed = precision != MAM4B_FP64;
  auto mark = [&](int k) {
    if (ev)
      cudaEventRecord(ev[k], s);
  };
  mark(0);
  launch_size(t, a, s);
  mark(1);
  launch_mode(t, a, s, mixed);
  mark(2);
  launch_pair(t, a, s, mixed);
  mark(3);
  if (ch) {
    const int block = 128;
    pre_chem_kernel<<<(unsigned)((a.ncell + block - 1) / block), block, 0, s>>>(a, *ch);
  } else {
    launch_pre(t, a, s, mixed, fuse);
  }
  mark(4);
  launch_soa(t, sms, a, s, precision);
  mark(5);
  // the adjoint's forward (npass set) has no post stage: adj_post_kernel
  // recomputes the suffix from the hand-off, and the forward's outputs are
  // not returned
  if (!a.npass)
    launch_post(t, a, s);
  mark(6);
  e = cudaGetLastError();
  if (e == cudaSuccess && launches)
    *launches += a.npass ? 5 : 6;
  return e;
}

void drop_graph(mam4b_ctx *ctx) {
  if (ctx->graph_exec)
    cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph)
    cudaGraphDestroy(ctx->graph);
  ctx->graph_exec = nullptr;
  ctx->graph = nullptr;
}

// The forward pipeline with the context's launch shape. With graph mode on
// and `graph` set (mam4b_step's device entry), the pipeline is captured on
// a private stream into a CUDA graph, instantiated once and replayed on s;
// a call with other arguments (pointers, sizes, precision, launch shape)
// recaptures and updates the instantiated graph in place, or
// re-instantiates it when the update is refused.
cudaError_t launch_pipeline(mam4b_ctx *ctx, const StepArgs &a, cudaStream_t s, int precision,
                            const ChemArgs *ch = nullptr, bool graph = false) {
  if (!graph || !ctx->use_graph || ch || !a.do_cond)
    return launch_pipeline_t(ctx->tune, ctx->sms, a, s, precision, ch, nullptr, &ctx->launches);
  const bool same = ctx->graph_exec && memcmp(&ctx->graph_args, &a, sizeof(StepArgs)) == 0 &&
                    ctx->graph_precision == precision &&
                    memcmp(&ctx->graph_tune, &ctx->tune, sizeof(mam4b_tuning)) == 0;
  cudaError_t e = cudaSuccess;
  if (!same) {
    if (!ctx->cap_stream)
      e = cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking);
    cudaGraph_t g = nullptr;
    if (e == cudaSuccess)
      e = cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
      const cudaError_t el = launch_pipeline_t(ctx->tune, ctx->sms, a, ctx->cap_stream, precision,
                                               nullptr, nullptr, nullptr);
      e = cudaStreamEndCapture(ctx->cap_stream, &g);
      if (e == cudaSuccess)
        e = el;
    }
    if (e == cudaSuccess && ctx->graph_exec) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(ctx->graph_exec, g, &info) != cudaSuccess) {
        (void)cudaGetLastError();  // the refusal is not an error of the step
        cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
      }
    }
    if (e == cudaSuccess && !ctx->graph_exec)
      e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
    if (ctx->graph)
      cudaGraphDestroy(ctx->graph);
    ctx->graph = g;
    if (e != cudaSuccess) {
      drop_graph(ctx);
      return e;
    }
    ctx->graph_args = a;
    ctx->graph_precision = precision;
    ctx->graph_tune = ctx->tune;
  }
  e = cudaGraphLaunch(ctx->graph_exec, s);
  if (e == cudaSuccess)
    ctx->launches += 6;
  return e;
}

cudaError_t ensure_host_streams(mam4b_ctx *ctx) {
  if (ctx->host_streams)
    return cudaSuccess;
  // created in order; on failure everything created so far is released
  int ns = 0, ne = 0;
  cudaEvent_t *evs[1 + kHostStreams + 2 * kMaxChunks];
  evs[ne] = &ctx->ev_start;
  cudaError_t e = cudaEventCreateWithFlags(evs[ne], cudaEventDisableTiming);
  if (e == cudaSuccess)
    ++ne;
  for (; ns < kHostStreams && e == cudaSuccess; ++ns) {
    e = cudaStreamCreateWithFlags(&ctx->hs[ns], cudaStreamNonBlocking);
    if (e != cudaSuccess)
      break;
  }
  for (int k = 0; k < kHostStreams && e == cudaSuccess; ++k) {
    evs[ne] = &ctx->ev_done[k];
    e = cudaEventCreateWithFlags(evs[ne], cudaEventDisableTiming);
    if (e == cudaSuccess)
      ++ne;
  }
  for (int i = 0; i < kMaxChunks && e == cudaSuccess; ++i) {
    evs[ne] = &ctx->ev_in[i];
    e = cudaEventCreateWithFlags(evs[ne], cudaEventDisableTiming);
    if (e != cudaSuccess)
      break;
    ++ne;
    evs[ne] = &ctx->ev_comp[i];
    e = cudaEventCreateWithFlags(evs[ne], cudaEventDisableTiming);
    if (e == cudaSuccess)
      ++ne;
  }
  if (e != cudaSuccess) {
    for (int j = 0; j < ns; ++j)
      cudaStreamDestroy(ctx->hs[j]);
    for (int j = 0; j < ne; ++j)
      cudaEventDestroy(*evs[j]);
    return e;
  }
  ctx->host_streams = true;
  return cudaSuccess;
}

// Per-device state of mam4b_step_slab_noalloc, filled once per device by
// noalloc_setup with that device current.
struct NoAllocDevice {
  bool ready;
  double *scratch;  // device address of g_noalloc_scratch on this device
  int sms;          // SMs of the device (the solver's persistent grid)
};
NoAllocDevice g_noalloc[64];

cudaError_t noalloc_setup(int dev) {
  std::lock_guard<std::mutex> lk(g_init_mu);
  if (dev < 0 || dev >= 64)
    return cudaErrorInvalidDevice;
  if (g_noalloc[dev].ready)
    return cudaSuccess;
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess)
    return e;
  if (!g_consts_ready[dev]) {
    // derived constants without a temporary allocation: staged in the
    // scratch array (no step can be using it before set-up ends)
    StepConsts *stage = reinterpret_cast<StepConsts *>(p);
    init_consts_kernel<<<1, 1>>>(stage);
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
      e = cudaMemcpyToSymbol(c_k, stage, sizeof(StepConsts), 0, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess)
      e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
      return e;
    g_consts_ready[dev] = true;
  }
  int sms = 0;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess)
    return e;
  g_noalloc[dev].scratch = static_cast<double *>(p);
  g_noalloc[dev].sms = sms;
  g_noalloc[dev].ready = true;
  return cudaSuccess;
}
// ------------------------------------------------------- tuning files
// A tuning file is a flat JSON object with the integer fields of
// mam4b_tuning under their own names and the device name it was chosen on
// ("device": "NVIDIA B200"), e.g. as written by mam4xx_b200/autotune.py.
const char *const kTuningKeys[] = {"size_block", "size_regs", "mode_block", "pair_block",
                                   "pre_block", "pre_regs", "post_block", "post_regs",
                                   "soa_block", "soa_regs", "soa_blocks_per_sm",
                                   "cells_per_thread", "inline_scale"};
int *tuning_field(mam4b_tuning &t, int k) {
  int *f[] = {&t.size_block, &t.size_regs, &t.mode_block, &t.pair_block, &t.pre_block,
              &t.pre_regs, &t.post_block, &t.post_regs, &t.soa_block, &t.soa_regs,
              &t.soa_blocks_per_sm, &t.cells_per_thread, &t.inline_scale};
  return f[k];
}

// Value text after "key": in json, or nullptr.
const char *json_value(const char *json, const char *key) {
  char pat[64];
  snprintf(pat, sizeof(pat), "\"%s\"", key);
  const char *p = strstr(json, pat);
  if (!p)
    return nullptr;
  p += strlen(pat);
  while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')
    ++p;
  if (*p != ':')
    return nullptr;
  ++p;
  while (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')
    ++p;
  return p;
}

mam4b_status parse_tuning(const char *json, mam4b_tuning *t, char *device, size_t device_len) {
  mam4b_tuning r;
  mam4b_default_tuning(&r);
  for (int k = 0; k < (int)(sizeof(kTuningKeys) / sizeof(kTuningKeys[0])); ++k) {
    const char *v = json_value(json, kTuningKeys[k]);
    if (!v)
      return MAM4B_ERR_INVALID_ARGUMENT;
    char *end = nullptr;
    const long x = strtol(v, &end, 10);
    if (end == v || x < 0 || x > 4096)
      return MAM4B_ERR_INVALID_ARGUMENT;
    *tuning_field(r, k) = (int)x;
  }
  if (!valid_tuning(r))
    return MAM4B_ERR_INVALID_ARGUMENT;
  if (device && device_len) {
    device[0] = '\0';
    const char *v = json_value(json, "device");
    if (v && *v == '"') {
      const char *q = strchr(v + 1, '"');
      if (q) {
        size_t n = (size_t)(q - v - 1);
        if (n >= device_len)
          n = device_len - 1;
        memcpy(device, v + 1, n);
        device[n] = '\0';
      }
    }
  }
  *t = r;
  return MAM4B_OK;
}

mam4b_status read_tuning_file(const char *path, mam4b_tuning *t, char *device, size_t device_len) {
  FILE *f = fopen(path, "rb");
  if (!f)
    return MAM4B_ERR_INVALID_ARGUMENT;
  char buf[4096];
  const size_t n = fread(buf, 1, sizeof(buf) - 1, f);
  fclose(f);
  buf[n] = '\0';
  return parse_tuning(buf, t, device, device_len);
}

// The tuning a new context starts with: the file named by MAM4B_TUNING_FILE,
// else mam4b_tuning.json next to this library, when it exists, parses and
// was chosen on a device of the current device's name; else the defaults.
void initial_tuning(int dev, mam4b_tuning *t) {
  mam4b_default_tuning(t);
  char path[1024] = {0};
  const char *env = getenv("MAM4B_TUNING_FILE");
  if (env && *env) {
    snprintf(path, sizeof(path), "%s", env);
  } else {
    Dl_info info;
    if (!dladdr((void *)&initial_tuning, &info) || !info.dli_fname)
      return;
    snprintf(path, sizeof(path), "%s", info.dli_fname);
    char *slash = strrchr(path, '/');
    if (!slash)
      return;
    snprintf(slash + 1, sizeof(path) - (size_t)(slash + 1 - path), "mam4b_tuning.json");
  }
  mam4b_tuning r;
  char name[256];
  if (read_tuning_file(path, &r, name, sizeof(name)) != MAM4B_OK)
    return;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || strcmp(prop.name, name) != 0)
    return;
  *t = r;
}
}  // namespace

extern "C" {

int mam4b_abi_version(void) { return MAM4B_ABI_VERSION; }

void mam4b_default_tuning(mam4b_tuning *t) {
  if (!t)
    return;
  t->size_block = 128;
  t->size_regs = 128;
  t->mode_block = 128;
  t->pair_block = 128;
  t->pre_block = 128;
  t->pre_regs = 255;
  t->post_block = 128;
  t->post_regs = 128;
  t->soa_block = 256;
  t->soa_regs = 64;
  t->soa_blocks_per_sm = 4;
  t->cells_per_thread = 1;
  t->inline_scale = 0;
}

mam4b_status mam4b_tuning_from_json(const char *path, mam4b_tuning *t, char *device,
                                    size_t device_len) {
  if (!path || !t)
    return MAM4B_ERR_INVALID_ARGUMENT;
  return read_tuning_file(path, t, device, device_len);
}

mam4b_status mam4b_get_tuning(const mam4b_ctx *ctx, mam4b_tuning *t) {
  if (!ctx || !t)
    return MAM4B_ERR_INVALID_ARGUMENT;
  *t = ctx->tune;
  return MAM4B_OK;
}

mam4b_status mam4b_set_tuning(mam4b_ctx *ctx, const mam4b_tuning *t) {
  if (!ctx || !t || !valid_tuning(*t))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_set_tuning", cudaSuccess);
  ctx->tune = *t;
  return MAM4B_OK;
}

mam4b_status mam4b_set_adjoint_checkpoint(mam4b_ctx *ctx, int interval) {
  if (!ctx || (interval != 1 && interval != 4))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_set_adjoint_checkpoint: interval 1 or 4",
                   cudaSuccess);
  ctx->adj_ck = interval;
  return MAM4B_OK;
}

mam4b_status mam4b_set_graph_mode(mam4b_ctx *ctx, int enable) {
  if (!ctx)
    return MAM4B_ERR_INVALID_ARGUMENT;
  ctx->use_graph = enable != 0;
  if (!ctx->use_graph)
    drop_graph(ctx);
  return MAM4B_OK;
}

void mam4b_default_config(mam4b_config *cfg) {
  if (!cfg)
    return;
  cfg->do_cond = 1;
  cfg->do_rename = 1;
  cfg->do_newnuc = 1;
  cfg->do_coag = 1;
  cfg->gaexch_h2so4_uptake_optaa = 2;
  cfg->newnuc_h2so4_conc_optaa = 2;
  cfg->n_so4_monolayers_pcage = 8;
}

mam4b_status mam4b_create(mam4b_ctx **out, const mam4b_config *cfg) {
  if (!out)
    return MAM4B_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  mam4b_config c;
  if (cfg)
    c = *cfg;
  else
    mam4b_default_config(&c);
  if (!valid_config(&c))
    return MAM4B_ERR_INVALID_ARGUMENT;
  mam4b_ctx *ctx = new (std::nothrow) mam4b_ctx();
  if (!ctx)
    return MAM4B_ERR_INVALID_ARGUMENT;
  ctx->cfg = c;
  ctx->launches = 0;
  cudaError_t e = cudaGetDevice(&ctx->device);
  if (e == cudaSuccess)
    e = ensure_consts(ctx->device);
  if (e == cudaSuccess)
    e = cudaMalloc(&ctx->d_flags, sizeof(unsigned));
  if (e == cudaSuccess)
    e = cudaMemset(ctx->d_flags, 0, sizeof(unsigned));
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->device);
  if (e != cudaSuccess) {
    if (ctx->d_flags)
      cudaFree(ctx->d_flags);
    delete ctx;
    return MAM4B_ERR_CUDA;
  }
  initial_tuning(ctx->device, &ctx->tune);
  *out = ctx;
  return MAM4B_OK;
}

mam4b_status mam4b_destroy(mam4b_ctx *ctx) {
  if (!ctx)
    return MAM4B_ERR_INVALID_ARGUMENT;
  drop_graph(ctx);
  if (ctx->cap_stream)
    cudaStreamDestroy(ctx->cap_stream);
  cudaFree(ctx->d_coltab);
  cudaFree(ctx->d_flags);
  cudaFree(ctx->d_in);
  cudaFree(ctx->d_out);
  cudaFree(ctx->d_pblh);
  cudaFree(ctx->d_soa);
  cudaFree(ctx->d_hand);
  cudaFree(ctx->d_task);
  cudaFree(ctx->d_order);
  cudaFree(ctx->d_aux);
  cudaFree(ctx->d_counters);
  cudaFree(ctx->d_ck);
  cudaFree(ctx->d_ck2);
  cudaFree(ctx->d_abar);
  cudaFree(ctx->d_lbar);
  cudaFree(ctx->d_npass);
  cudaFree(ctx->d_bins);
  cudaFree(ctx->d_optics_lw);
  cudaFree(ctx->d_optics_scr);
  cudaFree(ctx->d_optics_sw);
  cudaFree(ctx->d_trop);
  cudaFree(ctx->d_dmx);
  cudaFree(ctx->d_coag_cc);
  if (ctx->host_streams) {
    for (int k = 0; k < kHostStreams; ++k) {
      cudaStreamDestroy(ctx->hs[k]);
      cudaEventDestroy(ctx->ev_done[k]);
    }
    for (int i = 0; i < kMaxChunks; ++i) {
      cudaEventDestroy(ctx->ev_in[i]);
      cudaEventDestroy(ctx->ev_comp[i]);
    }
    cudaEventDestroy(ctx->ev_start);
  }
  delete ctx;
  return MAM4B_OK;
}

mam4b_status mam4b_step(mam4b_ctx *ctx, const mam4b_state_view *in, const mam4b_tend_view *out,
                        int ncol, int nlev, double dt, int precision, void *stream) {
  if (!ctx || !in || !out || ncol < 0 || nlev <= 0 || !(dt > 0.0) || !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step", cudaSuccess);
  if (precision != MAM4B_FP64 && precision != MAM4B_MIXED && precision != MAM4B_MIXED_FAST)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step: precision", cudaSuccess);
  StepArgs a;
  memset(&a, 0, sizeof(a));
  bool diag = false;
  for (int f = 0; f < MAM4B_NIN; ++f) {
    if (!in->field[f])
      return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step: null input field", cudaSuccess);
    a.in[f] = in->field[f];
  }
  if (!in->pblh)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step: null pblh", cudaSuccess);
  a.pblh = in->pblh;
  for (int f = 0; f < MAM4B_NOUT; ++f) {
    if (!out->field[f])
      return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step: null output field", cudaSuccess);
    a.out[f] = out->field[f];
  }
  for (int f = 0; f < MAM4B_NDIAG; ++f) {
    a.diag[f] = out->diag[f];
    diag = diag || (out->diag[f] != nullptr);
  }
  set_step_config(ctx, a, (long long)ncol * nlev, nlev, dt);
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (a.ncell == 0)
    return MAM4B_OK;
  const int block = 128;
  const long long grid = (a.ncell + block - 1) / block;
  if (a.ncell > 0x7fffffffLL)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step: too many cells", cudaSuccess);
  cudaError_t e;
  if (diag && precision != MAM4B_FP64)
    return set_err(ctx, MAM4B_ERR_NOT_SUPPORTED,
                   "mam4b_step: process diagnostics are FP64 only", cudaSuccess);
  if (diag) {
    // per-process diagnostics: one thread per cell, start to end
    full_kernel<true><<<(unsigned)grid, block, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess)
      return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_step launch", e);
    ctx->launches += 1;
    return MAM4B_OK;
  }
  e = ensure_solver_scratch(ctx, (size_t)a.ncell);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_step scratch", e);
  set_step_scratch(ctx, a, 0, 0);
  e = launch_pipeline(ctx, a, s, precision, nullptr, true);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_step launch", e);
  return MAM4B_OK;
}

mam4b_status mam4b_step_slab(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                             double *out_slab, size_t ld, int ncol, int nlev, double dt,
                             int precision, void *stream) {
  if (!ctx || !in_slab || !pblh || !out_slab || ncol < 0 || nlev <= 0 ||
      ld < (size_t)ncol * (size_t)nlev)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step_slab", cudaSuccess);
  mam4b_state_view iv;
  mam4b_tend_view ov;
  memset(&iv, 0, sizeof(iv));
  memset(&ov, 0, sizeof(ov));
  for (int f = 0; f < MAM4B_NIN; ++f)
    iv.field[f] = in_slab + (size_t)f * ld;
  iv.pblh = pblh;
  for (int f = 0; f < MAM4B_NOUT; ++f)
    ov.field[f] = out_slab + (size_t)f * ld;
  return mam4b_step(ctx, &iv, &ov, ncol, nlev, dt, precision, stream);
}

// Autotuner (include/mam4b.h): times every candidate launch shape of each
// pipeline stage on the caller's batch, stage by stage from events
// recorded between the launches (a stage's time does not depend on the
// other stages' shapes), keeps the fastest shape of each stage, then the
// fastest cells-per-thread of the whole-cell kernels, and adopts the result
// when the whole pipeline is faster with it than with the defaults.
mam4b_status mam4b_autotune(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                            double *out_slab, size_t ld, int ncol, int nlev, double dt,
                            int precision, int reps, void *stream, mam4b_tuning *best,
                            float *default_ms, float *best_ms) {
  const char *what = "mam4b_autotune";
  if (!ctx || !in_slab || !pblh || !out_slab || ncol <= 0 || nlev <= 0 || !(dt > 0.0) ||
      ld < (size_t)ncol * (size_t)nlev || reps < 1 || reps > 100 ||
      (long long)ncol * nlev > 0x7fffffffLL ||
      (precision != MAM4B_FP64 && precision != MAM4B_MIXED && precision != MAM4B_MIXED_FAST))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  if (!ctx->cfg.do_cond)
    return set_err(ctx, MAM4B_ERR_NOT_SUPPORTED, "mam4b_autotune: condensation off (one kernel)",
                   cudaSuccess);
  StepArgs a;
  memset(&a, 0, sizeof(a));
  for (int f = 0; f < MAM4B_NIN; ++f)
    a.in[f] = in_slab + (size_t)f * ld;
  a.pblh = pblh;
  for (int f = 0; f < MAM4B_NOUT; ++f)
    a.out[f] = out_slab + (size_t)f * ld;
  set_step_config(ctx, a, (long long)ncol * nlev, nlev, dt);
  cudaError_t e = ensure_solver_scratch(ctx, (size_t)a.ncell);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  set_step_scratch(ctx, a, 0, 0);
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t ev[7];
  int nev = 0;
  for (; nev < 7; ++nev)
    if ((e = cudaEventCreate(&ev[nev])) != cudaSuccess)
      break;
  // per-stage candidates
  const int blocks[3] = {64, 128, 256};
  std::vector<mam4b_tuning> cand[6];
  mam4b_tuning d;
  mam4b_default_tuning(&d);
  for (int b : blocks) {
    for (int r : {255, 128, 96}) {
      mam4b_tuning t = d;
      t.size_block = b;
      t.size_regs = r;
      if (valid_tuning(t))
        cand[0].push_back(t);
    }
    mam4b_tuning t = d;
    t.mode_block = b;
    cand[1].push_back(t);
    t = d;
    t.pair_block = b;
    cand[2].push_back(t);
    for (int r : {255, 168, 128}) {
      t = d;
      t.pre_block = b;
      t.pre_regs = r;
      if (valid_tuning(t))
        cand[3].push_back(t);
      t = d;
      t.post_block = b;
      t.post_regs = r;
      if (valid_tuning(t))
        cand[5].push_back(t);
    }
  }
  for (int b : {128, 256})
    for (int r : {64, 96, 128}) {
      const int resident = (int)(65536 / ((long long)b * r));
      for (int bps : {resident, resident / 2}) {
        mam4b_tuning t = d;
        t.soa_block = b;
        t.soa_regs = r;
        t.soa_blocks_per_sm = bps < 1 ? 1 : (bps > 16 ? 16 : bps);
        if (valid_tuning(t))
          cand[4].push_back(t);
      }
    }
  size_t kmax = 0;
  for (auto &c : cand)
    kmax = std::max(kmax, c.size());
  std::vector<float> stage_ms[6];
  for (int k = 0; k < 6; ++k)
    stage_ms[k].assign(cand[k].size(), 1e30f);
  auto combine = [&](size_t i) {
    // stage k of the combined shape from candidate i of stage k
    mam4b_tuning t = d;
    const mam4b_tuning &c0 = cand[0][i % cand[0].size()];
    t.size_block = c0.size_block;
    t.size_regs = c0.size_regs;
    t.mode_block = cand[1][i % cand[1].size()].mode_block;
    t.pair_block = cand[2][i % cand[2].size()].pair_block;
    const mam4b_tuning &c3 = cand[3][i % cand[3].size()];
    t.pre_block = c3.pre_block;
    t.pre_regs = c3.pre_regs;
    const mam4b_tuning &c4 = cand[4][i % cand[4].size()];
    t.soa_block = c4.soa_block;
    t.soa_regs = c4.soa_regs;
    t.soa_blocks_per_sm = c4.soa_blocks_per_sm;
    const mam4b_tuning &c5 = cand[5][i % cand[5].size()];
    t.post_block = c5.post_block;
    t.post_regs = c5.post_regs;
    return t;
  };
  auto run = [&](const mam4b_tuning &t, float *stages, float *total) -> cudaError_t {
    cudaError_t r = launch_pipeline_t(t, ctx->sms, a, s, precision, nullptr, ev, nullptr);
    if (r == cudaSuccess)
      r = cudaEventSynchronize(ev[6]);
    float ms;
    for (int k = 0; r == cudaSuccess && k < 6; ++k) {
      r = cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      if (stages)
        stages[k] = ms;
    }
    if (r == cudaSuccess && total)
      r = cudaEventElapsedTime(total, ev[0], ev[6]);
    return r;
  };
  // warm-up
  if (e == cudaSuccess)
    e = run(d, nullptr, nullptr);
  for (size_t i = 0; e == cudaSuccess && i < kmax; ++i) {
    const mam4b_tuning t = combine(i);
    for (int r = 0; e == cudaSuccess && r < reps; ++r) {
      float st[6];
      e = run(t, st, nullptr);
      for (int k = 0; e == cudaSuccess && k < 6; ++k) {
        const size_t j = i % cand[k].size();
        if (i < cand[k].size())
          stage_ms[k][j] = std::min(stage_ms[k][j], st[k]);
      }
    }
  }
  mam4b_tuning b = d;
  if (e == cudaSuccess) {
    size_t arg[6];
    for (int k = 0; k < 6; ++k)
      arg[k] = (size_t)(std::min_element(stage_ms[k].begin(), stage_ms[k].end()) -
                        stage_ms[k].begin());
    b.size_block = cand[0][arg[0]].size_block;
    b.size_regs = cand[0][arg[0]].size_regs;
    b.mode_block = cand[1][arg[1]].mode_block;
    b.pair_block = cand[2][arg[2]].pair_block;
    b.pre_block = cand[3][arg[3]].pre_block;
    b.pre_regs = cand[3][arg[3]].pre_regs;
    b.soa_block = cand[4][arg[4]].soa_block;
    b.soa_regs = cand[4][arg[4]].soa_regs;
    b.soa_blocks_per_sm = cand[4][arg[4]].soa_blocks_per_sm;
    b.post_block = cand[5][arg[5]].post_block;
    b.post_regs = cand[5][arg[5]].post_regs;
  }
  // cells per thread of the whole-cell kernels, then whole-pipeline times
  auto total_of = [&](const mam4b_tuning &t, float &ms) -> cudaError_t {
    ms = 1e30f;
    cudaError_t r = cudaSuccess;
    for (int k = 0; r == cudaSuccess && k < reps; ++k) {
      float x;
      r = run(t, nullptr, &x);
      ms = std::min(ms, x);
    }
    return r;
  };
  float t_best = 1e30f;
  for (int cpt : {1, 2, 4}) {
    mam4b_tuning t = b;
    t.cells_per_thread = cpt;
    float ms = 1e30f;
    if (e == cudaSuccess)
      e = total_of(t, ms);
    if (e == cudaSuccess && ms < t_best) {
      t_best = ms;
      b.cells_per_thread = cpt;
    }
  }
  // short SOA loops finished in pre: changes the work of pre, soa and post
  // together, so it is chosen on the whole step
  for (int sc : {1, 4, 16, 64}) {
    mam4b_tuning t = b;
    t.inline_scale = sc;
    float ms = 1e30f;
    if (e == cudaSuccess)
      e = total_of(t, ms);
    if (e == cudaSuccess && ms < t_best) {
      t_best = ms;
      b.inline_scale = sc;
    }
  }
  float t_def = 1e30f;
  if (e == cudaSuccess)
    e = total_of(d, t_def);
  if (e == cudaSuccess)
    e = total_of(b, t_best);
  for (int k = 0; k < nev; ++k)
    cudaEventDestroy(ev[k]);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  if (!(t_best < t_def)) {
    b = d;
    t_best = t_def;
  }
  ctx->tune = b;
  if (best)
    *best = b;
  if (default_ms)
    *default_ms = t_def;
  if (best_ms)
    *best_ms = t_best;
  return MAM4B_OK;
}

// The step with gas-phase and aqueous chemistry ahead of amicphys (FP64):
// the forward pipeline with the chemistry in its pre stage; slabs of ld
// doubles per field.
mam4b_status mam4b_step_chem_slab(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                                  const double *chem_in, double *out_slab, double *chem_out,
                                  size_t ld, int ncol, int nlev, double dt, void *stream) {
  const char *what = "mam4b_step_chem_slab";
  if (!ctx || !in_slab || !pblh || !chem_in || !out_slab || !chem_out || ncol < 0 ||
      nlev <= 0 || ld < (size_t)ncol * (size_t)nlev || !(dt > 0.0) || !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  StepArgs a;
  memset(&a, 0, sizeof(a));
  for (int f = 0; f < MAM4B_NIN; ++f)
    a.in[f] = in_slab + (size_t)f * ld;
  a.pblh = pblh;
  for (int f = 0; f < MAM4B_NOUT; ++f)
    a.out[f] = out_slab + (size_t)f * ld;
  set_step_config(ctx, a, (long long)ncol * nlev, nlev, dt);
  ChemArgs ch;
  ch.in = chem_in;
  ch.out = chem_out;
  ch.ld = ld;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (a.ncell == 0)
    return MAM4B_OK;
  if (a.ncell > 0x7fffffffLL)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  cudaError_t e = ensure_solver_scratch(ctx, (size_t)a.ncell);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  set_step_scratch(ctx, a, 0, 0);
  e = launch_pipeline(ctx, a, s, MAM4B_FP64, &ch);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  return MAM4B_OK;
}

static cudaError_t grow(double **p, size_t *cap, size_t need) {
  if (*cap >= need)
    return cudaSuccess;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(p, need * sizeof(double));
  if (e == cudaSuccess)
    *cap = need;
  return e;
}

mam4b_status mam4b_step_host(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                             double *out_slab, size_t ld, int ncol, int nlev, double dt,
                             int precision, void *stream) {
  if (!ctx || !in_slab || !pblh || !out_slab || ncol < 0 || nlev <= 0 ||
      ld < (size_t)ncol * (size_t)nlev || !(dt > 0.0) || !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step_host", cudaSuccess);
  if (precision != MAM4B_FP64 && precision != MAM4B_MIXED && precision != MAM4B_MIXED_FAST)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step_host: precision", cudaSuccess);
  const size_t n = (size_t)ncol * (size_t)nlev;
  if (n > 0x7fffffffULL)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step_host: too many cells", cudaSuccess);
  cudaStream_t us = (cudaStream_t)stream;
  ctx->last_stream = us;
  if (n == 0)
    return MAM4B_OK;
  cudaError_t e = grow(&ctx->d_in, &ctx->cap_in, (size_t)MAM4B_NIN * n);
  if (e == cudaSuccess)
    e = grow(&ctx->d_out, &ctx->cap_out, (size_t)MAM4B_NOUT * n);
  if (e == cudaSuccess)
    e = grow(&ctx->d_pblh, &ctx->cap_pblh, (size_t)ncol);
  if (e == cudaSuccess)
    e = ensure_solver_scratch(ctx, n);
  if (e == cudaSuccess)
    e = ensure_host_streams(ctx);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_step_host scratch", e);
  // chunks of whole columns: the first ones a quarter and a half of the
  // steady size, so that the copy-out engine starts early; at most
  // kMaxChunks (the steady size grows for very large batches)
  int chunk_cols = (int)(kHostChunkCells / nlev);
  if (chunk_cols < 1)
    chunk_cols = 1;
  if ((ncol + chunk_cols - 1) / chunk_cols > kMaxChunks - 2)
    chunk_cols = (ncol + kMaxChunks - 3) / (kMaxChunks - 2);
  int chunk_start[kMaxChunks + 1];
  int nchunk = 0;
  for (int col = 0; col < ncol; ++nchunk) {
    chunk_start[nchunk] = col;
    const int want = nchunk == 0 ? (chunk_cols + 3) / 4 : nchunk == 1 ? (chunk_cols + 1) / 2 : chunk_cols;
    col += want < ncol - col ? want : ncol - col;
  }
  chunk_start[nchunk] = ncol;
  // the internal streams start after the work already queued on us
  e = cudaEventRecord(ctx->ev_start, us);
  for (int k = 0; k < kHostStreams && e == cudaSuccess; ++k)
    e = cudaStreamWaitEvent(ctx->hs[k], ctx->ev_start, 0);
  const size_t dp = n * sizeof(double), hp = ld * sizeof(double);
  cudaStream_t s_in = ctx->hs[0], s_out = ctx->hs[kHostStreams - 1];
  for (int i = 0; i < nchunk && e == cudaSuccess; ++i) {
    cudaStream_t s = ctx->hs[1 + i % kComputeStreams];
    const int col0 = chunk_start[i];
    const int ncc = chunk_start[i + 1] - col0;
    const size_t c0 = (size_t)col0 * nlev, nc = (size_t)ncc * nlev;
    // field f of the chunk: nc doubles at f*ld + c0 on the host, f*n + c0 on the device
    e = cudaMemcpy2DAsync(ctx->d_in + c0, dp, in_slab + c0, hp, nc * sizeof(double), MAM4B_NIN,
                          cudaMemcpyHostToDevice, s_in);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ctx->d_pblh + col0, pblh + col0, (size_t)ncc * sizeof(double),
                          cudaMemcpyHostToDevice, s_in);
    if (e == cudaSuccess)
      e = cudaEventRecord(ctx->ev_in[i], s_in);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(s, ctx->ev_in[i], 0);
    if (e != cudaSuccess)
      break;
    StepArgs a;
    memset(&a, 0, sizeof(a));
    for (int f = 0; f < MAM4B_NIN; ++f)
      a.in[f] = ctx->d_in + (size_t)f * n + c0;
    a.pblh = ctx->d_pblh + col0;
    for (int f = 0; f < MAM4B_NOUT; ++f)
      a.out[f] = ctx->d_out + (size_t)f * n + c0;
    set_step_config(ctx, a, (long long)nc, nlev, dt);
    set_step_scratch(ctx, a, c0, i);
    e = launch_pipeline(ctx, a, s, precision);
    if (e == cudaSuccess)
      e = cudaEventRecord(ctx->ev_comp[i], s);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(s_out, ctx->ev_comp[i], 0);
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(out_slab + c0, hp, ctx->d_out + c0, dp, nc * sizeof(double),
                            MAM4B_NOUT, cudaMemcpyDeviceToHost, s_out);
  }
  // us waits for every internal stream, then the call returns
  for (int k = 0; k < kHostStreams; ++k) {
    cudaError_t e2 = cudaEventRecord(ctx->ev_done[k], ctx->hs[k]);
    if (e2 == cudaSuccess)
      e2 = cudaStreamWaitEvent(us, ctx->ev_done[k], 0);
    if (e == cudaSuccess)
      e = e2;
  }
  cudaError_t e3 = cudaStreamSynchronize(us);
  if (e == cudaSuccess)
    e = e3;
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_step_host", e);
  return MAM4B_OK;
}

// The step on per-column arrays (include/mam4b.h, mam4b_step_columns):
// gather the columns into the context's staging slabs, the pipeline, then
// add the tendencies to (and write the mode outputs into) the caller's
// columns. Two pointer tables go to the device per call, synchronously.
mam4b_status mam4b_step_columns(mam4b_ctx *ctx, const mam4b_column *cols, int ncol, int nlev,
                                double dt, int precision, void *stream) {
  const char *what = "mam4b_step_columns";
  if (!ctx || !cols || ncol < 0 || nlev <= 0 || !(dt > 0.0) || !isfinite(dt) ||
      (long long)ncol * nlev > 0x7fffffffLL ||
      (precision != MAM4B_FP64 && precision != MAM4B_MIXED && precision != MAM4B_MIXED_FAST))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  for (int c = 0; c < ncol; ++c)
    for (int f = 0; f < MAM4B_NIN; ++f)
      if (!cols[c].in[f])
        return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step_columns: null input column",
                       cudaSuccess);
  if (ncol == 0)
    return MAM4B_OK;
  const size_t ncell = (size_t)ncol * nlev;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  cudaError_t e = grow(&ctx->d_in, &ctx->cap_in, (size_t)MAM4B_NIN * ncell);
  if (e == cudaSuccess)
    e = grow(&ctx->d_out, &ctx->cap_out, (size_t)MAM4B_NOUT * ncell);
  if (e == cudaSuccess)
    e = grow(&ctx->d_pblh, &ctx->cap_pblh, (size_t)ncol);
  const size_t ntab = (size_t)(MAM4B_NIN + MAM4B_NOUT) * ncol;
  if (e == cudaSuccess && ctx->cap_coltab < ntab) {
    cudaFree(ctx->d_coltab);
    ctx->d_coltab = nullptr;
    ctx->cap_coltab = 0;
    e = cudaMalloc(&ctx->d_coltab, ntab * sizeof(void *));
    if (e == cudaSuccess)
      ctx->cap_coltab = ntab;
  }
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_step_columns scratch", e);
  // tables [input fields][col], then [output fields][col]; pblh per column
  ctx->h_coltab.assign(ntab + (size_t)ncol, nullptr);
  double *pb = reinterpret_cast<double *>(ctx->h_coltab.data() + ntab);
  for (int c = 0; c < ncol; ++c) {
    for (int f = 0; f < MAM4B_NIN; ++f)
      ctx->h_coltab[(size_t)f * ncol + c] = const_cast<double *>(cols[c].in[f]);
    for (int f = 0; f < MAM4B_NUM_PROG; ++f)
      ctx->h_coltab[(size_t)(MAM4B_NIN + f) * ncol + c] = cols[c].tend[f];
    for (int f = 0; f < MAM4B_NOUT - MAM4B_NUM_PROG; ++f)
      ctx->h_coltab[(size_t)(MAM4B_NIN + MAM4B_NUM_PROG + f) * ncol + c] = cols[c].mode_out[f];
    pb[c] = cols[c].pblh;
  }
  static_assert(sizeof(double) == sizeof(void *), "pblh shares the pointer staging");
  e = cudaMemcpyAsync(ctx->d_coltab, ctx->h_coltab.data(), ntab * sizeof(void *),
                      cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ctx->d_pblh, pb, (size_t)ncol * sizeof(double), cudaMemcpyHostToDevice, s);
  // the host staging is reused by the next call: wait for the copies
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s);
  const int block = 128;
  const unsigned gx = (unsigned)((ncell + block - 1) / block);
  if (e == cudaSuccess) {
    gather_columns_kernel<<<dim3(gx, MAM4B_NIN), block, 0, s>>>(
        reinterpret_cast<const double *const *>(ctx->d_coltab), ctx->d_in, ncol, nlev);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  const mam4b_status st = mam4b_step_slab(ctx, ctx->d_in, ctx->d_pblh, ctx->d_out, ncell, ncol,
                                          nlev, dt, precision, stream);
  if (st != MAM4B_OK)
    return st;
  scatter_columns_kernel<<<dim3(gx, MAM4B_NOUT), block, 0, s>>>(
      reinterpret_cast<double *const *>(ctx->d_coltab) + (size_t)MAM4B_NIN * ncol, ctx->d_out,
      ncol, nlev, MAM4B_NUM_PROG);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

mam4b_status mam4b_synchronize(mam4b_ctx *ctx) {
  if (!ctx)
    return MAM4B_ERR_INVALID_ARGUMENT;
  const cudaError_t e = cudaStreamSynchronize(ctx->last_stream);
  return e == cudaSuccess ? MAM4B_OK : set_err(ctx, MAM4B_ERR_CUDA, "mam4b_synchronize", e);
}

// Allocation-free step for callers that cannot call cudaMalloc (a host
// model whose memory pool owns the GPU's memory, or that forbids the
// device-wide synchronisation of cudaMalloc/cudaFree once it runs). Same
// kernels as mam4b_step, with their scratch in g_noalloc_scratch. Nothing
// here allocates: set-up uses cudaGetSymbolAddress, a kernel, copies into
// the constant bank and occupancy queries; each step clears the counters
// with cudaMemsetAsync and launches the six pipeline kernels (size, mode,
// pair, pre, soa, post), or the one full_kernel when condensation is off.
// All calls share the array, so calls that overlap on the GPU race.
mam4b_status mam4b_step_slab_noalloc(const mam4b_config *cfg, const double *in_slab,
                                     const double *pblh, double *out_slab, size_t ld, int ncol,
                                     int nlev, double dt, uint32_t *flags, void *stream) {
  mam4b_config c;
  if (cfg)
    c = *cfg;
  else
    mam4b_default_config(&c);
  if (!valid_config(&c) || !in_slab || !pblh || !out_slab || ncol < 0 || nlev <= 0 ||
      !(dt > 0.0) || !isfinite(dt) || ld < (size_t)ncol * (size_t)nlev)
    return MAM4B_ERR_INVALID_ARGUMENT;
  const long long ncell = (long long)ncol * nlev;
  if (ncell > (long long)MAM4B_NOALLOC_MAX_CELLS)
    return MAM4B_ERR_TOO_MANY_CELLS;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess)
    e = noalloc_setup(dev);
  if (e != cudaSuccess)
    return MAM4B_ERR_CUDA;
  if (ncell == 0)
    return MAM4B_OK;
  const NoAllocDevice &nd = g_noalloc[dev];
  StepArgs a;
  memset(&a, 0, sizeof(a));
  for (int f = 0; f < MAM4B_NIN; ++f)
    a.in[f] = in_slab + (size_t)f * ld;
  a.pblh = pblh;
  for (int f = 0; f < MAM4B_NOUT; ++f)
    a.out[f] = out_slab + (size_t)f * ld;
  unsigned *tail = reinterpret_cast<unsigned *>(nd.scratch + kNoAllocTail);
  a.counters = tail;  // CNT_WORDS queue counters, then the spare flag word
  a.flags = flags ? reinterpret_cast<unsigned *>(flags) : tail + CNT_WORDS;
  a.soa = nd.scratch + kNoAllocSoa;
  a.hand = nd.scratch + kNoAllocHand;
  a.task = reinterpret_cast<int *>(nd.scratch + kNoAllocTask);
  a.order = reinterpret_cast<int *>(nd.scratch + kNoAllocOrder);
  a.aux = nd.scratch + kNoAllocAux;
  a.ncell = ncell;
  a.nlev = nlev;
  a.dt = dt;
  a.do_cond = c.do_cond;
  a.do_rename = c.do_rename;
  a.do_newnuc = c.do_newnuc;
  a.do_coag = c.do_coag;
  a.optaa = c.gaexch_h2so4_uptake_optaa;
  a.nmono = c.n_so4_monolayers_pcage;
  cudaStream_t s = (cudaStream_t)stream;
  // the counters (and the spare flag word) must start every step at zero
  e = cudaMemsetAsync(tail, 0, (CNT_WORDS + 1) * sizeof(unsigned), s);
  if (e != cudaSuccess)
    return MAM4B_ERR_CUDA;
  const int block = 128;
  const unsigned grid = (unsigned)((ncell + block - 1) / block);
  if (!a.do_cond) {
    // no SOA loop to pipeline (and no scratch used)
    full_kernel<false><<<grid, block, 0, s>>>(a);
  } else {
    // the default launch shape (mam4b_default_tuning)
    mam4b_tuning t;
    mam4b_default_tuning(&t);
    launch_size(t, a, s);
    launch_mode(t, a, s, false);
    launch_pair(t, a, s, false);
    launch_pre(t, a, s);
    launch_soa(t, nd.sms, a, s, MAM4B_FP64);
    launch_post(t, a, s);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? MAM4B_OK : MAM4B_ERR_CUDA;
}

// Reverse-mode adjoint (include/mam4b.h). With condensation on: the
// forward pipeline (without its post stage) into the context's output
// scratch, then eight reverse launches (suffix, the counting sort of the
// SOA loops, the loops, front, water uptake, calcsize); otherwise one
// thread per cell (adjoint_kernel).
mam4b_status mam4b_adjoint_slab(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                                const double *out_bar, double *in_bar, size_t ld, int ncol,
                                int nlev, double dt, void *stream) {
  return mam4b_adjoint_slab_ex(ctx, in_slab, pblh, out_bar, in_bar, ld, ncol, nlev, dt,
                               MAM4B_FP64, stream);
}

mam4b_status mam4b_adjoint_slab_ex(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                                   const double *out_bar, double *in_bar, size_t ld, int ncol,
                                   int nlev, double dt, int precision, void *stream) {
  if (!ctx || !in_slab || !pblh || !out_bar || !in_bar || ncol < 0 || nlev <= 0 ||
      ld < (size_t)ncol * (size_t)nlev || !(dt > 0.0) || !isfinite(dt) ||
      (precision != MAM4B_FP64 && precision != MAM4B_MIXED && precision != MAM4B_MIXED_FAST))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_adjoint_slab", cudaSuccess);
  if (!ctx->cfg.do_cond && !ctx->cfg.do_newnuc)
    return set_err(ctx, MAM4B_ERR_NOT_SUPPORTED,
                   "mam4b_adjoint_slab: needs condensation or nucleation on", cudaSuccess);
  if (precision == MAM4B_MIXED_FAST || (precision == MAM4B_MIXED && !ctx->cfg.do_cond))
    return set_err(ctx, MAM4B_ERR_NOT_SUPPORTED,
                   "mam4b_adjoint_slab: precision not supported (FP64; MIXED with condensation on)",
                   cudaSuccess);
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  const long long ncell = (long long)ncol * nlev;
  if (ncell == 0)
    return MAM4B_OK;
  if (ncell > 0x7fffffffLL)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_adjoint_slab: too many cells", cudaSuccess);
  const adj::AdjCfg cfg = {ctx->cfg.do_cond, ctx->cfg.do_rename, ctx->cfg.do_newnuc,
                           ctx->cfg.do_coag, ctx->cfg.gaexch_h2so4_uptake_optaa,
                           ctx->cfg.n_so4_monolayers_pcage};
  cudaError_t e = cudaSuccess;
  if (!ctx->cfg.do_cond) {
    if (!ctx->d_ck) {
      int dev = 0, sms = 0, per_sm = 0;
      e = cudaGetDevice(&dev);
      if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel, 128, 0);
      if (e == cudaSuccess) {
        ctx->adj_grid = sms * (per_sm > 0 ? per_sm : 1);
        e = cudaMalloc(&ctx->d_ck, (size_t)6 * adj::kSoaCkMax * ctx->adj_grid * 128 * sizeof(double));
      }
      if (e != cudaSuccess) {
        ctx->d_ck = nullptr;
        return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_adjoint_slab scratch", e);
      }
    }
    AdjArgs a;
    a.in = in_slab;
    a.pblh = pblh;
    a.ybar = out_bar;
    a.xbar = in_bar;
    a.ld = ld;
    a.ncell = ncell;
    a.nlev = nlev;
    a.dt = dt;
    a.cfg = cfg;
    a.ck = ctx->d_ck;
    adjoint_kernel<<<ctx->adj_grid, 128, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess)
      return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_adjoint_slab launch", e);
    ctx->launches += 1;
    return MAM4B_OK;
  }
  // pipelined adjoint
  const size_t n = (size_t)ncell;
  e = grow(&ctx->d_out, &ctx->cap_out, (size_t)MAM4B_NOUT * n);
  if (e == cudaSuccess)
    e = ensure_solver_scratch(ctx, n);
  if (e == cudaSuccess && ctx->cap_adj < n) {
    cudaFree(ctx->d_abar);
    cudaFree(ctx->d_lbar);
    cudaFree(ctx->d_npass);
    ctx->d_abar = ctx->d_lbar = nullptr;
    ctx->d_npass = nullptr;
    ctx->cap_adj = 0;
    e = cudaMalloc(&ctx->d_abar, (size_t)AB_FIELDS * n * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMalloc(&ctx->d_lbar, (size_t)LB_FIELDS * n * sizeof(double));
    if (e == cudaSuccess)
      e = cudaMalloc(&ctx->d_npass, n * sizeof(int));
    if (e == cudaSuccess && !ctx->d_bins)
      e = cudaMalloc(&ctx->d_bins, 2 * kPassBins * sizeof(unsigned));
    if (e == cudaSuccess)
      ctx->cap_adj = n;
  }
  const int ck_interval = ctx->adj_ck > 1 ? ctx->adj_ck : 1;
  if (e == cudaSuccess && ctx->d_ck2 && ctx->ck2_slots < adj_soa_slots(ck_interval)) {
    cudaFree(ctx->d_ck2);
    ctx->d_ck2 = nullptr;
    ctx->ck2_slots = 0;
  }
  if (e == cudaSuccess && !ctx->d_ck2) {
    int dev = 0, sms = 0, per_sm = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adj_soa_kernel<1, false>,
                                                        kSoaBlock, 0);
    if (e == cudaSuccess) {
      ctx->adj_soa_grid = sms * (per_sm > 0 ? per_sm : 1);
      const int slots = adj_soa_slots(ck_interval);
      e = cudaMalloc(&ctx->d_ck2, (size_t)6 * slots * ctx->adj_soa_grid * kSoaBlock * sizeof(double));
      if (e != cudaSuccess)
        ctx->d_ck2 = nullptr;
      else
        ctx->ck2_slots = slots;
    }
  }
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_adjoint_slab scratch", e);
  AdjPipeArgs p;
  memset(&p, 0, sizeof(p));
  for (int f = 0; f < MAM4B_NIN; ++f)
    p.s.in[f] = in_slab + (size_t)f * ld;
  p.s.pblh = pblh;
  for (int f = 0; f < MAM4B_NOUT; ++f)
    p.s.out[f] = ctx->d_out + (size_t)f * n;
  set_step_config(ctx, p.s, ncell, nlev, dt);
  set_step_scratch(ctx, p.s, 0, 0);
  p.ybar = out_bar;
  p.xbar = in_bar;
  p.ld = ld;
  p.abar = ctx->d_abar;
  p.lbar = ctx->d_lbar;
  p.ck = ctx->d_ck2;
  p.bins = ctx->d_bins;
  p.cfg = cfg;
  p.s.npass = ctx->d_npass;
  e = launch_pipeline(ctx, p.s, s, precision);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(ctx->d_bins, 0, kPassBins * sizeof(unsigned), s);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_adjoint_slab forward", e);
  const int block = 128;
  const unsigned grid = (unsigned)((ncell + block - 1) / block);
  const unsigned sort_grid = (unsigned)std::min<long long>((ncell + 255) / 256, 4 * 148);
  adj_post_kernel<<<grid, block, 0, s>>>(p);
  adj_hist_kernel<<<sort_grid, 256, 0, s>>>(p);
  adj_scan_kernel<<<1, 1024, 0, s>>>(p);
  adj_sort_kernel<<<sort_grid, 256, 0, s>>>(p);
  const bool fast = precision == MAM4B_MIXED;
  if (ck_interval == 4 && fast)
    adj_soa_kernel<4, true><<<ctx->adj_soa_grid, kSoaBlock, 0, s>>>(p);
  else if (ck_interval == 4)
    adj_soa_kernel<4, false><<<ctx->adj_soa_grid, kSoaBlock, 0, s>>>(p);
  else if (fast)
    adj_soa_kernel<1, true><<<ctx->adj_soa_grid, kSoaBlock, 0, s>>>(p);
  else
    adj_soa_kernel<1, false><<<ctx->adj_soa_grid, kSoaBlock, 0, s>>>(p);
  adj_pre_kernel<<<grid, block, 0, s>>>(p);
  adj_mode_kernel<<<dim3(grid, NMODE), block, 0, s>>>(p);
  adj_fin_kernel<<<grid, block, 0, s>>>(p);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_adjoint_slab launch", e);
  ctx->launches += 8;
  return MAM4B_OK;
}

// The step on mam4::TracersView-layout arrays (state_q tracer order,
// utils.hpp:205-259): a field table into the caller's rows, then the step.
mam4b_status mam4b_step_tracers(mam4b_ctx *ctx, const double *q, const double *qqcw,
                                size_t tracer_stride, const double *temperature,
                                const double *pressure, const double *height,
                                const double *cloud_fraction, const double *pblh,
                                double *ptend_q, double *ptend_qqcw, double *mode_out,
                                size_t mode_stride, int ncol, int nlev, double dt,
                                int precision, void *stream) {
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !q || !qqcw || !temperature || !pressure || !height || !cloud_fraction || !pblh ||
      !ptend_q || !ptend_qqcw || !mode_out || ncol < 0 || nlev <= 0 || tracer_stride < n ||
      mode_stride < n)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_step_tracers", cudaSuccess);
  constexpr int kQv = 0, kH2so4 = 11, kSoag = 14, kAero = 15;
  mam4b_state_view iv;
  mam4b_tend_view ov;
  memset(&iv, 0, sizeof(iv));
  memset(&ov, 0, sizeof(ov));
  iv.field[MAM4B_IN_T] = temperature;
  iv.field[MAM4B_IN_P] = pressure;
  iv.field[MAM4B_IN_ZM] = height;
  iv.field[MAM4B_IN_QV] = q + (size_t)kQv * tracer_stride;
  iv.field[MAM4B_IN_CLD] = cloud_fraction;
  iv.field[MAM4B_IN_H2SO4] = q + (size_t)kH2so4 * tracer_stride;
  iv.field[MAM4B_IN_SOAG] = q + (size_t)kSoag * tracer_stride;
  ov.field[MAM4B_OUT_TEND + 0] = ptend_q + (size_t)kH2so4 * tracer_stride;
  ov.field[MAM4B_OUT_TEND + 1] = ptend_q + (size_t)kSoag * tracer_stride;
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    iv.field[MAM4B_IN_AER_I + p] = q + (size_t)(kAero + p) * tracer_stride;
    iv.field[MAM4B_IN_AER_C + p] = qqcw + (size_t)(kAero + p) * tracer_stride;
    ov.field[MAM4B_OUT_TEND + 2 + p] = ptend_q + (size_t)(kAero + p) * tracer_stride;
    ov.field[MAM4B_OUT_TEND + 27 + p] = ptend_qqcw + (size_t)(kAero + p) * tracer_stride;
  }
  for (int k = 0; k < 16; ++k)
    ov.field[MAM4B_OUT_DGN_A + k] = mode_out + (size_t)k * mode_stride;
  iv.pblh = pblh;
  return mam4b_step(ctx, &iv, &ov, ncol, nlev, dt, precision, stream);
}

// longwave optics tables: the reference's per-type species refractive
// indices mapped to modes by species type (set_device_specrefindex,
// modal_aero_opt.hpp:142-190), water, grids and absorption tables
mam4b_status mam4b_optics_lw_set_tables(mam4b_ctx *ctx, const mam4b_optics_lw_tables *t) {
  const char *what = "mam4b_optics_lw_set_tables";
  if (!ctx || !t || !t->specrefindex || !t->water_refindex || !t->refrtab || !t->refitab ||
      !t->absp)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  double *h = (double *)malloc(sizeof(double) * opt::kTableDoubles);
  if (!h)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_optics_lw_set_tables: host memory",
                   cudaSuccess);
  memset(h, 0, sizeof(double) * opt::kTableDoubles);
  for (int m = 0; m < NMODE; ++m)
    for (int s = 0; s < K::nspec(m); ++s)
      for (int b = 0; b < opt::kLwBands; ++b) {
        const int type = act::spectype(m, s) - 1;
        const size_t src = 2 * ((size_t)b * MAM4B_OPTICS_NTYPES + type);
        h[opt::kSpecRe + (m * 7 + s) * opt::kLwBands + b] = t->specrefindex[src];
        h[opt::kSpecIm + (m * 7 + s) * opt::kLwBands + b] = t->specrefindex[src + 1];
      }
  for (int b = 0; b < opt::kLwBands; ++b) {
    h[opt::kWaterRe + b] = t->water_refindex[2 * b];
    h[opt::kWaterIm + b] = t->water_refindex[2 * b + 1];
  }
  memcpy(h + opt::kRefr, t->refrtab, sizeof(double) * 4 * opt::kLwBands * opt::kPrefr);
  memcpy(h + opt::kRefi, t->refitab, sizeof(double) * 4 * opt::kLwBands * opt::kPrefi);
  memcpy(h + opt::kAbsp, t->absp,
         sizeof(double) * 4 * opt::kLwBands * opt::kNcoef * opt::kPrefr * opt::kPrefi);
  cudaError_t e = cudaSuccess;
  if (!ctx->d_optics_lw)
    e = cudaMalloc(&ctx->d_optics_lw, sizeof(double) * opt::kTableDoubles);
  if (e == cudaSuccess)
    e = cudaMemcpy(ctx->d_optics_lw, h, sizeof(double) * opt::kTableDoubles,
                   cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  return MAM4B_OK;
}

// shortwave optics tables (layouts of mam4b_optics_sw_tables)
mam4b_status mam4b_optics_sw_set_tables(mam4b_ctx *ctx, const mam4b_optics_sw_tables *t) {
  const char *what = "mam4b_optics_sw_set_tables";
  if (!ctx || !t || !t->specrefindex || !t->water_refindex || !t->refrtab || !t->refitab ||
      !t->extp || !t->absp || !t->asmp)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  double *h = (double *)malloc(sizeof(double) * opt::kSwTableDoubles);
  if (!h)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_optics_sw_set_tables: host memory",
                   cudaSuccess);
  memset(h, 0, sizeof(double) * opt::kSwTableDoubles);
  for (int m = 0; m < NMODE; ++m)
    for (int s = 0; s < K::nspec(m); ++s)
      for (int b = 0; b < opt::kSwBands; ++b) {
        const int type = act::spectype(m, s) - 1;
        const size_t src = 2 * ((size_t)b * MAM4B_OPTICS_NTYPES + type);
        h[opt::kSwSpecRe + (m * 7 + s) * opt::kSwBands + b] = t->specrefindex[src];
        h[opt::kSwSpecIm + (m * 7 + s) * opt::kSwBands + b] = t->specrefindex[src + 1];
      }
  for (int b = 0; b < opt::kSwBands; ++b) {
    h[opt::kSwWaterRe + b] = t->water_refindex[2 * b];
    h[opt::kSwWaterIm + b] = t->water_refindex[2 * b + 1];
  }
  memcpy(h + opt::kSwRefr, t->refrtab, sizeof(double) * 4 * opt::kSwBands * opt::kPrefr);
  memcpy(h + opt::kSwRefi, t->refitab, sizeof(double) * 4 * opt::kSwBands * opt::kPrefi);
  memcpy(h + opt::kSwExt, t->extp, sizeof(double) * 4 * opt::kSwBands * opt::kSwTab);
  memcpy(h + opt::kSwAbs, t->absp, sizeof(double) * 4 * opt::kSwBands * opt::kSwTab);
  memcpy(h + opt::kSwAsm, t->asmp, sizeof(double) * 4 * opt::kSwBands * opt::kSwTab);
  cudaError_t e = cudaSuccess;
  if (!ctx->d_optics_sw)
    e = cudaMalloc(&ctx->d_optics_sw, sizeof(double) * opt::kSwTableDoubles);
  if (e == cudaSuccess)
    e = cudaMemcpy(ctx->d_optics_sw, h, sizeof(double) * opt::kSwTableDoubles,
                   cudaMemcpyHostToDevice);
  free(h);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  return MAM4B_OK;
}

// modal_aero_opt::modal_aero_sw (modal_aero_opt.hpp:536-878), batched
mam4b_status mam4b_optics_sw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                             const double *pdeldry, double *out, double *aodvis, int ncol,
                             int nlev, double dt, void *stream) {
  const char *what = "mam4b_optics_sw";
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !in_slab || !pdeldry || !out || ncol < 0 || nlev <= 0 || ld < n || !(dt > 0.0) ||
      !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  if (!ctx->d_optics_sw)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_optics_sw: tables not set",
                   cudaSuccess);
  OpticsSwArgs w;
  memset(&w, 0, sizeof(w));
  for (int f = 0; f < MAM4B_NIN; ++f)
    w.base.in[f] = in_slab + (size_t)f * ld;
  w.base.pdeldry = pdeldry;
  w.base.tables = ctx->d_optics_sw;
  w.base.ld = ld;
  w.base.ncell = (long long)n;
  w.base.dt = dt;
  w.out = out;
  w.aodvis = aodvis;
  w.ncol = ncol;
  w.nlev = nlev;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (n == 0)
    return MAM4B_OK;
  cudaError_t e = grow(&ctx->d_optics_scr, &ctx->cap_optics_scr, (size_t)SS_FIELDS * n);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_optics_sw scratch", e);
  w.base.scr = ctx->d_optics_scr;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  optics_size_kernel<<<grid, block, 0, s>>>(w.base);
  optics_sw_mode_kernel<<<dim3(grid, NMODE), block, 0, s>>>(w);
  // at most 1,024 blocks of cells per band: each block stages its band's
  // tables once and then steps several groups of cells
  optics_sw_band_kernel<<<dim3(opt::kSwBands, grid < 1024u ? grid : 1024u), block, 0, s>>>(w);
  int launches = 3;
  if (aodvis) {
    optics_sw_aod_kernel<<<(unsigned)((ncol + block - 1) / block), block, 0, s>>>(w);
    ++launches;
  }
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += launches;
  return MAM4B_OK;
}

// modal_aero_opt::modal_aero_lw_k (modal_aero_opt.hpp:879-989), batched
mam4b_status mam4b_optics_lw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                             const double *pdeldry, double *tauxar, int ncol, int nlev,
                             double dt, void *stream) {
  const char *what = "mam4b_optics_lw";
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !in_slab || !pdeldry || !tauxar || ncol < 0 || nlev <= 0 || ld < n ||
      !(dt > 0.0) || !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  if (!ctx->d_optics_lw)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_optics_lw: tables not set",
                   cudaSuccess);
  OpticsLwArgs a;
  for (int f = 0; f < MAM4B_NIN; ++f)
    a.in[f] = in_slab + (size_t)f * ld;
  a.pdeldry = pdeldry;
  a.tables = ctx->d_optics_lw;
  a.tau = tauxar;
  a.ld = ld;
  a.ncell = (long long)n;
  a.dt = dt;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (n == 0)
    return MAM4B_OK;
  cudaError_t e = grow(&ctx->d_optics_scr, &ctx->cap_optics_scr, (size_t)OS_FIELDS * n);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_optics_lw scratch", e);
  a.scr = ctx->d_optics_scr;
  const int block = 128;
  const unsigned grid = (unsigned)((n + block - 1) / block);
  optics_size_kernel<<<grid, block, 0, s>>>(a);
  optics_mode_kernel<<<dim3(grid, NMODE), block, 0, s>>>(a);
  // at most 1,024 blocks of cells per band, as the shortwave band kernel
  optics_band_kernel<<<dim3(opt::kLwBands, grid < 1024u ? grid : 1024u), block, 0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 3;
  return MAM4B_OK;
}

// Tropopause levels of the columns into trop (caller's array, or the
// context's when NULL); r gets the layout fields.
static mam4b_status rad_props_tropopause(mam4b_ctx *ctx, const char *what, RadArgs &r,
                                         const double *in_slab, const double *pint,
                                         const double *zi, int *trop_level, cudaStream_t s) {
  r.temp = in_slab + (size_t)MAM4B_IN_T * r.ld;
  r.pmid = in_slab + (size_t)MAM4B_IN_P * r.ld;
  r.pint = pint;
  r.zi = zi;
  r.trop = trop_level;
  if (!r.trop) {
    if (ctx->cap_trop < (size_t)r.ncol) {
      cudaFree(ctx->d_trop);
      ctx->d_trop = nullptr;
      ctx->cap_trop = 0;
      const cudaError_t e = cudaMalloc(&ctx->d_trop, (size_t)r.ncol * sizeof(int));
      if (e != cudaSuccess)
        return set_err(ctx, MAM4B_ERR_CUDA, what, e);
      ctx->cap_trop = (size_t)r.ncol;
    }
    r.trop = ctx->d_trop;
  }
  const int block = 128, per_block = block / 32;
  const size_t smem = (size_t)per_block * 4 * r.nlev * sizeof(double);
  if (smem > 48 * 1024)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  tropopause_kernel<<<(unsigned)((r.ncol + per_block - 1) / per_block), block, smem, s>>>(r);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

// aero_rad_props_sw (aero_rad_props.hpp:250-338), batched
mam4b_status mam4b_aero_rad_props_sw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                                     const double *pdeldry, const double *pint, const double *zi,
                                     const double *ext_sw, const double *ssa_sw,
                                     const double *af_sw, double *out, double *aodvis,
                                     int *trop_level, int ncol, int nlev, double dt,
                                     void *stream) {
  const char *what = "mam4b_aero_rad_props_sw";
  if (!ctx || !pint || !zi || !ext_sw || !ssa_sw || !af_sw || nlev < 2)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  mam4b_status st = mam4b_optics_sw(ctx, in_slab, ld, pdeldry, out, aodvis, ncol, nlev, dt, stream);
  if (st != MAM4B_OK || ncol == 0)
    return st;
  cudaStream_t s = (cudaStream_t)stream;
  RadArgs r;
  memset(&r, 0, sizeof(r));
  r.ld = ld;
  r.ncol = ncol;
  r.nlev = nlev;
  r.ext = ext_sw;
  r.ssa = ssa_sw;
  r.af = af_sw;
  r.out = out;
  st = rad_props_tropopause(ctx, what, r, in_slab, pint, zi, trop_level, s);
  if (st != MAM4B_OK)
    return st;
  const int block = 128;
  const size_t n = (size_t)ncol * nlev;
  volcanic_sw_kernel<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(r);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

// aero_rad_props_lw (aero_rad_props.hpp:339-410), batched
mam4b_status mam4b_aero_rad_props_lw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                                     const double *pdeldry, const double *pint, const double *zi,
                                     const double *ext_lw, double *odap, int *trop_level,
                                     int ncol, int nlev, double dt, void *stream) {
  const char *what = "mam4b_aero_rad_props_lw";
  if (!ctx || !pint || !zi || !ext_lw || nlev < 2)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  mam4b_status st = mam4b_optics_lw(ctx, in_slab, ld, pdeldry, odap, ncol, nlev, dt, stream);
  if (st != MAM4B_OK || ncol == 0)
    return st;
  cudaStream_t s = (cudaStream_t)stream;
  RadArgs r;
  memset(&r, 0, sizeof(r));
  r.ld = ld;
  r.ncol = ncol;
  r.nlev = nlev;
  r.ext = ext_lw;
  r.out = odap;
  st = rad_props_tropopause(ctx, what, r, in_slab, pint, zi, trop_level, s);
  if (st != MAM4B_OK)
    return st;
  const int block = 128;
  const size_t n = (size_t)ncol * nlev;
  volcanic_lw_kernel<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(r);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

// ndrop::dropmixnuc (ndrop.hpp:1393-1714), one block per column
mam4b_status mam4b_dropmixnuc(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                              const double *mix_in, const double *pint, const double *kvh,
                              double *out, int ncol, int nlev, int top_lev, int vertical_mix,
                              double dt, void *stream) {
  const char *what = "mam4b_dropmixnuc";
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !in_slab || !mix_in || !pint || !kvh || !out || ncol < 0 || nlev < 2 || ld < n ||
      top_lev < 1 || top_lev > nlev - 2 || !(dt > 0.0) || !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  const size_t smem = (size_t)nlev * (DM_LEVEL_FIELDS + 3 * NMODE + 4 * NPOP) * sizeof(double);
  if (smem > 200 * 1024)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_dropmixnuc: too many levels",
                   cudaSuccess);
  DropmixArgs a;
  memset(&a, 0, sizeof(a));
  for (int f = 0; f < MAM4B_NIN; ++f)
    a.in[f] = in_slab + (size_t)f * ld;
  a.mix = mix_in;
  a.pint = pint;
  a.kvh = kvh;
  a.out = out;
  a.flags = ctx->d_flags;
  a.ld = ld;
  a.ncol = ncol;
  a.nlev = nlev;
  a.top_lev = top_lev;
  a.vertical_mix = vertical_mix ? 1 : 0;
  a.dt = dt;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (n == 0)
    return MAM4B_OK;
  cudaError_t e = grow(&ctx->d_dmx, &ctx->cap_dmx, (size_t)DA_FIELDS * n);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_dropmixnuc scratch", e);
  a.act = ctx->d_dmx;
  e = cudaFuncSetAttribute(dropmix_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  dropmix_act_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(a);
  // one thread per level (whole warps, at most 128; larger columns loop)
  const int block = nlev >= 128 ? 128 : ((nlev + 31) / 32) * 32;
  dropmix_kernel<<<(unsigned)ncol, block, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 2;
  return MAM4B_OK;
}

// ndrop get_activate_frac (ndrop.hpp:699-765), batched
mam4b_status mam4b_activate(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                            const double *air_density, const double *updraft, double *out,
                            int ncol, int nlev, void *stream) {
  const char *what = "mam4b_activate";
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !in_slab || !air_density || !updraft || !out || ncol < 0 || nlev <= 0 || ld < n)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  ActivateArgs a;
  a.temp = in_slab + (size_t)MAM4B_IN_T * ld;
  for (int p = 0; p < NPOP; ++p)
    a.aer[p] = in_slab + (size_t)(MAM4B_IN_AER_I + p) * ld;
  a.rho = air_density;
  a.w = updraft;
  a.out = out;
  a.ld = ld;
  a.ncell = (long long)n;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (n == 0)
    return MAM4B_OK;
  const int block = 128;
  activate_kernel<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

// mo_setsox::setsox_single_level (mo_setsox.hpp:944-1254), batched
mam4b_status mam4b_setsox(mam4b_ctx *ctx, const double *pressure, const double *temperature,
                          const double *lwc, const double *cloud_fraction,
                          const double *cloud_number, const double *air_density, double *qin,
                          double *qcw, size_t ld, double *dqdt_aqso4, double *dqdt_aqh2so4,
                          int ncol, int nlev, double dt, void *stream) {
  const char *what = "mam4b_setsox";
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !pressure || !temperature || !lwc || !cloud_fraction || !cloud_number ||
      !air_density || !qin || !qcw || ncol < 0 || nlev <= 0 || ld < n || !(dt > 0.0) ||
      !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  SetsoxArgs a;
  a.press = pressure;
  a.temp = temperature;
  a.lwc = lwc;
  a.cldfrc = cloud_fraction;
  a.cldnum = cloud_number;
  a.xhnm = air_density;
  a.qin = qin;
  a.qcw = qcw;
  a.dso4 = dqdt_aqso4;
  a.dh2so4 = dqdt_aqh2so4;
  a.ld = ld;
  a.ncell = (long long)n;
  a.dt = dt;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (n == 0)
    return MAM4B_OK;
  const int block = 128;
  setsox_kernel<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

// gas_phase_chemistry (gas_phase_chemistry.hpp:40-117), batched
mam4b_status mam4b_gas_chemistry(mam4b_ctx *ctx, const double *temperature,
                                 const double *photo_rates, const double *extfrc,
                                 const double *invariants, const double *het_rates, double *qq,
                                 size_t ld, int ncol, int nlev, double dt, void *stream) {
  const char *what = "mam4b_gas_chemistry";
  const size_t n = (size_t)(ncol > 0 ? ncol : 0) * (size_t)(nlev > 0 ? nlev : 0);
  if (!ctx || !temperature || !photo_rates || !extfrc || !invariants || !het_rates || !qq ||
      ncol < 0 || nlev <= 0 || ld < n || !(dt > 0.0) || !isfinite(dt))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  GasChemArgs a;
  a.temp = temperature;
  a.photo = photo_rates;
  a.extfrc = extfrc;
  a.inv = invariants;
  a.het = het_rates;
  a.qq = qq;
  a.ld = ld;
  a.ncell = (long long)n;
  a.dt = dt;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (n == 0)
    return MAM4B_OK;
  const int block = 128;
  gaschem_kernel<<<(unsigned)((n + block - 1) / block), block, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

static bool copy_prog_fields(const mam4b_prog_fields *f, ProgFields &o) {
  if (!f)
    return false;
  for (int m = 0; m < NMODE; ++m) {
    o.n_i[m] = f->n_mode_i[m];
    o.n_c[m] = f->n_mode_c[m];
    for (int x = 0; x < NAER; ++x) {
      o.q_i[m][x] = f->q_aero_i[m][x];
      o.q_c[m][x] = f->q_aero_c[m][x];
    }
  }
  return true;
}

// CalcSize::compute_tendencies (calcsize.hpp:963-1220), batched
mam4b_status mam4b_calcsize_process(mam4b_ctx *ctx, const mam4b_calcsize_config *cfg,
                                    const mam4b_prog_fields *progs,
                                    const mam4b_prog_fields *tends,
                                    double *const dgncur_i[MAM4B_NUM_MODES],
                                    double *const dgncur_c[MAM4B_NUM_MODES], int ncol,
                                    int nlev, double dt, void *stream) {
  const char *what = "mam4b_calcsize_process";
  if (!ctx || ncol < 0 || nlev <= 0 || !(dt > 0.0) || !isfinite(dt) || !dgncur_i || !dgncur_c)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  CalcSizeArgs a;
  memset(&a, 0, sizeof(a));
  if (!copy_prog_fields(progs, a.progs) || !copy_prog_fields(tends, a.tends))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  a.do_aitacc_transfer = cfg ? (cfg->do_aitacc_transfer != 0) : 1;
  a.do_adjust = cfg ? (cfg->do_adjust != 0) : 1;
  // every field the process reads or writes must be given
  for (int m = 0; m < NMODE; ++m) {
    if (!dgncur_i[m] || !dgncur_c[m] || !a.progs.n_i[m] || !a.progs.n_c[m])
      return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_calcsize_process: null field",
                     cudaSuccess);
    a.dgn_i[m] = dgncur_i[m];
    a.dgn_c[m] = dgncur_c[m];
    const bool tn = a.do_adjust && !(a.do_aitacc_transfer && m <= 1);
    const bool tx = a.do_aitacc_transfer && m <= 1;
    if ((tn || tx) && (!a.tends.n_i[m] || !a.tends.n_c[m]))
      return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_calcsize_process: null tendency",
                     cudaSuccess);
    for (int s = 0; s < K::nspec(m); ++s) {
      if (!a.progs.q_i[m][s] || !a.progs.q_c[m][s])
        return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_calcsize_process: null field",
                       cudaSuccess);
    }
  }
  if (a.do_aitacc_transfer) {
    const int acc_s[4] = {0, 2, 5, 6}, ait_s[4] = {0, 1, 2, 3};
    for (int k = 0; k < 4; ++k)
      if (!a.tends.q_i[0][acc_s[k]] || !a.tends.q_c[0][acc_s[k]] || !a.tends.q_i[1][ait_s[k]] ||
          !a.tends.q_c[1][ait_s[k]])
        return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT,
                       "mam4b_calcsize_process: null tendency", cudaSuccess);
  }
  a.ncell = (long long)ncol * nlev;
  a.dt = dt;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (a.ncell == 0)
    return MAM4B_OK;
  const int block = 128;
  calcsize_process_kernel<<<(unsigned)((a.ncell + block - 1) / block), block, 0, s>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 1;
  return MAM4B_OK;
}

// Coagulation::compute_tendencies (coagulation.hpp:1198-1209), batched
mam4b_status mam4b_coagulation_process(mam4b_ctx *ctx, const double *temperature,
                                       const double *pressure,
                                       const double *const wet_density[MAM4B_NUM_MODES],
                                       const double *const wet_diameter_i[MAM4B_NUM_MODES],
                                       const mam4b_prog_fields *progs,
                                       const mam4b_prog_fields *tends, int ncol, int nlev,
                                       double dt, void *stream) {
  const char *what = "mam4b_coagulation_process";
  if (!ctx || ncol < 0 || nlev <= 0 || !(dt > 0.0) || !isfinite(dt) || !temperature ||
      !pressure || !wet_density || !wet_diameter_i)
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  CoagProcessArgs a;
  memset(&a, 0, sizeof(a));
  if (!copy_prog_fields(progs, a.progs) || !copy_prog_fields(tends, a.tends))
    return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, what, cudaSuccess);
  a.temp = temperature;
  a.pmid = pressure;
  for (int m = 0; m < NMODE; ++m) {
    if (!wet_density[m] || !wet_diameter_i[m] || !a.progs.n_i[m] || !a.tends.n_i[m])
      return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT, "mam4b_coagulation_process: null field",
                     cudaSuccess);
    a.wet_density[m] = wet_density[m];
    a.dgn_awet[m] = wet_diameter_i[m];
    for (int x = 0; x < NAER; ++x)
      if (!a.progs.q_i[m][x] || !a.tends.q_i[m][x])
        return set_err(ctx, MAM4B_ERR_INVALID_ARGUMENT,
                       "mam4b_coagulation_process: null field", cudaSuccess);
  }
  a.ncell = (long long)ncol * nlev;
  a.dt = dt;
  cudaStream_t s = (cudaStream_t)stream;
  ctx->last_stream = s;
  if (a.ncell == 0)
    return MAM4B_OK;
  cudaError_t e = grow(&ctx->d_coag_cc, &ctx->cap_coag_cc, (size_t)12 * a.ncell);
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  a.cc = ctx->d_coag_cc;
  const int block = 128;
  const unsigned grid = (unsigned)((a.ncell + block - 1) / block);
  coag_pair_process_kernel<<<dim3(grid, 3), block, 0, s>>>(a);
  coag_process_kernel<<<grid, block, 0, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, what, e);
  ctx->launches += 2;
  return MAM4B_OK;
}

mam4b_status mam4b_last_status(mam4b_ctx *ctx, uint32_t *flags) {
  if (!ctx || !flags)
    return MAM4B_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize(ctx->last_stream);
  unsigned h = 0;
  if (e == cudaSuccess)
    e = cudaMemcpy(&h, ctx->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess)
    e = cudaMemset(ctx->d_flags, 0, sizeof(unsigned));
  if (e != cudaSuccess)
    return set_err(ctx, MAM4B_ERR_CUDA, "mam4b_last_status", e);
  *flags = h;
  return (h & MAM4B_FLAGS_ERROR_MASK) ? MAM4B_ERR_DEVICE_FLAGS : MAM4B_OK;
}

void mam4b_last_error(mam4b_ctx *ctx, char *buf, size_t len) {
  if (!buf || len == 0)
    return;
  const char *m = ctx ? ctx->err : "null context";
  snprintf(buf, len, "%s", m);
}

uint64_t mam4b_launch_count(mam4b_ctx *ctx) { return ctx ? (uint64_t)ctx->launches : 0; }

}  // extern "C"
