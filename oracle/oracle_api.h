/*
 * oracle_api.h -- batched CPU entry points shared by the two CPU oracles.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links these.
 *
 *   mam4ref_*  : oracle/_ref/libmam4ref.so, the mam4xx reference headers
 *                (src/mam4xx headers) compiled unchanged with g++ against the
 *                host shim in oracle/shim (oracle/ref/ref_step.cpp).
 *   mam4orc_*  : oracle/libmam4oracle.so, the plain-C restatement of the
 *                same algorithm (oracle/mam4_oracle.c).
 *
 * The full-step entry uses the field-major layout of include/mam4b.h:
 * in[f*ld_in + cell], out[f*ld_out + cell], diag[f*ld_diag + cell].
 * pblh is given per cell. Stage-level entries use cell-major arrays.
 */
#ifndef MAM4_ORACLE_API_H
#define MAM4_ORACLE_API_H

#include <stddef.h>
#include "../include/mam4b.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_DECLARE(P)                                                      \
  int P##_step(int ncell, const double *in, size_t ld_in,                      \
               const double *pblh_cell, double *out, size_t ld_out,            \
               double *diag, size_t ld_diag, double dt,                        \
               const mam4b_config *cfg, int nthreads);                         \
  /* calcsize: state_q, qqcw [ncell][40] kg/kg; outputs [ncell][4], [40] */    \
  void P##_calcsize(int ncell, const double *state_q, const double *qqcw,      \
                    double dt, double *dgncur_a, double *dgncur_c,             \
                    double *ptend, double *dqqcwdt);                           \
  /* water uptake: state_q [ncell][40]; dgncur_a [ncell][4] */                 \
  void P##_water_uptake(int ncell, const double *state_q, const double *temp,  \
                        const double *pmid, const double *cld,                 \
                        const double *dgncur_a, double *dgncur_awet,           \
                        double *qaerwat, double *wetdens);                     \
  /* amicphys: qq, qqcw [ncell][31] in/out (mol/mol, #/kmol); diag may be   \
     NULL or [ncell][5][31] */                                                 \
  void P##_amicphys(int ncell, const mam4b_config *cfg, double dt,             \
                    const double *temp, const double *pmid, const double *zm,  \
                    const double *pblh, const double *qv, const double *cld,   \
                    double *qq, double *qqcw, const double *dgncur_a,          \
                    const double *dgncur_awet, const double *wetdens,          \
                    double *diag);                                             \
  /* H2SO4 quasi-analytic update for one box (4 modes) */                      \
  void P##_h2so4_update(double dt, double qgas_netprod_otrproc,                \
                        const double *uptkaer, double *qgas_cur,               \
                        double *qgas_avg, double *qaer_cur);                   \
  double P##_bm0ij(int n1, int n2a, int n2n);                                  \
  double P##_bm3i(int n1, int n2a, int n2n);                                   \
  /* primary-carbon aging for one subarea; arrays [7][4] species-major */      \
  void P##_aging(unsigned n_so4_monolayers_pcage, const double *dgn_a,         \
                 double *qnum_cur, double *qnum_del_cond,                      \
                 double *qnum_del_coag, double *qaer_cur,                      \
                 double *qaer_del_cond, double *qaer_del_coag,                 \
                 double *qaer_del_coag_in);

ORACLE_DECLARE(mam4ref)
ORACLE_DECLARE(mam4orc)

/* Extra port-only instrumentation: SOA sub-step count of the clear
 * subarea per cell (0 when condensation does not run). */
void mam4orc_soa_niter(int ncell, const double *in, size_t ld_in,
                       const double *pblh_cell, double dt,
                       const mam4b_config *cfg, int *niter, int nthreads);

#ifdef __cplusplus
}
#endif

#endif
