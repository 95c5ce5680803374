/*
 * mam4b.h -- C ABI of the B200-native MAM4 gas-aerosol microphysics step.
 *
 * One "step" advances every grid cell (column x level) through the
 * sequence that mam4xx's host model runs per cell:
 *
 *   calcsize     mam4::modal_aero_calcsize::modal_aero_calcsize_sub
 *                (src/mam4xx/modal_aero_calcsize.hpp:750)
 *   water uptake mam4::water_uptake::modal_aero_water_uptake_dr
 *                (src/mam4xx/water_uptake.hpp:481)
 *   amicphys     mam4::microphysics::modal_aero_amicphys_intr
 *                (src/mam4xx/mam4_amicphys.hpp:2120): H2SO4/SOAG
 *                condensation, Aitken->accumulation renaming, H2SO4-H2O
 *                nucleation, Brownian coagulation, primary-carbon aging,
 *                over clear and cloudy subareas.
 *
 * The entry points replace the host's team dispatch
 *   Kokkos::parallel_for(team_policy, ... process.compute_tendencies(...))
 * (src/validation/aero_process.hpp:114-122, the AeroProcess plug-in API):
 * one call processes a whole batch of columns on a CUDA stream.
 *
 * Data layout ("state" and "tendency" views). Every field is a plain
 * array of doubles with one entry per cell, cell index = col*nlev + lev
 * (the same flattening as a ColumnView per column laid end to end).
 * Fields are passed as a table of pointers so that each field can live in
 * its own allocation (a Prognostics-style view per species) or inside one
 * slab with a leading dimension; reads and writes are coalesced per field.
 *
 * Units follow mam4::Prognostics: aerosol and gas mass mixing ratios in
 * kg/kg, aerosol numbers in #/kg; tendencies in the same units per second.
 *
 * Error behaviour: every entry point returns a mam4b_status; nothing is
 * thrown across the boundary and no device trap is ever raised. Per-cell
 * conditions found on the device (non-finite input, condensation sub-step
 * limit reached) are OR-ed into a status word that mam4b_last_status()
 * returns after the stream has been synchronised.
 */
#ifndef MAM4B_H
#define MAM4B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MAM4B_ABI_VERSION 1

/* ---------------------------------------------------------------- sizes */
#define MAM4B_NUM_MODES 4     /* accumulation, aitken, coarse, primary C  */
#define MAM4B_NUM_AERO 7      /* SOA, SO4, POM, BC, NaCl, DST, MOM          */
#define MAM4B_NUM_POPS 25     /* 21 species-in-mode masses + 4 numbers      */
#define MAM4B_GAS_PCNST 31    /* amicphys tracer work array length          */
#define MAM4B_NUM_PROG 52     /* H2SO4, SOAG, 25 interstitial, 25 cloud     */

/*
 * Input fields (MAM4B_NIN per cell).
 * Aerosol populations follow the E3SM state_q order of indices 15..39
 * (src/mam4xx/utils.hpp:222-259): for each mode (accumulation, aitken,
 * coarse, primary carbon) the species masses in mam4::mode_aero_species
 * order (src/mam4xx/aero_modes.hpp:214-243), then the mode number:
 *   0-6  acc  SO4 POM SOA BC DST NaCl MOM, 7 acc number
 *   8-11 ait  SO4 SOA NaCl MOM,            12 ait number
 *   13-19 cor DST NaCl SO4 BC POM SOA MOM, 20 coarse number
 *   21-23 pca POM BC MOM,                  24 pca number
 */
enum {
  MAM4B_IN_T = 0,      /* temperature [K]                                  */
  MAM4B_IN_P = 1,      /* mid-level pressure [Pa]                          */
  MAM4B_IN_ZM = 2,     /* mid-level height above surface [m]               */
  MAM4B_IN_QV = 3,     /* water vapour mixing ratio [kg/kg]                */
  MAM4B_IN_CLD = 4,    /* cloud fraction [-]                               */
  MAM4B_IN_H2SO4 = 5,  /* H2SO4 gas [kg/kg]                                */
  MAM4B_IN_SOAG = 6,   /* SOA precursor gas [kg/kg]                        */
  MAM4B_IN_AER_I = 7,  /* 25 interstitial populations                      */
  MAM4B_IN_AER_C = 32, /* 25 cloud-borne populations                       */
  MAM4B_NIN = 57
};

/*
 * Output fields (MAM4B_NOUT per cell).
 *   0..51  tendency of the 52 prognostics in input order
 *          (H2SO4, SOAG, 25 interstitial, 25 cloud-borne), per second,
 *          = (value after the step - value before) / dt
 *   52..55 dry geometric-mean diameter of the interstitial modes [m]
 *   56..59 wet geometric-mean diameter [m]
 *   60..63 wet density [kg/m3]
 *   64..67 aerosol water [kg/kg]
 */
enum {
  MAM4B_OUT_TEND = 0,
  MAM4B_OUT_DGN_A = 52,
  MAM4B_OUT_DGN_AWET = 56,
  MAM4B_OUT_WETDENS = 60,
  MAM4B_OUT_QAERWAT = 64,
  MAM4B_NOUT = 68
};

/*
 * Optional per-process diagnostics: the grid-cell mean tendencies of the
 * 31 amicphys tracers [mol/mol/s or #/kmol/s] for condensation, renaming,
 * nucleation, coagulation and cloud-borne renaming, as written by
 * modal_aero_amicphys_intr into gas_aero_exchange_* (mam4_amicphys.hpp:
 * 2355-2374). Field index = process*31 + tracer.
 */
enum { MAM4B_NDIAG = 5 * MAM4B_GAS_PCNST };

typedef enum mam4b_status {
  MAM4B_OK = 0,
  MAM4B_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad config    */
  MAM4B_ERR_CUDA = 2,             /* a CUDA runtime call failed            */
  MAM4B_ERR_NOT_SUPPORTED = 3,    /* option not built into this library    */
  MAM4B_ERR_DEVICE_FLAGS = 4,     /* cell-level flags raised on the device */
  MAM4B_ERR_TOO_MANY_CELLS = 5    /* batch larger than the fixed scratch of
                                     mam4b_step_slab_noalloc              */
} mam4b_status;

/* Cell-level condition bits reported by mam4b_last_status().
 * NONFINITE_* are errors. SOA_NITER_LIMIT is informational: the SOA
 * condensation sub-stepping reached the reference's own cap of 1000
 * iterations (gasaerexch_soaexch.hpp:93,172-173) in some cell; as in the
 * reference, that cell keeps the state reached at the cap. */
#define MAM4B_FLAG_NONFINITE_INPUT 0x1u
#define MAM4B_FLAG_SOA_NITER_LIMIT 0x2u
#define MAM4B_FLAG_NONFINITE_OUTPUT 0x4u
#define MAM4B_FLAGS_ERROR_MASK (MAM4B_FLAG_NONFINITE_INPUT | MAM4B_FLAG_NONFINITE_OUTPUT)

/* Arithmetic of the step. The mixed forms run the bulk in FP32 (water
 * uptake and Kohler equilibrium, the H2SO4 uptake coefficients, the
 * coagulation coefficients) and keep FP64 in calcsize, the H2SO4 implicit
 * exponential update, the renaming transfer fractions, the nucleation rate
 * fits (their polynomials cancel to a few digits in FP32), aging and every
 * state update and sum that carries species mass. Where an FP32 value
 * decides a branch at its threshold (the SOA loop's 1e-15 uptake cut-off,
 * the coagulation table index), the FP64 value is used. MAM4B_MIXED runs
 * the SOA sub-stepping with an FP64 state and FP64 semi-implicit update and
 * FP32 step control (saturation ratios, departures from equilibrium, the
 * sub-step length); MAM4B_MIXED_FAST runs the whole loop in FP32, which is
 * faster but leaves the results of many cells 1e-4..1e-2 away from FP64
 * (the loop amplifies rounding near equilibrium). Per-process diagnostics
 * are FP64 only. */
typedef enum mam4b_precision {
  MAM4B_FP64 = 0,       /* plain double precision throughout              */
  MAM4B_MIXED = 1,      /* FP32 bulk, FP64 condensation state and update  */
  MAM4B_MIXED_FAST = 2  /* FP32 bulk and FP32 SOA sub-stepping            */
} mam4b_precision;

/*
 * Process switches and options; mirrors mam4::microphysics::AmicPhysConfig
 * (src/mam4xx/mam4_amicphys.hpp:223-237) plus the aging parameter
 * n_so4_monolayers_pcage (src/mam4xx/aging.hpp:31).
 */
typedef struct mam4b_config {
  int do_cond;
  int do_rename;
  int do_newnuc;
  int do_coag;
  int gaexch_h2so4_uptake_optaa; /* 1 sequential, 2 simultaneous          */
  int newnuc_h2so4_conc_optaa;   /* accepted, unused (as in the reference) */
  unsigned n_so4_monolayers_pcage;
} mam4b_config;

/* Pointer tables. in[f] / out[f] point at ncell doubles (device memory). */
typedef struct mam4b_state_view {
  const double *field[MAM4B_NIN];
  const double *pblh; /* planetary boundary layer height per column [m]  */
} mam4b_state_view;

typedef struct mam4b_tend_view {
  double *field[MAM4B_NOUT];
  double *diag[MAM4B_NDIAG]; /* all NULL: diagnostics not written        */
} mam4b_tend_view;

typedef struct mam4b_ctx mam4b_ctx;

/* Fills *cfg with the defaults used by E3SM (all processes on,
 * options 2/2, 8 monolayers). */
void mam4b_default_config(mam4b_config *cfg);

/* Creates a context bound to the current CUDA device. The context owns the
 * device status word; one context per stream. */
mam4b_status mam4b_create(mam4b_ctx **ctx, const mam4b_config *cfg);
mam4b_status mam4b_destroy(mam4b_ctx *ctx);

/*
 * Runs one step over ncol*nlev cells, asynchronously on `stream`
 * (a cudaStream_t; NULL = legacy default stream). All pointers are device
 * pointers. Replaces AeroProcess<MicrophysicsProcess>::compute_tendencies
 * dispatched over all columns (src/validation/aero_process.hpp:114).
 */
mam4b_status mam4b_step(mam4b_ctx *ctx, const mam4b_state_view *in,
                        const mam4b_tend_view *out, int ncol, int nlev,
                        double dt, int precision, void *stream);

/*
 * Same step on a slab: in_slab holds MAM4B_NIN fields of ld doubles each,
 * out_slab MAM4B_NOUT fields of ld doubles each, pblh ncol doubles.
 */
mam4b_status mam4b_step_slab(mam4b_ctx *ctx, const double *in_slab,
                             const double *pblh, double *out_slab, size_t ld,
                             int ncol, int nlev, double dt, int precision,
                             void *stream);

/*
 * Launch shape of the forward step's kernels (no counterpart in the
 * reference, whose only knob is the Kokkos team size of its column loop,
 * src/validation/validation.hpp:25-30). The step runs as six kernels: size
 * (calcsize, one thread per cell), mode (water uptake, one thread per cell
 * and mode), pair (coagulation coefficients, one thread per cell and mode
 * pair), pre (each cell up to the SOA condensation loop), soa (the
 * persistent loop solver) and post (the rest of each cell). Blocks are 64,
 * 128 or 256 threads (128 or 256 for soa); *_regs selects the compiled
 * register cap of a kernel (size 255, 128 or 96; pre and post 255, 168 or 128;
 * soa 64, 96 or 128; block x regs <= 65536); soa_blocks_per_sm sizes the
 * solver's persistent grid (1..16 blocks per SM); cells_per_thread (1, 2,
 * 4) is how many cells each thread of size and post steps, i.e.
 * 32 x cells_per_thread cells per warp; inline_scale (0 = off, 1, 4, 16,
 * 64): cells whose first SOA sub-step is at least 1/inline_scale of the time
 * step (short loops, predicted from the first sub-step) run their loop and
 * finish inside pre, without the hand-off to the solver and post kernels
 * (FP64 and MAM4B_MIXED; not in the adjoint's forward). Every shape computes
 * the same results bit for bit; only the speed differs.
 */
typedef struct mam4b_tuning {
  int size_block, size_regs;
  int mode_block, pair_block;
  int pre_block, pre_regs;
  int post_block, post_regs;
  int soa_block, soa_regs, soa_blocks_per_sm;
  int cells_per_thread;
  int inline_scale;
} mam4b_tuning;

/* The built-in shape (size 128/128, mode 128, pair 128, pre 128/255, post
 * 128/128, soa 256/64 x 4 per SM, one cell per thread, no inline loops). */
void mam4b_default_tuning(mam4b_tuning *t);

/* A context starts with the shape in the file named by the environment
 * variable MAM4B_TUNING_FILE, else in mam4b_tuning.json next to this
 * library, when that file parses, is valid and was chosen on a device of the
 * current device's name; else with the defaults. */
mam4b_status mam4b_get_tuning(const mam4b_ctx *ctx, mam4b_tuning *t);
/* MAM4B_ERR_INVALID_ARGUMENT for a shape outside the values above. */
mam4b_status mam4b_set_tuning(mam4b_ctx *ctx, const mam4b_tuning *t);

/* Reads a tuning file: a flat JSON object with the integer fields of
 * mam4b_tuning under their own names and "device": "<device name>" (copied
 * to device, which may be NULL). No CUDA call. */
mam4b_status mam4b_tuning_from_json(const char *path, mam4b_tuning *t, char *device,
                                    size_t device_len);

/*
 * Project autotuner: times the candidate shapes of every stage on the given
 * batch (device slabs as for mam4b_step_slab, `reps` timed repetitions of
 * each, 1..100), picks the fastest per stage and the fastest
 * cells_per_thread, and sets the result on ctx when the whole step is
 * faster with it than with the defaults (else the defaults). best,
 * default_ms and best_ms (may be NULL) receive the shape and the two
 * whole-step times [ms]. Synchronous; out_slab is overwritten with the
 * step's results. Needs condensation on (the pipelined step).
 */
mam4b_status mam4b_autotune(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                            double *out_slab, size_t ld, int ncol, int nlev, double dt,
                            int precision, int reps, void *stream, mam4b_tuning *best,
                            float *default_ms, float *best_ms);

/*
 * Graph mode (off by default). When on, mam4b_step and mam4b_step_slab
 * capture the step's kernels (pipelined form: condensation on, no
 * diagnostics) into a CUDA graph on the first call and replay it with one
 * graph launch on `stream` while the call's arguments (pointers, sizes,
 * dt, precision, launch shape) stay the same; a call with other arguments
 * recaptures the graph and updates it in place. The capture runs on a
 * private stream of the context. Results are identical to the plain
 * launches.
 */
mam4b_status mam4b_set_graph_mode(mam4b_ctx *ctx, int enable);

/*
 * One column of a host model that keeps one array per field and column
 * (mam4::Atmosphere / Prognostics / Diagnostics / Tendencies ColumnViews,
 * src/mam4xx/atmosphere.hpp:70-118, aero_config.hpp:74-130): device
 * pointers to nlev doubles each.
 *   in[MAM4B_NIN]   the step's inputs in MAM4B_IN_* order (populations in
 *                   the E3SM state_q order of the header's table)
 *   pblh            the column's boundary-layer height [m]
 *   tend[52]        tendency columns of the 52 prognostics (H2SO4, SOAG, 25
 *                   interstitial, 25 cloud-borne); the step ADDS its
 *                   tendency to each (as processes add to a shared
 *                   Tendencies); NULL: not written
 *   mode_out[16]    dry diameter, wet diameter, wet density and aerosol water
 *                   of the 4 interstitial modes (outputs 52..67), written;
 *                   NULL: not written
 */
typedef struct mam4b_column {
  const double *in[MAM4B_NIN];
  double pblh;
  double *tend[MAM4B_NUM_PROG];
  double *mode_out[MAM4B_NOUT - MAM4B_NUM_PROG];
} mam4b_column;

/*
 * The step on ncol such columns (cols: a host array): gathers them into the
 * context's staging slabs, runs the step and adds/writes the results into
 * the columns, on `stream`. This is the batched entry behind the C++
 * mam4::MicrophysicsProcess (include/mam4b_microphysics.hpp): it replaces
 * the host's parallel_for(team_policy, ...) over columns of
 * AeroProcess::compute_tendencies (src/validation/aero_process.hpp:114).
 * Copies the column tables to the device synchronously; the kernels are
 * asynchronous on `stream`.
 */
mam4b_status mam4b_step_columns(mam4b_ctx *ctx, const mam4b_column *cols, int ncol, int nlev,
                                double dt, int precision, void *stream);

/* Waits for the work of the context's last call (its stream); returns
 * MAM4B_ERR_CUDA when that work failed. */
mam4b_status mam4b_synchronize(mam4b_ctx *ctx);

/*
 * Host-buffer convenience: copies the host slabs to the device, runs the
 * step and copies the results back, all on `stream`, then synchronises.
 * Scratch device memory is kept in ctx and reused across calls.
 */
mam4b_status mam4b_step_host(mam4b_ctx *ctx, const double *in_slab,
                             const double *pblh, double *out_slab, size_t ld,
                             int ncol, int nlev, double dt, int precision,
                             void *stream);

/*
 * Allocation-free step (no counterpart in the reference: mam4xx allocates
 * its work views itself). For callers that cannot call cudaMalloc: host
 * models whose memory pool has reserved the GPU's memory up front, and
 * host models that forbid allocation after start-up because cudaMalloc and
 * cudaFree can synchronise the whole device and stall their other streams.
 * The same step as mam4b_step_slab (FP64, no diagnostics, same results),
 * with the whole pipeline scratch (the SOA solver's loop state, the
 * hand-off between the pipeline kernels, the work queue and its counters,
 * the per-cell auxiliaries) in one fixed device array inside the library
 * instead of context-owned allocations:
 * MAM4B_NOALLOC_MAX_CELLS cells at most, about 13 MB, held on every GPU
 * that loads the library until the process exits. No context is needed.
 *
 *   cfg      process switches (NULL = mam4b_default_config)
 *   in_slab, pblh, out_slab, ld, ncol, nlev, dt  as for mam4b_step_slab
 *   flags    optional device pointer to one word into which the step ORs
 *            its MAM4B_FLAG_* bits; the caller clears it (NULL = dropped)
 *   stream   cudaStream_t the step is queued on (NULL = legacy default)
 *
 * Returns MAM4B_ERR_TOO_MANY_CELLS, before touching the device, when
 * ncol*nlev > MAM4B_NOALLOC_MAX_CELLS; split larger batches by columns.
 * The first call on a device does a one-time set-up with that device
 * current (finds the array's device address, fills the constant tables)
 * and synchronises the device; make that first call, for instance with
 * ncol = 0, which does only the set-up, before any stream capture. Every
 * call shares the one array and leaves its contents behind: two calls
 * whose work overlaps on a device (other streams, other host threads)
 * race and give wrong results; serialise them.
 */
#define MAM4B_NOALLOC_MAX_CELLS 16384
mam4b_status mam4b_step_slab_noalloc(const mam4b_config *cfg, const double *in_slab,
                                     const double *pblh, double *out_slab, size_t ld,
                                     int ncol, int nlev, double dt, uint32_t *flags,
                                     void *stream);

/*
 * Reverse-mode adjoint of the FP64 step (no counterpart in the reference,
 * which has no derivatives): for every cell, in_bar = (d out / d in)^T
 * out_bar, where out are the MAM4B_NOUT outputs of mam4b_step_slab at the
 * state in_slab and out_bar their cotangents (MAM4B_NOUT fields of ld
 * doubles). in_bar receives MAM4B_NIN fields of ld doubles: the gradients
 * with respect to temperature, water vapour, H2SO4, SOAG and the 50 aerosol
 * populations; the pressure, height and cloud-fraction rows are written as
 * zero (these are held fixed), and the boundary-layer height has no
 * cotangent. The derivative is that of the branch the forward takes at the
 * given state (max/min clips, process thresholds and the SOA sub-step count
 * are not differentiated across). With condensation on, the SOA loops are
 * reversed by a persistent kernel whose threads keep the loop state (6
 * doubles) before every sub-step (the default) or only a checkpoint every
 * 4 sub-steps, recomputing each block of 4 from its checkpoint
 * (mam4b_set_adjoint_checkpoint). Memory of those states, allocated on
 * the first call and kept by the context: 6 x 1,001 doubles per thread
 * (every sub-step) or 6 x 255 (every 4), for SMs x 2 x 256 threads; on a
 * 148-SM B200, 3.64 GB or 0.93 GB, whatever the batch size. Without
 * condensation, one thread per cell recomputes from checkpoints every 4
 * sub-steps. Uses the context's config; asynchronous on `stream`. Device
 * pointers.
 */
mam4b_status mam4b_adjoint_slab(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                                const double *out_bar, double *in_bar, size_t ld, int ncol,
                                int nlev, double dt, void *stream);

/*
 * The adjoint of one precision form of the step (no counterpart in the
 * reference): MAM4B_FP64 is mam4b_adjoint_slab. MAM4B_MIXED (condensation
 * on) runs the forward sweep as the MAM4B_MIXED step does (single-precision
 * water uptake, uptake and coagulation coefficients; the SOA loop in double
 * precision with approximate reciprocals and fused multiply-adds) and
 * reverses its SOA loops with the same arithmetic; every other reverse
 * process is the FP64 one. Its gradient is that of the MAM4B_MIXED step up
 * to rounding. MAM4B_MIXED_FAST: MAM4B_ERR_NOT_SUPPORTED.
 */
mam4b_status mam4b_adjoint_slab_ex(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                                   const double *out_bar, double *in_bar, size_t ld, int ncol,
                                   int nlev, double dt, int precision, void *stream);

/*
 * SOA sub-step states of the adjoint (no counterpart in the reference):
 * interval 1 stores the state before every sub-step (fastest), interval 4
 * keeps a checkpoint every 4 sub-steps and recomputes the others in the
 * reverse sweep (a quarter of the memory, more arithmetic). The gradient
 * is the same bit for bit. MAM4B_ERR_INVALID_ARGUMENT for other intervals.
 */
mam4b_status mam4b_set_adjoint_checkpoint(mam4b_ctx *ctx, int interval);

/*
 * Step on tracer arrays (E3SM state_q tracer order, the layout of
 * mam4::TracersView, src/mam4xx/mam4_types.hpp:46-50: tracer, column,
 * level). For hosts that keep their aerosol state as tracer arrays rather
 * than per-species views: the step reads and writes them in place through
 * its field table, with no repacking pass (the mmr -> vmr conversion of
 * utils.hpp:112-360 / conversions.hpp:56-75 is done inside the kernels).
 *
 *   q, qqcw        interstitial and cloud-borne tracers [kg/kg, #/kg]:
 *                  tracer t of cell c at q[t*tracer_stride + c], c = col*nlev
 *                  + lev; the order of extract_stateq_from_prognostics
 *                  (utils.hpp:205-259): 0 qv, 1 qc, 2 qi, 3 nc, 4 ni, 9..14
 *                  O3 H2O2 H2SO4 SO2 DMS SOAG, 15..39 the 25 aerosol
 *                  populations of the input table above. Read: q rows 0, 11,
 *                  14, 15..39 and qqcw rows 15..39.
 *   temperature, pressure, height, cloud_fraction  one value per cell
 *   pblh           one value per column
 *   ptend_q, ptend_qqcw  tendencies in the same tracer layout and stride:
 *                  rows 11, 14, 15..39 of ptend_q and 15..39 of ptend_qqcw
 *                  are written, every other row is left as it is.
 *   mode_out       16 rows of mode_stride doubles: dry diameter, wet
 *                  diameter, wet density, aerosol water of the 4 modes.
 * Same kernels and results as mam4b_step. Asynchronous on `stream`.
 */
#define MAM4B_TRACER_COUNT 40
mam4b_status mam4b_step_tracers(mam4b_ctx *ctx, const double *q, const double *qqcw,
                                size_t tracer_stride, const double *temperature,
                                const double *pressure, const double *height,
                                const double *cloud_fraction, const double *pblh,
                                double *ptend_q, double *ptend_qqcw, double *mode_out,
                                size_t mode_stride, int ncol, int nlev, double dt,
                                int precision, void *stream);

/*
 * Longwave aerosol optics, batched over cells:
 * mam4::modal_aero_opt::modal_aero_lw_k (src/mam4xx/modal_aero_opt.hpp:
 * 879-989). Per cell: dry and wet mode diameters and aerosol water
 * (calcsize and water uptake, as in the step), then for every mode and
 * longwave band the volume-mixed complex refractive index of species and
 * water, bilinear interpolation of the Chebyshev coefficients of specific
 * absorption in the mode's refractive-index table, and the layer's
 * absorption optical depth tauxar = max(0, absorption) x wet volume x
 * rho_water x pdeldry / g, summed over modes.
 *
 * The tables (in the host model read from its optics files) are set once
 * per context with mam4b_optics_lw_set_tables (host arrays, copied):
 *   specrefindex    [16 bands][MAM4B_OPTICS_NTYPES species types] complex,
 *                   as (real, imaginary) pairs: the refractive index of
 *                   each species type of get_e3sm_parameters (ndrop.hpp:
 *                   44-114), mapped to the modes by species type
 *   water_refindex  [16] complex, (real, imaginary) pairs
 *   refrtab, refitab  [4 modes][16][7] and [4][16][10]: the real and
 *                   imaginary refractive-index grids of each table
 *   absp            [4][16][5 coefficients][7][10]: Chebyshev coefficients
 *                   of specific absorption
 * mam4b_optics_lw reads the step's input layout (MAM4B_NIN fields of ld
 * doubles; qv, T, p, cloud fraction and both aerosol phases), pdeldry (dry
 * pressure thickness, Pa, one per cell) and writes tauxar, 16 fields of ld
 * doubles. Asynchronous on `stream`.
 */
#define MAM4B_OPTICS_NTYPES 14
#define MAM4B_OPTICS_LW_BANDS 16
typedef struct mam4b_optics_lw_tables {
  const double *specrefindex;
  const double *water_refindex;
  const double *refrtab;
  const double *refitab;
  const double *absp;
} mam4b_optics_lw_tables;
mam4b_status mam4b_optics_lw_set_tables(mam4b_ctx *ctx, const mam4b_optics_lw_tables *tables);
mam4b_status mam4b_optics_lw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                             const double *pdeldry, double *tauxar, int ncol, int nlev,
                             double dt, void *stream);

/*
 * Shortwave aerosol optics, batched over cells: mam4::modal_aero_opt::
 * modal_aero_sw (src/mam4xx/modal_aero_opt.hpp:536-878). Per cell, mode
 * and shortwave band (14): the mode sizes as for the longwave, the
 * volume-mixed refractive index, the Chebyshev coefficients of specific
 * extinction, absorption and asymmetry interpolated in the mode's tables,
 * extinction exp(Chebyshev) (geometric optics above 25 um surface radius),
 * the single-scattering albedo and the layer products; summed over the
 * modes per band. Tables per context (host arrays, copied):
 *   specrefindex [14 bands][MAM4B_OPTICS_NTYPES] and water_refindex [14],
 *   complex as (real, imaginary) pairs; refrtab [4][14][7], refitab
 *   [4][14][10]; extp, absp, asmp [4][14][5][7][10]
 * out: 4 x 14 fields of ld doubles, tauxar[band] (optical depth), then
 * wa (x single-scattering albedo), ga (x asymmetry), fa (x asymmetry^2).
 * aodvis: NULL or one value per column, the visible-band (index 9) optical
 * depth summed over levels and modes. The reference's extra layer above
 * the model top (constant values) is not produced. Asynchronous on
 * `stream`.
 */
#define MAM4B_OPTICS_SW_BANDS 14
typedef struct mam4b_optics_sw_tables {
  const double *specrefindex;
  const double *water_refindex;
  const double *refrtab;
  const double *refitab;
  const double *extp;
  const double *absp;
  const double *asmp;
} mam4b_optics_sw_tables;
mam4b_status mam4b_optics_sw_set_tables(mam4b_ctx *ctx, const mam4b_optics_sw_tables *tables);
mam4b_status mam4b_optics_sw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                             const double *pdeldry, double *out, double *aodvis, int ncol,
                             int nlev, double dt, void *stream);

/*
 * Aerosol activation, batched over cells: the per-cell part of mam4xx's
 * droplet nucleation, get_activate_frac (src/mam4xx/ndrop.hpp:699-765):
 * number, volume and hygroscopicity of the 4 interstitial modes (loadaer),
 * then the Abdul-Razzak & Ghan activated fractions for the updraft
 * (activate_modal with maxsat, maximum updraft 10 m/s). A consumer of the
 * aerosol state the step produces.
 *
 *   in_slab     the step's input layout (MAM4B_NIN fields of ld doubles);
 *               reads temperature and the 25 interstitial populations
 *   air_density [kg/m3] and updraft (subgrid vertical velocity, m/s), one
 *               per cell; the aerosol is loaded at the same level
 *   out         17 fields of ld doubles: activated number fraction of the 4
 *               modes, activated mass fraction, their fluxes (fraction x
 *               updraft, m/s), and the flux at full activation; all zero
 *               where there is no accumulation-mode aerosol or no updraft
 * Mode number bounds of loadaer: the modes' nominal volume-to-number
 * ratios at their maximum and minimum diameters. Asynchronous on `stream`.
 */
mam4b_status mam4b_activate(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                            const double *air_density, const double *updraft, double *out,
                            int ncol, int nlev, void *stream);

/*
 * The radiation-facing aerosol optics of the host model, batched over
 * columns: aero_rad_props_sw and aero_rad_props_lw
 * (src/mam4xx/aero_rad_props.hpp:250-338, 339-410). The modal optics of
 * mam4b_optics_sw / mam4b_optics_lw (same arguments, same tables), then the
 * WMO lapse-rate tropopause of each column (tropopause_twmo,
 * src/mam4xx/tropopause.hpp:81-233) and the volcanic (CMIP6) stratospheric
 * aerosol over them: averaged half and half at the tropopause level,
 * replacing the modal values above it.
 *
 *   pint, zi   interface pressure [Pa] and height above the surface [m],
 *              nlev + 1 per column (top first): element col*(nlev+1) + k
 *   ext_sw, ssa_sw, af_sw  [MAM4B_OPTICS_SW_BANDS][ld]: volcanic extinction
 *              [1/m], single-scattering albedo and asymmetry per cell
 *   ext_lw     [MAM4B_OPTICS_LW_BANDS][ld]: volcanic extinction [1/m]
 *   out, odap  as mam4b_optics_sw's out and mam4b_optics_lw's tauxar
 *   aodvis     NULL or per column: the visible optical depth of the modal
 *              aerosol (before the volcanic values, as in the reference)
 *   trop_level NULL or [ncol] ints (out): the tropopause level of each
 *              column, 0 where none is found (the reference's value then)
 * The tropopause search needs nlev >= 2; the reference fixes nlev at its
 * build's level count. Asynchronous on `stream`.
 */
mam4b_status mam4b_aero_rad_props_sw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                                     const double *pdeldry, const double *pint, const double *zi,
                                     const double *ext_sw, const double *ssa_sw,
                                     const double *af_sw, double *out, double *aodvis,
                                     int *trop_level, int ncol, int nlev, double dt,
                                     void *stream);
mam4b_status mam4b_aero_rad_props_lw(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                                     const double *pdeldry, const double *pint, const double *zi,
                                     const double *ext_lw, double *odap, int *trop_level,
                                     int ncol, int nlev, double dt, void *stream);

/*
 * Droplet activation and vertical mixing, batched over columns:
 * mam4::ndrop::dropmixnuc (src/mam4xx/ndrop.hpp:1393-1714). Per level,
 * from top_lev down: release of aerosol where the cloud shrank and
 * activation where it grew (update_from_newcld), activation at cloud base
 * from the level below (update_from_cldn_profile); then explicit,
 * sub-stepped vertical mixing of droplets and of interstitial and
 * cloud-borne aerosol (update_from_explmix); then tendencies and CCN.
 *
 *   in_slab    the step's input layout: temperature, pressure, height,
 *              cloud fraction (the new one), the 25 interstitial
 *              populations (state_q) and the 25 cloud-borne ones (qqcw)
 *   mix_in     MAM4B_DROPMIX_NIN fields of ld doubles (below)
 *   pint, kvh  interface pressure [Pa] and vertical diffusivity [m2/s],
 *              nlev + 1 per column (top first): element col*(nlev+1) + k
 *   out        MAM4B_DROPMIX_NOUT fields of ld doubles (below); above
 *              top_lev the droplet number is the input one, wtke is set,
 *              and every other field is zero (the cloud-borne aerosol is
 *              removed there, as the reference does)
 *   top_lev    first level treated, 1 <= top_lev <= nlev - 2 (the
 *              reference reads one level above it)
 *   vertical_mix  enable_aero_vertical_mix
 * factnum starts at zero; rpdel is 1 / pdel. One block of 128 threads per
 * column; about 1 KB of shared memory per level (at most ~200 levels).
 * Asynchronous on `stream`.
 */
enum {
  MAM4B_DROPMIX_IN_PDEL = 0,    /* layer pressure thickness [Pa] */
  MAM4B_DROPMIX_IN_CLDO = 1,    /* cloud fraction of the previous step */
  MAM4B_DROPMIX_IN_NCLDWTR = 2, /* cloud droplet number [#/kg] */
  MAM4B_DROPMIX_IN_WSUB = 3,    /* subgrid vertical velocity [m/s] */
  MAM4B_DROPMIX_NIN = 4
};
enum {
  MAM4B_DROPMIX_OUT_QCLD = 0,     /* droplet number after mixing [#/kg] */
  MAM4B_DROPMIX_OUT_TENDND = 1,   /* droplet number tendency [#/kg/s] */
  MAM4B_DROPMIX_OUT_NSOURCE = 2,  /* droplet number source [#/kg/s] */
  MAM4B_DROPMIX_OUT_NDROPMIX = 3, /* droplet number mixing [#/kg/s] */
  MAM4B_DROPMIX_OUT_NDROPCOL = 4, /* column droplet number of the level [#/m2] */
  MAM4B_DROPMIX_OUT_WTKE = 5,     /* turbulent vertical velocity [m/s] */
  MAM4B_DROPMIX_OUT_FACTNUM = 6,  /* 4 activated number fractions */
  MAM4B_DROPMIX_OUT_CCN = 10,     /* CCN at 0.02..1 % supersaturation [#/cm3], 6 */
  MAM4B_DROPMIX_OUT_PTEND = 16,   /* 25 interstitial tendencies [kg/kg/s, #/kg/s] */
  MAM4B_DROPMIX_OUT_QQCW = 41,    /* 25 cloud-borne populations after */
  MAM4B_DROPMIX_NOUT = 66
};
mam4b_status mam4b_dropmixnuc(mam4b_ctx *ctx, const double *in_slab, size_t ld,
                              const double *mix_in, const double *pint, const double *kvh,
                              double *out, int ncol, int nlev, int top_lev, int vertical_mix,
                              double dt, void *stream);

/*
 * Aqueous-phase sulfate chemistry in cloud water, batched over cells:
 * mam4::mo_setsox::setsox_single_level (src/mam4xx/mo_setsox.hpp:944-1254),
 * the cloud-chemistry stage that runs before amicphys in the host model.
 * Per cell: the pH of cloud water (bisection on the electro-neutrality
 * equation), S(IV) oxidation by H2O2 and by O3 over dt, uptake of H2SO4 gas
 * by the droplets; the sulfate formed goes to the cloud-borne SO4 of the
 * accumulation, aitken and coarse modes in proportion to their activated
 * number.
 *
 *   pressure [Pa], temperature [K], lwc (cloud liquid water, kg/kg),
 *   cloud_fraction, cloud_number (droplets, #/kg), air_density (total
 *   number density, #/cm3): one value per cell
 *   qin, qcw   the 31 amicphys tracers (mol/mol, #/kmol; order of
 *              MAM4B_GAS_PCNST: O3 H2O2 H2SO4 SO2 DMS SOAG, then the
 *              populations) of the gas/interstitial and of the cloud-borne
 *              phase, [31][ld], updated in place: qin O3..SO2 are read and
 *              H2O2, H2SO4, SO2 written; qcw SO4 and numbers of the modes
 *              read, SO4 of modes 1-3 written
 *   dqdt_aqso4, dqdt_aqh2so4  NULL or [3][ld]: the cloud-borne SO4
 *              tendencies of modes 1-3 from aqueous oxidation and from
 *              H2SO4 uptake [mol/mol/s] (zero where the cell has no cloud
 *              water)
 * The reference's mbar and pdel arguments are not used by its computation
 * and are not taken. Asynchronous on `stream`.
 */
mam4b_status mam4b_setsox(mam4b_ctx *ctx, const double *pressure, const double *temperature,
                          const double *lwc, const double *cloud_fraction,
                          const double *cloud_number, const double *air_density, double *qin,
                          double *qcw, size_t ld, double *dqdt_aqso4, double *dqdt_aqh2so4,
                          int ncol, int nlev, double dt, void *stream);

/*
 * Gas-phase chemistry, batched over cells:
 * mam4::microphysics::gas_phase_chemistry (src/mam4xx/gas_phase_chemistry.hpp:
 * 40-117), the chemistry stage that runs before cloud chemistry and
 * amicphys in the host model, for the mechanism of
 * src/mam4xx/gas_chem_mechanism.hpp: reaction rates (setrxt, usrrxt,
 * adjrxt), then imp_sol's implicit Euler step with Newton-Raphson iteration
 * and step control (src/mam4xx/gas_chem.hpp:234-424).
 *
 *   temperature [K], photo_rates (the one photolysis rate, of H2O2, 1/s):
 *              one value per cell
 *   extfrc     [MAM4B_GAS_EXTCNT][ld] external forcing [molecules/cm3/s]
 *   invariants [MAM4B_GAS_NFS][ld] invariant densities [molecules/cm3]
 *              (0 total air, 1 N2, 2 O2, 3 H2O, 4 OH, 5 NO3, 6 HO2, 7 O3:
 *              mo_setinv::setinv_single_level)
 *   het_rates  [MAM4B_GAS_PCNST][ld] wet-removal rates [1/s] (row 0 unused)
 *   qq         [MAM4B_GAS_PCNST][ld] the 31 tracers [mol/mol, #/kmol],
 *              updated in place (tracer 0, O3, is neither read nor written)
 * Asynchronous on `stream`.
 */
#define MAM4B_GAS_EXTCNT 9
#define MAM4B_GAS_NFS 8
mam4b_status mam4b_gas_chemistry(mam4b_ctx *ctx, const double *temperature,
                                 const double *photo_rates, const double *extfrc,
                                 const double *invariants, const double *het_rates, double *qq,
                                 size_t ld, int ncol, int nlev, double dt, void *stream);

/*
 * The step with the chemistry that precedes amicphys in the host model,
 * fused per cell: calcsize, water uptake and the calcsize update as in
 * mam4b_step; then gas-phase chemistry (gas_phase_chemistry, as
 * mam4b_gas_chemistry) and aqueous chemistry (setsox_single_level, as
 * mam4b_setsox) on the cell's 31 tracers; then modal_aero_amicphys_intr
 * (src/mam4xx/mam4_amicphys.hpp:2120) with the states the chemistry leaves:
 * q_pregaschem before gas chemistry, q_precldchem and qqcw_precldchem before
 * aqueous chemistry, qq and qqcw after it. With distinct states the
 * H2SO4 production of the other processes (gaexch_h2so4_uptake_optaa = 2)
 * feeds condensation, and cloud-chemistry growth feeds renaming.
 *
 *   in_slab, pblh, out_slab  the step's layouts (MAM4B_NIN / MAM4B_NOUT
 *              fields of ld doubles); out_slab's tendencies are relative to
 *              the inputs, so they include the chemistry
 *   chem_in    MAM4B_CHEM_NIN fields of ld doubles (below); the total air
 *              density of aqueous chemistry is the invariant density 0
 *   chem_out   MAM4B_CHEM_NOUT fields of ld doubles: tendencies [kg/kg/s]
 *              of O3 (zero: neither chemistry changes it), H2O2, SO2, DMS
 * FP64, one thread per cell. Asynchronous on `stream`.
 */
enum {
  MAM4B_CHEM_IN_O3 = 0,      /* O3, H2O2, SO2, DMS mass mixing ratios [kg/kg] */
  MAM4B_CHEM_IN_H2O2 = 1,
  MAM4B_CHEM_IN_SO2 = 2,
  MAM4B_CHEM_IN_DMS = 3,
  MAM4B_CHEM_IN_PHOTO = 4,   /* H2O2 photolysis rate [1/s] */
  MAM4B_CHEM_IN_EXTFRC = 5,  /* MAM4B_GAS_EXTCNT external forcings [molecules/cm3/s] */
  MAM4B_CHEM_IN_INV = 14,    /* MAM4B_GAS_NFS invariant densities [molecules/cm3] */
  MAM4B_CHEM_IN_HET = 22,    /* MAM4B_GAS_PCNST wet-removal rates [1/s] (first unused) */
  MAM4B_CHEM_IN_LWC = 53,    /* cloud liquid water [kg/kg] */
  MAM4B_CHEM_IN_CLDNUM = 54, /* cloud droplet number [#/kg] */
  MAM4B_CHEM_NIN = 55
};
enum { MAM4B_CHEM_OUT_TEND = 0, MAM4B_CHEM_NOUT = 4 };
mam4b_status mam4b_step_chem_slab(mam4b_ctx *ctx, const double *in_slab, const double *pblh,
                                  const double *chem_in, double *out_slab, double *chem_out,
                                  size_t ld, int ncol, int nlev, double dt, void *stream);

/*
 * Per-process entries: the batched form of two mam4xx AeroProcess
 * implementations, for host models that call the processes one at a time
 * instead of the whole step. Their state is Prognostics-style: one device
 * array per (mode, index), one entry per cell (cell = col*nlev + lev, the
 * ColumnViews of mam4::Prognostics, src/mam4xx/aero_config.hpp:74-124,
 * laid end to end). Mass mixing ratios in kg/kg, numbers in #/kg,
 * tendencies per second. The second index of q_aero_* follows each
 * reference process (they differ): see the entries.
 */
typedef struct mam4b_prog_fields {
  double *n_mode_i[MAM4B_NUM_MODES];
  double *n_mode_c[MAM4B_NUM_MODES];
  double *q_aero_i[MAM4B_NUM_MODES][MAM4B_NUM_AERO];
  double *q_aero_c[MAM4B_NUM_MODES][MAM4B_NUM_AERO];
} mam4b_prog_fields;

/* CalcSize::Config (src/mam4xx/calcsize.hpp:835-842); both default to 1. */
typedef struct mam4b_calcsize_config {
  int do_aitacc_transfer; /* aitken <-> accumulation exchange             */
  int do_adjust;          /* number adjustment toward the size bounds     */
} mam4b_calcsize_config;

/*
 * CalcSize::compute_tendencies (src/mam4xx/calcsize.hpp:963-1220) over a
 * batch of columns. Reads progs->n_mode_{i,c}[m] and
 * progs->q_aero_{i,c}[m][s] for the species s of mode m in the mode's own
 * order (aero_modes.hpp:214-243: accumulation SO4 POM SOA BC DST NaCl MOM,
 * aitken SO4 SOA NaCl MOM, coarse DST NaCl SO4 BC POM SOA MOM, primary
 * carbon POM BC MOM). Writes dgncur_i[m], dgncur_c[m] (dry geometric-mean
 * diameters [m], 4 device arrays each). Tendencies as the reference: the
 * number tendencies of the modes it adjusts are overwritten; the aitken <->
 * accumulation transfers are added to the number and common-species
 * tendencies already in tends; other tendency arrays are not touched (only
 * the fields read or written must be non-null). cfg NULL = defaults.
 * Asynchronous on `stream`.
 */
mam4b_status mam4b_calcsize_process(mam4b_ctx *ctx, const mam4b_calcsize_config *cfg,
                                    const mam4b_prog_fields *progs,
                                    const mam4b_prog_fields *tends,
                                    double *const dgncur_i[MAM4B_NUM_MODES],
                                    double *const dgncur_c[MAM4B_NUM_MODES], int ncol,
                                    int nlev, double dt, void *stream);

/*
 * Coagulation::compute_tendencies (src/mam4xx/coagulation.hpp:1198-1209,
 * coagulation_rates_1box :1121-1183) over a batch of columns: Brownian
 * coagulation of the aitken, accumulation and primary-carbon interstitial
 * modes over dt. Reads temperature [K], pressure [Pa], the wet density
 * [kg/m3] and wet diameter [m] of the 4 modes, progs->n_mode_i[m] and
 * progs->q_aero_i[m][a] for all 7 AeroIds a of every mode (SOA SO4 POM BC
 * NaCl DST MOM, mam4::AeroId order, as that routine indexes them: all 28
 * arrays non-null). As the reference: tends->n_mode_i / q_aero_i +=
 * (after - before) / dt, and progs->n_mode_i / q_aero_i are overwritten
 * with the state after coagulation. Cloud-borne fields are not used.
 * Asynchronous on `stream`.
 */
mam4b_status mam4b_coagulation_process(mam4b_ctx *ctx, const double *temperature,
                                       const double *pressure,
                                       const double *const wet_density[MAM4B_NUM_MODES],
                                       const double *const wet_diameter_i[MAM4B_NUM_MODES],
                                       const mam4b_prog_fields *progs,
                                       const mam4b_prog_fields *tends, int ncol, int nlev,
                                       double dt, void *stream);

/* Synchronises the context's last stream, stores in *flags the OR of the
 * MAM4B_FLAG_* bits raised since the previous call (then clears them), and
 * returns MAM4B_ERR_DEVICE_FLAGS if any bit of MAM4B_FLAGS_ERROR_MASK is
 * set, MAM4B_OK otherwise. */
mam4b_status mam4b_last_status(mam4b_ctx *ctx, uint32_t *flags);

/* Copies a description of the last error into buf (NUL-terminated). */
void mam4b_last_error(mam4b_ctx *ctx, char *buf, size_t len);

/* Number of kernels launched by this context since creation. */
uint64_t mam4b_launch_count(mam4b_ctx *ctx);

int mam4b_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MAM4B_H */
