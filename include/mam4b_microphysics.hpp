// mam4b_microphysics.hpp -- the B200 microphysics step as a mam4xx
// AeroProcess implementation (C++ host side of the C ABI in mam4b.h).
//
// mam4::MicrophysicsProcess has the shape AeroProcess<Impl> requires
// (src/validation/aero_process.hpp:19-129): a Config, name(), init(),
// validate() and compute_tendencies() over mam4::AeroConfig, ThreadTeam,
// Atmosphere, Surface, Prognostics, Diagnostics and Tendencies
// (src/mam4xx/aero_config.hpp:74-239, atmosphere.hpp). It is a host-side
// implementation: the step runs as CUDA kernels launched through the C ABI,
// which cannot be nested inside a device team, so
//
//   * compute_tendencies_columns() is the batched entry that replaces the
//     host's Kokkos::parallel_for(team_policy, ...) over all columns
//     (one mam4b_step_columns call for the whole batch), and
//   * compute_tendencies() is the per-team form for host teams (a batch of
//     one column; it synchronises the stream).
//
// The containers' ColumnViews must hold device-accessible memory (CUDA
// device or managed memory). Field mapping (mam4::utils packing of state_q,
// utils.hpp:222-259): Atmosphere temperature, pressure, height,
// vapor_mixing_ratio, cloud_fraction, planetary_boundary_layer_height;
// Prognostics q_gas[H2SO4], q_gas[SOAG], per mode the first
// num_species_mode(m) entries of q_aero_i[m][] / q_aero_c[m][] (species in
// mode order, aero_modes.hpp:214-243) and n_mode_i[m] / n_mode_c[m];
// Tendencies: the same fields, to which the step adds its tendencies;
// Diagnostics: dry_geometric_mean_diameter_i, wet_geometric_mean_diameter_i
// and wet_density of each mode are written (where their views are set).
#ifndef MAM4B_MICROPHYSICS_HPP
#define MAM4B_MICROPHYSICS_HPP

#include <mam4xx/mam4.hpp>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mam4b.h"

namespace mam4 {

class MicrophysicsProcess {
public:
  /// Process switches of amicphys (mam4b_config, AmicPhysConfig of
  /// mam4_amicphys.hpp:223-237) and the arithmetic (mam4b_precision).
  struct Config {
    mam4b_config physics;
    int precision;
    Config() : precision(MAM4B_FP64) { mam4b_default_config(&physics); }
  };

  MicrophysicsProcess() = default;

  const char *name() const { return "MAM4 microphysics step (calcsize, water uptake, amicphys)"; }

  /// Creates the device context (on the current CUDA device).
  void init(const AeroConfig &aero_config, const Config &config) {
    (void)aero_config;
    config_ = config;
    mam4b_ctx *h = nullptr;
    if (mam4b_create(&h, &config_.physics) != MAM4B_OK)
      throw std::runtime_error("MicrophysicsProcess: mam4b_create failed");
    ctx_ = std::shared_ptr<mam4b_ctx>(h, [](mam4b_ctx *c) { mam4b_destroy(c); });
  }

  /// Non-negative atmosphere and prognostics, as the reference processes
  /// check (atmosphere.hpp, aero_config.hpp quantities_nonnegative).
  bool validate(const AeroConfig &aero_config, const ThreadTeam &team,
                const Atmosphere &atmosphere, const Surface &surface,
                const Prognostics &prognostics) const {
    (void)aero_config;
    (void)surface;
    return atmosphere.quantities_nonnegative(team) && prognostics.quantities_nonnegative(team);
  }

  /// Per-team form (host teams): one column, synchronous.
  void compute_tendencies(const AeroConfig &aero_config, const ThreadTeam &team, Real t, Real dt,
                          const Atmosphere &atmosphere, const Surface &surface,
                          const Prognostics &prognostics, const Diagnostics &diagnostics,
                          const Tendencies &tendencies) const {
    (void)aero_config;
    (void)team;
    compute_tendencies_columns(t, dt, 1, &atmosphere, &surface, &prognostics, &diagnostics,
                               &tendencies, nullptr);
    if (mam4b_synchronize(ctx_.get()) != MAM4B_OK)
      throw std::runtime_error("MicrophysicsProcess: the step failed on the device");
  }

  /// Batched form: every column of the host model in one call on `stream`
  /// (a cudaStream_t; nullptr = legacy default stream).
  void compute_tendencies_columns(Real t, Real dt, int ncol, const Atmosphere *atmosphere,
                                  const Surface *surface, const Prognostics *prognostics,
                                  const Diagnostics *diagnostics, const Tendencies *tendencies,
                                  void *stream) const {
    (void)t;
    (void)surface;
    if (!ctx_)
      throw std::runtime_error("MicrophysicsProcess: init() was not called");
    if (ncol <= 0)
      return;
    const int nlev = atmosphere[0].num_levels();
    std::vector<mam4b_column> cols((size_t)ncol);
    for (int c = 0; c < ncol; ++c) {
      if (atmosphere[c].num_levels() != nlev)
        throw std::invalid_argument("MicrophysicsProcess: columns differ in levels");
      cols[(size_t)c] = column(atmosphere[c], prognostics[c],
                               diagnostics ? &diagnostics[c] : nullptr, tendencies[c]);
    }
    const mam4b_status st = mam4b_step_columns(ctx_.get(), cols.data(), ncol, nlev, dt,
                                               config_.precision, stream);
    if (st != MAM4B_OK) {
      char msg[256];
      mam4b_last_error(ctx_.get(), msg, sizeof(msg));
      throw std::runtime_error(std::string("MicrophysicsProcess: ") + msg);
    }
  }

  /// The C-ABI column of one set of containers (the mapping above).
  static mam4b_column column(const Atmosphere &atm, const Prognostics &prog,
                             const Diagnostics *diag, const Tendencies &tend) {
    mam4b_column col = {};
    col.in[MAM4B_IN_T] = atm.temperature.data();
    col.in[MAM4B_IN_P] = atm.pressure.data();
    col.in[MAM4B_IN_ZM] = atm.height.data();
    col.in[MAM4B_IN_QV] = atm.vapor_mixing_ratio.data();
    col.in[MAM4B_IN_CLD] = atm.cloud_fraction.data();
    const int h2so4 = static_cast<int>(GasId::H2SO4), soag = static_cast<int>(GasId::SOAG);
    col.in[MAM4B_IN_H2SO4] = prog.q_gas[h2so4].data();
    col.in[MAM4B_IN_SOAG] = prog.q_gas[soag].data();
    col.pblh = atm.planetary_boundary_layer_height;
    col.tend[0] = tend.q_gas[h2so4].data();
    col.tend[1] = tend.q_gas[soag].data();
    int p = 0;
    for (int m = 0; m < AeroConfig::num_modes(); ++m) {
      for (int a = 0; a < num_species_mode(m); ++a, ++p) {
        col.in[MAM4B_IN_AER_I + p] = prog.q_aero_i[m][a].data();
        col.in[MAM4B_IN_AER_C + p] = prog.q_aero_c[m][a].data();
        col.tend[2 + p] = tend.q_aero_i[m][a].data();
        col.tend[27 + p] = tend.q_aero_c[m][a].data();
      }
      col.in[MAM4B_IN_AER_I + p] = prog.n_mode_i[m].data();
      col.in[MAM4B_IN_AER_C + p] = prog.n_mode_c[m].data();
      col.tend[2 + p] = tend.n_mode_i[m].data();
      col.tend[27 + p] = tend.n_mode_c[m].data();
      ++p;
      if (diag) {
        col.mode_out[m] = diag->dry_geometric_mean_diameter_i[m].data();
        col.mode_out[4 + m] = diag->wet_geometric_mean_diameter_i[m].data();
        col.mode_out[8 + m] = diag->wet_density[m].data();
      }
    }
    return col;
  }

  mam4b_ctx *context() const { return ctx_.get(); }

private:
  Config config_;
  std::shared_ptr<mam4b_ctx> ctx_;  // shared by the copies AeroProcess makes
};

}  // namespace mam4

#endif
