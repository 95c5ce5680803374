// microphysics_process_check.cpp -- test harness of the C++ process
// include/mam4b_microphysics.hpp over the mam4xx reference containers.
//
// TEST INFRASTRUCTURE ONLY (tests/cpp/_build/libmam4b_process_check.so,
// built by tests/cpp/build_process_check.py where the mam4xx tree is
// present; the reference headers come through the host shim in
// oracle/shim). It fills mam4::Atmosphere, Prognostics, Diagnostics and
// Tendencies per column from a field-major input slab (the layout of
// include/mam4b.h) with views over CUDA managed memory, runs
// mam4::MicrophysicsProcess either through the reference's own
// mam4::AeroProcess<> wrapper one column at a time (validate +
// compute_tendencies, src/validation/aero_process.hpp:19-129) or through
// its batched entry over all columns, and returns the tendencies and mode
// outputs in the slab layout, for comparison with mam4b_step_slab.

#include <aero_process.hpp>
#include <mam4xx/mam4.hpp>

#include "../../include/mam4b_microphysics.hpp"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

namespace {

using mam4::ColumnView;
using mam4::Real;

struct Managed {
  std::vector<double *> bufs;
  double *get(size_t n) {
    double *p = nullptr;
    if (cudaMallocManaged(&p, n * sizeof(double)) != cudaSuccess)
      return nullptr;
    std::memset(p, 0, n * sizeof(double));
    bufs.push_back(p);
    return p;
  }
  ~Managed() {
    for (double *p : bufs)
      cudaFree(p);
  }
};

}  // namespace

// Returns 0 on success; 1 on a failed allocation, 2 on a failed validate(),
// 3 on an exception (message in err).
extern "C" int mam4b_process_check(int ncol, int nlev, const double *in_slab, const double *pblh,
                                   double dt, int batched, double *tend_out, double *mode_out,
                                   char *err, int errlen) {
  const size_t ncell = (size_t)ncol * nlev;
  Managed mem;
  double *in = mem.get((size_t)MAM4B_NIN * ncell);
  double *tend = mem.get((size_t)MAM4B_NUM_PROG * ncell);
  double *mode = mem.get((size_t)12 * ncell);
  double *zeros = mem.get(ncell + ncol);  // unused atmosphere and gas fields
  if (!in || !tend || !mode || !zeros)
    return 1;
  std::memcpy(in, in_slab, (size_t)MAM4B_NIN * ncell * sizeof(double));
  auto field = [&](double *base, int f, int c) { return base + (size_t)f * ncell + (size_t)c * nlev; };
  std::vector<mam4::Atmosphere> atm;
  std::vector<mam4::Surface> sfc((size_t)ncol);
  std::vector<mam4::Prognostics> prog, tends;
  std::vector<mam4::Diagnostics> diag;
  for (int c = 0; c < ncol; ++c) {
    const ColumnView z0(zeros, nlev), zi(zeros, nlev + 1);
    atm.emplace_back(nlev, ColumnView(field(in, MAM4B_IN_T, c), nlev),
                     ColumnView(field(in, MAM4B_IN_P, c), nlev),
                     ColumnView(field(in, MAM4B_IN_QV, c), nlev), z0, z0, z0, z0,
                     ColumnView(field(in, MAM4B_IN_ZM, c), nlev), z0, zi,
                     ColumnView(field(in, MAM4B_IN_CLD, c), nlev), z0, pblh[c]);
    mam4::Prognostics p(nlev), t(nlev);
    mam4::Diagnostics d(nlev);
    for (int g = 0; g < mam4::AeroConfig::num_gas_ids(); ++g) {
      p.q_gas[g] = p.q_gas_avg[g] = t.q_gas[g] = t.q_gas_avg[g] = z0;
    }
    const int h2so4 = static_cast<int>(mam4::GasId::H2SO4);
    const int soag = static_cast<int>(mam4::GasId::SOAG);
    p.q_gas[h2so4] = ColumnView(field(in, MAM4B_IN_H2SO4, c), nlev);
    p.q_gas[soag] = ColumnView(field(in, MAM4B_IN_SOAG, c), nlev);
    t.q_gas[h2so4] = ColumnView(field(tend, 0, c), nlev);
    t.q_gas[soag] = ColumnView(field(tend, 1, c), nlev);
    int slot = 0;
    for (int m = 0; m < mam4::AeroConfig::num_modes(); ++m) {
      for (int a = 0; a < mam4::AeroConfig::num_aerosol_ids(); ++a)
        p.q_aero_i[m][a] = p.q_aero_c[m][a] = t.q_aero_i[m][a] = t.q_aero_c[m][a] = z0;
      for (int a = 0; a < mam4::num_species_mode(m); ++a, ++slot) {
        p.q_aero_i[m][a] = ColumnView(field(in, MAM4B_IN_AER_I + slot, c), nlev);
        p.q_aero_c[m][a] = ColumnView(field(in, MAM4B_IN_AER_C + slot, c), nlev);
        t.q_aero_i[m][a] = ColumnView(field(tend, 2 + slot, c), nlev);
        t.q_aero_c[m][a] = ColumnView(field(tend, 27 + slot, c), nlev);
      }
      p.n_mode_i[m] = ColumnView(field(in, MAM4B_IN_AER_I + slot, c), nlev);
      p.n_mode_c[m] = ColumnView(field(in, MAM4B_IN_AER_C + slot, c), nlev);
      t.n_mode_i[m] = ColumnView(field(tend, 2 + slot, c), nlev);
      t.n_mode_c[m] = ColumnView(field(tend, 27 + slot, c), nlev);
      ++slot;
      d.dry_geometric_mean_diameter_i[m] = ColumnView(field(mode, m, c), nlev);
      d.wet_geometric_mean_diameter_i[m] = ColumnView(field(mode, 4 + m, c), nlev);
      d.wet_density[m] = ColumnView(field(mode, 8 + m, c), nlev);
    }
    prog.push_back(p);
    tends.push_back(t);
    diag.push_back(d);
  }
  try {
    const mam4::AeroConfig aero_config;
    const mam4::MicrophysicsProcess::Config cfg;
    if (batched) {
      mam4::MicrophysicsProcess impl;
      impl.init(aero_config, cfg);
      impl.compute_tendencies_columns(0.0, dt, ncol, atm.data(), sfc.data(), prog.data(),
                                      diag.data(), tends.data(), nullptr);
      if (mam4b_synchronize(impl.context()) != MAM4B_OK)
        throw std::runtime_error("device step failed");
    } else {
      mam4::AeroProcess<mam4::MicrophysicsProcess> process(aero_config, cfg);
      Kokkos::TeamMember team;
      for (int c = 0; c < ncol; ++c) {
        if (!process.validate(team, atm[c], sfc[c], prog[c]))
          return 2;
        process.compute_tendencies(team, 0.0, dt, atm[c], sfc[c], prog[c], diag[c], tends[c]);
      }
    }
  } catch (const std::exception &e) {
    if (err && errlen > 0)
      std::snprintf(err, (size_t)errlen, "%s", e.what());
    return 3;
  }
  if (cudaDeviceSynchronize() != cudaSuccess)
    return 3;
  std::memcpy(tend_out, tend, (size_t)MAM4B_NUM_PROG * ncell * sizeof(double));
  std::memcpy(mode_out, mode, (size_t)12 * ncell * sizeof(double));
  return 0;
}

// The field mapping of MicrophysicsProcess::column() without a device: one
// column of containers over host arrays laid out like the slabs above;
// writes, for every pointer of the resulting mam4b_column, the slab field
// it points at (-1 for NULL, -2 for a pointer outside the slabs):
// in[57], tend[52], mode_out[16]. Also checks name() and validate().
extern "C" int mam4b_process_check_mapping(int nlev, int *in_field, int *tend_field,
                                           int *mode_field) {
  std::vector<double> in((size_t)MAM4B_NIN * nlev, 1.0), tend((size_t)MAM4B_NUM_PROG * nlev),
      mode((size_t)12 * nlev), zeros((size_t)nlev + 1);
  auto col = [&](std::vector<double> &v, int f) { return ColumnView(v.data() + (size_t)f * nlev, nlev); };
  const ColumnView z0(zeros.data(), nlev), zi(zeros.data(), nlev + 1);
  mam4::Atmosphere atm(nlev, col(in, MAM4B_IN_T), col(in, MAM4B_IN_P), col(in, MAM4B_IN_QV), z0, z0,
                       z0, z0, col(in, MAM4B_IN_ZM), z0, zi, col(in, MAM4B_IN_CLD), z0, 500.0);
  mam4::Prognostics p(nlev), t(nlev);
  mam4::Diagnostics d(nlev);
  for (int g = 0; g < mam4::AeroConfig::num_gas_ids(); ++g)
    p.q_gas[g] = p.q_gas_avg[g] = t.q_gas[g] = t.q_gas_avg[g] = z0;
  p.q_gas[static_cast<int>(mam4::GasId::H2SO4)] = col(in, MAM4B_IN_H2SO4);
  p.q_gas[static_cast<int>(mam4::GasId::SOAG)] = col(in, MAM4B_IN_SOAG);
  t.q_gas[static_cast<int>(mam4::GasId::H2SO4)] = col(tend, 0);
  t.q_gas[static_cast<int>(mam4::GasId::SOAG)] = col(tend, 1);
  int slot = 0;
  for (int m = 0; m < mam4::AeroConfig::num_modes(); ++m) {
    for (int a = 0; a < mam4::AeroConfig::num_aerosol_ids(); ++a)
      p.q_aero_i[m][a] = p.q_aero_c[m][a] = t.q_aero_i[m][a] = t.q_aero_c[m][a] = z0;
    for (int a = 0; a < mam4::num_species_mode(m); ++a, ++slot) {
      p.q_aero_i[m][a] = col(in, MAM4B_IN_AER_I + slot);
      p.q_aero_c[m][a] = col(in, MAM4B_IN_AER_C + slot);
      t.q_aero_i[m][a] = col(tend, 2 + slot);
      t.q_aero_c[m][a] = col(tend, 27 + slot);
    }
    p.n_mode_i[m] = col(in, MAM4B_IN_AER_I + slot);
    p.n_mode_c[m] = col(in, MAM4B_IN_AER_C + slot);
    t.n_mode_i[m] = col(tend, 2 + slot);
    t.n_mode_c[m] = col(tend, 27 + slot);
    ++slot;
    d.dry_geometric_mean_diameter_i[m] = col(mode, m);
    d.wet_geometric_mean_diameter_i[m] = col(mode, 4 + m);
    d.wet_density[m] = col(mode, 8 + m);
  }
  const mam4b_column c = mam4::MicrophysicsProcess::column(atm, p, &d, t);
  auto which = [&](const double *ptr, const std::vector<double> &v, int nf) {
    if (!ptr)
      return -1;
    if (ptr < v.data() || ptr >= v.data() + (size_t)nf * nlev || (ptr - v.data()) % nlev)
      return -2;
    return (int)((ptr - v.data()) / nlev);
  };
  for (int f = 0; f < MAM4B_NIN; ++f)
    in_field[f] = which(c.in[f], in, MAM4B_NIN);
  for (int f = 0; f < MAM4B_NUM_PROG; ++f)
    tend_field[f] = which(c.tend[f], tend, MAM4B_NUM_PROG);
  for (int f = 0; f < MAM4B_NOUT - MAM4B_NUM_PROG; ++f)
    mode_field[f] = which(c.mode_out[f], mode, 12);
  mam4::MicrophysicsProcess impl;
  Kokkos::TeamMember team;
  const bool ok = impl.validate(mam4::AeroConfig(), team, atm, mam4::Surface(), p);
  in[(size_t)MAM4B_IN_T * nlev] = -1.0;  // a negative temperature fails validation
  const bool bad = impl.validate(mam4::AeroConfig(), team, atm, mam4::Surface(), p);
  return (c.pblh == 500.0 && ok && !bad && std::strlen(impl.name()) > 0) ? 0 : 1;
}
