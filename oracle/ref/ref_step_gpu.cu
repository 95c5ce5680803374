// ref_step_gpu.cu -- the mam4xx reference headers compiled for the GPU.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref/libmam4ref_gpu.so). The reference
// headers (src/mam4xx/modal_aero_calcsize.hpp, water_uptake.hpp,
// mam4_amicphys.hpp and their includes) are included read-only from the
// mam4xx source tree and compiled unchanged by nvcc against the host/device
// shim in oracle/shim, with CUDA's math library and without FMA contraction
// (--fmad=false), like the product kernels. One thread runs the step of one
// grid cell, composed exactly as oracle/ref/ref_step.cpp composes it on the
// host (step_cell there; no per-process diagnostics here):
//   pack state_q/qqcw (utils.hpp:222-259) -> modal_aero_calcsize_sub
//   (modal_aero_calcsize.hpp:750) -> modal_aero_water_uptake_dr
//   (water_uptake.hpp:481) -> calcsize tendencies applied for one step ->
//   mmr -> vmr (gas_chem_mechanism.hpp:31-38) -> modal_aero_amicphys_intr
//   (mam4_amicphys.hpp:2120) -> vmr -> mmr, tendency = (after - before)/dt.
//
// It differs from the host build of the same headers only through the math
// library, so comparing the product kernels with it bit for bit checks
// their algorithm against the reference itself.

#include <mam4xx/mam4_amicphys.hpp>
#include <mam4xx/modal_aero_calcsize.hpp>
#include <mam4xx/water_uptake.hpp>

#include "../oracle_api.h"

#include <cuda_runtime.h>

namespace {

using mam4::Real;
using CalcsizeData = mam4::modal_aero_calcsize::CalcsizeData;

constexpr double kMwDryAir = 28.966; // kg/kmol

__host__ __device__ bool is_number_slot(int i31) {
  return i31 == 13 || i31 == 18 || i31 == 26 || i31 == 30;
}
// mmr <-> vmr factors of the 31 tracers (gas_chem_mechanism.hpp:31-38),
// evaluated on the host from the mechanism's molecular weights and kept in
// constant memory for the device (the namespace array is a host object)
struct UnitFactors {
  double to_vmr[31], to_mmr[31];
};
__constant__ UnitFactors c_units;
UnitFactors host_units() {
  UnitFactors u;
  for (int i = 0; i < 31; ++i) {
    u.to_vmr[i] = is_number_slot(i) ? kMwDryAir : kMwDryAir / mam4::gas_chemistry::adv_mass[i];
    u.to_mmr[i] = is_number_slot(i) ? 1.0 / kMwDryAir : mam4::gas_chemistry::adv_mass[i] / kMwDryAir;
  }
  return u;
}
__host__ __device__ double to_vmr_factor(int i31) {
#if defined(__CUDA_ARCH__)
  return c_units.to_vmr[i31];
#else
  static const UnitFactors u = host_units();
  return u.to_vmr[i31];
#endif
}
__host__ __device__ double to_mmr_factor(int i31) {
#if defined(__CUDA_ARCH__)
  return c_units.to_mmr[i31];
#else
  static const UnitFactors u = host_units();
  return u.to_mmr[i31];
#endif
}

__host__ __device__ mam4::microphysics::AmicPhysConfig amicphys_config(const mam4b_config &c) {
  mam4::microphysics::AmicPhysConfig a;
  a.do_cond = c.do_cond != 0;
  a.do_rename = c.do_rename != 0;
  a.do_newnuc = c.do_newnuc != 0;
  a.do_coag = c.do_coag != 0;
  a.gaexch_h2so4_uptake_optaa = c.gaexch_h2so4_uptake_optaa;
  a.newnuc_h2so4_conc_optaa = c.newnuc_h2so4_conc_optaa;
  return a;
}

__host__ __device__ void step_cell(const CalcsizeData &cd, const double *in, size_t ld, size_t c,
                          double pblh, double *out, size_t ldo, double dt,
                          const mam4b_config &cfg) {
  auto IN = [&](int f) { return in[(size_t)f * ld + c]; };
  Real state_q[40] = {}, qqcw[40] = {};
  state_q[0] = IN(MAM4B_IN_QV);
  state_q[11] = IN(MAM4B_IN_H2SO4);
  state_q[14] = IN(MAM4B_IN_SOAG);
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    state_q[15 + p] = IN(MAM4B_IN_AER_I + p);
    qqcw[15 + p] = IN(MAM4B_IN_AER_C + p);
  }
  const Real temp = IN(MAM4B_IN_T), pmid = IN(MAM4B_IN_P);
  const Real cld = IN(MAM4B_IN_CLD);

  // calcsize on copies (ref_step.cpp calcsize_cell)
  Real dgncur_a[4], dgncur_c[4], ptend[40], dqqcwdt[40];
  {
    for (int i = 0; i < 40; ++i) {
      ptend[i] = 0;
      dqqcwdt[i] = 0;
    }
    Real sq[40], cw[40];
    for (int i = 0; i < 40; ++i) {
      sq[i] = state_q[i];
      cw[i] = qqcw[i];
    }
    mam4::modal_aero_calcsize::modal_aero_calcsize_sub(sq, cw, dt, cd, dgncur_a, dgncur_c,
                                                       ptend, dqqcwdt);
  }
  // water uptake on copies (ref_step.cpp water_uptake_cell)
  Real dgncur_awet[4], qaerwat[4], wetdens[4];
  {
    Real sq[40], dgn[4];
    for (int i = 0; i < 40; ++i)
      sq[i] = state_q[i];
    for (int m = 0; m < 4; ++m)
      dgn[m] = dgncur_a[m];
    mam4::water_uptake::modal_aero_water_uptake_dr(
        cd.nspec_amode, cd.specdens_amode, cd.spechygro, cd.lspectype_amode, sq, temp, pmid,
        cld, dgn, dgncur_awet, qaerwat, wetdens);
  }
  for (int i = 15; i < 40; ++i) {
    state_q[i] = mam4::max(0.0, state_q[i] + ptend[i] * dt);
    qqcw[i] = mam4::max(0.0, qqcw[i] + dqqcwdt[i] * dt);
  }
  Real qq[31], qqcw31[31];
  for (int i = 0; i < 31; ++i) {
    qq[i] = state_q[9 + i] * to_vmr_factor(i);
    qqcw31[i] = qqcw[9 + i] * to_vmr_factor(i);
  }
  // amicphys without diagnostics (ref_step.cpp amicphys_cell)
  {
    using View2D = mam4::microphysics::View2D;
    View2D d[5];
    Real q_pregaschem[31], q_precldchem[31], qqcw_precldchem[31];
    for (int i = 0; i < 31; ++i) {
      q_pregaschem[i] = qq[i];
      q_precldchem[i] = qq[i];
      qqcw_precldchem[i] = qqcw31[i];
    }
    const Real pdel_unused = 0.0; // passed through, never read by amicphys
    mam4::microphysics::modal_aero_amicphys_intr(
        amicphys_config(cfg), dt, cfg.n_so4_monolayers_pcage, temp, pmid, pdel_unused,
        IN(MAM4B_IN_ZM), pblh, IN(MAM4B_IN_QV), cld, qq, qqcw31, 0, d[0], d[1], d[2], d[3],
        d[4], q_pregaschem, q_precldchem, qqcw_precldchem, dgncur_a, dgncur_awet, wetdens);
  }
  auto OUT = [&](int f) -> double & { return out[(size_t)f * ldo + c]; };
  OUT(MAM4B_OUT_TEND + 0) = (qq[2] * to_mmr_factor(2) - IN(MAM4B_IN_H2SO4)) / dt;
  OUT(MAM4B_OUT_TEND + 1) = (qq[5] * to_mmr_factor(5) - IN(MAM4B_IN_SOAG)) / dt;
  for (int p = 0; p < MAM4B_NUM_POPS; ++p) {
    const int i31 = 6 + p;
    OUT(MAM4B_OUT_TEND + 2 + p) = (qq[i31] * to_mmr_factor(i31) - IN(MAM4B_IN_AER_I + p)) / dt;
    OUT(MAM4B_OUT_TEND + 27 + p) =
        (qqcw31[i31] * to_mmr_factor(i31) - IN(MAM4B_IN_AER_C + p)) / dt;
  }
  for (int m = 0; m < 4; ++m) {
    OUT(MAM4B_OUT_DGN_A + m) = dgncur_a[m];
    OUT(MAM4B_OUT_DGN_AWET + m) = dgncur_awet[m];
    OUT(MAM4B_OUT_WETDENS + m) = wetdens[m];
    OUT(MAM4B_OUT_QAERWAT + m) = qaerwat[m];
  }
}

__global__ void __launch_bounds__(64) ref_step_kernel(int n, const double *in, size_t ld,
                                                      const double *pblh_cell, double *out,
                                                      size_t ldo, double dt, mam4b_config cfg,
                                                      const CalcsizeData *cd) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n)
    return;
  step_cell(*cd, in, ld, (size_t)c, pblh_cell[c], out, ldo, dt, cfg);
}

__global__ void read_assert_count(unsigned long long *dst) {
  *dst = mam4shim::dev_assert_failures;
  mam4shim::dev_assert_failures = 0;
}

} // namespace

// The same composition run on the host through the nvcc build of the shim
// (glibc libm): equal to mam4ref_step bit for bit, which checks the shim's
// device mode on the CPU.
extern "C" int mam4refgpu_step_on_host(int ncell, const double *in, size_t ld_in,
                                       const double *pblh_cell, double *out, size_t ld_out,
                                       double dt, const mam4b_config *cfg) {
  CalcsizeData hd;
  hd.initialize();
  for (int c = 0; c < ncell; ++c)
    step_cell(hd, in, ld_in, (size_t)c, pblh_cell[c], out, ld_out, dt, *cfg);
  return 0;
}

// Host arrays in, host arrays out (field-major, like mam4ref_step). Writes
// the number of failed reference kernel asserts of the call to *n_asserts
// (may be NULL). Returns 0, or 2 when a CUDA call failed.
extern "C" int mam4refgpu_step(int ncell, const double *in, size_t ld_in,
                               const double *pblh_cell, double *out, size_t ld_out, double dt,
                               const mam4b_config *cfg, unsigned long long *n_asserts) {
  if (n_asserts)
    *n_asserts = 0;
  if (ncell <= 0)
    return 0;
  CalcsizeData hd;
  hd.initialize();
  const size_t n = (size_t)ncell;
  double *d_in = nullptr, *d_pb = nullptr, *d_out = nullptr;
  CalcsizeData *d_cd = nullptr;
  unsigned long long *d_cnt = nullptr;
  // the reference's per-cell working arrays live on the thread's stack
  // (about 16 KB per thread: ptxas -v of ref_step_kernel)
  cudaError_t e = cudaDeviceSetLimit(cudaLimitStackSize, 24 * 1024);
  if (e == cudaSuccess) e = cudaMalloc(&d_in, MAM4B_NIN * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_pb, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, MAM4B_NOUT * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_cd, sizeof(CalcsizeData));
  if (e == cudaSuccess) e = cudaMalloc(&d_cnt, sizeof(unsigned long long));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_cd, &hd, sizeof(CalcsizeData), cudaMemcpyHostToDevice);
  const UnitFactors units = host_units();
  if (e == cudaSuccess)
    e = cudaMemcpyToSymbol(c_units, &units, sizeof(UnitFactors));
  for (int f = 0; f < MAM4B_NIN && e == cudaSuccess; ++f)
    e = cudaMemcpy(d_in + f * n, in + f * ld_in, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_pb, pblh_cell, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    read_assert_count<<<1, 1>>>(d_cnt);  // clears the counter
    ref_step_kernel<<<(ncell + 63) / 64, 64>>>(ncell, d_in, n, d_pb, d_out, n, dt, *cfg, d_cd);
    read_assert_count<<<1, 1>>>(d_cnt);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaDeviceSynchronize();
  for (int f = 0; f < MAM4B_NOUT && e == cudaSuccess; ++f)
    e = cudaMemcpy(out + f * ld_out, d_out + f * n, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && n_asserts)
    e = cudaMemcpy(n_asserts, d_cnt, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d_in);
  cudaFree(d_pb);
  cudaFree(d_out);
  cudaFree(d_cd);
  cudaFree(d_cnt);
  return e == cudaSuccess ? 0 : 2;
}
