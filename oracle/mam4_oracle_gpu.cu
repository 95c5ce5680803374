// mam4_oracle_gpu.cu -- the plain-C restatement (mam4_oracle.c) compiled for
// the GPU: the "libm-matched diagnostic oracle".
//
// TEST INFRASTRUCTURE ONLY (oracle/libmam4oracle_gpu.so). One thread runs
// the restatement's step for one cell, with CUDA's math library and, like
// the product kernel, without FMA contraction (--fmad=false). Comparing it
// with the product kernel isolates algorithmic differences (same libm on
// both sides); comparing it with the host build of the same source
// isolates the effect of CUDA's libm versus glibc.
#define ORACLE_GPU 1
#include "mam4_oracle.c"

#include <cuda_runtime.h>

__global__ void oracle_step_kernel(int n, const double *in, size_t ld, const double *pblh_cell,
                                   double *out, size_t ldo, double *diag, size_t ldd, double dt,
                                   mam4b_config cfg) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n)
    return;
  calcsize_data cd;
  calcsize_init(&cd);
  step_cell(&cd, in, ld, (size_t)c, pblh_cell[c], out, ldo, diag, ldd, dt, &cfg);
}

// Host arrays in, host arrays out (field-major, like mam4orc_step).
extern "C" int mam4orcgpu_step(int ncell, const double *in, size_t ld_in,
                               const double *pblh_cell, double *out, size_t ld_out,
                               double *diag, size_t ld_diag, double dt,
                               const mam4b_config *cfg) {
  if (ncell <= 0)
    return 0;
  const size_t n = (size_t)ncell;
  double *d_in = nullptr, *d_pb = nullptr, *d_out = nullptr, *d_dg = nullptr;
  cudaError_t e = cudaMalloc(&d_in, MAM4B_NIN * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_pb, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, MAM4B_NOUT * n * sizeof(double));
  if (e == cudaSuccess && diag) e = cudaMalloc(&d_dg, MAM4B_NDIAG * n * sizeof(double));
  for (int f = 0; f < MAM4B_NIN && e == cudaSuccess; ++f)
    e = cudaMemcpy(d_in + f * n, in + f * ld_in, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_pb, pblh_cell, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    oracle_step_kernel<<<(ncell + 63) / 64, 64>>>(ncell, d_in, n, d_pb, d_out, n, d_dg, n, dt, *cfg);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaDeviceSynchronize();
  for (int f = 0; f < MAM4B_NOUT && e == cudaSuccess; ++f)
    e = cudaMemcpy(out + f * ld_out, d_out + f * n, n * sizeof(double), cudaMemcpyDeviceToHost);
  for (int f = 0; diag && f < MAM4B_NDIAG && e == cudaSuccess; ++f)
    e = cudaMemcpy(diag + f * ld_diag, d_dg + f * n, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d_in);
  cudaFree(d_pb);
  cudaFree(d_out);
  cudaFree(d_dg);
  return e == cudaSuccess ? 0 : 2;
}
