// fp_peaks.cu -- measurement helper (libmam4b_peaks.so): the FP64 and FP32
// vector peak of the device, the denominator of the step's FP64 roofline.
//
// Every thread runs 8 independent fused multiply-add chains (a = a*b + c)
// in registers; 4 blocks of 256 threads per SM keep every FMA pipe busy.
// FLOPs = 2 per FMA. The result is stored so that nothing is eliminated.
#include <cuda_runtime.h>

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T *out, T b, T c, int iters) {
  const unsigned tid = blockIdx.x * blockDim.x + threadIdx.x;
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    a[k] = (T)(tid & 1023) * (T)1e-3 + (T)k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      a[k] = fma(a[k], b, c);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    s += a[k];
  out[tid] = s;
}

template <typename T>
int measure(double *gflops, double *ms_best) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 1;
  const int block = 256, grid = sms * 4, iters = 16384;
  T *out = nullptr;
  if (cudaMalloc(&out, (size_t)grid * block * sizeof(T)) != cudaSuccess)
    return 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    fma_chain_kernel<T><<<grid, block>>>(out, (T)0.9999999, (T)1e-7, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best)  // the first launch warms up
      best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess)
    return 1;
  *ms_best = best;
  *gflops = 2.0 * 8.0 * (double)iters * grid * block / (best * 1e-3) / 1e9;
  return 0;
}

}  // namespace

// fp64 != 0: double precision, else single. Returns 0 on success.
extern "C" int mam4b_peak_gflops(int fp64, double *gflops, double *ms) {
  if (!gflops || !ms)
    return 1;
  return fp64 ? measure<double>(gflops, ms) : measure<float>(gflops, ms);
}
