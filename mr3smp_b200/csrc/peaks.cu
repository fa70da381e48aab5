// peaks.cu -- in-run FP64 peak measurement used as the roofline denominator.
//
// The MRRR kernels are bound by FP64 division (one per Sturm-count step) and
// FP64 arithmetic, not by tensor cores or copies.  These two kernels measure,
// on the device in use, the throughput of IEEE double division and of FP64
// fused multiply-add with many independent chains per SM.
#include <cuda_runtime.h>

#include "mr3_cuda.h"

namespace {
__global__ void k_peak_div(double *out, int iters) {
  double x0 = 1.0 + threadIdx.x * 1e-6, x1 = x0 + 0.25, x2 = x0 + 0.5, x3 = x0 + 0.75;
  for (int i = 0; i < iters; i++) {
    x0 = 0.75 / (x0 + 1.5);
    x1 = 0.75 / (x1 + 1.5);
    x2 = 0.75 / (x2 + 1.5);
    x3 = 0.75 / (x3 + 1.5);
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3;
}

__global__ void k_peak_fma(double *out, int iters) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = 1.0 + (threadIdx.x + k) * 1e-6;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = fma(x[k], 0.999999, 1e-7);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

extern "C" int mr3_cuda_fp64_peaks(int device, double *fma_tflops, double *div_gops) {
  if (cudaSetDevice(device) != cudaSuccess) return MR3_EMISC;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MR3_EMISC;
  const int blocks = prop.multiProcessorCount * 8, threads = 256;
  double *out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return MR3_EMISC;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float ms = 0.f;
  const int it_div = 4000, it_fma = 20000;
  k_peak_div<<<blocks, threads>>>(out, 100);
  cudaEventRecord(e0);
  k_peak_div<<<blocks, threads>>>(out, it_div);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  *div_gops = 4.0 * blocks * threads * (double)it_div / (ms * 1e-3) * 1e-9;
  k_peak_fma<<<blocks, threads>>>(out, 100);
  cudaEventRecord(e0);
  k_peak_fma<<<blocks, threads>>>(out, it_fma);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(&ms, e0, e1);
  *fma_tflops = 2.0 * 8.0 * blocks * threads * (double)it_fma / (ms * 1e-3) * 1e-12;
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return err == cudaSuccess ? MR3_OK : MR3_EMISC;
}
