/* FP32 throughput probe: the denominator of the pair kernels' roofline.
 *
 * The pair terms run on the FP32 (non-tensor) pipe, for which no measured
 * peak is supplied with the GPU, so it is measured here the same way the HBM
 * and GEMM peaks are: a kernel that does nothing but independent FP32 FMAs on
 * every SM, timed with CUDA events. Reported as TFLOP/s with FMA = 2 FLOP.
 */
#include <cuda_runtime.h>

#include "../../include/raspa_gpu.h"

#define PROBE_CHAINS 8

__global__ void __launch_bounds__(256) k_fma_probe(float *out, int iters, float a, float b)
{
  float x[PROBE_CHAINS];
#pragma unroll
  for (int c = 0; c < PROBE_CHAINS; c++) x[c] = threadIdx.x * 1e-3f + c;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int c = 0; c < PROBE_CHAINS; c++) x[c] = fmaf(x[c], a, b);
  }
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < PROBE_CHAINS; c++) s += x[c];
  if (s == 1.2345f) out[threadIdx.x] = s;   /* keeps the chains live; never true in practice */
}

extern "C" int rgpu_fp32_peak_probe(double *tflops, double *seconds)
{
  if (!tflops) return RGPU_E_INVALID;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return RGPU_E_NODEVICE;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  if (cudaMalloc((void **)&out, 256 * sizeof(float)) != cudaSuccess) return RGPU_E_CUDA;
  const int blocks = sms * 8, threads = 256, iters = 1 << 16;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_probe<<<blocks, threads>>>(out, 256, 0.999f, 1e-3f);   /* warm-up */
  float best = 1e30f;
  for (int rep = 0; rep < 3; rep++) {
    cudaEventRecord(e0);
    k_fma_probe<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return RGPU_E_CUDA;
  const double flop = 2.0 * PROBE_CHAINS * (double)iters * blocks * threads;
  *tflops = flop / (best * 1e-3) / 1e12;
  if (seconds) *seconds = best * 1e-3;
  return RGPU_SUCCESS;
}
