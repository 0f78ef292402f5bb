// Measurement aid for bench.py, built into its own library (libhv_peaks.so)
// and never called by the engine: the FP64 FMA throughput of the device,
// the denominator of the FP64 roofline fraction. Each thread runs eight
// independent FMA chains so the pipe, not latency, is the limit.
#include <cuda_runtime.h>

namespace {
__global__ void fma_chains(double* out, int iters, double a, double b) {
  double r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = threadIdx.x * 1e-9 + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fma(r[k], a, b);
  }
  double s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}
}  // namespace

extern "C" __attribute__((visibility("default"))) int hv_peak_fp64(int device, double* tflops) {
  if (cudaSetDevice(device) != cudaSuccess) return 1;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  double* out = nullptr;
  if (cudaMalloc(&out, 8) != cudaSuccess) return 1;
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    fma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  double flops = 2.0 * 8.0 * iters * double(blocks) * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
