// Peak FP32 FMA rate of the SMs: the compute roofline of the plain FP32
// (SIMT) Legendre contraction.  Every thread advances kFmaChains independent
// FMA chains, enough independent work that each SM sub-partition always has
// an FMA ready to issue; 2048 threads run on every SM.

#include "dino_internal.cuh"

namespace dino {
namespace {

constexpr int kFmaChains = 8;
constexpr int kFmaThreads = 256;

__global__ void __launch_bounds__(kFmaThreads)
    fma_peak_kernel(float* out, int iters, float a, float b) {
  float x[kFmaChains];
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) x[c] = 1e-3f * (float)(threadIdx.x + c);
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c) x[c] = fmaf(x[c], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) s += x[c];
  // The chains converge to b / (1 - a) > 0, so this store never happens; it
  // keeps the arithmetic live.
  if (s == -1.0f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace dino

extern "C" DINO_API int dino_measure_fp32_fma_peak(int32_t iters, double* tflops) {
  DINO_REQUIRE(tflops != nullptr && iters > 0, DINO_ERR_ARG,
               "dino_measure_fp32_fma_peak: bad argument");
  int dev = 0, sms = 0, max_threads = 0;
  DINO_CHECK_CUDA(cudaGetDevice(&dev));
  DINO_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  DINO_CHECK_CUDA(
      cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
  const int blocks = sms * (max_threads / dino::kFmaThreads);
  float* out = nullptr;
  DINO_CHECK_CUDA(cudaMalloc(&out, sizeof(float) * (size_t)blocks * dino::kFmaThreads));
  cudaEvent_t e0, e1;
  DINO_CHECK_CUDA(cudaEventCreate(&e0));
  DINO_CHECK_CUDA(cudaEventCreate(&e1));
  dino::fma_peak_kernel<<<blocks, dino::kFmaThreads>>>(out, iters, 0.9999f, 1e-4f);
  DINO_CHECK_CUDA(cudaEventRecord(e0, 0));
  dino::fma_peak_kernel<<<blocks, dino::kFmaThreads>>>(out, iters, 0.9999f, 1e-4f);
  DINO_CHECK_CUDA(cudaEventRecord(e1, 0));
  int rc = dino::check_launch("fma_peak");
  float ms = 0.f;
  if (rc == DINO_OK) {
    DINO_CHECK_CUDA(cudaEventSynchronize(e1));
    DINO_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double flops = 2.0 * dino::kFmaChains * (double)iters * blocks * dino::kFmaThreads;
    *tflops = flops / (ms * 1e-3) / 1e12;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return rc;
}
