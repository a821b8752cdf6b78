// Device FP64 throughput, measured in-process: the denominator of the FP64 roofline fractions.
//
// Two microkernels run on every SM, each with enough independent chains per warp to keep its pipe
// busy: the FP64 tensor-core MMA (mma.sync m8n8k4 f64, the instruction the element-matrix products
// of the assembly issue) and the FP64 FMA pipe. Each is timed with CUDA events on a private stream
// (best of three), flops counted as 2 per multiply-add.
#include <cuda_runtime.h>

#include <algorithm>

#include "hfk_internal.h"

namespace {

constexpr int PEAK_CHAINS = 8;

__global__ void __launch_bounds__(256) peak_dmma_kernel(int iters, double seed, double* sink) {
  const double a = seed + 1e-9 * threadIdx.x, b = seed - 1e-9 * threadIdx.x;
  double c[PEAK_CHAINS][2];
#pragma unroll
  for (int k = 0; k < PEAK_CHAINS; ++k) c[k][0] = c[k][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < PEAK_CHAINS; ++k)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[k][0]), "+d"(c[k][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PEAK_CHAINS; ++k) s += c[k][0] + c[k][1];
  if (s == -1.0) sink[threadIdx.x] = s;  // never true for seed > 0: keeps the chains live
}

__global__ void __launch_bounds__(256) peak_dfma_kernel(int iters, double seed, double* sink) {
  double x[PEAK_CHAINS];
#pragma unroll
  for (int k = 0; k < PEAK_CHAINS; ++k) x[k] = seed + 1e-3 * k + 1e-9 * threadIdx.x;
  const double m = 0.999999, ad = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < PEAK_CHAINS; ++k) x[k] = fma(x[k], m, ad);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < PEAK_CHAINS; ++k) s += x[k];
  if (s == -1.0) sink[threadIdx.x] = s;
}

template <typename K>
double best_ms(K kernel, int grid, int iters, double* sink, cudaStream_t s) {
  cudaEvent_t e0, e1;
  HFK_CUDA(cudaEventCreate(&e0));
  HFK_CUDA(cudaEventCreate(&e1));
  kernel<<<grid, 256, 0, s>>>(iters / 8, 1.0, sink);  // warm-up (clocks, instruction cache)
  HFK_CUDA(cudaGetLastError());
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    HFK_CUDA(cudaEventRecord(e0, s));
    kernel<<<grid, 256, 0, s>>>(iters, 1.0, sink);
    HFK_CUDA(cudaGetLastError());
    HFK_CUDA(cudaEventRecord(e1, s));
    HFK_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    HFK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

}  // namespace

extern "C" int hfk_device_peak_fp64(double* dmma_tflops, double* dfma_tflops) {
  HFK_API_BEGIN
  HFK_REQUIRE(dmma_tflops && dfma_tflops, HFK_ERR_ARG, "null argument");
  int dev = 0, sms = 0;
  HFK_CUDA(cudaGetDevice(&dev));
  HFK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaStream_t s;
  HFK_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  double* sink = nullptr;
  HFK_CUDA(cudaMalloc(&sink, 256 * sizeof(double)));
  const int grid = sms * 8;  // 8 CTAs of 8 warps per SM: 64 warps, the SM's limit
  const int it_mma = 128, it_fma = 1024;  // about 0.1 s a run at the nominal FP64 rate
  const double ms_mma = best_ms(peak_dmma_kernel, grid, it_mma, sink, s);
  const double ms_fma = best_ms(peak_dfma_kernel, grid, it_fma, sink, s);
  const double threads = (double)grid * 256;
  // an m8n8k4 MMA is 8*8*4 multiply-adds per warp; an FMA one per thread
  *dmma_tflops = (threads / 32) * it_mma * PEAK_CHAINS * 2.0 * 256 / (ms_mma * 1e-3) / 1e12;
  *dfma_tflops = threads * it_fma * PEAK_CHAINS * 2.0 / (ms_fma * 1e-3) / 1e12;
  cudaFree(sink);
  cudaStreamDestroy(s);
  HFK_API_END
}
