// FP64 throughput of this GPU, for the benchmark's FP64 roofline of the contact and solver
// kernels (no counterpart in the reference).  Every thread runs eight independent chains of
// fused multiply-adds (fma, one DFMA instruction each, two flops), long enough to hide the
// pipeline latency, on a grid of 8 CTAs of 256 threads per SM; the kernel time comes from
// CUDA events around it.  The library's own kernels are built without contraction
// (-fmad=false), so each of their multiplies and adds is one instruction: their FP64 flop rate
// tops out at half this figure.
#include <cuda_runtime.h>

#include "abd_common.cuh"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_dfma_chains(int iters, double* sink) {
  double a[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) a[c] = 1.0 + 1e-9 * (threadIdx.x + c);
  const double m = 0.999999999, k = 1e-12;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = fma(a[c], m, k);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += a[c];
  if (s == 12345.678) *sink = s;  // keeps the chains live; never true
}

}  // namespace

extern "C" int abd_fp64_peak(double* tflops) {
  if (!tflops) return ABD_ERR_INVALID;
  int dev = 0, sms = 0;
  if (ABD_NOTE(cudaGetDevice(&dev)) || ABD_NOTE(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)))
    return ABD_ERR_CUDA;
  double* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int r = ABD_OK;
  if (ABD_NOTE(cudaMalloc(&sink, sizeof(double))) || ABD_NOTE(cudaEventCreate(&e0)) || ABD_NOTE(cudaEventCreate(&e1)))
    r = ABD_ERR_CUDA;
  const int blocks = 8 * sms, iters = 1 << 14;
  float best = 0.f;
  for (int rep = 0; r == ABD_OK && rep < 4; ++rep) {  // the first launch warms up
    cudaEventRecord(e0, 0);
    k_dfma_chains<<<blocks, 256>>>(iters, sink);
    cudaEventRecord(e1, 0);
    if (ABD_NOTE(cudaEventSynchronize(e1)) != cudaSuccess) {
      r = ABD_ERR_CUDA;
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best == 0.f || ms < best)) best = ms;
  }
  if (sink) cudaFree(sink);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (r != ABD_OK || best <= 0.f) return r ? r : ABD_ERR_CUDA;
  const double flops = 2.0 * kChains * (double)iters * 256.0 * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return ABD_OK;
}
