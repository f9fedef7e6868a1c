// Single-CTA exclusive scan used for small offset tables (body rows, radix histograms).
#pragma once
#include <cuda_runtime.h>

namespace abd {
namespace {

// exclusive scan of data[0..count) in place by one CTA of 1024 threads; *total (optional)
// receives the sum
__global__ void k_scan_excl(int* data, int count, int* total) {
  __shared__ int buf[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int start = 0; start < count; start += 1024) {
    const int i = start + threadIdx.x;
    const int v = i < count ? data[i] : 0;
    buf[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int add = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
      __syncthreads();
      buf[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < count) data[i] = carry + buf[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += buf[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

}  // namespace
}  // namespace abd
