// Exact, order-independent summation of FP64 values.
//
// Every reduction of the step (energies, the assembled gradient and Hessian blocks, the dot
// products of the Newton and Krylov iterations) is summed in fixed point instead of in
// floating point: each value is truncated to a multiple of 2^kXB0 and split into 32-bit
// digits that are added to 64-bit integer limbs.  Integer addition is associative, so the
// total does not depend on the order in which threads, warps, CTAs or atomics deliver the
// terms; it is rounded to FP64 once (round to nearest, ties to even).  A CPU restatement
// that sums the same terms therefore obtains the same bits, which is what makes whole time
// steps reproducible between the GPU and the oracle despite the condition number of the
// stiff contact systems (an accumulated rounding difference of one ulp in H or g is amplified
// by cond(H) ~ 1e10 in the Newton step).
//
// Range: digit i has weight 2^(kXB0 + 32 i), i < kXD.  Terms below 2^kXB0 (~1.6e-58) are
// dropped, terms of magnitude >= 2^128 raise XS_RANGE; each limb absorbs 2^31 additions.
#pragma once

#include <stdint.h>

namespace abd {

constexpr int kXD = 10;      // 32-bit digits
constexpr int kXB0 = -192;   // weight exponent of digit 0

enum : long long { XS_NAN = 1, XS_PINF = 2, XS_NINF = 4, XS_RANGE = 8 };

struct XSum {
  long long d[kXD];
  long long flags;
};

__device__ inline void xs_zero(XSum& s) {
#pragma unroll
  for (int i = 0; i < kXD; ++i) s.d[i] = 0;
  s.flags = 0;
}

// |x| truncated to the fixed-point grid = (u0 + u1 2^32 + u2 2^64) 2^(kXB0 + 32 j); the signed
// digits are returned in d0..d2.  Returns false when x contributes nothing (zero, below the
// grid, or non-finite / out of range, reported in fl).
__device__ inline bool xs_split(double x, int& j, long long& d0, long long& d1, long long& d2, long long& fl) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
  const int ex = (int)((bits >> 52) & 0x7ff);
  const unsigned long long frac = bits & 0xfffffffffffffULL;
  const bool neg = (bits >> 63) != 0;
  fl = 0;
  if (ex == 0x7ff) {
    fl = frac ? XS_NAN : (neg ? XS_NINF : XS_PINF);
    return false;
  }
  unsigned long long m = ex ? (frac | (1ULL << 52)) : frac;
  int sft = (ex ? ex : 1) - 1075 - kXB0;  // position of the mantissa's unit bit on the grid
  if (sft < 0) {
    if (sft <= -64) return false;
    m >>= -sft;
    sft = 0;
  }
  if (!m) return false;
  j = sft >> 5;
  const unsigned __int128 v = (unsigned __int128)m << (sft & 31);
  const unsigned long long u0 = (unsigned long long)v & 0xffffffffULL;
  const unsigned long long u1 = (unsigned long long)(v >> 32) & 0xffffffffULL;
  const unsigned long long u2 = (unsigned long long)(v >> 64);
  if (j + (u2 ? 2 : (u1 ? 1 : 0)) >= kXD) {
    fl = XS_RANGE;
    return false;
  }
  d0 = neg ? -(long long)u0 : (long long)u0;
  d1 = neg ? -(long long)u1 : (long long)u1;
  d2 = neg ? -(long long)u2 : (long long)u2;
  return true;
}

// register accumulator (no dynamic indexing of the limbs)
__device__ inline void xs_add(XSum& s, double x) {
  int j;
  long long d0, d1, d2, fl;
  if (!xs_split(x, j, d0, d1, d2, fl)) {
    s.flags |= fl;
    return;
  }
#pragma unroll
  for (int i = 0; i < kXD; ++i) s.d[i] += (i == j ? d0 : 0) + (i == j + 1 ? d1 : 0) + (i == j + 2 ? d2 : 0);
}

// accumulator in shared or global memory, updated with atomics (any order gives the same sum)
__device__ inline void xs_add_atomic(XSum* s, double x) {
  int j;
  long long d0, d1, d2, fl;
  if (!xs_split(x, j, d0, d1, d2, fl)) {
    if (fl) atomicOr((unsigned long long*)&s->flags, (unsigned long long)fl);
    return;
  }
  atomicAdd((unsigned long long*)&s->d[j], (unsigned long long)d0);
  if (d1 && j + 1 < kXD) atomicAdd((unsigned long long*)&s->d[j + 1], (unsigned long long)d1);
  if (d2 && j + 2 < kXD) atomicAdd((unsigned long long*)&s->d[j + 2], (unsigned long long)d2);
}

__device__ inline void xs_merge(XSum& s, const XSum& t) {
#pragma unroll
  for (int i = 0; i < kXD; ++i) s.d[i] += t.d[i];
  s.flags |= t.flags;
}

// warp-wide sum of every lane's accumulator (all lanes receive it)
__device__ inline void xs_warp_sum(XSum& s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int i = 0; i < kXD; ++i) s.d[i] += __shfl_xor_sync(0xffffffffu, s.d[i], o);
    s.flags |= __shfl_xor_sync(0xffffffffu, s.flags, o);
  }
}

// CTA-wide sum; the result is valid in thread 0.  sh: nwarps accumulators of shared memory.
__device__ inline void xs_block_sum(XSum& s, XSum* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  xs_warp_sum(s);
  if (lane == 0) sh[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < nw; ++w) xs_merge(s, sh[w]);
  __syncthreads();
}

__device__ inline int clz128(unsigned __int128 v) {
  const unsigned long long hi = (unsigned long long)(v >> 64), lo = (unsigned long long)v;
  return hi ? __clzll((long long)hi) : 64 + __clzll((long long)lo);
}

// The exact sum rounded to FP64 (to nearest, ties to even).
__device__ inline double xs_round(const XSum& s) {
  if (s.flags & (XS_NAN | XS_RANGE)) return __longlong_as_double(0x7ff8000000000000LL);
  if (s.flags & XS_PINF) return (s.flags & XS_NINF) ? __longlong_as_double(0x7ff8000000000000LL) : INFINITY;
  if (s.flags & XS_NINF) return -INFINITY;
  long long d[kXD + 1];
#pragma unroll
  for (int i = 0; i < kXD; ++i) d[i] = s.d[i];
  d[kXD] = 0;
  // carries: digits 0..kXD-1 into [0, 2^32), the rest into d[kXD] (signed)
#pragma unroll
  for (int i = 0; i < kXD; ++i) {
    const long long c = d[i] >> 32;  // arithmetic shift: floor division
    d[i] -= c * 4294967296LL;
    d[i + 1] += c;
  }
  const bool neg = d[kXD] < 0;
  if (neg) {
    // magnitude: negate and propagate again
#pragma unroll
    for (int i = 0; i <= kXD; ++i) d[i] = -d[i];
#pragma unroll
    for (int i = 0; i < kXD; ++i) {
      const long long c = d[i] >> 32;
      d[i] -= c * 4294967296LL;
      d[i + 1] += c;
    }
  }
  // d[kXD] now holds at most a few bits above digit kXD-1; fold it in as digit kXD
  int h = -1;
#pragma unroll
  for (int i = 0; i <= kXD; ++i)
    if (d[i] != 0) h = i;
  if (h < 0) return 0.0;
  const unsigned long long t2 = (unsigned long long)d[h];
  const unsigned long long t1 = h >= 1 ? (unsigned long long)d[h - 1] : 0ULL;
  const unsigned long long t0 = h >= 2 ? (unsigned long long)d[h - 2] : 0ULL;
  bool sticky = false;
#pragma unroll
  for (int i = 0; i <= kXD; ++i)
    if (i < h - 2 && d[i] != 0) sticky = true;
  const unsigned __int128 w = ((unsigned __int128)t2 << 64) | ((unsigned __int128)t1 << 32) | (unsigned __int128)t0;
  const int msb = 127 - clz128(w);  // >= 64 since t2 != 0
  const int drop = msb - 52;
  unsigned long long mant = (unsigned long long)(w >> drop);
  const unsigned __int128 rem = w & ((((unsigned __int128)1) << drop) - 1);
  const unsigned __int128 half = ((unsigned __int128)1) << (drop - 1);
  if (rem > half || (rem == half && (sticky || (mant & 1ULL)))) ++mant;
  const double r = ldexp((double)mant, drop + 32 * (h - 2) + kXB0);
  return neg ? -r : r;
}

}  // namespace abd
