// r3d_common.cuh -- device helpers shared by the pass kernels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "r3d_fft.cuh"
#include "r3d_internal.h"

namespace r3d {

// Debug builds (-DR3D_DEBUG_BOUNDS, the library's `debug` target): the
// iteration kernels check the index of each global access against its
// array's extent; a failed check sets bit 2 of the solve's error word and
// skips the access, and the host reports R3D_ECUDA.  Release builds compile
// the checks away.
#ifdef R3D_DEBUG_BOUNDS
__device__ __forceinline__ bool r3d_in_bounds(int *err, long long i, long long n) {
  if (i >= 0 && i < n) return true;
  atomicOr(err, 2);
  return false;
}
#define R3D_IN(d, i, n) r3d_in_bounds(&(d).ctl->err, (long long)(i), (long long)(n))
#else
#define R3D_IN(d, i, n) true
#endif

// ------------------------------------------------------------------ helpers
struct Batch {
  const Desc *d;       // [ns]
  const int *prefix;   // [ns + 1] CTA prefix of this pass
  int ns;
};

__device__ __forceinline__ int find_solve(const Batch &b, int cta) {
  int lo = 0, hi = b.ns - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (b.prefix[mid] <= cta)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <typename R>
__device__ __forceinline__ R closure_g(int clos, int pse_n, R earg) {
  // calculate_cuda.cu:1-16 (KH, HNC); PSE-n: sum_{i<=n} t*^i / i! for t* > 0.
  if (clos == HNC) return exp(earg);
  if (earg >= (R)0) {
    if (clos == KH || pse_n == 1) return (R)1 + earg;
    R term = (R)1, sum = (R)1;
    for (int i = 1; i <= pse_n; ++i) {
      term *= earg / (R)i;
      sum += term;
    }
    return sum;
  }
  return exp(earg);
}

template <typename R>
__device__ __forceinline__ bool solve_running(const Desc &d) {
  return d.ctl->status == RUNNING;
}

// Shared-memory carve-up: twiddles, digit-reversal table, pack twiddles, data.
template <typename C>
struct Smem {
  C *tw;
  int16_t *perm;
  C *ptw;  // half-sample twiddles e^{-i pi a / n}
  C *buf;
};
template <typename C>
__device__ __forceinline__ Smem<C> carve(char *sm, int L, int Lp) {
  Smem<C> s;
  s.tw = (C *)sm;
  size_t off = sizeof(C) * L;
  s.ptw = (C *)(sm + off);
  off += sizeof(C) * Lp;
  s.perm = (int16_t *)(sm + off);
  off += ((sizeof(int16_t) * L + 15) / 16) * 16;
  s.buf = (C *)(sm + off);
  return s;
}
// e^{-i pi a / n} for a in [0, L)
template <typename C>
__device__ void half_twiddles(C *ptw, int L, int n) {
  for (int a = threadIdx.x; a < L; a += blockDim.x) {
    double s, c;
    sincospi(-(double)a / (double)n, &s, &c);
    ptw[a].x = c;
    ptw[a].y = s;
  }
}


// Block-wide sum; valid in thread 0.  `red` holds kThreads/32 doubles.
__device__ __forceinline__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
  return s;
}

// K block-wide sums behind one pair of barriers, each added in the same
// order as block_sum (the warp's butterfly, then the warps in order), so the
// results equal K block_sum calls bit for bit; valid in thread 0.  `red`
// holds K * kThreads/32 doubles.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double *red) {
  constexpr int NW = kThreads / 32;
#pragma unroll
  for (int k = 0; k < K; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * NW + wid] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[k * NW + i];
      v[k] = s;
    }
}

}  // namespace r3d
