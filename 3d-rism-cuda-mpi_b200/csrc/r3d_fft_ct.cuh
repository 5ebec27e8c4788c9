// r3d_fft_ct.cuh -- compile-time-length FFT engine for the grid passes.
//
// Every pass keeps its tile in shared memory as PC "columns" of L complex
// elements, element (row r, column p) at buf[r * LD + p].  A CTA of kThreads
// threads is laid out column-fastest (p = tid % PC, row group g = tid / PC),
// so every shared-memory access of a warp touches consecutive columns and is
// free of bank conflicts; global loads/stores of the y/z passes are coalesced
// along the same columns, and the x passes store their rows transposed with
// an odd leading dimension.
//
// L, PC, LD and the radix plan are template constants, so all index
// arithmetic folds to shifts and multiplies.  Forward transforms are in-place
// decimation in time (input scattered to digit-reversed rows on load),
// inverse transforms in-place decimation in frequency (output gathered from
// digit-reversed rows on store); both unnormalised.  Twiddles come from
// per-length tables in global memory (read through L1).
#pragma once

#include "r3d_fft.cuh"
#include "r3d_internal.h"

namespace r3d {

// radices of L, outermost first (8s, then 4, 2, 3, 5)
struct Fac {
  int n;
  int r[12];
};
__host__ __device__ constexpr Fac factorize(int L) {
  Fac f{0, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
  int m = L;
  while (m > 1 && f.n < 12) {
    int r = (m % 8 == 0 && m != 16) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2
            : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : m;
    f.r[f.n++] = r;
    m /= r;
  }
  return f;
}
__host__ __device__ constexpr bool supported_length(int L) {
  Fac f = factorize(L);
  int p = 1;
  for (int i = 0; i < f.n; ++i) {
    if (f.r[i] != 2 && f.r[i] != 3 && f.r[i] != 4 && f.r[i] != 5 && f.r[i] != 8) return false;
    p *= f.r[i];
  }
  return p == L;
}
// product of radices s..n-1 (the sub-length below stage s)
__host__ __device__ constexpr int sub_len(int L, int s) {
  Fac f = factorize(L);
  int p = 1;
  for (int i = s; i < f.n; ++i) p *= f.r[i];
  return p;
}
// digit-reversed position of natural index I
template <int L>
__device__ __forceinline__ int digit_rev(int I) {
  constexpr Fac f = factorize(L);
  int P = 0, M = L;
#pragma unroll
  for (int k = 0; k < f.n; ++k) {
    M /= f.r[k];
    P += (I % f.r[k]) * M;
    I /= f.r[k];
  }
  return P;
}

template <int DIR, typename C>
__device__ __forceinline__ C tw_load(const C *tw, int e) {
  C w = tw[e];
  return DIR < 0 ? w : cconj(w);
}

// One DIT stage (radix R = f.r[S], sub-length M) on all PC columns, by NT
// threads (thread tid of the group).
template <int L, int PC, int LD, int S, int DIR, int NT, typename C>
__device__ __forceinline__ void ct_dit_stage(C *buf, const C *tw, int tid) {
  constexpr Fac f = factorize(L);
  constexpr int R = f.r[S];
  constexpr int M = sub_len(L, S + 1);
  constexpr int NB = L / R;       // butterflies per column
  constexpr int TR = NT / PC;     // row groups
  constexpr int TWS = L / (R * M);
  const int p = tid % PC, g = tid / PC;
  if (g >= TR) return;  // NT not a multiple of PC: the remainder idles
#pragma unroll
  for (int b0 = 0; b0 < NB; b0 += TR) {
    const int b = b0 + g;
    if (NB % TR == 0 || b < NB) {
      const int blk = b / M, k = b % M;
      C *base = buf + (blk * R * M + k) * LD + p;
      C a[R];
#pragma unroll
      for (int j = 0; j < R; ++j) a[j] = base[j * M * LD];
      if (M > 1) {
#pragma unroll
        for (int j = 1; j < R; ++j) a[j] = cmul(a[j], tw_load<DIR>(tw, j * k * TWS));
      }
      dftp<R, DIR>(a);
#pragma unroll
      for (int u = 0; u < R; ++u) base[u * M * LD] = a[u];
    }
  }
}

// One DIF stage (radix R = f.r[S], block length Lb = R*M).
template <int L, int PC, int LD, int S, int DIR, int NT, typename C>
__device__ __forceinline__ void ct_dif_stage(C *buf, const C *tw, int tid) {
  constexpr Fac f = factorize(L);
  constexpr int R = f.r[S];
  constexpr int M = sub_len(L, S + 1);
  constexpr int NB = L / R;
  constexpr int TR = NT / PC;
  constexpr int TWS = L / (R * M);
  const int p = tid % PC, g = tid / PC;
  if (g >= TR) return;  // NT not a multiple of PC: the remainder idles
#pragma unroll
  for (int b0 = 0; b0 < NB; b0 += TR) {
    const int b = b0 + g;
    if (NB % TR == 0 || b < NB) {
      const int blk = b / M, k = b % M;
      C *base = buf + (blk * R * M + k) * LD + p;
      C a[R];
#pragma unroll
      for (int j = 0; j < R; ++j) a[j] = base[j * M * LD];
      dftp<R, DIR>(a);
      if (M > 1) {
#pragma unroll
        for (int u = 1; u < R; ++u) a[u] = cmul(a[u], tw_load<DIR>(tw, u * k * TWS));
      }
#pragma unroll
      for (int u = 0; u < R; ++u) base[u * M * LD] = a[u];
    }
  }
}

// barrier of the thread group: the CTA (NT = kThreads) or one warp (NT = 32)
template <int NT>
__device__ __forceinline__ void group_sync() {
  if constexpr (NT == 32)
    __syncwarp();
  else
    __syncthreads();
}

template <int L, int PC, int LD, int S, int DIR, int NT, typename C>
__device__ __forceinline__ void ct_dit_from(C *buf, const C *tw, int tid) {
  if constexpr (S >= 0) {
    ct_dit_stage<L, PC, LD, S, DIR, NT>(buf, tw, tid);
    group_sync<NT>();
    ct_dit_from<L, PC, LD, S - 1, DIR, NT>(buf, tw, tid);
  }
}
template <int L, int PC, int LD, int S, int DIR, int NT, typename C>
__device__ __forceinline__ void ct_dif_from(C *buf, const C *tw, int tid) {
  constexpr Fac f = factorize(L);
  if constexpr (S < f.n) {
    ct_dif_stage<L, PC, LD, S, DIR, NT>(buf, tw, tid);
    group_sync<NT>();
    ct_dif_from<L, PC, LD, S + 1, DIR, NT>(buf, tw, tid);
  }
}

// Forward (DIT) transform of all PC columns; rows must be digit-reversed.
// Ends with __syncthreads.
template <int L, int PC, int LD, int DIR, typename C>
__device__ __forceinline__ void ct_fft_dit(C *buf, const C *tw) {
  constexpr Fac f = factorize(L);
  ct_dit_from<L, PC, LD, f.n - 1, DIR, kThreads>(buf, tw, threadIdx.x);
}
// Inverse-direction (DIF) transform; output rows digit-reversed.
template <int L, int PC, int LD, int DIR, typename C>
__device__ __forceinline__ void ct_fft_dif(C *buf, const C *tw) {
  ct_dif_from<L, PC, LD, 0, DIR, kThreads>(buf, tw, threadIdx.x);
}
// The same transforms by one warp on its own tile (lane = lane index); they
// end with __syncwarp.
template <int L, int PC, int LD, int DIR, typename C>
__device__ __forceinline__ void ct_fft_dit_warp(C *buf, const C *tw, int lane) {
  constexpr Fac f = factorize(L);
  ct_dit_from<L, PC, LD, f.n - 1, DIR, 32>(buf, tw, lane);
}
template <int L, int PC, int LD, int DIR, typename C>
__device__ __forceinline__ void ct_fft_dif_warp(C *buf, const C *tw, int lane) {
  ct_dif_from<L, PC, LD, 0, DIR, 32>(buf, tw, lane);
}

}  // namespace r3d
