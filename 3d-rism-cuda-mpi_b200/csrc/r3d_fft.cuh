// r3d_fft.cuh -- shared-memory mixed-radix FFT engine for sm_100a.
//
// A CTA transforms `nseq` complex sequences of length L that sit in shared
// memory.  Element i of sequence s lives at
//     buf[(s / sdiv) * sA + (s % sdiv) * sB + i * is]
// so one routine serves row-major tiles (x pass), column tiles (y pass) and
// site-by-column tiles (z pass) without copies.
//
// Forward transforms use in-place decimation in time (input scattered to
// mixed-radix digit-reversed positions when it is loaded, output natural);
// inverse transforms use in-place decimation in frequency (input natural,
// output digit-reversed, gathered when it is stored).  Both are unnormalised.
// Radices 2, 3, 4, 5 and 8 have dedicated butterflies; any other prime factor
// goes through a generic DFT loop.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace r3d {

template <typename R> struct Cx;
template <> struct Cx<float> { using T = float2; };
template <> struct Cx<double> { using T = double2; };

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) { return {a.x + b.x, a.y + b.y}; }
template <typename C>
__device__ __forceinline__ C csub(C a, C b) { return {a.x - b.x, a.y - b.y}; }
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename C>
__device__ __forceinline__ C cconj(C a) { return {a.x, -a.y}; }
// multiply by (DIR * i)
template <int DIR, typename C>
__device__ __forceinline__ C cmuli(C a) {
  return DIR < 0 ? C{a.y, -a.x} : C{-a.y, a.x};
}

// Per-CTA plan of one transform length, tables in shared memory.
template <typename C>
struct SPlan {
  int L, nrad;
  int8_t rad[12];
  const C *tw;          // tw[e] = exp(-2 pi i e / L)
  const int16_t *perm;  // perm[I] = digit-reversed position of natural index I
};

// Fill twiddles and the digit-reversal table (all threads of the CTA).
template <typename C>
__device__ void splan_init(C *tw, int16_t *perm, int L, const int8_t *rad,
                           int nrad) {
  for (int e = threadIdx.x; e < L; e += blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)e / (double)L, &s, &c);
    tw[e].x = c;
    tw[e].y = s;
    // I = j1 + p1 j2 + p1 p2 j3 + ...  ->  P = j1 L/p1 + j2 L/(p1 p2) + ...
    int I = e, P = 0, M = L;
    for (int k = 0; k < nrad; ++k) {
      int p = rad[k];
      M /= p;
      P += (I % p) * M;
      I /= p;
    }
    perm[e] = (int16_t)P;
  }
}

template <int DIR, typename C>
__device__ __forceinline__ C twid(const C *tw, int e) {
  C w = tw[e];
  return DIR < 0 ? w : cconj(w);
}

// ------------------------------------------------------------------ DFTs
template <int DIR, typename C>
__device__ __forceinline__ void dft2(C &a0, C &a1) {
  C t = a0;
  a0 = cadd(t, a1);
  a1 = csub(t, a1);
}
template <int DIR, typename C>
__device__ __forceinline__ void dft4(C &a0, C &a1, C &a2, C &a3) {
  C s02 = cadd(a0, a2), d02 = csub(a0, a2);
  C s13 = cadd(a1, a3), d13 = cmuli<DIR>(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}
template <int DIR, typename C>
__device__ __forceinline__ void dft3(C &a0, C &a1, C &a2) {
  using R = decltype(a0.x);
  const R h = (R)0.86602540378443864676;  // sqrt(3)/2
  C s = cadd(a1, a2), d = csub(a1, a2);
  C m = {a0.x - (R)0.5 * s.x, a0.y - (R)0.5 * s.y};
  C r = cmuli<DIR>(C{h * d.x, h * d.y});
  a0 = cadd(a0, s);
  a1 = cadd(m, r);
  a2 = csub(m, r);
}
template <int DIR, typename C>
__device__ __forceinline__ void dft5(C &a0, C &a1, C &a2, C &a3, C &a4) {
  using R = decltype(a0.x);
  const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
  const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
  C p14 = cadd(a1, a4), m14 = csub(a1, a4);
  C p23 = cadd(a2, a3), m23 = csub(a2, a3);
  C b1 = {a0.x + c1 * p14.x + c2 * p23.x, a0.y + c1 * p14.y + c2 * p23.y};
  C b2 = {a0.x + c2 * p14.x + c1 * p23.x, a0.y + c2 * p14.y + c1 * p23.y};
  C r1 = cmuli<DIR>(C{s1 * m14.x + s2 * m23.x, s1 * m14.y + s2 * m23.y});
  C r2 = cmuli<DIR>(C{s2 * m14.x - s1 * m23.x, s2 * m14.y - s1 * m23.y});
  a0 = cadd(a0, cadd(p14, p23));
  a1 = cadd(b1, r1);
  a4 = csub(b1, r1);
  a2 = cadd(b2, r2);
  a3 = csub(b2, r2);
}
template <int DIR, typename C>
__device__ __forceinline__ void dft8(C *a) {
  using R = decltype(a[0].x);
  const R q = (R)0.70710678118654752440;
  dft4<DIR>(a[0], a[2], a[4], a[6]);
  dft4<DIR>(a[1], a[3], a[5], a[7]);
  // W8^1 = q (1 + DIR i), W8^2 = DIR i, W8^3 = q (-1 + DIR i)
  C o1 = a[3], o2 = a[5], o3 = a[7];
  C w1o = cadd(C{q * o1.x, q * o1.y}, cmuli<DIR>(C{q * o1.x, q * o1.y}));
  C w2o = cmuli<DIR>(o2);
  C w3o = csub(cmuli<DIR>(C{q * o3.x, q * o3.y}), C{q * o3.x, q * o3.y});
  C e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6], o0 = a[1];
  a[0] = cadd(e0, o0);
  a[4] = csub(e0, o0);
  a[1] = cadd(e1, w1o);
  a[5] = csub(e1, w1o);
  a[2] = cadd(e2, w2o);
  a[6] = csub(e2, w2o);
  a[3] = cadd(e3, w3o);
  a[7] = csub(e3, w3o);
}

template <int P, int DIR, typename C>
__device__ __forceinline__ void dftp(C *a) {
  if constexpr (P == 2) dft2<DIR>(a[0], a[1]);
  if constexpr (P == 3) dft3<DIR>(a[0], a[1], a[2]);
  if constexpr (P == 4) dft4<DIR>(a[0], a[1], a[2], a[3]);
  if constexpr (P == 5) dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
  if constexpr (P == 8) dft8<DIR>(a);
}

// ------------------------------------------------------------- stages
// DIT stage: radix P, sub-length m; butterflies (blk, k) over all sequences.
template <int P, int DIR, typename C>
__device__ void stage_dit(C *buf, int nseq, int sdiv, int sA, int sB, int is,
                          int L, int m, const C *tw) {
  const int pm = P * m, nb = L / P, tws = L / pm;
  const int total = nseq * nb;
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    int sq = w / nb, b = w - sq * nb;
    int blk = b / m, k = b - blk * m;
    C *base = buf + (sq / sdiv) * sA + (sq % sdiv) * sB + (blk * pm + k) * is;
    C a[P];
#pragma unroll
    for (int j = 0; j < P; ++j) a[j] = base[j * m * is];
    if (m > 1) {
#pragma unroll
      for (int j = 1; j < P; ++j) a[j] = cmul(a[j], twid<DIR>(tw, j * k * tws));
    }
    dftp<P, DIR>(a);
#pragma unroll
    for (int u = 0; u < P; ++u) base[u * m * is] = a[u];
  }
}

// DIF stage: radix P, block length P*m.
template <int P, int DIR, typename C>
__device__ void stage_dif(C *buf, int nseq, int sdiv, int sA, int sB, int is,
                          int L, int m, const C *tw) {
  const int pm = P * m, nb = L / P, tws = L / pm;
  const int total = nseq * nb;
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    int sq = w / nb, b = w - sq * nb;
    int blk = b / m, k = b - blk * m;
    C *base = buf + (sq / sdiv) * sA + (sq % sdiv) * sB + (blk * pm + k) * is;
    C a[P];
#pragma unroll
    for (int j = 0; j < P; ++j) a[j] = base[j * m * is];
    dftp<P, DIR>(a);
    if (m > 1) {
#pragma unroll
      for (int u = 1; u < P; ++u) a[u] = cmul(a[u], twid<DIR>(tw, u * k * tws));
    }
#pragma unroll
    for (int u = 0; u < P; ++u) base[u * m * is] = a[u];
  }
}

// Generic prime radix (direct DFT through the twiddle table).
template <int DIR, typename C, bool DIT>
__device__ void stage_gen(C *buf, int nseq, int sdiv, int sA, int sB, int is,
                          int L, int p, int m, const C *tw) {
  const int pm = p * m, nb = L / p, tws = L / pm, wp = L / p;
  const int total = nseq * nb;
  for (int w = threadIdx.x; w < total; w += blockDim.x) {
    int sq = w / nb, b = w - sq * nb;
    int blk = b / m, k = b - blk * m;
    C *base = buf + (sq / sdiv) * sA + (sq % sdiv) * sB + (blk * pm + k) * is;
    C a[16], o[16];
    for (int j = 0; j < p; ++j) {
      a[j] = base[j * m * is];
      if (DIT && j) a[j] = cmul(a[j], twid<DIR>(tw, j * k * tws));
    }
    for (int u = 0; u < p; ++u) {
      C acc = a[0];
      for (int j = 1; j < p; ++j)
        acc = cadd(acc, cmul(a[j], twid<DIR>(tw, ((j * u) % p) * wp)));
      o[u] = acc;
    }
    for (int u = 0; u < p; ++u) {
      C v = o[u];
      if (!DIT && u) v = cmul(v, twid<DIR>(tw, u * k * tws));
      base[u * m * is] = v;
    }
  }
}

// Forward (DIT) transform; input must be in digit-reversed order.
template <int DIR, typename C>
__device__ void fft_dit(C *buf, int nseq, int sdiv, int sA, int sB, int is,
                        const SPlan<C> &pl) {
  int m = 1;
  for (int s = pl.nrad - 1; s >= 0; --s) {
    int p = pl.rad[s];
    switch (p) {
      case 2: stage_dit<2, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 3: stage_dit<3, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 4: stage_dit<4, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 5: stage_dit<5, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 8: stage_dit<8, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      default:
        stage_gen<DIR, C, true>(buf, nseq, sdiv, sA, sB, is, pl.L, p, m, pl.tw);
    }
    __syncthreads();
    m *= p;
  }
}

// Inverse-direction (DIF) transform; output left in digit-reversed order.
template <int DIR, typename C>
__device__ void fft_dif(C *buf, int nseq, int sdiv, int sA, int sB, int is,
                        const SPlan<C> &pl) {
  int Lb = pl.L;
  for (int s = 0; s < pl.nrad; ++s) {
    int p = pl.rad[s];
    int m = Lb / p;
    switch (p) {
      case 2: stage_dif<2, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 3: stage_dif<3, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 4: stage_dif<4, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 5: stage_dif<5, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      case 8: stage_dif<8, DIR>(buf, nseq, sdiv, sA, sB, is, pl.L, m, pl.tw); break;
      default:
        stage_gen<DIR, C, false>(buf, nseq, sdiv, sA, sB, is, pl.L, p, m, pl.tw);
    }
    __syncthreads();
    Lb = m;
  }
}

}  // namespace r3d
