// r3d_passes_sr.cu -- the iteration's y and z passes on the register-pass
// Stockham engine (r3d_fft_sr.cuh).  Compiled once per precision
// (R3D_CT_FP64 as r3d_passes_ct.cu).
//
// The tile-per-CTA and copy-engine y/z passes (r3d_passes_ct.cu,
// r3d_passes_tma.cu) run the in-place radix-8/4 engine: three shared-memory
// round trips per 256-point transform plus a global twiddle load per stage.
// Measured on B200 that made the z pass (forward z, OZ, inverse z over all
// sites) bound by shared-memory and L1 traffic, not by DRAM.  Here:
//   FY / IY   pass 0 reads the spectrum straight from global memory into
//             registers, the last pass writes it straight back: one
//             shared-memory round trip per transform (two for 512).
//   ZOZ       the forward z transform's last pass leaves every site's values
//             of the same k_z in one thread's registers; the OZ product
//             h_a(k) = sum_b chi_ab(|k|) c_b(k) (calculate_cuda.cu:39-52) and
//             the inverse transform's first pass run there, so the z pass
//             makes two shared-memory round trips in all.
// The spectrum stays in natural k_y order (the transform sorts itself), so
// these kernels pair with each other only.  Twiddles come from a per-CTA
// shared-memory copy of the length's table.
#include "r3d_async.cuh"
#include "r3d_common.cuh"
#include "r3d_fft_sr.cuh"

#ifndef R3D_CT_FP64
#define R3D_CT_FP64 1
#endif

namespace r3d {

#if R3D_CT_FP64
using PSR = P64;
#else
using PSR = PMix;
#endif

// --------------------------------------------------------------- y pass
// tile = PC x-columns of one (site, z) plane; shared memory [L = ny][PC] plus
// the twiddle table.  Forward (DIR -1): y half-sample twiddle on load.
// Inverse (+1): the reversed plan, conjugate half-sample twiddle on store.
template <typename P, int L, int PC, int DIR>
__global__ void __launch_bounds__(kThreads, 3) k_fy_sr(Batch b) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr SrPlan pl = sr_plan(L);
  constexpr bool INV = DIR > 0;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;
  C *tw = buf + L * PC;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, ptiles = hx / PC;
  const int pt = tile % ptiles;
  tile /= ptiles;
  const int z = tile % d.nz, v = tile / d.nz;
  const C *pw = (const C *)d.pwy;
  const long long wb = (long long)v * d.Nhs + (long long)z * L * hx + pt * PC, wn = d.n * d.Nhs;
  C *w = (C *)d.w + wb;
  for (int e = threadIdx.x; e < L; e += kThreads) tw[e] = ((const C *)d.twy)[e];

  // pass 0: global -> registers -> shared
  {
    constexpr int R = sr_radix(L, 0, INV), NS = 1, T = PC * (L / R);
    for (int task = threadIdx.x; task < T; task += kThreads) {
      const int p = task % PC, j = task / PC;
      C a[R];
      const C pj = pw[j];  // y = j + m L / R
      // all R loads issued before any of them is used (more loads in flight),
      // then the forward transform's half-sample twiddles
#pragma unroll
      for (int m = 0; m < R; ++m) {
        const int y = sr_in<L, R>(j, m);
        a[m] = R3D_IN(d, wb + (long long)y * hx + p, wn) ? w[(long long)y * hx + p] : C{0, 0};
      }
      if (!INV) {
#pragma unroll
        for (int m = 0; m < R; ++m) a[m] = cmul(a[m], sr_half_twiddle<R>(pj, m));
      }
      if constexpr (pl.n == 1) {
        sr_pass<L, R, NS, DIR>(a, tw, j);
#pragma unroll
        for (int m = 0; m < R; ++m) {
          const int y = sr_out<R, NS>(j, m);
          if (R3D_IN(d, wb + (long long)y * hx + p, wn))  // one pass: y = m
            w[(long long)y * hx + p] = INV ? cmul(a[m], cconj(sr_half_twiddle<R>(pj, m))) : a[m];
        }
      } else {
        sr_pass<L, R, NS, DIR>(a, tw, j);
#pragma unroll
        for (int m = 0; m < R; ++m) buf[sr_out<R, NS>(j, m) * PC + p] = a[m];
      }
    }
  }
  if constexpr (pl.n == 1) return;
  __syncthreads();  // also publishes tw
  // middle pass (512 = 8 x 8 x 8): shared -> registers, barrier, -> shared
  if constexpr (pl.n == 3) {
    constexpr int R = sr_radix(L, 1, INV), NS = sr_ns(L, 1, INV), T = PC * (L / R);
    constexpr int K = (T + kThreads - 1) / kThreads;
    C a[K][R];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = threadIdx.x + k * kThreads;
      if (T % kThreads == 0 || task < T) {
        const int p = task % PC, j = task / PC;
#pragma unroll
        for (int m = 0; m < R; ++m) a[k][m] = buf[sr_in<L, R>(j, m) * PC + p];
        sr_pass<L, R, NS, DIR>(a[k], tw, j);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = threadIdx.x + k * kThreads;
      if (T % kThreads == 0 || task < T) {
        const int p = task % PC, j = task / PC;
#pragma unroll
        for (int m = 0; m < R; ++m) buf[sr_out<R, NS>(j, m) * PC + p] = a[k][m];
      }
    }
    __syncthreads();
  }
  // last pass: shared -> registers -> global (natural k_y / y order)
  {
    constexpr int s = pl.n - 1;
    constexpr int R = sr_radix(L, s, INV), NS = sr_ns(L, s, INV), T = PC * (L / R);
    for (int task = threadIdx.x; task < T; task += kThreads) {
      const int p = task % PC, j = task / PC;
      C a[R];
#pragma unroll
      for (int m = 0; m < R; ++m) a[m] = buf[sr_in<L, R>(j, m) * PC + p];
      sr_pass<L, R, NS, DIR>(a, tw, j);
      static_assert(!INV || NS * R == L, "the inverse's last pass writes y = j + m L / R");
      const C pj = INV ? pw[j] : C{0, 0};
#pragma unroll
      for (int m = 0; m < R; ++m) {
        const int y = sr_out<R, NS>(j, m);
        if (R3D_IN(d, wb + (long long)y * hx + p, wn))
          w[(long long)y * hx + p] = INV ? cmul(a[m], cconj(sr_half_twiddle<R>(pj, m))) : a[m];
      }
    }
  }
}

// --------------------------------------------------------------- x passes
// Rows of nx = 2L reals of one site, packed as the L-point complex sequence
// z_m = (f_m - i f_{m+L}) e^{-i pi m / nx} (the odd-frequency real-to-complex
// packing of r3d_passes_ct.cu), transformed by the Stockham engine.  A tile
// is PC consecutive rows (row = y + ny z); shared memory holds the rows with
// one complex of padding per 16 (index p + p/16), which keeps the
// transposing accesses of the passes free of bank conflicts.
template <int L>
__device__ __forceinline__ constexpr int sr_xrow() {
  return L + L / 16 + 1;
}
template <int L>
__device__ __forceinline__ constexpr int sr_xi(int p) {
  return p + p / 16;
}

// The iteration's FX on the Stockham engine: closure (KH/HNC/PSE-n) and
// c_s = g - 1 - t_s (- c_ref) per voxel (trm1mt, calculate_cuda.cu:18-24),
// the g it evaluated stored for IX, the checkerboard sign, packing and the
// forward x transform; the first pass computes its inputs straight from
// global memory, the last writes the half spectrum w[site][z][y][p].
template <typename P, int L, int PC>
__global__ void __launch_bounds__(kThreads) k_fx_sr(Batch b) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  constexpr SrPlan pl = sr_plan(L);
  constexpr int LR = sr_xrow<L>(), NX = 2 * L;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;  // [PC][LR]
  C *tw = buf + PC * LR;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int tile = blockIdx.x - b.prefix[si];
  const int tps = (d.ny * d.nz) / PC;  // tiles per site
  const int v = tile / tps;
  const long long row0 = (long long)(tile % tps) * PC;
  const int ny = d.ny;
  for (int e = threadIdx.x; e < L; e += kThreads) tw[e] = ((const C *)d.twx)[e];
  const C *pw = (const C *)d.pwx;
  const long long base0 = (long long)v * d.Ns + row0 * NX;
  const T *t = (const T *)d.t + base0;
  const R *u = (const R *)d.u + base0;
  const R *cref = d.cref ? (const R *)d.cref + base0 : nullptr;
  T *gq = (T *)d.gq + base0;
  C *w = (C *)d.w + (long long)v * d.Nhs + row0 * L;
  // pass 0: closure and packing straight from global memory
  {
    constexpr int R0 = pl.r[0], J = L / R0, TT = PC * J;
    for (int task = threadIdx.x; task < TT; task += kThreads) {
      const int j = task % J, r = task / J;
      const long long row = row0 + r;
      const int par = (int)((row % ny + row / ny) & 1);
      const long long rb = (long long)r * NX;
      C a[R0];
#pragma unroll
      for (int q = 0; q < R0; ++q) {
        const int m = sr_in<L, R0>(j, q);
        if (!R3D_IN(d, base0 + rb + m + L, d.n * d.Ns)) {
          a[q] = C{0, 0};
          continue;
        }
        const double t0 = t[rb + m], t1 = t[rb + m + L];
        const double g0 = closure_g<double>(d.clos, d.pse_n, -(double)u[rb + m] + t0);
        const double g1 = closure_g<double>(d.clos, d.pse_n, -(double)u[rb + m + L] + t1);
        gq[rb + m] = (T)g0;
        gq[rb + m + L] = (T)g1;
        double c0 = g0 - 1.0 - t0, c1 = g1 - 1.0 - t1;
        if (cref) {
          c0 -= (double)cref[rb + m];
          c1 -= (double)cref[rb + m + L];
        }
        R f0 = (R)c0, f1 = (R)c1;
        if ((m + par) & 1) f0 = -f0;
        if ((m + L + par) & 1) f1 = -f1;
        a[q] = cmul(C{f0, -f1}, pw[m]);
      }
      sr_pass<L, R0, 1, -1>(a, tw, j);
      if constexpr (pl.n == 1) {
#pragma unroll
        for (int q = 0; q < R0; ++q) w[(long long)r * L + sr_out<R0, 1>(j, q)] = a[q];
      } else {
#pragma unroll
        for (int q = 0; q < R0; ++q) buf[r * LR + sr_xi<L>(sr_out<R0, 1>(j, q))] = a[q];
      }
    }
  }
  if constexpr (pl.n == 1) return;
  __syncthreads();
  if constexpr (pl.n == 3) {  // middle pass, in place
    constexpr int R1 = pl.r[1], NS1 = sr_ns(L, 1, false), J = L / R1, TT = PC * J;
    constexpr int K = (TT + kThreads - 1) / kThreads;
    C a[K][R1];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = threadIdx.x + k * kThreads;
      if (TT % kThreads == 0 || task < TT) {
        const int j = task % J, r = task / J;
#pragma unroll
        for (int q = 0; q < R1; ++q) a[k][q] = buf[r * LR + sr_xi<L>(sr_in<L, R1>(j, q))];
        sr_pass<L, R1, NS1, -1>(a[k], tw, j);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int task = threadIdx.x + k * kThreads;
      if (TT % kThreads == 0 || task < TT) {
        const int j = task % J, r = task / J;
#pragma unroll
        for (int q = 0; q < R1; ++q) buf[r * LR + sr_xi<L>(sr_out<R1, NS1>(j, q))] = a[k][q];
      }
    }
    __syncthreads();
  }
  {  // last pass -> the half spectrum (natural p order)
    constexpr int s = pl.n - 1;
    constexpr int RS = pl.r[s], NSs = sr_ns(L, s, false), J = L / RS, TT = PC * J;
    for (int task = threadIdx.x; task < TT; task += kThreads) {
      const int j = task % J, r = task / J;
      C a[RS];
#pragma unroll
      for (int q = 0; q < RS; ++q) a[q] = buf[r * LR + sr_xi<L>(sr_in<L, RS>(j, q))];
      sr_pass<L, RS, NSs, -1>(a, tw, j);
#pragma unroll
      for (int q = 0; q < RS; ++q) w[(long long)r * L + sr_out<RS, NSs>(j, q)] = a[q];
    }
  }
}

// The iteration's IX on the Stockham engine: inverse x transform (reversed
// plan) of `per` consecutive tiles, unpacking, R = h + 1 - g with the g FX
// left (calculate_cuda.cu:54-60), sum R^2 (cal_rms.cu:14-26) and, past AN2's
// Picard warm-up, the five theta dots per site (anderson_cuda.cu:25-67) into
// this CTA's row of partials (per site, in tile order: deterministic).
template <typename P, int L, int PC>
__global__ void __launch_bounds__(kThreads) k_ix_sr(Batch b, int per) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  constexpr SrPlan pl = sr_plan(L);
  constexpr int LR = sr_xrow<L>(), NX = 2 * L;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;  // [PC][LR]
  C *tw = buf + PC * LR;
  __shared__ double red6[6 * (kThreads / 32)];
  __shared__ double sums[kPartials];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int ny = d.ny;
  const int tps = (d.ny * d.nz) / PC;
  const int ntile = d.n * tps;
  const bool dots = d.mixer == MIX_AN2 && d.ctl->count_left <= 0;
  for (int e = threadIdx.x; e < L; e += kThreads) tw[e] = ((const C *)d.twx)[e];
  for (int k = threadIdx.x; k < kPartials; k += kThreads) sums[k] = 0;
  const C *pw = (const C *)d.pwx;
  const long long niv = (long long)d.n * d.Ns;
  double a_ss = 0, a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0;
  int cur_v = -1;
  auto flush = [&]() {
    if (cur_v < 0) return;
    double q[6] = {a_ss, a0, a1, a2, a3, a4};
    block_sums<6>(q, red6);
    if (threadIdx.x == 0) {
      sums[0] += q[0];
      if (dots)
        for (int k = 0; k < 5; ++k) sums[1 + 5 * cur_v + k] += q[1 + k];
    }
    a_ss = a0 = a1 = a2 = a3 = a4 = 0;
  };
  for (int it = 0; it < per; ++it) {
    const int tile = cta * per + it;
    if (tile >= ntile) break;
    const int v = tile / tps;
    const long long row0 = (long long)(tile % tps) * PC;
    if (v != cur_v) {  // uniform over the CTA
      flush();
      cur_v = v;
    }
    const C *w = (const C *)d.w + (long long)v * d.Nhs + row0 * L;
    __syncthreads();  // buf of the previous tile fully read
    {  // pass 0 (radix R_{P-1}): global -> registers -> shared
      constexpr int R0 = sr_radix(L, 0, true), J = L / R0, TT = PC * J;
      for (int task = threadIdx.x; task < TT; task += kThreads) {
        const int j = task % J, r = task / J;
        C a[R0];
#pragma unroll
        for (int q = 0; q < R0; ++q) a[q] = w[(long long)r * L + sr_in<L, R0>(j, q)];
        sr_pass<L, R0, 1, 1>(a, tw, j);
#pragma unroll
        for (int q = 0; q < R0; ++q) buf[r * LR + sr_xi<L>(sr_out<R0, 1>(j, q))] = a[q];
      }
    }
    __syncthreads();
    if constexpr (pl.n == 3) {
      constexpr int R1 = sr_radix(L, 1, true), NS1 = sr_ns(L, 1, true), J = L / R1,
                    TT = PC * J, K = (TT + kThreads - 1) / kThreads;
      C a[K][R1];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int task = threadIdx.x + k * kThreads;
        if (TT % kThreads == 0 || task < TT) {
          const int j = task % J, r = task / J;
#pragma unroll
          for (int q = 0; q < R1; ++q) a[k][q] = buf[r * LR + sr_xi<L>(sr_in<L, R1>(j, q))];
          sr_pass<L, R1, NS1, 1>(a[k], tw, j);
        }
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int task = threadIdx.x + k * kThreads;
        if (TT % kThreads == 0 || task < TT) {
          const int j = task % J, r = task / J;
#pragma unroll
          for (int q = 0; q < R1; ++q) buf[r * LR + sr_xi<L>(sr_out<R1, NS1>(j, q))] = a[k][q];
        }
      }
      __syncthreads();
    }
    {  // last pass, unpacking and the residual
      constexpr int s = pl.n - 1;
      constexpr int RS = sr_radix(L, s, true), NSs = sr_ns(L, s, true), J = L / RS,
                    TT = PC * J;
      for (int task = threadIdx.x; task < TT; task += kThreads) {
        const int j = task % J, r = task / J;
        const long long row = row0 + r;
        const int par = (int)((row % ny + row / ny) & 1);
        const long long gb = (long long)v * d.Ns + row * NX;
        const T *gq = (const T *)d.gq + gb;
        const R *lr = (const R *)d.lr + gb, *p0 = (const R *)d.hist_b + gb,
                *q0 = (const R *)d.hist_b + niv + gb;
        R *res = (R *)d.res + gb;
        C a[RS];
        if constexpr (pl.n == 1) {
#pragma unroll
          for (int q = 0; q < RS; ++q) a[q] = w[(long long)r * L + sr_in<L, RS>(j, q)];
        } else {
#pragma unroll
          for (int q = 0; q < RS; ++q) a[q] = buf[r * LR + sr_xi<L>(sr_in<L, RS>(j, q))];
        }
        sr_pass<L, RS, NSs, 1>(a, tw, j);
#pragma unroll
        for (int q = 0; q < RS; ++q) {
          const int m = sr_out<RS, NSs>(j, q);
          if (!R3D_IN(d, gb + m + L, niv)) continue;
          const C zc = cmul(a[q], cconj(pw[m]));
          R h0 = zc.x, h1 = -zc.y;
          if ((m + par) & 1) h0 = -h0;
          if ((m + L + par) & 1) h1 = -h1;
          const double g0 = gq[m], g1 = gq[m + L];
          const R r0 = (R)((double)h0 + (double)lr[m] - g0);
          const R r1 = (R)((double)h1 + (double)lr[m + L] - g1);
          res[m] = r0;
          res[m + L] = r1;
          a_ss += (double)r0 * r0 + (double)r1 * r1;
          if (dots) {
            const double t10 = (double)r0 - p0[m], t20 = (double)r0 - q0[m];
            const double t11 = (double)r1 - p0[m + L], t21 = (double)r1 - q0[m + L];
            a0 += r0 * t10 + r1 * t11;
            a1 += r0 * t20 + r1 * t21;
            a2 += t10 * t10 + t11 * t11;
            a3 += t10 * t20 + t11 * t21;
            a4 += t20 * t20 + t21 * t21;
          }
        }
      }
    }
  }
  flush();
  __syncthreads();
  double *part = d.partials + (size_t)cta * kPartials;
  for (int k = threadIdx.x; k < kPartials; k += kThreads) part[k] = sums[k];
}

// --------------------------------------------------------------- z pass
// Position of (site v, z, column p) in the z pass's shared tile: rows of PC
// columns with one spare row after every 16, so that rows 16 apart (the
// stride of a radix-16 pass's writes) fall on other banks.
template <int L>
__device__ __forceinline__ constexpr int sr_zrows() {
  return L + L / 16 + 1;
}
template <int L, int PC>
__device__ __forceinline__ int sr_zi(int v, int z, int p) {
  return (v * sr_zrows<L>() + z + z / 16) * PC + p;
}

// One Stockham pass in place on the shared-memory tile [site][L][PC] of NS
// sites: every thread reads and transforms all of its tasks, then (after a
// barrier, since a pass writes other positions than it reads) writes them.
template <int L, int R, int NSs, int DIR, int NS, int PC, int NT, typename C>
__device__ __forceinline__ void sr_tile_pass(C *buf, const C *tw) {
  constexpr int T = NS * PC * (L / R), K = (T + NT - 1) / NT;
  C a[K][R];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = threadIdx.x + k * NT;
    if (T % NT == 0 || task < T) {
      const int p = task % PC, q = task / PC, j = q % (L / R), v = q / (L / R);
#pragma unroll
      for (int m = 0; m < R; ++m) a[k][m] = buf[sr_zi<L, PC>(v, sr_in<L, R>(j, m), p)];
      sr_pass<L, R, NSs, DIR>(a[k], tw, j);
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const int task = threadIdx.x + k * NT;
    if (T % NT == 0 || task < T) {
      const int p = task % PC, q = task / PC, j = q % (L / R), v = q / (L / R);
#pragma unroll
      for (int m = 0; m < R; ++m) buf[sr_zi<L, PC>(v, sr_out<R, NSs>(j, m), p)] = a[k][m];
    }
  }
  __syncthreads();
}

// OZ at one k point: c[0..NS) -> h_a = sum_b chi_ab(|k|) c_b, with the chi
// row of the point's |k| shell (cubic cells: shell (ax^2 + ay^2 + az^2 - 3)
// / 8 over the odd integers a = 2j - n + 1, k_x index 2p; else the table)
template <typename R>
__device__ __forceinline__ const R *sr_chi_row(const Desc &d, long long ax, long long ay, int kz,
                                               long long gi) {
  size_t shell;
  if (d.cubic) {
    const long long az = 2 * kz - d.nz + 1;
    shell = (size_t)((ax * ax + ay * ay + az * az - 3) / 8);
  } else {
    shell = d.kidx[gi];
  }
  return (const R *)d.chi + shell * d.chis;
}
template <typename R, int NS, typename C>
__device__ __forceinline__ void sr_oz_apply(C *c, const R *ch) {
  R x[NS * NS];
  if constexpr ((NS * NS) % 4 == 0 && sizeof(R) == 4) {
#pragma unroll
    for (int q = 0; q < NS * NS / 4; ++q) {
      const float4 v4 = reinterpret_cast<const float4 *>(ch)[q];
      x[4 * q] = v4.x;
      x[4 * q + 1] = v4.y;
      x[4 * q + 2] = v4.z;
      x[4 * q + 3] = v4.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < NS * NS; ++q) x[q] = ch[q];
  }
  C in[NS];
#pragma unroll
  for (int v = 0; v < NS; ++v) in[v] = c[v];
#pragma unroll
  for (int v = 0; v < NS; ++v) {
    R hr = 0, hi = 0;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      hr += in[q].x * x[v * NS + q];
      hi += in[q].y * x[v * NS + q];
    }
    c[v] = C{hr, hi};
  }
}

// the same chi row applied to two k points
template <typename R, int NS, typename C>
__device__ __forceinline__ void sr_oz_apply2(C *c1, C *c2, const R *ch) {
  R x[NS * NS];
  if constexpr ((NS * NS) % 4 == 0 && sizeof(R) == 4) {
#pragma unroll
    for (int q = 0; q < NS * NS / 4; ++q) {
      const float4 v4 = reinterpret_cast<const float4 *>(ch)[q];
      x[4 * q] = v4.x;
      x[4 * q + 1] = v4.y;
      x[4 * q + 2] = v4.z;
      x[4 * q + 3] = v4.w;
    }
  } else {
#pragma unroll
    for (int q = 0; q < NS * NS; ++q) x[q] = ch[q];
  }
  C i1[NS], i2[NS];
#pragma unroll
  for (int v = 0; v < NS; ++v) {
    i1[v] = c1[v];
    i2[v] = c2[v];
  }
#pragma unroll
  for (int v = 0; v < NS; ++v) {
    R h1r = 0, h1i = 0, h2r = 0, h2i = 0;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      const R xq = x[v * NS + q];
      h1r += i1[q].x * xq;
      h1i += i1[q].y * xq;
      h2r += i2[q].x * xq;
      h2i += i2[q].y * xq;
    }
    c1[v] = C{h1r, h1i};
    c2[v] = C{h2r, h2i};
  }
}

template <typename R, int NS, typename C>
__device__ __forceinline__ void sr_oz_point(C *c, const Desc &d, long long ax, long long ay,
                                            int kz, long long gi) {
  sr_oz_apply<R, NS>(c, sr_chi_row<R>(d, ax, ay, kz, gi));
}

// The z pass on a tile of PC x-columns at one k_y, all NS sites, all z;
// shared memory [site][L = nz][PC] plus the twiddle table.  Forward z
// transform (half-sample twiddle on load), OZ, inverse z transform
// (conjugate half-sample twiddle on store).  OZREG: the forward transform's
// last pass, the OZ and the inverse transform's first pass run on registers
// holding every site of a task (one shared-memory round trip less, NS *
// R_last complex values per thread); else the OZ is a pass of its own over
// the shared tile.  Two kernels run it: one tile per CTA (k_zoz_sr), and one
// persistent CTA per SM that streams its next tile in while it transforms
// the current one (k_zoz_srp).

// From the forward transform's second pass (its first has filled the tile)
// through the inverse transform's second-to-last pass, on the shared tile.
template <typename P, int L, int PC, int NS, int NT, bool OZREG>
__device__ __forceinline__ void sr_zoz_middle(typename Cx<typename P::R>::T *buf,
                                              const typename Cx<typename P::R>::T *tw,
                                              const Desc &d, int pt, long long ay,
                                              long long gbase, long long zs) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr SrPlan pl = sr_plan(L);
  constexpr int RL = pl.r[pl.n - 1];  // forward last radix = inverse first
  constexpr int NSL = L / RL;         // N of the forward last pass
  (void)NSL;
  (void)RL;
  auto at = [&](int v, int z, int p) -> C & { return buf[sr_zi<L, PC>(v, z, p)]; };
  if constexpr (pl.n == 3) sr_tile_pass<L, pl.r[1], sr_ns(L, 1, false), -1, NS, PC, NT>(buf, tw);
  if constexpr (OZREG && pl.n > 1) {
    // forward last pass -> OZ -> inverse first pass, every site of a task in
    // registers; written back after a barrier (the passes are in place)
    constexpr int TO = PC * NSL, KO = (TO + NT - 1) / NT;
    C a[KO][NS][RL];
#pragma unroll
    for (int k = 0; k < KO; ++k) {
      const int task = threadIdx.x + k * NT;
      if (TO % NT == 0 || task < TO) {
        const int p = task % PC, j = task / PC;
#pragma unroll
        for (int v = 0; v < NS; ++v) {
#pragma unroll
          for (int m = 0; m < RL; ++m) a[k][v][m] = at(v, sr_in<L, RL>(j, m), p);
          sr_pass<L, RL, NSL, -1>(a[k][v], tw, j);
        }
        const long long ax = 4 * (pt * PC + p) - d.nx + 1;
#pragma unroll
        for (int m = 0; m < RL; ++m) {  // element m is k_z = j + m NSL
          const int kz = j + m * NSL;
          C c[NS];
#pragma unroll
          for (int v = 0; v < NS; ++v) c[v] = a[k][v][m];
          sr_oz_point<R, NS>(c, d, ax, ay, kz, kz * zs + gbase + p);
#pragma unroll
          for (int v = 0; v < NS; ++v) a[k][v][m] = c[v];
        }
#pragma unroll
        for (int v = 0; v < NS; ++v) sr_pass<L, RL, 1, 1>(a[k][v], tw, j);
      }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KO; ++k) {
      const int task = threadIdx.x + k * NT;
      if (TO % NT == 0 || task < TO) {
        const int p = task % PC, j = task / PC;
#pragma unroll
        for (int v = 0; v < NS; ++v)
#pragma unroll
          for (int m = 0; m < RL; ++m) at(v, sr_out<RL, 1>(j, m), p) = a[k][v][m];
      }
    }
    __syncthreads();
  } else {
    if constexpr (pl.n > 1) sr_tile_pass<L, RL, NSL, -1, NS, PC, NT>(buf, tw);
    {  // OZ, in place.  k_z and L - 1 - k_z (the same |k| shell) form a pair;
       // NS lanes of a warp take one pair, lane q the output site q: it reads
       // row q of the shell's chi matrix (the group reads the whole row
       // block at once, a gather from L2 in NS * NS * 4 contiguous bytes),
       // every site's input (shared-memory broadcast within the group) and
       // writes its site's outputs after the group has read.
      constexpr int G = 32 / NS, TP = PC * (L / 2), NW = NT / 32;
      // pairs a group takes, and how many of their chi rows are in flight
      // at once (the rows come from L2: issued together, their latency is
      // paid once per U pairs)
      constexpr int IT = (TP + NW * G - 1) / (NW * G), U = IT < 4 ? IT : 4;
      const int lane = threadIdx.x & 31, q = lane % NS, grp = lane / NS;
      const bool lane_on = grp < G;
      const int first = (threadIdx.x >> 5) * G + grp;
#pragma unroll 1
      for (int i0 = 0; i0 < IT; i0 += U) {
        R x[U][NS];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int pair = first + (i0 + u) * NW * G;
          if (lane_on && i0 + u < IT && pair < TP) {
            const int p = pair % PC, kz = pair / PC;
            const R *ch = sr_chi_row<R>(d, 4 * (pt * PC + p) - d.nx + 1, ay, kz,
                                        (long long)kz * zs + gbase + p) + q * NS;
            if constexpr (NS == 4 && sizeof(R) == 4) {
              const float4 v4 = *reinterpret_cast<const float4 *>(ch);
              x[u][0] = v4.x, x[u][1] = v4.y, x[u][2] = v4.z, x[u][3] = v4.w;
            } else if constexpr (NS == 2 && sizeof(R) == 4) {
              const float2 v2 = *reinterpret_cast<const float2 *>(ch);
              x[u][0] = v2.x, x[u][1] = v2.y;
            } else {
#pragma unroll
              for (int b = 0; b < NS; ++b) x[u][b] = ch[b];
            }
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int pair = first + (i0 + u) * NW * G;
          const bool on = lane_on && i0 + u < IT && pair < TP;
          const int p = pair % PC, kz = pair / PC, kz2 = L - 1 - kz;
          C c1[NS], c2[NS];
          if (on) {
#pragma unroll
            for (int b = 0; b < NS; ++b) {
              c1[b] = at(b, kz, p);
              c2[b] = at(b, kz2, p);
            }
          }
          __syncwarp();
          if (on) {
            R h1r = 0, h1i = 0, h2r = 0, h2i = 0;
#pragma unroll
            for (int b = 0; b < NS; ++b) {
              h1r += c1[b].x * x[u][b];
              h1i += c1[b].y * x[u][b];
              h2r += c2[b].x * x[u][b];
              h2i += c2[b].y * x[u][b];
            }
            at(q, kz, p) = C{h1r, h1i};
            at(q, kz2, p) = C{h2r, h2i};
          }
          __syncwarp();
        }
      }
    }
    __syncthreads();
    if constexpr (pl.n > 1) sr_tile_pass<L, RL, 1, 1, NS, PC, NT>(buf, tw);
  }
  if constexpr (pl.n == 3) sr_tile_pass<L, sr_radix(L, 1, true), sr_ns(L, 1, true), 1, NS, PC, NT>(buf, tw);
}

// The inverse transform's last pass: shared tile -> registers -> global
// (w = the tile's first column of site 0, wb its offset in the spectrum).
template <typename P, int L, int PC, int NS, int NT>
__device__ __forceinline__ void sr_zoz_last(const typename Cx<typename P::R>::T *buf,
                                            const typename Cx<typename P::R>::T *tw,
                                            const Desc &d, typename Cx<typename P::R>::T *w,
                                            const typename Cx<typename P::R>::T *pw,
                                            long long wb, long long wn, long long zs) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr SrPlan pl = sr_plan(L);
  auto at = [&](int v, int z, int p) -> const C & { return buf[sr_zi<L, PC>(v, z, p)]; };
  (void)wb;
  (void)wn;
  (void)d;
  {
    constexpr int s = pl.n - 1;
    constexpr int R = sr_radix(L, s, true), NSs = sr_ns(L, s, true), T = NS * PC * (L / R);
    static_assert(NSs * R == L, "the last pass writes z = j + m L / R");
    for (int task = threadIdx.x; task < T; task += NT) {
      const int p = task % PC, q = task / PC, j = q % (L / R), v = q / (L / R);
      C e[R];
#pragma unroll
      for (int m = 0; m < R; ++m) e[m] = at(v, sr_in<L, R>(j, m), p);
      sr_pass<L, R, NSs, 1>(e, tw, j);
      const C pj = pw[j];
#pragma unroll
      for (int m = 0; m < R; ++m) {
        const int z = sr_out<R, NSs>(j, m);
        const long long gi = v * d.Nhs + z * zs + p;
        if (R3D_IN(d, wb + gi, wn)) w[gi] = cmul(e[m], cconj(sr_half_twiddle<R>(pj, m)));
      }
    }
  }
}

template <typename P, int L, int PC, int NS, int NT, bool OZREG>
__global__ void __launch_bounds__(NT, (OZREG || NT > 256) ? 1 : 2) k_zoz_sr(Batch b) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr SrPlan pl = sr_plan(L);
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;  // [site][z (padded)][p]
  C *tw = buf + NS * sr_zrows<L>() * PC;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, ptiles = hx / PC;
  const int pt = tile % ptiles, y = tile / ptiles;
  const long long zs = (long long)d.ny * hx;
  const C *pw = (const C *)d.pwz;
  C *w = (C *)d.w + (long long)y * hx + pt * PC;
  const long long wn = d.n * d.Nhs, wb = (long long)y * hx + pt * PC;
  (void)wn;
  (void)wb;
  for (int e = threadIdx.x; e < L; e += NT) tw[e] = ((const C *)d.twz)[e];
  const long long ay = 2 * y - d.ny + 1;
  const long long gbase = (long long)y * hx + pt * PC;
  auto at = [&](int v, int z, int p) -> C & { return buf[sr_zi<L, PC>(v, z, p)]; };

  // forward pass 0: global -> registers -> shared (the loads of up to 16
  // values' worth of tasks are issued together: more loads in flight)
  {
    constexpr int R0 = pl.r[0], T = NS * PC * (L / R0), K0 = (T + NT - 1) / NT;
    constexpr int KB = K0 * R0 <= 16 ? K0 : 1;
#pragma unroll 1
    for (int k0 = 0; k0 < K0; k0 += KB) {
      C a[KB][R0];
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) {
        const int task = threadIdx.x + (k0 + kk) * NT;
        if (k0 + kk < K0 && (T % NT == 0 || task < T)) {
          const int p = task % PC, q = task / PC, j = q % (L / R0), v = q / (L / R0);
#pragma unroll
          for (int m = 0; m < R0; ++m) {
            const long long gi = v * d.Nhs + sr_in<L, R0>(j, m) * zs + p;
            a[kk][m] = R3D_IN(d, wb + gi, wn) ? w[gi] : C{0, 0};
          }
        }
      }
#pragma unroll
      for (int kk = 0; kk < KB; ++kk) {
        const int task = threadIdx.x + (k0 + kk) * NT;
        if (k0 + kk < K0 && (T % NT == 0 || task < T)) {
          const int p = task % PC, q = task / PC, j = q % (L / R0), v = q / (L / R0);
#pragma unroll
          for (int m = 0; m < R0; ++m) a[kk][m] = cmul(a[kk][m], sr_half_twiddle<R0>(pw[j], m));
          sr_pass<L, R0, 1, -1>(a[kk], tw, j);
#pragma unroll
          for (int m = 0; m < R0; ++m) at(v, sr_out<R0, 1>(j, m), p) = a[kk][m];
        }
      }
    }
    __syncthreads();
  }
  sr_zoz_middle<P, L, PC, NS, NT, OZREG>(buf, tw, d, pt, ay, gbase, zs);
  sr_zoz_last<P, L, PC, NS, NT>(buf, tw, d, w, pw, wb, wn, zs);
}

// Persistent z pass: gridDim.x CTAs (one per SM) walk the launch's tiles t =
// blockIdx.x, blockIdx.x + gridDim.x, ...  A second tile buffer takes the
// next tile's spectrum with 16-byte asynchronous copies (cp.async) while the
// current tile is transformed, so that the DRAM reads of tile t + gridDim.x
// overlap the transforms of tile t; the forward transform's first pass reads
// the staged tile.  The OZ runs as a shared-memory pass (OZREG false).
template <typename P, int L, int PC, int NS, int NT>
__global__ void __launch_bounds__(NT, 1) k_zoz_srp(Batch b, int ntiles) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr int TS = NS * sr_zrows<L>() * PC;  // complex values of one tile buffer
  constexpr int CW = 16 / (int)sizeof(C);      // complex values of one 16-byte copy
  constexpr int CH = PC / CW;                  // copies per row of a site
  static_assert(PC % CW == 0, "tile rows of whole 16-byte copies");
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem, *stage = buf + TS, *tw = stage + TS;
  // every solve of a launch has this launch's geometry: one twiddle table
  for (int e = threadIdx.x; e < L; e += NT) tw[e] = ((const C *)b.d[0].twz)[e];
  // the copies of tile t into stage (none for a solve that is not running)
  auto fetch = [&](int t) {
    const int si = find_solve(b, t);
    const Desc &d = b.d[si];
    if (d.ctl->status == RUNNING) {
      const int tile = t - b.prefix[si];
      const int hx = d.hx, ptiles = hx / PC, pt = tile % ptiles, y = tile / ptiles;
      const long long zs = (long long)d.ny * hx;
      const long long wb = (long long)y * hx + pt * PC, wn = d.n * d.Nhs;
      const C *w = (const C *)d.w + wb;
      (void)wn;
      for (int c = threadIdx.x; c < NS * L * CH; c += NT) {
        const int q = c % CH, row = c / CH, z = row % L, v = row / L;
        const long long gi = v * d.Nhs + z * zs + q * CW;
        if (R3D_IN(d, wb + gi, wn)) cp_async16(stage + sr_zi<L, PC>(v, z, q * CW), w + gi);
      }
    }
    cp_async_commit();
  };
  if ((int)blockIdx.x < ntiles) fetch(blockIdx.x);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();  // stage holds tile t; the last tile's final pass has read buf
    const int si = find_solve(b, t);
    const Desc &d = b.d[si];
    const bool run = d.ctl->status == RUNNING;  // the same for the whole CTA
    const int tile = t - b.prefix[si];
    const int hx = d.hx, ptiles = hx / PC, pt = tile % ptiles, y = tile / ptiles;
    const long long zs = (long long)d.ny * hx;
    const long long wb = (long long)y * hx + pt * PC, wn = d.n * d.Nhs;
    const C *pw = (const C *)d.pwz;
    if (run) {  // forward pass 0: stage -> registers -> buf
      constexpr int R0 = sr_plan(L).r[0], T = NS * PC * (L / R0);
      for (int task = threadIdx.x; task < T; task += NT) {
        const int p = task % PC, q = task / PC, j = q % (L / R0), v = q / (L / R0);
        C a[R0];
        const C pj = pw[j];
#pragma unroll
        for (int m = 0; m < R0; ++m)
          a[m] = cmul(stage[sr_zi<L, PC>(v, sr_in<L, R0>(j, m), p)], sr_half_twiddle<R0>(pj, m));
        sr_pass<L, R0, 1, -1>(a, tw, j);
#pragma unroll
        for (int m = 0; m < R0; ++m) buf[sr_zi<L, PC>(v, sr_out<R0, 1>(j, m), p)] = a[m];
      }
    }
    __syncthreads();  // stage is free for the next tile
    if (t + (int)gridDim.x < ntiles) fetch(t + gridDim.x);
    if (!run) continue;
    sr_zoz_middle<P, L, PC, NS, NT, false>(buf, tw, d, pt, 2LL * y - d.ny + 1,
                                           (long long)y * hx + pt * PC, zs);
    sr_zoz_last<P, L, PC, NS, NT>(buf, tw, d, (C *)d.w + wb, pw, wb, wn, zs);
  }
  cp_async_wait_all();
}

// ------------------------------------------------------------ launchers
// Tiles: FY PC columns (16 FP32 / 8 FP64: 128-byte rows); ZOZ about 32 FP32
// (16 FP64) spectrum columns over all sites (half of that for 512-point
// columns), a power of two per site.
template <typename P>
constexpr int sr_pc_y() {
  return sizeof(typename P::R) == 4 ? 16 : 8;
}
#ifndef R3D_SR_ZBASE32
#define R3D_SR_ZBASE32 32
#endif
#ifndef R3D_SR_ZHI
#define R3D_SR_ZHI 256
#endif
template <typename P>
constexpr int sr_pc_z(int L, int ns) {
  int base = (sizeof(typename P::R) == 4 ? R3D_SR_ZBASE32 : 16) / (L >= 512 ? 2 : 1);
  int pc = 1;
  while (pc * 2 * ns <= base) pc *= 2;
  return pc;
}
// threads of the z pass: register OZ: one OZ task (all sites) per thread,
// 64..256; shared OZ: one task of the largest-radix pass per thread, 64..256
// (two CTAs per SM; measured faster than one CTA of 512 at 256^3 and 512^3
// with four sites), a whole number of warps: the OZ pass deals pairs out by
// warp
template <typename P>
constexpr int sr_threads_z(int L, int ns, bool ozreg) {
  int t = ozreg ? sr_pc_z<P>(L, ns) * (L / sr_plan(L).r[sr_plan(L).n - 1])
                : ns * sr_pc_z<P>(L, ns) * (L / sr_max_radix(L));
  t = (t + 31) / 32 * 32;
  const int hi = ozreg ? 256 : R3D_SR_ZHI;
  return t < 64 ? 64 : (t > hi ? hi : t);
}

// threads of the persistent z pass: one task of the largest-radix pass per
// thread, 64..512 whole warps
template <typename P>
constexpr int sr_threads_zp(int L, int ns) {
  int t = ns * sr_pc_z<P>(L, ns) * (L / sr_max_radix(L));
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : (t > 512 ? 512 : t);
}
// tile rows of the persistent z pass are whole 16-byte copies
template <typename P>
constexpr bool sr_zp_ok(int L, int ns) {
  return sr_pc_z<P>(L, ns) % (16 / (int)sizeof(typename Cx<typename P::R>::T)) == 0;
}

#define R3D_SR_LENGTHS(X) X(16) X(24) X(32) X(40) X(48) X(64) X(72) X(80) X(96) X(128) X(144) X(160) X(192) X(256) X(512)

#if R3D_CT_FP64
size_t sr_smem_y(int L, int PC, size_t csz) { return csz * (size_t)L * (PC + 1); }
size_t sr_smem_z(int L, int PC, int ns, size_t csz) {
  return csz * ((size_t)ns * (L + L / 16 + 1) * PC + L);
}
bool sr_length_supported(int L) { return sr_length_ok(L); }
// the persistent z pass: two tile buffers and the twiddle table
size_t sr_smem_zp(int L, int PC, int ns, size_t csz) {
  return csz * (2 * (size_t)ns * (L + L / 16 + 1) * PC + L);
}
#endif

template <typename K>
static void sr_allow(K kern) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
}

template <typename P>
int sr_pc_y_of() { return sr_pc_y<P>(); }
template <typename P>
int sr_pc_z_of(int L, int ns) { return (ns >= 1 && ns <= 4) ? sr_pc_z<P>(L, ns) : 0; }

// false: no kernel for the length
template <typename P>
bool sr_launch_fy(int L, int dir, Batch b, int grid, size_t smem, cudaStream_t s) {
  constexpr int PC = sr_pc_y<P>();
#define R3D_SRY(LL)                                                  \
  if (L == LL) {                                                     \
    if (dir < 0)                                                     \
      k_fy_sr<P, LL, PC, -1><<<grid, kThreads, smem, s>>>(b);        \
    else                                                             \
      k_fy_sr<P, LL, PC, 1><<<grid, kThreads, smem, s>>>(b);         \
    return true;                                                     \
  }
  R3D_SR_LENGTHS(R3D_SRY)
#undef R3D_SRY
  return false;
}

template <typename P, int NS, bool OZREG>
static bool sr_launch_zoz_ns(int L, Batch b, int grid, size_t smem, cudaStream_t s) {
#define R3D_SRZ(LL)                                                              \
  if (L == LL) {                                                                 \
    constexpr int PC = sr_pc_z<P>(LL, NS), NT = sr_threads_z<P>(LL, NS, OZREG);  \
    k_zoz_sr<P, LL, PC, NS, NT, OZREG><<<grid, NT, smem, s>>>(b);                \
    return true;                                                                 \
  }
  R3D_SR_LENGTHS(R3D_SRZ)
#undef R3D_SRZ
  return false;
}
// ozreg: the OZ on registers (variant 3) or as a shared-memory pass (4)
template <typename P>
bool sr_launch_zoz(int L, int ns, bool ozreg, Batch b, int grid, size_t smem, cudaStream_t s) {
  switch (ns * 2 + (ozreg ? 1 : 0)) {
    case 2: return sr_launch_zoz_ns<P, 1, false>(L, b, grid, smem, s);
    case 3: return sr_launch_zoz_ns<P, 1, true>(L, b, grid, smem, s);
    case 4: return sr_launch_zoz_ns<P, 2, false>(L, b, grid, smem, s);
    case 5: return sr_launch_zoz_ns<P, 2, true>(L, b, grid, smem, s);
    case 6: return sr_launch_zoz_ns<P, 3, false>(L, b, grid, smem, s);
    case 7: return sr_launch_zoz_ns<P, 3, true>(L, b, grid, smem, s);
    case 8: return sr_launch_zoz_ns<P, 4, false>(L, b, grid, smem, s);
    case 9: return sr_launch_zoz_ns<P, 4, true>(L, b, grid, smem, s);
    default: return false;
  }
}

// The persistent z pass over ntiles tiles with `grid` CTAs (false: no
// kernel for the length and sites).
template <typename P, int NS>
static bool sr_launch_zozp_ns(int L, Batch b, int ntiles, int grid, size_t smem, cudaStream_t s) {
#define R3D_SRZP(LL)                                                        \
  if (L == LL) {                                                            \
    if constexpr (sr_zp_ok<P>(LL, NS)) {                                    \
      constexpr int PC = sr_pc_z<P>(LL, NS), NT = sr_threads_zp<P>(LL, NS);  \
      k_zoz_srp<P, LL, PC, NS, NT><<<grid, NT, smem, s>>>(b, ntiles);       \
      return true;                                                          \
    }                                                                       \
    return false;                                                           \
  }
  R3D_SR_LENGTHS(R3D_SRZP)
#undef R3D_SRZP
  return false;
}
template <typename P>
bool sr_launch_zozp(int L, int ns, Batch b, int ntiles, int grid, size_t smem, cudaStream_t s) {
  grid = grid < ntiles ? grid : ntiles;
  if (grid < 1) return true;  // no tiles
  switch (ns) {
    case 1: return sr_launch_zozp_ns<P, 1>(L, b, ntiles, grid, smem, s);
    case 2: return sr_launch_zozp_ns<P, 2>(L, b, ntiles, grid, smem, s);
    case 3: return sr_launch_zozp_ns<P, 3>(L, b, ntiles, grid, smem, s);
    case 4: return sr_launch_zozp_ns<P, 4>(L, b, ntiles, grid, smem, s);
    default: return false;
  }
}
// resident CTAs per SM of the persistent z pass (0: no kernel, or it does
// not fit); its shared-memory attribute must be set (sr_allow_geometry)
template <typename P, int NS>
static int sr_occupancy_zozp_ns(int L, size_t smem) {
  int nb = 0;
#define R3D_SRZO(LL)                                                                       \
  if (L == LL) {                                                                           \
    if constexpr (sr_zp_ok<P>(LL, NS)) {                                                   \
      constexpr int PC = sr_pc_z<P>(LL, NS), NT = sr_threads_zp<P>(LL, NS);                 \
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_zoz_srp<P, LL, PC, NS, NT>, \
                                                        NT, smem) != cudaSuccess) {       \
        cudaGetLastError();                                                                \
        nb = 0;                                                                            \
      }                                                                                    \
    }                                                                                      \
  }
  R3D_SR_LENGTHS(R3D_SRZO)
#undef R3D_SRZO
  return nb;
}
template <typename P>
int sr_occupancy_zozp(int L, int ns, size_t smem) {
  switch (ns) {
    case 1: return sr_occupancy_zozp_ns<P, 1>(L, smem);
    case 2: return sr_occupancy_zozp_ns<P, 2>(L, smem);
    case 3: return sr_occupancy_zozp_ns<P, 3>(L, smem);
    case 4: return sr_occupancy_zozp_ns<P, 4>(L, smem);
    default: return 0;
  }
}
template <typename P>
int sr_zp_supported(int L, int ns) {
  int ok = 0;
#define R3D_SRZS(LL) \
  if (L == LL) ok = ns == 1 ? sr_zp_ok<P>(LL, 1) : ns == 2 ? sr_zp_ok<P>(LL, 2) : ns == 3 ? sr_zp_ok<P>(LL, 3) : ns == 4 ? sr_zp_ok<P>(LL, 4) : 0;
  R3D_SR_LENGTHS(R3D_SRZS)
#undef R3D_SRZS
  return ok;
}

template <typename P, int LL, int NS>
static void sr_allow_zoz() {
  sr_allow(k_zoz_sr<P, LL, sr_pc_z<P>(LL, NS), NS, sr_threads_z<P>(LL, NS, false), false>);
  sr_allow(k_zoz_sr<P, LL, sr_pc_z<P>(LL, NS), NS, sr_threads_z<P>(LL, NS, true), true>);
  if constexpr (sr_zp_ok<P>(LL, NS))
    sr_allow(k_zoz_srp<P, LL, sr_pc_z<P>(LL, NS), NS, sr_threads_zp<P>(LL, NS)>);
}

// x passes: PC rows per tile, PC * (L / R_0) tasks filling the CTA
template <int L>
constexpr int sr_pc_x() {  // a power of two (it divides the rows of a site)
  constexpr int J = L / sr_plan(L).r[0];
  int pc = 1;
  while (pc * 2 * J <= kThreads) pc *= 2;
  return pc;
}
#if R3D_CT_FP64
int sr_pc_x_of(int L) {
#define R3D_SRPX(LL) \
  if (L == LL) return sr_pc_x<LL>();
  R3D_SR_LENGTHS(R3D_SRPX)
#undef R3D_SRPX
  return 0;
}
size_t sr_smem_x(int L, int PC, size_t csz) {
  return csz * ((size_t)PC * (L + L / 16 + 1) + L);
}
#endif
template <typename P>
bool sr_launch_fx(int L, Batch b, int grid, size_t smem, cudaStream_t s) {
#define R3D_SRX(LL)                                                       \
  if (L == LL) {                                                          \
    k_fx_sr<P, LL, sr_pc_x<LL>()><<<grid, kThreads, smem, s>>>(b);        \
    return true;                                                          \
  }
  R3D_SR_LENGTHS(R3D_SRX)
#undef R3D_SRX
  return false;
}
template <typename P>
bool sr_launch_ix(int L, Batch b, int grid, size_t smem, cudaStream_t s, int per) {
#define R3D_SRX(LL)                                                       \
  if (L == LL) {                                                          \
    k_ix_sr<P, LL, sr_pc_x<LL>()><<<grid, kThreads, smem, s>>>(b, per);   \
    return true;                                                          \
  }
  R3D_SR_LENGTHS(R3D_SRX)
#undef R3D_SRX
  return false;
}

// The kernels of one geometry: x passes of length hx, y of ny, z with its
// OZ over ns sites of nz (both OZ forms).  Setting the attribute loads the
// kernel, so a solve loads only the lengths it uses.
template <typename P>
void sr_allow_geometry(int hx, int ny, int nz, int ns) {
  constexpr int PC = sr_pc_y<P>();
#define R3D_SRG(LL)                                                   \
  if (hx == LL) {                                                     \
    sr_allow(k_fx_sr<P, LL, sr_pc_x<LL>()>);                          \
    sr_allow(k_ix_sr<P, LL, sr_pc_x<LL>()>);                          \
  }                                                                   \
  if (ny == LL) {                                                     \
    sr_allow(k_fy_sr<P, LL, PC, -1>);                                 \
    sr_allow(k_fy_sr<P, LL, PC, 1>);                                  \
  }                                                                   \
  if (nz == LL) {                                                     \
    if (ns == 1) sr_allow_zoz<P, LL, 1>();                            \
    if (ns == 2) sr_allow_zoz<P, LL, 2>();                            \
    if (ns == 3) sr_allow_zoz<P, LL, 3>();                            \
    if (ns == 4) sr_allow_zoz<P, LL, 4>();                            \
  }
  R3D_SR_LENGTHS(R3D_SRG)
#undef R3D_SRG
}

template bool sr_launch_fx<PSR>(int, Batch, int, size_t, cudaStream_t);
template bool sr_launch_ix<PSR>(int, Batch, int, size_t, cudaStream_t, int);
template bool sr_launch_fy<PSR>(int, int, Batch, int, size_t, cudaStream_t);
template bool sr_launch_zoz<PSR>(int, int, bool, Batch, int, size_t, cudaStream_t);
template void sr_allow_geometry<PSR>(int, int, int, int);
template bool sr_launch_zozp<PSR>(int, int, Batch, int, int, size_t, cudaStream_t);
template int sr_occupancy_zozp<PSR>(int, int, size_t);
template int sr_zp_supported<PSR>(int, int);
template int sr_pc_y_of<PSR>();
template int sr_pc_z_of<PSR>(int, int);

}  // namespace r3d
