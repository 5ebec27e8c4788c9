// r3d_passes_ct.cu -- the five grid passes on the compile-time FFT engine
// (r3d_fft_ct.cuh).  Compiled once per precision: R3D_CT_FP64 = 1 builds the
// FP64 instantiations, 0 the mixed-precision ones.  The passes compute the
// same quantities as the runtime-length passes in r3d_kernels.cu (which stay
// as the fallback for lengths outside kCtLengths); see that file for the
// algorithm and the reference lines each step follows.
#include "r3d_common.cuh"
#include "r3d_fft_ct.cuh"
#include "r3d_async.cuh"

#ifndef R3D_CT_FP64
#define R3D_CT_FP64 1
#endif

namespace r3d {

#if R3D_CT_FP64
using PCT = P64;
#else
using PCT = PMix;
#endif

// ------------------------------------------------------------------ FX
// tile = PC consecutive rows (row = y + ny z) of one site; smem [L][PC+1].
template <typename P, int L, int PC, int MODE>
__global__ void __launch_bounds__(kThreads)
    k_fx_ct(Batch b, const typename P::R *src) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  constexpr int LD = PC + 1;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;
  __shared__ int par[PC];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (MODE == 1 && d.ctl->status != RUNNING) return;
  const int tile = blockIdx.x - b.prefix[si];
  const int tps = (d.ny * d.nz) / PC;  // tiles per site
  const int v = tile / tps;
  const long long row0 = (long long)(tile % tps) * PC;
  const int nx = d.nx, ny = d.ny;
  if (threadIdx.x < PC) {
    long long row = row0 + threadIdx.x;
    par[threadIdx.x] = (int)((row % ny + row / ny) & 1);
  }
  __syncthreads();
  const C *pw = (const C *)d.pwx;
  const T *t = (const T *)d.t;
  const R *u = (const R *)d.u, *cref = (const R *)d.cref;
#pragma unroll 4
  for (int e = threadIdx.x; e < PC * L; e += kThreads) {
    const int r = e / L, m = e % L;
    const long long base = (long long)v * d.Ns + (row0 + r) * nx;
    R f0, f1;
    if (MODE == 0) {
      f0 = src[base + m];
      f1 = src[base + m + L];
    } else {
      // trm1mt on the short-range parts (calculate_cuda.cu:18-24)
      const double t0 = t[base + m], t1 = t[base + m + L];
      const double g0 = closure_g<double>(d.clos, d.pse_n, -(double)u[base + m] + t0);
      const double g1 = closure_g<double>(d.clos, d.pse_n, -(double)u[base + m + L] + t1);
      ((T *)d.gq)[base + m] = g0;
      ((T *)d.gq)[base + m + L] = g1;
      double c0 = g0 - 1.0 - t0, c1 = g1 - 1.0 - t1;
      if (cref) {
        c0 -= (double)cref[base + m];
        c1 -= (double)cref[base + m + L];
      }
      f0 = (R)c0;
      f1 = (R)c1;
    }
    if ((m + par[r]) & 1) f0 = -f0;
    if ((m + L + par[r]) & 1) f1 = -f1;
    buf[digit_rev<L>(m) * LD + r] = cmul(C{f0, -f1}, pw[m]);
  }
  __syncthreads();
  ct_fft_dit<L, PC, LD, -1>(buf, (const C *)d.twx);
  C *w = (C *)d.w + (long long)v * d.Nhs + row0 * L;
#pragma unroll
  for (int e = threadIdx.x; e < PC * L; e += kThreads) {
    const int r = e / L, p = e % L;
    w[(long long)r * L + p] = buf[p * LD + r];
  }
}

// ------------------------------------------------------------------ FY
// tile = PC x-columns of one (site, z) plane; smem [L = ny][PC].
template <typename P, int L, int PC, int DIR>
__global__ void __launch_bounds__(kThreads)
    k_fy_ct(Batch b, int check) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (check && d.ctl->status != RUNNING) return;
  int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, ptiles = hx / PC;
  const int pt = tile % ptiles;
  tile /= ptiles;
  const int z = tile % d.nz, v = tile / d.nz;
  const C *pw = (const C *)d.pwy;
  C *w = (C *)d.w + (long long)v * d.Nhs + (long long)z * L * hx + pt * PC;
  if (DIR < 0) {
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int p = e % PC, y = e / PC;
      buf[digit_rev<L>(y) * PC + p] = cmul(w[(long long)y * hx + p], pw[y]);
    }
    __syncthreads();
    ct_fft_dit<L, PC, PC, -1>(buf, (const C *)d.twy);
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int p = e % PC, y = e / PC;
      w[(long long)y * hx + p] = buf[y * PC + p];
    }
  } else {
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int p = e % PC, y = e / PC;
      buf[y * PC + p] = w[(long long)y * hx + p];
    }
    __syncthreads();
    ct_fft_dif<L, PC, PC, 1>(buf, (const C *)d.twy);
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int p = e % PC, y = e / PC;
      w[(long long)y * hx + p] = cmul(buf[digit_rev<L>(y) * PC + p], cconj(pw[y]));
    }
  }
}

// ------------------------------------------------------------------ ZOZ
// tile = PC x-columns at one y, all n sites; smem [site][L = nz][PC].
// Forward z, (mqvfk when d.fk is set), Ornstein-Zernike, inverse z.
// ZMAJOR: the tile is [z][site][p] (all sites' columns side by side, one
// transform over NS * PC columns); else [site][z][p]
template <typename P, int L, int PC, int NS, bool ZMAJOR = false>
__device__ __forceinline__ void ct_oz(typename Cx<typename P::R>::T *buf, const Desc &d,
                                      int y, int pt) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr int M = NS > 0 ? NS : kMaxSites;
  const int n = NS > 0 ? NS : d.n;
  const long long zs = (long long)d.ny * d.hx;
  const long long off = (long long)y * d.hx + pt * PC;
  const R *chi = (const R *)d.chi;
  const double2 *fk = (const double2 *)d.fk;
  // shell of |k|: cubic cells use s = ax^2 + ay^2 + az^2 over the odd
  // integers a = 2j - n + 1 (shell (s - 3) / 8), others the kidx table
  const long long ay = 2 * y - d.ny + 1;
#pragma unroll 2
  for (int e = threadIdx.x; e < PC * L; e += kThreads) {
    const int p = e % PC, z = e / PC;
    const long long gi = z * zs + off + p;
    size_t shell;
    if (d.cubic) {
      const long long ax = 4 * (pt * PC + p) - d.nx + 1, az = 2 * z - d.nz + 1;
      shell = (size_t)((ax * ax + ay * ay + az * az - 3) / 8);
    } else {
      shell = d.kidx[gi];
    }
    const R *ch = chi + shell * d.chis;
    R x[M * M];
    if constexpr (NS > 0 && (NS * NS) % 4 == 0 && sizeof(R) == 4) {  // 16-byte rows
#pragma unroll
      for (int q = 0; q < NS * NS / 4; ++q) {
        const float4 v4 = reinterpret_cast<const float4 *>(ch)[q];
        x[4 * q] = v4.x;
        x[4 * q + 1] = v4.y;
        x[4 * q + 2] = v4.z;
        x[4 * q + 3] = v4.w;
      }
    } else if constexpr (NS > 0 && (NS * NS) % 2 == 0 && sizeof(R) == 8) {
#pragma unroll
      for (int q = 0; q < NS * NS / 2; ++q) {
        const double2 v2 = reinterpret_cast<const double2 *>(ch)[q];
        x[2 * q] = v2.x;
        x[2 * q + 1] = v2.y;
      }
    } else {
#pragma unroll
      for (int q = 0; q < M * M; ++q)
        if (q < n * n) x[q] = ch[q];
    }
    C c[M];
#pragma unroll
    for (int q = 0; q < M; ++q)
      if (q < n) c[q] = buf[ZMAJOR ? (z * NS + q) * PC + p : (q * L + z) * PC + p];
    if (fk) {  // mqvfk (refresh pipeline only)
      const double2 f = fk[gi];
#pragma unroll
      for (int q = 0; q < M; ++q)
        if (q < n) {
          c[q].x -= (R)(d.qv[q] * f.x);
          c[q].y -= (R)(d.qv[q] * f.y);
        }
    }
#pragma unroll
    for (int a = 0; a < M; ++a) {
      if (a < n) {
        R hr = 0, hi = 0;
#pragma unroll
        for (int q = 0; q < M; ++q) {
          if (q < n) {
            const R xq = x[a * n + q];
            hr += c[q].x * xq;
            hi += c[q].y * xq;
          }
        }
        buf[ZMAJOR ? (z * NS + a) * PC + p : (a * L + z) * PC + p] = C{hr, hi};
      }
    }
  }
}

// z transform, OZ and inverse z transform of one tile with the NS sites'
// columns side by side: smem [z][site][p], rows digit-reversed for the DIT
template <typename P, int L, int PC, int NS>
__device__ __forceinline__ void zoz_sites(typename Cx<typename P::R>::T *buf, const Desc &d,
                                          typename Cx<typename P::R>::T *w, long long zs,
                                          const typename Cx<typename P::R>::T *pw,
                                          const typename Cx<typename P::R>::T *tw, int ky,
                                          int pt) {
  using C = typename Cx<typename P::R>::T;
  constexpr int W = NS * PC;  // columns of the transform
#pragma unroll 4
  for (int e = threadIdx.x; e < W * L; e += kThreads) {
    const int p = e % PC, v = (e / PC) % NS, z = e / W;
    buf[(digit_rev<L>(z) * NS + v) * PC + p] = cmul(w[v * d.Nhs + z * zs + p], pw[z]);
  }
  __syncthreads();
  ct_fft_dit<L, W, W, -1>(buf, tw);
  ct_oz<P, L, PC, NS, true>(buf, d, ky, pt);
  __syncthreads();
  ct_fft_dif<L, W, W, 1>(buf, tw);
#pragma unroll 4
  for (int e = threadIdx.x; e < W * L; e += kThreads) {
    const int p = e % PC, v = (e / PC) % NS, z = e / W;
    w[v * d.Nhs + z * zs + p] = cmul(buf[(digit_rev<L>(z) * NS + v) * PC + p], cconj(pw[z]));
  }
}

// check: bit 0 = skip solves not running; bit 1 = w's y rows are in the
// digit-reversed ky order of the copy-engine y pass (ky from d.yrev)
template <typename P, int L, int PC>
__global__ void __launch_bounds__(kThreads, sizeof(typename P::R) == 4 ? 3 : 2)
    k_zoz_ct(Batch b, int check) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if ((check & 1) && d.ctl->status != RUNNING) return;
  const int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, n = d.n, ptiles = hx / PC;
  const int pt = tile % ptiles, y = tile / ptiles;
  const int ky = (check & 2) ? d.yrev[y] : y;
  const long long zs = (long long)d.ny * hx;
  const C *pw = (const C *)d.pwz, *tw = (const C *)d.twz;
  C *w = (C *)d.w + (long long)y * hx + pt * PC;
  // up to four sites: one transform over all sites' columns ([z][site][p]),
  // a quarter of the barriers of one transform per site
  switch (n) {
    case 1: zoz_sites<P, L, PC, 1>(buf, d, w, zs, pw, tw, ky, pt); return;
    case 2: zoz_sites<P, L, PC, 2>(buf, d, w, zs, pw, tw, ky, pt); return;
    case 3: zoz_sites<P, L, PC, 3>(buf, d, w, zs, pw, tw, ky, pt); return;
    case 4: zoz_sites<P, L, PC, 4>(buf, d, w, zs, pw, tw, ky, pt); return;
    default: break;
  }
  for (int v = 0; v < n; ++v) {
    const C *wv = w + (long long)v * d.Nhs;
    C *bv = buf + v * L * PC;
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int p = e % PC, z = e / PC;
      bv[digit_rev<L>(z) * PC + p] = cmul(wv[z * zs + p], pw[z]);
    }
  }
  __syncthreads();
  for (int v = 0; v < n; ++v) ct_fft_dit<L, PC, PC, -1>(buf + v * L * PC, tw);
  switch (n) {
    case 1: ct_oz<P, L, PC, 1>(buf, d, ky, pt); break;
    case 2: ct_oz<P, L, PC, 2>(buf, d, ky, pt); break;
    case 3: ct_oz<P, L, PC, 3>(buf, d, ky, pt); break;
    case 4: ct_oz<P, L, PC, 4>(buf, d, ky, pt); break;
    default: ct_oz<P, L, PC, 0>(buf, d, ky, pt); break;
  }
  __syncthreads();
  for (int v = 0; v < n; ++v) ct_fft_dif<L, PC, PC, 1>(buf + v * L * PC, tw);
  for (int v = 0; v < n; ++v) {
    C *wv = w + (long long)v * d.Nhs;
    const C *bv = buf + v * L * PC;
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int p = e % PC, z = e / PC;
      wv[z * zs + p] = cmul(bv[digit_rev<L>(z) * PC + p], cconj(pw[z]));
    }
  }
}

// ------------------------------------------------------------------ IX
// tiles as FX; a CTA handles `per` consecutive tiles.  MODE 0 writes the
// real grid to dst; MODE 1 forms g, R = h + 1 - g (calculate_cuda.cu:54-60),
// sum R^2 (cal_rms.cu) and, past AN2's Picard warm-up, the five theta dots
// per site (anderson_cuda.cu:25-67) into this CTA's partials.
#ifndef R3D_IX_MINB
#define R3D_IX_MINB 2
#endif
#ifndef R3D_IX_UNROLL
#define R3D_IX_UNROLL 1
#endif
#define R3D_PRAGMA(x) _Pragma(#x)
#define R3D_UNROLL_N(n) R3D_PRAGMA(unroll n)
#define R3D_UNROLL(n) R3D_UNROLL_N(n)
// rows of up to 128 reals: four resident CTAs (64 registers) instead of two,
// since at those lengths the kernel waits on its global loads
template <typename P, int L, int PC, int MODE>
__global__ void __launch_bounds__(kThreads, L <= 64 ? 4 : R3D_IX_MINB)
    k_ix_ct(Batch b, typename P::R *dst, int per) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  constexpr int LD = PC + 1;
  extern __shared__ __align__(16) char smem[];
  C *buf = (C *)smem;
  __shared__ int par[PC];
  __shared__ double red6[6 * (kThreads / 32)];
  __shared__ double sums[kPartials];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (MODE == 1 && d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int nx = d.nx, ny = d.ny;
  const int tps = (d.ny * d.nz) / PC;
  const int ntile = d.n * tps;
  const bool dots = MODE == 1 && d.mixer == MIX_AN2 && d.ctl->count_left <= 0;
  const C *pw = (const C *)d.pwx, *tw = (const C *)d.twx;
  const T *gq = (const T *)d.gq;
  const R *lr = (const R *)d.lr;
  R *res = (R *)d.res;
  const R *rp = (const R *)d.hist_b;
  const long long niv = (long long)d.n * d.Ns;
  if (MODE == 1)
    for (int k = threadIdx.x; k < kPartials; k += kThreads) sums[k] = 0;
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
    if (MODE == 1 && v != cur_v) {
      flush();
      cur_v = v;
    }
    __syncthreads();
    if (threadIdx.x < PC) {
      long long row = row0 + threadIdx.x;
      par[threadIdx.x] = (int)((row % ny + row / ny) & 1);
    }
    const C *w = (const C *)d.w + (long long)v * d.Nhs + row0 * L;
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, p = e % L;
      buf[p * LD + r] = w[(long long)r * L + p];
    }
    __syncthreads();
    ct_fft_dif<L, PC, LD, 1>(buf, tw);
    R3D_UNROLL(R3D_IX_UNROLL)
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, m = e % L;
      const C zc = cmul(buf[digit_rev<L>(m) * LD + r], cconj(pw[m]));
      R h0 = zc.x, h1 = -zc.y;
      if ((m + par[r]) & 1) h0 = -h0;
      if ((m + L + par[r]) & 1) h1 = -h1;
      const long long base = (long long)v * d.Ns + (row0 + r) * nx;
      if (MODE == 0) {
        dst[base + m] = h0;
        dst[base + m + L] = h1;
      } else {
        const double g0 = gq[base + m], g1 = gq[base + m + L];
        const R r0 = (R)((double)h0 + (double)lr[base + m] - g0);
        const R r1 = (R)((double)h1 + (double)lr[base + m + L] - g1);
        res[base + m] = r0;
        res[base + m + L] = r1;
        a_ss += (double)r0 * r0 + (double)r1 * r1;
        if (dots) {
          const double p0 = rp[base + m], p1 = rp[base + m + L];
          const double q0 = rp[niv + base + m], q1 = rp[niv + base + m + L];
          const double t10 = (double)r0 - p0, t20 = (double)r0 - q0;
          const double t11 = (double)r1 - p1, t21 = (double)r1 - q1;
          a0 += r0 * t10 + r1 * t11;
          a1 += r0 * t20 + r1 * t21;
          a2 += t10 * t10 + t11 * t11;
          a3 += t10 * t20 + t11 * t21;
          a4 += t20 * t20 + t21 * t21;
        }
      }
    }
  }
  if (MODE == 0) return;
  flush();
  __syncthreads();
  double *part = d.partials + (size_t)cta * kPartials;
  for (int k = threadIdx.x; k < kPartials; k += kThreads) part[k] = sums[k];
}

// ------------------------------------------------- IX with bulk staging
// The iteration's IX (MODE 1) with the per-voxel inputs staged by the bulk
// copy engine: a tile's PC rows of one site are one contiguous block in each
// of gq, lr and the two AN2 residual slots, so one cp.async.bulk per array
// brings the next tile into shared memory while the current one is being
// transformed and reduced (two stages, one mbarrier each).
template <typename P, int L, int PC>
struct IxStage {  // byte layout of one stage of staged inputs
  static constexpr int NX = 2 * L;
  static constexpr size_t gq = 0;
  static constexpr size_t lr = gq + (size_t)PC * NX * sizeof(typename P::T);
  static constexpr size_t r0 = lr + (size_t)PC * NX * sizeof(typename P::R);
  static constexpr size_t r1 = r0 + (size_t)PC * NX * sizeof(typename P::R);
  static constexpr size_t w = r1 + (size_t)PC * NX * sizeof(typename P::R);  // spectrum rows
  static constexpr size_t bytes = w + (size_t)PC * L * 2 * sizeof(typename P::R);
};
#if R3D_CT_FP64
size_t ct_smem_ixb(int L, int PC, size_t csz, size_t rsz, size_t tsz) {
  const size_t buf = ((csz * (size_t)L * (PC + 1) + 127) / 128) * 128;
  const size_t stage = (size_t)PC * 2 * L * (tsz + 3 * rsz) + (size_t)PC * L * csz;
  return buf + 2 * stage;
}
#endif

// half-size tiles (PC 4 / 2) are the occupancy variant: three CTAs per SM
template <typename P, int L, int PC>
__global__ void __launch_bounds__(kThreads, PC < (sizeof(typename P::R) == 4 ? 8 : 4) ? 3 : 1)
    k_ix_bulk(Batch b, int per) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  using St = IxStage<P, L, PC>;
  constexpr int LD = PC + 1, NX = 2 * L;
  constexpr size_t BUF = ((sizeof(C) * (size_t)L * LD + 127) / 128) * 128;
  extern __shared__ __align__(128) char smem[];
  C *buf = (C *)smem;
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int par[PC];
  __shared__ double red6[6 * (kThreads / 32)];
  __shared__ double sums[kPartials];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int ny = d.ny;
  const int tps = (d.ny * d.nz) / PC;
  const int ntile = d.n * tps;
  const int first = cta * per;
  const int count = min(per, ntile - first);
  if (count <= 0) return;
  const bool dots = d.mixer == MIX_AN2 && d.ctl->count_left <= 0;
  const C *pw = (const C *)d.pwx, *tw = (const C *)d.twx;
  R *res = (R *)d.res;
  const long long niv = (long long)d.n * d.Ns;
  const uint32_t tbytes = PC * NX * sizeof(T), rbytes = PC * NX * sizeof(R);
  const uint32_t wbytes = PC * L * sizeof(C);
  const uint32_t stage_tx = tbytes + rbytes + wbytes + (dots ? 2 * rbytes : 0);
  const Desc *dp = &d;
  char *const stages = smem + BUF;
  uint64_t *const bars = bar;
  // thread 0: the copies of one tile into stage st (no captures by reference:
  // they would keep the loop's variables in local memory)
  auto issue = [=](int tile, int st) {
    const int v = tile / tps;
    const long long base = (long long)v * dp->Ns + (long long)(tile % tps) * PC * NX;
    char *sb = stages + st * St::bytes;
    uint64_t *br = bars + st;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(br, stage_tx);
    bulk_g2s(sb + St::gq, (const T *)dp->gq + base, tbytes, br);
    bulk_g2s(sb + St::lr, (const R *)dp->lr + base, rbytes, br);
    bulk_g2s(sb + St::w,
             (const C *)dp->w + (long long)v * dp->Nhs + (long long)(tile % tps) * PC * L,
             wbytes, br);
    if (dots) {
      bulk_g2s(sb + St::r0, (const R *)dp->hist_b + base, rbytes, br);
      bulk_g2s(sb + St::r1, (const R *)dp->hist_b + niv + base, rbytes, br);
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int k = threadIdx.x; k < kPartials; k += kThreads) sums[k] = 0;
  __syncthreads();
  if (threadIdx.x == 0) issue(first, 0);
  double a_ss = 0, a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0;
  int cur_v = -1;
  uint32_t phase = 0;  // bit st: parity of the next wait on stage st
  bool failed = false;
  int stop = -1;  // iteration at which a staged copy's wait ran out
  for (int it = 0; it < count; ++it) {
    const int tile = first + it, st = it & 1;
    const int v = tile / tps;
    const long long row0 = (long long)(tile % tps) * PC;
    if (v != cur_v) {  // uniform: flush the previous site's sums
      if (cur_v >= 0) {
        double q[6] = {a_ss, a0, a1, a2, a3, a4};
        block_sums<6>(q, red6);
        if (threadIdx.x == 0) {
          sums[0] += q[0];
          if (dots)
            for (int k = 0; k < 5; ++k) sums[1 + 5 * cur_v + k] += q[1 + k];
        }
        a_ss = a0 = a1 = a2 = a3 = a4 = 0;
      }
      cur_v = v;
    }
    // the other stage is free (its readers passed the barrier at the end of
    // the previous iteration): prefetch the next tile into it
    if (threadIdx.x == 0 && it + 1 < count) issue(tile + 1, st ^ 1);
    if (threadIdx.x < PC) {
      const long long row = row0 + threadIdx.x;
      par[threadIdx.x] = (int)((row % ny + row / ny) & 1);
    }
    if (!mbar_wait(&bar[st], (phase >> st) & 1, d.wait_polls)) failed = true;
    phase ^= 1u << st;
    const char *sb = smem + BUF + st * St::bytes;
    const C *ws = (const C *)(sb + St::w);
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, p = e % L;
      buf[p * LD + r] = ws[r * L + p];
    }
    __syncthreads();
    ct_fft_dif<L, PC, LD, 1>(buf, tw);
    const T *gs = (const T *)(sb + St::gq);
    const R *ls = (const R *)(sb + St::lr);
    const R *q0s = (const R *)(sb + St::r0), *q1s = (const R *)(sb + St::r1);
    const long long gbase = (long long)v * d.Ns + row0 * NX;
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, m = e % L;
      const C zc = cmul(buf[digit_rev<L>(m) * LD + r], cconj(pw[m]));
      R h0 = zc.x, h1 = -zc.y;
      if ((m + par[r]) & 1) h0 = -h0;
      if ((m + L + par[r]) & 1) h1 = -h1;
      const int i0 = r * NX + m, i1 = i0 + L;
      const double g0 = gs[i0], g1 = gs[i1];
      const R r0 = (R)((double)h0 + (double)ls[i0] - g0);
      const R r1 = (R)((double)h1 + (double)ls[i1] - g1);
      res[gbase + i0] = r0;
      res[gbase + i1] = r1;
      a_ss += (double)r0 * r0 + (double)r1 * r1;
      if (dots) {
        const double t10 = (double)r0 - q0s[i0], t20 = (double)r0 - q1s[i0];
        const double t11 = (double)r1 - q0s[i1], t21 = (double)r1 - q1s[i1];
        a0 += r0 * t10 + r1 * t11;
        a1 += r0 * t20 + r1 * t21;
        a2 += t10 * t10 + t11 * t11;
        a3 += t10 * t20 + t11 * t21;
        a4 += t20 * t20 + t21 * t21;
      }
    }
    if (__syncthreads_or(failed)) {  // buf, par and this stage are free again
      stop = it;
      break;
    }
  }
  if (stop >= 0) {  // flag the solve, wait (bounded) for the copies in flight, give up
    if (threadIdx.x == 0) atomicExch(&d.ctl->err, 1);
    const int st = stop & 1;
    mbar_wait(&bar[st], ((phase >> st) & 1) ^ 1);
    if (stop + 1 < count) mbar_wait(&bar[st ^ 1], (phase >> (st ^ 1)) & 1);
    return;
  }
  {
    double q[6] = {a_ss, a0, a1, a2, a3, a4};
    block_sums<6>(q, red6);
    if (threadIdx.x == 0) {
      sums[0] += q[0];
      if (dots)
        for (int k = 0; k < 5; ++k) sums[1 + 5 * cur_v + k] += q[1 + k];
    }
  }
  __syncthreads();
  double *part = d.partials + (size_t)cta * kPartials;
  for (int k = threadIdx.x; k < kPartials; k += kThreads) part[k] = sums[k];
}

// ------------------------------------------------- FX with bulk staging
// The iteration's FX (closure + forward x transform) with t, u and c_ref
// staged by the bulk copy engine: a tile's PC rows of one site are one
// contiguous block of each array, brought into shared memory while the
// previous tile is transformed (two stages, one mbarrier each).
template <typename P, int L, int PC>
struct FxStage {
  static constexpr int NX = 2 * L;
  static constexpr size_t t = 0;
  static constexpr size_t u = t + (size_t)PC * NX * sizeof(typename P::T);
  static constexpr size_t cref = u + (size_t)PC * NX * sizeof(typename P::R);
  static constexpr size_t bytes = cref + (size_t)PC * NX * sizeof(typename P::R);
};
#if R3D_CT_FP64
size_t ct_smem_fxb(int L, int PC, size_t csz, size_t rsz, size_t tsz) {
  const size_t buf = ((csz * (size_t)L * (PC + 1) + 127) / 128) * 128;
  return buf + 2 * (size_t)PC * 2 * L * (tsz + 2 * rsz);
}
#endif

template <typename P, int L, int PC>
__global__ void __launch_bounds__(kThreads, 1)
    k_fx_bulk(Batch b, int per) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  using St = FxStage<P, L, PC>;
  constexpr int LD = PC + 1, NX = 2 * L;
  constexpr size_t BUF = ((sizeof(C) * (size_t)L * LD + 127) / 128) * 128;
  extern __shared__ __align__(128) char smem[];
  C *buf = (C *)smem;
  __shared__ __align__(8) uint64_t bar[2];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int ny = d.ny;
  const int tps = (d.ny * d.nz) / PC;
  const int ntile = d.n * tps;
  const int first = cta * per;
  const int count = min(per, ntile - first);
  if (count <= 0) return;
  const bool has_cref = d.cref != nullptr;
  const C *pw = (const C *)d.pwx, *tw = (const C *)d.twx;
  const uint32_t tbytes = PC * NX * sizeof(T), rbytes = PC * NX * sizeof(R);
  const uint32_t stage_tx = tbytes + rbytes + (has_cref ? rbytes : 0);
  const Desc *dp = &d;
  char *const stages = smem + BUF;
  uint64_t *const bars = bar;
  auto issue = [=](int tile, int st) {  // thread 0: the copies of one tile
    const int v = tile / tps;
    const long long base = (long long)v * dp->Ns + (long long)(tile % tps) * PC * NX;
    char *sb = stages + st * St::bytes;
    uint64_t *br = bars + st;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(br, stage_tx);
    bulk_g2s(sb + St::t, (const T *)dp->t + base, tbytes, br);
    bulk_g2s(sb + St::u, (const R *)dp->u + base, rbytes, br);
    if (has_cref) bulk_g2s(sb + St::cref, (const R *)dp->cref + base, rbytes, br);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) issue(first, 0);
  uint32_t phase = 0;  // bit st: parity of the next wait on stage st
  bool failed = false;
  int stop = -1;
  for (int it = 0; it < count; ++it) {
    const int tile = first + it, st = it & 1;
    const int v = tile / tps;
    const long long row0 = (long long)(tile % tps) * PC;
    if (threadIdx.x == 0 && it + 1 < count) issue(tile + 1, st ^ 1);
    // parity (y + z) & 1 of row row0 + r in registers (no shared array and
    // no barrier): y0 and z0 of the tile's first row, y wrapping into the
    // next z-plane at most once (the planner keeps PC <= ny)
    const int y0 = (int)(row0 % ny), pz0 = (int)((y0 + row0 / ny) & 1);
    if (!mbar_wait(&bar[st], (phase >> st) & 1, d.wait_polls)) failed = true;
    phase ^= 1u << st;
    const char *sb = smem + BUF + st * St::bytes;
    const T *ts = (const T *)(sb + St::t);
    const R *us = (const R *)(sb + St::u), *cs = (const R *)(sb + St::cref);
    T *gqg = (T *)d.gq + (long long)v * d.Ns + row0 * NX;
#pragma unroll 4
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, m = e % L;
      const int i0 = r * NX + m, i1 = i0 + L;
      // trm1mt on the short-range parts (calculate_cuda.cu:18-24)
      const double t0 = ts[i0], t1 = ts[i1];
      const double g0 = closure_g<double>(d.clos, d.pse_n, -(double)us[i0] + t0);
      const double g1 = closure_g<double>(d.clos, d.pse_n, -(double)us[i1] + t1);
      gqg[i0] = g0;
      gqg[i1] = g1;
      double c0 = g0 - 1.0 - t0, c1 = g1 - 1.0 - t1;
      if (has_cref) {
        c0 -= (double)cs[i0];
        c1 -= (double)cs[i1];
      }
      R f0 = (R)c0, f1 = (R)c1;
      const int pr = (pz0 + r + (y0 + r >= ny ? 1 - ny : 0)) & 1;
      if ((m + pr) & 1) f0 = -f0;
      if ((m + L + pr) & 1) f1 = -f1;
      buf[digit_rev<L>(m) * LD + r] = cmul(C{f0, -f1}, pw[m]);
    }
    __syncthreads();
    ct_fft_dit<L, PC, LD, -1>(buf, tw);
    C *w = (C *)d.w + (long long)v * d.Nhs + row0 * L;
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, p = e % L;
      w[(long long)r * L + p] = buf[p * LD + r];
    }
    if (__syncthreads_or(failed)) {  // buf, par and this stage are free again
      stop = it;
      break;
    }
  }
  if (stop >= 0) {  // flag the solve, wait (bounded) for the copies in flight, give up
    if (threadIdx.x == 0) atomicExch(&d.ctl->err, 1);
    const int st = stop & 1;
    mbar_wait(&bar[st], ((phase >> st) & 1) ^ 1);
    if (stop + 1 < count) mbar_wait(&bar[st ^ 1], (phase >> (st ^ 1)) & 1);
  }
}

// -------------------------------------------- AN2 mix fused into FX
// The mixed path's AN2 update of t (anderson_cuda.cu:1-22, with the t slots
// as FP32 differences of successive t, as k_mix_an2) fused with the next
// evaluation's FX: t, the residual and the four history rows of a tile are
// staged by the bulk copy engine together with u and c_ref; each element's
// new t is formed, stored with its history entries, and goes straight into
// the closure and the forward x transform.  Against the separate mix and FX
// kernels this reads t once instead of twice and saves a launch.  The mix
// requested by the previous iteration's reduce (mix_flag) is applied; the
// first evaluation of a solve (mix_flag 0) is a plain FX.
template <typename P, int L, int PC>
struct MfxStage {
  static constexpr int NX = 2 * L;
  static constexpr size_t t = 0;  // FP64
  static constexpr size_t u = t + (size_t)PC * NX * 8;
  static constexpr size_t cref = u + (size_t)PC * NX * 4;
  static constexpr size_t res = cref + (size_t)PC * NX * 4;
  static constexpr size_t dn = res + (size_t)PC * NX * 4;   // newest t difference slot
  static constexpr size_t dl = dn + (size_t)PC * NX * 4;    // the other one
  static constexpr size_t r0 = dl + (size_t)PC * NX * 4;    // residual slots 0, 1
  static constexpr size_t r1 = r0 + (size_t)PC * NX * 4;
  static constexpr size_t bytes = r1 + (size_t)PC * NX * 4;
};
#if R3D_CT_FP64
size_t ct_smem_mfx(int L, int PC) {
  const size_t buf = ((8 * (size_t)L * (PC + 1) + 127) / 128) * 128;
  return buf + 2 * (size_t)PC * 2 * L * (8 + 7 * 4);
}
#endif

#if !R3D_CT_FP64
// two resident CTAs (three, at 80 registers, spilled and ran 30 % slower at
// rows of 96 reals)
template <int L, int PC>
__global__ void __launch_bounds__(kThreads, 2)
    k_mfx_bulk(Batch b, int per, int allow_mix) {
  using P = PMix;
  using R = float;
  using C = float2;
  using St = MfxStage<P, L, PC>;
  constexpr int LD = PC + 1, NX = 2 * L;
  constexpr size_t BUF = ((sizeof(C) * (size_t)L * LD + 127) / 128) * 128;
  extern __shared__ __align__(128) char smem[];
  C *buf = (C *)smem;
  __shared__ __align__(8) uint64_t bar[2];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  const Ctl *ctl = d.ctl;
  if (ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int ny = d.ny;
  const int tps = (d.ny * d.nz) / PC;
  const int ntile = d.n * tps;
  const int first = cta * per;
  const int count = min(per, ntile - first);
  if (count <= 0) return;
  const bool mix = allow_mix && ctl->mix_flag != 0;
  const bool picard = ctl->coef[2] < 0;
  const long long niv = (long long)d.n * d.Ns;
  const long long boff = (long long)ctl->coef[3] * niv, noff = niv - boff;
  const double s1 = ctl->coef[0], s2 = ctl->coef[1], mm = d.m;
  const bool old0 = boff == 0;  // slot 0 holds the older entry
  const bool has_cref = d.cref != nullptr;
  const C *pw = (const C *)d.pwx, *tw = (const C *)d.twx;
  const uint32_t tbytes = PC * NX * 8, rbytes = PC * NX * 4;
  const uint32_t stage_tx = tbytes + rbytes + (has_cref ? rbytes : 0) +
                            (mix ? (picard ? 1 : 5) * rbytes : 0);
  const Desc *dp = &d;
  char *const stages = smem + BUF;
  uint64_t *const bars = bar;
  auto issue = [=](int tile, int st) {  // thread 0: the copies of one tile
    const int v = tile / tps;
    const long long base = (long long)v * dp->Ns + (long long)(tile % tps) * PC * NX;
    char *sb = stages + st * St::bytes;
    uint64_t *br = bars + st;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(br, stage_tx);
    bulk_g2s(sb + St::t, (const double *)dp->t + base, tbytes, br);
    bulk_g2s(sb + St::u, (const R *)dp->u + base, rbytes, br);
    if (has_cref) bulk_g2s(sb + St::cref, (const R *)dp->cref + base, rbytes, br);
    if (mix) {
      bulk_g2s(sb + St::res, (const R *)dp->res + base, rbytes, br);
      if (!picard) {
        bulk_g2s(sb + St::dn, (const R *)dp->hist_a + noff + base, rbytes, br);
        bulk_g2s(sb + St::dl, (const R *)dp->hist_a + boff + base, rbytes, br);
        bulk_g2s(sb + St::r0, (const R *)dp->hist_b + base, rbytes, br);
        bulk_g2s(sb + St::r1, (const R *)dp->hist_b + niv + base, rbytes, br);
      }
    }
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) issue(first, 0);
  uint32_t phase = 0;
  bool failed = false;
  int stop = -1;
  for (int it = 0; it < count; ++it) {
    const int tile = first + it, st = it & 1;
    const int v = tile / tps;
    const long long row0 = (long long)(tile % tps) * PC;
    if (threadIdx.x == 0 && it + 1 < count) issue(tile + 1, st ^ 1);
    // parity (y + z) & 1 of row row0 + r in registers (no shared array and
    // no barrier): y0 and z0 of the tile's first row, y wrapping into the
    // next z-plane at most once (the planner keeps PC <= ny)
    const int y0 = (int)(row0 % ny), pz0 = (int)((y0 + row0 / ny) & 1);
    if (!mbar_wait(&bar[st], (phase >> st) & 1, d.wait_polls)) failed = true;
    phase ^= 1u << st;
    const char *sb = smem + BUF + st * St::bytes;
    const double *ts = (const double *)(sb + St::t);
    const R *us = (const R *)(sb + St::u), *cs = (const R *)(sb + St::cref);
    const R *rs = (const R *)(sb + St::res), *dns = (const R *)(sb + St::dn),
            *dls = (const R *)(sb + St::dl), *r0s = (const R *)(sb + St::r0),
            *r1s = (const R *)(sb + St::r1);
    const long long gbase = (long long)v * d.Ns + row0 * NX;
    double *tg = (double *)d.t + gbase;
    R *ddg = (R *)d.hist_a + boff + gbase, *rpg = (R *)d.hist_b + boff + gbase;
    double *gqg = (double *)d.gq + gbase;
#pragma unroll 2
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, m = e % L;
      double tv[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = r * NX + m + h * L;
        double tt = ts[i];
        if (mix) {
          const double rr = rs[i];
          double tn;
          if (picard) {  // newdt0: t_{k+1} = t_k + R_k
            tn = tt + rr;
          } else {  // newdt
            const double dnew = dns[i], dold = (double)dls[i] + dnew;
            const double e0 = old0 ? dold : dnew, e1 = old0 ? dnew : dold;
            const double rp0 = r0s[i], rp1 = r1s[i];
            const double uu = tt + s1 * e0 + s2 * e1;
            const double vv = tt + rr + s1 * (e0 + rp0 - rr) + s2 * (e1 + rp1 - rr);
            tn = uu + mm * (vv - uu);
          }
          ddg[i] = (R)(tt - tn);
          rpg[i] = (R)rr;
          tg[i] = tn;
          tt = tn;
        }
        tv[h] = tt;
      }
      // trm1mt on the short-range parts (calculate_cuda.cu:18-24)
      const int i0 = r * NX + m, i1 = i0 + L;
      const double g0 = closure_g<double>(d.clos, d.pse_n, -(double)us[i0] + tv[0]);
      const double g1 = closure_g<double>(d.clos, d.pse_n, -(double)us[i1] + tv[1]);
      gqg[i0] = g0;
      gqg[i1] = g1;
      double c0 = g0 - 1.0 - tv[0], c1 = g1 - 1.0 - tv[1];
      if (has_cref) {
        c0 -= (double)cs[i0];
        c1 -= (double)cs[i1];
      }
      R f0 = (R)c0, f1 = (R)c1;
      const int pr = (pz0 + r + (y0 + r >= ny ? 1 - ny : 0)) & 1;
      if ((m + pr) & 1) f0 = -f0;
      if ((m + L + pr) & 1) f1 = -f1;
      buf[digit_rev<L>(m) * LD + r] = cmul(C{f0, -f1}, pw[m]);
    }
    __syncthreads();
    ct_fft_dit<L, PC, LD, -1>(buf, tw);
    C *w = (C *)d.w + (long long)v * d.Nhs + row0 * L;
#pragma unroll
    for (int e = threadIdx.x; e < PC * L; e += kThreads) {
      const int r = e / L, p = e % L;
      w[(long long)r * L + p] = buf[p * LD + r];
    }
    if (__syncthreads_or(failed)) {  // buf, par and this stage are free again
      stop = it;
      break;
    }
  }
  if (stop >= 0) {  // flag the solve, wait (bounded) for the copies in flight, give up
    if (threadIdx.x == 0) atomicExch(&d.ctl->err, 1);
    const int st = stop & 1;
    mbar_wait(&bar[st], ((phase >> st) & 1) ^ 1);
    if (stop + 1 < count) mbar_wait(&bar[st ^ 1], (phase >> (st ^ 1)) & 1);
  }
}
#endif

// ------------------------------------------------------- warp tiles
// The iteration's x passes with one tile of PCW rows per warp: each warp
// loads, transforms (warp-synchronous radix stages) and stores its own tile,
// so no warp waits at a CTA barrier and the warps of an SM overlap the
// memory phases of some tiles with the transforms of others.  CTAs are
// persistent; the warps of a solve's CTAs stride over its tiles.
constexpr int kWarps = kThreads / 32;

#if R3D_CT_FP64
size_t ct_smem_warp(int L, int PCW, size_t csz) {
  return (size_t)kWarps * L * (PCW + 1) * csz;
}
#endif

template <typename P, int L, int PCW>
__global__ void __launch_bounds__(kThreads, sizeof(typename P::R) == 4 ? 3 : 2)
    k_fx_warp(Batch b) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  constexpr int LD = PCW + 1, NX = 2 * L;
  extern __shared__ __align__(16) char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C *buf = (C *)smem + warp * (L * LD);
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si], nct = b.prefix[si + 1] - b.prefix[si];
  const int ny = d.ny, tps = (d.ny * d.nz) / PCW, ntile = d.n * tps;
  const bool has_cref = d.cref != nullptr;
  const C *pw = (const C *)d.pwx, *tw = (const C *)d.twx;
  const T *t = (const T *)d.t;
  const R *u = (const R *)d.u, *cref = (const R *)d.cref;
  for (int tile = cta * kWarps + warp; tile < ntile; tile += nct * kWarps) {
    const int v = tile / tps;
    const long long row0 = (long long)(tile % tps) * PCW;
    const long long base0 = (long long)v * d.Ns + row0 * NX;
    const T *tt = t + base0;
    const R *ut = u + base0, *ct = cref + (has_cref ? base0 : 0);
    T *gt = (T *)d.gq + base0;
    const int pr0 = (int)((row0 % ny + row0 / ny) & 1);
    const int y0 = (int)(row0 % ny);
#pragma unroll 1
    for (int e = lane; e < PCW * L; e += 32) {
      const int r = e / L, m = e % L;
      const int i0 = r * NX + m, i1 = i0 + L;
      // parity of row0 + r: (y + z) & 1, y wrapping into the next z-plane
      const int par = (pr0 + r + ((y0 + r) >= ny ? 1 : 0) * (1 - ny)) & 1;
      // trm1mt on the short-range parts (calculate_cuda.cu:18-24)
      const double t0 = tt[i0], t1 = tt[i1];
      const double g0 = closure_g<double>(d.clos, d.pse_n, -(double)ut[i0] + t0);
      const double g1 = closure_g<double>(d.clos, d.pse_n, -(double)ut[i1] + t1);
      gt[i0] = g0;
      gt[i1] = g1;
      double c0 = g0 - 1.0 - t0, c1 = g1 - 1.0 - t1;
      if (has_cref) {
        c0 -= (double)ct[i0];
        c1 -= (double)ct[i1];
      }
      R f0 = (R)c0, f1 = (R)c1;
      if ((m + par) & 1) f0 = -f0;
      if ((m + L + par) & 1) f1 = -f1;
      buf[digit_rev<L>(m) * LD + r] = cmul(C{f0, -f1}, pw[m]);
    }
    __syncwarp();
    ct_fft_dit_warp<L, PCW, LD, -1>(buf, tw, lane);
    C *w = (C *)d.w + (long long)v * d.Nhs + row0 * L;
#pragma unroll 4
    for (int e = lane; e < PCW * L; e += 32) {
      const int r = e / L, p = e % L;
      w[(long long)r * L + p] = buf[p * LD + r];
    }
    __syncwarp();
  }
}

// IX with warp tiles: the residual, its sum of squares and AN2's theta dots
// (as k_ix_ct MODE 1).  Each warp keeps its own per-site sums (its tiles in
// order), and the CTA adds the warps' sums in warp order, so the partials do
// not depend on scheduling.
template <typename P, int L, int PCW>
__global__ void __launch_bounds__(kThreads, sizeof(typename P::R) == 4 ? 3 : 2)
    k_ix_warp(Batch b) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  constexpr int LD = PCW + 1, NX = 2 * L;
  extern __shared__ __align__(16) char smem[];
  __shared__ double wsum[kWarps][kPartials];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  C *buf = (C *)smem + warp * (L * LD);
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si], nct = b.prefix[si + 1] - b.prefix[si];
  const int ny = d.ny, tps = (d.ny * d.nz) / PCW, ntile = d.n * tps;
  const bool dots = d.mixer == MIX_AN2 && d.ctl->count_left <= 0;
  const C *pw = (const C *)d.pwx, *tw = (const C *)d.twx;
  const T *gq = (const T *)d.gq;
  const R *lr = (const R *)d.lr;
  const R *rp = (const R *)d.hist_b;
  R *res = (R *)d.res;
  const long long niv = (long long)d.n * d.Ns;
  for (int k = lane; k < kPartials; k += 32) wsum[warp][k] = 0;
  double a_ss = 0, a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0;
  int cur_v = -1;
  auto flush = [&]() {  // warp-uniform
    if (cur_v < 0) return;
    double q[6] = {a_ss, a0, a1, a2, a3, a4};
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) q[k] += __shfl_xor_sync(0xffffffffu, q[k], o);
    if (lane == 0) {
      wsum[warp][0] += q[0];
      if (dots)
#pragma unroll
        for (int k = 0; k < 5; ++k) wsum[warp][1 + 5 * cur_v + k] += q[1 + k];
    }
    a_ss = a0 = a1 = a2 = a3 = a4 = 0;
  };
  __syncwarp();
  for (int tile = cta * kWarps + warp; tile < ntile; tile += nct * kWarps) {
    const int v = tile / tps;
    const long long row0 = (long long)(tile % tps) * PCW;
    if (v != cur_v) {
      flush();
      cur_v = v;
    }
    const C *w = (const C *)d.w + (long long)v * d.Nhs + row0 * L;
#pragma unroll 4
    for (int e = lane; e < PCW * L; e += 32) {
      const int r = e / L, p = e % L;
      buf[p * LD + r] = w[e];
    }
    __syncwarp();
    ct_fft_dif_warp<L, PCW, LD, 1>(buf, tw, lane);
    const long long base0 = (long long)v * d.Ns + row0 * NX;
    const T *gt = gq + base0;
    const R *lt = lr + base0, *p0t = rp + base0, *q0t = rp + niv + base0;
    R *rt = res + base0;
    const int pr0 = (int)((row0 % ny + row0 / ny) & 1);
    const int y0 = (int)(row0 % ny);
#pragma unroll 1
    for (int e = lane; e < PCW * L; e += 32) {
      const int r = e / L, m = e % L;
      const int par = (pr0 + r + ((y0 + r) >= ny ? 1 : 0) * (1 - ny)) & 1;
      const C zc = cmul(buf[digit_rev<L>(m) * LD + r], cconj(pw[m]));
      R h0 = zc.x, h1 = -zc.y;
      if ((m + par) & 1) h0 = -h0;
      if ((m + L + par) & 1) h1 = -h1;
      const int i0 = r * NX + m, i1 = i0 + L;
      const double g0 = gt[i0], g1 = gt[i1];
      const R r0 = (R)((double)h0 + (double)lt[i0] - g0);
      const R r1 = (R)((double)h1 + (double)lt[i1] - g1);
      rt[i0] = r0;
      rt[i1] = r1;
      a_ss += (double)r0 * r0 + (double)r1 * r1;
      if (dots) {
        const double p0 = p0t[i0], p1 = p0t[i1];
        const double q0 = q0t[i0], q1 = q0t[i1];
        const double t10 = (double)r0 - p0, t20 = (double)r0 - q0;
        const double t11 = (double)r1 - p1, t21 = (double)r1 - q1;
        a0 += r0 * t10 + r1 * t11;
        a1 += r0 * t20 + r1 * t21;
        a2 += t10 * t10 + t11 * t11;
        a3 += t10 * t20 + t11 * t21;
        a4 += t20 * t20 + t21 * t21;
      }
    }
    __syncwarp();
  }
  flush();
  __syncthreads();
  double *part = d.partials + (size_t)cta * kPartials;
  for (int k = threadIdx.x; k < kPartials; k += kThreads) {
    double x = 0;
#pragma unroll
    for (int j = 0; j < kWarps; ++j) x += wsum[j][k];
    part[k] = x;
  }
}

// ------------------------------------------------------------ launchers
#define R3D_CT_LENGTHS(X) X(16) X(24) X(32) X(40) X(48) X(64) X(72) X(80) X(96) X(128) X(144) X(160) X(192) X(256) X(512)

#if R3D_CT_FP64
size_t ct_smem_x(int L, int PC, size_t csz) { return csz * (size_t)L * (PC + 1); }
size_t ct_smem_y(int L, int PC, size_t csz) { return csz * (size_t)L * PC; }
size_t ct_smem_z(int L, int PC, int n, size_t csz) { return csz * (size_t)L * PC * n; }
bool ct_length_ok(int L) {
#define R3D_OK_L(LL) if (L == LL) return true;
  R3D_CT_LENGTHS(R3D_OK_L)
#undef R3D_OK_L
  return false;
}
#endif

// Every instantiation is opted into large dynamic shared memory by
// ct_allow_smem (called at context setup: the attribute cannot be set while a
// stream is being captured into a graph).
template <typename K>
static void allow_smem(K kern) {
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
}

// Returns false when (L, PC) has no compile-time instantiation.
template <typename P>
bool ct_launch_fx(int L, int PC, Batch b, int grid, size_t smem, cudaStream_t s, int mode,
                  const void *src) {
  using R = typename P::R;
#define R3D_FX(LL)                                                                 \
  if (L == LL && PC == (sizeof(R) == 4 ? 32 : 16)) {                              \
    constexpr int PCC = sizeof(R) == 4 ? 32 : 16;                                  \
    if (mode == 0) {                                                               \
      k_fx_ct<P, LL, PCC, 0><<<grid, kThreads, smem, s>>>(b, (const R *)src);      \
    } else {                                                                       \
      k_fx_ct<P, LL, PCC, 1><<<grid, kThreads, smem, s>>>(b, nullptr);             \
    }                                                                              \
    return true;                                                                   \
  }
  R3D_CT_LENGTHS(R3D_FX)
#undef R3D_FX
  return false;
}

template <typename P>
bool ct_launch_fy(int L, int PC, Batch b, int grid, size_t smem, cudaStream_t s, int dir,
                  int check) {
#define R3D_FY_PC(LL, PCC)                                                  \
  if (L == LL && PC == PCC) {                                               \
    if (dir < 0) {                                                          \
      k_fy_ct<P, LL, PCC, -1><<<grid, kThreads, smem, s>>>(b, check);       \
    } else {                                                                \
      k_fy_ct<P, LL, PCC, 1><<<grid, kThreads, smem, s>>>(b, check);        \
    }                                                                       \
    return true;                                                            \
  }
#define R3D_FY(LL) R3D_FY_PC(LL, 8) R3D_FY_PC(LL, 16)
  R3D_CT_LENGTHS(R3D_FY)
#undef R3D_FY
#undef R3D_FY_PC
  return false;
}

template <typename P>
bool ct_launch_zoz(int L, int PC, Batch b, int grid, size_t smem, cudaStream_t s, int check) {
#define R3D_Z_PC(LL, PCC)                                                 \
  if (L == LL && PC == PCC) {                                             \
    k_zoz_ct<P, LL, PCC><<<grid, kThreads, smem, s>>>(b, check);          \
    return true;                                                          \
  }
#define R3D_Z(LL) R3D_Z_PC(LL, 4) R3D_Z_PC(LL, 8)
  R3D_CT_LENGTHS(R3D_Z)
#undef R3D_Z
#undef R3D_Z_PC
  return false;
}

template <typename P>
bool ct_launch_ix(int L, int PC, Batch b, int grid, size_t smem, cudaStream_t s, int mode,
                  void *dst, int per) {
  using R = typename P::R;
#define R3D_IX(LL)                                                                   \
  if (L == LL && PC == (sizeof(R) == 4 ? 32 : 16)) {                                \
    constexpr int PCC = sizeof(R) == 4 ? 32 : 16;                                    \
    if (mode == 0) {                                                                 \
      k_ix_ct<P, LL, PCC, 0><<<grid, kThreads, smem, s>>>(b, (R *)dst, per);         \
    } else {                                                                         \
      k_ix_ct<P, LL, PCC, 1><<<grid, kThreads, smem, s>>>(b, nullptr, per);          \
    }                                                                                \
    return true;                                                                     \
  }
  R3D_CT_LENGTHS(R3D_IX)
#undef R3D_IX
  return false;
}

template <typename P>
bool ct_launch_ixb(int L, int PC, Batch b, int grid, size_t smem, cudaStream_t s, int per) {
#define R3D_IXB(LL)                                                             \
  if (L == LL && PC == (sizeof(typename P::R) == 4 ? 8 : 4)) {                 \
    constexpr int PCC = sizeof(typename P::R) == 4 ? 8 : 4;                     \
    k_ix_bulk<P, LL, PCC><<<grid, kThreads, smem, s>>>(b, per);                \
    return true;                                                                \
  }
  R3D_CT_LENGTHS(R3D_IXB)
#undef R3D_IXB
  // half the rows per tile: long rows (two stages fit) and the occupancy variant
#define R3D_IXB_HALF(LL)                                                        \
  if (L == LL && PC == (sizeof(typename P::R) == 4 ? 4 : 2)) {                 \
    constexpr int PCC = sizeof(typename P::R) == 4 ? 4 : 2;                     \
    k_ix_bulk<P, LL, PCC><<<grid, kThreads, smem, s>>>(b, per);                \
    return true;                                                                \
  }
  R3D_CT_LENGTHS(R3D_IXB_HALF)
#undef R3D_IXB_HALF
  // two rows per tile for the longest FP32 rows (the occupancy variant there)
  if constexpr (sizeof(typename P::R) == 4) {
    if (L == 256 && PC == 2) {
      k_ix_bulk<P, 256, 2><<<grid, kThreads, smem, s>>>(b, per);
      return true;
    }
    if (L == 512 && PC == 2) {
      k_ix_bulk<P, 512, 2><<<grid, kThreads, smem, s>>>(b, per);
      return true;
    }
  }
  return false;
}

template <typename P>
bool ct_launch_fxb(int L, int PC, Batch b, int grid, size_t smem, cudaStream_t s, int per) {
#define R3D_FXB(LL)                                                             \
  if (L == LL && PC == (sizeof(typename P::R) == 4 ? 8 : 4)) {                 \
    constexpr int PCC = sizeof(typename P::R) == 4 ? 8 : 4;                     \
    k_fx_bulk<P, LL, PCC><<<grid, kThreads, smem, s>>>(b, per);                \
    return true;                                                                \
  }
  R3D_CT_LENGTHS(R3D_FXB)
#undef R3D_FXB
#define R3D_FXB_HALF(LL)                                                        \
  if (L == LL && PC == (sizeof(typename P::R) == 4 ? 4 : 2)) {                 \
    constexpr int PCC = sizeof(typename P::R) == 4 ? 4 : 2;                     \
    k_fx_bulk<P, LL, PCC><<<grid, kThreads, smem, s>>>(b, per);                \
    return true;                                                                \
  }
  R3D_FXB_HALF(256)
  R3D_FXB_HALF(512)
#undef R3D_FXB_HALF
  return false;
}

// The mix-fused FX (mixed precision; false: no kernel for the length).
// Rows per tile: 8 for rows of up to 128 reals (a tile of 4 short rows
// leaves threads idle and pays the tile's barriers for few elements), 4, and
// 2 for rows of 1024 reals.
constexpr int mfx_pc(int L) { return L >= 512 ? 2 : L <= 64 ? 8 : 4; }
template <typename P>
bool ct_launch_mfx(int L, Batch b, int grid, size_t smem, cudaStream_t s, int per,
                   int allow_mix) {
#if !R3D_CT_FP64
#define R3D_MFX(LL)                                                          \
  if (L == LL) {                                                             \
    k_mfx_bulk<LL, mfx_pc(LL)><<<grid, kThreads, smem, s>>>(b, per, allow_mix); \
    return true;                                                             \
  }
  R3D_CT_LENGTHS(R3D_MFX)
#undef R3D_MFX
#endif
  return false;
}
template <typename P>
int ct_occupancy_mfx(int L, size_t smem) {
  int nb = 0;
#if !R3D_CT_FP64
#define R3D_OMFX(LL)                                                                        \
  if (L == LL) {                                                                            \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_mfx_bulk<LL, mfx_pc(LL)>, kThreads, \
                                                  smem);                                    \
    return nb;                                                                              \
  }
  R3D_CT_LENGTHS(R3D_OMFX)
#undef R3D_OMFX
#endif
  return nb;
}
#if R3D_CT_FP64
int ct_mfx_pc(int L) { return mfx_pc(L); }
#endif

// Resident CTAs per SM of the bulk-staged FX (which = 0) or IX (1) for
// length L, PC rows per tile and `smem` dynamic bytes (0: not instantiated).
template <typename P>
int ct_occupancy_bulk(int which, int L, int PC, size_t smem) {
  int nb = 0;
#define R3D_OCC(LL, PCC)                                                              \
  if (L == LL && PC == PCC) {                                                         \
    if (which == 0)                                                                   \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_fx_bulk<P, LL, PCC>, kThreads, \
                                                    smem);                            \
    else                                                                              \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ix_bulk<P, LL, PCC>, kThreads, \
                                                    smem);                            \
    return nb;                                                                        \
  }
#define R3D_OCC_FULL(LL) R3D_OCC(LL, (sizeof(typename P::R) == 4 ? 8 : 4))
  R3D_CT_LENGTHS(R3D_OCC_FULL)
  R3D_OCC(256, (sizeof(typename P::R) == 4 ? 4 : 2))
  R3D_OCC(512, (sizeof(typename P::R) == 4 ? 4 : 2))
#undef R3D_OCC_FULL
  // the IX's half-size tiles at the other lengths
#define R3D_OCC_IXH(LL)                                                                    \
  if (which == 1 && L == LL && PC == (sizeof(typename P::R) == 4 ? 4 : 2)) {              \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(                                         \
        &nb, k_ix_bulk<P, LL, (sizeof(typename P::R) == 4 ? 4 : 2)>, kThreads, smem);      \
    return nb;                                                                             \
  }
  R3D_CT_LENGTHS(R3D_OCC_IXH)
#undef R3D_OCC_IXH
  if constexpr (sizeof(typename P::R) == 4) {
    if (which == 1 && PC == 2 && (L == 256 || L == 512)) {
      if (L == 256)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ix_bulk<P, 256, 2>, kThreads, smem);
      else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ix_bulk<P, 512, 2>, kThreads, smem);
      return nb;
    }
  }
#undef R3D_OCC
  return 0;
}

// warp-tile x passes: PCW = 4 rows per warp, 2 for rows of 256 or more
// complex points
template <typename P>
bool ct_launch_xw(int which, int L, int PCW, Batch b, int grid, size_t smem, cudaStream_t s) {
#define R3D_XW(LL, PP)                                               \
  if (L == LL && PCW == PP) {                                        \
    if (which == 0)                                                  \
      k_fx_warp<P, LL, PP><<<grid, kThreads, smem, s>>>(b);          \
    else                                                             \
      k_ix_warp<P, LL, PP><<<grid, kThreads, smem, s>>>(b);          \
    return true;                                                     \
  }
#define R3D_XW4(LL) R3D_XW(LL, 4)
  R3D_CT_LENGTHS(R3D_XW4)
  R3D_XW(256, 2)
  R3D_XW(512, 2)
#undef R3D_XW4
#undef R3D_XW
  return false;
}
template <typename P>
int ct_occupancy_xw(int which, int L, int PCW, size_t smem) {
  int nb = 0;
#define R3D_OXW(LL, PP)                                                                  \
  if (L == LL && PCW == PP) {                                                            \
    if (which == 0)                                                                      \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_fx_warp<P, LL, PP>, kThreads, smem); \
    else                                                                                 \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ix_warp<P, LL, PP>, kThreads, smem); \
    return nb;                                                                           \
  }
#define R3D_OXW4(LL) R3D_OXW(LL, 4)
  R3D_CT_LENGTHS(R3D_OXW4)
  R3D_OXW(256, 2)
  R3D_OXW(512, 2)
#undef R3D_OXW4
#undef R3D_OXW
  return 0;
}

template <typename P>
void ct_allow_smem_all() {
  using R = typename P::R;
  constexpr int PX = sizeof(R) == 4 ? 32 : 16;
#define R3D_ATTR(LL)                                                      \
  allow_smem(k_fx_ct<P, LL, PX, 0>);                                      \
  allow_smem(k_fx_ct<P, LL, PX, 1>);                                      \
  allow_smem(k_ix_ct<P, LL, PX, 0>);                                      \
  allow_smem(k_ix_ct<P, LL, PX, 1>);                                      \
  allow_smem(k_fy_ct<P, LL, 8, -1>);                                      \
  allow_smem(k_fy_ct<P, LL, 8, 1>);                                       \
  allow_smem(k_fy_ct<P, LL, 16, -1>);                                     \
  allow_smem(k_fy_ct<P, LL, 16, 1>);                                      \
  allow_smem(k_zoz_ct<P, LL, 4>);                                         \
  allow_smem(k_zoz_ct<P, LL, 8>);                                         \
  allow_smem(k_ix_bulk<P, LL, (sizeof(typename P::R) == 4 ? 8 : 4)>);      \
  allow_smem(k_ix_bulk<P, LL, (sizeof(typename P::R) == 4 ? 4 : 2)>);      \
  allow_smem(k_fx_bulk<P, LL, (sizeof(typename P::R) == 4 ? 8 : 4)>);       \
  allow_smem(k_fx_warp<P, LL, 4>);                                        \
  allow_smem(k_ix_warp<P, LL, 4>);
  R3D_CT_LENGTHS(R3D_ATTR)
#undef R3D_ATTR
  allow_smem(k_fx_bulk<P, 256, (sizeof(typename P::R) == 4 ? 4 : 2)>);
  allow_smem(k_fx_bulk<P, 512, (sizeof(typename P::R) == 4 ? 4 : 2)>);
  if constexpr (sizeof(typename P::R) == 4) {
    allow_smem(k_ix_bulk<P, 256, 2>);
    allow_smem(k_ix_bulk<P, 512, 2>);
  }
  allow_smem(k_fx_warp<P, 256, 2>);
  allow_smem(k_fx_warp<P, 512, 2>);
#if !R3D_CT_FP64
#define R3D_AMFX(LL) allow_smem(k_mfx_bulk<LL, mfx_pc(LL)>);
  R3D_CT_LENGTHS(R3D_AMFX)
#undef R3D_AMFX
#endif
  allow_smem(k_ix_warp<P, 256, 2>);
  allow_smem(k_ix_warp<P, 512, 2>);
}
template void ct_allow_smem_all<PCT>();

template bool ct_launch_fx<PCT>(int, int, Batch, int, size_t, cudaStream_t, int, const void *);
template bool ct_launch_fy<PCT>(int, int, Batch, int, size_t, cudaStream_t, int, int);
template bool ct_launch_zoz<PCT>(int, int, Batch, int, size_t, cudaStream_t, int);
template bool ct_launch_ix<PCT>(int, int, Batch, int, size_t, cudaStream_t, int, void *, int);
template bool ct_launch_ixb<PCT>(int, int, Batch, int, size_t, cudaStream_t, int);
template bool ct_launch_fxb<PCT>(int, int, Batch, int, size_t, cudaStream_t, int);
template bool ct_launch_mfx<PCT>(int, Batch, int, size_t, cudaStream_t, int, int);
template int ct_occupancy_mfx<PCT>(int, size_t);
template int ct_occupancy_bulk<PCT>(int, int, int, size_t);
template bool ct_launch_xw<PCT>(int, int, int, Batch, int, size_t, cudaStream_t);
template int ct_occupancy_xw<PCT>(int, int, int, size_t);

}  // namespace r3d
