// r3d_kernels.cu -- sm_100a kernels of the 3D-RISM solve.
//
// One iteration (the reference's RISM3D::calculate + cal_rms + AN2::calculate,
// calculate.cu:4-65, cal_rms.cu:14-26, anderson.cu:43-130) is five grid passes
// plus two tiny control kernels:
//
//   FX   closure + c_s + checkerboard + packed real->complex x transform
//   FY   y transform of the half spectrum                     (in place)
//   ZOZ  z transform, Ornstein-Zernike h_a(k) = sum_b chi_ab(|k|) c_b(k),
//        inverse z transform                                  (in place)
//   IY   inverse y transform                                  (in place)
//   IX   inverse packed x transform + g, residual R = h + 1 - g,
//        sum R^2 and the AN2 Gram dots (per-CTA partials)
//
// Long-range electrostatics and refinement.  The reference adds
// q_v beta phi_L(r) to c in r space (trm1mt) and subtracts q_v beta phi_L(k) in
// k space (mqvfk).  Here the solve runs on the short-range parts
// t_s = t - q_v beta phi_L(r) and u_s = beta u - q_v beta phi_L(r), so that
// c_s = g - 1 - t_s, and h is split around a frozen c_ref:
//   h_a = F^-1[ sum_b chi_ab F(c_s,b - c_ref,b) ] + h_ref,a
//   h_ref,a = F^-1[ sum_b chi_ab (F(c_ref,b) - q_b beta phi_L(k)) ]
// with h_ref computed in FP64 (the "refresh", which with c_ref = 0 is the
// setup's long-range term).  This is the reference's iteration exactly; in the
// mixed path the FP32 transforms only ever see the small correction
// c_s - c_ref, so their rounding noise shrinks as the solve converges instead
// of flooring the residual at ~1e-6.
//   reduce/coef (1 CTA)  RMS, convergence, mixing coefficients on the device
//   mix   AN2 or history-M Anderson update of t
//
// The transform is the reference's half-shifted one (fft3d.cu):
//   F(k) = dv sum_r f(r) e^{-i k.r},  r = (i - n/2) dr,  k = 2 pi (j - n/2 + 1/2)/L
// computed as: checkerboard (-1)^{x+y+z} on r, odd-frequency DFT per axis
// (x via a half-length packed complex FFT, y/z via a half-sample twiddle), and
// the constant per-point phase dv*C(k) is folded into phi_L(k) and chi, so the
// iteration never applies it.  All passes take a descriptor table so that one
// launch can serve many solves of different grids (batching).
#include <cuda_runtime.h>
#include <algorithm>
#include <type_traits>
#include <math.h>
#include <stdint.h>

#include "r3d_common.cuh"

namespace r3d {

// ======================================================================
// FX: forward x pass.  MODE 0: plain real input `src` ([n][N]);
// MODE 1: closure fused (reads t, u, fr).
// ======================================================================
template <typename P, int MODE>
__global__ void __launch_bounds__(kThreads)
    k_fwd_x(Batch b, const typename P::R *src) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) char smem[];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (MODE == 1 && !solve_running<R>(d)) return;
  const int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, nx = d.nx, ny = d.ny, n = d.n, S = d.rows;
  Smem<C> sm = carve<C>(smem, hx, hx);
  splan_init(sm.tw, sm.perm, hx, d.rad_x, d.nrad_x);
  half_twiddles(sm.ptw, hx, nx);
  __syncthreads();
  SPlan<C> pl{hx, d.nrad_x, {}, sm.tw, sm.perm};
  for (int k = 0; k < d.nrad_x; ++k) pl.rad[k] = d.rad_x[k];

  const long long row0 = (long long)tile * S;
  const T *t = (const T *)d.t;
  const R *u = (const R *)d.u, *cref = (const R *)d.cref;
  const int total = n * S * hx;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    int m = e % hx, sr = e / hx, r = sr % S, v = sr / S;
    long long row = row0 + r;
    int y = (int)(row % ny), z = (int)(row / ny);
    long long base = (long long)v * d.Ns + row * nx;
    R f0, f1;
    if (MODE == 0) {
      f0 = src[base + m];
      f1 = src[base + m + hx];
    } else {
      // trm1mt on the short-range parts: c_s = g - 1 - t_s (closure in the
      // state precision, rounded once to the grid type)
      double t0 = t[base + m], t1 = t[base + m + hx];
      double g0 = closure_g<double>(d.clos, d.pse_n, -(double)u[base + m] + t0);
      double g1 = closure_g<double>(d.clos, d.pse_n, -(double)u[base + m + hx] + t1);
      ((T *)d.gq)[base + m] = g0;
      ((T *)d.gq)[base + m + hx] = g1;
      double c0 = g0 - 1.0 - t0, c1 = g1 - 1.0 - t1;
      if (cref) {
        c0 -= (double)cref[base + m];
        c1 -= (double)cref[base + m + hx];
      }
      f0 = (R)c0;
      f1 = (R)c1;
    }
    if ((m + y + z) & 1) f0 = -f0;
    if ((m + hx + y + z) & 1) f1 = -f1;
    C zc = cmul(C{f0, -f1}, sm.ptw[m]);
    sm.buf[sr * hx + sm.perm[m]] = zc;
  }
  __syncthreads();
  fft_dit<-1>(sm.buf, n * S, 1 << 30, 0, hx, 1, pl);
  C *w = (C *)d.w;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    int p = e % hx, sr = e / hx, r = sr % S, v = sr / S;
    w[(long long)v * d.Nhs + (row0 + r) * hx + p] = sm.buf[sr * hx + p];
  }
}

// ======================================================================
// FY / IY: y transform of the half spectrum, tile = (site, z, x-columns).
// ======================================================================
template <typename P, int DIR>
__global__ void __launch_bounds__(kThreads)
    k_fft_y(Batch b, int check_status) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) char smem[];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (check_status && !solve_running<R>(d)) return;
  int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, ny = d.ny, nz = d.nz, PC = d.ycols;
  const int ptiles = hx / PC;
  const int pt = tile % ptiles;
  tile /= ptiles;
  const int z = tile % nz, v = tile / nz;
  Smem<C> sm = carve<C>(smem, ny, ny);
  splan_init(sm.tw, sm.perm, ny, d.rad_y, d.nrad_y);
  half_twiddles(sm.ptw, ny, ny);
  __syncthreads();
  SPlan<C> pl{ny, d.nrad_y, {}, sm.tw, sm.perm};
  for (int k = 0; k < d.nrad_y; ++k) pl.rad[k] = d.rad_y[k];
  C *w = (C *)d.w + (long long)v * d.Nhs + (long long)z * ny * hx + pt * PC;
  const int total = ny * PC;
  if (DIR < 0) {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, y = e / PC;
      sm.buf[sm.perm[y] * PC + p] = cmul(w[(long long)y * hx + p], sm.ptw[y]);
    }
    __syncthreads();
    fft_dit<-1>(sm.buf, PC, 1 << 30, 0, 1, PC, pl);
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, y = e / PC;
      w[(long long)y * hx + p] = sm.buf[y * PC + p];
    }
  } else {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, y = e / PC;
      sm.buf[y * PC + p] = w[(long long)y * hx + p];
    }
    __syncthreads();
    fft_dif<1>(sm.buf, PC, 1 << 30, 0, 1, PC, pl);
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, y = e / PC;
      w[(long long)y * hx + p] = cmul(sm.buf[sm.perm[y] * PC + p], cconj(sm.ptw[y]));
    }
  }
}

// ======================================================================
// ZOZ: tile = (y, x-columns), all sites.  MODE 0: forward z only;
// MODE 1: inverse z only; MODE 2: forward z + mqvfk + OZ + inverse z.
// ======================================================================
template <typename R, int NS>
__device__ __forceinline__ void oz_point(typename Cx<R>::T *buf, int n, int stride,
                                         const R *chi, const double2 *fk,
                                         const double *qv) {
  using C = typename Cx<R>::T;
  constexpr int M = NS > 0 ? NS : kMaxSites;
  const int nn = NS > 0 ? NS : n;
  C c[M];
#pragma unroll
  for (int bb = 0; bb < M; ++bb)
    if (bb < nn) c[bb] = buf[bb * stride];
  if (fk) {  // mqvfk (refresh pipeline only)
    const double2 f = *fk;
#pragma unroll
    for (int bb = 0; bb < M; ++bb)
      if (bb < nn) {
        c[bb].x -= (R)(qv[bb] * f.x);
        c[bb].y -= (R)(qv[bb] * f.y);
      }
  }
#pragma unroll
  for (int a = 0; a < M; ++a) {
    if (a < nn) {
      R hr = 0, hi = 0;  // oz: h_a = sum_b chi[a][b] c_b
#pragma unroll
      for (int bb = 0; bb < M; ++bb) {
        if (bb < nn) {
          R x = chi[a * nn + bb];
          hr += c[bb].x * x;
          hi += c[bb].y * x;
        }
      }
      buf[a * stride] = C{hr, hi};
    }
  }
}

template <typename P, int MODE>
__global__ void __launch_bounds__(kThreads)
    k_zoz(Batch b, int check_status) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) char smem[];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (check_status && !solve_running<R>(d)) return;
  int tile = blockIdx.x - b.prefix[si];
  const int hx = d.hx, ny = d.ny, nz = d.nz, n = d.n, PC = d.zcols;
  const int ptiles = hx / PC;
  const int pt = tile % ptiles, y = tile / ptiles;
  Smem<C> sm = carve<C>(smem, nz, nz);
  splan_init(sm.tw, sm.perm, nz, d.rad_z, d.nrad_z);
  half_twiddles(sm.ptw, nz, nz);
  __syncthreads();
  SPlan<C> pl{nz, d.nrad_z, {}, sm.tw, sm.perm};
  for (int k = 0; k < d.nrad_z; ++k) pl.rad[k] = d.rad_z[k];
  const long long zs = (long long)ny * hx;  // z stride in the half spectrum
  C *w = (C *)d.w + (long long)y * hx + pt * PC;
  const int total = n * nz * PC;
  const int sA = nz * PC;
  if (MODE != 1) {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, vz = e / PC, z = vz % nz, v = vz / nz;
      sm.buf[(v * nz + sm.perm[z]) * PC + p] =
          cmul(w[(long long)v * d.Nhs + z * zs + p], sm.ptw[z]);
    }
    __syncthreads();
    fft_dit<-1>(sm.buf, n * PC, PC, sA, 1, PC, pl);
  } else {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, vz = e / PC, z = vz % nz, v = vz / nz;
      sm.buf[(v * nz + z) * PC + p] = w[(long long)v * d.Nhs + z * zs + p];
    }
    __syncthreads();
  }
  if (MODE == 0) {
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % PC, vz = e / PC, z = vz % nz, v = vz / nz;
      w[(long long)v * d.Nhs + z * zs + p] = sm.buf[(v * nz + z) * PC + p];
    }
    return;
  }
  if (MODE == 2) {
    const uint32_t *kidx = d.kidx + (long long)y * hx + pt * PC;
    const double2 *fk = d.fk ? (const double2 *)d.fk + (long long)y * hx + pt * PC : nullptr;
    const R *chi = (const R *)d.chi;
    const int nn = n * n;
    for (int e = threadIdx.x; e < nz * PC; e += blockDim.x) {
      int p = e % PC, z = e / PC;
      const R *ch = chi + (size_t)kidx[z * zs + p] * d.chis;
      const double2 *f = fk ? fk + z * zs + p : nullptr;
      C *bp = sm.buf + z * PC + p;
      switch (n) {
        case 1: oz_point<R, 1>(bp, n, sA, ch, f, d.qv); break;
        case 2: oz_point<R, 2>(bp, n, sA, ch, f, d.qv); break;
        case 3: oz_point<R, 3>(bp, n, sA, ch, f, d.qv); break;
        case 4: oz_point<R, 4>(bp, n, sA, ch, f, d.qv); break;
        default: oz_point<R, 0>(bp, n, sA, ch, f, d.qv); break;
      }
    }
    __syncthreads();
  }
  fft_dif<1>(sm.buf, n * PC, PC, sA, 1, PC, pl);
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    int p = e % PC, vz = e / PC, z = vz % nz, v = vz / nz;
    w[(long long)v * d.Nhs + z * zs + p] =
        cmul(sm.buf[(v * nz + sm.perm[z]) * PC + p], cconj(sm.ptw[z]));
  }
}

// ======================================================================
// IX: inverse x pass.  MODE 0: plain real output `dst` ([n][N]);
// MODE 1: g, residual R = h + 1 - g (calculate_cuda.cu:54-60), partial sums
// of R^2 (cal_rms.cu) and, when AN2 is past its Picard warm-up, the five
// theta dots per site (anderson_cuda.cu:25-67).  A CTA handles `per` tiles.
// ======================================================================
template <typename P, int MODE>
__global__ void __launch_bounds__(kThreads)
    k_inv_x(Batch b, typename P::R *dst, int per) {
  using R = typename P::R;
  using T = typename P::T;
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) char smem[];
  __shared__ double red[8 * (kThreads / 32)];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (MODE == 1 && !solve_running<R>(d)) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int hx = d.hx, nx = d.nx, ny = d.ny, n = d.n, S = d.rows;
  Smem<C> sm = carve<C>(smem, hx, hx);
  splan_init(sm.tw, sm.perm, hx, d.rad_x, d.nrad_x);
  half_twiddles(sm.ptw, hx, nx);
  __syncthreads();
  SPlan<C> pl{hx, d.nrad_x, {}, sm.tw, sm.perm};
  for (int k = 0; k < d.nrad_x; ++k) pl.rad[k] = d.rad_x[k];

  const bool dots = MODE == 1 && d.mixer == MIX_AN2 && d.ctl->count_left <= 0;
  const T *gq = (const T *)d.gq;
  const R *lr = (const R *)d.lr;
  R *res = (R *)d.res;
  const R *rp = (const R *)d.hist_b;
  const long long niv = (long long)n * d.Ns;
  double acc_ss = 0;
  double acc[kMaxSites][5];
  for (int v = 0; v < kMaxSites; ++v)
    for (int k = 0; k < 5; ++k) acc[v][k] = 0;

  const C *w = (const C *)d.w;
  const int ntile = d.tiles_x;
  for (int it = 0; it < per; ++it) {
    const int tile = cta * per + it;
    if (tile >= ntile) break;
    const long long row0 = (long long)tile * S;
    const int total = n * S * hx;
    __syncthreads();
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int p = e % hx, sr = e / hx, r = sr % S, v = sr / S;
      sm.buf[sr * hx + p] = w[(long long)v * d.Nhs + (row0 + r) * hx + p];
    }
    __syncthreads();
    fft_dif<1>(sm.buf, n * S, 1 << 30, 0, hx, 1, pl);
    for (int v = 0; v < n; ++v) {
      const R q = (R)d.qv[v];
      (void)q;
      double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
      for (int e = threadIdx.x; e < S * hx; e += blockDim.x) {
        int m = e % hx, r = e / hx, sr = v * S + r;
        long long row = row0 + r;
        int y = (int)(row % ny), z = (int)(row / ny);
        C zc = cmul(sm.buf[sr * hx + sm.perm[m]], cconj(sm.ptw[m]));
        R h0 = zc.x, h1 = -zc.y;
        if ((m + y + z) & 1) h0 = -h0;
        if ((m + hx + y + z) & 1) h1 = -h1;
        long long base = (long long)v * d.Ns + row * nx;
        if (MODE == 0) {
          dst[base + m] = h0;
          dst[base + m + hx] = h1;
        } else {
          const double g0 = gq[base + m], g1 = gq[base + m + hx];
          // tr: R = h + 1 - g with h = h_s - L, evaluated in FP64 and rounded
          // once (R is small near convergence, g need not be)
          R r0 = (R)((double)h0 + (double)lr[base + m] - g0);
          R r1 = (R)((double)h1 + (double)lr[base + m + hx] - g1);
          res[base + m] = r0;
          res[base + m + hx] = r1;
          acc_ss += (double)r0 * r0 + (double)r1 * r1;
          if (dots) {
            R a0 = rp[base + m], a1 = rp[base + m + hx];
            R b0 = rp[niv + base + m], b1 = rp[niv + base + m + hx];
            double t10 = (double)r0 - a0, t20 = (double)r0 - b0;
            double t11 = (double)r1 - a1, t21 = (double)r1 - b1;
            s0 += r0 * t10 + r1 * t11;
            s1 += r0 * t20 + r1 * t21;
            s2 += t10 * t10 + t11 * t11;
            s3 += t10 * t20 + t11 * t21;
            s4 += t20 * t20 + t21 * t21;
          }
        }
      }
      if (dots) {
        acc[v][0] += s0;
        acc[v][1] += s1;
        acc[v][2] += s2;
        acc[v][3] += s3;
        acc[v][4] += s4;
      }
    }
  }
  if (MODE == 0) return;
  double *part = d.partials + (size_t)cta * kPartials;
  {
    double q[6] = {acc_ss, acc[0][0], acc[0][1], acc[0][2], acc[0][3], acc[0][4]};
    block_sums<6>(q, red);
    if (threadIdx.x == 0) {
      part[0] = q[0];
      if (dots)
        for (int k = 0; k < 5; ++k) part[1 + k] = q[1 + k];
    }
  }
  if (dots) {
    for (int v = 1; v < n; ++v) {
      double q[5] = {acc[v][0], acc[v][1], acc[v][2], acc[v][3], acc[v][4]};
      block_sums<5>(q, red);
      if (threadIdx.x == 0)
        for (int k = 0; k < 5; ++k) part[1 + 5 * v + k] = q[k];
    }
  }
}

// ======================================================================
// Control kernels (1 CTA per solve).
// ======================================================================
// leg (anderson.cu:105-130): 2x2 Gaussian elimination, no pivoting.
__device__ void leg2(double *a, double *x, double *bb) {
  double p = a[0];
  a[1] /= p;
  double r = bb[0] /= p;
  double q = a[2];
  a[3] -= q * a[1];
  bb[1] -= q * r;
  x[1] = bb[1] / a[3];
  x[0] = bb[0] - a[1] * x[1];
}

// Dense solve with partial pivoting (ANM); returns false when singular.
__device__ bool solve_pp(double *A, double *x, int m) {
  for (int k = 0; k < m; ++k) {
    int piv = k;
    double best = fabs(A[k * m + k]);
    for (int i = k + 1; i < m; ++i)
      if (fabs(A[i * m + k]) > best) {
        best = fabs(A[i * m + k]);
        piv = i;
      }
    if (!(best > 1e-300)) return false;
    if (piv != k) {
      for (int j = 0; j < m; ++j) {
        double tt = A[k * m + j];
        A[k * m + j] = A[piv * m + j];
        A[piv * m + j] = tt;
      }
      double tt = x[k];
      x[k] = x[piv];
      x[piv] = tt;
    }
    for (int i = k + 1; i < m; ++i) {
      double f = A[i * m + k] / A[k * m + k];
      for (int j = k; j < m; ++j) A[i * m + j] -= f * A[k * m + j];
      x[i] -= f * x[k];
    }
  }
  for (int k = m - 1; k >= 0; --k) {
    double acc = x[k];
    for (int j = k + 1; j < m; ++j) acc -= A[k * m + j] * x[j];
    x[k] = acc / A[k * m + k];
  }
  for (int k = 0; k < m; ++k)
    if (!isfinite(x[k])) return false;
  return true;
}

// Reduce the IX partials of every solve: RMS and convergence/divergence
// (iterate.cu:48-59, cal_rms.cu:14-26).  Grid = one CTA per solve.
// AN2 coefficients (anderson.cu:54-73) are computed here too, so that the
// mix kernel only reads them.  `force` = mix regardless of convergence
// (the explicit anderson() API call).
__global__ void __launch_bounds__(kThreads)
    k_reduce(const Desc *descs, const int *ix_ctas, int mode_force) {
  __shared__ double red[8 * (kThreads / 32)];
  __shared__ double sums[kPartials];
  const Desc &d = descs[blockIdx.x];
  Ctl *c = d.ctl;
  if (c->status != RUNNING && mode_force == 0) {
    if (threadIdx.x == 0) c->mix_flag = 0;
    return;
  }
  const int nct = ix_ctas[blockIdx.x];
  const bool dots = d.mixer == MIX_AN2 && c->count_left <= 0;
  const int np = dots ? 1 + 5 * d.n : 1;
  // eight columns at a time: every thread sums its rows (i, i + blockDim,
  // ...) of each column with all the chunk's loads in flight, then one
  // block reduction per chunk -- the same additions in the same order as a
  // column at a time
  for (int k0 = 0; k0 < np; k0 += 8) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = 0;
    for (int i = threadIdx.x; i < nct; i += blockDim.x) {
      const double *row = d.partials + (size_t)i * kPartials + k0;
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k0 + k < np) v[k] += row[k];
    }
    block_sums<8>(v, red);
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k0 + k < np) sums[k0 + k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  if (mode_force == 2) {  // calculate() only: record the rms, decide nothing
    c->ss = sums[0];
    c->rms = sqrt(sums[0] / ((double)d.N * d.n));
    c->step += 1;
    return;
  }
  if (mode_force == 0) {
    c->ss = sums[0];
    c->rms = sqrt(sums[0] / ((double)d.N * d.n));
    c->step += 1;
    if (c->step <= c->maxstep) d.rmslog[c->step - 1] = c->rms;
    if (!isfinite(c->rms) || c->err) {  // err: a kernel's bounded wait ran out
      c->status = DIVERGED;
      c->mix_flag = 0;
      return;
    }
    if (c->rms <= c->tol) {
      c->status = CONVERGED;
      c->mix_flag = 0;
      return;
    }
    // The last allowed evaluation ends the solve without a mix: t stays the
    // t of that evaluation, whose g and h the results are computed from.
    if (c->step >= c->maxstep) {
      c->status = MAXSTEP;
      c->mix_flag = 0;
      return;
    }
  }
  c->mix_flag = 1;
  if (d.mixer == MIX_AN2) {
    if (c->count_left > 0) {  // newdt0 (Picard) step
      c->count_left -= 1;
      c->coef[0] = 0;
      c->coef[1] = 0;
      c->coef[2] = -1.0;  // marker: Picard
      c->coef[3] = (double)c->binary;
    } else {
      double a[4], cc[2], x[2];
      cc[0] = cc[1] = a[0] = a[1] = a[3] = 0.0;
      for (int v = 0; v < d.n; ++v) {  // cal_theta, anderson.cu:81-102
        cc[0] += sums[1 + 5 * v + 0] * d.irho[v];
        cc[1] += sums[1 + 5 * v + 1] * d.irho[v];
        a[0] += sums[1 + 5 * v + 2] * d.irho[v];
        a[1] += sums[1 + 5 * v + 3] * d.irho[v];
        a[3] += sums[1 + 5 * v + 4] * d.irho[v];
      }
      a[2] = a[1];
      leg2(a, x, cc);
      c->coef[0] = x[0] + d.mp * ((c->binary == 0) ? 0 : 1);
      c->coef[1] = x[1] + d.mp * ((c->binary == 0) ? 1 : 0);
      c->coef[2] = 1.0;
      c->coef[3] = (double)c->binary;
    }
    c->binary = (c->binary == 0) ? 1 : 0;
  }
}

// AN2 mix: newdt0 / newdt (anderson_cuda.cu:1-22), all sites in one launch.
// Each CTA owns one chunk of kMixChunk consecutive elements of the [site][x]
// arrays; every thread loads its kMixPer elements of all six streams before
// it stores anything, so each thread keeps 6 * kMixPer loads in flight.
constexpr int kMixPer = 4;
constexpr int kMixChunk = kThreads * kMixPer;

template <typename P>
__global__ void __launch_bounds__(kThreads)
    k_mix_an2(Batch b) {
  using R = typename P::R;
  using T = typename P::T;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  const Ctl *c = d.ctl;
  if (!c->mix_flag) return;
  const long long niv = (long long)d.n * d.Ns;
  const long long i0 = (long long)(blockIdx.x - b.prefix[si]) * kMixChunk + threadIdx.x;
  T *__restrict__ t = (T *)d.t;
  const R *__restrict__ r = (const R *)d.res;
  R *__restrict__ rp = (R *)d.hist_b;
  const bool picard = c->coef[2] < 0;
  const long long boff = (long long)c->coef[3] * niv;
  if (!R3D_IN(d, boff, 2 * niv)) return;  // the ping-pong slot is 0 or 1
  const double s1 = c->coef[0], s2 = c->coef[1], m = d.m;
  T tv[kMixPer];
  R rv[kMixPer];
  if constexpr (sizeof(R) < sizeof(T)) {
    // Mixed precision: the t slots hold FP32 differences of successive
    // states, D_k = t_k - t_{k+1}, written when t_{k+1} is made.  At step k
    // the newest slot (1 - binary) holds t_{k-1} - t_k and the other
    // t_{k-2} - t_{k-1}; the mix needs only t_slot - t_k, which is D_new and
    // D_old + D_new.  Slot traffic halves against FP64 copies of t.
    R *__restrict__ dd = (R *)d.hist_a;
    const long long noff = (long long)(1 - (int)c->coef[3]) * niv;
    if (picard) {  // t_{k+1} = t_k + R_k: D_k = -R_k
#pragma unroll
      for (int k = 0; k < kMixPer; ++k) {
        const long long i = i0 + k * kThreads;
        if (i < niv) {
          tv[k] = t[i];
          rv[k] = r[i];
        }
      }
#pragma unroll
      for (int k = 0; k < kMixPer; ++k) {
        const long long i = i0 + k * kThreads;
        if (i < niv) {
          dd[boff + i] = -rv[k];
          rp[boff + i] = rv[k];
          t[i] = tv[k] + (T)rv[k];
        }
      }
      return;
    }
    R dn[kMixPer], dl[kMixPer], b0[kMixPer], b1[kMixPer];
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) {
        tv[k] = t[i];
        rv[k] = r[i];
        dn[k] = dd[noff + i];
        dl[k] = dd[boff + i];
        b0[k] = rp[i];
        b1[k] = rp[i + niv];
      }
    }
    const bool old0 = boff == 0;  // slot 0 holds the older entry
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) {
        const double tt = tv[k], rr = rv[k];
        const double dnew = dn[k], dold = (double)dl[k] + dnew;
        const double e0 = old0 ? dold : dnew, e1 = old0 ? dnew : dold;  // t_slot - t_k
        const double rp0 = b0[k], rp1 = b1[k];
        const double uu = tt + s1 * e0 + s2 * e1;
        const double vv = tt + rr + s1 * (e0 + rp0 - rr) + s2 * (e1 + rp1 - rr);
        const double tn = uu + m * (vv - uu);
        dd[boff + i] = (R)(tt - tn);
        rp[boff + i] = rv[k];
        t[i] = (T)tn;
      }
    }
    return;
  }
  T *__restrict__ tp = (T *)d.hist_a;
  if (picard) {
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) {
        tv[k] = t[i];
        rv[k] = r[i];
      }
    }
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) {
        tp[boff + i] = tv[k];
        rp[boff + i] = rv[k];
        t[i] = tv[k] + (T)rv[k];
      }
    }
    return;
  }
  T a0[kMixPer], a1[kMixPer];
  R b0[kMixPer], b1[kMixPer];
#pragma unroll
  for (int k = 0; k < kMixPer; ++k) {
    const long long i = i0 + k * kThreads;
    if (i < niv) {
      tv[k] = t[i];
      rv[k] = r[i];
      a0[k] = tp[i];
      a1[k] = tp[i + niv];
      b0[k] = rp[i];
      b1[k] = rp[i + niv];
    }
  }
#pragma unroll
  for (int k = 0; k < kMixPer; ++k) {
    const long long i = i0 + k * kThreads;
    if (i < niv) {
      const double tt = tv[k], rr = rv[k];
      const double tp0 = a0[k], tp1 = a1[k], rp0 = b0[k], rp1 = b1[k];
      const double uu = tt + s1 * (tp0 - tt) + s2 * (tp1 - tt);
      const double vv = tt + rr + s1 * (tp0 + rp0 - tt - rr) + s2 * (tp1 + rp1 - tt - rr);
      tp[boff + i] = tv[k];
      rp[boff + i] = rv[k];
      t[i] = (T)(uu + m * (vv - uu));
    }
  }
}

// ANM dots: <f_k, f_slot> (1/rho weighted) for the newest residual against
// every stored residual.  Writes per-CTA partials [slot].
template <typename P>
__global__ void __launch_bounds__(kThreads)
    k_anm_dots(Batch b) {
  // The dots of the new residual with itself and with the stored residuals,
  // eight slots per pass: each pass reads the residual once and its slots
  // once, with 16-byte vector loads.
  using R = typename P::R;
  using V = typename std::conditional<sizeof(R) == 4, float4, double2>::type;
  constexpr int VEC = 16 / sizeof(R);
  constexpr int G = 8;
  __shared__ double red[8 * (kThreads / 32)];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  const Ctl *c = d.ctl;
  if (c->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int nct = b.prefix[si + 1] - b.prefix[si];
  const int H1 = d.history + 1;
  const long long niv = (long long)d.n * d.Ns;
  const R *f = (const R *)d.hist_a;
  const R *res = (const R *)d.res;
  double *part = d.partials + (size_t)cta * kPartials;
  const int m = c->hcount;
  // vector loads when every site's block starts on a 16-byte boundary
  const long long nv = d.Ns % VEC == 0 ? d.N / VEC : 0;
  const long long stride = (long long)nct * blockDim.x;
  for (int i0 = 0; i0 <= m; i0 += G) {
    const int ng = min(G, m + 1 - i0);
    const R *src[G];
#pragma unroll
    for (int g = 0; g < G; ++g) {
      // i == 0: self dot; i >= 1: history slot (head - i) mod H1
      const int i = i0 + g;
      const int slot = (c->hhead - i + 2 * H1) % H1;
      src[g] = (i == 0 || g >= ng) ? res : f + (long long)slot * niv;
    }
    double acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = 0;
    for (int v = 0; v < d.n; ++v) {
      const long long off = (long long)v * d.Ns;
      double sv[G];
#pragma unroll
      for (int g = 0; g < G; ++g) sv[g] = 0;
      const V *a = reinterpret_cast<const V *>(res + off);
      for (long long q = (long long)cta * blockDim.x + threadIdx.x; q < nv; q += stride) {
        const V x = a[q];
#pragma unroll
        for (int g = 0; g < G; ++g) {
          if (g < ng) {
            const V y = reinterpret_cast<const V *>(src[g] + off)[q];
            if constexpr (VEC == 4) {
              sv[g] += (double)x.x * (double)y.x + (double)x.y * (double)y.y +
                       (double)x.z * (double)y.z + (double)x.w * (double)y.w;
            } else {
              sv[g] += (double)x.x * (double)y.x + (double)x.y * (double)y.y;
            }
          }
        }
      }
      for (long long e = nv * VEC + (long long)cta * blockDim.x + threadIdx.x; e < d.N; e += stride)
#pragma unroll
        for (int g = 0; g < G; ++g)
          if (g < ng) sv[g] += (double)res[off + e] * (double)src[g][off + e];
#pragma unroll
      for (int g = 0; g < G; ++g) acc[g] += sv[g] * d.irho[v];
    }
    // one block sum per used slot (a block_sums<G> here raised the kernel
    // to 170 registers and halved its resident CTAs)
#pragma unroll
    for (int g = 0; g < G; ++g) {
      if (g < ng) {
        const double s = block_sum(acc[g], red);
        if (threadIdx.x == 0) part[1 + i0 + g] = s;
      }
    }
  }
}

// ANM coefficients: update the ring Gram, solve for alpha (1 thread/solve).
__global__ void k_anm_coef(const Desc *descs, const int *ctas, int force) {
  const Desc &d = descs[blockIdx.x];
  Ctl *c = d.ctl;
  if (threadIdx.x != 0) return;
  if (!c->mix_flag) return;
  const int nct = ctas[blockIdx.x];
  const int H = d.history, H1 = H + 1, m = c->hcount;
  double dot[kMaxHistory + 1];
  for (int i = 0; i <= m; ++i) {
    double s = 0;
    for (int k = 0; k < nct; ++k) s += d.partials[(size_t)k * kPartials + 1 + i];
    dot[i] = s;
  }
  const int head = c->hhead;
  // Gram rows of the newest residual (stored under the head slot)
  c->gram[head * H1 + head] = dot[0];
  int slot[kMaxHistory];
  for (int i = 1; i <= m; ++i) {
    slot[i - 1] = (head - i + 2 * H1) % H1;
    c->gram[head * H1 + slot[i - 1]] = dot[i];
    c->gram[slot[i - 1] * H1 + head] = dot[i];
  }
  double A[kMaxHistory * kMaxHistory], x[kMaxHistory];
  const double Fkk = dot[0];
  for (int i = 0; i < m; ++i) {
    x[i] = Fkk - dot[i + 1];
    for (int j = 0; j < m; ++j)
      A[i * m + j] = Fkk - dot[i + 1] - dot[j + 1] +
                     c->gram[slot[i] * H1 + slot[j]];
  }
  bool ok = m > 0 && solve_pp(A, x, m);
  double wsum = 0;
  for (int i = 0; i < m; ++i) {
    if (!ok) x[i] = 0;
    wsum += x[i];
  }
  c->coef[0] = 1.0 - wsum;  // weight of the newest pair
  for (int i = 0; i < m; ++i) {
    c->coef[1 + i] = x[i];
    c->mix_slots[i] = slot[i];
  }
  c->mix_m = m;
  c->mix_head = head;
  // the newest pair joins the history
  c->hhead = (head + 1) % H1;
  if (c->hcount < H) c->hcount += 1;
  (void)force;
}

// ANM mix: t_{k+1} = w_k (t_k + beta R_k) + sum_i alpha_i z_i ; the newest
// pair (R_k, z_k = t_k + beta R_k) is written into the ring under `head`.
// Chunked like k_mix_an2.
template <typename P>
__global__ void __launch_bounds__(kThreads)
    k_mix_anm(Batch b) {
  using R = typename P::R;
  using T = typename P::T;
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  const Ctl *c = d.ctl;
  if (!c->mix_flag) return;
  const long long niv = (long long)d.n * d.Ns;
  const long long i0 = (long long)(blockIdx.x - b.prefix[si]) * kMixChunk + threadIdx.x;
  const int head = c->mix_head, m = c->mix_m;
  T *__restrict__ t = (T *)d.t;
  const R *__restrict__ res = (const R *)d.res;
  R *__restrict__ f = (R *)d.hist_a;
  const double beta = d.beta, w0 = c->coef[0];
  if (!R3D_IN(d, head, d.history + 1) || !R3D_IN(d, m, d.history + 1)) return;
#ifdef R3D_DEBUG_BOUNDS
  for (int q = 0; q < m; ++q)
    if (!R3D_IN(d, c->mix_slots[q], d.history + 1)) return;
#endif
  if constexpr (sizeof(R) < sizeof(T)) {
    // Mixed precision: the history of z_i = t_i + beta R_i is kept as FP32
    // differences of successive entries, E_i = z_i - z_{i+1} (stored under
    // entry i's slot), plus D = t_k - t_{k+1} of the last mix.  With w0 =
    // 1 - sum alpha_i,
    //   t_{k+1} = z_k + sum_i alpha_i (z_i - z_k) = z_k + sum_b C_b E_{k-b},
    // C_b = sum of alpha over the entries of age >= b; the newest difference
    // E_{k-1} = D_{k-1} + beta (R_{k-1} - R_k) is formed here.  Against FP64
    // copies of z this reads 4 instead of 8 bytes per history entry.
    R *__restrict__ er = (R *)d.hist_b;
    R *__restrict__ dp = er + (long long)(d.history + 1) * niv;  // D of the last mix
    double cb[kMaxHistory];
    {
      double run = 0;
      for (int q = m - 1; q >= 0; --q) {
        run += c->coef[1 + q];
        cb[q] = run;  // C_{q+1}: entries of age q+1 and older
      }
    }
    if ((niv & 3) == 0) {
      // Four consecutive elements per thread (16-byte loads of every FP32
      // stream, the chunk's elements [4 tid, 4 tid + 4)), and the history
      // read four slots at a time: 64 bytes of loads in flight per thread in
      // the sum over the ring.  Every slot and stream starts on a 16-byte
      // boundary when niv is a multiple of 4.
      const long long iv = (long long)(blockIdx.x - b.prefix[si]) * kMixChunk + 4 * threadIdx.x;
      if (iv >= niv) return;
      const float4 r4 = *reinterpret_cast<const float4 *>(res + iv);
      const double2 ta = *reinterpret_cast<const double2 *>(t + iv);
      const double2 tb = *reinterpret_cast<const double2 *>(t + iv + 2);
      const double rk[4] = {r4.x, r4.y, r4.z, r4.w}, tk[4] = {ta.x, ta.y, tb.x, tb.y};
      double acc[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[e] = tk[e] + beta * rk[e];
      if (m >= 1) {
        const long long s0 = (long long)c->mix_slots[0] * niv;
        const float4 d4 = *reinterpret_cast<const float4 *>(dp + iv);
        const float4 f4 = *reinterpret_cast<const float4 *>(f + s0 + iv);
        const double dd[4] = {d4.x, d4.y, d4.z, d4.w}, ff[4] = {f4.x, f4.y, f4.z, f4.w};
        float e1f[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double e1 = dd[e] + beta * (ff[e] - rk[e]);
          e1f[e] = (float)e1;
          acc[e] += cb[0] * e1;
        }
        *reinterpret_cast<float4 *>(er + s0 + iv) = make_float4(e1f[0], e1f[1], e1f[2], e1f[3]);
      }
      int q = 1;
      for (; q + 3 < m; q += 4) {
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          v[u] = *reinterpret_cast<const float4 *>(er + (long long)c->mix_slots[q + u] * niv + iv);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const double cu = cb[q + u];
          acc[0] += cu * v[u].x;
          acc[1] += cu * v[u].y;
          acc[2] += cu * v[u].z;
          acc[3] += cu * v[u].w;
        }
      }
      for (; q < m; ++q) {
        const float4 v = *reinterpret_cast<const float4 *>(er + (long long)c->mix_slots[q] * niv + iv);
        const double cq = cb[q];
        acc[0] += cq * v.x;
        acc[1] += cq * v.y;
        acc[2] += cq * v.z;
        acc[3] += cq * v.w;
      }
      *reinterpret_cast<float4 *>(f + (long long)head * niv + iv) = r4;
      *reinterpret_cast<float4 *>(dp + iv) =
          make_float4((float)(tk[0] - acc[0]), (float)(tk[1] - acc[1]), (float)(tk[2] - acc[2]),
                      (float)(tk[3] - acc[3]));
      *reinterpret_cast<double2 *>(t + iv) = make_double2(acc[0], acc[1]);
      *reinterpret_cast<double2 *>(t + iv + 2) = make_double2(acc[2], acc[3]);
      return;
    }
    double acc[kMixPer], tk[kMixPer];
    R rk[kMixPer];
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) {
        rk[k] = res[i];
        tk[k] = (double)t[i];
        acc[k] = tk[k] + beta * (double)rk[k];
      }
    }
    if (m >= 1) {
      const long long s0 = (long long)c->mix_slots[0] * niv;
#pragma unroll
      for (int k = 0; k < kMixPer; ++k) {
        const long long i = i0 + k * kThreads;
        if (i < niv) {
          const double e1 = (double)dp[i] + beta * ((double)f[s0 + i] - (double)rk[k]);
          er[s0 + i] = (R)e1;
          acc[k] += cb[0] * e1;
        }
      }
    }
    int q = 1;
    for (; q + 1 < m; q += 2) {  // two history slots per step
      const R *__restrict__ ea = er + (long long)c->mix_slots[q] * niv;
      const R *__restrict__ eb = er + (long long)c->mix_slots[q + 1] * niv;
      const double ca = cb[q], cc = cb[q + 1];
#pragma unroll
      for (int k = 0; k < kMixPer; ++k) {
        const long long i = i0 + k * kThreads;
        if (i < niv) acc[k] += ca * (double)ea[i] + cc * (double)eb[i];
      }
    }
    if (q < m) {
      const R *__restrict__ eq = er + (long long)c->mix_slots[q] * niv;
      const double cq = cb[q];
#pragma unroll
      for (int k = 0; k < kMixPer; ++k) {
        const long long i = i0 + k * kThreads;
        if (i < niv) acc[k] += cq * (double)eq[i];
      }
    }
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) {
        f[(long long)head * niv + i] = rk[k];
        dp[i] = (R)(tk[k] - acc[k]);
        t[i] = (T)acc[k];
      }
    }
    return;
  }
  T *__restrict__ zr = (T *)d.hist_b;
  double acc[kMixPer], rk[kMixPer], zk[kMixPer];
#pragma unroll
  for (int k = 0; k < kMixPer; ++k) {
    const long long i = i0 + k * kThreads;
    if (i < niv) {
      rk[k] = res[i];
      zk[k] = (double)t[i] + beta * rk[k];
      acc[k] = w0 * zk[k];
    }
  }
  int j = 0;
  for (; j + 1 < m; j += 2) {  // two history slots per step: twice the loads in flight
    const T *__restrict__ za = zr + (long long)c->mix_slots[j] * niv;
    const T *__restrict__ zb = zr + (long long)c->mix_slots[j + 1] * niv;
    const double ca = c->coef[1 + j], cb = c->coef[2 + j];
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) acc[k] += ca * (double)za[i] + cb * (double)zb[i];
    }
  }
  if (j < m) {
    const T *__restrict__ zj = zr + (long long)c->mix_slots[j] * niv;
    const double cj = c->coef[1 + j];
#pragma unroll
    for (int k = 0; k < kMixPer; ++k) {
      const long long i = i0 + k * kThreads;
      if (i < niv) acc[k] += cj * (double)zj[i];
    }
  }
#pragma unroll
  for (int k = 0; k < kMixPer; ++k) {
    const long long i = i0 + k * kThreads;
    if (i < niv) {
      f[(long long)head * niv + i] = (R)rk[k];
      zr[(long long)head * niv + i] = (T)zk[k];
      t[i] = (T)acc[k];
    }
  }
}

// ======================================================================
// Setup kernels: potentials (cal_LJ.cu, cal_Coulomb.cu, cal_potential.cu,
// initialize_tuv.cu), phi_L(k), shell indices.
// ======================================================================
struct AtomTab {
  const double *x, *y, *z, *q;  // [nu]
  const double *sig2, *eps4;    // [n][nu]: sigma_uv^2, 4 eps_uv
  int nu;
};

constexpr int kAtomTile = 128;

// Grid potentials, all sites per voxel: LJ (cal_LJ.cu:56-81), Coulomb in real
// space (cal_Coulomb.cu:40-62); writes u[v] = beta u_LJ + q_v beta (phi -
// phi_L), fr = beta phi_L(r), t0[v] = 0 (the short-range side of init_tuv's
// t0 = q_v fr).
//
// The pair sums are the reference's, arranged so that one atom-voxel pair
// costs one FP64 reciprocal square root and no division:
//   1/r = rsqrt(r^2);  (sigma/r)^6 = sigma^6 (1/r^2)^3, clamped at 1/cut^6,
//   which is the reference's clamp of (r/sigma)^2 from below at cut^2
//   raised to the third power (four operations per site and pair);
//   e^{-r} of the long-range kernel (1 - e^{-r})/r is evaluated only for
//   r <= 38 A: beyond, 1 - e^{-r} rounds to 1 in FP64, as it does in the
//   reference, and most pairs of a protein-sized grid are that far apart.
// Each thread owns V voxels adjacent in x (nx a multiple of V), which share
// an atom's y/z distance terms and its shared-memory loads.
template <typename P, int NS, int V>
__global__ void __launch_bounds__(kThreads)
    k_potential(Desc d, AtomTab at, double ikbt, double ubeta, double dx,
                double dy, double dz, int coulomb, double *fr64) {
  using R = typename P::R;
  using T = typename P::T;
  constexpr int M = NS > 0 ? NS : kMaxSites;
  __shared__ double2 sxy[kAtomTile], szq[kAtomTile];
  __shared__ double2 sse[M][kAtomTile];  // (sigma^6, 4 eps) per site
  const long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = it * V < d.N;
  const long long ip = live ? it * V : 0;
  const int n = d.n;
  const int x = (int)(ip % d.nx), y = (int)((ip / d.nx) % d.ny),
            z = (int)(ip / ((long long)d.nx * d.ny));
  const double ry = (y - d.ny / 2) * dy, rz = (z - d.nz / 2) * dz;
  double rx[V];
#pragma unroll
  for (int j = 0; j < V; ++j) rx[j] = (x + j - d.nx / 2) * dx;
  double lj[V][M], e[V], f[V];
#pragma unroll
  for (int j = 0; j < V; ++j) {
    e[j] = f[j] = 0;
#pragma unroll
    for (int v = 0; v < M; ++v) lj[j][v] = 0;
  }
  // cal_LJ.cu:11: (r/sigma)^2 >= (2e-3)^2, i.e. (sigma/r)^6 <= 1 / (2e-3)^6
  const double smax6 = 1.0 / (2.0e-3 * 2.0e-3 * 2.0e-3 * 2.0e-3 * 2.0e-3 * 2.0e-3);
  for (int a0 = 0; a0 < at.nu; a0 += kAtomTile) {
    const int na = min(kAtomTile, at.nu - a0);
    __syncthreads();
    for (int i = threadIdx.x; i < na; i += blockDim.x) {
      sxy[i] = make_double2(at.x[a0 + i], at.y[a0 + i]);
      szq[i] = make_double2(at.z[a0 + i], at.q[a0 + i]);
      for (int v = 0; v < n; ++v) {
        const double s2 = at.sig2[v * at.nu + a0 + i];
        sse[v][i] = make_double2(s2 * s2 * s2, at.eps4[v * at.nu + a0 + i]);
      }
    }
    __syncthreads();
    for (int i = 0; i < na; ++i) {
      const double2 axy = sxy[i], azq = szq[i];
      const double ddy = ry - axy.y, ddz = rz - azq.x;
      const double yz2 = fma(ddy, ddy, ddz * ddz);
      double r2[V], ir[V], ir6[V];
#pragma unroll
      for (int j = 0; j < V; ++j) {
        const double ddx = rx[j] - axy.x;
        r2[j] = fma(ddx, ddx, yz2);
        ir[j] = rsqrt(r2[j]);
        const double ir2 = ir[j] * ir[j];
        ir6[j] = ir2 * ir2 * ir2;
      }
#pragma unroll
      for (int v = 0; v < M; ++v) {
        if (NS > 0 || v < n) {
          const double2 se = sse[v][i];
#pragma unroll
          for (int j = 0; j < V; ++j) {
            const double s6 = fmin(se.x * ir6[j], smax6);
            lj[j][v] = fma(se.y, fma(s6, s6, -s6), lj[j][v]);
          }
        }
      }
      if (coulomb) {
#pragma unroll
        for (int j = 0; j < V; ++j) {
          if (r2[j] >= 1.0e-10) {  // r >= 1e-5 A
            const double qr = azq.y * ir[j];
            const double ra = r2[j] * ir[j];
            e[j] += qr;
            if (ra <= 38.0)  // a branch, so that far pairs skip the exponential
              f[j] = fma(qr, 1.0 - exp(-ra), f[j]);
            else
              f[j] += qr;  // = fma(qr, 1 - 0, f)
          } else {
            f[j] += azq.y;
          }
        }
      }
    }
  }
  if (!live) return;
  R *u = (R *)d.u, *fr = (R *)d.fr;
  T *t = (T *)d.t;
#pragma unroll
  for (int j = 0; j < V; ++j) {
    const long long q = ip + j;
    const double bfr = f[j] * ubeta, bde = e[j] * ubeta;  // betar
    fr[q] = (R)bfr;
    if (fr64) fr64[q] = bfr;
#pragma unroll
    for (int v = 0; v < M; ++v) {
      if (NS > 0 || v < n) {
        u[(long long)v * d.Ns + q] = (R)(lj[j][v] * ikbt + d.qv[v] * bde - d.qv[v] * bfr);
        t[(long long)v * d.Ns + q] = (T)0;
      }
    }
  }
}

// ======================================================================
// Post-solve per-atom integrals over g (cal_grad.cu:41-90, cal_euv.cu:29-65,
// cal_ad1.cu, cal_ad2.cu), all atoms, sites and voxels in one launch: a CTA
// takes one chunk of voxels and 256 atoms (one per thread); the chunk goes
// through shared memory in tiles (g of every site and the voxel positions),
// every thread sums its atom's terms over the tile, and the chunk's sums go
// to partials [chunk][atom][k] that k_atom_reduce adds up.  Per atom
// (k): 0-2 the force integrand sum_v rho_v g (24 eps s6 (2 s6 - 1) / r^2 +
// q_u q_v cc / r^3) (x, y, z of voxel - atom), 3 the lambda derivative
// (LJ: 24 eps s6 (2 s6 - 1) / lambda, r >= sigma lambda / 2; otherwise the
// Coulomb term q_u q_v cc / r), 4.. the energy per site rho_v g (4 eps s6
// (s6 - 1) + q_u q_v cc / r); terms only for r >= sigma_uv / 2.
// ======================================================================
constexpr int kIntTile = 256;  // voxels per shared-memory tile

template <int NS>
__global__ void __launch_bounds__(kThreads)
    k_atom_integrals(IntAtoms at, const double *g, long long N, int nx, int ny, int nz,
                     double dx, double dy, double dz, long long chunk, double *part) {
  constexpr int M = NS > 0 ? NS : kMaxSites;
  __shared__ double sg[M][kIntTile];
  __shared__ double sx[kIntTile], sy[kIntTile], sz[kIntTile];
  const int n = NS > 0 ? NS : at.n;
  const int a = blockIdx.y * blockDim.x + threadIdx.x;
  const bool live = a < at.nu;
  const double ax = live ? at.x[a] : 0, ay = live ? at.y[a] : 0, az = live ? at.z[a] : 0;
  const double qa = live ? at.q[a] : 0;
  double sig[M], eps[M];
#pragma unroll
  for (int v = 0; v < M; ++v) {
    sig[v] = (live && v < n) ? at.sig[v * at.nu + a] : 0;
    eps[v] = (live && v < n) ? at.eps[v * at.nu + a] : 0;
  }
  double fx = 0, fy = 0, fz = 0, ad = 0, e[M];
#pragma unroll
  for (int v = 0; v < M; ++v) e[v] = 0;
  const long long c0 = blockIdx.x * chunk, c1 = min(N, c0 + chunk);
  for (long long t0 = c0; t0 < c1; t0 += kIntTile) {
    const int nt = (int)min((long long)kIntTile, c1 - t0);
    __syncthreads();
    for (int i = threadIdx.x; i < nt; i += blockDim.x) {
      const long long ip = t0 + i;
      const int x = (int)(ip % nx), y = (int)((ip / nx) % ny), z = (int)(ip / ((long long)nx * ny));
      sx[i] = (x - nx / 2) * dx;
      sy[i] = (y - ny / 2) * dy;
      sz[i] = (z - nz / 2) * dz;
      for (int v = 0; v < n; ++v) sg[v][i] = g[(long long)v * N + ip];
    }
    __syncthreads();
    if (!live) continue;
    for (int i = 0; i < nt; ++i) {
      const double ddx = sx[i] - ax, ddy = sy[i] - ay, ddz = sz[i] - az;
      const double r2 = ddx * ddx + ddy * ddy + ddz * ddz;
      const double r1 = sqrt(r2);
#pragma unroll
      for (int v = 0; v < M; ++v) {
        if (NS == 0 && v >= n) break;
        const double gv = sg[v][i];
        const double qq = qa * at.qv[v] * at.cc;
        const double s2 = sig[v] * sig[v] / r2, s6 = s2 * s2 * s2;
        const double w = at.rhov[v] * gv;
        if (r1 >= sig[v] * 0.5) {
          const double fm = (eps[v] * 24.0 * s6 / r2 * (2.0 * s6 - 1.0) + qq / (r2 * r1)) * w;
          fx += fm * ddx;
          fy += fm * ddy;
          fz += fm * ddz;
          e[v] += (eps[v] * 4.0 * s6 * (s6 - 1.0) + qq / r1) * w;
          if (!at.ad1) ad += qq / r1 * w;
        }
        if (at.ad1 && r1 >= sig[v] * at.lambda * 0.5)
          ad += eps[v] * 24.0 * s6 * (2.0 * s6 - 1.0) / at.lambda * w;
      }
    }
  }
  if (!live) return;
  const int K = 4 + n;
  double *o = part + ((long long)blockIdx.x * at.nu + a) * K;
  o[0] = fx;
  o[1] = fy;
  o[2] = fz;
  o[3] = ad;
  for (int v = 0; v < n; ++v) o[4 + v] = e[v];
}

// out[a][k] = sum over the chunks of part[chunk][a][k]
__global__ void k_atom_reduce(const double *part, int nchunk, long long nk, double *out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nk;
       i += (long long)gridDim.x * blockDim.x) {
    double s = 0;
    for (int c = 0; c < nchunk; ++c) s += part[(long long)c * nk + i];
    out[i] = s;
  }
}

void launch_atom_integrals(const IntAtoms &at, const double *g, long long N, const int *grid,
                           const double *dr, double *part, int nchunk, double *out,
                           cudaStream_t s) {
  const long long chunk = (N + nchunk - 1) / nchunk;
  dim3 gr(nchunk, (at.nu + kThreads - 1) / kThreads);
#define R3D_INT(NS)                                                                      \
  k_atom_integrals<NS><<<gr, kThreads, 0, s>>>(at, g, N, grid[0], grid[1], grid[2], dr[0], \
                                               dr[1], dr[2], chunk, part)
  switch (at.n) {
    case 1: R3D_INT(1); break;
    case 2: R3D_INT(2); break;
    case 3: R3D_INT(3); break;
    case 4: R3D_INT(4); break;
    default: R3D_INT(0); break;
  }
#undef R3D_INT
  const long long nk = (long long)at.nu * (4 + at.n);
  k_atom_reduce<<<(int)std::min<long long>((nk + kThreads - 1) / kThreads, 1184), kThreads, 0,
                  s>>>(part, nchunk, nk, out);
}

// Per-axis phase tables e^{-i k_j x_u} (FP64): ex[u][p] (k index j = 2p),
// ey[u][y], ez[u][z].
__global__ void k_phase_tables(double2 *ex, double2 *ey, double2 *ez,
                               const double *ax, const double *ay,
                               const double *az, int nu, int nx, int ny,
                               int nz, double bx, double by, double bz) {
  const int hx = nx / 2;
  const long long tot = (long long)nu * (hx + ny + nz);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    int u = (int)(i / (hx + ny + nz)), j = (int)(i % (hx + ny + nz));
    double k, r;
    double2 *dst;
    if (j < hx) {
      k = 2.0 * M_PI * (2 * j - nx / 2.0 + 0.5) / bx;
      r = ax[u];
      dst = ex + (long long)u * hx + j;
    } else if (j < hx + ny) {
      j -= hx;
      k = 2.0 * M_PI * (j - ny / 2.0 + 0.5) / by;
      r = ay[u];
      dst = ey + (long long)u * ny + j;
    } else {
      j -= hx + ny;
      k = 2.0 * M_PI * (j - nz / 2.0 + 0.5) / bz;
      r = az[u];
      dst = ez + (long long)u * nz + j;
    }
    double s, c;
    sincos(k * r, &s, &c);
    *dst = make_double2(c, -s);
  }
}

// phi_L(k) in transform units: fk = ubeta sum_u 4 pi q_u / (k^2 (k^2+1))
// e^{-i k.r_u} (cal_Coulomb.cu:65-95), divided by dv * C(k) with
// C(k) = -i (-1)^{jx+jy+jz+(nx+ny+nz)/2}.
//
// The structure factor is a complex matrix product over the atoms:
//   S[p][c] = sum_u ex[u][p] w[u][c],  w[u][c] = q_u ey[u][y] ez[u][z],
// c = y + ny z the (k_y, k_z) column.  A CTA owns kFkT k_x values x kFkT
// columns; atoms come in chunks of kFkA through shared memory (the chunk's
// ex rows, and its w formed once per CTA and reused by every k_x), and each
// thread accumulates 4 x 4 outputs in registers, each over the atoms in
// order: four FP64 FMAs per atom and output.
constexpr int kFkT = 64, kFkA = 16;
__global__ void __launch_bounds__(kThreads, 2)
    k_fk(Desc d, double2 *fk64, const double2 *ex, const double2 *ey,
         const double2 *ez, const double *q, int nu, double ubeta, double bx,
         double by, double bz, double dv) {
  __shared__ double2 sx[kFkA][kFkT], sw[kFkA][kFkT];
  const int hx = d.hx, ny = d.ny;
  const long long ncol = (long long)ny * d.nz;
  const int ptiles = (hx + kFkT - 1) / kFkT;
  const int p0 = (int)(blockIdx.x % ptiles) * kFkT;
  const long long c0 = (long long)(blockIdx.x / ptiles) * kFkT;
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  for (int a0 = 0; a0 < nu; a0 += kFkA) {
    __syncthreads();
    for (int e = threadIdx.x; e < kFkA * kFkT; e += kThreads) {
      const int a = e / kFkT, j = e % kFkT, u = a0 + a;
      const int p = p0 + j;
      sx[a][j] = (u < nu && p < hx) ? ex[(long long)u * hx + p] : make_double2(0.0, 0.0);
      const long long c = c0 + j;
      double2 w = make_double2(0.0, 0.0);
      if (u < nu && c < ncol) {
        const int y = (int)(c % ny), z = (int)(c / ny);
        const double2 by2 = ey[(long long)u * ny + y], bz2 = ez[(long long)u * d.nz + z];
        const double qq = q[u];
        w = make_double2(qq * (by2.x * bz2.x - by2.y * bz2.y),
                         qq * (by2.x * bz2.y + by2.y * bz2.x));
      }
      sw[a][j] = w;
    }
    __syncthreads();
#pragma unroll 4
    for (int a = 0; a < kFkA; ++a) {
      double2 xv[4], wv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) xv[i] = sx[a][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) wv[j] = sw[a][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x = fma(-xv[i].y, wv[j].y, fma(xv[i].x, wv[j].x, acc[i][j].x));
          acc[i][j].y = fma(xv[i].y, wv[j].x, fma(xv[i].x, wv[j].y, acc[i][j].y));
        }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int p = p0 + tx + 16 * i;
    if (p >= hx) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const long long c = c0 + ty + 16 * j;
      if (c >= ncol) continue;
      const int y = (int)(c % ny), z = (int)(c / ny);
      const double kx = 2.0 * M_PI * (2 * p - d.nx / 2.0 + 0.5) / bx;
      const double ky = 2.0 * M_PI * (y - d.ny / 2.0 + 0.5) / by;
      const double kz = 2.0 * M_PI * (z - d.nz / 2.0 + 0.5) / bz;
      const double rk2 = kx * kx + ky * ky + kz * kz;
      const double rk4i = 1.0 / (rk2 * (rk2 + 1.0));
      const double sc = 4.0 * M_PI * rk4i * ubeta;
      const double re = acc[i][j].x * sc, im = acc[i][j].y * sc;
      // divide by dv * C:  (re + i im) * conj(C) / dv, conj(C) = i * sigma
      const int par = (2 * p + y + z + (d.nx + d.ny + d.nz) / 2) & 1;
      const double sg = par ? -1.0 : 1.0;
      fk64[p + (long long)hx * c] = make_double2(-im * sg / dv, re * sg / dv);
    }
  }
}

// Refresh, step 1: freeze c_ref = c_s(t) in the grid type, and an FP64 copy
// of exactly the stored values for the FP64 transform.
template <typename P>
__global__ void k_cref(Desc d, double *c64) {
  using R = typename P::R;
  using T = typename P::T;
  const long long niv = (long long)d.n * d.Ns;
  const T *t = (const T *)d.t;
  const R *u = (const R *)d.u;
  R *cref = (R *)d.cref;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < niv;
       i += (long long)gridDim.x * blockDim.x) {
    double g = closure_g<double>(d.clos, d.pse_n, -(double)u[i] + (double)t[i]);
    R c = (R)(g - 1.0 - (double)t[i]);
    cref[i] = c;
    c64[i] = (double)c;
  }
}

// Refresh, step 2: lr = 1 + h_ref (h_ref from the FP64 transform).
template <typename P>
__global__ void k_lr_update(const double *href, typename P::R *lr, long long niv) {
  using R = typename P::R;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < niv;
       i += (long long)gridDim.x * blockDim.x)
    lr[i] = (R)(1.0 + href[i]);
}

// Shell index of each half-spectrum point.  Cubic boxes: (s - 3) / 8 with
// s = ax^2 + ay^2 + az^2 over the odd integers a = 2j - n + 1; otherwise a
// lookup in the host-built table of (|ax|, |ay|, |az|) tuples.
__global__ void k_kidx(Desc d, const uint32_t *tuple_idx, int cubic) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Nh) return;
  const int hx = d.hx;
  int p = (int)(i % hx), y = (int)((i / hx) % d.ny),
      z = (int)(i / ((long long)hx * d.ny));
  int ax = 4 * p - d.nx + 1, ay = 2 * y - d.ny + 1, az = 2 * z - d.nz + 1;
  uint32_t s;
  if (cubic) {
    long long ss = (long long)ax * ax + (long long)ay * ay + (long long)az * az;
    s = (uint32_t)((ss - 3) / 8);
  } else {
    int ix = (abs(ax) - 1) / 2, iy = (abs(ay) - 1) / 2, iz = (abs(az) - 1) / 2;
    s = tuple_idx[((long long)iz * (d.ny / 2) + iy) * (d.nx / 2) + ix];
  }
  ((uint32_t *)d.kidx)[i] = s;
}

// ======================================================================
// Thermodynamics (cal_exchem.cu:55-155, cal_pmv.cu:27-57): per-site sums of
// the closure functional, HNC functional, GF functional and c = h - t.
// g is rebuilt from (tg, u), h = R - 1 + g; c uses the current t.
// ======================================================================
template <typename P>
__global__ void __launch_bounds__(kThreads)
    k_thermo(Desc d, const typename P::T *tg, double *out /* [ctas][n][4] */) {
  using R = typename P::R;
  using T = typename P::T;
  __shared__ double red[8 * (kThreads / 32)];
  const T *t = (const T *)d.t;
  const R *u = (const R *)d.u, *res = (const R *)d.res;
  const R *fr = (const R *)d.fr;
  for (int v = 0; v < d.n; ++v) {
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < d.N;
         x += (long long)gridDim.x * blockDim.x) {
      long long i = (long long)v * d.Ns + x;
      // physical t = t_s + q_v beta phi_L(r); t* = t - beta u = t_s - u_s
      double tt = (double)t[i] + d.qv[v] * (double)fr[x];
      double ts = -(double)u[i] + (double)tg[i];
      double g = closure_g<double>(d.clos, d.pse_n, ts);
      double h = (double)res[i] - 1.0 + g;
      double c = h - tt;
      double ehnc = h * 0.5 * tt - c;
      double egf = -(h * 0.5 + 1.0) * c;
      double esc;
      if (d.clos == HNC) {
        esc = ehnc;
      } else if (h > 0.0) {
        if (d.clos == KH || d.pse_n == 1) {
          esc = egf;
        } else {
          double term = 1.0;
          for (int k = 1; k <= d.pse_n + 1; ++k) term *= ts / k;
          esc = 0.5 * h * h - c - 0.5 * h * c - term;
        }
      } else {
        esc = ehnc;
      }
      a0 += esc;
      a1 += ehnc;
      a2 += egf;
      a3 += c;
    }
    double q[4] = {a0, a1, a2, a3};
    block_sums<4>(q, red);
    if (threadIdx.x == 0) {
      double *o = out + ((size_t)blockIdx.x * d.n + v) * 4;
      o[0] = q[0];
      o[1] = q[1];
      o[2] = q[2];
      o[3] = q[3];
    }
  }
}

// g (and h) grids for read-back: g = closure(t - u), h = R - 1 + g.
template <typename P>
__global__ void k_gh(Desc d, const typename P::T *tg, double *g, double *h) {
  using R = typename P::R;
  const long long niv = (long long)d.n * d.N;  // dense output [site][N]
  const R *u = (const R *)d.u, *res = (const R *)d.res;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < niv;
       j += (long long)gridDim.x * blockDim.x) {
    const long long i = (j / d.N) * d.Ns + j % d.N;
    double gv = closure_g<double>(d.clos, d.pse_n, -(double)u[i] + (double)tg[i]);
    if (g) g[j] = gv;
    if (h) h[j] = (double)res[i] - 1.0 + gv;
  }
}

template <typename R>
__global__ void k_to_double(const R *src, double *dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
template <typename R>
__global__ void k_from_double(const double *src, R *dst, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (R)src[i];
}
// short-range -> physical: dst = src + sign * q_v fr  (per-site grids)
template <typename P, typename X>
__global__ void k_shift_qfr(Desc d, const X *src, double *dst, double sign) {
  using R = typename P::R;
  const long long niv = (long long)d.n * d.N;  // dense output [site][N]
  const R *fr = (const R *)d.fr;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < niv;
       j += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(j / d.N);
    const long long x = j % d.N;
    const double f = sign != 0.0 ? sign * d.qv[v] * (double)fr[x] : 0.0;
    dst[j] = (double)src[(long long)v * d.Ns + x] + f;
  }
}
// physical -> short-range: dst = src - q_v fr
template <typename P>
__global__ void k_set_short(Desc d, const double *src, typename P::T *dst) {
  using R = typename P::R;
  using T = typename P::T;
  const long long niv = (long long)d.n * d.N;  // dense input [site][N]
  const R *fr = (const R *)d.fr;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < niv;
       j += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(j / d.N);
    const long long x = j % d.N;
    dst[(long long)v * d.Ns + x] = (T)(src[j] - d.qv[v] * (double)fr[x]);
  }
}

// Twiddle table entries e^{i pi scale e} for e in [0, count).
__global__ void k_twiddle(double2 *o64, float2 *o32, int count, double scale) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(scale * (double)e, &s, &c);
    if (o64) o64[e] = make_double2(c, s);
    if (o32) o32[e] = make_float2((float)c, (float)s);
  }
}

// ======================================================================
// Host-side launch wrappers
// ======================================================================
size_t smem_x(int hx, int n, int S, size_t csz) {
  return csz * hx * 2 + ((2 * hx + 15) / 16) * 16 + csz * (size_t)n * S * hx;
}
size_t smem_y(int ny, int P, size_t csz) {
  return csz * ny * 2 + ((2 * ny + 15) / 16) * 16 + csz * (size_t)ny * P;
}
size_t smem_z(int nz, int n, int P, size_t csz) {
  return csz * nz * 2 + ((2 * nz + 15) / 16) * 16 + csz * (size_t)n * nz * P;
}

template <typename P>
static void set_smem_attrs(size_t maxbytes) {
  const int mb = (int)maxbytes;
  const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaFuncSetAttribute(k_fwd_x<P, 0>, a, mb);
  cudaFuncSetAttribute(k_fwd_x<P, 1>, a, mb);
  cudaFuncSetAttribute(k_fft_y<P, -1>, a, mb);
  cudaFuncSetAttribute(k_fft_y<P, 1>, a, mb);
  cudaFuncSetAttribute(k_zoz<P, 0>, a, mb);
  cudaFuncSetAttribute(k_zoz<P, 1>, a, mb);
  cudaFuncSetAttribute(k_zoz<P, 2>, a, mb);
  cudaFuncSetAttribute(k_inv_x<P, 0>, a, mb);
  cudaFuncSetAttribute(k_inv_x<P, 1>, a, mb);
}

// Resident CTAs per SM of the grid-stride streaming kernels (mixers), so
// that their grids are exactly one wave.
int dot_blocks_per_sm(bool fp64) {
  int b = 0;
  if (fp64)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_anm_dots<P64>, kThreads, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_anm_dots<PMix>, kThreads, 0);
  return b > 0 ? b : 1;
}
int mix_chunk() { return kMixChunk; }

void launch_twiddle(double2 *o64, float2 *o32, int count, double scale, cudaStream_t s) {
  k_twiddle<<<(count + kThreads - 1) / kThreads, kThreads, 0, s>>>(o64, o32, count, scale);
}

template <typename P>
void ct_allow_smem_all();

template <typename P>
void tma_allow_smem_all();
void kernels_set_smem(bool fp64, size_t maxbytes) {
  static bool ct_done[2] = {false, false};
  if (fp64)
    set_smem_attrs<P64>(maxbytes);
  else
    set_smem_attrs<PMix>(maxbytes);
  if (!ct_done[fp64]) {  // compile-time-engine passes, once per process
    if (fp64) {
      ct_allow_smem_all<P64>();
      tma_allow_smem_all<P64>();
    } else {
      ct_allow_smem_all<PMix>();
      tma_allow_smem_all<PMix>();
    }
    ct_done[fp64] = true;
  }
}

// Pass launchers.  `grid` = total CTAs of the pass over all solves in the
// batch; `smem` = dynamic shared memory (max over solves).
template <typename P>
void launch_fwd_x(Batch b, int grid, size_t smem, cudaStream_t s, int mode,
                  const void *src) {
  using R = typename P::R;
  if (mode == 0)
    k_fwd_x<P, 0><<<grid, kThreads, smem, s>>>(b, (const R *)src);
  else
    k_fwd_x<P, 1><<<grid, kThreads, smem, s>>>(b, nullptr);
}
template <typename P>
void launch_fft_y(Batch b, int grid, size_t smem, cudaStream_t s, int dir,
                  int check) {
  if (dir < 0)
    k_fft_y<P, -1><<<grid, kThreads, smem, s>>>(b, check);
  else
    k_fft_y<P, 1><<<grid, kThreads, smem, s>>>(b, check);
}
template <typename P>
void launch_zoz(Batch b, int grid, size_t smem, cudaStream_t s, int mode,
                int check) {
  if (mode == 0)
    k_zoz<P, 0><<<grid, kThreads, smem, s>>>(b, check);
  else if (mode == 1)
    k_zoz<P, 1><<<grid, kThreads, smem, s>>>(b, check);
  else
    k_zoz<P, 2><<<grid, kThreads, smem, s>>>(b, check);
}
template <typename P>
void launch_inv_x(Batch b, int grid, size_t smem, cudaStream_t s, int mode,
                  void *dst, int per) {
  using R = typename P::R;
  if (mode == 0)
    k_inv_x<P, 0><<<grid, kThreads, smem, s>>>(b, (R *)dst, per);
  else
    k_inv_x<P, 1><<<grid, kThreads, smem, s>>>(b, nullptr, per);
}
void launch_reduce(const Desc *d, const int *ctas, int ns, int force,
                   cudaStream_t s) {
  k_reduce<<<ns, kThreads, 0, s>>>(d, ctas, force);
}
// Control words of ns solves, gathered for one read-back:
// out[4 i ..] = status, completed steps, rms, error word.
__global__ void k_ctl_gather(const Desc *descs, int ns, double *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += gridDim.x * blockDim.x) {
    const Ctl *c = descs[i].ctl;
    out[4 * i + 0] = c->status;
    out[4 * i + 1] = c->step;
    out[4 * i + 2] = c->rms;
    out[4 * i + 3] = c->err;
  }
}
void launch_ctl_gather(const Desc *d, int ns, double *out, cudaStream_t s) {
  k_ctl_gather<<<(ns + kThreads - 1) / kThreads, kThreads, 0, s>>>(d, ns, out);
}
template <typename P>
void launch_mix_an2(Batch b, int grid, cudaStream_t s) {
  k_mix_an2<P><<<grid, kThreads, 0, s>>>(b);
}
// Mixed AN2: the t of the last evaluation when the last step also mixed
// (maxstep): t_k = t_{k+1} + D_k, D_k in slot `slot` of the t differences.
__global__ void k_t_restore(const double *t, const float *dslot, double *out, long long niv) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < niv) out[i] = t[i] + (double)dslot[i];
}
void launch_t_restore(const void *t, const void *dslot, void *out, long long niv,
                      cudaStream_t s) {
  k_t_restore<<<(unsigned)((niv + kThreads - 1) / kThreads), kThreads, 0, s>>>(
      (const double *)t, (const float *)dslot, (double *)out, niv);
}
template <typename P>
void launch_anm(Batch b, int grid, const Desc *d, const int *ctas, int ns,
                cudaStream_t s, int stage) {
  if (stage == 0)
    k_anm_dots<P><<<grid, kThreads, 0, s>>>(b);
  else if (stage == 1)
    k_anm_coef<<<ns, 32, 0, s>>>(d, ctas, 0);
  else
    k_mix_anm<P><<<grid, kThreads, 0, s>>>(b);
}
template <typename P>
void launch_potential(const Desc &d, const AtomTab &at, double ikbt,
                      double ubeta, const double *dr, int coulomb,
                      double *fr64, cudaStream_t s) {
  // two voxels per thread (nx is even); four measured 9% slower on a B200
  constexpr int V = 2;
  const long long thr = (d.N + V - 1) / V;
  int grid = (int)((thr + kThreads - 1) / kThreads);
#define R3D_POT(NS)                                                           \
  k_potential<P, NS, V><<<grid, kThreads, 0, s>>>(d, at, ikbt, ubeta, dr[0], \
                                                  dr[1], dr[2], coulomb, fr64)
  switch (d.n) {
    case 1: R3D_POT(1); break;
    case 2: R3D_POT(2); break;
    case 3: R3D_POT(3); break;
    case 4: R3D_POT(4); break;
    default: R3D_POT(0); break;
  }
#undef R3D_POT
}
void launch_phase_tables(double2 *ex, double2 *ey, double2 *ez,
                         const double *ax, const double *ay, const double *az,
                         int nu, int nx, int ny, int nz, const double *box,
                         cudaStream_t s) {
  k_phase_tables<<<1184, kThreads, 0, s>>>(ex, ey, ez, ax, ay, az, nu, nx, ny,
                                           nz, box[0], box[1], box[2]);
}
void launch_fk(const Desc &d, double2 *fk64, const double2 *ex,
               const double2 *ey, const double2 *ez, const double *q, int nu,
               double ubeta, const double *box, double dv, cudaStream_t s) {
  const long long ncol = (long long)d.ny * d.nz;
  const long long tiles = (long long)((d.hx + kFkT - 1) / kFkT) * ((ncol + kFkT - 1) / kFkT);
  k_fk<<<(int)tiles, kThreads, 0, s>>>(d, fk64, ex, ey, ez, q, nu, ubeta, box[0],
                                       box[1], box[2], dv);
}
template <typename P>
void launch_cref(const Desc &d, double *c64, cudaStream_t s) {
  k_cref<P><<<1184, kThreads, 0, s>>>(d, c64);
}
template <typename P>
void launch_lr_update(const double *href, void *lr, long long niv,
                      cudaStream_t s) {
  k_lr_update<P><<<1184, kThreads, 0, s>>>(href, (typename P::R *)lr, niv);
}
void launch_kidx(const Desc &d, const uint32_t *tuple_idx, int cubic,
                 cudaStream_t s) {
  int grid = (int)((d.Nh + kThreads - 1) / kThreads);
  k_kidx<<<grid, kThreads, 0, s>>>(d, tuple_idx, cubic);
}
template <typename P>
void launch_thermo(const Desc &d, const void *tg, double *out, int ctas,
                   cudaStream_t s) {
  k_thermo<P><<<ctas, kThreads, 0, s>>>(d, (const typename P::T *)tg, out);
}
template <typename P>
void launch_gh(const Desc &d, const void *tg, double *g, double *h,
               cudaStream_t s) {
  k_gh<P><<<1184, kThreads, 0, s>>>(d, (const typename P::T *)tg, g, h);
}
// element-type conversions: x = 0 grid type R, x = 1 state type T
template <typename P>
void launch_to_double(const void *src, double *dst, long long n, int x,
                      cudaStream_t s) {
  if (x == 0)
    k_to_double<typename P::R><<<1184, kThreads, 0, s>>>((const typename P::R *)src, dst, n);
  else
    k_to_double<typename P::T><<<1184, kThreads, 0, s>>>((const typename P::T *)src, dst, n);
}
template <typename P>
void launch_from_double(const double *src, void *dst, long long n, int x,
                        cudaStream_t s) {
  if (x == 0)
    k_from_double<typename P::R><<<1184, kThreads, 0, s>>>(src, (typename P::R *)dst, n);
  else
    k_from_double<typename P::T><<<1184, kThreads, 0, s>>>(src, (typename P::T *)dst, n);
}
template <typename P>
void launch_shift_qfr(const Desc &d, const void *src, double *dst, double sign,
                      int x, cudaStream_t s) {
  if (x == 0)
    k_shift_qfr<P, typename P::R><<<1184, kThreads, 0, s>>>(
        d, (const typename P::R *)src, dst, sign);
  else
    k_shift_qfr<P, typename P::T><<<1184, kThreads, 0, s>>>(
        d, (const typename P::T *)src, dst, sign);
}
template <typename P>
void launch_set_short(const Desc &d, const double *src, void *dst,
                      cudaStream_t s) {
  k_set_short<P><<<1184, kThreads, 0, s>>>(d, src, (typename P::T *)dst);
}

#define R3D_INST(P)                                                            \
  template void launch_fwd_x<P>(Batch, int, size_t, cudaStream_t, int,         \
                                const void *);                                 \
  template void launch_fft_y<P>(Batch, int, size_t, cudaStream_t, int, int);   \
  template void launch_zoz<P>(Batch, int, size_t, cudaStream_t, int, int);     \
  template void launch_inv_x<P>(Batch, int, size_t, cudaStream_t, int, void *, \
                                int);                                          \
  template void launch_mix_an2<P>(Batch, int, cudaStream_t);                   \
  template void launch_anm<P>(Batch, int, const Desc *, const int *, int,      \
                              cudaStream_t, int);                              \
  template void launch_potential<P>(const Desc &, const AtomTab &, double,     \
                                    double, const double *, int, double *,     \
                                    cudaStream_t);                             \
  template void launch_cref<P>(const Desc &, double *, cudaStream_t);          \
  template void launch_lr_update<P>(const double *, void *, long long,         \
                                    cudaStream_t);                             \
  template void launch_thermo<P>(const Desc &, const void *, double *, int,    \
                                 cudaStream_t);                                \
  template void launch_gh<P>(const Desc &, const void *, double *, double *,   \
                             cudaStream_t);                                    \
  template void launch_to_double<P>(const void *, double *, long long, int,    \
                                    cudaStream_t);                             \
  template void launch_from_double<P>(const double *, void *, long long, int,  \
                                      cudaStream_t);                           \
  template void launch_shift_qfr<P>(const Desc &, const void *, double *,      \
                                    double, int, cudaStream_t);                \
  template void launch_set_short<P>(const Desc &, const double *, void *,      \
                                    cudaStream_t);
R3D_INST(P64)
R3D_INST(PMix)

}  // namespace r3d
