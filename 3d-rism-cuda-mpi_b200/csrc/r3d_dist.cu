// r3d_dist.cu -- one rank's pointwise steps of a solve split over GPUs
// (r3d_dist_*; slabs.py's DistSolve drives them, with r3d_slab_transform for
// the transforms and NCCL for the all-to-alls and the sums).
//
// The reference splits a solve over MPI ranks: each rank owns a pencil of
// every array, calculate() runs its pointwise steps on that pencil
// (calculate_cuda.cu: trm1mt, mqvfk, oz, tr) and the mixer its AN2 update
// (anderson_cuda.cu), while cal_rms.cu:23 and anderson.cu:95 sum the RMS and
// the theta dots over ranks.  These kernels are those steps on one rank's
// slabs, in FP64 (the reference's precision): z-slabs of the real-space
// arrays, y-slabs of the half spectrum.  Every call is asynchronous on the
// caller's stream (NULL: the default stream) and returns the launch status.
#include <cuda_runtime.h>

#include <string>

#include "../../include/rism3d_b200.h"
#include "r3d_common.cuh"

namespace r3d {
void set_last_error(const std::string &m);
}  // namespace r3d

using namespace r3d;

namespace {

constexpr int kDistThreads = 256;
constexpr int kDistBlocks = 296;  // CTAs per site of the residual sums (two per SM)

struct Charges {
  double q[kMaxSites];
};

int dist_fail(int code, const std::string &m) {
  set_last_error("r3d_dist: " + m);
  return code;
}

// the caller's device is current again when the call returns
struct DeviceScope {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceScope(int device) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess) err = cudaSetDevice(device);
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

int launched() {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? R3D_OK : dist_fail(R3D_ECUDA, cudaGetErrorString(e));
}

int grid_for(long long count) {
  const long long b = (count + kDistThreads - 1) / kDistThreads;
  return (int)(b < 148LL * 8 ? b : 148LL * 8);
}

// trm1mt (calculate_cuda.cu:18-24) on the full t: g = closure(-u + t),
// c = g - 1 - t + q_v beta phi_L(r)
__global__ void k_dist_closure(int n, long long nloc, int clos, int pse_n, const double *du,
                               const double *t, const double *fr, Charges qv, double *g,
                               double *c) {
  const long long total = (long long)n * nloc;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int v = (int)(i / nloc);
    const long long j = i - (long long)v * nloc;
    const double tt = t[i];
    const double gg = closure_g<double>(clos, pse_n, -du[i] + tt);
    g[i] = gg;
    c[i] = gg - 1.0 - tt + qv.q[v] * fr[j];
  }
}

// mqvfk and oz (calculate_cuda.cu:39-52) at each half-spectrum point of the
// rank's y-slab, in place: H_v = sum_v' chi_vv' (C_v' - q_v' fk)
__global__ void k_dist_oz(int n, long long nk, const double *chi, const double2 *fk, Charges qv,
                          double2 *spec) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nk;
       k += (long long)gridDim.x * blockDim.x) {
    const double2 f = fk[k];
    double2 cs[kMaxSites];
    for (int b = 0; b < n; ++b) {
      const double2 x = spec[(long long)b * nk + k];
      cs[b] = make_double2(x.x - qv.q[b] * f.x, x.y - qv.q[b] * f.y);
    }
    for (int a = 0; a < n; ++a) {
      double hr = 0.0, hi = 0.0;
      for (int b = 0; b < n; ++b) {
        const double x = chi[((long long)a * n + b) * nk + k];
        hr += cs[b].x * x;
        hi += cs[b].y * x;
      }
      spec[(long long)a * nk + k] = make_double2(hr, hi);
    }
  }
}

// tr (calculate_cuda.cu:54-60): R = scale h + 1 - g; per CTA of site v:
// sum R^2 and, when dots, the five AN2 theta dots against the two stored
// residuals (anderson_cuda.cu:25-67) -> part[(v * kDistBlocks + cta) * 6 + k]
__global__ void __launch_bounds__(kDistThreads)
    k_dist_residual(long long nloc, double scale, const double *h, const double *g,
                    const double *rp0, const double *rp1, int dots, double *r, double *part) {
  __shared__ double red[6 * (kDistThreads / 32)];
  const int v = blockIdx.y;
  const long long off = (long long)v * nloc;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nloc;
       j += (long long)gridDim.x * blockDim.x) {
    const long long i = off + j;
    const double rr = h[i] * scale + 1.0 - g[i];
    r[i] = rr;
    a[0] += rr * rr;
    if (dots) {
      const double t1 = rr - rp0[i], t2 = rr - rp1[i];
      a[1] += rr * t1;
      a[2] += rr * t2;
      a[3] += t1 * t1;
      a[4] += t1 * t2;
      a[5] += t2 * t2;
    }
  }
  block_sums<6>(a, red);
  if (threadIdx.x == 0) {
    double *o = part + ((long long)v * gridDim.x + blockIdx.x) * 6;
    for (int k = 0; k < 6; ++k) o[k] = a[k];
  }
}

// the partials in a fixed order: sums[0] = sum R^2 over sites, sums[1 + 5 v
// + k] the dots of site v
__global__ void k_dist_sums(int n, const double *part, double *sums) {
  __shared__ double red[kDistThreads / 32];
  for (int q = 0; q < 1 + 5 * n; ++q) {
    const int v = q == 0 ? -1 : (q - 1) / 5, k = q == 0 ? 0 : 1 + (q - 1) % 5;
    double s = 0.0;
    if (v < 0) {
      for (int i = threadIdx.x; i < n * kDistBlocks; i += blockDim.x) s += part[(long long)i * 6];
    } else {
      for (int i = threadIdx.x; i < kDistBlocks; i += blockDim.x)
        s += part[((long long)v * kDistBlocks + i) * 6 + k];
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) sums[q] = s;
  }
}

// newdt0 / newdt (anderson_cuda.cu:1-22): the current t and R go to slot
// `binary`, t becomes t + R (Picard) or the AN2 combination
__global__ void k_dist_mix(long long count, double *t, const double *r, double *tp0,
                           double *tp1, double *rp0, double *rp1, int binary, int picard,
                           double s1, double s2, double m) {
  double *tpb = binary ? tp1 : tp0, *rpb = binary ? rp1 : rp0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const double tt = t[i], rr = r[i];
    double tn;
    if (picard) {
      tn = tt + rr;
    } else {
      const double a0 = tp0[i], a1 = tp1[i], b0 = rp0[i], b1 = rp1[i];
      const double u = tt + s1 * (a0 - tt) + s2 * (a1 - tt);
      const double w = tt + rr + s1 * (a0 + b0 - tt - rr) + s2 * (a1 + b1 - tt - rr);
      tn = u + m * (w - u);
    }
    tpb[i] = tt;
    rpb[i] = rr;
    t[i] = tn;
  }
}

// history-m Anderson: up to kDistHist stored residuals per call
constexpr int kDistHist = 16;
struct Slots {
  const double *p[kDistHist];
};

// <r, r> and <r, f_i> per CTA of site v, one pass over r and the f_i:
// part[((v * kDistBlocks + cta) * (kDistHist + 1)) + k]
__global__ void __launch_bounds__(kDistThreads)
    k_dist_anm_dots(long long nloc, const double *r, Slots f, int m, double *part) {
  __shared__ double red[kDistThreads / 32];
  const int v = blockIdx.y;
  const long long off = (long long)v * nloc;
  double a[kDistHist + 1];
#pragma unroll
  for (int k = 0; k <= kDistHist; ++k) a[k] = 0.0;
  for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < nloc;
       j += (long long)gridDim.x * blockDim.x) {
    const double rr = r[off + j];
    a[0] += rr * rr;
#pragma unroll
    for (int k = 0; k < kDistHist; ++k)
      if (k < m) a[1 + k] += rr * f.p[k][off + j];
  }
  double *o = part + ((long long)v * gridDim.x + blockIdx.x) * (kDistHist + 1);
#pragma unroll
  for (int k = 0; k <= kDistHist; ++k) {
    if (k <= m) {  // the same for every thread of the CTA
      const double s = block_sum(a[k], red);
      if (threadIdx.x == 0) o[k] = s;
    }
  }
}

// the partials in a fixed order, site by site with the weights 1 / rho_v
__global__ void k_dist_anm_sums(int n, int m, Charges irho, const double *part, double *sums) {
  __shared__ double red[kDistThreads / 32];
  for (int k = 0; k <= m; ++k) {
    double tot = 0.0;
    for (int v = 0; v < n; ++v) {
      double s = 0.0;
      for (int i = threadIdx.x; i < kDistBlocks; i += blockDim.x)
        s += part[((long long)v * kDistBlocks + i) * (kDistHist + 1) + k];
      s = block_sum(s, red);
      tot += s * irho.q[v];  // meaningful in thread 0
    }
    if (threadIdx.x == 0) sums[k] = tot;
  }
}

// t_new = w0 t + sum a_i x_i + beta (w0 r + sum a_i f_i)
__global__ void k_dist_anm_mix(long long count, const double *t, const double *r, Slots x,
                               Slots f, Charges alpha, int m, double w0, double beta,
                               double *tn) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    double xb = w0 * t[i], fb = w0 * r[i];
    for (int k = 0; k < m; ++k) {
      xb += alpha.q[k] * x.p[k][i];
      fb += alpha.q[k] * f.p[k][i];
    }
    tn[i] = xb + beta * fb;
  }
}

bool charges(int n, const double *qv, Charges &c) {
  if (n < 1 || n > kMaxSites || !qv) return false;
  for (int v = 0; v < n; ++v) c.q[v] = qv[v];
  return true;
}

}  // namespace

extern "C" int r3d_dist_closure(int device, int n, long long nloc, int closure, int pse_n,
                                const double *d_u, const double *d_t, const double *d_fr,
                                const double *qv, double *d_g, double *d_c, void *stream) {
  Charges q;
  if (!charges(n, qv, q) || nloc < 1 || !d_u || !d_t || !d_fr || !d_g || !d_c ||
      closure < R3D_KH || closure > R3D_PSE || pse_n < 1)
    return dist_fail(R3D_EINVAL, "closure: bad arguments");
  DeviceScope ds(device);
  if (ds.err != cudaSuccess) return dist_fail(R3D_ECUDA, cudaGetErrorString(ds.err));
  k_dist_closure<<<grid_for(n * nloc), kDistThreads, 0, (cudaStream_t)stream>>>(
      n, nloc, closure, pse_n, d_u, d_t, d_fr, q, d_g, d_c);
  return launched();
}

extern "C" int r3d_dist_oz(int device, int n, long long nk, const double *d_chi,
                           const double *d_fk, const double *qv, double *d_spec, void *stream) {
  Charges q;
  if (!charges(n, qv, q) || nk < 1 || !d_chi || !d_fk || !d_spec)
    return dist_fail(R3D_EINVAL, "oz: bad arguments");
  DeviceScope ds(device);
  if (ds.err != cudaSuccess) return dist_fail(R3D_ECUDA, cudaGetErrorString(ds.err));
  k_dist_oz<<<grid_for(nk), kDistThreads, 0, (cudaStream_t)stream>>>(
      n, nk, d_chi, (const double2 *)d_fk, q, (double2 *)d_spec);
  return launched();
}

extern "C" int r3d_dist_residual(int device, int n, long long nloc, double scale,
                                 const double *d_h, const double *d_g, const double *d_rp0,
                                 const double *d_rp1, int dots, double *d_r, double *d_sums,
                                 void *stream) {
  if (n < 1 || n > kMaxSites || nloc < 1 || !d_h || !d_g || !d_r || !d_sums ||
      (dots && (!d_rp0 || !d_rp1)))
    return dist_fail(R3D_EINVAL, "residual: bad arguments");
  DeviceScope ds(device);
  if (ds.err != cudaSuccess) return dist_fail(R3D_ECUDA, cudaGetErrorString(ds.err));
  cudaStream_t s = (cudaStream_t)stream;
  double *part = d_sums + 1 + 5 * kMaxSites;
  k_dist_residual<<<dim3(kDistBlocks, n), kDistThreads, 0, s>>>(nloc, scale, d_h, d_g, d_rp0,
                                                               d_rp1, dots, d_r, part);
  k_dist_sums<<<1, kDistThreads, 0, s>>>(n, part, d_sums);
  return launched();
}

extern "C" int r3d_dist_mix(int device, long long count, double *d_t, const double *d_r,
                            double *d_tp0, double *d_tp1, double *d_rp0, double *d_rp1,
                            int binary, int picard, double s1, double s2, double m,
                            void *stream) {
  if (count < 1 || !d_t || !d_r || !d_tp0 || !d_tp1 || !d_rp0 || !d_rp1 || binary < 0 ||
      binary > 1)
    return dist_fail(R3D_EINVAL, "mix: bad arguments");
  DeviceScope ds(device);
  if (ds.err != cudaSuccess) return dist_fail(R3D_ECUDA, cudaGetErrorString(ds.err));
  k_dist_mix<<<grid_for(count), kDistThreads, 0, (cudaStream_t)stream>>>(
      count, d_t, d_r, d_tp0, d_tp1, d_rp0, d_rp1, binary, picard, s1, s2, m);
  return launched();
}

extern "C" int r3d_dist_anm_dots(int device, int n, long long nloc, const double *d_r, int m,
                                 const double *const *d_hist, const double *irho,
                                 double *d_sums, void *stream) {
  Charges w;
  if (!charges(n, irho, w) || nloc < 1 || !d_r || !d_sums || m < 0 || m > kDistHist ||
      (m > 0 && !d_hist))
    return dist_fail(R3D_EINVAL, "anm_dots: bad arguments");
  Slots f{};
  for (int k = 0; k < m; ++k) {
    if (!d_hist[k]) return dist_fail(R3D_EINVAL, "anm_dots: NULL history slot");
    f.p[k] = d_hist[k];
  }
  DeviceScope ds(device);
  if (ds.err != cudaSuccess) return dist_fail(R3D_ECUDA, cudaGetErrorString(ds.err));
  cudaStream_t s = (cudaStream_t)stream;
  double *part = d_sums + 1 + kDistHist;
  k_dist_anm_dots<<<dim3(kDistBlocks, n), kDistThreads, 0, s>>>(nloc, d_r, f, m, part);
  k_dist_anm_sums<<<1, kDistThreads, 0, s>>>(n, m, w, part, d_sums);
  return launched();
}

extern "C" int r3d_dist_anm_mix(int device, long long count, const double *d_t,
                                const double *d_r, int m, const double *const *d_x,
                                const double *const *d_f, const double *alpha, double beta,
                                double *d_tn, void *stream) {
  Charges a{};
  if (count < 1 || !d_t || !d_r || !d_tn || m < 0 || m > kDistHist ||
      (m > 0 && (!d_x || !d_f || !alpha)))
    return dist_fail(R3D_EINVAL, "anm_mix: bad arguments");
  Slots x{}, f{};
  double w0 = 1.0;
  for (int k = 0; k < m; ++k) {
    if (!d_x[k] || !d_f[k]) return dist_fail(R3D_EINVAL, "anm_mix: NULL history slot");
    x.p[k] = d_x[k];
    f.p[k] = d_f[k];
    a.q[k] = alpha[k];
    w0 -= alpha[k];
  }
  DeviceScope ds(device);
  if (ds.err != cudaSuccess) return dist_fail(R3D_ECUDA, cudaGetErrorString(ds.err));
  k_dist_anm_mix<<<grid_for(count), kDistThreads, 0, (cudaStream_t)stream>>>(
      count, d_t, d_r, x, f, a, m, w0, beta, d_tn);
  return launched();
}
