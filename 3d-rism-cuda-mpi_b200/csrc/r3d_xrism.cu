// r3d_xrism.cu -- 1D XRISM solve of the bulk solvent on the GPU: the tables
// the reference reads as .xvk (src-cuda-mpi/solvent_read.cc:10-94) and ships
// without the program that makes them.
//
// Equations (extended RISM, Hirata and Rossky 1981; KH closure, Kovalenko
// and Hirata 1999; modified DIIS, Kovalenko, Ten-no and Hirata 1999), on the
// reader's site classes A = |sym| - 1 with representative atom rep(A):
//   W_AB(k) = sum_{b in B, same molecule as rep(A)} j0(k |r_rep(A) - r_b|)
//   D = diag(rhov), rhov[B] = sum of the class's atom densities
//   C(k) = C_s(k) - s^2 cc q_A q_B 4 pi e^{-k^2/4} / k^2      (erf(r)/r part)
//   H = (I - W C D)^-1 W C W^T,  T(k) = H_sym - C_s(k)
//   closure on t = h - c_s: g = closure(-u_LJ - s^2 cc q_A q_B erfc(r)/r + t)
//   xvv[A][B](k) = W_AB + rhov[B] H_AB           (calculate_cuda.cu:39-52)
// r_i = i dr, k_j = j pi/(N dr), i, j = 1..N-1; the transforms are discrete
// sine transforms on that pair of grids.
//
// Device layout (FP64): per-pair rows [p][Ns] (pairs A <= B, element 0 of a
// row unused and zero), a DIIS ring of H (t, f) rows, the best t of the
// stage, W as [A][B][Ns] (row j), and one control block.  One evaluation is
// five launches, captured in a CUDA graph a few evaluations at a time:
//   xr_mix   (wide)     t of the next evaluation: DIIS combination, the
//                       stage's best state (rollback) or nothing
//   xr_fwd   (per pair) closure -> r c_s(r) -> sine transform -> C_s(k)
//   xr_oz    (per k)    the natv x natv OZ solve -> k T(k)
//   xr_inv   (per pair) sine transform -> t_new(r) -> f = t_new - t
//   xr_dots  (wide)     <f, f_n> against the ring; the last CTA reduces,
//                       updates the Gram matrix, decides (converged, next
//                       stage, rollback, mix) and solves the DIIS system
// The sine transform of length N runs in one CTA: the half-length complex
// FFT of y_i = sin(pi i/N)(f_i + f_{N-i}) + (f_i - f_{N-i})/2 (N/2 points in
// shared memory, radix-2 decimation in frequency with up to four stages
// fused in registers), then S_{2m} = -Im Y_m and S_{2m+1} = S_{2m-1} + Re Y_m
// (a block scan).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rism3d_b200.h"
#include "r3d_internal.h"

namespace r3d {
void set_last_error(const std::string &m);  // r3d_last_error(NULL) reports it
}

namespace {

using namespace r3d;

constexpr int kXMaxV = 16;
constexpr int kXMaxP = kXMaxV * (kXMaxV + 1) / 2;
constexpr int kXMaxH = 31;    // DIIS entries: the bordered system fits one warp
constexpr int kXNT = 512;     // threads of the per-pair transform CTAs
constexpr int kXWide = 256;   // threads of the wide kernels
constexpr int kXMaxN = 16384;
constexpr int kXRollbacks = 8;
constexpr int kXChunk = 1024;  // elements per CTA of xr_dots

namespace phys {  // src-cuda-mpi/physical.h:5-14
constexpr double avogadro = 6.02214076e23;
constexpr double bohr = 0.5291771500001;
constexpr double boltzmann = 1.380649e-23;
constexpr double hartree = 4.359744722207185e-18;
}  // namespace phys

enum XMode : int { XM_NONE = 0, XM_MIX = 1, XM_ROLLBACK = 2 };

struct XCtl {
  int status;       // Status
  int steps;        // evaluations, all stages
  int stage_steps;  // evaluations of the current stage
  int stage;        // 1..nladder
  int head;         // ring slot of the next evaluation's t (and its f)
  int nh;           // DIIS entries held
  int mode;         // what xr_mix does before the next evaluation
  int save_best;    // xr_mix copies t of slot `best_src` into tb
  int best_src;
  int nsrc;
  int src[kXMaxH];
  int rollbacks;
  unsigned int counter;  // xr_dots CTAs done
  int err;
  double s2;    // charge scale squared of the stage
  double eta;   // DIIS step of the stage
  double best;  // best RMS of the stage
  double rms;
  double coef[kXMaxH];
  double gram[kXMaxH * kXMaxH];
};

struct XP {
  int N, Ns, M;  // points, row stride, N/2
  int P, nv, H, nladder, maxstep;
  int closure, pse_n;
  double tol, mix, dr, dk;
  double *ring_t, *ring_f, *tb;  // [H][P][Ns], [H][P][Ns], [P][Ns]
  const double *ulj, *uc;        // [P][Ns]
  const double *om;              // [nv][nv][Ns], row j = 1..N
  const double *cl;              // [Ns]
  const double2 *E;              // [N]: (cos, sin)(pi i / N)
  double2 *zf, *zi;              // [P][M]: packed inputs of the two transforms
  double *cs, *hk, *tn;          // [P][Ns]: C_s(k), H_sym(k), t_new(r)
  double *tkx;                   // [P][Ns]: k T(k) (generic OZ path only)
  double *c0;                    // [P]
  double *partials;              // [nblk_dots][32]
  int nblk_dots;
  XCtl *ctl;
  signed char pa[kXMaxP], pb[kXMaxP];
  double q[kXMaxV], rhov[kXMaxV];
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double xr_closure(int clos, int pse_n, double x) {
  if (clos == HNC || x <= 0.0) return exp(x);
  double term = 1.0, sum = 1.0;
  int n = clos == PSE ? pse_n : 1;
  for (int m = 1; m <= n; ++m) {
    term *= x / m;
    sum += term;
  }
  return sum;
}

__device__ __forceinline__ int zpad(int i) { return i + (i >> 5); }
__device__ __forceinline__ int dpad(int i) { return i + (i >> 5); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ bool xr_running(const XCtl *c) {
  return *(volatile const int *)&c->status == RUNNING;
}

// Pack the sine transform's input: y_i = s_i (a + b) + (a - b)/2 and
// y_{N-i} = s_i (a + b) - (a - b)/2 with a = f_i, b = f_{N-i}, s_i =
// sin(pi i/N), into z_n = y_{2n} + i y_{2n+1} (i and N - i have the same
// parity, so the same component).  i = 1..M; y_0 stays 0.
__device__ __forceinline__ void pack_pair(double2 *z, int N, int i, double s, double a, double b) {
  double *zd = (double *)z;
  const double sym = s * (a + b), asy = 0.5 * (a - b);
  const int h = i & 1;
  zd[2 * (i >> 1) + h] = sym + asy;
  if (2 * i != N) zd[2 * ((N - i) >> 1) + h] = sym - asy;
}

// q radix-2 decimation-in-frequency stages starting at span L, fused in
// registers: group g holds Z[base + e*S], e < 2^q, S = L / 2^q.  The
// twiddle of element e at stage t is e^{-2 pi i u / Lt} with u = j +
// (e mod 2^{q-t}) S: one table load per stage (e^{-2 pi i j / Lt}) times a
// 2^q-th root of unity held in registers.
template <int Q>
__device__ void fft_pass(double2 *Z, const double2 *tw, int lgM, int lgL) {
  constexpr int G = 1 << Q;
  const int lgS = lgL - Q;
  const int S = 1 << lgS;
  const int ngroups = 1 << (lgM - Q);
  double2 root[G / 2];  // e^{-2 pi i k / 2^Q}
#pragma unroll
  for (int k = 0; k < G / 2; ++k) root[k] = tw[k << (lgM - Q)];
  for (int g = threadIdx.x; g < ngroups; g += blockDim.x) {
    const int b = g >> lgS, j = g & (S - 1);
    const int base = (b << lgL) + j;
    double2 x[G];
#pragma unroll
    for (int e = 0; e < G; ++e) x[e] = Z[zpad(base + e * S)];
#pragma unroll
    for (int t = 0; t < Q; ++t) {
      const int d = G >> (t + 1);
      const double2 wj = tw[j << (lgM - lgL + t)];  // e^{-2 pi i j / Lt}
#pragma unroll
      for (int e = 0; e < G; ++e) {
        if (e & d) continue;
        const int k = (e & (2 * d - 1)) << t;  // (e mod 2^{Q-t}) 2^t
        const double2 w = k == 0 ? wj : cmul(wj, root[k]);
        const double2 a = x[e], c = x[e + d];
        x[e] = make_double2(a.x + c.x, a.y + c.y);
        x[e + d] = cmul(make_double2(a.x - c.x, a.y - c.y), w);
      }
    }
#pragma unroll
    for (int e = 0; e < G; ++e) Z[zpad(base + e * S)] = x[e];
  }
}

// Sine transform S_j = sum_{i=1}^{N-1} f_i sin(pi i j / N) of one row, in
// one CTA, from its packed input z (pack_pair; M = N/2 complex, global).
// On return F[dpad(j)] holds S_j (j = 1..N-1) in shared memory.  Shared
// memory: Z (M + M/32 complex), tw (M/2 complex); F aliases Z.
__device__ void sine_transform(const XP &p, const double2 *z, double2 *Z, double2 *tw,
                               double *F) {
  const int N = p.N, M = p.M, tid = threadIdx.x, nt = blockDim.x;
  {  // all loads in flight before the shared-memory stores
    double2 v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int n = tid + c * nt;
      if (n < M) v[c] = z[n];
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      const int n = tid + c * nt;
      if (n < M) Z[zpad(n)] = v[c];
    }
  }
  for (int k = tid; k < M / 2; k += nt) {  // e^{-2 pi i k / M} = conj E[4k]
    double2 e = p.E[4 * k];
    tw[k] = make_double2(e.x, -e.y);
  }
  __syncthreads();
  // log2(M) stages in passes of up to four
  const int lgM = 31 - __clz(M);
  for (int lgL = lgM; lgL > 0;) {
    const int q = lgL >= 4 ? 4 : lgL;
    if (q == 4) fft_pass<4>(Z, tw, lgM, lgL);
    else if (q == 3) fft_pass<3>(Z, tw, lgM, lgL);
    else if (q == 2) fft_pass<2>(Z, tw, lgM, lgL);
    else fft_pass<1>(Z, tw, lgM, lgL);
    __syncthreads();
    lgL -= q;
  }
  // Y_m = (Z_m + conj Z_{M-m})/2 + e^{-2 pi i m/N} (Z_m - conj Z_{M-m})/(2i);
  // Z is in bit-reversed order
  const int lg = lgM;
  const int C = (M + nt - 1) / nt;  // m per thread (<= 16 for M <= 8192)
  const int m0 = tid * C;
  double ry[16], iy[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    ry[c] = 0.0;
    iy[c] = 0.0;
    const int m = m0 + c;
    if (c < C && m < M) {
      const int mr = (int)(__brev((unsigned)m) >> (32 - lg));
      const int mc = (int)(__brev((unsigned)((M - m) & (M - 1))) >> (32 - lg));
      const double2 zm = Z[zpad(mr)], zc = Z[zpad(mc)];
      const double er = 0.5 * (zm.x + zc.x), ei = 0.5 * (zm.y - zc.y);
      const double orr = 0.5 * (zm.y + zc.y), oi = -0.5 * (zm.x - zc.x);
      const double2 e2 = p.E[2 * m];
      const double wr = e2.x, wi = -e2.y;
      ry[c] = er + (wr * orr - wi * oi);
      iy[c] = ei + (wr * oi + wi * orr);
    }
  }
  // S_{2m+1} = Re Y_0 / 2 + sum_{m'=1}^{m} Re Y_{m'}: chunk prefix + block scan
  double run = 0.0;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int m = m0 + c;
    if (c < C && m < M) {
      run += m == 0 ? 0.5 * ry[c] : ry[c];
      ry[c] = run;
    }
  }
  __shared__ double wsum[kXNT / 32];
  double incl = run;
  const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();  // also: every thread has read Z
  if (wid == 0) {
    double v = lane < nt / 32 ? wsum[lane] : 0.0;
    double w = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      double u = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += u;
    }
    if (lane < nt / 32) wsum[lane] = w - v;  // exclusive
  }
  __syncthreads();
  const double off = wsum[wid] + (incl - run);
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int m = m0 + c;
    if (c < C && m < M) {
      if (m > 0) F[dpad(2 * m)] = -iy[c];
      F[dpad(2 * m + 1)] = off + ry[c];
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------------ kernels
// t of the next evaluation at r_i and r_{N-i} (DIIS combination, the stage's
// best state, or the head slot as it is), the closure there and the packed
// input of the forward transform.  grid (M / 256, P).
__global__ void __launch_bounds__(kXWide) xr_mix(XP p) {
  XCtl *c = p.ctl;
  if (!xr_running(c)) return;
  __shared__ int s_mode, s_head, s_nsrc, s_save, s_best;
  __shared__ double s_eta, s_s2;
  __shared__ int s_src[kXMaxH];
  __shared__ double s_coef[kXMaxH];
  if (threadIdx.x == 0) {
    s_mode = c->mode;
    s_head = c->head;
    s_nsrc = c->nsrc;
    s_save = c->save_best;
    s_best = c->best_src;
    s_eta = c->eta;
    s_s2 = c->s2;
  }
  __syncthreads();
  if (threadIdx.x < s_nsrc && s_mode == XM_MIX) {
    s_src[threadIdx.x] = c->src[threadIdx.x];
    s_coef[threadIdx.x] = c->coef[threadIdx.x];
  }
  __syncthreads();
  const int pr = blockIdx.y;
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i > p.M) return;
  const size_t rows = (size_t)p.P * p.Ns, row = (size_t)pr * p.Ns;
  const int mode = s_mode, n = s_nsrc;
  const double eta = s_eta, s2 = s_s2;
  // i = M is its own mirror: one pass (a second would read the head slot
  // after this thread rewrote it)
  const int nh = i == p.M ? 1 : 2;
  double f[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (h >= nh) {
      f[1] = f[0];
      break;
    }
    const int q = h == 0 ? i : p.N - i;
    const size_t e = row + q;
    double t;
    if (mode == XM_NONE) {
      t = p.ring_t[(size_t)s_head * rows + e];
    } else if (mode == XM_ROLLBACK) {
      t = p.tb[e];
      p.ring_t[(size_t)s_head * rows + e] = t;
    } else {
      t = 0.0;
      for (int k = 0; k < n; ++k) {
        const size_t o = (size_t)s_src[k] * rows + e;
        t += s_coef[k] * (p.ring_t[o] + eta * p.ring_f[o]);
      }
      if (s_save) p.tb[e] = p.ring_t[(size_t)s_best * rows + e];
      // the head slot may be a source (ring full): read above already
      p.ring_t[(size_t)s_head * rows + e] = t;
    }
    const double g = xr_closure(p.closure, p.pse_n, -(p.ulj[e] + s2 * p.uc[e]) + t);
    f[h] = (q * p.dr) * (g - 1.0 - t);
  }
  pack_pair(p.zf + (size_t)pr * p.M, p.N, i, p.E[i].y, f[0], f[1]);
}

extern __shared__ __align__(16) unsigned char xr_smem[];

// forward transform of one pair: C_s(k_j) = 4 pi dr / k_j S_j[r c_s]
__global__ void __launch_bounds__(kXNT) xr_fwd(XP p) {
  if (!xr_running(p.ctl)) return;
  const int pr = blockIdx.x;
  double2 *Z = (double2 *)xr_smem;
  double2 *tw = Z + (p.M + (p.M >> 5));
  double *F = (double *)Z;
  sine_transform(p, p.zf + (size_t)pr * p.M, Z, tw, F);
  double *out = p.cs + (size_t)pr * p.Ns;
  const double sc = 4.0 * M_PI * p.dr / p.dk;
  for (int j = 1 + threadIdx.x; j < p.N; j += blockDim.x) out[j] = sc / j * F[dpad(j)];
}

// inverse transform of one pair: t_new(r_i) = dk / (2 pi^2 r_i) S_i[k T]
__global__ void __launch_bounds__(kXNT) xr_inv(XP p) {
  if (!xr_running(p.ctl)) return;
  const int pr = blockIdx.x;
  double2 *Z = (double2 *)xr_smem;
  double2 *tw = Z + (p.M + (p.M >> 5));
  double *F = (double *)Z;
  sine_transform(p, p.zi + (size_t)pr * p.M, Z, tw, F);
  double *out = p.tn + (size_t)pr * p.Ns;
  const double sc = p.dk / (2.0 * M_PI * M_PI * p.dr);
  for (int i = 1 + threadIdx.x; i < p.N; i += blockDim.x) out[i] = sc / i * F[dpad(i)];
}

// The OZ at one k for NV (compile time, <= 6) site classes, matrices in
// registers: h[pair] = H_sym(k_j).
template <int NV>
__device__ __forceinline__ void oz_point(const XP &p, int j, double s2, double *h) {
  constexpr int V = NV;
  constexpr int PP = NV * (NV + 1) / 2;
  const double clj = p.cl[j];
  double W[V][V], C[V][V], A[V][V], B[V][V];
#pragma unroll
  for (int a = 0; a < V; ++a)
#pragma unroll
    for (int b = 0; b < V; ++b) W[a][b] = p.om[((size_t)a * V + b) * p.Ns + j];
  {
    int pr = 0;
#pragma unroll
    for (int a = 0; a < V; ++a)
#pragma unroll
      for (int b = a; b < V; ++b, ++pr) {
        const double v = p.cs[(size_t)pr * p.Ns + j] + s2 * p.q[a] * p.q[b] * clj;
        C[a][b] = v;
        C[b][a] = v;
      }
  }
#pragma unroll
  for (int a = 0; a < V; ++a) {
    double wc[V];
#pragma unroll
    for (int b = 0; b < V; ++b) {
      double v = 0.0;
#pragma unroll
      for (int e = 0; e < V; ++e) v += W[a][e] * C[e][b];
      wc[b] = v;
      A[a][b] = (a == b ? 1.0 : 0.0) - v * p.rhov[b];
    }
#pragma unroll
    for (int b = 0; b < V; ++b) {
      double v = 0.0;
#pragma unroll
      for (int e = 0; e < V; ++e) v += wc[e] * W[b][e];
      B[a][b] = v;
    }
  }
  // Gaussian elimination with partial pivoting (row swaps by selects)
#pragma unroll
  for (int c = 0; c < V; ++c) {
    int piv = c;
    double best = fabs(A[c][c]);
#pragma unroll
    for (int r = c + 1; r < V; ++r)
      if (fabs(A[r][c]) > best) { best = fabs(A[r][c]); piv = r; }
#pragma unroll
    for (int r = c + 1; r < V; ++r) {
      if (r == piv) {
#pragma unroll
        for (int x = 0; x < V; ++x) {
          double t = A[c][x]; A[c][x] = A[r][x]; A[r][x] = t;
          t = B[c][x]; B[c][x] = B[r][x]; B[r][x] = t;
        }
      }
    }
    const double inv = 1.0 / A[c][c];
#pragma unroll
    for (int r = c + 1; r < V; ++r) {
      const double m = A[r][c] * inv;
#pragma unroll
      for (int x = 0; x < V; ++x) {
        if (x >= c) A[r][x] -= m * A[c][x];
        B[r][x] -= m * B[c][x];
      }
    }
  }
#pragma unroll
  for (int c = V - 1; c >= 0; --c) {
#pragma unroll
    for (int x = 0; x < V; ++x) {
      double s = B[c][x];
#pragma unroll
      for (int y = c + 1; y < V; ++y) s -= A[c][y] * B[y][x];
      B[c][x] = s / A[c][c];
    }
  }
  {
    int pr = 0;
#pragma unroll
    for (int a = 0; a < V; ++a)
#pragma unroll
      for (int b = a; b < V; ++b, ++pr) h[pr] = 0.5 * (B[a][b] + B[b][a]);
    (void)PP;
  }
}

// OZ at k_j and k_{N-j} per thread (j = 1..M), H_sym stored for the table,
// T = H_sym - C_s packed (times k) as the inverse transform's input.
template <int NV>
__global__ void __launch_bounds__(128) xr_oz(XP p) {
  if (!xr_running(p.ctl)) return;
  const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j > p.M) return;
  constexpr int PP = NV * (NV + 1) / 2;
  const double s2 = p.ctl->s2;
  const int j2 = p.N - j;
  double h1[PP], h2[PP];
  oz_point<NV>(p, j, s2, h1);
  if (j2 != j) oz_point<NV>(p, j2, s2, h2);
  const double s = p.E[j].y;
#pragma unroll
  for (int pr = 0; pr < PP; ++pr) {
    const size_t o = (size_t)pr * p.Ns;
    const double a = j * p.dk * (h1[pr] - p.cs[o + j]);
    p.hk[o + j] = h1[pr];
    double b = a;
    if (j2 != j) {
      b = j2 * p.dk * (h2[pr] - p.cs[o + j2]);
      p.hk[o + j2] = h2[pr];
    }
    pack_pair(p.zi + (size_t)pr * p.M, p.N, j, s, a, b);
  }
}

// The same for any nv <= 16, one k per thread, rolled loops (matrices in
// local memory); k T(k) goes to tkx and xr_pack_inv packs it.
__global__ void __launch_bounds__(128) xr_oz_any(XP p) {
  if (!xr_running(p.ctl)) return;
  const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= p.N) return;
  const int nv = p.nv;
  const double k = j * p.dk, s2 = p.ctl->s2, clj = p.cl[j];
  double W[kXMaxV][kXMaxV], C[kXMaxV][kXMaxV], A[kXMaxV][kXMaxV], B[kXMaxV][kXMaxV];
#pragma unroll 1
  for (int a = 0; a < nv; ++a)
#pragma unroll 1
    for (int b = 0; b < nv; ++b) W[a][b] = p.om[((size_t)a * nv + b) * p.Ns + j];
#pragma unroll 1
  for (int pr = 0; pr < p.P; ++pr) {
    const int a = p.pa[pr], b = p.pb[pr];
    const double v = p.cs[(size_t)pr * p.Ns + j] + s2 * p.q[a] * p.q[b] * clj;
    C[a][b] = v;
    C[b][a] = v;
  }
#pragma unroll 1
  for (int a = 0; a < nv; ++a) {
    double wc[kXMaxV];
#pragma unroll 1
    for (int b = 0; b < nv; ++b) {
      double v = 0.0;
#pragma unroll 1
      for (int e = 0; e < nv; ++e) v += W[a][e] * C[e][b];
      wc[b] = v;
      A[a][b] = (a == b ? 1.0 : 0.0) - v * p.rhov[b];
    }
#pragma unroll 1
    for (int b = 0; b < nv; ++b) {
      double v = 0.0;
#pragma unroll 1
      for (int e = 0; e < nv; ++e) v += wc[e] * W[b][e];
      B[a][b] = v;
    }
  }
#pragma unroll 1
  for (int c = 0; c < nv; ++c) {
    int piv = c;
#pragma unroll 1
    for (int r = c + 1; r < nv; ++r)
      if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
    if (piv != c) {
#pragma unroll 1
      for (int x = 0; x < nv; ++x) {
        double t = A[c][x]; A[c][x] = A[piv][x]; A[piv][x] = t;
        t = B[c][x]; B[c][x] = B[piv][x]; B[piv][x] = t;
      }
    }
    const double inv = 1.0 / A[c][c];
#pragma unroll 1
    for (int r = c + 1; r < nv; ++r) {
      const double m = A[r][c] * inv;
#pragma unroll 1
      for (int x = c; x < nv; ++x) A[r][x] -= m * A[c][x];
#pragma unroll 1
      for (int x = 0; x < nv; ++x) B[r][x] -= m * B[c][x];
    }
  }
#pragma unroll 1
  for (int c = nv - 1; c >= 0; --c)
#pragma unroll 1
    for (int x = 0; x < nv; ++x) {
      double s = B[c][x];
#pragma unroll 1
      for (int y = c + 1; y < nv; ++y) s -= A[c][y] * B[y][x];
      B[c][x] = s / A[c][c];
    }
#pragma unroll 1
  for (int pr = 0; pr < p.P; ++pr) {
    const int a = p.pa[pr], b = p.pb[pr];
    const size_t o = (size_t)pr * p.Ns + j;
    const double h = 0.5 * (B[a][b] + B[b][a]);
    p.hk[o] = h;
    p.tkx[o] = k * (h - p.cs[o]);
  }
}

// packs tkx into the inverse transform's input (generic OZ path); grid
// (M / 256, P)
__global__ void __launch_bounds__(kXWide) xr_pack_inv(XP p) {
  if (!xr_running(p.ctl)) return;
  const int pr = blockIdx.y;
  const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j > p.M) return;
  const double *t = p.tkx + (size_t)pr * p.Ns;
  pack_pair(p.zi + (size_t)pr * p.M, p.N, j, p.E[j].y, t[j], t[p.N - j]);
}

// bordered DIIS system [G 1; 1^T 0] c = e_n (order m = n + 1 <= 32) by one
// warp, without block barriers: row r lives in the registers of lane r
// (columns unrolled, so every index is static); partial pivoting leaves the
// rows in place and publishes each column's pivot row to shared memory, one
// reciprocal per column; the back substitution reads the pivot rows there.
// G: the Gram matrix of the n entries (oldest first), stride 33.  Called by
// warp 0 (all 32 lanes).
__device__ void diis_solve_warp(const double *G, int n, double *coef) {
  __shared__ double Pv[kXMaxH + 1][33];  // pivot row of each column; [32] = rhs
  const int lane = threadIdx.x & 31;
  const int m = n + 1;
  double sc = 0.0;
  for (int i = 0; i < n; ++i) sc = fmax(sc, G[i * 33 + i]);
  sc = sc > 0.0 ? 1.0 / sc : 1.0;
  double row[32];
#pragma unroll
  for (int x = 0; x < 32; ++x) {
    double v = 0.0;
    if (lane < m && x < m) {
      if (lane < n && x < n) v = G[lane * 33 + x] * sc;
      else if (lane < n || x < n) v = 1.0;  // the border; the corner is 0
    }
    row[x] = v;
  }
  double rhs = lane == n ? 1.0 : 0.0;
  bool used = lane >= m;  // lanes past the system never pivot
  bool ok = true;
#pragma unroll
  for (int col = 0; col < 32; ++col) {
    if (col >= m) break;
    double best = used ? -1.0 : fabs(row[col]);
    int bl = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int ol = __shfl_xor_sync(0xffffffffu, bl, o);
      if (ob > best || (ob == best && ol < bl)) { best = ob; bl = ol; }
    }
    if (!(best > 1e-300)) {  // the same in every lane
      ok = false;
      break;
    }
    if (lane == bl) {
      used = true;
#pragma unroll
      for (int x = 0; x < 32; ++x)
        if (x >= col) Pv[col][x] = row[x];
      Pv[col][32] = rhs;
    }
    __syncwarp();
    if (!used) {
      const double mult = row[col] / Pv[col][col];
#pragma unroll
      for (int x = 0; x < 32; ++x)
        if (x > col) row[x] -= mult * Pv[col][x];
      rhs -= mult * Pv[col][32];
    }
  }
  __syncwarp();
  double sol = 0.0;
  if (ok) {
    for (int col = m - 1; col >= 0; --col) {
      double term = (lane > col && lane < m) ? Pv[col][lane] * sol : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) term += __shfl_xor_sync(0xffffffffu, term, o);
      const double v = (Pv[col][32] - term) / Pv[col][col];
      if (lane == col) sol = v;
    }
  }
  const bool fin = __all_sync(0xffffffffu, ok && (lane >= n || isfinite(sol)));
  if (lane < n) coef[lane] = fin ? sol : (lane == n - 1 ? 1.0 : 0.0);
}

// f = t_new - t of the evaluation into the ring, <f, f_n> against the ring
// entries in one pass; the last CTA reduces (fixed order), updates the Gram
// matrix, decides (converged, next stage, rollback, mix) and solves the
// DIIS system.  Every CTA stages the control fields and the Gram block at
// its start, so the last one finds them in shared memory.
__global__ void __launch_bounds__(kXWide) xr_dots(XP p) {
  XCtl *c = p.ctl;
  if (!xr_running(c)) return;
  const int H = p.H;
  __shared__ int s_head, s_nn, s_stage, s_stage_steps, s_rollbacks;
  __shared__ double s_best, s_eta;
  __shared__ int slot[kXMaxH];
  __shared__ double G[32 * 33];  // Gram of the nn entries, oldest first
  __shared__ double dots[kXMaxH];
  __shared__ bool last;
  if (threadIdx.x == 0) {
    s_head = c->head;
    s_nn = c->nh < H ? c->nh + 1 : H;  // entries after the push
    s_stage = c->stage;
    s_stage_steps = c->stage_steps;
    s_rollbacks = c->rollbacks;
    s_best = c->best;
    s_eta = c->eta;
  }
  __syncthreads();
  const int head = s_head, nn = s_nn;
  if (threadIdx.x < nn) slot[threadIdx.x] = (head - (nn - 1) + (int)threadIdx.x + H) % H;
  __syncthreads();
  for (int e = threadIdx.x; e < nn * nn; e += blockDim.x) {
    const int a = e / nn, b = e - a * nn;
    G[a * 33 + b] = c->gram[slot[a] * H + slot[b]];
  }
  // this CTA's chunk of kXChunk elements: f = t_new - t into the ring and
  // into shared memory, then warp w dots the chunk with entries w, w + 8, ...
  // (coalesced rows, every load of a lane independent of the others)
  const size_t rows = (size_t)p.P * p.Ns;
  const size_t e0 = (size_t)blockIdx.x * kXChunk;
  const double *t0 = p.ring_t + (size_t)head * rows;
  double *f0 = p.ring_f + (size_t)head * rows;
  __shared__ double fs[kXChunk];
  for (int k = threadIdx.x; k < kXChunk; k += blockDim.x) {
    const size_t e = e0 + k;
    double f = 0.0;
    if (e < rows) {
      f = p.tn[e] - t0[e];  // zero on the unused row elements
      f0[e] = f;
    }
    fs[k] = f;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int n = wid; n < nn; n += kXWide / 32) {
    const double *fn = p.ring_f + (size_t)slot[n] * rows + e0;
    double acc = 0.0;
    if (n == nn - 1) {  // the newest entry is this evaluation's f
#pragma unroll 8
      for (int k = lane; k < kXChunk; k += 32) acc += fs[k] * fs[k];
    } else {
#pragma unroll 8
      for (int k = lane; k < kXChunk; k += 32)
        if (e0 + k < rows) acc += fs[k] * fn[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) p.partials[(size_t)blockIdx.x * 32 + n] = acc;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&c->counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // ---- the last CTA
  {  // 8 threads per entry sum the partials of all CTAs (fixed order)
    const int n = threadIdx.x >> 3, part = threadIdx.x & 7;
    double s = 0.0;
    if (n < nn)
      for (int b = part; b < p.nblk_dots; b += 8)
        s += ((volatile double *)p.partials)[(size_t)b * 32 + n];
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, 8);
    if (part == 0 && n < nn) dots[n] = s;
  }
  __syncthreads();
  if (threadIdx.x < nn) {  // the newest entry's row and column
    const double d = dots[threadIdx.x];
    G[(nn - 1) * 33 + threadIdx.x] = d;
    G[threadIdx.x * 33 + nn - 1] = d;
    c->gram[head * H + slot[threadIdx.x]] = d;
    c->gram[slot[threadIdx.x] * H + head] = d;
  }
  __syncthreads();
  __shared__ int decide;  // 0 stop, 1 next stage, 2 rollback, 3 mix
  if (threadIdx.x == 0) {
    c->counter = 0;
    const double err = sqrt(G[(nn - 1) * 33 + nn - 1] / ((double)p.P * (p.N - 1)));
    const int stage = s_stage;
    const int stage_steps = s_stage_steps + 1;
    const double best = s_best;
    c->rms = err;
    c->steps += 1;
    c->stage_steps = stage_steps;
    c->save_best = 0;
    const double stol = stage == p.nladder ? p.tol : fmax(p.tol, 1e-5);
    int dcs = 3;
    if (err < stol) {
      if (stage == p.nladder) {
        c->status = CONVERGED;
        dcs = 0;
      } else {  // next stage from this t, fresh history
        const double s = (double)(stage + 1) / p.nladder;
        c->stage = stage + 1;
        c->s2 = s * s;
        c->stage_steps = 0;
        c->best = INFINITY;
        c->eta = p.mix;
        c->rollbacks = 0;
        c->nh = 0;
        c->mode = XM_NONE;
        dcs = 1;
      }
    } else if (stage_steps >= p.maxstep) {
      c->status = MAXSTEP;
      dcs = 0;
    } else if (!(err <= 10.0 * best)) {
      const int rb = s_rollbacks + 1;
      c->rollbacks = rb;
      if (!isfinite(best) || rb > kXRollbacks) {
        c->status = DIVERGED;
        dcs = 0;
      } else {
        c->mode = XM_ROLLBACK;
        c->nh = 0;
        c->eta = 0.5 * s_eta;
        c->head = (head + 1) % H;
        dcs = 2;
      }
    } else {
      if (err < best) {
        c->best = err;
        c->save_best = 1;
        c->best_src = head;
      }
      c->nh = nn;
      c->nsrc = nn;
      c->mode = XM_MIX;
      c->head = (head + 1) % H;
    }
    decide = dcs;
  }
  __syncthreads();
  if (decide == 3 && threadIdx.x < 32) {
    if (threadIdx.x < nn) c->src[threadIdx.x] = slot[threadIdx.x];
    diis_solve_warp(G, nn, c->coef);
  }
}

// c_s(k=0) = 4 pi dr sum r^2 c_s(r) of each pair at the converged t (full
// charges), for the compressibility; one CTA per pair
__global__ void __launch_bounds__(kXWide) xr_c0(XP p) {
  const int pr = blockIdx.x;
  const size_t e0 = (size_t)p.ctl->head * p.P * p.Ns + (size_t)pr * p.Ns;
  const size_t u0 = (size_t)pr * p.Ns;
  double acc = 0.0;
  for (int i = 1 + threadIdx.x; i < p.N; i += blockDim.x) {
    const double t = p.ring_t[e0 + i];
    const double g = xr_closure(p.closure, p.pse_n, -(p.ulj[u0 + i] + p.uc[u0 + i]) + t);
    const double r = i * p.dr;
    acc += r * r * (g - 1.0 - t);
  }
  __shared__ double red[kXWide / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    p.c0[pr] = 4.0 * M_PI * p.dr * s;
  }
}

// table rows j = 1..N: xvv[j-1][A][B] = W_AB + rhov[B] H_AB (row N: W)
__global__ void xr_table(XP p, double *xvv) {
  const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j > p.N) return;
  const int nv = p.nv;
  for (int a = 0; a < nv; ++a)
    for (int b = 0; b < nv; ++b) {
      double v = p.om[((size_t)a * nv + b) * p.Ns + j];
      if (j < p.N) {
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        const int pr = lo * nv - lo * (lo - 1) / 2 + (hi - lo);
        v += p.rhov[b] * p.hk[(size_t)pr * p.Ns + j];
      }
      xvv[((size_t)(j - 1) * nv + a) * nv + b] = v;
    }
}

// ------------------------------------------------------------------- host
int xfail(int code, const std::string &m) {
  set_last_error("xrism: " + m);
  return code;
}

#define XCK(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      rc = xfail(R3D_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
      goto done;                                                              \
    }                                                                         \
  } while (0)

template <int NV>
void launch_oz_nv(const XP &p, cudaStream_t st) {
  xr_oz<NV><<<(p.M + 127) / 128, 128, 0, st>>>(p);
}

void launch_oz(const XP &p, cudaStream_t st) {
  switch (p.nv) {
    case 1: launch_oz_nv<1>(p, st); break;
    case 2: launch_oz_nv<2>(p, st); break;
    case 3: launch_oz_nv<3>(p, st); break;
    case 4: launch_oz_nv<4>(p, st); break;
    case 5: launch_oz_nv<5>(p, st); break;
    case 6: launch_oz_nv<6>(p, st); break;
    default:
      xr_oz_any<<<(p.N - 1 + 127) / 128, 128, 0, st>>>(p);
      xr_pack_inv<<<dim3((p.M + kXWide - 1) / kXWide, p.P), kXWide, 0, st>>>(p);
      break;
  }
}

size_t transform_smem(int M) {
  return sizeof(double2) * ((size_t)M + (M >> 5) + M / 2);
}

// one evaluation: 5 launches (6 for more than six site classes)
void enqueue_eval(const XP &p, cudaStream_t st) {
  xr_mix<<<dim3((p.M + kXWide - 1) / kXWide, p.P), kXWide, 0, st>>>(p);
  xr_fwd<<<p.P, kXNT, transform_smem(p.M), st>>>(p);
  launch_oz(p, st);
  xr_inv<<<p.P, kXNT, transform_smem(p.M), st>>>(p);
  xr_dots<<<p.nblk_dots, kXWide, 0, st>>>(p);
}

std::string check_atoms(const r3d_xrism_atom *at, int natom, int &nv, int *rep) {
  if (!at || natom < 1) return "no atoms";
  nv = 0;
  for (int i = 0; i < natom; ++i) nv = std::max(nv, std::abs(at[i].sym));
  if (nv < 1 || nv > kXMaxV) return "site classes (|sym|) must be 1.." + std::to_string(kXMaxV);
  for (int a = 0; a < nv; ++a) rep[a] = -1;
  for (int i = 0; i < natom; ++i) {
    const int a = std::abs(at[i].sym) - 1;
    if (a < 0) return "atom " + std::to_string(i) + " has sym 0";
    if (rep[a] < 0) {
      rep[a] = i;
      continue;
    }
    const r3d_xrism_atom &r = at[rep[a]];
    if (at[i].species != r.species || at[i].sigma != r.sigma || at[i].epsilon != r.epsilon ||
        at[i].charge != r.charge || at[i].density != r.density)
      return "atoms of site class " + std::to_string(a + 1) +
             " differ in species, LJ, charge or density";
  }
  for (int a = 0; a < nv; ++a)
    if (rep[a] < 0) return "site class " + std::to_string(a + 1) + " has no atom";
  for (int i = 0; i < natom; ++i)
    if (!(at[i].density >= 0.0) || !(at[i].sigma >= 0.0) || !(at[i].epsilon >= 0.0))
      return "negative density, sigma or epsilon";
  return "";
}

}  // namespace

extern "C" {

void r3d_xrism_default_opts(r3d_xrism_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->ntab = 8192;
  o->dr = 0.05;
  o->temperature = 298.15;
  o->closure = R3D_KH;
  o->pse_n = 1;
  o->tol = 1e-10;
  o->maxstep = 10000;
  o->history = 20;
  o->mix = 0.3;
  o->nladder = 5;
  o->verbose = 0;
}

int r3d_xrism_solve(const r3d_xrism_opts *opts, const r3d_xrism_atom *atoms, int natom,
                    double *xvv, r3d_xrism_result *res) {
  if (!opts || !res) return xfail(R3D_EINVAL, "null opts or result");
  std::memset(res, 0, sizeof(*res));
  const r3d_xrism_opts &o = *opts;
  const int N = o.ntab;
  if (N < 64 || N > kXMaxN || (N & (N - 1)))
    return xfail(R3D_EINVAL, "ntab must be a power of two in [64, " + std::to_string(kXMaxN) + "]");
  if (!(o.dr > 0.0) || !(o.temperature > 0.0) || !(o.tol > 0.0) || !(o.mix > 0.0))
    return xfail(R3D_EINVAL, "dr, temperature, tol and mix must be positive");
  if (o.history < 1 || o.history > kXMaxH)
    return xfail(R3D_EINVAL, "history must be 1.." + std::to_string(kXMaxH));
  if (o.nladder < 1 || o.maxstep < 1) return xfail(R3D_EINVAL, "nladder and maxstep must be >= 1");
  if (o.closure != R3D_KH && o.closure != R3D_HNC && o.closure != R3D_PSE)
    return xfail(R3D_EINVAL, "unknown closure");
  if (o.closure == R3D_PSE && (o.pse_n < 1 || o.pse_n > 10))
    return xfail(R3D_EINVAL, "pse_n must be 1..10");
  int nv = 0, rep[kXMaxV];
  {
    std::string m = check_atoms(atoms, natom, nv, rep);
    if (!m.empty()) return xfail(R3D_EINVAL, m);
  }
  const int P = nv * (nv + 1) / 2, H = o.history;
  const int Ns = N + 64;  // row stride off the power of two
  const int M = N / 2;
  const double dk = M_PI / (N * o.dr);
  const double kT = phys::boltzmann * o.temperature;
  const double cc = phys::hartree * phys::bohr / kT;
  const double rt = phys::avogadro * kT;

  // host tables
  std::vector<double> ulj((size_t)P * Ns, 0.0), uc((size_t)P * Ns, 0.0);
  std::vector<double> om((size_t)nv * nv * Ns, 0.0), cl(Ns, 0.0);
  std::vector<double2> E(N);
  XP p;
  std::memset(&p, 0, sizeof(p));
  for (int a = 0, pr = 0; a < nv; ++a)
    for (int b = a; b < nv; ++b, ++pr) {
      p.pa[pr] = (signed char)a;
      p.pb[pr] = (signed char)b;
      const r3d_xrism_atom &x = atoms[rep[a]], &y = atoms[rep[b]];
      const double s = 0.5 * (x.sigma + y.sigma), e = std::sqrt(x.epsilon * y.epsilon);
      for (int i = 1; i < N; ++i) {
        const double r = i * o.dr, sr6 = std::pow(s / r, 6);
        ulj[(size_t)pr * Ns + i] = 4.0 * e * (sr6 * sr6 - sr6) / rt;
        uc[(size_t)pr * Ns + i] = cc * x.charge * y.charge * std::erfc(r) / r;
      }
    }
  for (int a = 0; a < nv; ++a) {
    const r3d_xrism_atom &x = atoms[rep[a]];
    p.q[a] = x.charge;
    for (int i = 0; i < natom; ++i) {
      if (atoms[i].species != x.species) continue;
      const int b = std::abs(atoms[i].sym) - 1;
      const double dx = x.x - atoms[i].x, dy = x.y - atoms[i].y, dz = x.z - atoms[i].z;
      const double l = std::sqrt(dx * dx + dy * dy + dz * dz);
      for (int j = 1; j <= N; ++j) {
        const double k = j * dk;
        om[((size_t)a * nv + b) * Ns + j] += (i == rep[a] || l == 0.0) ? 1.0 : std::sin(k * l) / (k * l);
      }
    }
  }
  for (int i = 0; i < natom; ++i)
    p.rhov[std::abs(atoms[i].sym) - 1] += atoms[i].density * phys::avogadro * 1.0e-27;
  for (int j = 1; j < N; ++j) {
    const double k = j * dk;
    cl[j] = -cc * 4.0 * M_PI * std::exp(-0.25 * k * k) / (k * k);
  }
  for (int i = 0; i < N; ++i) E[i] = make_double2(std::cos(M_PI * i / N), std::sin(M_PI * i / N));

  int rc = R3D_OK;
  cudaStream_t st = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  char *dmem = nullptr;
  XCtl *hctl = nullptr;
  const int nblk_dots =
      std::max(1, (int)(((size_t)P * Ns + kXChunk - 1) / kXChunk));
  const size_t rowsz = (size_t)P * Ns * sizeof(double);
  const size_t zsz = (size_t)P * M * sizeof(double2);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o2 = off;
    off += (bytes + 255) & ~(size_t)255;
    return o2;
  };
  const size_t o_rt = take((size_t)H * rowsz), o_rf = take((size_t)H * rowsz), o_tb = take(rowsz),
               o_ulj = take(rowsz), o_uc = take(rowsz),
               o_om = take((size_t)nv * nv * Ns * sizeof(double)), o_cl = take(Ns * sizeof(double)),
               o_E = take(N * sizeof(double2)), o_zf = take(zsz), o_zi = take(zsz),
               o_cs = take(rowsz), o_hk = take(rowsz), o_tn = take(rowsz),
               o_tkx = take(nv > 6 ? rowsz : 256), o_c0 = take(P * sizeof(double)),
               o_part = take((size_t)nblk_dots * 32 * sizeof(double)),
               o_ctl = take(sizeof(XCtl)),
               o_tab = take((size_t)N * nv * nv * sizeof(double));
  const size_t smem = transform_smem(M);
  XCtl c0;
  std::vector<double> c0h(P);
  float ms = 0.f;
  const int per_graph = 8;
  long long max_evals = (long long)o.maxstep * o.nladder;

  int prev_device = -1;
  XCK(cudaGetDevice(&prev_device));
  XCK(cudaSetDevice(o.device));
  XCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  XCK(cudaMalloc(&dmem, off));
  XCK(cudaMallocHost(&hctl, sizeof(XCtl)));
  XCK(cudaMemsetAsync(dmem, 0, off, st));
  p.N = N;
  p.Ns = Ns;
  p.M = M;
  p.P = P;
  p.nv = nv;
  p.H = H;
  p.nladder = o.nladder;
  p.maxstep = o.maxstep;
  p.closure = o.closure;
  p.pse_n = o.closure == R3D_PSE ? o.pse_n : 1;
  p.tol = o.tol;
  p.mix = o.mix;
  p.dr = o.dr;
  p.dk = dk;
  p.ring_t = (double *)(dmem + o_rt);
  p.ring_f = (double *)(dmem + o_rf);
  p.tb = (double *)(dmem + o_tb);
  p.ulj = (const double *)(dmem + o_ulj);
  p.uc = (const double *)(dmem + o_uc);
  p.om = (const double *)(dmem + o_om);
  p.cl = (const double *)(dmem + o_cl);
  p.E = (const double2 *)(dmem + o_E);
  p.zf = (double2 *)(dmem + o_zf);
  p.zi = (double2 *)(dmem + o_zi);
  p.cs = (double *)(dmem + o_cs);
  p.hk = (double *)(dmem + o_hk);
  p.tn = (double *)(dmem + o_tn);
  p.tkx = (double *)(dmem + o_tkx);
  p.c0 = (double *)(dmem + o_c0);
  p.partials = (double *)(dmem + o_part);
  p.nblk_dots = nblk_dots;
  p.ctl = (XCtl *)(dmem + o_ctl);
  XCK(cudaMemcpyAsync(dmem + o_ulj, ulj.data(), rowsz, cudaMemcpyHostToDevice, st));
  XCK(cudaMemcpyAsync(dmem + o_uc, uc.data(), rowsz, cudaMemcpyHostToDevice, st));
  XCK(cudaMemcpyAsync(dmem + o_om, om.data(), om.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  XCK(cudaMemcpyAsync(dmem + o_cl, cl.data(), cl.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  XCK(cudaMemcpyAsync(dmem + o_E, E.data(), E.size() * sizeof(double2), cudaMemcpyHostToDevice, st));
  std::memset(&c0, 0, sizeof(c0));
  c0.status = RUNNING;
  c0.stage = 1;
  {
    const double s = 1.0 / o.nladder;
    c0.s2 = s * s;
  }
  c0.eta = o.mix;
  c0.best = INFINITY;
  c0.mode = XM_NONE;
  XCK(cudaMemcpyAsync(p.ctl, &c0, sizeof(c0), cudaMemcpyHostToDevice, st));
  XCK(cudaFuncSetAttribute(xr_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  XCK(cudaFuncSetAttribute(xr_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  XCK(cudaEventCreate(&ev0));
  XCK(cudaEventCreate(&ev1));
  XCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  for (int r = 0; r < per_graph; ++r) enqueue_eval(p, st);
  XCK(cudaStreamEndCapture(st, &graph));
  XCK(cudaGraphInstantiate(&gexec, graph, 0));
  XCK(cudaEventRecord(ev0, st));
  for (long long done_evals = 0;; done_evals += per_graph) {
    XCK(cudaGraphLaunch(gexec, st));
    XCK(cudaMemcpyAsync(hctl, p.ctl, sizeof(XCtl), cudaMemcpyDeviceToHost, st));
    XCK(cudaStreamSynchronize(st));
    if (o.verbose)
      std::printf(" xrism stage %d step %d rms %.6e\n", hctl->stage, hctl->steps, hctl->rms);
    if (hctl->status != RUNNING) break;
    if (done_evals > max_evals + per_graph) {  // bounded on the host too
      rc = xfail(R3D_ECUDA, "iteration control did not stop");
      goto done;
    }
  }
  XCK(cudaEventRecord(ev1, st));
  XCK(cudaEventSynchronize(ev1));
  XCK(cudaEventElapsedTime(&ms, ev0, ev1));
  res->natv = nv;
  res->steps = hctl->steps;
  res->rms = hctl->rms;
  res->ms_device = ms;
  res->status = hctl->status == CONVERGED ? R3D_CONVERGED
                : hctl->status == DIVERGED ? R3D_DIVERGED
                                           : R3D_MAXSTEP;
  res->xt = NAN;
  if (hctl->status == CONVERGED) {
    double *dtab = (double *)(dmem + o_tab);
    xr_c0<<<P, kXWide, 0, st>>>(p);
    xr_table<<<(N + 127) / 128, 128, 0, st>>>(p, dtab);
    XCK(cudaGetLastError());
    if (xvv)
      XCK(cudaMemcpyAsync(xvv, dtab, (size_t)N * nv * nv * sizeof(double), cudaMemcpyDeviceToHost, st));
    XCK(cudaMemcpyAsync(c0h.data(), p.c0, P * sizeof(double), cudaMemcpyDeviceToHost, st));
    XCK(cudaStreamSynchronize(st));
    // isothermal compressibility: 1/(kT (sum_species rho_s - sum_AB rhov_A rhov_B c_s,AB(0)))
    double rs = 0.0, scs = 0.0;
    for (int i = 0; i < natom; ++i) {
      bool first = true;
      for (int j = 0; j < i; ++j)
        if (atoms[j].species == atoms[i].species) first = false;
      if (first) rs += atoms[i].density * phys::avogadro * 1.0e-27;
    }
    for (int a = 0; a < nv; ++a)
      for (int b = 0; b < nv; ++b) {
        const int lo = std::min(a, b), hi = std::max(a, b);
        const int pr = lo * nv - lo * (lo - 1) / 2 + (hi - lo);
        scs += p.rhov[a] * p.rhov[b] * c0h[pr];
      }
    res->xt = 1.0 / (kT * 1.0e30 * (rs - scs));
  }
done:
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (st) cudaStreamSynchronize(st);
  if (dmem) cudaFree(dmem);
  if (hctl) cudaFreeHost(hctl);
  if (st) cudaStreamDestroy(st);
  if (prev_device >= 0) cudaSetDevice(prev_device);  // the caller's current device
  return rc;
}

int r3d_xrism_read_deck(const char *path, r3d_xrism_atom *atoms, int max_atoms, int *natom,
                        r3d_xrism_opts *opts) {
  if (!path || !atoms || !natom || !opts) return xfail(R3D_EINVAL, "null argument");
  std::ifstream f(path);
  if (!f) return xfail(R3D_EIO, std::string("cannot open ") + path);
  std::vector<std::string> lines;
  for (std::string l; std::getline(f, l) && lines.size() < 4096;) lines.push_back(l);
  if (lines.size() < 5) return xfail(R3D_EINVAL, std::string("truncated deck ") + path);
  // solvent_read.cc:33-49: "## num natv ntab dr dk", "## nspec T xt", atoms
  int num = 0, natv = 0, ntab = 0;
  double dr = 0, temper = 0;
  {
    std::istringstream h(lines[1]);
    std::string d;
    if (!(h >> d >> num >> natv >> ntab >> dr)) return xfail(R3D_EINVAL, "bad header line 2");
    std::istringstream h2(lines[2]);
    int ns;
    if (!(h2 >> d >> ns >> temper)) return xfail(R3D_EINVAL, "bad header line 3");
  }
  if (num < 1 || num > max_atoms || (int)lines.size() < 4 + num)
    return xfail(R3D_EINVAL, "atom count " + std::to_string(num) + " out of range");
  for (int i = 0; i < num; ++i) {
    std::istringstream a(lines[4 + i]);
    std::string d, name;
    r3d_xrism_atom &x = atoms[i];
    std::memset(&x, 0, sizeof(x));
    if (!(a >> d >> name >> x.species >> x.sym >> x.sigma >> x.epsilon >> x.charge >> x.x >> x.y >>
          x.z >> x.density))
      return xfail(R3D_EINVAL, "bad atom line " + std::to_string(i + 1));
    std::snprintf(x.name, sizeof(x.name), "%s", name.c_str());
  }
  *natom = num;
  opts->ntab = ntab;
  opts->dr = dr;
  opts->temperature = temper;
  return R3D_OK;
}

int r3d_xrism_write_xvk(const char *path, const r3d_xrism_opts *opts, const r3d_xrism_atom *atoms,
                        int natom, const double *xvv, double xt) {
  if (!path || !opts || !atoms || !xvv) return xfail(R3D_EINVAL, "null argument");
  int nv = 0, rep[kXMaxV];
  {
    std::string m = check_atoms(atoms, natom, nv, rep);
    if (!m.empty()) return xfail(R3D_EINVAL, m);
  }
  FILE *fp = std::fopen(path, "w");
  if (!fp) return xfail(R3D_EIO, std::string("cannot write ") + path);
  int nspec = 0;
  for (int i = 0; i < natom; ++i) {
    bool first = true;
    for (int j = 0; j < i; ++j)
      if (atoms[j].species == atoms[i].species) first = false;
    nspec += first;
  }
  const int N = opts->ntab;
  std::fprintf(fp, "##  reduced xvv(k) data with solvent parameters\n");
  std::fprintf(fp, "## %9d %7d %7d %15.8f %15.8f\n", natom, nv, N, opts->dr, M_PI / (N * opts->dr));
  std::fprintf(fp, "## %4d %16.8f %16.8E\n", nspec, opts->temperature, xt);
  std::fprintf(fp, "## ATOM SPC SYM sig[Angs]   eps[J/mol]  charge[e]    ---X---     ---Y---     ---Z---    density[M]\n");
  for (int i = 0; i < natom; ++i) {
    const r3d_xrism_atom &a = atoms[i];
    std::fprintf(fp, "## %-6s %3d %3d %12.8f %14.8f %12.8f %12.8f %12.8f %12.8f %14.8f\n",
                 a.name[0] ? a.name : "X", a.species, a.sym, a.sigma, a.epsilon, a.charge, a.x, a.y,
                 a.z, a.density);
  }
  std::fprintf(fp, "##\n");
  for (int j = 0; j < N; ++j) {
    for (int v = 0; v < nv * nv; ++v) std::fprintf(fp, " %23.16E", xvv[(size_t)j * nv * nv + v]);
    std::fprintf(fp, "\n");
  }
  const bool ok = std::fclose(fp) == 0;
  return ok ? R3D_OK : xfail(R3D_EIO, std::string("write failed: ") + path);
}

}  // extern "C"
