/*
 * xrism_oracle.c -- FP64 CPU oracle of the 1D XRISM solvent solve that makes
 * .xvk tables (TEST INFRASTRUCTURE, not the product).
 *
 * The reference repository ships .xvk tables (example/h2o_vv.xvk,
 * example/naclaq_vv.xvk, example/kclaq_vv.xvk, example_milc/ctip3p.xvk) but
 * not the 1D program that made them; its reader fixes the format
 * (src-cuda-mpi/solvent_read.cc:31-85: header "## num natv ntab dr dk",
 * "## nspecies T xt", atom lines "## name spc sym sig eps q x y z dens[M]",
 * then ntab rows of natv*natv values [iv2][iv1] at k = (i+1) pi/(dr ntab)),
 * and its use of the table fixes what the values are
 * (src-cuda-mpi/calculate_cuda.cu:39-52: h_v = sum_v' c_v' xvv[v][v'], so
 * xvv[v][v'] = sum over the sites b of class v' of w_ab(k) + rho_b h_ab(k)).
 *
 * This file restates the published extended RISM equations (Hirata and
 * Rossky, Chem. Phys. Lett. 83, 329 (1981)) with the Kovalenko-Hirata
 * closure (J. Chem. Phys. 110, 10095 (1999)) and a modified DIIS mixer in
 * the form of Kovalenko, Ten-no and Hirata (J. Comput. Chem. 20, 928
 * (1999)).  Pinned: with the reference's physical constants
 * (src-cuda-mpi/physical.h:5-14) and a Coulomb split erf(r/1 A)/r it
 * re-makes the four shipped tables from their own atom tables -- water and
 * 0.2 M NaCl / KCl at 300 K to 1.3-3.1e-7, their compressibility column to
 * 2-5e-7 relative, and the 298.15 K ctip3p water to 1.2e-7 once its H
 * positions (printed to 5 decimals) are recovered from the table's own
 * large-k rows (tests/test_xrism.py).
 *
 * Sites are reduced to the reader's classes (|sym|): rep(A) is the first
 * atom of class A, n_B rho_B = rhov[B] the summed site density, and
 *   W~_AB(k) = sum_{b in B, same molecule as rep(A)} j0(k |r_rep(A) - r_b|)
 *   H = (I - W~ C D)^-1 W~ C W~^T,  D = diag(rhov)
 *   xvv[A][B] = W~_AB + rhov[B] H_AB.
 * Coulomb: u_s = u_LJ + cc q_A q_B erfc(r)/r in r space; C = C_s + C_L with
 * C_L(k) = -cc q_A q_B 4 pi exp(-k^2/4)/k^2 added analytically; the state is
 * t = h - c_s on r_i = i dr, i = 1..N-1; the transforms are the discrete
 * sine transform on that grid (k_j = j pi/(N dr)), which leaves k_N = pi/dr
 * with h = 0 (the table's last row is W~ alone).
 * Charges are switched on over a ladder of nladder stages (q scaled by
 * s/nladder); every stage but the last stops at RMS 1e-5.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define XR_MAXV 16
#define XR_MAXH 32

static const double kAvogadro = 6.02214076e23;   /* physical.h:5  */
static const double kBohr = 0.5291771500001;      /* physical.h:8  */
static const double kBoltzmann = 1.380649e-23;    /* physical.h:11 */
static const double kHartree = 4.359744722207185e-18; /* physical.h:14 */

/* ---- FFT (radix-2, in place, e^{-2 pi i jk/L}); L a power of two ------- */
static void fft_c(double *re, double *im, int L, const double *cw, const double *sw) {
  for (int i = 1, j = 0; i < L; ++i) {
    int bit = L >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double t = re[i]; re[i] = re[j]; re[j] = t;
      t = im[i]; im[i] = im[j]; im[j] = t;
    }
  }
  for (int len = 2; len <= L; len <<= 1) {
    int half = len >> 1, step = L / len;
    for (int s = 0; s < L; s += len)
      for (int k = 0; k < half; ++k) {
        double wr = cw[k * step], wi = -sw[k * step];
        int a = s + k, b = a + half;
        double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - xr; im[b] = im[a] - xi;
        re[a] += xr; im[a] += xi;
      }
  }
}

/* S_j = sum_{i=1}^{N-1} f_i sin(pi i j / N), j = 1..N-1, via the odd
 * extension of length 2N: its DFT is -2i S_j.  f, S indexed 1..N-1 (f[0]
 * unused); work: 4N doubles; cw/sw: cos/sin(2 pi k/(2N)), k < N. */
static void dst1(const double *f, double *S, int N, double *work,
                 const double *cw, const double *sw) {
  int L = 2 * N;
  double *re = work, *im = work + L;
  re[0] = 0; re[N] = 0;
  for (int i = 1; i < N; ++i) { re[i] = f[i]; re[L - i] = -f[i]; }
  memset(im, 0, sizeof(double) * L);
  fft_c(re, im, L, cw, sw);
  for (int j = 1; j < N; ++j) S[j] = -0.5 * im[j];
}

/* Exported for the tests: the transform above on one vector. */
void orc_dst1(const double *f, double *S, int N) {
  double *work = malloc(sizeof(double) * 4 * N);
  double *cw = malloc(sizeof(double) * N), *sw = malloc(sizeof(double) * N);
  for (int k = 0; k < N; ++k) { cw[k] = cos(M_PI * k / N); sw[k] = sin(M_PI * k / N); }
  dst1(f, S, N, work, cw, sw);
  free(work); free(cw); free(sw);
}

/* small dense solve A X = B (n x n, nrhs columns), partial pivoting;
 * returns 0 when a pivot vanishes */
static int gauss(double *A, double *B, int n, int nrhs) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (fabs(A[r * n + c]) > fabs(A[p * n + c])) p = r;
    if (!(fabs(A[p * n + c]) > 1e-300)) return 0;
    if (p != c) {
      for (int k = 0; k < n; ++k) { double t = A[c * n + k]; A[c * n + k] = A[p * n + k]; A[p * n + k] = t; }
      for (int k = 0; k < nrhs; ++k) { double t = B[c * nrhs + k]; B[c * nrhs + k] = B[p * nrhs + k]; B[p * nrhs + k] = t; }
    }
    double inv = 1.0 / A[c * n + c];
    for (int r = c + 1; r < n; ++r) {
      double m = A[r * n + c] * inv;
      if (m == 0.0) continue;
      for (int k = c; k < n; ++k) A[r * n + k] -= m * A[c * n + k];
      for (int k = 0; k < nrhs; ++k) B[r * nrhs + k] -= m * B[c * nrhs + k];
    }
  }
  for (int c = n - 1; c >= 0; --c)
    for (int k = 0; k < nrhs; ++k) {
      double s = B[c * nrhs + k];
      for (int j = c + 1; j < n; ++j) s -= A[c * n + j] * B[j * nrhs + k];
      B[c * nrhs + k] = s / A[c * n + c];
    }
  return 1;
}

/* MDIIS coefficients from the bordered Gram system [G 1; 1^T 0];
 * falls back to the newest entry alone when the system is singular. */
static void diis_coef(const double *G, int m, const int *slots, int n, int newest, double *c) {
  double A[(XR_MAXH + 1) * (XR_MAXH + 1)], b[XR_MAXH + 1];
  double sc = 0;
  for (int i = 0; i < n; ++i) sc = fmax(sc, G[slots[i] * m + slots[i]]);
  sc = sc > 0 ? 1.0 / sc : 1.0;
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) A[i * (n + 1) + j] = G[slots[i] * m + slots[j]] * sc;
    A[i * (n + 1) + n] = 1.0;
    A[n * (n + 1) + i] = 1.0;
    b[i] = 0.0;
  }
  A[n * (n + 1) + n] = 0.0;
  b[n] = 1.0;
  int ok = gauss(A, b, n + 1, 1);
  for (int i = 0; i < n && ok; ++i) ok = isfinite(b[i]);
  for (int i = 0; i < n; ++i) c[i] = ok ? b[i] : (slots[i] == newest ? 1.0 : 0.0);
}

/*
 * One 1D XRISM solve.  Atoms as the .xvk atom table: spc (species), sym
 * (class, sign ignored), sig [A], eps [J/mol], q [e], xyz [A], den [M].
 * xvv: [ntab][natv][natv] out.  info[0..4] out: xt [1/Pa], rms, evaluations,
 * status (0 converged, 1 maxstep, 2 diverged), natv.  Returns 0 on success,
 * else a negative code for bad input.
 */
int orc_xrism_solve(int natom, const int *spc, const int *sym, const double *sig,
                    const double *eps, const double *q, const double *xyz,
                    const double *den, double temper, int ntab, double dr,
                    int closure, int pse_n, double tol, int maxstep, int history,
                    double mix, int nladder, double *xvv, double *info) {
  const int N = ntab, M = N - 1;
  if (natom < 1 || N < 16 || (N & (N - 1)) || dr <= 0 || temper <= 0) return -1;
  if (history < 1 || history > XR_MAXH || nladder < 1 || maxstep < 1) return -1;
  int natv = 0;
  for (int i = 0; i < natom; ++i) natv = abs(sym[i]) > natv ? abs(sym[i]) : natv;
  if (natv < 1 || natv > XR_MAXV) return -2;
  int rep[XR_MAXV];
  for (int A = 0; A < natv; ++A) rep[A] = -1;
  double rhov[XR_MAXV] = {0};
  for (int i = 0; i < natom; ++i) {
    int A = abs(sym[i]) - 1;
    if (A < 0) return -2;
    if (rep[A] < 0) rep[A] = i;
    int r0 = rep[A];
    if (spc[i] != spc[r0] || sig[i] != sig[r0] || eps[i] != eps[r0] || q[i] != q[r0] ||
        den[i] != den[r0])
      return -3;
    rhov[A] += den[i] * kAvogadro * 1.0e-27;
  }
  for (int A = 0; A < natv; ++A)
    if (rep[A] < 0) return -2;
  const int P = natv * (natv + 1) / 2;
  int pa[XR_MAXV * (XR_MAXV + 1) / 2], pb[XR_MAXV * (XR_MAXV + 1) / 2], pidx[XR_MAXV][XR_MAXV];
  for (int A = 0, p = 0; A < natv; ++A)
    for (int B = A; B < natv; ++B, ++p) { pa[p] = A; pb[p] = B; pidx[A][B] = pidx[B][A] = p; }

  const double dk = M_PI / (N * dr);
  const double kT = kBoltzmann * temper;
  const double cc = kHartree * kBohr / kT;                 /* A */
  const double rt = kAvogadro * kT;                        /* J/mol */
  /* per-pair short-range potential, long-range C_L(k) / (q_A q_B) */
  double *us_lj = malloc(sizeof(double) * P * N), *us_c = malloc(sizeof(double) * P * N);
  double *om = malloc(sizeof(double) * natv * natv * N);   /* [j][A][B], j = 0..N-1 <-> k_{j+1} */
  double *cl = malloc(sizeof(double) * N);                 /* -cc 4 pi e^{-k^2/4}/k^2 */
  for (int p = 0; p < P; ++p) {
    int a = rep[pa[p]], b = rep[pb[p]];
    double s = 0.5 * (sig[a] + sig[b]), e = sqrt(eps[a] * eps[b]);
    for (int i = 1; i < N; ++i) {
      double r = i * dr, sr6 = pow(s / r, 6);
      us_lj[p * N + i] = 4.0 * e * (sr6 * sr6 - sr6) / rt;
      us_c[p * N + i] = cc * q[a] * q[b] * erfc(r) / r;
    }
  }
  for (int j = 0; j < N; ++j) {
    double k = (j + 1) * dk;
    cl[j] = -cc * 4.0 * M_PI * exp(-0.25 * k * k) / (k * k);
    for (int A = 0; A < natv; ++A)
      for (int B = 0; B < natv; ++B) om[(j * natv + A) * natv + B] = 0.0;
    for (int A = 0; A < natv; ++A) {
      int a = rep[A];
      for (int b = 0; b < natom; ++b) {
        if (spc[b] != spc[a]) continue;
        int B = abs(sym[b]) - 1;
        double dx = xyz[3 * a] - xyz[3 * b], dy = xyz[3 * a + 1] - xyz[3 * b + 1],
               dz = xyz[3 * a + 2] - xyz[3 * b + 2];
        double l = sqrt(dx * dx + dy * dy + dz * dz);
        om[(j * natv + A) * natv + B] += (b == a || l == 0.0) ? 1.0 : sin(k * l) / (k * l);
      }
    }
  }
  const int H = history;
  double *tr = calloc((size_t)H * P * N, sizeof(double));   /* t ring   [slot][p][i] */
  double *fr = calloc((size_t)H * P * N, sizeof(double));   /* f ring   */
  double *cs = malloc(sizeof(double) * P * N);               /* r c_s(r), then C_s(k) */
  double *tk = malloc(sizeof(double) * P * N);               /* k T(k), then t_new */
  double *G = calloc(H * H, sizeof(double));
  double *tb = calloc((size_t)P * N, sizeof(double));  /* best t of the stage */
  double *cw = malloc(sizeof(double) * N), *sw = malloc(sizeof(double) * N);
  for (int k = 0; k < N; ++k) { cw[k] = cos(M_PI * k / N); sw[k] = sin(M_PI * k / N); }
  double qA[XR_MAXV];
  for (int A = 0; A < natv; ++A) qA[A] = q[rep[A]];

  int head = 0, nh = 0, steps = 0, status = 1;
  int slots[XR_MAXH];
  double err = 0;
  for (int stage = 1; stage <= nladder; ++stage) {
    const double s = (double)stage / nladder, s2 = s * s;
    const double stol = stage == nladder ? tol : fmax(tol, 1e-5);
    double best = INFINITY, eta = mix;
    int rollbacks = 0;
    nh = 0;
    status = 1;
    for (int it = 0; it < maxstep; ++it) {
      double *t = tr + (size_t)head * P * N, *f = fr + (size_t)head * P * N;
      /* closure -> r c_s(r) */
      for (int p = 0; p < P; ++p)
        for (int i = 1; i < N; ++i) {
          double tt = t[p * N + i];
          double x = -(us_lj[p * N + i] + s2 * us_c[p * N + i]) + tt, g;
          if (closure == 1 || x <= 0.0) {
            g = exp(x);
          } else {
            double term = 1.0, sum = 1.0;
            int n = closure == 2 ? pse_n : 1;
            for (int m = 1; m <= n; ++m) { term *= x / m; sum += term; }
            g = sum;
          }
          cs[p * N + i] = (i * dr) * (g - 1.0 - tt);
        }
      /* forward transforms: C_s(k_j) = 4 pi dr / k_j S_j[r c_s] */
#pragma omp parallel for schedule(static)
      for (int p = 0; p < P; ++p) {
        double *work = malloc(sizeof(double) * 4 * N), *S = malloc(sizeof(double) * N);
        dst1(cs + p * N, S, N, work, cw, sw);
        for (int j = 1; j < N; ++j) cs[p * N + j] = 4.0 * M_PI * dr / (j * dk) * S[j];
        free(work); free(S);
      }
      /* OZ per k: H = (I - W C D)^-1 W C W^T; k T(k) = k (H_sym - C_s) */
#pragma omp parallel for schedule(static)
      for (int j = 1; j < N; ++j) {
        const double *W = om + (size_t)(j - 1) * natv * natv;
        double C[XR_MAXV * XR_MAXV], WC[XR_MAXV * XR_MAXV], Am[XR_MAXV * XR_MAXV],
            Bm[XR_MAXV * XR_MAXV];
        for (int A = 0; A < natv; ++A)
          for (int B = 0; B < natv; ++B)
            C[A * natv + B] = cs[pidx[A][B] * N + j] + s2 * qA[A] * qA[B] * cl[j - 1];
        for (int A = 0; A < natv; ++A)
          for (int B = 0; B < natv; ++B) {
            double v = 0;
            for (int E = 0; E < natv; ++E) v += W[A * natv + E] * C[E * natv + B];
            WC[A * natv + B] = v;
          }
        for (int A = 0; A < natv; ++A)
          for (int B = 0; B < natv; ++B) {
            Am[A * natv + B] = (A == B ? 1.0 : 0.0) - WC[A * natv + B] * rhov[B];
            double v = 0;
            for (int E = 0; E < natv; ++E) v += WC[A * natv + E] * W[B * natv + E];
            Bm[A * natv + B] = v;
          }
        gauss(Am, Bm, natv, natv);
        double k = j * dk;
        for (int p = 0; p < P; ++p) {
          double h = 0.5 * (Bm[pa[p] * natv + pb[p]] + Bm[pb[p] * natv + pa[p]]);
          tk[p * N + j] = k * (h - cs[p * N + j]);
        }
      }
      /* inverse transforms: t(r_i) = dk / (2 pi^2 r_i) S_i[k T]; residual */
#pragma omp parallel for schedule(static)
      for (int p = 0; p < P; ++p) {
        double *work = malloc(sizeof(double) * 4 * N), *S = malloc(sizeof(double) * N);
        dst1(tk + p * N, S, N, work, cw, sw);
        for (int i = 1; i < N; ++i)
          f[p * N + i] = dk / (2.0 * M_PI * M_PI * (i * dr)) * S[i] - t[p * N + i];
        free(work); free(S);
      }
      ++steps;
      double ss = 0;
      for (int p = 0; p < P; ++p)
        for (int i = 1; i < N; ++i) ss += f[p * N + i] * f[p * N + i];
      err = sqrt(ss / ((double)P * M));
      if (err < stol) { status = 0; break; }
      int next = (head + 1) % H;
      double *tn = tr + (size_t)next * P * N;
      if (!(err <= 10.0 * best)) {
        /* the step left the basin: go back to the best state of the stage,
         * drop the history and halve the step */
        if (!isfinite(best) || ++rollbacks > 8) { status = 2; break; }
        memcpy(tn, tb, sizeof(double) * P * N);
        nh = 0;
        eta *= 0.5;
        head = next;
        continue;
      }
      if (err < best) {
        best = err;
        memcpy(tb, t, sizeof(double) * P * N);
      }
      /* push (t, f) of slot head; Gram row of the new entry */
      nh = nh < H ? nh + 1 : H;
      for (int n = 0; n < nh; ++n) slots[n] = (head - (nh - 1) + n + H) % H;  /* oldest first */
      for (int n = 0; n < nh; ++n) {
        const double *g2 = fr + (size_t)slots[n] * P * N;
        double d = 0;
        for (int p = 0; p < P; ++p)
          for (int i = 1; i < N; ++i) d += f[p * N + i] * g2[p * N + i];
        G[head * H + slots[n]] = G[slots[n] * H + head] = d;
      }
      double c[XR_MAXH];
      diis_coef(G, H, slots, nh, head, c);
      /* next may be the oldest slot (ring full): each element reads every slot
       * before it writes its own */
      for (int p = 0; p < P; ++p)
        for (int i = 1; i < N; ++i) {
          double v = 0;
          for (int n = 0; n < nh; ++n) {
            size_t o = (size_t)slots[n] * P * N + p * N + i;
            v += c[n] * (tr[o] + eta * fr[o]);
          }
          tn[p * N + i] = v;
        }
      head = next;
    }
    if (status != 0) break;
  }
  /* table: rows j = 1..N-1 from the last evaluation's OZ, row N = W~ */
  double xt = NAN;
  if (status == 0) {
    const double *t = tr + (size_t)head * P * N;
    /* re-evaluate c_s(r) and the OZ at the converged t for the table and
     * the compressibility (sum over species densities minus
     * sum_AB rhov_A rhov_B c_s,AB(k=0)) */
    double c0[XR_MAXV * (XR_MAXV + 1) / 2];
    for (int p = 0; p < P; ++p) {
      double acc = 0;
      for (int i = 1; i < N; ++i) {
        double tt = t[p * N + i];
        double x = -(us_lj[p * N + i] + us_c[p * N + i]) + tt, g;
        if (closure == 1 || x <= 0.0) {
          g = exp(x);
        } else {
          double term = 1.0, sum = 1.0;
          int n = closure == 2 ? pse_n : 1;
          for (int m = 1; m <= n; ++m) { term *= x / m; sum += term; }
          g = sum;
        }
        double r = i * dr;
        cs[p * N + i] = r * (g - 1.0 - tt);
        acc += r * r * (g - 1.0 - tt);
      }
      c0[p] = 4.0 * M_PI * dr * acc;
    }
    for (int p = 0; p < P; ++p) {
      double *work = malloc(sizeof(double) * 4 * N), *S = malloc(sizeof(double) * N);
      dst1(cs + p * N, S, N, work, cw, sw);
      for (int j = 1; j < N; ++j) cs[p * N + j] = 4.0 * M_PI * dr / (j * dk) * S[j];
      free(work); free(S);
    }
    for (int j = 1; j <= N; ++j) {
      const double *W = om + (size_t)(j - 1) * natv * natv;
      double *X = xvv + (size_t)(j - 1) * natv * natv;
      if (j == N) {
        memcpy(X, W, sizeof(double) * natv * natv);
        continue;
      }
      double C[XR_MAXV * XR_MAXV], WC[XR_MAXV * XR_MAXV], Am[XR_MAXV * XR_MAXV],
          Bm[XR_MAXV * XR_MAXV];
      for (int A = 0; A < natv; ++A)
        for (int B = 0; B < natv; ++B)
          C[A * natv + B] = cs[pidx[A][B] * N + j] + qA[A] * qA[B] * cl[j - 1];
      for (int A = 0; A < natv; ++A)
        for (int B = 0; B < natv; ++B) {
          double v = 0;
          for (int E = 0; E < natv; ++E) v += W[A * natv + E] * C[E * natv + B];
          WC[A * natv + B] = v;
        }
      for (int A = 0; A < natv; ++A)
        for (int B = 0; B < natv; ++B) {
          Am[A * natv + B] = (A == B ? 1.0 : 0.0) - WC[A * natv + B] * rhov[B];
          double v = 0;
          for (int E = 0; E < natv; ++E) v += WC[A * natv + E] * W[B * natv + E];
          Bm[A * natv + B] = v;
        }
      gauss(Am, Bm, natv, natv);
      for (int A = 0; A < natv; ++A)
        for (int B = 0; B < natv; ++B) {
          double h = 0.5 * (Bm[A * natv + B] + Bm[B * natv + A]);
          X[A * natv + B] = W[A * natv + B] + rhov[B] * h;
        }
    }
    /* species densities: den of each species' first atom */
    double rs = 0;
    for (int i = 0; i < natom; ++i) {
      int first = 1;
      for (int j = 0; j < i; ++j)
        if (spc[j] == spc[i]) first = 0;
      if (first) rs += den[i] * kAvogadro * 1.0e-27;
    }
    double sc = 0;
    for (int A = 0; A < natv; ++A)
      for (int B = 0; B < natv; ++B) sc += rhov[A] * rhov[B] * c0[pidx[A][B]];
    xt = 1.0 / (kT * 1.0e30 * (rs - sc));
  }
  info[0] = xt;
  info[1] = err;
  info[2] = steps;
  info[3] = status;
  info[4] = natv;
  free(us_lj); free(us_c); free(om); free(cl); free(tr); free(fr); free(cs); free(tk);
  free(G); free(tb); free(cw); free(sw);
  return 0;
}
