/*
 * rism_oracle.c -- FP64 CPU oracle for the 3D-RISM solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * solver's algorithm (rismical-dev/3D-RISM-CUDA-MPI, src-cuda-mpi/), used by
 * the test-suite, the smoke check and the benchmark's CPU-baseline arm as the
 * checker.  It is never linked into, called by, or shipped with the CUDA
 * product.  Each function names the reference file:line it restates.  The
 * data layout deliberately follows the reference (full complex k grid,
 * per-voxel chi expansion, sort-based |k| shells) so that it checks the
 * product's very different GPU layout against the reference's semantics.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp, -ffp-contract=off).
 */
#define _GNU_SOURCE
#include "rism_oracle.h"

#include <ctype.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Deterministic parallel sums: the index range is cut into kSumBlocks
 * fixed blocks, each summed in order, and the block sums are added in block
 * order, so results do not depend on the thread count or on scheduling. */
enum { kSumBlocks = 64 };
static long blk_lo(long n, int b) { return (long)((double)n * b / kSumBlocks); }

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* physical.h:5-17 */
static const double kAvogadro = 6.02214076e23;
static const double kBohr = 0.5291771500001;
static const double kBoltzmann = 1.380649e-23;
static const double kHartree = 4.359744722207185e-18;

typedef struct { double re, im; } cplx;

static char g_err[1024];
static void set_err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}
const char *orc_last_error(void) { return g_err; }

struct orc_solver {
  /* control (read_input.cu:32-52) */
  char outlist[64];
  int ksave;
  int clos, pse_n;
  char fsolvent[1024];
  char inpdir[1024];
  char fname[1024];
  double convergence;
  int maxstep;
  int count;
  double mix_m, mix_mp;
  int mixer, history;
  double damping;
  int adswitch;
  double lambda;
  int zero;
  /* cell (cell.cc:8-26) */
  double box[3], dr[3], shift[3], volume, dv;
  int grid[3];
  long ngrid;
  /* solute (solute.cu) */
  int nu;
  double *sig, *eps, *q, *r;
  /* solvent (solvent_read.cc) */
  int natv, ntab;
  double temper, xt;
  double *sigv, *epsv, *qv, *rhov, *ttab, *xvv; /* xvv[iv2][iv1][ntab] */
  /* k grid and chi */
  int nga;
  double *ga;
  int *indga;
  double *xk; /* [a][b][ngrid] */
  /* potentials */
  double *du, *de, *fr;
  cplx *fk;
  /* iteration state */
  double *t, *tr;
  cplx *guv, *huv;
  cplx *dkf;
  int *dir, *dik;
  /* AN2 (anderson.cu) */
  double *tp, *rp;
  int binary;
  int count_left;
  /* ANM history */
  double *hx, *hf; /* [slot][n*ngrid] */
  int hcount, hhead;
  int initialized;
};

/* ------------------------------------------------------------------ */
/* tokeniser helpers                                                  */

typedef struct {
  char **tok;
  int n, pos;
  char *buf;
} toks;

static int read_file(const char *path, char **out) {
  FILE *f = fopen(path, "rb");
  if (!f) return -1;
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  char *b = (char *)malloc((size_t)n + 1);
  if (fread(b, 1, (size_t)n, f) != (size_t)n) {
    fclose(f);
    free(b);
    return -1;
  }
  b[n] = 0;
  fclose(f);
  *out = b;
  return 0;
}

static int tokenize(const char *path, toks *t) {
  memset(t, 0, sizeof *t);
  if (read_file(path, &t->buf)) return -1;
  int cap = 256;
  t->tok = (char **)malloc(sizeof(char *) * cap);
  char *p = t->buf;
  while (*p) {
    while (*p && isspace((unsigned char)*p)) ++p;
    if (!*p) break;
    char *s = p;
    while (*p && !isspace((unsigned char)*p)) ++p;
    if (*p) *p++ = 0;
    if (t->n == cap) {
      cap *= 2;
      t->tok = (char **)realloc(t->tok, sizeof(char *) * cap);
    }
    t->tok[t->n++] = s;
  }
  return 0;
}
static void free_toks(toks *t) {
  free(t->tok);
  free(t->buf);
}
static const char *next_tok(toks *t) {
  return t->pos < t->n ? t->tok[t->pos++] : NULL;
}
static int tok_double(toks *t, double *v) {
  const char *s = next_tok(t);
  if (!s) return -1;
  char *e;
  *v = strtod(s, &e);
  return e == s ? -1 : 0;
}
static int tok_int(toks *t, int *v) {
  const char *s = next_tok(t);
  if (!s) return -1;
  char *e;
  long x = strtol(s, &e, 10);
  if (e == s) return -1;
  *v = (int)x;
  return 0;
}

/* ------------------------------------------------------------------ */
/* input (read_input.cu:21-97, solute.cu:6-54, cell.cc:8-26)           */

static int is_natural(const char *s) { /* read_input.cu:7-19 */
  char *e;
  long v = strtol(s, &e, 10);
  if (e == s || *e) return 0;
  return v >= 0;
}

static void solute_centering(orc_solver *s) { /* solute.cu:18-48 */
  double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
  double mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int n = 0; n < s->nu; ++n)
    for (int d = 0; d < 3; ++d) {
      double v = s->r[3 * n + d];
      if (mn[d] > v) mn[d] = v;
      if (mx[d] < v) mx[d] = v;
    }
  for (int d = 0; d < 3; ++d) s->shift[d] = round(-(mx[d] - mn[d]) / 2 - mn[d]);
  for (int n = 0; n < s->nu; ++n)
    for (int d = 0; d < 3; ++d) s->r[3 * n + d] += s->shift[d];
}

static int read_xvk(orc_solver *s, const char *path); /* below */

orc_solver *orc_load(const char *inp, const char *structure, int centering,
                     int q0, const char *xvk_override) {
  orc_solver *s = (orc_solver *)calloc(1, sizeof *s);
  toks t;
  if (tokenize(inp, &t)) {
    set_err("cannot open input file %s", inp);
    free(s);
    return NULL;
  }
  const char *tk;
  char version[64] = "";
  if (!(tk = next_tok(&t))) goto bad;
  snprintf(s->outlist, sizeof s->outlist, "%s", tk);
  if (tok_int(&t, &s->ksave)) goto bad;
  if (!(tk = next_tok(&t))) goto bad;
  snprintf(version, sizeof version, "%s", tk);
  if (strcmp(version, "20220301") != 0) { /* read_input.cu:33-36 */
    set_err("This input file is for old version.");
    goto fail;
  }
  if (!(tk = next_tok(&t))) goto bad;
  if (!strcmp(tk, "KH")) { /* read_input.cu:38-47 */
    s->clos = ORC_CLOS_KH;
    s->pse_n = 1;
  } else if (!strcmp(tk, "HNC")) {
    s->clos = ORC_CLOS_HNC;
  } else if (!strncmp(tk, "PSE", 3)) { /* extension: PSE-n or PSEn */
    const char *d = tk + 3;
    if (*d == '-') ++d;
    s->clos = ORC_CLOS_PSE;
    s->pse_n = atoi(d);
    if (s->pse_n < 1) {
      set_err("Unexpected closure switch");
      goto fail;
    }
  } else {
    set_err("Unexpected closure switch");
    goto fail;
  }
  if (!(tk = next_tok(&t))) goto bad;
  snprintf(s->fsolvent, sizeof s->fsolvent, "%s", tk);
  if (tok_double(&t, &s->convergence) || tok_int(&t, &s->maxstep)) goto bad;
  if (tok_int(&t, &s->count) || tok_double(&t, &s->mix_m) ||
      tok_double(&t, &s->mix_mp))
    goto bad;
  for (int d = 0; d < 3; ++d)
    if (tok_double(&t, &s->box[d])) goto bad;
  for (int d = 0; d < 3; ++d)
    if (tok_int(&t, &s->grid[d])) goto bad;
  toks st;
  toks *src = &t;
  int have_struct = structure && structure[0];
  if (have_struct) {
    if (tokenize(structure, &st)) {
      set_err("cannot open structure file %s", structure);
      goto fail;
    }
    src = &st;
  }
  tk = next_tok(src);
  if (!tk || !is_natural(tk)) {
    set_err("Number of solute atom is not a natural number.");
    if (have_struct) free_toks(&st);
    goto fail;
  }
  s->nu = atoi(tk);
  s->sig = (double *)calloc(s->nu + 1, sizeof(double));
  s->eps = (double *)calloc(s->nu + 1, sizeof(double));
  s->q = (double *)calloc(s->nu + 1, sizeof(double));
  s->r = (double *)calloc(3 * s->nu + 3, sizeof(double));
  for (int iu = 0; iu < s->nu; ++iu) {
    if (tok_double(src, &s->sig[iu]) || tok_double(src, &s->eps[iu]) ||
        tok_double(src, &s->q[iu]) || tok_double(src, &s->r[3 * iu]) ||
        tok_double(src, &s->r[3 * iu + 1]) ||
        tok_double(src, &s->r[3 * iu + 2])) {
      set_err("truncated solute record %d", iu);
      if (have_struct) free_toks(&st);
      goto fail;
    }
  }
  if (have_struct) free_toks(&st);
  free_toks(&t);
  if (centering) solute_centering(s);
  s->zero = q0;
  if (q0)
    for (int n = 0; n < s->nu; ++n) s->q[n] = 0.0; /* solute.cu:50-54 */
  /* cell.cc:8-26 */
  for (int d = 0; d < 3; ++d) {
    if (s->grid[d] <= 0 || (s->grid[d] & 1) || !(s->box[d] > 0)) {
      set_err("grid must be positive and even and box positive");
      orc_free(s);
      return NULL;
    }
  }
  s->volume = s->box[0] * s->box[1] * s->box[2];
  s->ngrid = (long)s->grid[0] * s->grid[1] * s->grid[2];
  s->dv = s->volume / s->ngrid;
  for (int d = 0; d < 3; ++d) s->dr[d] = s->box[d] / s->grid[d];
  /* set_fname.cu:5-12 */
  {
    const char *base = have_struct ? structure : inp;
    snprintf(s->fname, sizeof s->fname, "%s", base);
    char *dot = strrchr(s->fname, '.');
    if (dot) *dot = 0;
    snprintf(s->inpdir, sizeof s->inpdir, "%s", inp);
    char *sl = strrchr(s->inpdir, '/');
    if (sl)
      sl[1] = 0;
    else
      s->inpdir[0] = 0;
  }
  s->mixer = ORC_MIX_AN2;
  s->history = 2;
  s->damping = s->mix_m;
  {
    const char *xp = xvk_override;
    char alt[2200];
    if (!xp) {
      FILE *f = fopen(s->fsolvent, "r");
      if (f) {
        fclose(f);
        xp = s->fsolvent;
      } else {
        snprintf(alt, sizeof alt, "%s%s", s->inpdir, s->fsolvent);
        xp = alt;
      }
    }
    if (read_xvk(s, xp)) {
      orc_free(s);
      return NULL;
    }
  }
  return s;
bad:
  set_err("truncated or malformed input file %s", inp);
fail:
  free_toks(&t);
  orc_free(s);
  return NULL;
}

/* solvent_read.cc:10-94 */
static int read_xvk(orc_solver *s, const char *path) {
  char *buf;
  if (read_file(path, &buf)) {
    set_err("Solvent file could not be opened!");
    return -1;
  }
  /* split into lines */
  int nlines = 0, cap = 1024;
  char **lines = (char **)malloc(sizeof(char *) * cap);
  char *p = buf;
  while (*p) {
    if (nlines == cap) {
      cap *= 2;
      lines = (char **)realloc(lines, sizeof(char *) * cap);
    }
    lines[nlines++] = p;
    char *e = strchr(p, '\n');
    if (!e) break;
    *e = 0;
    p = e + 1;
  }
  int num = 0;
  double drx = 0;
  int ok = nlines > 4;
  if (ok) {
    char d0[64];
    double dk;
    ok = sscanf(lines[1], "%63s %d %d %d %lf %lf", d0, &num, &s->natv, &s->ntab,
                &drx, &dk) >= 5;
    char d1[64], d2[64];
    ok = ok && sscanf(lines[2], "%63s %63s %lf %lf", d1, d2, &s->temper,
                      &s->xt) == 4;
  }
  if (!ok || num <= 0 || s->natv <= 0 || s->ntab <= 3 ||
      nlines < num + 5) {
    set_err("malformed solvent file %s", path);
    free(lines);
    free(buf);
    return -1;
  }
  int natv = s->natv, ntab = s->ntab;
  double *sig = (double *)malloc(sizeof(double) * num);
  double *eps = (double *)malloc(sizeof(double) * num);
  double *q = (double *)malloc(sizeof(double) * num);
  double *den = (double *)malloc(sizeof(double) * num);
  int *sol = (int *)malloc(sizeof(int) * num);
  for (int i = 0; i < num; ++i) {
    char a[64], b[64], c[64], x[64], y[64], z[64];
    if (sscanf(lines[4 + i], "%63s %63s %63s %d %lf %lf %lf %63s %63s %63s %lf",
               a, b, c, &sol[i], &sig[i], &eps[i], &q[i], x, y, z,
               &den[i]) != 11) {
      set_err("malformed solvent atom line %d", i);
      free(lines);
      free(buf);
      return -1;
    }
  }
  s->sigv = (double *)calloc(natv, sizeof(double));
  s->epsv = (double *)calloc(natv, sizeof(double));
  s->qv = (double *)calloc(natv, sizeof(double));
  s->rhov = (double *)calloc(natv, sizeof(double));
  for (int i = 0; i < num; ++i) { /* solvent_read.cc:70-76 */
    int i2 = abs(sol[i]) - 1;
    if (i2 < 0 || i2 >= natv) {
      set_err("solvent site symbol out of range");
      free(lines);
      free(buf);
      return -1;
    }
    s->sigv[i2] = sig[i];
    s->epsv[i2] = eps[i];
    s->qv[i2] = q[i];
    s->rhov[i2] += den[i];
  }
  for (int i = 0; i < natv; ++i) s->rhov[i] *= (kAvogadro * 1.0e-27);
  free(sig);
  free(eps);
  free(q);
  free(den);
  free(sol);
  /* table rows follow the line after the atom lines (solvent_read.cc:51-57) */
  s->xvv = (double *)malloc(sizeof(double) * natv * natv * ntab);
  long need = (long)natv * natv * ntab, got = 0;
  for (int li = num + 5; li < nlines && got < need; ++li) {
    char *q2 = lines[li];
    for (;;) {
      while (*q2 && isspace((unsigned char)*q2)) ++q2;
      if (!*q2) break;
      char *e;
      double v = strtod(q2, &e);
      if (e == q2) break;
      long row = got / (natv * natv);
      int k = (int)(got % (natv * natv));
      int iv2 = k / natv, iv1 = k % natv;
      s->xvv[((long)iv2 * natv + iv1) * ntab + row] = v;
      ++got;
      q2 = e;
      if (got == need) break;
    }
  }
  free(lines);
  free(buf);
  if (got != need) {
    set_err("solvent table truncated: %ld of %ld values", got, need);
    return -1;
  }
  double dk = M_PI / (drx * ntab); /* solvent_read.cc:81-85 */
  s->ttab = (double *)malloc(sizeof(double) * ntab);
  for (int i = 0; i < ntab; ++i) s->ttab[i] = dk * (i + 1);
  return 0;
}

void orc_free(orc_solver *s) {
  if (!s) return;
  void *ptrs[] = {s->sig, s->eps, s->q, s->r, s->sigv, s->epsv, s->qv,
                  s->rhov, s->ttab, s->xvv, s->ga, s->indga, s->xk, s->du,
                  s->de, s->fr, s->fk, s->t, s->tr, s->guv, s->huv, s->dkf,
                  s->dir, s->dik, s->tp, s->rp, s->hx, s->hf};
  for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; ++i) free(ptrs[i]);
  free(s);
}

void orc_set_ad(orc_solver *s, double lambda, int adswitch) {
  s->lambda = lambda;
  s->adswitch = adswitch;
}
void orc_set_closure(orc_solver *s, int clos, int pse_n) {
  s->clos = clos;
  s->pse_n = clos == ORC_CLOS_KH ? 1 : pse_n;
}
void orc_set_mixer(orc_solver *s, int kind, int history, double damping) {
  s->mixer = kind;
  s->history = history;
  s->damping = damping;
}

/* ------------------------------------------------------------------ */
/* 1D mixed-radix complex FFT (project-written; the reference calls    */
/* cuFFT Z2Z at fft3d.cu:61-63).  Forward uses e^{-2 pi i jk/n}.        */

typedef struct {
  int n;
  int nf;
  int fac[64]; /* pairs (radix, remaining) */
  cplx *tw;    /* e^{-2 pi i j/n} */
} fplan;

static void fplan_init(fplan *p, int n) {
  p->n = n;
  p->tw = (cplx *)malloc(sizeof(cplx) * n);
  for (int j = 0; j < n; ++j) {
    double a = -2.0 * M_PI * j / n;
    p->tw[j].re = cos(a);
    p->tw[j].im = sin(a);
  }
  int m = n, k = 0;
  while (m > 1) {
    int r;
    if (m % 4 == 0)
      r = 4;
    else if (m % 2 == 0)
      r = 2;
    else if (m % 3 == 0)
      r = 3;
    else if (m % 5 == 0)
      r = 5;
    else {
      r = m;
      for (int d = 7; d * d <= m; d += 2)
        if (m % d == 0) {
          r = d;
          break;
        }
    }
    m /= r;
    p->fac[2 * k] = r;
    p->fac[2 * k + 1] = m;
    ++k;
  }
  p->nf = k;
}
static void fplan_free(fplan *p) { free(p->tw); }

static void fft_work(cplx *out, const cplx *in, long fstride, long istride,
                     const int *fac, const fplan *p, int inverse) {
  int rdx = fac[0], m = fac[1];
  if (m == 1) {
    for (int j = 0; j < rdx; ++j) out[j] = in[(long)j * fstride * istride];
  } else {
    for (int j = 0; j < rdx; ++j)
      fft_work(out + (long)j * m, in + (long)j * fstride * istride,
               fstride * rdx, istride, fac + 2, p, inverse);
  }
  int n = p->n;
  cplx scratch[64];
  cplx *sc = rdx <= 64 ? scratch : (cplx *)malloc(sizeof(cplx) * rdx);
  for (int k = 0; k < m; ++k) {
    for (int q = 0; q < rdx; ++q) {
      long e = ((long)q * k * fstride) % n;
      cplx w = p->tw[e];
      if (inverse) w.im = -w.im;
      cplx a = out[k + (long)q * m];
      sc[q].re = a.re * w.re - a.im * w.im;
      sc[q].im = a.re * w.im + a.im * w.re;
    }
    for (int u = 0; u < rdx; ++u) {
      double sr = 0, si = 0;
      for (int q = 0; q < rdx; ++q) {
        long e = ((long)q * u * (n / rdx)) % n;
        cplx w = p->tw[e];
        if (inverse) w.im = -w.im;
        sr += sc[q].re * w.re - sc[q].im * w.im;
        si += sc[q].re * w.im + sc[q].im * w.re;
      }
      out[k + (long)u * m].re = sr;
      out[k + (long)u * m].im = si;
    }
  }
  if (sc != scratch) free(sc);
}

/* in-place 1D transform of a line (gathered into a buffer) */
static void fft_line(const fplan *p, cplx *line, cplx *tmp, int inverse) {
  if (p->n == 1) return;
  fft_work(tmp, line, 1, 1, p->fac, p, inverse);
  memcpy(line, tmp, sizeof(cplx) * p->n);
}

/* 3D unnormalised transform along all axes, x fastest */
static void fft3_raw(cplx *a, const int *g, int inverse) {
  int nx = g[0], ny = g[1], nz = g[2];
  fplan px, py, pz;
  fplan_init(&px, nx);
  fplan_init(&py, ny);
  fplan_init(&pz, nz);
  int nmax = nx > ny ? nx : ny;
  if (nz > nmax) nmax = nz;
#pragma omp parallel
  {
    cplx *line = (cplx *)malloc(sizeof(cplx) * nmax);
    cplx *tmp = (cplx *)malloc(sizeof(cplx) * nmax);
#pragma omp for schedule(static)
    for (long yz = 0; yz < (long)ny * nz; ++yz) {
      cplx *row = a + yz * nx;
      fft_line(&px, row, tmp, inverse);
    }
#pragma omp for schedule(static)
    for (long xz = 0; xz < (long)nx * nz; ++xz) {
      long x = xz % nx, z = xz / nx;
      for (int y = 0; y < ny; ++y) line[y] = a[x + nx * (y + (long)ny * z)];
      fft_line(&py, line, tmp, inverse);
      for (int y = 0; y < ny; ++y) a[x + nx * (y + (long)ny * z)] = line[y];
    }
#pragma omp for schedule(static)
    for (long xy = 0; xy < (long)nx * ny; ++xy) {
      for (int z = 0; z < nz; ++z) line[z] = a[xy + (long)nx * ny * z];
      fft_line(&pz, line, tmp, inverse);
      for (int z = 0; z < nz; ++z) a[xy + (long)nx * ny * z] = line[z];
    }
    free(line);
    free(tmp);
  }
  fplan_free(&px);
  fplan_free(&py);
  fplan_free(&pz);
}

/* phase and sign tables: setkf/setir/setik (fft3d_cuda.cu:94-128) */
static void fft_tables(const int *g, cplx *dkf, int *dir, int *dik) {
  int nx = g[0], ny = g[1], nz = g[2];
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        long ip = x + (long)nx * (y + (long)ny * z);
        int xi = (int)(x - nx / 2.0), yi = (int)(y - ny / 2.0),
            zi = (int)(z - nz / 2.0);
        double dkr = M_PI / nx * xi + M_PI / ny * yi + M_PI / nz * zi;
        dkf[ip].re = cos(dkr);
        dkf[ip].im = -sin(dkr);
        int s = ((x + y + z) % 2 == 0) ? 1 : -1;
        dir[ip] = s;
        dik[ip] = s;
      }
}

/* FFT3D::forward / backward (fft3d.cu:81-163): timekf, 3 x cufft, timeirvolf */
static void fft3_forward(cplx *a, const int *g, const cplx *dkf,
                         const int *dir, const int *dik, double volf) {
  long n = (long)g[0] * g[1] * g[2];
#pragma omp parallel for schedule(static)
  for (long ip = 0; ip < n; ++ip) { /* timekf */
    double tr = a[ip].re * dir[ip], ti = a[ip].im * dir[ip];
    a[ip].re = tr * dkf[ip].re - ti * dkf[ip].im;
    a[ip].im = ti * dkf[ip].re + tr * dkf[ip].im;
  }
  fft3_raw(a, g, 0);
#pragma omp parallel for schedule(static)
  for (long ip = 0; ip < n; ++ip) { /* timeirvolf */
    a[ip].re = a[ip].re * dik[ip] * volf;
    a[ip].im = a[ip].im * dik[ip] * volf;
  }
}
static void fft3_backward(cplx *a, const int *g, const cplx *dkf,
                          const int *dir, const int *dik, double volb) {
  long n = (long)g[0] * g[1] * g[2];
#pragma omp parallel for schedule(static)
  for (long ip = 0; ip < n; ++ip) { /* timeirvolb */
    a[ip].re = a[ip].re * dik[ip];
    a[ip].im = a[ip].im * dik[ip];
  }
  fft3_raw(a, g, 1);
#pragma omp parallel for schedule(static)
  for (long ip = 0; ip < n; ++ip) { /* timekb */
    double tr = a[ip].re * dir[ip] * volb, ti = a[ip].im * dir[ip] * volb;
    double re = tr * dkf[ip].re + ti * dkf[ip].im;
    double im = ti * dkf[ip].re - tr * dkf[ip].im;
    a[ip].re = re;
    a[ip].im = im;
  }
}

int orc_fft3d(int nx, int ny, int nz, const double *box, double *data,
              int dir) {
  int g[3] = {nx, ny, nz};
  long n = (long)nx * ny * nz;
  cplx *dkf = (cplx *)malloc(sizeof(cplx) * n);
  int *dr = (int *)malloc(sizeof(int) * n), *dk = (int *)malloc(sizeof(int) * n);
  fft_tables(g, dkf, dr, dk);
  double vol = box[0] * box[1] * box[2];
  if (dir == -1)
    fft3_forward((cplx *)data, g, dkf, dr, dk, vol / n);
  else
    fft3_backward((cplx *)data, g, dkf, dr, dk, 1.0 / vol);
  free(dkf);
  free(dr);
  free(dk);
  return 0;
}

/* ------------------------------------------------------------------ */
/* k grid shells (initialize_g.cu:7-63) and chi spline                 */

static const double *g_sort_key;
static int cmp_idx(const void *a, const void *b) {
  long i = *(const long *)a, j = *(const long *)b;
  double x = g_sort_key[i], y = g_sort_key[j];
  if (x < y) return -1;
  if (x > y) return 1;
  return (i > j) - (i < j);
}

static void initialize_g(orc_solver *s) {
  int nx = s->grid[0], ny = s->grid[1], nz = s->grid[2];
  long n = s->ngrid;
  double *g2 = (double *)malloc(sizeof(double) * n);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) { /* setg */
        long ip = x + (long)nx * (y + (long)ny * z);
        double kx = 2.0 * M_PI * (x - nx / 2.0 + 0.5) / s->box[0];
        double ky = 2.0 * M_PI * (y - ny / 2.0 + 0.5) / s->box[1];
        double kz = 2.0 * M_PI * (z - nz / 2.0 + 0.5) / s->box[2];
        g2[ip] = kx * kx + ky * ky + kz * kz;
      }
  long *idx = (long *)malloc(sizeof(long) * n);
  for (long i = 0; i < n; ++i) idx[i] = i;
  g_sort_key = g2;
  qsort(idx, n, sizeof(long), cmp_idx);
  s->indga = (int *)malloc(sizeof(int) * n);
  s->ga = (double *)malloc(sizeof(double) * n);
  double ga2o = -1.0;
  int nga = 0;
  for (long i = 0; i < n; ++i) {
    long igs = idx[i];
    double ga2 = g2[igs];
    if (ga2 > ga2o) {
      s->ga[nga++] = sqrt(ga2);
      ga2o = ga2;
    }
    s->indga[igs] = nga - 1;
  }
  s->nga = nga;
  free(idx);
  free(g2);
}

/* spline.cc:4-43 (natural cubic spline coefficients) */
static void spline_coe(const double *xp, const double *yp, int np,
                       double *c0, double *c1, double *c2) {
  double *a = (double *)calloc(np + 1, sizeof(double));
  double *b = (double *)calloc(np + 1, sizeof(double));
  double *c = (double *)calloc(np + 1, sizeof(double));
  double *d = (double *)calloc(np + 1, sizeof(double));
  double *sv = (double *)calloc(np + 1, sizeof(double));
  int n = np - 2;
  for (int k = 1; k <= n; ++k) {
    double hl = xp[k] - xp[k - 1];
    double hr = xp[k + 1] - xp[k];
    a[k] = hl / (hl + hr);
    b[k] = 1 - a[k];
    double q1 = (yp[k + 1] - yp[k]) / hr;
    double q2 = (yp[k] - yp[k - 1]) / hl;
    c[k] = 6.0 * ((q1 - q2) / (hl + hr));
    d[k] = 2.0;
  }
  for (int k = 1; k < n; ++k) {
    b[k] = b[k] / d[k];
    c[k] = c[k] / d[k];
    d[k + 1] = d[k + 1] - a[k + 1] * b[k];
    c[k + 1] = c[k + 1] - a[k + 1] * c[k];
  }
  sv[n] = c[n] / d[n];
  for (int k = n - 1; k >= 1; --k) sv[k] = c[k] - b[k] * sv[k + 1];
  sv[0] = sv[n + 1] = 0.0;
  for (int k = 0; k <= n; ++k) {
    double h = xp[k + 1] - xp[k];
    c1[k] = sv[k] / 2.0;
    c2[k] = (sv[k + 1] - sv[k]) / (6.0 * h);
    c0[k] = (yp[k + 1] - yp[k]) / h - c1[k] * h - c2[k] * h * h;
  }
  free(a);
  free(b);
  free(c);
  free(d);
  free(sv);
}

/* splint.cc:4-20 */
static double splint(const double *xp, const double *yp, const double *c0,
                     const double *c1, const double *c2, int np, double x) {
  int klo = 0, khi = np - 1;
  while (khi - klo > 1) {
    int k = (khi + klo) >> 1;
    if (xp[k] > x)
      khi = k;
    else
      klo = k;
  }
  int k = klo;
  double t = x - xp[k];
  return (((c2[k] * t + c1[k]) * t + c0[k]) * t + yp[k]);
}

/* Solvent::spline (solvent_spline.cu:7-96) */
static int solvent_spline(orc_solver *s) {
  int natv = s->natv, ntab = s->ntab, nga = s->nga;
  if (s->ga[nga - 1] > s->ttab[ntab - 1]) {
    set_err("insufficient maximal T tabulated");
    return -1;
  }
  int ntab1 = 0;
  for (int n = 0; n < ntab; ++n)
    if (s->ttab[n] < s->ga[0]) ntab1 = n;
  int ntab2 = ntab - 1;
  for (int n = ntab - 1; n > 0; --n)
    if (s->ttab[n] > s->ga[nga - 1]) ntab2 = n;
  int np = ntab2 - ntab1 + 1;
  double *x = (double *)malloc(sizeof(double) * np);
  double *y = (double *)malloc(sizeof(double) * np);
  double *c0 = (double *)malloc(sizeof(double) * np);
  double *c1 = (double *)malloc(sizeof(double) * np);
  double *c2 = (double *)malloc(sizeof(double) * np);
  double *xa = (double *)malloc(sizeof(double) * nga);
  long n = s->ngrid;
  s->xk = (double *)malloc(sizeof(double) * natv * natv * n);
  for (int iv2 = 0; iv2 < natv; ++iv2)
    for (int iv1 = 0; iv1 < natv; ++iv1) {
      const double *tab = s->xvv + ((long)iv2 * natv + iv1) * ntab;
      for (int k = 0; k < np; ++k) {
        x[k] = s->ttab[ntab1 + k];
        y[k] = tab[ntab1 + k];
      }
      spline_coe(x, y, np, c0, c1, c2);
      double wvv = iv1 == iv2 ? 1.0 : 0.0;
      for (int i = 0; i < nga; ++i) {
        double v = splint(x, y, c0, c1, c2, np, s->ga[i]);
        xa[i] = wvv + (v - wvv); /* solvent_spline.cu:57-69 */
      }
      double *dst = s->xk + ((long)iv2 * natv + iv1) * n;
      for (long ig = 0; ig < n; ++ig) dst[ig] = xa[s->indga[ig]];
    }
  free(x);
  free(y);
  free(c0);
  free(c1);
  free(c2);
  free(xa);
  return 0;
}

/* ------------------------------------------------------------------ */
/* potentials (cal_LJ.cu:4-81, cal_Coulomb.cu:4-95, cal_potential.cu)  */

static void cal_potential(orc_solver *s) {
  int nx = s->grid[0], ny = s->grid[1], nz = s->grid[2];
  long n = s->ngrid;
  int natv = s->natv, nu = s->nu;
  s->du = (double *)calloc(natv * n, sizeof(double));
  s->de = (double *)calloc(n, sizeof(double));
  s->fr = (double *)calloc(n, sizeof(double));
  s->fk = (cplx *)calloc(n, sizeof(cplx));
  double lambda1 = s->adswitch == 1 ? s->lambda : 1.0;
  double *siguv = (double *)malloc(sizeof(double) * nu * natv);
  double *epsuv = (double *)malloc(sizeof(double) * nu * natv);
  for (int iv = 0; iv < natv; ++iv)
    for (int iu = 0; iu < nu; ++iu) {
      siguv[iu + nu * iv] = (s->sig[iu] + s->sigv[iv]) * 0.5 * lambda1;
      epsuv[iu + nu * iv] = sqrt(s->eps[iu] * s->epsv[iv]);
    }
  const double cut = 2.0e-3, cut2 = cut * cut;
  double ikbt = 1.0 / (kAvogadro * kBoltzmann * s->temper);
  for (int iv = 0; iv < natv; ++iv) {
    double *du = s->du + iv * n;
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < n; ++ip) { /* LJ kernel, cal_LJ.cu:56-81 */
      int x = (int)(ip % nx), y = (int)((ip / nx) % ny),
          z = (int)(ip / ((long)nx * ny));
      double rx = (x - nx / 2) * s->dr[0];
      double ry = (y - ny / 2) * s->dr[1];
      double rz = (z - nz / 2) * s->dr[2];
      double acc = 0.0;
      for (int iu = 0; iu < nu; ++iu) {
        int iuv = iu + nu * iv;
        double dx = rx - s->r[3 * iu], dy = ry - s->r[3 * iu + 1],
               dz = rz - s->r[3 * iu + 2];
        double r2 = dx * dx + dy * dy + dz * dz;
        double rs2 = r2 / (siguv[iuv] * siguv[iuv]);
        if (rs2 < cut2) rs2 = cut2;
        double irs6 = 1.0 / (rs2 * rs2 * rs2);
        acc += epsuv[iuv] * 4.0 * irs6 * (irs6 - 1.0);
      }
      du[ip] = acc * ikbt;
    }
  }
  free(siguv);
  free(epsuv);
  if (s->adswitch != 1) {
    double lambda2 = s->adswitch == 2 ? s->lambda : 1.0;
    double ubeta = kHartree * kBohr / (kBoltzmann * s->temper) * lambda2;
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < n; ++ip) { /* coulomb, cal_Coulomb.cu:40-62 */
      int x = (int)(ip % nx), y = (int)((ip / nx) % ny),
          z = (int)(ip / ((long)nx * ny));
      double rx = (x - nx / 2) * s->dr[0];
      double ry = (y - ny / 2) * s->dr[1];
      double rz = (z - nz / 2) * s->dr[2];
      double e = 0.0, f = 0.0;
      for (int iu = 0; iu < nu; ++iu) {
        double dx = rx - s->r[3 * iu], dy = ry - s->r[3 * iu + 1],
               dz = rz - s->r[3 * iu + 2];
        double ra = sqrt(dx * dx + dy * dy + dz * dz);
        if (ra >= 1.0e-5) {
          double qr = s->q[iu] / ra;
          e += qr;
          f += qr * (1 - exp(-ra));
        } else {
          f += s->q[iu];
        }
      }
      s->de[ip] = e * ubeta; /* betar */
      s->fr[ip] = f * ubeta;
    }
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < n; ++ip) { /* fk, cal_Coulomb.cu:65-79 */
      int x = (int)(ip % nx), y = (int)((ip / nx) % ny),
          z = (int)(ip / ((long)nx * ny));
      double kx = 2.0 * M_PI * (x - nx / 2.0 + 0.5) / s->box[0];
      double ky = 2.0 * M_PI * (y - ny / 2.0 + 0.5) / s->box[1];
      double kz = 2.0 * M_PI * (z - nz / 2.0 + 0.5) / s->box[2];
      double rk2 = kx * kx + ky * ky + kz * kz;
      double rk4i = 1.0 / (rk2 * (rk2 + 1.0));
      double re = 0.0, im = 0.0;
      for (int iu = 0; iu < nu; ++iu) {
        double ruk = kx * s->r[3 * iu] + ky * s->r[3 * iu + 1] +
                     kz * s->r[3 * iu + 2];
        double tmp = 4.0 * M_PI * s->q[iu] * rk4i;
        re += tmp * cos(ruk);
        im -= tmp * sin(ruk);
      }
      s->fk[ip].re = re * ubeta; /* betak */
      s->fk[ip].im = im * ubeta;
    }
  }
  for (int iv = 0; iv < natv; ++iv) /* set_du, cal_potential.cu:19-21 */
    for (long ip = 0; ip < n; ++ip) s->du[iv * n + ip] += s->qv[iv] * s->de[ip];
}

int orc_initialize(orc_solver *s) {
  long n = s->ngrid;
  int natv = s->natv;
  initialize_g(s);
  if (solvent_spline(s)) return -1;
  cal_potential(s);
  s->t = (double *)malloc(sizeof(double) * natv * n);
  s->tr = (double *)calloc(natv * n, sizeof(double));
  s->guv = (cplx *)calloc(natv * n, sizeof(cplx));
  s->huv = (cplx *)calloc(natv * n, sizeof(cplx));
  for (int iv = 0; iv < natv; ++iv) /* init_tuv, initialize_tuv.cu:19-23 */
    for (long ip = 0; ip < n; ++ip) s->t[iv * n + ip] = s->qv[iv] * s->fr[ip];
  s->dkf = (cplx *)malloc(sizeof(cplx) * n);
  s->dir = (int *)malloc(sizeof(int) * n);
  s->dik = (int *)malloc(sizeof(int) * n);
  fft_tables(s->grid, s->dkf, s->dir, s->dik);
  /* AN2::initialize (anderson.cu:20-40) */
  s->tp = (double *)calloc(2 * natv * n, sizeof(double));
  s->rp = (double *)calloc(2 * natv * n, sizeof(double));
  s->binary = 0;
  s->count_left = s->count;
  s->hcount = 0;
  s->hhead = 0;
  if (s->mixer == ORC_MIX_ANM) {
    int h = s->history > 0 ? s->history : 1;
    s->hx = (double *)malloc(sizeof(double) * h * natv * n);
    s->hf = (double *)malloc(sizeof(double) * h * natv * n);
  }
  s->initialized = 1;
  return 0;
}

/* closures (calculate_cuda.cu:1-16; PSE-n extension) */
static double closure_g(int clos, int pse_n, double earg) {
  if (clos == ORC_CLOS_HNC) return exp(earg);
  if (earg >= 0.0) {
    if (clos == ORC_CLOS_KH || pse_n == 1) return 1.0 + earg;
    double term = 1.0, sum = 1.0;
    for (int i = 1; i <= pse_n; ++i) {
      term *= earg / i;
      sum += term;
    }
    return sum;
  }
  return exp(earg);
}

/* RISM3D::calculate (calculate.cu:4-65) + cal_rms (cal_rms.cu:14-26) */
double orc_calculate(orc_solver *s) {
  long n = s->ngrid;
  int natv = s->natv;
  for (int iv = 0; iv < natv; ++iv) {
    double *tr = s->tr + iv * n, *t = s->t + iv * n, *du = s->du + iv * n;
    cplx *gu = s->guv + iv * n;
    double qv = s->qv[iv];
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < n; ++ip) {
      tr[ip] = closure_g(s->clos, s->pse_n, -du[ip] + t[ip]); /* kh/hnc */
      gu[ip].re = tr[ip] - 1.0 - t[ip] + qv * s->fr[ip];      /* trm1mt */
      gu[ip].im = 0.0;
    }
    fft3_forward(gu, s->grid, s->dkf, s->dir, s->dik, s->dv);
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < n; ++ip) { /* mqvfk */
      gu[ip].re -= qv * s->fk[ip].re;
      gu[ip].im -= qv * s->fk[ip].im;
    }
  }
  for (int iv = 0; iv < natv; ++iv) { /* oz, calculate_cuda.cu:39-52 */
    cplx *hu = s->huv + iv * n;
    const double *x = s->xk + (long)iv * natv * n;
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < n; ++ip) {
      double hr = 0.0, hi = 0.0;
      for (int jv = 0; jv < natv; ++jv) {
        hr += s->guv[jv * n + ip].re * x[jv * n + ip];
        hi += s->guv[jv * n + ip].im * x[jv * n + ip];
      }
      hu[ip].re = hr;
      hu[ip].im = hi;
    }
  }
  double ss = 0.0;
  for (int iv = 0; iv < natv; ++iv) {
    cplx *hu = s->huv + iv * n, *gu = s->guv + iv * n;
    double *tr = s->tr + iv * n;
    fft3_backward(hu, s->grid, s->dkf, s->dir, s->dik, 1.0 / s->volume);
    double part[kSumBlocks];
#pragma omp parallel for schedule(static)
    for (int b = 0; b < kSumBlocks; ++b) {
      double acc = 0.0;
      for (long ip = blk_lo(n, b); ip < blk_lo(n, b + 1); ++ip) { /* tr, calculate_cuda.cu:54-60 */
        gu[ip].re = tr[ip];
        tr[ip] = hu[ip].re + 1.0 - gu[ip].re;
        acc += tr[ip] * tr[ip];
      }
      part[b] = acc;
    }
    for (int b = 0; b < kSumBlocks; ++b) ss += part[b];
  }
  return sqrt(ss / ((double)n * natv));
}

/* leg (anderson.cu:105-130): Gaussian elimination without pivoting */
static void leg(double *a, double *x, double *b, int n, int nn) {
  int i, j, k, k1;
  double sm, p, q, r;
  double *ai, *ak;
  for (k = 0, ak = a; k < n - 1; ++k, ak += nn) {
    k1 = k + 1;
    p = ak[k];
    for (j = k1; j < n; ++j) ak[j] /= p;
    r = b[k] /= p;
    for (i = k1, ai = ak + nn; i < n; ++i, ai += nn) {
      q = ai[k];
      for (j = k1; j < n; ++j) ai[j] -= q * ak[j];
      b[i] -= q * r;
    }
  }
  x[n - 1] = b[n - 1] / ak[n - 1];
  for (k = n - 2, ak = a + nn * (n - 2); k >= 0; --k, ak -= nn) {
    k1 = k + 1;
    sm = b[k];
    for (j = k1; j < n; ++j) sm -= ak[j] * x[j];
    x[k] = sm;
  }
}

/* AN2::calculate (anderson.cu:43-78, anderson_cuda.cu:1-67) */
static void mix_an2(orc_solver *s) {
  long n = s->ngrid;
  int natv = s->natv;
  long niv = (long)natv * n;
  if (s->count_left > 0) {
    --s->count_left;
    long boff = (long)s->binary * niv;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < niv; ++i) { /* newdt0 */
      s->tp[boff + i] = s->t[i];
      s->rp[boff + i] = s->tr[i];
      s->t[i] += s->tr[i];
    }
  } else {
    double a[4], c[2], x[2];
    c[0] = c[1] = a[0] = a[1] = a[3] = 0.0;
    for (int iv = 0; iv < natv; ++iv) { /* cal_theta + theta30 */
      double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
      const double *tr = s->tr + iv * n, *r0 = s->rp + iv * n,
                   *r1 = s->rp + niv + iv * n;
      double part[kSumBlocks][5];
#pragma omp parallel for schedule(static)
      for (int b = 0; b < kSumBlocks; ++b) {
        double q0 = 0, q1 = 0, q2 = 0, q3 = 0, q4 = 0;
        for (long ip = blk_lo(n, b); ip < blk_lo(n, b + 1); ++ip) {
          double t1 = tr[ip] - r0[ip];
          double t2 = tr[ip] - r1[ip];
          q0 += tr[ip] * t1;
          q1 += tr[ip] * t2;
          q2 += t1 * t1;
          q3 += t1 * t2;
          q4 += t2 * t2;
        }
        part[b][0] = q0;
        part[b][1] = q1;
        part[b][2] = q2;
        part[b][3] = q3;
        part[b][4] = q4;
      }
      for (int b = 0; b < kSumBlocks; ++b) {
        s0 += part[b][0];
        s1 += part[b][1];
        s2 += part[b][2];
        s3 += part[b][3];
        s4 += part[b][4];
      }
      double irho = 1.0 / s->rhov[iv];
      c[0] += s0 * irho;
      c[1] += s1 * irho;
      a[0] += s2 * irho;
      a[1] += s3 * irho;
      a[3] += s4 * irho;
    }
    a[2] = a[1];
    leg(a, x, c, 2, 2);
    double s1 = x[0] + s->mix_mp * ((s->binary == 0) ? 0 : 1);
    double s2 = x[1] + s->mix_mp * ((s->binary == 0) ? 1 : 0);
    double m = s->mix_m;
    long boff = (long)s->binary * niv;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < niv; ++i) { /* newdt, anderson_cuda.cu:11-22 */
      double t = s->t[i], r = s->tr[i];
      double tp0 = s->tp[i], tp1 = s->tp[i + niv];
      double rp0 = s->rp[i], rp1 = s->rp[i + niv];
      double u = t + s1 * (tp0 - t) + s2 * (tp1 - t);
      double v = t + r + s1 * (tp0 + rp0 - t - r) + s2 * (tp1 + rp1 - t - r);
      s->tp[i + boff] = t;
      s->rp[i + boff] = r;
      s->t[i] = u + m * (v - u);
    }
  }
  s->binary = (s->binary == 0) ? 1 : 0;
}

/* Small dense solve with partial pivoting; returns 0 if singular. */
static int solve_pp(double *A, double *b, int m) {
  for (int k = 0; k < m; ++k) {
    int piv = k;
    double best = fabs(A[k * m + k]);
    for (int i = k + 1; i < m; ++i)
      if (fabs(A[i * m + k]) > best) {
        best = fabs(A[i * m + k]);
        piv = i;
      }
    if (!(best > 1e-300)) return 0;
    if (piv != k) {
      for (int j = 0; j < m; ++j) {
        double tmp = A[k * m + j];
        A[k * m + j] = A[piv * m + j];
        A[piv * m + j] = tmp;
      }
      double tmp = b[k];
      b[k] = b[piv];
      b[piv] = tmp;
    }
    for (int i = k + 1; i < m; ++i) {
      double f = A[i * m + k] / A[k * m + k];
      for (int j = k; j < m; ++j) A[i * m + j] -= f * A[k * m + j];
      b[i] -= f * b[k];
    }
  }
  for (int k = m - 1; k >= 0; --k) {
    double acc = b[k];
    for (int j = k + 1; j < m; ++j) acc -= A[k * m + j] * b[j];
    b[k] = acc / A[k * m + k];
  }
  for (int k = 0; k < m; ++k)
    if (!isfinite(b[k])) return 0;
  return 1;
}

/* History-M Anderson with damping beta (extension).  With f = residual and
 * weights 1/rho_v (as in anderson.cu:96-100), alpha minimises
 * ||f_k + sum_i alpha_i (f_i - f_k)|| over the stored history i, and
 * t_{k+1} = t_k + sum alpha_i (t_i - t_k) + beta (f_k + sum alpha_i (f_i - f_k)).
 * The current pair (t_k, f_k) then joins the history, evicting the oldest. */
static void mix_anm(orc_solver *s) {
  long n = s->ngrid;
  int natv = s->natv;
  long niv = (long)natv * n;
  int H = s->history > 0 ? s->history : 1;
  int m = s->hcount;
  double beta = s->damping;
  double alpha[64] = {0};
  if (m > 0) {
    double A[64 * 64], c[64];
    int slot[64];
    for (int i = 0; i < m; ++i) slot[i] = (s->hhead - 1 - i + 2 * H) % H;
    for (int i = 0; i < m; ++i) {
      c[i] = 0;
      for (int j = 0; j < m; ++j) A[i * m + j] = 0;
    }
    for (int iv = 0; iv < natv; ++iv) {
      double irho = 1.0 / s->rhov[iv];
      const double *fk = s->tr + iv * n;
      for (int i = 0; i < m; ++i) {
        const double *fi = s->hf + (long)slot[i] * niv + iv * n;
        double ci = 0, part[kSumBlocks];
#pragma omp parallel for schedule(static)
        for (int b = 0; b < kSumBlocks; ++b) {
          double acc = 0.0;
          for (long ip = blk_lo(n, b); ip < blk_lo(n, b + 1); ++ip)
            acc += fk[ip] * (fk[ip] - fi[ip]);
          part[b] = acc;
        }
        for (int b = 0; b < kSumBlocks; ++b) ci += part[b];
        c[i] += ci * irho;
        for (int j = 0; j <= i; ++j) {
          const double *fj = s->hf + (long)slot[j] * niv + iv * n;
          double aij = 0;
#pragma omp parallel for schedule(static)
          for (int b = 0; b < kSumBlocks; ++b) {
            double acc = 0.0;
            for (long ip = blk_lo(n, b); ip < blk_lo(n, b + 1); ++ip)
              acc += (fk[ip] - fi[ip]) * (fk[ip] - fj[ip]);
            part[b] = acc;
          }
          for (int b = 0; b < kSumBlocks; ++b) aij += part[b];
          A[i * m + j] += aij * irho;
        }
      }
    }
    for (int i = 0; i < m; ++i)
      for (int j = i + 1; j < m; ++j) A[i * m + j] = A[j * m + i];
    for (int i = 0; i < m; ++i) alpha[i] = c[i];
    if (!solve_pp(A, alpha, m))
      for (int i = 0; i < m; ++i) alpha[i] = 0.0;
    double wsum = 0;
    for (int i = 0; i < m; ++i) wsum += alpha[i];
    double w0 = 1.0 - wsum;
    double *tn = (double *)malloc(sizeof(double) * niv);
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < niv; ++ip) {
      double xb = w0 * s->t[ip], fb = w0 * s->tr[ip];
      for (int i = 0; i < m; ++i) {
        long o = (long)slot[i] * niv + ip;
        xb += alpha[i] * s->hx[o];
        fb += alpha[i] * s->hf[o];
      }
      tn[ip] = xb + beta * fb;
    }
    /* the current pair replaces the oldest slot only after the update */
    long dst = (long)s->hhead * niv;
    memcpy(s->hx + dst, s->t, sizeof(double) * niv);
    memcpy(s->hf + dst, s->tr, sizeof(double) * niv);
    memcpy(s->t, tn, sizeof(double) * niv);
    free(tn);
  } else {
    long dst = (long)s->hhead * niv;
    memcpy(s->hx + dst, s->t, sizeof(double) * niv);
    memcpy(s->hf + dst, s->tr, sizeof(double) * niv);
#pragma omp parallel for schedule(static)
    for (long ip = 0; ip < niv; ++ip) s->t[ip] += beta * s->tr[ip];
  }
  s->hhead = (s->hhead + 1) % H;
  if (s->hcount < H) ++s->hcount;
}

void orc_mix(orc_solver *s) {
  if (s->mixer == ORC_MIX_ANM)
    mix_anm(s);
  else
    mix_an2(s);
}

/* RISM3D::iterate (iterate.cu:48-82) */
int orc_iterate(orc_solver *s, int maxstep_override, int *steps, double *rms,
                int *status) {
  int maxstep = maxstep_override > 0 ? maxstep_override : s->maxstep;
  int conver = 0, diverge = 0, istep;
  double r = 0.0;
  /* fresh mixer state, as AN2::initialize inside iterate (iterate.cu:39) */
  s->binary = 0;
  s->count_left = s->count;
  s->hcount = 0;
  s->hhead = 0;
  for (istep = 1; istep <= maxstep; ++istep) {
    r = orc_calculate(s);
    diverge = !isfinite(r);
    if (diverge) break;
    if (r <= s->convergence)
      conver = 1;
    else
      orc_mix(s);
    if (conver) break;
  }
  if (steps) *steps = istep > maxstep ? maxstep : istep;
  if (rms) *rms = r;
  if (status) *status = diverge ? 2 : (conver ? 0 : 1);
  return 0;
}

/* cal_exchem (cal_exchem.cu:4-155), cal_pmv (cal_pmv.cu:5-24),
 * cal_pressure (cal_pressure.cu:6-20) */
void orc_thermo(orc_solver *s, double *xmu, double *xmu2, double *pmv,
                double *pressure) {
  long n = s->ngrid;
  int natv = s->natv;
  double cuv = 0.0;
  for (int iv = 0; iv < natv; ++iv) {
    const cplx *hu = s->huv + iv * n;
    const double *t = s->t + iv * n, *du = s->du + iv * n;
    double e_sc = 0, e_hnc = 0, e_gf = 0, e_c = 0;
    for (long ip = 0; ip < n; ++ip) {
      double h = hu[ip].re, tt = t[ip], c = h - tt;
      double ehnc = h * 0.5 * tt - c;
      double egf = -(h * 0.5 + 1.0) * c;
      double esc;
      if (s->clos == ORC_CLOS_HNC) {
        esc = ehnc;
      } else if (h > 0.0) {
        if (s->clos == ORC_CLOS_KH || s->pse_n == 1) {
          esc = egf;
        } else {
          double ts = -du[ip] + tt, term = 1.0;
          for (int i = 1; i <= s->pse_n + 1; ++i) term *= ts / i;
          esc = 0.5 * h * h - c - 0.5 * h * c - term;
        }
      } else {
        esc = ehnc;
      }
      e_sc += esc;
      e_hnc += ehnc;
      e_gf += egf;
      e_c += c;
    }
    xmu[iv] = e_sc * s->rhov[iv] * s->dv;
    xmu[natv + iv] = e_gf * s->rhov[iv] * s->dv;
    xmu2[iv] = e_hnc * s->rhov[iv] * s->dv;
    cuv += e_c * s->rhov[iv];
  }
  cuv *= s->dv;
  double ibeta = kAvogadro * kBoltzmann * s->temper;
  *pmv = s->xt * (1.0 - cuv) * ibeta;
  double p = 0.0;
  for (int iv = 0; iv < natv; ++iv) p += s->rhov[iv];
  p *= 1.0e30 / kAvogadro;
  *pressure = 0.5 * (p + 1.0 / (s->xt * ibeta));
}

/* output_xmu.cu:7-82 */
int orc_write_xmu(orc_solver *s, const char *path) {
  int natv = s->natv;
  double *xmu = (double *)malloc(sizeof(double) * 2 * natv);
  double *xmu2 = (double *)malloc(sizeof(double) * natv);
  double pmv, pressure;
  orc_thermo(s, xmu, xmu2, &pmv, &pressure);
  char fbuf[1100];
  if (!path) {
    snprintf(fbuf, sizeof fbuf, "%s%s", s->fname, s->zero ? ".xmu0" : ".xmu");
    path = fbuf;
  }
  FILE *f = fopen(path, "w");
  if (!f) {
    free(xmu);
    free(xmu2);
    set_err("cannot write %s", path);
    return -1;
  }
  double ibeta = kAvogadro * kBoltzmann * s->temper;
  double xa = 0.0;
  for (int iv = 0; iv < natv; ++iv) xa += xmu[iv];
  double pcterm = -pressure * pmv * ibeta;
  fprintf(f, " $RESULTS\n");
  fprintf(f, "SFE_SC= %.5f !(J/mol)\n", ibeta * xa);
  for (int iv = 0; iv < natv; ++iv)
    fprintf(f, "  SFEC_SC(%d)= %.5f\n", iv, ibeta * xmu[iv]);
  fprintf(f, "\n");
  if (s->clos == ORC_CLOS_KH) {
    xa = 0.0;
    for (int iv = 0; iv < natv; ++iv) xa += xmu2[iv];
    fprintf(f, "SFE_SC_HNC= %.5f !(J/mol)\n", ibeta * xa);
    for (int iv = 0; iv < natv; ++iv)
      fprintf(f, "  SFEC_SC_HNC(%d)= %.5f\n", iv, ibeta * xmu2[iv]);
    fprintf(f, "\n");
  }
  xa = 0.0;
  for (int iv = 0; iv < natv; ++iv) xa += xmu[natv + iv];
  fprintf(f, "SFE_GF= %.5f !(J/mol)\n", ibeta * xa);
  for (int iv = 0; iv < natv; ++iv)
    fprintf(f, "  SFEC_GF(%d)= %.5f\n", iv, ibeta * xmu[natv + iv]);
  fprintf(f, "\n");
  fprintf(f, "PMV= %.5f !(L/mol)\n", pmv * 1000);
  fprintf(f, "Pressure= %.5f !(J/m^3)\n", ibeta * pressure);
  fprintf(f, "Correction_Term= %.5f !(J/mol)\n", pcterm);
  fprintf(f, " $END\n");
  fclose(f);
  free(xmu);
  free(xmu2);
  return 0;
}

/* ------------------------------------------------------------------ */
int orc_natv(const orc_solver *s) { return s->natv; }
long orc_ngrid(const orc_solver *s) { return s->ngrid; }
int orc_nu(const orc_solver *s) { return s->nu; }
void orc_grid(const orc_solver *s, int *grid, double *box, double *shift) {
  for (int d = 0; d < 3; ++d) {
    grid[d] = s->grid[d];
    box[d] = s->box[d];
    shift[d] = s->shift[d];
  }
}
void orc_solvent(const orc_solver *s, double *rhov, double *qv, double *sigv,
                 double *epsv, double *temper, double *xt) {
  for (int i = 0; i < s->natv; ++i) {
    rhov[i] = s->rhov[i];
    qv[i] = s->qv[i];
    sigv[i] = s->sigv[i];
    epsv[i] = s->epsv[i];
  }
  *temper = s->temper;
  *xt = s->xt;
}
void orc_solute(const orc_solver *s, double *sig, double *eps, double *q,
                double *r) {
  memcpy(sig, s->sig, sizeof(double) * s->nu);
  memcpy(eps, s->eps, sizeof(double) * s->nu);
  memcpy(q, s->q, sizeof(double) * s->nu);
  memcpy(r, s->r, sizeof(double) * 3 * s->nu);
}

int orc_get(const orc_solver *s, int which, double *out) {
  long n = s->ngrid;
  int natv = s->natv;
  if (!s->initialized) return -1;
  switch (which) {
    case 0:
      memcpy(out, s->du, sizeof(double) * natv * n);
      return 0;
    case 1:
      memcpy(out, s->t, sizeof(double) * natv * n);
      return 0;
    case 2:
      for (long i = 0; i < natv * n; ++i) out[i] = s->guv[i].re;
      return 0;
    case 3:
      for (long i = 0; i < natv * n; ++i) out[i] = s->huv[i].re;
      return 0;
    case 4:
      memcpy(out, s->tr, sizeof(double) * natv * n);
      return 0;
    case 5:
      memcpy(out, s->fr, sizeof(double) * n);
      return 0;
    case 6:
      memcpy(out, s->fk, sizeof(cplx) * n);
      return 0;
    case 7:
      memcpy(out, s->xk, sizeof(double) * natv * natv * n);
      return 0;
  }
  return -1;
}

int orc_set_t(orc_solver *s, const double *t) {
  if (!s->initialized) return -1;
  memcpy(s->t, t, sizeof(double) * s->natv * s->ngrid);
  return 0;
}
