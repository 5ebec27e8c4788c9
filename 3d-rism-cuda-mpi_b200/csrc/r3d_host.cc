// r3d_host.cc -- host-side input surface of the B200 3D-RISM solver:
// the .inp / .xvk readers, the chi shell table and the .xmu writer.
//
// Format and semantics follow the reference solver:
//   .inp      read_input.cu:21-97, solute.cu:6-54, set_fname.cu:5-12
//   .xvk      solvent_read.cc:10-94
//   shells    initialize_g.cu:7-63, solvent_spline.cu:7-96, spline.cc, splint.cc
//   .xmu      output_xmu.cu:7-82, cal_pressure.cu:6-20
#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "r3d_internal.h"

namespace r3d {

namespace phys {  // physical.h:5-17
constexpr double avogadro = 6.02214076e23;
constexpr double bohr = 0.5291771500001;
constexpr double boltzmann = 1.380649e-23;
constexpr double hartree = 4.359744722207185e-18;
}  // namespace phys

static bool slurp(const std::string &path, std::string &out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  out = ss.str();
  return true;
}

static std::vector<std::string> tokens(const std::string &s) {
  std::vector<std::string> t;
  size_t i = 0, n = s.size();
  while (i < n) {
    while (i < n && std::isspace((unsigned char)s[i])) ++i;
    size_t j = i;
    while (j < n && !std::isspace((unsigned char)s[j])) ++j;
    if (j > i) t.emplace_back(s.substr(i, j - i));
    i = j;
  }
  return t;
}

static bool to_d(const std::string &s, double &v) {
  char *e;
  v = std::strtod(s.c_str(), &e);
  return e != s.c_str();
}
static bool to_i(const std::string &s, int &v) {
  char *e;
  long x = std::strtol(s.c_str(), &e, 10);
  if (e == s.c_str()) return false;
  v = (int)x;
  return true;
}
static bool natural(const std::string &s) {  // read_input.cu:7-19
  char *e;
  long v = std::strtol(s.c_str(), &e, 10);
  return e != s.c_str() && *e == 0 && v >= 0;
}

std::string parse_inp(Problem &p, const std::string &inp,
                      const std::string &structure, bool centering, bool q0) {
  std::string text;
  if (!slurp(inp, text)) return "cannot open input file " + inp;
  std::vector<std::string> t = tokens(text);
  size_t k = 0;
  auto next = [&](std::string &s) {
    if (k >= t.size()) return false;
    s = t[k++];
    return true;
  };
  std::string s, version, clos;
  if (!next(p.outlist) || !next(s) || !to_i(s, p.ksave) || !next(version))
    return "truncated input file " + inp;
  if (version != "20220301") return "This input file is for old version.";
  if (!next(clos)) return "truncated input file " + inp;
  if (clos == "KH") {
    p.clos = KH;
    p.pse_n = 1;
  } else if (clos == "HNC") {
    p.clos = HNC;
    p.pse_n = 1;
  } else if (clos.compare(0, 3, "PSE") == 0) {  // extension: PSE-n / PSEn
    const char *d = clos.c_str() + 3;
    if (*d == '-') ++d;
    p.clos = PSE;
    p.pse_n = std::atoi(d);
    if (p.pse_n < 1) return "Unexpected closure switch";
  } else {
    return "Unexpected closure switch";
  }
  std::string a, b, c;
  if (!next(p.fsolvent)) return "truncated input file " + inp;
  if (!next(a) || !next(b) || !to_d(a, p.convergence) || !to_i(b, p.maxstep))
    return "malformed convergence line in " + inp;
  if (!next(a) || !next(b) || !next(c) || !to_i(a, p.count) ||
      !to_d(b, p.mix_m) || !to_d(c, p.mix_mp))
    return "malformed mixing line in " + inp;
  for (int d = 0; d < 3; ++d)
    if (!next(a) || !to_d(a, p.box[d])) return "malformed box in " + inp;
  for (int d = 0; d < 3; ++d)
    if (!next(a) || !to_i(a, p.grid[d])) return "malformed grid in " + inp;
  std::vector<std::string> st;
  size_t sk = 0;
  const std::vector<std::string> *src = &t;
  size_t *pk = &k;
  if (!structure.empty()) {
    std::string stext;
    if (!slurp(structure, stext)) return "cannot open structure file " + structure;
    st = tokens(stext);
    src = &st;
    pk = &sk;
  }
  if (*pk >= src->size() || !natural((*src)[*pk]))
    return "Number of solute atom is not a natural number.";
  int nu = std::atoi((*src)[(*pk)++].c_str());
  p.sig.assign(nu, 0);
  p.eps.assign(nu, 0);
  p.q.assign(nu, 0);
  p.r.assign(3 * nu, 0);
  for (int iu = 0; iu < nu; ++iu) {
    double v[6];
    for (int j = 0; j < 6; ++j) {
      if (*pk >= src->size() || !to_d((*src)[(*pk)++], v[j]))
        return "truncated solute record " + std::to_string(iu);
    }
    p.sig[iu] = v[0];
    p.eps[iu] = v[1];
    p.q[iu] = v[2];
    p.r[3 * iu] = v[3];
    p.r[3 * iu + 1] = v[4];
    p.r[3 * iu + 2] = v[5];
  }
  for (int d = 0; d < 3; ++d) {
    if (p.grid[d] < 4 || (p.grid[d] & 1) || p.grid[d] > 2048 || !(p.box[d] > 0))
      return "grid must be even, 4..2048, and the box positive";
  }
  p.shift[0] = p.shift[1] = p.shift[2] = 0.0;
  if (centering && nu > 0) {  // solute.cu:18-48, integer-rounded shift
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX};
    double mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int n = 0; n < nu; ++n)
      for (int d = 0; d < 3; ++d) {
        mn[d] = std::min(mn[d], p.r[3 * n + d]);
        mx[d] = std::max(mx[d], p.r[3 * n + d]);
      }
    for (int d = 0; d < 3; ++d) p.shift[d] = std::round(-(mx[d] - mn[d]) / 2 - mn[d]);
    for (int n = 0; n < nu; ++n)
      for (int d = 0; d < 3; ++d) p.r[3 * n + d] += p.shift[d];
  }
  p.zero = q0;
  if (q0) std::fill(p.q.begin(), p.q.end(), 0.0);  // solute.cu:50-54
  std::string base = structure.empty() ? inp : structure;  // set_fname.cu
  size_t dot = base.rfind('.');
  p.fname = dot == std::string::npos ? base : base.substr(0, dot);
  p.has_solute = true;
  return "";
}

std::string parse_xvk(Problem &p, const std::string &path) {
  std::string text;
  if (!slurp(path, text)) return "Solvent file could not be opened!";
  std::vector<std::string> lines;
  {
    size_t i = 0;
    while (i <= text.size()) {
      size_t j = text.find('\n', i);
      if (j == std::string::npos) j = text.size();
      lines.emplace_back(text.substr(i, j - i));
      if (j == text.size()) break;
      i = j + 1;
    }
  }
  if (lines.size() < 5) return "malformed solvent file " + path;
  int num = 0;
  double dr = 0;
  {
    std::vector<std::string> h = tokens(lines[1]);
    if (h.size() < 5 || !to_i(h[1], num) || !to_i(h[2], p.natv) ||
        !to_i(h[3], p.ntab) || !to_d(h[4], dr))
      return "malformed solvent header in " + path;
    std::vector<std::string> h2 = tokens(lines[2]);
    if (h2.size() < 4 || !to_d(h2[2], p.temper) || !to_d(h2[3], p.xt))
      return "malformed solvent temperature line in " + path;
  }
  if (num <= 0 || p.natv <= 0 || p.natv > kMaxSites || p.ntab < 4 ||
      (int)lines.size() < num + 5 || !(dr > 0))
    return "unsupported solvent file " + path;
  const int natv = p.natv, ntab = p.ntab;
  p.sigv.assign(natv, 0);
  p.epsv.assign(natv, 0);
  p.qv.assign(natv, 0);
  p.rhov.assign(natv, 0);
  for (int i = 0; i < num; ++i) {  // solvent_read.cc:47-49, 70-76
    std::vector<std::string> a = tokens(lines[4 + i]);
    int sym;
    double sg, ep, q, den;
    if (a.size() < 11 || !to_i(a[3], sym) || !to_d(a[4], sg) ||
        !to_d(a[5], ep) || !to_d(a[6], q) || !to_d(a[10], den))
      return "malformed solvent atom line " + std::to_string(i);
    int i2 = std::abs(sym) - 1;
    if (i2 < 0 || i2 >= natv) return "solvent site symbol out of range";
    p.sigv[i2] = sg;
    p.epsv[i2] = ep;
    p.qv[i2] = q;
    p.rhov[i2] += den;
  }
  for (int i = 0; i < natv; ++i) p.rhov[i] *= phys::avogadro * 1.0e-27;
  p.xvv.assign((size_t)natv * natv * ntab, 0.0);
  size_t need = (size_t)natv * natv * ntab, got = 0;
  for (size_t li = num + 5; li < lines.size() && got < need; ++li) {
    const char *q = lines[li].c_str();
    for (;;) {
      while (*q && std::isspace((unsigned char)*q)) ++q;
      if (!*q) break;
      char *e;
      double v = std::strtod(q, &e);
      if (e == q) break;
      size_t row = got / (natv * natv);
      int kk = (int)(got % (natv * natv));
      int iv2 = kk / natv, iv1 = kk % natv;
      p.xvv[((size_t)iv2 * natv + iv1) * ntab + row] = v;
      ++got;
      q = e;
      if (got == need) break;
    }
  }
  if (got != need) return "solvent table truncated in " + path;
  double dk = M_PI / (dr * ntab);  // solvent_read.cc:81-85
  p.ttab.resize(ntab);
  for (int i = 0; i < ntab; ++i) p.ttab[i] = dk * (i + 1);
  p.has_solvent = true;
  return "";
}

// ------------------------------------------------------------ FFT plans
int factor_length(int L, int8_t *rad) {
  int k = 0, m = L;
  while (m > 1 && k < kMaxRadices) {
    int r;
    if (m % 8 == 0 && m != 16)
      r = 8;
    else if (m % 4 == 0)
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
      if (r > 16) return -1;  // prime factor beyond the generic butterfly
    }
    rad[k++] = (int8_t)r;
    m /= r;
  }
  return m == 1 ? k : -1;
}

// ----------------------------------------------------- chi shell table
// natural cubic spline coefficients (spline.cc:4-43)
static void spline_coe(const double *xp, const double *yp, int np, double *c0,
                       double *c1, double *c2) {
  std::vector<double> a(np + 1), b(np + 1), c(np + 1), d(np + 1), s(np + 1);
  int n = np - 2;
  for (int k = 1; k <= n; ++k) {
    double hl = xp[k] - xp[k - 1], hr = xp[k + 1] - xp[k];
    a[k] = hl / (hl + hr);
    b[k] = 1 - a[k];
    double q1 = (yp[k + 1] - yp[k]) / hr, q2 = (yp[k] - yp[k - 1]) / hl;
    c[k] = 6.0 * ((q1 - q2) / (hl + hr));
    d[k] = 2.0;
  }
  for (int k = 1; k < n; ++k) {
    b[k] = b[k] / d[k];
    c[k] = c[k] / d[k];
    d[k + 1] = d[k + 1] - a[k + 1] * b[k];
    c[k + 1] = c[k + 1] - a[k + 1] * c[k];
  }
  s[n] = c[n] / d[n];
  for (int k = n - 1; k >= 1; --k) s[k] = c[k] - b[k] * s[k + 1];
  s[0] = s[n + 1] = 0.0;
  for (int k = 0; k <= n; ++k) {
    double h = xp[k + 1] - xp[k];
    c1[k] = s[k] / 2.0;
    c2[k] = (s[k + 1] - s[k]) / (6.0 * h);
    c0[k] = (yp[k + 1] - yp[k]) / h - c1[k] * h - c2[k] * h * h;
  }
}
// splint.cc:4-20
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
  double t = x - xp[klo];
  return (((c2[klo] * t + c1[klo]) * t + c0[klo]) * t + yp[klo]);
}

std::string build_shells(const Problem &p, ShellTable &st) {
  const int nx = p.grid[0], ny = p.grid[1], nz = p.grid[2];
  const bool cubic = nx == ny && ny == nz && p.box[0] == p.box[1] && p.box[1] == p.box[2];
  st.cubic = cubic;
  std::vector<double> ga;  // |k| of every shell, ascending
  if (cubic) {
    // |k|^2 = (pi/L)^2 s, s = ax^2+ay^2+az^2 over odd a in [-(n-1), n-1];
    // shell (s-3)/8 (every s = 3 mod 8 up to the maximum gets a slot).
    long long smax = 3LL * (nx - 1) * (nx - 1);
    st.nshell = (int)((smax - 3) / 8 + 1);
    ga.resize(st.nshell);
    const double f = M_PI / p.box[0];
    for (int i = 0; i < st.nshell; ++i) ga[i] = f * std::sqrt((double)(3 + 8LL * i));
  } else {
    // unique |k|^2 over (|ax|,|ay|,|az|) tuples (initialize_g.cu:26-45)
    const int hx = nx / 2, hy = ny / 2, hz = nz / 2;
    const size_t nt = (size_t)hx * hy * hz;
    std::vector<double> key(nt);
    for (int iz = 0; iz < hz; ++iz)
      for (int iy = 0; iy < hy; ++iy)
        for (int ix = 0; ix < hx; ++ix) {
          // same expression as setg: k = 2 pi (j - n/2 + 1/2) / L with
          // j = n/2 + i (the k > 0 member of each +-k pair)
          double kx = 2.0 * M_PI * (ix + 0.5) / p.box[0];
          double ky = 2.0 * M_PI * (iy + 0.5) / p.box[1];
          double kz = 2.0 * M_PI * (iz + 0.5) / p.box[2];
          key[((size_t)iz * hy + iy) * hx + ix] = kx * kx + ky * ky + kz * kz;
        }
    std::vector<uint32_t> order(nt);
    for (size_t i = 0; i < nt; ++i) order[i] = (uint32_t)i;
    std::sort(order.begin(), order.end(),
              [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    st.tuple_idx.assign(nt, 0);
    double prev = -1.0;
    int ns = 0;
    for (size_t i = 0; i < nt; ++i) {
      double k2 = key[order[i]];
      if (k2 > prev) {
        ga.push_back(std::sqrt(k2));
        prev = k2;
        ++ns;
      }
      st.tuple_idx[order[i]] = (uint32_t)(ns - 1);
    }
    st.nshell = ns;
  }
  // spline of chi on the shells (solvent_spline.cu:7-96)
  const int natv = p.natv, ntab = p.ntab, nga = st.nshell;
  const std::vector<double> &tt = p.ttab;
  if (ga[nga - 1] > tt[ntab - 1]) return "insufficient maximal T tabulated";
  int ntab1 = 0;
  for (int n = 0; n < ntab; ++n)
    if (tt[n] < ga[0]) ntab1 = n;
  int ntab2 = ntab - 1;
  for (int n = ntab - 1; n > 0; --n)
    if (tt[n] > ga[nga - 1]) ntab2 = n;
  const int np = ntab2 - ntab1 + 1;
  if (np < 3) return "solvent table too coarse for this grid";
  std::vector<double> x(np), y(np), c0(np), c1(np), c2(np);
  st.chi.assign((size_t)nga * natv * natv, 0.0);
  for (int iv2 = 0; iv2 < natv; ++iv2)
    for (int iv1 = 0; iv1 < natv; ++iv1) {
      const double *tab = p.xvv.data() + ((size_t)iv2 * natv + iv1) * ntab;
      for (int k = 0; k < np; ++k) {
        x[k] = tt[ntab1 + k];
        y[k] = tab[ntab1 + k];
      }
      spline_coe(x.data(), y.data(), np, c0.data(), c1.data(), c2.data());
      const double wvv = iv1 == iv2 ? 1.0 : 0.0;
      for (int i = 0; i < nga; ++i) {
        double v = splint(x.data(), y.data(), c0.data(), c1.data(), c2.data(), np, ga[i]);
        // oz (calculate_cuda.cu:39-52): h_a = sum_b c_b xvv[a][b]
        st.chi[((size_t)i * natv + iv2) * natv + iv1] = wvv + (v - wvv);
      }
    }
  return "";
}

// --------------------------------------------------------------- .xmu
// .guv (output_guv.cu:19-49): int natv, int grid[3], double box[3],
// double shift[3], then g of every site as z-planes of x-fastest rows.
std::string write_guv(const Problem &p, const double *g, const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return "cannot write " + path;
  const int hdr[4] = {p.natv, p.grid[0], p.grid[1], p.grid[2]};
  const size_t n = (size_t)p.natv * p.grid[0] * p.grid[1] * p.grid[2];
  bool ok = std::fwrite(hdr, sizeof(int), 4, f) == 4 &&
            std::fwrite(p.box, sizeof(double), 3, f) == 3 &&
            std::fwrite(p.shift, sizeof(double), 3, f) == 3 &&
            std::fwrite(g, sizeof(double), n, f) == n;
  ok = std::fclose(f) == 0 && ok;
  return ok ? "" : "short write to " + path;
}

// .huv / .cuv text (output_huv.cu, output_cuv.cu at one rank): box, grid,
// the solute (q sig eps x y z per atom), natv, then one line per grid point
// with the value of every site; iostream's default formatting.
std::string write_grid_text(const Problem &p, const double *v, const std::string &path) {
  std::ofstream out(path);
  if (!out) return "cannot write " + path;
  out << p.box[0] << " " << p.box[1] << " " << p.box[2] << " " << std::endl
      << p.grid[0] << " " << p.grid[1] << " " << p.grid[2] << " " << std::endl
      << p.q.size() << std::endl;
  for (size_t iu = 0; iu < p.q.size(); ++iu)
    out << p.q[iu] << " " << p.sig[iu] << " " << p.eps[iu] << " " << p.r[3 * iu] << " "
        << p.r[3 * iu + 1] << " " << p.r[3 * iu + 2] << std::endl;
  out << p.natv << std::endl;
  const size_t N = (size_t)p.grid[0] * p.grid[1] * p.grid[2];
  for (size_t ig = 0; ig < N; ++ig) {
    for (int iv = 0; iv < p.natv; ++iv) out << v[(size_t)iv * N + ig] << " ";
    out << "\n";
  }
  out.flush();
  return out ? "" : "short write to " + path;
}

// .tuv (write_tuv.cu): "nx ny nz natv", then t of every site, one value per
// line, iostream's default formatting.
std::string write_tuv(const Problem &p, const double *t, const std::string &path) {
  std::ofstream out(path);
  if (!out) return "cannot write " + path;
  out << p.grid[0] << " " << p.grid[1] << " " << p.grid[2] << " " << p.natv << std::endl;
  const size_t n = (size_t)p.natv * p.grid[0] * p.grid[1] * p.grid[2];
  for (size_t i = 0; i < n; ++i) out << t[i] << "\n";
  out.flush();
  return out ? "" : "short write to " + path;
}

// read_tuv.cu: the grid and site count must match the problem (the
// reference only prints the mismatch; here it is an error).
std::string read_tuv(const Problem &p, double *t, const std::string &path) {
  std::ifstream in(path);
  if (!in) return "cannot read " + path;
  int g0 = 0, g1 = 0, g2 = 0, nv = 0;
  if (!(in >> g0 >> g1 >> g2 >> nv)) return path + ": bad header";
  if (g0 != p.grid[0] || g1 != p.grid[1] || g2 != p.grid[2] || nv != p.natv)
    return path + ": saved grid " + std::to_string(g0) + "x" + std::to_string(g1) + "x" +
           std::to_string(g2) + " with " + std::to_string(nv) + " sites does not match";
  const size_t n = (size_t)p.natv * p.grid[0] * p.grid[1] * p.grid[2];
  for (size_t i = 0; i < n; ++i)
    if (!(in >> t[i])) return path + ": truncated";
  return "";
}

// Per-atom files, iostream formatting: kind 'd' .gra (output_grad.cu: three
// values per atom), 'b' .euv (output_euv.cu: fixed, the sum over sites then
// each site), 'a' lambda derivative (output_ad.cu: one value per atom).
std::string write_atom_file(const Problem &p, char kind, const double *v,
                            const std::string &path) {
  std::ofstream out(path);
  if (!out) return "cannot write " + path;
  const size_t nu = p.q.size(), n = (size_t)p.natv;
  for (size_t a = 0; a < nu; ++a) {
    if (kind == 'd') {
      out << v[3 * a] << " " << v[3 * a + 1] << " " << v[3 * a + 2] << std::endl;
    } else if (kind == 'b') {
      double sum = 0;
      for (size_t iv = 0; iv < n; ++iv) sum += v[a * n + iv];
      out << std::fixed << sum;
      for (size_t iv = 0; iv < n; ++iv) out << " " << std::fixed << v[a * n + iv];
      out << std::endl;
    } else {
      out << v[a] << std::endl;
    }
  }
  return out ? "" : "short write to " + path;
}

std::string write_xmu(const Problem &p, const double *xmu, const double *xmu2,
                      double pmv, double pressure, const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return "cannot write " + path;
  const int natv = p.natv;
  const double ibeta = phys::avogadro * phys::boltzmann * p.temper;
  double xa = 0.0;
  for (int iv = 0; iv < natv; ++iv) xa += xmu[iv];
  const double pcterm = -pressure * pmv * ibeta;
  std::fprintf(f, " $RESULTS\n");
  std::fprintf(f, "SFE_SC= %.5f !(J/mol)\n", ibeta * xa);
  for (int iv = 0; iv < natv; ++iv)
    std::fprintf(f, "  SFEC_SC(%d)= %.5f\n", iv, ibeta * xmu[iv]);
  std::fprintf(f, "\n");
  if (p.clos == KH) {
    xa = 0.0;
    for (int iv = 0; iv < natv; ++iv) xa += xmu2[iv];
    std::fprintf(f, "SFE_SC_HNC= %.5f !(J/mol)\n", ibeta * xa);
    for (int iv = 0; iv < natv; ++iv)
      std::fprintf(f, "  SFEC_SC_HNC(%d)= %.5f\n", iv, ibeta * xmu2[iv]);
    std::fprintf(f, "\n");
  }
  xa = 0.0;
  for (int iv = 0; iv < natv; ++iv) xa += xmu[natv + iv];
  std::fprintf(f, "SFE_GF= %.5f !(J/mol)\n", ibeta * xa);
  for (int iv = 0; iv < natv; ++iv)
    std::fprintf(f, "  SFEC_GF(%d)= %.5f\n", iv, ibeta * xmu[natv + iv]);
  std::fprintf(f, "\n");
  std::fprintf(f, "PMV= %.5f !(L/mol)\n", pmv * 1000);
  std::fprintf(f, "Pressure= %.5f !(J/m^3)\n", ibeta * pressure);
  std::fprintf(f, "Correction_Term= %.5f !(J/mol)\n", pcterm);
  std::fprintf(f, " $END\n");
  std::fclose(f);
  return "";
}

}  // namespace r3d
