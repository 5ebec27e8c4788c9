// r3d_internal.h -- internal types shared by the host runtime and the CUDA
// kernels of the B200 3D-RISM solver.  Nothing here is part of the C-ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace r3d {

constexpr int kMaxSites = 16;    // unique solvent sites per solve
constexpr int kMaxRadices = 12;  // factors of one FFT length
constexpr int kMaxHistory = 32;  // ANM history depth
constexpr int kThreads = 256;    // CTA size of every grid pass

enum Closure : int { KH = 0, HNC = 1, PSE = 2 };
enum Mixer : int { MIX_AN2 = 0, MIX_ANM = 1 };
enum Status : int { RUNNING = 0, CONVERGED = 1, DIVERGED = 2, MAXSTEP = 3 };

// ---------------------------------------------------------------------------
// Host-side problem description (what read_input.cu / solvent_read.cc build).
struct Problem {
  // control (.inp)
  std::string outlist = "m";
  int ksave = 0;
  int clos = KH, pse_n = 1;
  std::string fsolvent;
  double convergence = 1e-6;
  int maxstep = 10000;
  int count = 2;
  double mix_m = 0.6, mix_mp = 0.2;
  double box[3] = {0, 0, 0};
  int grid[3] = {0, 0, 0};
  double shift[3] = {0, 0, 0};
  std::string fname;  // output stem (set_fname.cu)
  bool zero = false;  // -z
  int adswitch = 0;
  double lambda = 1.0;
  // solute
  std::vector<double> sig, eps, q, r;  // r: xyz AoS
  // solvent (.xvk)
  int natv = 0, ntab = 0;
  double temper = 0, xt = 0;
  std::vector<double> sigv, epsv, qv, rhov, ttab;
  std::vector<double> xvv;  // [iv2][iv1][ntab]
  bool has_solute = false, has_solvent = false;
};

// Parsers / writers (r3d_host.cc).  Return "" on success, else the message.
std::string parse_inp(Problem &p, const std::string &inp,
                      const std::string &structure, bool centering, bool q0);
std::string parse_xvk(Problem &p, const std::string &path);
// Grid files (output_guv.cu:19-49, output_huv.cu, output_cuv.cu,
// write_tuv.cu, read_tuv.cu): grids [site][z][y][x], N = nx ny nz per site.
std::string write_guv(const Problem &p, const double *g, const std::string &path);
std::string write_grid_text(const Problem &p, const double *v, const std::string &path);
std::string write_tuv(const Problem &p, const double *t, const std::string &path);
std::string read_tuv(const Problem &p, double *t, const std::string &path);
std::string write_atom_file(const Problem &p, char kind, const double *v, const std::string &path);
std::string write_xmu(const Problem &p, const double *xmu, const double *xmu2,
                      double pmv, double pressure, const std::string &path);

// chi shell table: values of chi_ab at every |k| shell of the half spectrum
// (reference: initialize_g.cu + solvent_spline.cu).  `kidx_host` is empty for
// cubic boxes (the device derives the shell from the odd-integer norm).
struct ShellTable {
  int nshell = 0;
  bool cubic = false;
  std::vector<double> chi;          // [nshell][a][b]
  std::vector<uint32_t> tuple_idx;  // non-cubic: [|az|/2][|ay|/2][|ax|/2]
};
std::string build_shells(const Problem &p, ShellTable &st);

// FFT factor plan: radices outermost first.
int factor_length(int L, int8_t *rad);

// Precision of one solve: R = grid type (half spectra, u, L, residual and
// residual history), T = state type (t and its mixing history).  The mixed
// path keeps T in FP64: g = e^{t-u} multiplies any rounding of t by g (up to
// ~30 at ion contact peaks), which an FP32 t would put at ~1e-5 in R.
struct P64 {
  using R = double;
  using T = double;
};
struct PMix {
  using R = float;
  using T = double;
};

// ---------------------------------------------------------------------------
// Device-side control block of one solve (lives in device memory).
struct Ctl {
  int status;      // Status
  int step;        // completed calculate() evaluations
  int maxstep;
  int mix_flag;    // mix requested by the last solve step
  int count_left;  // AN2 Picard warm-up steps left
  int binary;      // AN2 ping-pong slot
  int hcount;      // ANM valid history entries
  int hhead;       // ANM ring head (slot receiving the newest pair)
  double tol;
  double rms;
  double ss;       // sum R^2
  double coef[kMaxHistory + 4];  // mixing coefficients
  double gram[(kMaxHistory + 1) * (kMaxHistory + 1)];  // ANM <f_i, f_j>
  int mix_head;                  // ANM: ring slot of the newest pair
  int mix_m;                     // ANM: history entries used by this mix
  int mix_slots[kMaxHistory];    // ANM: their ring slots
  int err;                       // device-side error word
};

// Per-solve descriptor read by every pass kernel (device memory).
struct Desc {
  int nx, ny, nz, n;  // grid and unique solvent sites
  int hx;             // nx / 2 (length of the packed x transform)
  long long N, Nh;    // voxels, half-spectrum points (hx*ny*nz)
  // site / slot strides of the per-site arrays (elements): N and Nh padded
  // off powers of two so that the many streams of one kernel do not all
  // land on the same DRAM channels
  long long Ns, Nhs;
  int clos, pse_n;
  int mixer, history;
  double beta;        // ANM damping
  double m, mp;       // AN2 parameters
  double irho[kMaxSites];
  double qv[kMaxSites];
  // tile shapes
  int rows;     // FX/IX rows per CTA
  int ycols;    // FY/IY x-columns per CTA
  int zcols;    // ZOZ x-columns per CTA
  int tiles_x, tiles_y, tiles_z;  // CTAs per pass
  int partial_base;  // first partial slot of this solve
  // FFT plans (radices outermost first)
  int8_t rad_x[kMaxRadices], rad_y[kMaxRadices], rad_z[kMaxRadices];
  int nrad_x, nrad_y, nrad_z;
  // compile-time-engine passes: columns per tile, 0 = runtime-length engine
  int ct_x, ct_y, ct_z;
  int cubic;  // nx = ny = nz and a cubic cell: shell index computed, no kidx
  int chis;   // chi row stride (elements): n*n rounded up to a multiple of 4
  // twiddle tables of the compile-time engine (complex, grid type):
  // tw* = e^{-2 pi i e / L}, pw* = half-sample e^{-i pi a / n} of each pass
  const void *twx, *pwx, *twy, *pwy, *twz, *pwz;
  // buffers (typed by the kernel's real type)
  // u = beta u - q_v beta phi_L(r) and t = t - q_v beta phi_L(r) (the
  // short-range parts); cref = frozen c_s of the last refresh (or null);
  // lr = 1 + h_ref with h_ref = F^-1[chi (F(cref) - q beta phi_L(k))];
  // fk = beta phi_L(k) in transform units (FP64; subtracted in the OZ step
  // only when non-null, i.e. in the refresh pipeline)
  void *u, *t, *fr, *res, *w, *fk, *chi, *lr, *cref;
  // gq: g = closure(-u + t) as the iteration's FX evaluated it (state type,
  // FP64), left for the IX of the same evaluation, which reads it instead of
  // t and u and evaluates no closure.  (Stored in FP32, as g - 1, it added
  // enough noise to R near convergence to cost the mixed path 14 % more
  // iterations at 256^3.)
  void *gq;
  const uint32_t *kidx;  // [z][y][p] shell index of each half-spectrum point
  // AN2: tp, rp [2][n][N]; ANM: fring, zring [H+1][n][N] (res aliases a slot)
  void *hist_a, *hist_b;
  double *partials;  // [ctas][kPartials]
  double *rmslog;    // [maxstep] rms of every evaluation
  Ctl *ctl;
  // tensor maps (CUtensorMap) of the half spectrum w for the iteration's
  // y and z passes on the copy engine: 4D [site][z][y][x] in 8-byte
  // elements, boxes of PC x-columns by a y column (tm_y) or by a z column of
  // every site (tm_z); tma_pc_* = 0: not built
  struct alignas(64) Tmap {
    unsigned char b[128];
  };
  Tmap tm_y, tm_z;
  int tma_pc_y, tma_pc_z;
  const int *yrev;  // [ny]: ky index of each digit-reversed y row of w
  // polls of a staged pass's bounded wait for its copies before it gives up
  // (sets the error word); <= 0: the default, far beyond any copy's latency.
  // Set smaller only to exercise that error path (R3D_WAIT_POLLS).
  int wait_polls;
};

constexpr int kPartials = 1 + 5 * kMaxSites;  // sum R^2 + per-site dots

// Atoms of the post-solve per-atom integrals (k_atom_integrals)
struct IntAtoms {
  const double *x, *y, *z, *q;  // [nu], device
  const double *sig, *eps;      // [n][nu], device: sigma_uv (with the LJ lambda), sqrt(eps_u eps_v)
  double qv[kMaxSites], rhov[kMaxSites];
  int nu, n, ad1;  // ad1: the LJ lambda derivative (else the Coulomb one)
  double lambda, cc;
};

}  // namespace r3d
