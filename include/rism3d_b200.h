/*
 * rism3d_b200.h -- C-ABI of the B200-native 3D-RISM solver.
 *
 * The reference solver (rismical-dev/3D-RISM-CUDA-MPI) exposes no library
 * interface: its solve path is the C++ class RISM3D (src-cuda-mpi/rism3d.h:21-105)
 * driven by main() (main.cu:6-69).  This header is the drop-in boundary for
 * that path.  Each entry point names the reference member it replaces.
 *
 * Conventions
 *  - Every call returns an int status (R3D_OK on success); the message of the
 *    last failure is r3d_last_error(ctx).  Nothing calls exit().
 *  - A context owns all of its device memory and one CUDA stream.  A context
 *    is not thread-safe; distinct contexts may be used from distinct threads.
 *  - Grids are x-fastest: index = x + nx*(y + ny*z); per-site arrays are
 *    [site][z][y][x].  Host arrays are always FP64, whatever the precision.
 *  - Plain pointers and sizes only; no C++ or framework types.
 */
#ifndef RISM3D_B200_H
#define RISM3D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define R3D_OK 0
#define R3D_EINVAL 1   /* bad argument or unsupported problem */
#define R3D_EIO 2      /* file could not be read or written */
#define R3D_ECUDA 3    /* CUDA runtime error */
#define R3D_ENOMEM 4   /* device allocation failed */
#define R3D_ESTATE 5   /* call out of order (e.g. iterate before initialize) */
#define R3D_EBUDGET 6  /* problem does not fit the context's HBM budget */

/* precision */
#define R3D_FP64 0   /* everything in FP64 (parity path) */
#define R3D_MIXED 1  /* FP32 grids/FFT/closure/OZ; FP64 reductions and solves */

/* closures */
#define R3D_KH 0
#define R3D_HNC 1
#define R3D_PSE 2 /* PSE-n, n given separately; PSE-1 == KH */

/* mixers */
#define R3D_MIX_AN2 0 /* the reference's modified Anderson (anderson.cu) */
#define R3D_MIX_ANM 1 /* Anderson with history depth m and fixed damping */

/* solve outcome (iterate.cu:73-82) */
#define R3D_CONVERGED 0
#define R3D_MAXSTEP 1
#define R3D_DIVERGED 2

/* grids for r3d_get_grid */
#define R3D_GRID_U 0   /* beta*u_v(r), per site                        */
#define R3D_GRID_T 1   /* t_v(r) = h - c, per site                      */
#define R3D_GRID_G 2   /* g_v(r), per site                              */
#define R3D_GRID_H 3   /* h_v(r), per site                              */
#define R3D_GRID_R 4   /* residual h + 1 - g of the last evaluation     */
#define R3D_GRID_FR 5  /* beta*phi_L(r) (one grid)                      */
#define R3D_GRID_FK 6  /* beta*phi_L(k) on the stored half spectrum,
                          complex interleaved [z][y][p], k_x index 2p   */
#define R3D_GRID_FKT 7 /* the same in the transform units of the
                          iteration's passes and of r3d_slab_transform
                          (divided by dv C(k)): what a solve split over
                          GPUs subtracts from q_v-scaled c(k)           */
#define R3D_GRID_CHI 8 /* chi_vv'(|k|) on the stored half spectrum,
                          [v][v'][z][y][p] (the solvent susceptibility
                          the OZ step of calculate_cuda.cu:39-52 uses)  */

typedef struct r3d_ctx r3d_ctx;

typedef struct r3d_opts {
  int device;                    /* CUDA device ordinal                      */
  int precision;                 /* R3D_FP64 or R3D_MIXED                    */
  unsigned long long hbm_budget; /* bytes this context may hold; 0 = any     */
  int verbose;                   /* 1: print " Step = i Reside = rms"        */
} r3d_opts;

/* Context lifetime (replaces `new RISM3D` / delete, main.cu:14). */
int r3d_create(const r3d_opts *opts, r3d_ctx **out);
int r3d_destroy(r3d_ctx *ctx);
const char *r3d_last_error(const r3d_ctx *ctx); /* ctx may be NULL */

/* RISM3D::set_ad (set_ad.cu:5-8): -l (adswitch 1) / -e (adswitch 2). */
int r3d_set_ad(r3d_ctx *ctx, double lambda, int adswitch);

/* RISM3D::read_input (read_input.cu:21-97) with Solute::centering/zero
 * (solute.cu:18-54) and set_fname (set_fname.cu:5-12).  structure may be
 * NULL (atoms follow in the .inp).  Reads the control deck only. */
int r3d_load_inp(r3d_ctx *ctx, const char *inp, const char *structure,
                 int centering, int q0);

/* Solvent::read (solvent_read.cc:10-94).  path NULL: the file named in the
 * .inp, opened relative to the working directory, else next to the .inp. */
int r3d_load_xvk(r3d_ctx *ctx, const char *path);

/* In-memory problem (alternative to the two loaders). Arrays are copied. */
typedef struct r3d_problem {
  int grid[3];
  double box[3];
  int closure, pse_n;
  double convergence;
  int maxstep;
  int count;       /* AN2 Picard warm-up steps */
  double m, mp;    /* AN2 damping and newest-slot bias */
  int nu;          /* solute atoms */
  const double *sig, *eps, *q; /* [nu]; eps in J/mol, q in e */
  const double *xyz;           /* [nu][3], Angstrom (used as given) */
  int natv;        /* unique solvent sites */
  const double *sigv, *epsv, *qv, *rhov; /* [natv]; rhov in 1/A^3 */
  double temper, xt;           /* K, 1/Pa */
  int ntab;
  double dr;                   /* table spacing: k_i = (i+1) pi / (dr ntab) */
  const double *xvv;           /* [natv][natv][ntab] */
} r3d_problem;
int r3d_set_problem(r3d_ctx *ctx, const r3d_problem *p);

/* Extensions of the input surface (the .inp keeps the reference's format). */
int r3d_set_closure(r3d_ctx *ctx, int closure, int pse_n);
int r3d_set_mixer(r3d_ctx *ctx, int mixer, int history, double damping);
int r3d_set_control(r3d_ctx *ctx, double convergence, int maxstep);

/* RISM3D::initialize after read_input (initialize.cu:4-44): k shells and
 * chi (initialize_g.cu, solvent_spline.cu), potentials (cal_potential.cu,
 * cal_LJ.cu, cal_Coulomb.cu) and t0 (initialize_tuv.cu). */
int r3d_initialize(r3d_ctx *ctx);

/* RISM3D::calculate + cal_rms (calculate.cu:4-65, cal_rms.cu:14-26):
 * one Picard evaluation; *rms receives sqrt(sum R^2 / (N n)). */
int r3d_calculate(r3d_ctx *ctx, double *rms);

/* AN2::calculate (anderson.cu:43-78) or the history-m mixer: one update of t
 * from the last evaluation. */
int r3d_anderson(r3d_ctx *ctx);

/* RISM3D::iterate (iterate.cu:6-107): evaluate, test, mix until converged,
 * diverged or maxstep.  status: R3D_CONVERGED / R3D_MAXSTEP / R3D_DIVERGED. */
int r3d_iterate(r3d_ctx *ctx, int *steps, double *rms, int *status);

/* RISM3D::output 'm' branch (output.cu:23-46): xmu[2*natv] (closure SFE per
 * site, then GF per site), xmu2[natv] (HNC functional on a KH solution),
 * pmv (m^3/mol), pressure (P/kT) -- the values cal_exchem, cal_pmv and
 * cal_pressure return, before output_xmu's unit conversion. */
int r3d_thermo(r3d_ctx *ctx, double *xmu, double *xmu2, double *pmv,
               double *pressure);

/* output_xmu (output_xmu.cu:7-82). path NULL: <stem>.xmu (or .xmu0 for -z). */
int r3d_write_xmu(r3d_ctx *ctx, const char *path);

/* Device -> host copy of a grid (FP64), see R3D_GRID_*. */
int r3d_get_grid(r3d_ctx *ctx, int which, double *host);
/* Host -> device t (FP64 [natv][N]); e.g. a restart. */
int r3d_set_t(r3d_ctx *ctx, const double *host);

/* Problem facts. */
int r3d_info(const r3d_ctx *ctx, int *grid3, int *natv, long long *ngrid,
             int *nu);
/* Charges (e) and number densities (molecules/A^3) of the solvent's site
 * classes, natv values each, in the order of the grids' sites: the q_v and
 * rho_v of Solvent::read (solvent_read.cc:30-85) after r3d_load_xvk.  What a
 * solve split over GPUs (slabs.py's DistSolve) takes besides the grids. */
int r3d_solvent_sites(const r3d_ctx *ctx, double *qv, double *rhov);
/* Device bytes the context holds (after initialize) or will need (before). */
int r3d_device_bytes(const r3d_ctx *ctx, unsigned long long *bytes);
/* CUDA-event time of the last r3d_iterate loop, ms per iteration, and the
 * number of kernels one iteration launches. */
int r3d_iter_timing(const r3d_ctx *ctx, double *ms_per_iter,
                    int *kernels_per_iter);

/* Times of the last r3d_initialize, ms: [0] the grid potentials (LJ and
 * real-space Coulomb pair sums, cal_LJ.cu / cal_Coulomb.cu's real-space
 * part), [1] the k-space Coulomb sum (cal_Coulomb.cu's fk), [2] the
 * long-range h term, all CUDA-event times, and [3] the whole initialize
 * (host clock, shells and uploads included).  No counterpart in the
 * reference beyond its -DTEST timers (initialize.cu). */
int r3d_setup_timing(const r3d_ctx *ctx, double *ms);

/* Refreshes of the mixed path's FP64 long-range reference made by the
 * iterations since r3d_initialize (c_ref frozen at the current t, h_ref
 * recomputed in FP64), and their host-clock time in ms, launch to
 * completion.  No counterpart in the reference (its iteration is FP64
 * throughout); 0 on the FP64 path. */
int r3d_refresh_timing(const r3d_ctx *ctx, int *count, double *ms);

/* Advance the solve by exactly `nsteps` iterations (graph replays, no
 * convergence polling; converged or diverged solves do no further work) and
 * return their CUDA-event time in *ms.  No counterpart in the reference: the
 * benchmark and batch loops use it to time iterations without host syncs. */
int r3d_step(r3d_ctx *ctx, int nsteps, double *ms);

/* Per-kernel CUDA-event timing of one iteration's kernels, each launched
 * `reps` times in isolation: names (comma separated, <= len bytes), average
 * ms per launch and algorithmic bytes per launch (compulsory reads + writes
 * of the kernel's arrays).  Restores t afterwards and resets the mixer, so
 * the next iterate() starts from the same t.  *nk receives the kernel count
 * (arrays hold up to 16 entries). */
int r3d_profile_kernels(r3d_ctx *ctx, int reps, char *names, int len,
                        double *ms, double *bytes, int *nk);

/* State of the solve: completed evaluations, last RMS, and R3D_CONVERGED /
 * R3D_MAXSTEP / R3D_DIVERGED, or -1 while still running. */
int r3d_status(r3d_ctx *ctx, int *steps, double *rms, int *status);

/* Bytes copied host->device and device->host by this context so far. */
int r3d_transfer_bytes(const r3d_ctx *ctx, unsigned long long *h2d,
                       unsigned long long *d2h);

/* ---- grid files (RISM3D::output's 'g', 'h', 'c' and the .tuv restart) ----
 * path NULL: the deck's stem (set_fname.cu) with the reference's extension.
 * r3d_write_guv: output_guv.cu:19-49, binary: int natv, int grid[3],
 *   double box[3], double shift[3], then g per site as z-planes of x-fastest
 *   rows (default <stem>.guv).
 * r3d_write_huv / r3d_write_cuv: output_huv.cu / output_cuv.cu at one rank,
 *   text: box, grid, solute atoms (q sig eps x y z), natv, then one line per
 *   grid point with h (or c = h - t) of every site (default <stem>.huv0 /
 *   <stem>.cuv0, the rank-0 file names).
 * r3d_write_tuv: write_tuv.cu, text "nx ny nz natv" then t per site, one value
 *   per line (default <stem>.tuv).  r3d_iterate also writes it every ksave
 *   steps (ksave > 0) and at convergence (ksave != 0), as iterate.cu:63-70.
 * r3d_read_tuv: read_tuv.cu, then loads t into the solve (the reference reads
 *   the file but never copies it to the device); after r3d_initialize.
 * r3d_output: RISM3D::output (output.cu): the files of the letters of
 *   outlist (NULL: the deck's) -- m (.xmu), d (.gra), c, g, h, a (lambda
 *   derivative), b (.euv). */
int r3d_write_guv(r3d_ctx *ctx, const char *path);
int r3d_write_huv(r3d_ctx *ctx, const char *path);
int r3d_write_cuv(r3d_ctx *ctx, const char *path);
int r3d_write_tuv(r3d_ctx *ctx, const char *path);
int r3d_read_tuv(r3d_ctx *ctx, const char *path);
int r3d_output(r3d_ctx *ctx, const char *outlist);

/* ---- post-solve per-atom integrals over g ---------------------------------
 * cal_grad.cu:41-90 (grad, [nu][3], kcal/(mol A)), cal_euv.cu:29-65 (euv,
 * [nu][natv], J/mol), cal_ad1.cu / cal_ad2.cu (ad, [nu], kcal/mol: the LJ
 * lambda derivative after r3d_set_ad(ctx, lambda, 1), else the Coulomb one),
 * in the units the reference writes them; any output may be NULL.  One
 * launch covers every atom, site and voxel (the reference launches a full
 * grid per atom and site).  The writers produce output_grad.cu's .gra,
 * output_euv.cu's .euv and output_ad.cu's <stem>-<adswitch>-<lambda>
 * (path NULL: those names). */
int r3d_atom_integrals(r3d_ctx *ctx, double *grad, double *euv, double *ad);
int r3d_write_gra(r3d_ctx *ctx, const char *path);
int r3d_write_euv(r3d_ctx *ctx, const char *path);
int r3d_write_ad(r3d_ctx *ctx, const char *path);

/* FFT3D::execute (fft3d.cu:72-78), stand-alone test seam: the reference's
 * half-shifted 3D transform F(k) = dv sum_r f(r) e^{-i k.r} of a real grid.
 * dir -1: in = real [N], out = complex interleaved half spectrum [z][y][p]
 *         (k_x index 2p of the full grid, all k_y, k_z);
 * dir +1: in = that half spectrum, out = real f(r) = (1/V) sum_k F(k) e^{ik.r}.
 * Runs on `device` with `precision`; allocates and frees its own buffers. */
int r3d_fft3d(int device, int precision, int nx, int ny, int nz,
              const double *box, int dir, const double *in, double *out);

/* No counterpart in the reference.  r3d_fft3d (FP64) for callers that
 * cannot allocate device memory: code running while another framework owns
 * the device's memory pool, and real-time loops that must not enter the
 * allocator.  d_in / d_out are the caller's device buffers, in the layouts
 * of r3d_fft3d; the only working storage is one fixed array of
 * R3D_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds until
 * the process exits.  Grids with nx/2*ny*nz above
 * (R3D_NOALLOC_SCRATCH_BYTES - 16384) / 16 points (about 2.1 million:
 * 160^3) are rejected with R3D_EBUDGET.  All calls on a device share the
 * array: calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on each device looks up the array's address (under
 * a lock, so concurrent first calls from several host threads are safe); make
 * it before any stream capture.  stream may be NULL (the default stream);
 * the work is ordered after what the caller queued on that stream, and the
 * call returns after it has finished.  The caller's current device is
 * restored on return.  A CUDA error already pending in the process is
 * reported (R3D_ECUDA) and left pending.  Errors are reported by
 * r3d_last_error(NULL). */
#define R3D_NOALLOC_SCRATCH_BYTES (32u << 20)
int r3d_fft3d_noalloc(int device, int nx, int ny, int nz, const double *box,
                      int dir, const double *d_in, double *d_out, void *stream);

/* One rank's stages of the shifted 3D transform when a grid is split over
 * several GPUs (the reference's distributed FFT3D, fft3d.cu:81-163, with the
 * pencil decomposition of cell.cc:30-48; here z-slabs for the x and y passes
 * and y-slabs for the z pass, moved between by one all-to-all per direction,
 * which the caller runs -- slabs.py with NCCL).  Device buffers, FP64, on
 * `device` and `stream` (NULL: the default stream); the call returns when the
 * stage has finished.  (nx, ny, nz) are the slab's own extents:
 *   stage 0  d_real [nz][ny][nx] (a z-slab; it must start on an even global
 *            plane) -> d_spec [nz][ny][nx/2] complex: x and y transforms
 *   stage 1  d_spec [nz][ny][nx/2] (a y-slab, all z) -> z transform, in place
 *   stage 2  the inverse z transform, in place
 *   stage 3  d_spec (z-slab; destroyed) -> d_real: inverse y and x transforms
 * in unnormalised transform units (the constant phase dv C(k) of r3d_fft3d
 * left out; stages 0-1 then 2-3 return the grid times nx ny nz / 2). */
int r3d_slab_transform(int device, int stage, int nx, int ny, int nz, double *d_spec,
                       double *d_real, void *stream);
/* The same stages for nsites grids (solvent sites, 1 <= nsites <= 16) in one
 * call, each buffer holding them one after another ([site][slab]);
 * r3d_slab_transform is the one-site case.  A site count outside that range,
 * or slabs whose tiles for every site do not fit one CTA's shared memory, is
 * R3D_EINVAL. */
int r3d_slab_transform_sites(int device, int stage, int nsites, int nx, int ny, int nz,
                             double *d_spec, double *d_real, void *stream);

/* One rank's pointwise steps of a solve split over GPUs (slabs.py's DistSolve
 * runs the iteration: these, r3d_slab_transform, NCCL all-to-alls between
 * the slab layouts and all-reduces of the sums).  They are the steps of the
 * reference's calculate() and AN2 mixer on the rank's own pencil
 * (calculate_cuda.cu: trm1mt, mqvfk, oz, tr; anderson_cuda.cu:1-67), whose
 * sums cal_rms.cu:23 and anderson.cu:95 reduce over ranks.  FP64 device
 * buffers on `device`; each call is asynchronous on `stream` (NULL: the
 * default stream) and returns the launch status.  n <= 16 sites; qv (host,
 * n values) the site charges.
 *   r3d_dist_closure   z-slab: g = closure(-u + t), c = g - 1 - t + q_v fr
 *                      (u, t, g, c [n][nloc]; fr [nloc])
 *   r3d_dist_oz        y-slab, in place: spec_v <- sum_v' chi_vv' (spec_v' -
 *                      q_v' fk) (spec [n][nk] complex, chi [n][n][nk], fk
 *                      [nk] complex in transform units: R3D_GRID_FKT)
 *   r3d_dist_residual  z-slab: R = scale h + 1 - g and its sums into d_sums
 *                      ([0] sum R^2, [1 + 5v + k] the five AN2 theta dots of
 *                      site v when dots != 0); d_sums holds
 *                      R3D_DIST_SUMS_DOUBLES doubles (work space after the
 *                      sums)
 *   r3d_dist_mix       newdt0 (picard != 0: t += R) or newdt with the AN2
 *                      coefficients s1, s2 and damping m; t and R go to slot
 *                      `binary` (tp0/tp1, rp0/rp1) first */
#define R3D_DIST_SUMS_DOUBLES (1 + 5 * 16 + 16 * 296 * 6)
int r3d_dist_closure(int device, int n, long long nloc, int closure, int pse_n,
                     const double *d_u, const double *d_t, const double *d_fr,
                     const double *qv, double *d_g, double *d_c, void *stream);
int r3d_dist_oz(int device, int n, long long nk, const double *d_chi, const double *d_fk,
                const double *qv, double *d_spec, void *stream);
int r3d_dist_residual(int device, int n, long long nloc, double scale, const double *d_h,
                      const double *d_g, const double *d_rp0, const double *d_rp1, int dots,
                      double *d_r, double *d_sums, void *stream);
int r3d_dist_mix(int device, long long count, double *d_t, const double *d_r, double *d_tp0,
                 double *d_tp1, double *d_rp0, double *d_rp1, int binary, int picard,
                 double s1, double s2, double m, void *stream);
/* The history-m Anderson mixer of the split solve (the library's own
 * extension of AN2; no counterpart in the reference):
 *   r3d_dist_anm_dots  d_sums[0] = <R, R>, d_sums[1 + i] = <R, f_i> for the m
 *                      stored residuals d_hist[i] (host array of device
 *                      pointers, m <= 16), each summed over the rank's points
 *                      of every site with the weights irho[v] = 1 / rho_v
 *                      (host); d_sums holds R3D_DIST_ANM_SUMS_DOUBLES doubles
 *   r3d_dist_anm_mix   d_tn = w0 t + sum alpha_i x_i + beta (w0 R + sum
 *                      alpha_i f_i), w0 = 1 - sum alpha_i (alpha: host, m
 *                      values; d_x / d_f: host arrays of device pointers) */
#define R3D_DIST_ANM_SUMS_DOUBLES (1 + 16 + 16 * 296 * 17)
int r3d_dist_anm_dots(int device, int n, long long nloc, const double *d_r, int m,
                      const double *const *d_hist, const double *irho, double *d_sums,
                      void *stream);
int r3d_dist_anm_mix(int device, long long count, const double *d_t, const double *d_r, int m,
                     const double *const *d_x, const double *const *d_f, const double *alpha,
                     double beta, double *d_tn, void *stream);

/* ---- batches of independent solves --------------------------------------
 * The reference runs one solve per process (main.cu:63-65).  A batch iterates
 * many initialized contexts together: the solves of one geometry (grid,
 * solvent sites, mixer) share every kernel launch of an iteration, which is
 * what makes many small solves (48^3-128^3 grids, a few ms of work each) use
 * the whole GPU.  Each solve keeps its own closure, tolerance, maxstep and
 * mixer parameters and stops on its own; results are read per context
 * (r3d_status, r3d_thermo, r3d_write_xmu, r3d_get_grid).  All contexts of a
 * batch share the device and the precision; a context belongs to at most one
 * batch at a time and must not be used on its own during r3d_batch_iterate.
 * Errors are reported by r3d_last_error(NULL). */
typedef struct r3d_batch r3d_batch;
int r3d_batch_create(int device, r3d_batch **out);
/* Adds an initialized context (not owned: destroy it yourself, after the
 * batch). */
int r3d_batch_add(r3d_batch *b, r3d_ctx *ctx);
/* RISM3D::iterate (iterate.cu:6-107) for every solve of the batch at once:
 * fresh mixer state, iterations until every solve has converged, diverged
 * or reached its maxstep.  iterations: the largest step count of any solve;
 * ms: device time of the whole loop. */
int r3d_batch_iterate(r3d_batch *b, int *iterations, double *ms);
/* solves, geometry groups (launches per kernel of an iteration), kernels per
 * iteration of the batch's graph (after the first r3d_batch_iterate). */
int r3d_batch_info(const r3d_batch *b, int *solves, int *groups, int *kernels_per_iter);
/* Frees the batch's own buffers; its contexts stay valid. */
int r3d_batch_destroy(r3d_batch *b);

/* ---- serving: continuous batching of submitted solves ------------------
 * No counterpart in the reference (one solve per process).  A server owns
 * one device, one submission thread and an HBM budget.  Submitted decks are
 * admitted while the budget and max_active allow: each is initialized on its
 * own stream while the admitted solves keep iterating, then takes a slot of
 * its geometry class (grid, solvent sites, mixer); every kernel of an
 * iteration covers all slots of a class, so solves that arrived at different
 * times iterate together, and each one retires on convergence (or
 * divergence, or maxstep) without stopping the others.  With closure_ladder,
 * a PSE-n deck is solved as KH, then PSE-2, ..., PSE-n, each stage starting
 * from the previous one's t (the usual route to PSE-n convergence).  Each
 * result equals the result of the same solve run alone (r3d_iterate per
 * stage) on the same precision.  Errors: r3d_last_error(NULL). */
#define R3D_REQ_QUEUED 0
#define R3D_REQ_ACTIVE 1
#define R3D_REQ_DONE 2
#define R3D_REQ_FAILED 3

typedef struct r3d_server r3d_server;
typedef struct r3d_server_opts {
  int device;
  int precision;                 /* R3D_FP64 or R3D_MIXED */
  unsigned long long hbm_budget; /* bytes for admitted solves; 0: 85% of free memory */
  int max_active;                /* most solves admitted at once; 0: no limit */
  int chunk;                     /* iterations between admissions/retirements; 0: 8 */
  int closure_ladder;            /* 1: solve PSE-n decks as KH, PSE-2, ..., PSE-n */
} r3d_server_opts;

typedef struct r3d_result {
  int state;    /* R3D_REQ_* */
  int status;   /* R3D_CONVERGED / R3D_MAXSTEP / R3D_DIVERGED (state DONE) */
  int steps;    /* iterations of the last closure stage */
  int steps_total; /* iterations of all stages */
  int natv;
  double rms;
  double xmu[32], xmu2[16], pmv, pressure; /* r3d_thermo's outputs (state DONE) */
  double queued_s, admitted_s, finished_s; /* seconds since r3d_server_create */
  char error[256];                          /* state FAILED */
} r3d_result;

int r3d_server_create(const r3d_server_opts *opts, r3d_server **out);
/* Queues the deck (and .xvk; NULL: the one the deck names).  The deck is
 * parsed here, so a bad deck fails the call; ticket identifies the solve. */
int r3d_server_submit(r3d_server *s, const char *inp, const char *xvk, long long *ticket);
/* Current state (and results once done) of a ticket. */
int r3d_server_poll(r3d_server *s, long long ticket, r3d_result *out);
/* Waits up to timeout_s seconds (< 0: no limit) for DONE or FAILED, then
 * does what r3d_server_poll does. */
int r3d_server_wait(r3d_server *s, long long ticket, double timeout_s, r3d_result *out);
/* output_xmu's .xmu of a finished solve. */
int r3d_server_write_xmu(r3d_server *s, long long ticket, const char *path);
/* Forgets a finished ticket. */
int r3d_server_release(r3d_server *s, long long ticket);
/* Finishes every queued and admitted solve, then frees the server. */
int r3d_server_destroy(r3d_server *s);

/* ---- 1D XRISM solvent solve: making .xvk tables -------------------------
 * The reference reads its solvent susceptibility from an .xvk table
 * (solvent_read.cc:10-94) and ships no program that makes one.  These calls
 * make it: an extended-RISM (XRISM) solve of the bulk solvent on a radial
 * grid, written in the format solvent_read.cc:31-85 reads.
 *
 * The solvent is the .xvk atom table: one line per atom of each molecule
 * (species) with its site class `sym` (atoms whose |sym| agree are one site
 * of the 3D solve, solvent_read.cc:70-76), LJ sigma [A] and epsilon
 * [J/mol] (Lorentz-Berthelot mixing), charge [e], position [A] in its
 * molecule and density [M].  Grid: r_i = i dr and k_j = j pi/(ntab dr),
 * i, j = 1..ntab-1; ntab a power of two in [64, 16384].  Closure on
 * t = h - c_s with the Coulomb split erf(r/1 A)/r (its k-space part added
 * analytically); charges switched on over `nladder` stages (every stage but
 * the last stops at RMS 1e-5); modified-DIIS mixing of `history` entries
 * with step `mix`, halved (and the stage's best state restored) whenever
 * the RMS grows tenfold over the stage's best.  The table row j holds
 * xvv[A][B](k_j) = sum_{b in B} (w_ab(k_j) + rho_b h_ab(k_j)) (row ntab: the
 * intramolecular part alone), the quantity calculate_cuda.cu:39-52 uses.
 * Errors are reported by r3d_last_error(NULL). */
typedef struct r3d_xrism_atom {
  char name[8];      /* label written to the table                 */
  int species;       /* molecule index (SPC column), 1-based        */
  int sym;           /* site class (SYM column); sign ignored       */
  double sigma;      /* A                                           */
  double epsilon;    /* J/mol                                       */
  double charge;     /* e                                           */
  double x, y, z;    /* A, within the molecule                      */
  double density;    /* M (mol/L) of the molecule                   */
} r3d_xrism_atom;

typedef struct r3d_xrism_opts {
  int device;         /* CUDA device ordinal                         */
  int ntab;           /* grid points (power of two, 64..16384)        */
  double dr;          /* A                                           */
  double temperature; /* K                                           */
  int closure;        /* R3D_KH, R3D_HNC or R3D_PSE                   */
  int pse_n;          /* PSE order (R3D_PSE)                          */
  double tol;         /* RMS of the t update that ends the solve      */
  int maxstep;        /* evaluations per coupling stage               */
  int history;        /* DIIS entries, 1..32                          */
  double mix;         /* DIIS step                                    */
  int nladder;        /* charge-coupling stages, >= 1                 */
  int verbose;        /* 1: print the RMS of each evaluation          */
} r3d_xrism_opts;

typedef struct r3d_xrism_result {
  int status;        /* R3D_CONVERGED / R3D_MAXSTEP / R3D_DIVERGED   */
  int steps;         /* evaluations over all stages                  */
  int natv;          /* site classes (table is [ntab][natv][natv])   */
  double rms;        /* RMS of the last evaluation                   */
  double xt;         /* isothermal compressibility [1/Pa]            */
  double ms_device;  /* device time of the iterations                */
} r3d_xrism_result;

/* Defaults: KH, tol 1e-10, maxstep 10000, history 20, mix 0.3, nladder 5,
 * ntab 8192, dr 0.05, 298.15 K, device 0. */
void r3d_xrism_default_opts(r3d_xrism_opts *opts);
/* Reads the header and atom table of an .xvk (the table itself, if any, is
 * ignored) into atoms[0..max_atoms) and opts' ntab, dr and temperature. */
int r3d_xrism_read_deck(const char *path, r3d_xrism_atom *atoms, int max_atoms,
                        int *natom, r3d_xrism_opts *opts);
/* One solve on the GPU.  xvv (may be NULL): [ntab][natv][natv] host array,
 * natv = the largest |sym|.  The table is written only when the solve
 * converged (status R3D_CONVERGED); the call returns R3D_OK either way. */
int r3d_xrism_solve(const r3d_xrism_opts *opts, const r3d_xrism_atom *atoms, int natom,
                    double *xvv, r3d_xrism_result *result);
/* Writes the .xvk (solvent_read.cc:31-58 layout, one table row per line). */
int r3d_xrism_write_xvk(const char *path, const r3d_xrism_opts *opts,
                        const r3d_xrism_atom *atoms, int natom, const double *xvv,
                        double xt);

#ifdef __cplusplus
}
#endif
#endif /* RISM3D_B200_H */
