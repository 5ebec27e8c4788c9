/*
 * rism_oracle.h -- FP64 CPU oracle for the 3D-RISM solve (TEST INFRASTRUCTURE).
 *
 * This library is the checker, not the product. It restates, in plain C on
 * the CPU, the algorithm of the reference solver (rismical-dev/3D-RISM-CUDA-MPI,
 * directory src-cuda-mpi/) step by step, with every function citing the
 * reference file:line it follows. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference arm may load it. The CUDA product never
 * links or calls it.
 *
 * All quantities are FP64. Grids are x-fastest: index = x + nx*(y + ny*z).
 */
#ifndef RISM_ORACLE_H
#define RISM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_solver orc_solver;

/* Mixers: 0 = the reference's two-slot modified Anderson (AN2, anderson.cu),
 * 1 = history-M Anderson with fixed damping (extension; same normal
 * equations as AN2 generalised to M slots, no mp bias). */
enum { ORC_MIX_AN2 = 0, ORC_MIX_ANM = 1 };

/* Closures: KH / HNC follow calculate_cuda.cu:1-16; PSE-n is the
 * Kast-Kloss partial series expansion (extension, not in the reference). */
enum { ORC_CLOS_KH = 0, ORC_CLOS_HNC = 1, ORC_CLOS_PSE = 2 };

/* Load an .inp control file (+ optional separate structure file) and its .xvk
 * solvent file.  xvk_override may be NULL (then the file named in the .inp is
 * opened relative to the working directory, falling back to the .inp's
 * directory).  Returns NULL on error; orc_last_error() has the message. */
orc_solver *orc_load(const char *inp, const char *structure, int centering,
                     int q0, const char *xvk_override);
const char *orc_last_error(void);
void orc_free(orc_solver *s);

/* -l / -e switches of the reference CLI (set_ad.cu:5-8): adswitch 1 scales
 * the LJ sigma by lambda and drops Coulomb; 2 scales Coulomb by lambda.
 * Must be called before orc_initialize. */
void orc_set_ad(orc_solver *s, double lambda, int adswitch);
/* Closure / mixer overrides (extensions). pse_n >= 1 for ORC_CLOS_PSE. */
void orc_set_closure(orc_solver *s, int clos, int pse_n);
void orc_set_mixer(orc_solver *s, int kind, int history, double damping);

/* initialize_g + solvent spline + potentials + t0 (initialize.cu:4-44,
 * iterate.cu:31-35).  Returns 0 on success. */
int orc_initialize(orc_solver *s);
/* One Picard evaluation (calculate.cu:4-65); returns the RMS (cal_rms.cu). */
double orc_calculate(orc_solver *s);
/* One mixing step (anderson.cu:43-78 for AN2). */
void orc_mix(orc_solver *s);
/* Full loop (iterate.cu:48-82).  status: 0 converged, 1 maxstep, 2 diverged. */
int orc_iterate(orc_solver *s, int maxstep_override, int *steps, double *rms,
                int *status);
/* Thermodynamics (output.cu:23-46): xmu[2n] (closure SFE per site then GF per
 * site), xmu2[n] (HNC functional on a KH solution), pmv (m^3/mol) and
 * pressure (P/kT, mol/m^3 x ...), in the units cal_*.cu return them. */
void orc_thermo(orc_solver *s, double *xmu, double *xmu2, double *pmv,
                double *pressure);
/* Write the .xmu text file exactly as output_xmu.cu:7-82 does. */
int orc_write_xmu(orc_solver *s, const char *path);

/* Introspection for tests. */
int orc_natv(const orc_solver *s);
void orc_grid(const orc_solver *s, int *grid, double *box, double *shift);
long orc_ngrid(const orc_solver *s);
void orc_solvent(const orc_solver *s, double *rhov, double *qv, double *sigv,
                 double *epsv, double *temper, double *xt);
int orc_nu(const orc_solver *s);
void orc_solute(const orc_solver *s, double *sig, double *eps, double *q,
                double *r);
/* which: 0 u(=beta*u, per site), 1 t, 2 g, 3 h, 4 R (residual), 5 fr,
 *        6 fk (2*ngrid doubles, re/im interleaved, full shifted k grid),
 *        7 chi on the full k grid ([a][b][ngrid]). */
int orc_get(const orc_solver *s, int which, double *out);
int orc_set_t(orc_solver *s, const double *t);

/* Stand-alone shifted 3D transform (fft3d.cu semantics, test seam).
 * data: 2*nx*ny*nz doubles (complex interleaved), in place.
 * dir = -1 forward F(k)=dv*sum f e^{-ik.r}; +1 inverse f=(1/V) sum F e^{ik.r}. */
int orc_fft3d(int nx, int ny, int nz, const double *box, double *data, int dir);

#ifdef __cplusplus
}
#endif
#endif
