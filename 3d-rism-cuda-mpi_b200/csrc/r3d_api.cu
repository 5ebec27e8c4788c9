// r3d_api.cu -- C-ABI and host runtime of the B200 3D-RISM solver.
//
// A context mirrors one RISM3D object of the reference (rism3d.h:21-105):
// load the control/solute deck and the solvent table, initialise the grids,
// iterate, output.  All device memory is owned by the context; one iteration
// is captured once as a CUDA graph and replayed, with convergence decided on
// the device (see k_reduce) so the host only polls every few iterations.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rism3d_b200.h"
#include "r3d_fft_ct.cuh"
#include "r3d_internal.h"

namespace r3d {
struct Batch {
  const Desc *d;
  const int *prefix;
  int ns;
};
struct AtomTab {
  const double *x, *y, *z, *q;
  const double *sig2, *eps4;
  int nu;
};
size_t smem_x(int hx, int n, int S, size_t csz);
size_t smem_y(int ny, int P, size_t csz);
size_t smem_z(int nz, int n, int P, size_t csz);
void kernels_set_smem(bool fp64, size_t maxbytes);
int dot_blocks_per_sm(bool fp64);
int mix_chunk();
void launch_twiddle(double2 *o64, float2 *o32, int count, double scale, cudaStream_t s);
// compile-time-length passes (r3d_passes_ct.cu)
size_t ct_smem_x(int L, int PC, size_t csz);
size_t ct_smem_y(int L, int PC, size_t csz);
size_t ct_smem_z(int L, int PC, int n, size_t csz);
bool ct_length_ok(int L);
template <typename P>
bool ct_launch_fx(int, int, Batch, int, size_t, cudaStream_t, int, const void *);
template <typename P>
bool ct_launch_fy(int, int, Batch, int, size_t, cudaStream_t, int, int);
template <typename P>
bool ct_launch_zoz(int, int, Batch, int, size_t, cudaStream_t, int);
template <typename P>
bool ct_launch_ix(int, int, Batch, int, size_t, cudaStream_t, int, void *, int);
template <typename P>
bool ct_launch_ixb(int, int, Batch, int, size_t, cudaStream_t, int);
template <typename P>
bool ct_launch_fxb(int, int, Batch, int, size_t, cudaStream_t, int);
template <typename P>
bool ct_launch_mfx(int L, Batch b, int grid, size_t smem, cudaStream_t s, int per, int allow_mix);
template <typename P>
int ct_occupancy_mfx(int L, size_t smem);
size_t ct_smem_mfx(int L, int PC);
int ct_mfx_pc(int L);
size_t ct_smem_fxb(int L, int PC, size_t csz, size_t rsz, size_t tsz);
template <typename P>
int ct_occupancy_bulk(int which, int L, int PC, size_t smem);
template <typename P>
bool ct_launch_xw(int which, int L, int PCW, Batch b, int grid, size_t smem, cudaStream_t s);
template <typename P>
int ct_occupancy_xw(int which, int L, int PCW, size_t smem);
size_t ct_smem_warp(int L, int PCW, size_t csz);
template <typename P>
bool tma_launch_fy(int L, int dir, Batch b, int grid, size_t smem, cudaStream_t s, int per,
                   int nst);
template <typename P>
bool tma_launch_zoz(int L, Batch b, int grid, size_t smem, cudaStream_t s, int per, int nst);
template <typename P>
int tma_occupancy(int which, int L, size_t smem);
template <typename P>
void tma_allow_smem_all();
size_t ct_smem_ixb(int L, int PC, size_t csz, size_t rsz, size_t tsz);
// register-pass Stockham y/z passes (r3d_passes_sr.cu)
size_t sr_smem_y(int L, int PC, size_t csz);
size_t sr_smem_z(int L, int PC, int ns, size_t csz);
bool sr_length_supported(int L);
template <typename P>
bool sr_launch_fy(int L, int dir, Batch b, int grid, size_t smem, cudaStream_t s);
template <typename P>
bool sr_launch_zoz(int L, int ns, bool ozreg, Batch b, int grid, size_t smem, cudaStream_t s);
template <typename P>
int sr_pc_y_of();
template <typename P>
int sr_pc_z_of(int L, int ns);
template <typename P>
void sr_allow_geometry(int hx, int ny, int nz, int ns);
template <typename P>
bool sr_launch_zozp(int L, int ns, Batch b, int ntiles, int grid, size_t smem, cudaStream_t s);
template <typename P>
int sr_occupancy_zozp(int L, int ns, size_t smem);
template <typename P>
int sr_zp_supported(int L, int ns);
size_t sr_smem_zp(int L, int PC, int ns, size_t csz);
int sr_pc_x_of(int L);
size_t sr_smem_x(int L, int PC, size_t csz);
template <typename P>
bool sr_launch_fx(int L, Batch b, int grid, size_t smem, cudaStream_t s);
template <typename P>
bool sr_launch_ix(int L, Batch b, int grid, size_t smem, cudaStream_t s, int per);
template <typename P>
void launch_fwd_x(Batch, int, size_t, cudaStream_t, int, const void *);
template <typename P>
void launch_fft_y(Batch, int, size_t, cudaStream_t, int, int);
template <typename P>
void launch_zoz(Batch, int, size_t, cudaStream_t, int, int);
template <typename P>
void launch_inv_x(Batch, int, size_t, cudaStream_t, int, void *, int);
void launch_reduce(const Desc *, const int *, int, int, cudaStream_t);
void launch_ctl_gather(const Desc *, int, double *, cudaStream_t);
void launch_atom_integrals(const IntAtoms &, const double *, long long, const int *,
                           const double *, double *, int, double *, cudaStream_t);
template <typename P>
void launch_mix_an2(Batch, int, cudaStream_t);
void launch_t_restore(const void *t, const void *dslot, void *out, long long niv, cudaStream_t s);
template <typename P>
void launch_anm(Batch, int, const Desc *, const int *, int, cudaStream_t, int);
template <typename P>
void launch_potential(const Desc &, const AtomTab &, double, double,
                      const double *, int, double *, cudaStream_t);
void launch_phase_tables(double2 *, double2 *, double2 *, const double *,
                         const double *, const double *, int, int, int, int,
                         const double *, cudaStream_t);
void launch_fk(const Desc &, double2 *, const double2 *, const double2 *,
               const double2 *, const double *, int, double, const double *,
               double, cudaStream_t);
template <typename P>
void launch_cref(const Desc &, double *, cudaStream_t);
template <typename P>
void launch_lr_update(const double *, void *, long long, cudaStream_t);
void launch_kidx(const Desc &, const uint32_t *, int, cudaStream_t);
template <typename P>
void launch_thermo(const Desc &, const void *, double *, int, cudaStream_t);
template <typename P>
void launch_gh(const Desc &, const void *, double *, double *, cudaStream_t);
template <typename P>
void launch_to_double(const void *, double *, long long, int, cudaStream_t);
template <typename P>
void launch_from_double(const double *, void *, long long, int, cudaStream_t);
template <typename P>
void launch_shift_qfr(const Desc &, const void *, double *, double, int,
                      cudaStream_t);
template <typename P>
void launch_set_short(const Desc &, const double *, void *, cudaStream_t);

namespace phys {
constexpr double avogadro = 6.02214076e23;
constexpr double bohr = 0.5291771500001;
constexpr double boltzmann = 1.380649e-23;
constexpr double hartree = 4.359744722207185e-18;
}  // namespace phys

constexpr size_t kSmemBudget = 100 * 1024;  // per CTA: two CTAs per SM
constexpr size_t kSmemMax = 220 * 1024;
constexpr int kNumSM = 148;

// resident CTAs per SM of a bulk-staged pass (device query; smem-only
// estimate for host-only planning)
inline int bulk_per_sm(int device, bool fp64, int which, int L, int PC, size_t smem) {
  int nb = 0;
  if (device >= 0) {
    kernels_set_smem(fp64, kSmemMax);  // the occupancy query honours the opt-in limit
    if (which < 2)
      nb = fp64 ? ct_occupancy_bulk<P64>(which, L, PC, smem)
                : ct_occupancy_bulk<PMix>(which, L, PC, smem);
    else
      nb = fp64 ? ct_occupancy_xw<P64>(which - 2, L, PC, smem)
                : ct_occupancy_xw<PMix>(which - 2, L, PC, smem);
  }
  // 0 on a device: no kernel for (L, PC), or it does not fit -- the variant
  // is not offered; host-only planning estimates from shared memory
  if (device < 0) nb = std::max(1, (int)((228 * 1024) / (smem + 2048)));
  return nb;
}

}  // namespace r3d

using namespace r3d;

static thread_local std::string g_last_error;  // per calling thread
namespace r3d {
void set_last_error(const std::string &m) { g_last_error = m; }
}  // namespace r3d

// Launch geometry of the five grid passes for one (grid, sites, precision).
struct Geo {
  int tiles_x = 0, tiles_y = 0, tiles_z = 0, ix_ctas = 0, ix_per = 1, mix_ctas = 0,
      dot_ctas = 0;
  // the iteration's IX with bulk-staged inputs (ixb_pc = 0: not used): rows
  // per tile, CTAs, tiles per CTA, shared memory
  int ixb_pc = 0, ixb_ctas = 0, ixb_per = 1;
  size_t smixb = 0;
  int ixh_ctas = 0;  // CTAs of the same with half the rows per tile (autotuner's variant)
  // the iteration's FX with bulk-staged inputs (fxb_pc = 0: not used)
  int fxb_pc = 0, fxb_ctas = 0, fxb_per = 1;
  size_t smfxb = 0;
  // the iteration's FX / IX on warp tiles (pc = 0: not used): rows per warp
  // tile, CTAs per solve, shared memory
  int fxw_pc = 0, fxw_ctas = 0, ixw_pc = 0, ixw_ctas = 0;
  size_t smxw = 0;
  // the iteration's y and z passes on the tensor copy engine (yz_tma = 0:
  // the tile-per-CTA kernels): CTAs per solve, tiles per CTA, stages, smem
  // (yz_tma also carries the chosen y/z variant: 3 and 4 are the register-
  // pass Stockham y and z passes, with the OZ on registers / as a pass of
  // its own; yz_sr = 1 where those kernels cover the lengths and sites;
  // 5: variant 4 with the persistent z pass that streams its next tile in,
  // yz_srp = 1 where it exists: zp_ctas CTAs for any number of solves)
  int yz_tma = 0, fyt_pc = 0, fyt_ctas = 0, fyt_per = 1, fyt_nst = 0, zt_pc = 0, zt_ctas = 0,
      zt_per = 1, zt_nst = 0;
  size_t smfyt = 0, smzt = 0;
  int yz_sr = 0, fys_ctas = 0, zs_ctas = 0, yz_srp = 0, zp_ctas = 0;
  size_t smfys = 0, smzs = 0, smzp = 0;
  // the iteration's FX / IX on the Stockham engine (fxs_pc / ixs_pc = 0: not used;
  // x variant 4): rows per tile, CTAs (FX one tile each; IX ixs_per tiles)
  int fxs_pc = 0, ixs_pc = 0, fxs_ctas = 0, ixs_ctas = 0, ixs_per = 1;
  size_t smxs = 0;
  // the mixed path's AN2 mix fused into the iteration's FX (mfx_avail: the
  // kernel covers the geometry; mfx: in use -- the iteration then launches
  // no separate mix kernel)
  int mfx_avail = 0, mfx = 0, mfx_ctas = 0, mfx_per = 1;
  size_t smmfx = 0;
  size_t smx = 0, smy = 0, smz = 0;
};

struct r3d_ctx {
  r3d_opts opts{};
  Problem prob;
  std::string err;
  bool fp64 = true;
  size_t rsz = 8;
  int mixer = MIX_AN2, history = 2;
  double damping = -1;  // <0: use the .inp m
  std::string inp_dir;
  cudaStream_t stream = nullptr;
  bool initialized = false;
  // device memory
  std::vector<void *> allocs;
  size_t bytes = 0;
  void *u = nullptr, *t = nullptr, *fr = nullptr, *res = nullptr, *w = nullptr,
       *fk = nullptr, *chi = nullptr, *lr = nullptr, *gq = nullptr, *hist_a = nullptr,
       *hist_b = nullptr, *cref = nullptr, *chi64 = nullptr;
  double next_refresh = 0;  // mixed path: refresh when rms drops below this
  // the refresh schedule: the first at RMS refresh_first, then every time the
  // RMS has dropped by refresh_factor (R3D_REFRESH="first,factor" overrides).
  // Measured on the 256^3 NaCl deck: refreshing from 3e-2 on by factors of
  // 0.3 keeps the FP32 transforms' share of c small enough that the mixed
  // solve takes the FP64 solve's iterations (260-282 over the pass variants,
  // against 264-350 with refreshes at 1e-3 and 1e-5 only), for ~9 refreshes
  // of a few ms each.
  double refresh_first = 3e-2, refresh_factor = 0.3;
  // mixed path: the refresh's FP64 geometry and work buffer, kept from the
  // first refresh on (the FP64 path refreshes once, at setup, and frees it)
  bool rplanned = false;
  Desc rdesc{};
  Geo rgeo;
  char *rtmp = nullptr;
  void *tw64 = nullptr, *tw32 = nullptr;  // compile-time engine twiddles
  uint32_t *kidx = nullptr;
  double *partials = nullptr, *scratch = nullptr;
  void *tbuf = nullptr;  // mixed AN2: rebuilt t of the last evaluation (maxstep)
  int npart = 0;  // rows of partials
  size_t scratch_bytes = 0;
  Ctl *ctl = nullptr;
  Desc *ddesc = nullptr;
  int *dprefix = nullptr;  // [5][2]: prefix arrays of the passes + ix ctas
  Desc desc{};
  int nshell = 0;
  Geo geo;  // launch geometry of the iteration
  // graph of one iteration
  cudaGraphExec_t gexec = nullptr;
  double ms_per_iter = 0;
  int kernels_per_iter = 0;
  // CUDA-event times of the last initialize: potential pair sums, k-space
  // Coulomb sum, long-range h term (refresh), whole initialize (host clock)
  double setup_ms[4] = {0, 0, 0, 0};
  // refreshes of the FP64 reference during iterations since the last
  // initialize, and their host-clock time (launch to completion)
  int refreshes = 0;
  double refresh_ms = 0;
  unsigned long long h2d = 0, d2h = 0;  // bytes copied each way
  // pinned staging chunks of the grid copies to caller memory (first use)
  void *pin[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
};

// ------------------------------------------------------------------ utils
static int fail(r3d_ctx *c, int code, const std::string &m) {
  if (c) c->err = m;
  g_last_error = m;
  return code;
}
#define CK(call)                                                          \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess)                                                \
      return fail(c, R3D_ECUDA, std::string(#call) + ": " +               \
                                    cudaGetErrorString(e_));              \
  } while (0)

// Host<->device copies on the context's stream, counted for r3d_transfer_bytes.
static cudaError_t copy_h2d(r3d_ctx *c, void *dst, const void *src, size_t n,
                            cudaStream_t s) {
  c->h2d += n;
  return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s);
}
static cudaError_t copy_d2h(r3d_ctx *c, void *dst, const void *src, size_t n,
                            cudaStream_t s) {
  c->d2h += n;
  return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, s);
}

// A solve's device memory comes from one stream-ordered pool per device,
// allocated and freed on the solve's stream, and the pool keeps what is
// freed for the next solve.  cudaMalloc / cudaFree of a solve's gigabytes
// would synchronise the whole device -- a server's admissions would wait
// for the iterations in flight -- and returning and re-mapping the pages of
// every solve costs from milliseconds to a second per solve.  Memory the
// pool holds unused is counted as free by the admission checks and given
// back (trimmed) when an allocation does not fit.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pool[64];

static cudaMemPool_t solve_pool(int dev) {
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = dev;
    cudaMemPool_t mp = nullptr;
    if (cudaMemPoolCreate(&mp, &pp) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    unsigned long long keep = ~0ull;  // never give memory back at a sync
    cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pool[dev] = mp;
  }
  return g_pool[dev];
}

// Bytes the device's pool holds but no solve uses.
static size_t pool_spare(int dev) {
  cudaMemPool_t mp = solve_pool(dev);
  if (!mp) return 0;
  unsigned long long res = 0, used = 0;
  cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReservedMemCurrent, &res);
  cudaMemPoolGetAttribute(mp, cudaMemPoolAttrUsedMemCurrent, &used);
  return res > used ? (size_t)(res - used) : 0;
}

// bytes on stream s from device dev's pool; on a failure the pool's unused
// memory is released and the allocation tried once more
static cudaError_t pool_alloc(int dev, void **p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t mp = solve_pool(dev);
  if (!mp) return cudaErrorMemoryAllocation;
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, mp, s);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    cudaStreamSynchronize(s);
    cudaMemPoolTrimTo(mp, 0);
    e = cudaMallocFromPoolAsync(p, bytes, mp, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
  }
  return e;
}

static int dalloc(r3d_ctx *c, void **p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  cudaError_t e = pool_alloc(c->opts.device, p, bytes, c->stream);
  if (e != cudaSuccess)
    return fail(c, R3D_ENOMEM, "device allocation of " + std::to_string(bytes) +
                                   " bytes failed: " + cudaGetErrorString(e));
  c->allocs.push_back(*p);
  c->bytes += bytes;
  return R3D_OK;
}

// Frees on the solve's stream; every other stream that used the memory (a
// batch's, a server's) has finished with it when a solve is freed.
static void free_all(r3d_ctx *c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  c->gexec = nullptr;
  for (void *p : c->allocs) cudaFreeAsync(p, c->stream);
  c->allocs.clear();
  c->bytes = 0;
  c->rtmp = nullptr;
  c->initialized = false;
}

// ------------------------------------------------------------- lifetime
extern "C" int r3d_create(const r3d_opts *opts, r3d_ctx **out) {
  if (!out) return fail(nullptr, R3D_EINVAL, "out is NULL");
  *out = nullptr;
  r3d_ctx *c = new r3d_ctx();
  if (opts) c->opts = *opts;
  if (c->opts.precision != R3D_FP64 && c->opts.precision != R3D_MIXED) {
    delete c;
    return fail(nullptr, R3D_EINVAL, "precision must be R3D_FP64 or R3D_MIXED");
  }
  c->fp64 = c->opts.precision == R3D_FP64;
  c->rsz = c->fp64 ? 8 : 4;
  if (const char *er = getenv("R3D_REFRESH")) {
    double a = 0, f = 0;
    if (std::sscanf(er, "%lf,%lf", &a, &f) == 2 && a > 0 && f > 0 && f < 1) {
      c->refresh_first = a;
      c->refresh_factor = f;
    }
  }
  if (c->opts.device < 0) {  // host-only context: loaders, planning, no GPU
    *out = c;
    return R3D_OK;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    delete c;
    return fail(nullptr, R3D_ECUDA, std::string("no CUDA device: ") +
                                        cudaGetErrorString(e));
  }
  if (c->opts.device < 0 || c->opts.device >= ndev) {
    delete c;
    return fail(nullptr, R3D_EINVAL, "device ordinal out of range");
  }
  e = cudaSetDevice(c->opts.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(nullptr, R3D_ECUDA, std::string("stream: ") + cudaGetErrorString(e));
  }
  *out = c;
  return R3D_OK;
}

extern "C" int r3d_destroy(r3d_ctx *c) {
  if (!c) return R3D_OK;
  if (c->opts.device < 0) {
    delete c;
    return R3D_OK;
  }
  cudaSetDevice(c->opts.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_all(c);
  for (int k = 0; k < 2; ++k) {
    if (c->pin[k]) cudaFreeHost(c->pin[k]);
    if (c->pin_ev[k]) cudaEventDestroy(c->pin_ev[k]);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return R3D_OK;
}

extern "C" const char *r3d_last_error(const r3d_ctx *c) {
  return c ? c->err.c_str() : g_last_error.c_str();
}

// ---------------------------------------------------------------- input
extern "C" int r3d_set_ad(r3d_ctx *c, double lambda, int adswitch) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (c->initialized) return fail(c, R3D_ESTATE, "set_ad after initialize");
  c->prob.lambda = lambda;
  c->prob.adswitch = adswitch;
  return R3D_OK;
}

extern "C" int r3d_load_inp(r3d_ctx *c, const char *inp, const char *structure,
                            int centering, int q0) {
  if (!c || !inp) return fail(c, R3D_EINVAL, "ctx or inp is NULL");
  if (c->initialized) return fail(c, R3D_ESTATE, "load_inp after initialize");
  Problem p;
  p.adswitch = c->prob.adswitch;
  p.lambda = c->prob.lambda;
  std::string m = parse_inp(p, inp, structure ? structure : "", centering != 0, q0 != 0);
  if (!m.empty())
    return fail(c, m.rfind("cannot open", 0) == 0 ? R3D_EIO : R3D_EINVAL, m);
  // keep a solvent that was loaded before
  if (c->prob.has_solvent) {
    p.natv = c->prob.natv;
    p.ntab = c->prob.ntab;
    p.temper = c->prob.temper;
    p.xt = c->prob.xt;
    p.sigv = c->prob.sigv;
    p.epsv = c->prob.epsv;
    p.qv = c->prob.qv;
    p.rhov = c->prob.rhov;
    p.ttab = c->prob.ttab;
    p.xvv = c->prob.xvv;
    p.has_solvent = true;
  }
  c->prob = std::move(p);
  std::string ip(inp);
  size_t sl = ip.rfind('/');
  c->inp_dir = sl == std::string::npos ? std::string() : ip.substr(0, sl + 1);
  return R3D_OK;
}

extern "C" int r3d_load_xvk(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (c->initialized) return fail(c, R3D_ESTATE, "load_xvk after initialize");
  std::string p;
  if (path) {
    p = path;
  } else {
    if (c->prob.fsolvent.empty())
      return fail(c, R3D_ESTATE, "no solvent file named: load an .inp first");
    p = c->prob.fsolvent;
    FILE *f = std::fopen(p.c_str(), "r");
    if (f)
      std::fclose(f);
    else if (p[0] != '/')
      p = c->inp_dir + p;
  }
  std::string m = parse_xvk(c->prob, p);
  if (!m.empty())
    return fail(c, m.find("could not be opened") != std::string::npos ? R3D_EIO : R3D_EINVAL, m);
  return R3D_OK;
}

extern "C" int r3d_set_problem(r3d_ctx *c, const r3d_problem *q) {
  if (!c || !q) return fail(c, R3D_EINVAL, "ctx or problem is NULL");
  if (c->initialized) return fail(c, R3D_ESTATE, "set_problem after initialize");
  if (q->nu < 0 || q->natv <= 0 || q->natv > kMaxSites || q->ntab < 4 || !(q->dr > 0))
    return fail(c, R3D_EINVAL, "bad problem sizes");
  Problem p;
  p.adswitch = c->prob.adswitch;
  p.lambda = c->prob.lambda;
  for (int d = 0; d < 3; ++d) {
    p.grid[d] = q->grid[d];
    p.box[d] = q->box[d];
    if (p.grid[d] < 4 || (p.grid[d] & 1) || p.grid[d] > 2048 || !(p.box[d] > 0))
      return fail(c, R3D_EINVAL, "grid must be even, 4..2048, and the box positive");
  }
  p.clos = q->closure;
  p.pse_n = q->closure == R3D_KH ? 1 : std::max(1, q->pse_n);
  p.convergence = q->convergence;
  p.maxstep = q->maxstep;
  p.count = q->count;
  p.mix_m = q->m;
  p.mix_mp = q->mp;
  p.sig.assign(q->sig, q->sig + q->nu);
  p.eps.assign(q->eps, q->eps + q->nu);
  p.q.assign(q->q, q->q + q->nu);
  p.r.assign(q->xyz, q->xyz + 3 * q->nu);
  p.natv = q->natv;
  p.sigv.assign(q->sigv, q->sigv + q->natv);
  p.epsv.assign(q->epsv, q->epsv + q->natv);
  p.qv.assign(q->qv, q->qv + q->natv);
  p.rhov.assign(q->rhov, q->rhov + q->natv);
  p.temper = q->temper;
  p.xt = q->xt;
  p.ntab = q->ntab;
  p.xvv.assign(q->xvv, q->xvv + (size_t)q->natv * q->natv * q->ntab);
  double dk = M_PI / (q->dr * q->ntab);
  p.ttab.resize(q->ntab);
  for (int i = 0; i < q->ntab; ++i) p.ttab[i] = dk * (i + 1);
  p.fname = "r3d";
  p.has_solute = p.has_solvent = true;
  c->prob = std::move(p);
  return R3D_OK;
}

extern "C" int r3d_set_closure(r3d_ctx *c, int clos, int pse_n) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (clos < R3D_KH || clos > R3D_PSE || (clos == R3D_PSE && pse_n < 1))
    return fail(c, R3D_EINVAL, "unknown closure");
  c->prob.clos = clos;
  c->prob.pse_n = clos == R3D_KH ? 1 : pse_n;
  if (c->initialized) {
    c->desc.clos = c->prob.clos;
    c->desc.pse_n = c->prob.pse_n;
    CK(copy_h2d(c, c->ddesc, &c->desc, sizeof(Desc), c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  return R3D_OK;
}

extern "C" int r3d_set_mixer(r3d_ctx *c, int mixer, int history, double damping) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (c->initialized) return fail(c, R3D_ESTATE, "set_mixer after initialize");
  if (mixer != R3D_MIX_AN2 && mixer != R3D_MIX_ANM)
    return fail(c, R3D_EINVAL, "unknown mixer");
  if (mixer == R3D_MIX_ANM && (history < 1 || history > kMaxHistory))
    return fail(c, R3D_EINVAL, "history must be 1.." + std::to_string(kMaxHistory));
  c->mixer = mixer;
  c->history = mixer == R3D_MIX_AN2 ? 2 : history;
  c->damping = damping;
  return R3D_OK;
}

extern "C" int r3d_set_control(r3d_ctx *c, double convergence, int maxstep) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (convergence > 0) c->prob.convergence = convergence;
  if (maxstep > 0) c->prob.maxstep = maxstep;
  return R3D_OK;
}

// ------------------------------------------------------------ geometry
static int plan_geo(r3d_ctx *c, Desc &d, Geo &g, bool fp64, int nsites);
static bool ixb_config(int device, const Desc &d, bool fp64, int pcb, Geo &g);
static int plan_geometry(r3d_ctx *c, Desc &d) {
  return plan_geo(c, d, c->geo, c->fp64, c->prob.natv);
}

static int plan_geo(r3d_ctx *c, Desc &d, Geo &g, bool fp64, int nsites) {
  const Problem &p = c->prob;
  d.nx = p.grid[0];
  d.ny = p.grid[1];
  d.nz = p.grid[2];
  d.n = nsites;
  d.hx = d.nx / 2;
  d.N = (long long)d.nx * d.ny * d.nz;
  d.Nh = (long long)d.hx * d.ny * d.nz;
  d.Ns = d.N + 1536;   // 6 KB (FP32) / 12 KB (FP64) off a power of two
  d.Nhs = d.Nh + 768;
  d.nrad_x = factor_length(d.hx, d.rad_x);
  d.nrad_y = factor_length(d.ny, d.rad_y);
  d.nrad_z = factor_length(d.nz, d.rad_z);
  if (d.nrad_x < 0 || d.nrad_y < 0 || d.nrad_z < 0)
    return fail(c, R3D_EINVAL, "grid sizes must factor into primes <= 13");
  const size_t cs = fp64 ? 16 : 8;
  const int rowsN = d.ny * d.nz;
  // compile-time engine where the length and tile divide (else runtime engine)
  const int pcx = fp64 ? 16 : 32;
  d.ct_x = (ct_length_ok(d.hx) && rowsN % pcx == 0) ? pcx : 0;
  int pcy = fp64 ? 8 : 16;
  if (d.hx % pcy) pcy = 8;
  d.ct_y = (ct_length_ok(d.ny) && d.hx % pcy == 0) ? pcy : 0;
  int pcz = fp64 ? 4 : 8;
  if (d.hx % pcz) pcz = 4;
  d.ct_z = (ct_length_ok(d.nz) && d.hx % pcz == 0 &&
            ct_smem_z(d.nz, pcz, d.n, cs) <= kSmemMax) ? pcz : 0;
  int S = 16;
  while (S > 1 && (rowsN % S || smem_x(d.hx, d.n, S, cs) > kSmemBudget)) S >>= 1;
  while (S > 1 && rowsN / S < 2 * kNumSM) S >>= 1;
  int Py = fp64 ? 8 : 16;
  while (Py > 1 && (d.hx % Py || smem_y(d.ny, Py, cs) > kSmemBudget)) Py >>= 1;
  int Pz = fp64 ? 4 : 8;
  while (Pz > 1 && (d.hx % Pz || smem_z(d.nz, d.n, Pz, cs) > kSmemBudget)) Pz >>= 1;
  d.rows = S;
  d.ycols = Py;
  d.zcols = Pz;
  g.smx = smem_x(d.hx, d.n, S, cs);
  g.smy = smem_y(d.ny, Py, cs);
  g.smz = smem_z(d.nz, d.n, Pz, cs);
  d.tiles_x = rowsN / S;
  d.tiles_y = d.n * d.nz * (d.hx / Py);
  d.tiles_z = d.ny * (d.hx / Pz);
  if (d.ct_x) {
    d.tiles_x = d.n * (rowsN / d.ct_x);
    g.smx = ct_smem_x(d.hx, d.ct_x, cs);
  }
  if (d.ct_y) {
    d.tiles_y = d.n * d.nz * (d.hx / d.ct_y);
    g.smy = ct_smem_y(d.ny, d.ct_y, cs);
  }
  if (d.ct_z) {  // the runtime engine serves the other z modes on the same tiles
    d.zcols = d.ct_z;
    d.tiles_z = d.ny * (d.hx / d.ct_z);
    g.smz = std::max(ct_smem_z(d.nz, d.ct_z, d.n, cs), smem_z(d.nz, d.n, d.ct_z, cs));
  }
  if (g.smx > kSmemMax || g.smy > kSmemMax || g.smz > kSmemMax)
    return fail(c, R3D_EINVAL, "grid too large for one CTA's shared memory");
  g.tiles_x = d.tiles_x;
  g.tiles_y = d.tiles_y;
  g.tiles_z = d.tiles_z;
  g.ix_ctas = std::min(d.tiles_x, 4 * kNumSM);
  g.ix_per = (d.tiles_x + g.ix_ctas - 1) / g.ix_ctas;
  g.ix_ctas = (d.tiles_x + g.ix_per - 1) / g.ix_per;
  g.ixb_pc = 0;
  if (d.ct_x) {  // bulk-staged IX: as many CTAs as stay resident
    const int pcb = fp64 ? 4 : 8;
    if (!ixb_config(c->opts.device, d, fp64, pcb, g) && d.hx >= 256)
      ixb_config(c->opts.device, d, fp64, pcb / 2, g);  // long rows: half the rows per tile
    Geo h = g;  // the half-size tiles the autotuner may choose write as many partials rows
    g.ixh_ctas = (g.ixb_pc >= 2 && ixb_config(c->opts.device, d, fp64, g.ixb_pc / 2, h))
                     ? h.ixb_ctas : 0;
  }
  g.fxb_pc = 0;
  if (d.ct_x) {  // bulk-staged FX, sized like the IX above
    int pcb = fp64 ? 4 : 8;
    size_t sm = ct_smem_fxb(d.hx, pcb, cs, fp64 ? 8 : 4, 8);
    if (sm > 110 * 1024 && d.hx >= 256) {  // long rows: half the rows, two CTAs per SM
      pcb /= 2;
      sm = ct_smem_fxb(d.hx, pcb, cs, fp64 ? 8 : 4, 8);
    }
    if (rowsN % pcb == 0 && d.ny >= pcb && sm <= kSmemMax) {  // a tile's rows wrap z once at most
      const int tiles = d.n * (rowsN / pcb);
      const int per_sm = bulk_per_sm(c->opts.device, fp64, 0, d.hx, pcb, sm);
      if (per_sm > 0) {
        g.fxb_pc = pcb;
        g.smfxb = sm;
        g.fxb_ctas = std::min(tiles, kNumSM * per_sm);
        g.fxb_per = (tiles + g.fxb_ctas - 1) / g.fxb_ctas;
        g.fxb_ctas = (tiles + g.fxb_per - 1) / g.fxb_per;
      }
    }
  }
  g.fxw_pc = g.ixw_pc = 0;
  if (d.ct_x) {  // warp tiles: 4 rows per warp (2 for long rows)
    const int pcw = d.hx >= 256 ? 2 : 4;
    const size_t sm = ct_smem_warp(d.hx, pcw, cs);
    if (rowsN % pcw == 0 && sm + 6 * 1024 <= kSmemMax) {
      const int ctas = (d.n * (rowsN / pcw) + 7) / 8;
      g.smxw = sm;
      g.fxw_pc = g.ixw_pc = pcw;
      g.fxw_ctas = std::min(ctas, kNumSM * bulk_per_sm(c->opts.device, fp64, 2, d.hx, pcw, sm));
      g.ixw_ctas = std::min(ctas, kNumSM * bulk_per_sm(c->opts.device, fp64, 3, d.hx, pcw, sm));
      if (!g.fxw_ctas) g.fxw_pc = 0;
      if (!g.ixw_ctas) g.ixw_pc = 0;
    }
  }
  g.yz_tma = 0;
  {  // y and z passes on the tensor copy engine: lengths of the engine, 2-4 stages
    auto tma_len = [](int L) { return ct_length_ok(L) && L <= 512; };
    const int py = fp64 ? 4 : 8, pz = fp64 ? 2 : 4;
    const size_t sby = (size_t)py * d.ny * cs, sbz = (size_t)pz * d.nz * d.n * cs;
    auto stages = [&](size_t sb, size_t cap) {
      for (int k = 4; k >= 2; --k)
        if (k * sb <= cap) return k;
      return 0;
    };
    const int ny_st = stages(sby, 64 * 1024) ? stages(sby, 64 * 1024) : stages(sby, kSmemMax);
    const int nz_st = stages(sbz, 110 * 1024) ? stages(sbz, 110 * 1024) : stages(sbz, kSmemMax);
    if (tma_len(d.ny) && tma_len(d.nz) && d.hx % py == 0 && d.hx % pz == 0 && ny_st && nz_st &&
        c->opts.device >= 0) {
      g.yz_tma = 2;  // the autotuner may step down to 1 (copy-engine y only) or 0
      g.fyt_pc = py;
      g.zt_pc = pz;
      g.fyt_nst = ny_st;
      g.zt_nst = nz_st;
      g.smfyt = ny_st * sby;
      g.smzt = nz_st * sbz;
      const int ty = d.n * d.nz * (d.hx / py), tz = d.ny * (d.hx / pz);
      kernels_set_smem(fp64, kSmemMax);
      int oy = fp64 ? tma_occupancy<P64>(0, d.ny, g.smfyt) : tma_occupancy<PMix>(0, d.ny, g.smfyt);
      int oz = fp64 ? tma_occupancy<P64>(1, d.nz, g.smzt) : tma_occupancy<PMix>(1, d.nz, g.smzt);
      if (oy <= 0 || oz <= 0) g.yz_tma = 0;  // no kernels for these lengths
      oy = std::max(oy, 1);
      oz = std::max(oz, 1);
      g.fyt_ctas = std::min(ty, kNumSM * oy);
      g.fyt_per = (ty + g.fyt_ctas - 1) / g.fyt_ctas;
      g.fyt_ctas = (ty + g.fyt_per - 1) / g.fyt_per;
      g.zt_ctas = std::min(tz, kNumSM * oz);
      g.zt_per = (tz + g.zt_ctas - 1) / g.zt_ctas;
      g.zt_ctas = (tz + g.zt_per - 1) / g.zt_per;
    }
  }
  g.mfx_avail = g.mfx = 0;
  if (!fp64 && c->mixer == MIX_AN2 && d.ct_x && c->opts.device >= 0) {  // mix-fused FX
    const int pc = ct_mfx_pc(d.hx);
    const size_t sm = ct_smem_mfx(d.hx, pc);
    if (rowsN % pc == 0 && d.ny >= pc && sm <= kSmemMax) {  // rows wrap z once at most
      kernels_set_smem(false, kSmemMax);
      const int per_sm = ct_occupancy_mfx<PMix>(d.hx, sm);
      if (per_sm > 0) {
        const int tiles = d.n * (rowsN / pc);
        g.mfx_avail = 1;
        g.smmfx = sm;
        g.mfx_ctas = std::min(tiles, kNumSM * per_sm);
        g.mfx_per = (tiles + g.mfx_ctas - 1) / g.mfx_ctas;
        g.mfx_ctas = (tiles + g.mfx_per - 1) / g.mfx_per;
      }
    }
  }
  g.fxs_pc = g.ixs_pc = 0;
  if (c->opts.device >= 0 && sr_length_supported(d.hx)) {  // Stockham x passes
    const int pc = sr_pc_x_of(d.hx);
    const size_t sm = sr_smem_x(d.hx, pc, cs);
    if (pc > 0 && rowsN % pc == 0 && sm <= kSmemMax) {
      g.fxs_pc = g.ixs_pc = pc;
      g.smxs = sm;
      g.fxs_ctas = d.n * (rowsN / pc);
      g.ixs_ctas = std::min(g.fxs_ctas, 4 * kNumSM);
      g.ixs_per = (g.fxs_ctas + g.ixs_ctas - 1) / g.ixs_ctas;
      g.ixs_ctas = (g.fxs_ctas + g.ixs_per - 1) / g.ixs_per;
    }
  }
  g.yz_sr = 0;
  if (c->opts.device >= 0 && sr_length_supported(d.ny) && sr_length_supported(d.nz) &&
      d.n >= 1 && d.n <= 4) {  // register-pass Stockham y and z passes
    const int pcy = fp64 ? sr_pc_y_of<P64>() : sr_pc_y_of<PMix>();
    const int pcz = fp64 ? sr_pc_z_of<P64>(d.nz, d.n) : sr_pc_z_of<PMix>(d.nz, d.n);
    const size_t smy = sr_smem_y(d.ny, pcy, cs), smz = sr_smem_z(d.nz, pcz, d.n, cs);
    if (pcz > 0 && d.hx % pcy == 0 && d.hx % pcz == 0 && smy <= kSmemMax && smz <= kSmemMax) {
      g.yz_sr = 1;
      g.fys_ctas = d.n * d.nz * (d.hx / pcy);
      g.zs_ctas = d.ny * (d.hx / pcz);
      g.smfys = smy;
      g.smzs = smz;
    }
  }
  // large shared memory for the Stockham kernels of this geometry's lengths
  // (set here, before any capture; loads only the kernels the solve may use)
  if (g.fxs_pc || g.yz_sr) {
    if (fp64)
      sr_allow_geometry<P64>(g.fxs_pc ? d.hx : 0, g.yz_sr ? d.ny : 0, g.yz_sr ? d.nz : 0, d.n);
    else
      sr_allow_geometry<PMix>(g.fxs_pc ? d.hx : 0, g.yz_sr ? d.ny : 0, g.yz_sr ? d.nz : 0, d.n);
  }
  // the persistent z pass: whole 16-byte copies of tile rows (the rows of
  // the spectrum and the site stride 16-byte aligned), one CTA per SM or more
  g.yz_srp = g.zp_ctas = 0;
  g.smzp = 0;
  if (g.yz_sr && (fp64 ? sr_zp_supported<P64>(d.nz, d.n) : sr_zp_supported<PMix>(d.nz, d.n)) &&
      ((size_t)d.hx * cs) % 16 == 0 && ((size_t)d.Nhs * cs) % 16 == 0) {
    const int pcz = fp64 ? sr_pc_z_of<P64>(d.nz, d.n) : sr_pc_z_of<PMix>(d.nz, d.n);
    const size_t sm = sr_smem_zp(d.nz, pcz, d.n, cs);
    const int occ = sm > kSmemMax ? 0
                    : fp64 ? sr_occupancy_zozp<P64>(d.nz, d.n, sm)
                           : sr_occupancy_zozp<PMix>(d.nz, d.n, sm);
    if (occ > 0) {
      int nsm = kNumSM;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->opts.device);
      g.yz_srp = 1;
      g.smzp = sm;
      g.zp_ctas = occ * nsm;
    }
  }
  // mixers: one chunk of mix_chunk() elements per CTA; ANM dots: one full
  // wave of a grid-stride reduction
  const long long niv = (long long)d.n * d.Ns;
  g.mix_ctas = (int)((niv + mix_chunk() - 1) / mix_chunk());
  int nsm = kNumSM;
  if (c->opts.device >= 0) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->opts.device);
  const int bps = c->opts.device >= 0 ? dot_blocks_per_sm(fp64) : 4;
  g.dot_ctas = (int)std::min<long long>((d.N + kThreads - 1) / kThreads, (long long)nsm * bps);
  return R3D_OK;
}

// Geometry of the bulk-staged IX with pcb rows per tile (false: does not fit).
static bool ixb_config(int device, const Desc &d, bool fp64, int pcb, Geo &g) {
  // rows per tile with compiled kernels: 8 or 4 (FP32 grids; 2 as well for
  // rows of 256 or more), 4 or 2 (FP64)
  if (pcb != (fp64 ? 4 : 8) && pcb != (fp64 ? 2 : 4) && !(!fp64 && pcb == 2 && d.hx >= 256))
    return false;
  const size_t cs = fp64 ? 16 : 8;
  const int rowsN = d.ny * d.nz;
  const size_t sm = ct_smem_ixb(d.hx, pcb, cs, fp64 ? 8 : 4, 8);
  if (rowsN % pcb || sm > kSmemMax) return false;
  const int tiles = d.n * (rowsN / pcb);
  const int per_sm = bulk_per_sm(device, fp64, 1, d.hx, pcb, sm);
  if (per_sm <= 0) return false;
  g.ixb_pc = pcb;
  g.smixb = sm;
  g.ixb_ctas = std::min(tiles, kNumSM * per_sm);
  g.ixb_per = (tiles + g.ixb_ctas - 1) / g.ixb_ctas;
  g.ixb_ctas = (tiles + g.ixb_per - 1) / g.ixb_per;
  return true;
}

// ---------------------------------------------------------- pass dispatch
// Each pass runs on the compile-time engine when plan_geo chose it for this
// descriptor (d.ct_* != 0), else on the runtime-length engine.
// mode 1 with the mix-fused FX in use: allow_mix = 1 applies the mix the
// last reduce requested (the iteration's graph), 0 is a plain FX (calculate)
template <typename P>
static void pass_fx(const Desc &d, const Geo &g, Batch b, cudaStream_t s, int mode,
                    const void *src, int allow_mix = 0) {
  if (mode == 1 && g.mfx && ct_launch_mfx<P>(d.hx, b, g.mfx_ctas, g.smmfx, s, g.mfx_per, allow_mix))
    return;
  if (mode == 1 && g.fxs_pc && sr_launch_fx<P>(d.hx, b, g.fxs_ctas, g.smxs, s)) return;
  if (mode == 1 && g.fxw_pc && ct_launch_xw<P>(0, d.hx, g.fxw_pc, b, g.fxw_ctas, g.smxw, s))
    return;
  if (mode == 1 && g.fxb_pc &&
      ct_launch_fxb<P>(d.hx, g.fxb_pc, b, g.fxb_ctas, g.smfxb, s, g.fxb_per))
    return;
  if (!(d.ct_x && ct_launch_fx<P>(d.hx, d.ct_x, b, g.tiles_x, g.smx, s, mode, src)))
    launch_fwd_x<P>(b, g.tiles_x, g.smx, s, mode, src);
}
template <typename P>
static void pass_fy(const Desc &d, const Geo &g, Batch b, cudaStream_t s, int dir, int check) {
  if (!(d.ct_y && ct_launch_fy<P>(d.ny, d.ct_y, b, g.tiles_y, g.smy, s, dir, check)))
    launch_fft_y<P>(b, g.tiles_y, g.smy, s, dir, check);
}
template <typename P>
static void pass_zoz(const Desc &d, const Geo &g, Batch b, cudaStream_t s, int mode, int check) {
  // the compile-time engine implements the fused mode (2) only
  if (!(mode == 2 && d.ct_z && ct_launch_zoz<P>(d.nz, d.ct_z, b, g.tiles_z, g.smz, s, check)))
    launch_zoz<P>(b, g.tiles_z, g.smz, s, mode, check);
}
template <typename P>
static void pass_ix(const Desc &d, const Geo &g, Batch b, cudaStream_t s, int mode, void *dst) {
  if (mode == 1 && g.ixs_pc && sr_launch_ix<P>(d.hx, b, g.ixs_ctas, g.smxs, s, g.ixs_per)) return;
  if (mode == 1 && g.ixw_pc && ct_launch_xw<P>(1, d.hx, g.ixw_pc, b, g.ixw_ctas, g.smxw, s))
    return;
  if (mode == 1 && g.ixb_pc &&
      ct_launch_ixb<P>(d.hx, g.ixb_pc, b, g.ixb_ctas, g.smixb, s, g.ixb_per))
    return;
  if (!(d.ct_x && ct_launch_ix<P>(d.hx, d.ct_x, b, g.ix_ctas, g.smx, s, mode, dst, g.ix_per)))
    launch_inv_x<P>(b, g.ix_ctas, g.smx, s, mode, dst, g.ix_per);
}
// The iteration's y / z passes: on the tensor copy engine when the geometry
// has it (the three together: they share the digit-reversed ky layout of w),
// else the tile-per-CTA kernels.
template <typename P>
static void pass_fy_iter(const Desc &d, const Geo &g, Batch b, cudaStream_t s, int dir) {
  if (g.yz_tma >= 3 && sr_launch_fy<P>(d.ny, dir, b, g.fys_ctas, g.smfys, s)) return;
  if ((g.yz_tma == 1 || g.yz_tma == 2) &&
      tma_launch_fy<P>(d.ny, dir, b, g.fyt_ctas, g.smfyt, s, g.fyt_per, g.fyt_nst))
    return;
  pass_fy<P>(d, g, b, s, dir, 1);
}
template <typename P>
static void pass_zoz_iter(const Desc &d, const Geo &g, Batch b, cudaStream_t s) {
  if (g.yz_tma == 5 && g.yz_srp &&
      sr_launch_zozp<P>(d.nz, d.n, b, g.zs_ctas, g.zp_ctas, g.smzp, s))
    return;
  if (g.yz_tma >= 3 && sr_launch_zoz<P>(d.nz, d.n, g.yz_tma == 3, b, g.zs_ctas, g.smzs, s))
    return;
  if (g.yz_tma == 2 && tma_launch_zoz<P>(d.nz, b, g.zt_ctas, g.smzt, s, g.zt_per, g.zt_nst))
    return;
  if (g.yz_tma == 1 && ct_launch_zoz<P>(d.nz, d.ct_z, b, g.tiles_z, g.smz, s, 1 | 2)) return;
  pass_zoz<P>(d, g, b, s, 2, 1);
}

// CTAs of the iteration's IX (each writes one row of the partials k_reduce sums)
static int iter_ix_ctas(const Geo &g) {
  return g.ixs_pc ? g.ixs_ctas : g.ixw_pc ? g.ixw_ctas : g.ixb_pc ? g.ixb_ctas : g.ix_ctas;
}
// rows of partials the iteration's IX may need, whichever variant runs
static int max_ix_ctas(const Geo &g) {
  return std::max(std::max(std::max(std::max(g.ix_ctas, g.ixb_pc ? g.ixb_ctas : 0),
                                    g.ixw_pc ? g.ixw_ctas : 0),
                           g.ixh_ctas),
                  g.ixs_pc ? g.ixs_ctas : 0);
}
// CTAs of the iteration's FX
static int iter_fx_ctas(const Geo &g) {
  return g.mfx ? g.mfx_ctas : g.fxs_pc ? g.fxs_ctas : g.fxw_pc ? g.fxw_ctas
                                      : g.fxb_pc ? g.fxb_ctas : g.tiles_x;
}

// Launch prefixes of ns solves that share one geometry (a device int block):
// the CTA prefixes of the x, y, z, IX, mix and ANM-dot passes (ns + 1 entries
// each: solve i owns CTAs [p[i], p[i+1]) of the launch), then every solve's
// IX CTA count (rows of partials k_reduce sums) and ANM dot CTA count.
enum { PF_X, PF_Y, PF_Z, PF_IX, PF_MIX, PF_DOT, PF_IXC, PF_DOTC };
static int pf_off(int ns, int k) {
  return k <= PF_IXC ? k * (ns + 1) : PF_IXC * (ns + 1) + ns;
}
static int pf_len(int ns) { return PF_IXC * (ns + 1) + 2 * ns; }
static std::vector<int> make_prefix(const Geo &g, int ns) {
  std::vector<int> v(pf_len(ns));
  const int per[6] = {iter_fx_ctas(g),
                      g.yz_tma >= 3 ? g.fys_ctas : g.yz_tma ? g.fyt_ctas : g.tiles_y,
                      g.yz_tma >= 3 ? g.zs_ctas : g.yz_tma == 2 ? g.zt_ctas : g.tiles_z,
                      iter_ix_ctas(g), g.mix_ctas, g.dot_ctas};
  for (int k = 0; k < 6; ++k)
    for (int i = 0; i <= ns; ++i) v[pf_off(ns, k) + i] = i * per[k];
  for (int i = 0; i < ns; ++i) {
    v[pf_off(ns, PF_IXC) + i] = iter_ix_ctas(g);
    v[pf_off(ns, PF_DOTC) + i] = g.dot_ctas;
  }
  return v;
}
// Grid sizes of one launch over ns solves of geometry g.
static Geo scaled(const Geo &g, int ns) {
  Geo s = g;
  s.tiles_x *= ns;
  s.tiles_y *= ns;
  s.tiles_z *= ns;
  s.ix_ctas *= ns;
  s.ixb_ctas *= ns;
  s.fxb_ctas *= ns;
  s.fxw_ctas *= ns;
  s.ixw_ctas *= ns;
  s.fyt_ctas *= ns;
  s.zt_ctas *= ns;
  s.fys_ctas *= ns;
  s.zs_ctas *= ns;
  s.fxs_ctas *= ns;
  s.ixs_ctas *= ns;
  s.mfx_ctas *= ns;
  s.mix_ctas *= ns;
  s.dot_ctas *= ns;
  return s;
}

// Twiddle tables of the compile-time engine for one grid: [twx | pwx | twy |
// pwy | twz | pwz]; FP64 always (refresh pipeline), FP32 as well for the
// mixed path.  Sets the table pointers of d (grid type of the descriptor).
// cuTensorMapEncodeTiled from the driver, looked up once (no link-time
// dependency on the driver library)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return (EncodeTiledFn)p;
  }();
  return fn;
}

// natural index of digit-reversed position P of a length-L transform
static int digit_rev_inv_host(int L, int P) {
  const Fac f = factorize(L);
  int I = 0, M = L, scale = 1;
  for (int k = 0; k < f.n; ++k) {
    M /= f.r[k];
    const int dk = P / M;
    P -= dk * M;
    I += dk * scale;
    scale *= f.r[k];
  }
  return I;
}

// Tensor maps of w for the iteration's y and z passes (4D [site][z][y][x]
// in 8-byte elements, strides in bytes) and the ky table of the
// digit-reversed y rows.  Without the driver entry point the geometry falls
// back to the tile-per-CTA passes.
static int make_tmaps(r3d_ctx *c, Desc &d) {
  Geo &g = c->geo;
  d.tma_pc_y = d.tma_pc_z = 0;
  d.yrev = nullptr;
  if (!g.yz_tma) return R3D_OK;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) {
    g.yz_tma = 0;
    return R3D_OK;
  }
  const cuuint64_t cs = c->fp64 ? 16 : 8, e8 = cs / 8;
  const cuuint64_t dims[4] = {(cuuint64_t)d.hx * e8, (cuuint64_t)d.ny, (cuuint64_t)d.nz,
                              (cuuint64_t)d.n};
  const cuuint64_t strides[3] = {(cuuint64_t)d.hx * cs, (cuuint64_t)d.hx * d.ny * cs,
                                 (cuuint64_t)d.Nhs * cs};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const cuuint32_t by[4] = {(cuuint32_t)(g.fyt_pc * e8), (cuuint32_t)std::min(d.ny, 256), 1, 1};
  const cuuint32_t bz[4] = {(cuuint32_t)(g.zt_pc * e8), 1, (cuuint32_t)std::min(d.nz, 256), 1};
  CUresult r1 = enc((CUtensorMap *)&d.tm_y, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, d.w, dims, strides,
                    by, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  CUresult r2 = enc((CUtensorMap *)&d.tm_z, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, d.w, dims, strides,
                    bz, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r1 != CUDA_SUCCESS || r2 != CUDA_SUCCESS) {
    g.yz_tma = 0;
    return R3D_OK;
  }
  std::vector<int> yr(d.ny);
  for (int P = 0; P < d.ny; ++P) yr[P] = digit_rev_inv_host(d.ny, P);
  int *dy = nullptr;
  int rc = dalloc(c, (void **)&dy, yr.size() * sizeof(int));
  if (rc) return rc;
  CK(copy_h2d(c, dy, yr.data(), yr.size() * sizeof(int), c->stream));
  d.yrev = dy;
  d.tma_pc_y = g.fyt_pc;
  d.tma_pc_z = g.zt_pc;
  return R3D_OK;
}

static int make_twiddles(r3d_ctx *c, Desc &d, bool fp64_desc, void **t64, void **t32) {
  const int L[6] = {d.hx, d.hx, d.ny, d.ny, d.nz, d.nz};
  const double sc[6] = {-2.0 / d.hx, -1.0 / d.nx, -2.0 / d.ny, -1.0 / d.ny, -2.0 / d.nz,
                        -1.0 / d.nz};
  size_t tot = 0;
  for (int i = 0; i < 6; ++i) tot += L[i];
  int rc;
  if (!*t64 && (rc = dalloc(c, t64, tot * sizeof(double2)))) return rc;
  if (!fp64_desc && !*t32 && (rc = dalloc(c, t32, tot * sizeof(float2)))) return rc;
  size_t off = 0;
  const void *ptr[6];
  for (int i = 0; i < 6; ++i) {
    double2 *o64 = (double2 *)*t64 + off;
    float2 *o32 = fp64_desc ? nullptr : (float2 *)*t32 + off;
    launch_twiddle(o64, o32, L[i], sc[i], c->stream);
    ptr[i] = fp64_desc ? (const void *)o64 : (const void *)o32;
    off += L[i];
  }
  d.twx = ptr[0];
  d.pwx = ptr[1];
  d.twy = ptr[2];
  d.pwy = ptr[3];
  d.twz = ptr[4];
  d.pwz = ptr[5];
  CK(cudaGetLastError());
  return R3D_OK;
}
static void set_twiddles64(const void *t64, Desc &d) {
  const double2 *p = (const double2 *)t64;
  d.twx = p;
  d.pwx = p + d.hx;
  d.twy = p + 2 * d.hx;
  d.pwy = p + 2 * d.hx + d.ny;
  d.twz = p + 2 * d.hx + 2 * d.ny;
  d.pwz = p + 2 * d.hx + 2 * d.ny + d.nz;
}

// device bytes of the refresh's work buffer: FP64 c_ref / h_ref, n half
// spectra, descriptor, control block, launch prefixes
static size_t refresh_bytes(const Desc &d) {
  return (size_t)d.n * d.Ns * 8 + (size_t)d.n * d.Nhs * 16 + sizeof(Desc) + sizeof(Ctl) + 64;
}

// Refresh (also the setup's long-range term): freeze c_ref = c_s(t) (zero at
// setup) and set lr = 1 + h_ref, h_ref = F^-1[chi (F(c_ref) - q phi_L(k))],
// with the FP64 pass kernels.  Leaves t, R and the mixer state untouched: the
// residual of the current t is unchanged in exact arithmetic.
template <typename P>
static int refresh(r3d_ctx *c, bool zero) {
  const auto t_start = std::chrono::steady_clock::now();
  const Desc &d = c->desc;
  const int n = d.n;
  const long long N = d.Ns, Nh = d.Nhs;  // padded site strides
  cudaStream_t s = c->stream;
  if (!c->rplanned) {
    int rc = plan_geo(c, c->rdesc, c->rgeo, true, n);
    if (rc) return rc;
    c->rplanned = true;
  }
  Desc dr = c->rdesc;
  const Geo &g = c->rgeo;
  const size_t bytes = refresh_bytes(d);
  char *tmp = c->rtmp;
  if (!tmp) {
    if (c->fp64) {
      CK(pool_alloc(c->opts.device, (void **)&tmp, bytes, s));
    } else {
      int rc = dalloc(c, (void **)&c->rtmp, bytes);
      if (rc) return rc;
      tmp = c->rtmp;
    }
  }
  double *c64 = (double *)tmp;                      // c_ref, then h_ref
  double2 *w64 = (double2 *)(c64 + (size_t)n * N);  // n half spectra
  Desc *dd = (Desc *)(w64 + (size_t)n * Nh);
  Ctl *ctl = (Ctl *)((char *)dd + sizeof(Desc));
  int *pre = (int *)((char *)ctl + sizeof(Ctl));
  if (zero)
    CK(cudaMemsetAsync(c64, 0, (size_t)n * N * 8, s));
  else
    launch_cref<P>(d, c64, s);
  for (int v = 0; v < n; ++v) dr.qv[v] = d.qv[v];
  dr.clos = d.clos;
  dr.pse_n = d.pse_n;
  dr.w = w64;
  dr.chi = c->chi64;
  dr.chis = d.chis;
  dr.cubic = d.cubic;
  dr.kidx = c->kidx;
  dr.fk = c->fk;
  dr.ctl = ctl;
  set_twiddles64(c->tw64, dr);
  int pf[8] = {0, g.tiles_x, 0, g.tiles_y, 0, g.tiles_z, 0, g.ix_ctas};
  CK(cudaMemsetAsync(ctl, 0, sizeof(Ctl), s));
  CK(copy_h2d(c, dd, &dr, sizeof(Desc), s));
  CK(copy_h2d(c, pre, pf, sizeof(pf), s));
  kernels_set_smem(true, kSmemMax);
  pass_fx<P64>(dr, g, Batch{dd, pre, 1}, s, 0, c64);
  pass_fy<P64>(dr, g, Batch{dd, pre + 2, 1}, s, -1, 0);
  pass_zoz<P64>(dr, g, Batch{dd, pre + 4, 1}, s, 2, 0);
  pass_fy<P64>(dr, g, Batch{dd, pre + 2, 1}, s, 1, 0);
  pass_ix<P64>(dr, g, Batch{dd, pre + 6, 1}, s, 0, c64);
  launch_lr_update<P>(c64, c->lr, (long long)n * N, s);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  if (tmp != c->rtmp) cudaFreeAsync(tmp, s);
  if (!zero) {
    c->refreshes += 1;
    c->refresh_ms += std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t_start).count();
  }
  return R3D_OK;
}

static size_t plan_bytes(const r3d_ctx *c, const Desc &d, int nshell) {
  const size_t R = c->rsz, T = 8, N = (size_t)d.N, n = (size_t)d.n;
  size_t b = 0;
  b += 3 * n * N * R + 2 * n * N * T;  // u, res, lr (grid type), t, gq (state type)
  b += n * N * R;                  // w (n half spectra)
  b += N * R + N * 8;              // fr, fk (FP64 half spectrum)
  if (!c->fp64) b += n * N * R + (size_t)nshell * n * n * 8;  // cref, chi64
  b += refresh_bytes(d);           // refresh work buffer (kept on the mixed path)
  b += (size_t)d.Nh * 4;           // kidx
  b += (size_t)nshell * n * n * R;
  size_t slots = c->mixer == MIX_AN2 ? 2 : (size_t)c->history + 1;
  // mixer history (residuals, states; mixed: FP32 differences of states, and
  // for ANM one more FP32 array)
  b += slots * n * N * (R + (!c->fp64 ? R : T));
  if (c->mixer == MIX_ANM && !c->fp64) b += n * N * R;
  b += (size_t)std::max(max_ix_ctas(c->geo), c->geo.dot_ctas) * kPartials * 8;
  b += (size_t)(c->prob.maxstep + 1) * 8 + sizeof(Ctl) + sizeof(Desc) + 4096;
  return b;
}

// ------------------------------------------------------------ autotuning
// The iteration's x passes have two implementations each: one tile per CTA
// with loads through registers (k_fx_ct / k_ix_ct), or persistent CTAs whose
// inputs the bulk copy engine stages (k_fx_bulk / k_ix_bulk).  Which is
// faster depends on the row length, the sites and the precision, so the
// first solve of each geometry times both on its own buffers -- the mode-1 x
// passes write only w, gq, the residual and the partials, which every
// iteration rewrites -- and the choice holds for the process.
static std::mutex g_tune_mu;
// per geometry: the FX and IX variant (0 one tile per CTA, 1 bulk-staged,
// 2 warp tiles, 3 (IX) bulk-staged with half-size tiles)
static std::map<std::array<int, 5>, std::array<int, 3>> g_tune;  // + y/z on TMA

// The committed choice per geometry.  Results of a solve depend (in their
// last bits, which the Anderson iteration amplifies over hundreds of steps)
// on the variant: each one sums the residual and its dots in its own order.
// So the variant is a fixed function of the geometry -- this table, filled
// from timings taken on a B200 with R3D_AUTOTUNE=1 (which times every
// candidate and prints the row), else the rule in tune_rule -- and a solve
// gives the same iterations and results on every box and every run.
struct TuneRow {
  int nx, ny, nz, n, fp64;
  int fx, ix, yz;
  int mfx;  // mixed AN2: 1 = the mix fused into FX (when the geometry has it)
};
static const TuneRow kTuneTable[] = {
#include "r3d_tune_table.inc"
};

// Variants for a geometry with no row in the table (what the measured rows
// favour): bulk-staged x passes for rows of 128 or more complex points, else
// one tile per CTA (warp tiles for the shortest rows); the register-pass
// Stockham y and z passes where they cover the lengths and sites, else the
// copy-engine y passes with the tile-per-CTA z pass.
static std::array<int, 3> tune_rule(const Geo &g, const Desc &d) {
  std::array<int, 3> u{0, 0, 0};
  if (d.hx <= 32 && g.fxw_pc) u[0] = 2;
  else if (d.hx >= 128 && g.fxb_pc) u[0] = 1;
  if (d.hx <= 32 && g.ixw_pc) u[1] = 2;
  else if (d.hx >= 128 && g.ixb_pc) u[1] = 1;
  if (g.yz_sr)
    u[2] = 4;
  else if (g.yz_tma)
    u[2] = d.ct_z ? 1 : 2;
  return u;
}

template <typename P>
static int autotune_x(r3d_ctx *c) {
  Geo &g = c->geo;
  const Desc &d = c->desc;
  if (!g.fxb_pc && !g.ixb_pc && !g.fxw_pc && !g.ixw_pc && !g.fxs_pc && !g.yz_tma && !g.yz_sr)
    return R3D_OK;
  const std::array<int, 5> key{d.nx, d.ny, d.nz, d.n, c->fp64 ? 1 : 0};
  std::array<int, 3> use{0, 0, g.yz_tma};
  bool known = false;
  // R3D_X_VARIANT=0|1|2 replaces the timing by that variant where it exists
  // (diagnostics and the per-variant parity tests)
  if (const char *ev = getenv("R3D_X_VARIANT")) {
    const int k = std::atoi(ev);
    const bool fx = k == 0 || ((k == 1 || k == 3) && g.fxb_pc) || (k == 2 && g.fxw_pc) ||
                    (k == 4 && g.fxs_pc);
    const bool ix = k == 0 || ((k == 1 || k == 3) && g.ixb_pc) || (k == 2 && g.ixw_pc) ||
                    (k == 4 && g.ixs_pc);
    use = {fx ? (k == 3 ? 1 : k) : 0, ix ? k : 0, g.yz_tma};
    if (const char *ey = getenv("R3D_YZ_VARIANT")) {
      const int k = std::atoi(ey);
      use[2] = (k >= 3) ? (g.yz_sr ? (k >= 5 ? (g.yz_srp ? 5 : 4) : k) : 0)
                        : (k == 1 && !d.ct_z) ? 0 : std::min(k, g.yz_tma);
    }
    known = true;
  } else if (!getenv("R3D_AUTOTUNE")) {  // the committed table, else the fixed rule
    use = tune_rule(g, d);
    g.mfx = g.mfx_avail;  // the rule: fused where available
    for (const TuneRow &r : kTuneTable)
      if (r.nx == d.nx && r.ny == d.ny && r.nz == d.nz && r.n == d.n && r.fp64 == (c->fp64 ? 1 : 0)) {
        use = {r.fx, r.ix, r.yz};
        g.mfx = g.mfx_avail && r.mfx;
        break;
      }
    // a row naming a variant this geometry does not offer falls back to the rule
    const bool ok = (use[0] == 0 || (use[0] == 1 && g.fxb_pc) || (use[0] == 2 && g.fxw_pc) ||
                     (use[0] == 4 && g.fxs_pc)) &&
                    (use[1] == 0 || ((use[1] == 1 || use[1] == 3) && g.ixb_pc) ||
                     (use[1] == 2 && g.ixw_pc) || (use[1] == 4 && g.ixs_pc)) &&
                    (use[2] >= 3 ? (g.yz_sr && (use[2] <= 4 || (use[2] == 5 && g.yz_srp)))
                                 : (use[2] <= g.yz_tma && !(use[2] == 1 && !d.ct_z)));
    if (!ok) use = tune_rule(g, d);
    known = true;
  } else {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      use = it->second;
      known = true;
    }
  }
  // geometry with only variant k of the x passes
  auto only = [&](int k) {
    Geo o = g;
    if (k != 1) o.fxb_pc = o.ixb_pc = 0;
    if (k != 2) o.fxw_pc = o.ixw_pc = 0;
    if (k != 4) o.fxs_pc = o.ixs_pc = 0;
    return o;
  };
  if (!known) {
    cudaStream_t s = c->stream;
    int *pf = nullptr;
    // the bulk IX with half the rows per tile (more CTAs per SM)
    Geo half = g;
    const bool has_half = g.ixb_pc >= 2 &&
                          ixb_config(c->opts.device, d, c->fp64, g.ixb_pc / 2, half) &&
                          half.ixb_ctas <= c->npart;
    CK(cudaMalloc((void **)&pf, 30 * sizeof(int)));
    const int pre[30] = {0, d.tiles_x, 0, g.fxb_ctas, 0, g.fxw_ctas, 0, g.ix_ctas,
                         0, g.ixb_ctas, 0, g.ixw_ctas, 0, g.tiles_y, 0, g.tiles_z,
                         0, g.fyt_ctas, 0, g.zt_ctas, 0, half.ixb_ctas, 0, g.fys_ctas,
                         0, g.zs_ctas, 0, g.fxs_ctas, 0, g.ixs_ctas};
    CK(copy_h2d(c, pf, pre, sizeof(pre), s));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time = [&](auto &&launch) {
      launch();
      cudaEventRecord(e0, s);
      for (int i = 0; i < 10; ++i) launch();
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      return ms;
    };
    float best[2] = {0, 0};
    std::string report;  // candidate times, us per launch
    auto note = [&](const char *what, int k, float ms) {
      report += " " + std::string(what) + std::to_string(k) + "=" +
                std::to_string((int)(ms * 100.0f)) ;  // 10 launches: ms*100 = us/launch
    };
    for (int k = 0; k < 3; ++k) {
      const Geo o = only(k);
      const bool fx = k == 0 || (k == 1 ? g.fxb_pc : g.fxw_pc);
      const bool ix = k == 0 || (k == 1 ? g.ixb_pc : g.ixw_pc);
      if (fx) {
        const float ms = time([&] { pass_fx<P>(d, o, Batch{c->ddesc, pf + 2 * k, 1}, s, 1, nullptr); });
        note("fx", k, ms);
        if (k == 0 || ms < best[0]) best[0] = ms, use[0] = k;
      }
      if (ix) {
        const float ms =
            time([&] { pass_ix<P>(d, o, Batch{c->ddesc, pf + 6 + 2 * k, 1}, s, 1, nullptr); });
        note("ix", k, ms);
        if (k == 0 || ms < best[1]) best[1] = ms, use[1] = k;
      }
      if (k == 2 && g.fxs_pc) {  // variant 4: the Stockham engine
        const Geo o4 = only(4);
        const float mf = time([&] { pass_fx<P>(d, o4, Batch{c->ddesc, pf + 26, 1}, s, 1, nullptr); });
        note("fx", 4, mf);
        if (mf < best[0]) best[0] = mf, use[0] = 4;
        const float mi = time([&] { pass_ix<P>(d, o4, Batch{c->ddesc, pf + 28, 1}, s, 1, nullptr); });
        note("ix", 4, mi);
        if (mi < best[1]) best[1] = mi, use[1] = 4;
      }
      if (k == 1 && has_half) {  // variant 3: bulk IX, half the rows per tile
        Geo o3 = only(1);
        o3.ixb_pc = half.ixb_pc;
        o3.smixb = half.smixb;
        o3.ixb_ctas = half.ixb_ctas;
        o3.ixb_per = half.ixb_per;
        const float ms = time([&] { pass_ix<P>(d, o3, Batch{c->ddesc, pf + 20, 1}, s, 1, nullptr); });
        note("ix", 3, ms);
        if (ms < best[1]) best[1] = ms, use[1] = 3;
      }
    }
    if (g.yz_tma || g.yz_sr) {  // the y/z trio: tile-per-CTA, copy-engine y, copy-engine
                                // y and z, register-pass Stockham (OZ on registers / shared)
      float best2 = 0;
      for (int k = 0; k < 6; ++k) {
        if (k == 1 && !d.ct_z) continue;
        if ((k == 1 || k == 2) && !g.yz_tma) continue;
        if (k >= 3 && !g.yz_sr) continue;
        if (k == 5 && !g.yz_srp) continue;
        Geo o = g;
        o.yz_tma = k;
        const Batch by{c->ddesc, pf + (k >= 3 ? 22 : k ? 16 : 12), 1},
            bz{c->ddesc, pf + (k >= 3 ? 24 : k == 2 ? 18 : 14), 1};
        const float ms = time([&] {
          pass_fy_iter<P>(d, o, by, s, -1);
          pass_zoz_iter<P>(d, o, bz, s);
          pass_fy_iter<P>(d, o, by, s, 1);
        });
        note("yz", k, ms);
        if (k == 0 || ms < best2) best2 = ms, use[2] = k;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaError_t e = cudaGetLastError();
    cudaFree(pf);
    if (e != cudaSuccess) return fail(c, R3D_ECUDA, std::string("autotune: ") + cudaGetErrorString(e));
    std::fprintf(stderr, "r3d-tune row: {%d, %d, %d, %d, %d, %d, %d, %d, %d},  // us:%s\n", d.nx,
                 d.ny, d.nz, d.n, c->fp64 ? 1 : 0, use[0], use[1], use[2], g.mfx_avail ? 1 : 0,
                 report.c_str());
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = use;
  }
  if (!getenv("R3D_X_VARIANT") && getenv("R3D_AUTOTUNE")) g.mfx = g.mfx_avail;
  if (use[0] != 1) g.fxb_pc = 0;
  if (use[0] != 2) g.fxw_pc = 0;
  if (use[0] != 4) g.fxs_pc = 0;
  if (use[1] != 4) g.ixs_pc = 0;
  if (const char *em = getenv("R3D_MFX")) g.mfx = g.mfx_avail && std::atoi(em) != 0;
  if (use[1] == 3) {
    if (!(g.ixb_pc >= 2 && ixb_config(c->opts.device, d, c->fp64, g.ixb_pc / 2, g))) g.ixb_pc = 0;
  } else if (use[1] != 1) {
    g.ixb_pc = 0;
  }
  if (use[1] != 2) g.ixw_pc = 0;
  g.yz_tma = use[2];
  return R3D_OK;
}

template <typename P>
static int init_typed(r3d_ctx *c, const ShellTable &st) {
  using R = typename P::R;
  using T = typename P::T;
  Problem &p = c->prob;
  Desc &d = c->desc;
  cudaStream_t s = c->stream;
  const int n = d.n, nu = (int)p.q.size();
  const long long N = d.Ns, Nh = d.Nhs;  // padded site strides
  int rc;
  // grids
  if ((rc = dalloc(c, &c->u, n * N * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &c->t, n * N * sizeof(T)))) return rc;
  if ((rc = dalloc(c, &c->res, n * N * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &c->lr, n * N * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &c->w, n * Nh * 2 * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &c->fr, d.N * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &c->fk, d.Nh * sizeof(double2)))) return rc;
  if ((rc = dalloc(c, (void **)&c->kidx, d.Nh * 4))) return rc;
  const int chis = (n * n + 3) / 4 * 4;  // padded rows: aligned vector loads
  if ((rc = dalloc(c, &c->chi, (size_t)st.nshell * chis * sizeof(R)))) return rc;
  // AN2: hist_a = t slots (T), hist_b = residual slots (R);
  // ANM: hist_a = residual ring (R), hist_b = z ring (T)
  const size_t slots = c->mixer == MIX_AN2 ? 2 : (size_t)c->history + 1;
  // (mixed AN2: the t slots hold FP32 differences of successive t; mixed
  // ANM: hist_b holds FP32 differences of successive z and, after the ring,
  // the last mix's t difference)
  const size_t ha = c->mixer == MIX_AN2 ? (c->fp64 ? sizeof(T) : sizeof(R)) : sizeof(R);
  const size_t hb = c->mixer == MIX_AN2 ? sizeof(R) : (c->fp64 ? sizeof(T) : sizeof(R));
  const size_t bslots = slots + (c->mixer == MIX_ANM && !c->fp64 ? 1 : 0);
  if ((rc = dalloc(c, &c->hist_a, slots * n * N * ha))) return rc;
  if ((rc = dalloc(c, &c->hist_b, bslots * n * N * hb))) return rc;
  if ((rc = dalloc(c, &c->gq, n * N * sizeof(T)))) return rc;
  const int npart = std::max(max_ix_ctas(c->geo), c->geo.dot_ctas);
  if ((rc = dalloc(c, (void **)&c->partials, (size_t)npart * kPartials * 8))) return rc;
  c->npart = npart;
  double *rmslog;
  if ((rc = dalloc(c, (void **)&rmslog, (size_t)(p.maxstep + 1) * 8))) return rc;
  if ((rc = dalloc(c, (void **)&c->ctl, sizeof(Ctl)))) return rc;
  if ((rc = dalloc(c, (void **)&c->ddesc, sizeof(Desc)))) return rc;
  if ((rc = dalloc(c, (void **)&c->dprefix, pf_len(1) * sizeof(int)))) return rc;
  CK(cudaMemsetAsync(c->hist_a, 0, slots * n * N * ha, s));
  CK(cudaMemsetAsync(c->hist_b, 0, bslots * n * N * hb, s));
  CK(cudaMemsetAsync(c->res, 0, n * N * sizeof(R), s));
  CK(cudaMemsetAsync(c->u, 0, n * N * sizeof(R), s));
  CK(cudaMemsetAsync(c->t, 0, n * N * sizeof(T), s));
  CK(cudaMemsetAsync(c->lr, 0, n * N * sizeof(R), s));
  CK(cudaMemsetAsync(c->gq, 0, n * N * sizeof(T), s));
  CK(cudaMemsetAsync(c->w, 0, n * Nh * 2 * sizeof(R), s));
  CK(cudaMemsetAsync(c->fr, 0, d.N * sizeof(R), s));
  CK(cudaMemsetAsync(c->fk, 0, d.Nh * sizeof(double2), s));
  if (!c->fp64) {
    if ((rc = dalloc(c, &c->cref, n * N * sizeof(R)))) return rc;
    if ((rc = dalloc(c, &c->chi64, (size_t)st.nshell * ((n * n + 3) / 4 * 4) * 8))) return rc;
    CK(cudaMemsetAsync(c->cref, 0, n * N * sizeof(R), s));
  }
  CK(cudaMemsetAsync(c->partials, 0, (size_t)npart * kPartials * 8, s));

  d.clos = p.clos;
  d.pse_n = p.pse_n;
  d.mixer = c->mixer;
  d.history = c->history;
  d.beta = c->damping >= 0 ? c->damping : p.mix_m;
  d.m = p.mix_m;
  d.mp = p.mix_mp;
  for (int v = 0; v < n; ++v) {
    d.irho[v] = 1.0 / p.rhov[v];
    d.qv[v] = p.qv[v];
  }
  d.u = c->u;
  d.t = c->t;
  d.fr = c->fr;
  d.res = c->res;
  d.w = c->w;
  d.fk = nullptr;  // phi_L(k) enters through lr (see refresh)
  d.chi = c->chi;
  d.lr = c->lr;
  d.gq = c->gq;
  d.cref = c->cref;
  d.kidx = c->kidx;
  d.hist_a = c->hist_a;
  d.hist_b = c->hist_b;
  d.partials = c->partials;
  d.ctl = c->ctl;
  if ((rc = make_twiddles(c, d, c->fp64, &c->tw64, &c->tw32))) return rc;
  if ((rc = make_tmaps(c, d))) return rc;
  d.partial_base = 0;
  d.rmslog = rmslog;
  // Test hook of the error path of the staged passes: R3D_WAIT_POLLS=k makes
  // their bounded waits for staged copies give up after k polls, so that a
  // solve fails with R3D_ECUDA and the device stays usable.
  d.wait_polls = 0;
  if (const char *ew = getenv("R3D_WAIT_POLLS")) d.wait_polls = std::atoi(ew);

  // chi shell table, scaled by 2/N (the unnormalised transforms' factor)
  d.cubic = st.cubic ? 1 : 0;
  d.chis = chis;
  std::vector<double> chi64((size_t)st.nshell * chis, 0.0);
  {
    std::vector<R> chi(chi64.size(), (R)0);
    const double sc = 2.0 / (double)d.N;
    for (int sh = 0; sh < st.nshell; ++sh)
      for (int q = 0; q < n * n; ++q) {
        const size_t i = (size_t)sh * chis + q;
        chi64[i] = st.chi[(size_t)sh * n * n + q] * sc;
        chi[i] = (R)chi64[i];
      }
    CK(copy_h2d(c, c->chi, chi.data(), chi.size() * sizeof(R), s));
    if (c->fp64)
      c->chi64 = c->chi;
    else
      CK(copy_h2d(c, c->chi64, chi64.data(), chi64.size() * 8, s));
    CK(cudaStreamSynchronize(s));
  }
  // shell index of every half-spectrum point
  {
    uint32_t *dtuple = nullptr;
    if (!st.cubic) {
      if ((rc = dalloc(c, (void **)&dtuple, st.tuple_idx.size() * 4))) return rc;
      CK(copy_h2d(c, dtuple, st.tuple_idx.data(), st.tuple_idx.size() * 4, s));
    }
    launch_kidx(d, dtuple, st.cubic ? 1 : 0, s);
    CK(cudaGetLastError());
  }
  // potentials: atom tables (cal_LJ.cu:33-40 mixing rules)
  {
    const double lambda1 = p.adswitch == 1 ? p.lambda : 1.0;
    std::vector<double> ax(nu), ay(nu), az(nu), sig2((size_t)n * nu), eps4((size_t)n * nu);
    for (int iu = 0; iu < nu; ++iu) {
      ax[iu] = p.r[3 * iu];
      ay[iu] = p.r[3 * iu + 1];
      az[iu] = p.r[3 * iu + 2];
    }
    for (int v = 0; v < n; ++v)
      for (int iu = 0; iu < nu; ++iu) {
        double sg = (p.sig[iu] + p.sigv[v]) * 0.5 * lambda1;
        sig2[(size_t)v * nu + iu] = sg * sg;
        eps4[(size_t)v * nu + iu] = std::sqrt(p.eps[iu] * p.epsv[v]) * 4.0;
      }
    double *dat;
    const size_t natom = std::max(nu, 1);
    if ((rc = dalloc(c, (void **)&dat, (4 + 2 * (size_t)n) * natom * 8))) return rc;
    double *dx = dat, *dy = dat + natom, *dz = dat + 2 * natom, *dq = dat + 3 * natom;
    double *dsig = dat + 4 * natom, *deps = dsig + (size_t)n * natom;
    if (nu > 0) {
      CK(copy_h2d(c, dx, ax.data(), nu * 8, s));
      CK(copy_h2d(c, dy, ay.data(), nu * 8, s));
      CK(copy_h2d(c, dz, az.data(), nu * 8, s));
      CK(copy_h2d(c, dq, p.q.data(), nu * 8, s));
      for (int v = 0; v < n; ++v) {
        CK(copy_h2d(c, dsig + (size_t)v * natom, sig2.data() + (size_t)v * nu, nu * 8, s));
        CK(copy_h2d(c, deps + (size_t)v * natom, eps4.data() + (size_t)v * nu, nu * 8, s));
      }
    }
    AtomTab at{dx, dy, dz, dq, dsig, deps, nu};
    // the kernel indexes sig2/eps4 as [v * nu + i]; pass nu as the stride
    const double ikbt = 1.0 / (phys::avogadro * phys::boltzmann * p.temper);
    const int coulomb = p.adswitch != 1;
    const double lambda2 = p.adswitch == 2 ? p.lambda : 1.0;
    const double ubeta = phys::hartree * phys::bohr / (phys::boltzmann * p.temper) * lambda2;
    double dr[3] = {p.box[0] / d.nx, p.box[1] / d.ny, p.box[2] / d.nz};
    // FP64 phase tables of the k-space Coulomb sum (setup scratch)
    const size_t ntab = (size_t)std::max(nu, 1) * (d.hx + d.ny + d.nz);
    double2 *tabs = nullptr;
    cudaError_t e = pool_alloc(c->opts.device, (void **)&tabs, ntab * sizeof(double2), s);
    if (e != cudaSuccess) return fail(c, R3D_ENOMEM, "setup scratch");
    double *fr64 = nullptr;
    cudaEvent_t ev[4];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    CK(cudaEventRecord(ev[0], s));
    if (nu > 0) {
      if (natom != (size_t)nu) return fail(c, R3D_EINVAL, "internal: atom stride");
      launch_potential<P>(d, at, ikbt, ubeta, dr, coulomb, fr64, s);
      CK(cudaGetLastError());
    } else {
      CK(cudaMemsetAsync(c->u, 0, n * N * sizeof(R), s));
      CK(cudaMemsetAsync(c->t, 0, n * N * sizeof(T), s));
    }
    CK(cudaEventRecord(ev[1], s));
    if (coulomb && nu > 0) {
      double2 *ex = tabs, *ey = tabs + (size_t)nu * d.hx, *ez = ey + (size_t)nu * d.ny;
      launch_phase_tables(ex, ey, ez, dx, dy, dz, nu, d.nx, d.ny, d.nz, p.box, s);
      const double dv = p.box[0] * p.box[1] * p.box[2] / (double)d.N;
      launch_fk(d, (double2 *)c->fk, ex, ey, ez, dq, nu, ubeta, p.box, dv, s);
      CK(cudaGetLastError());
    }
    CK(cudaEventRecord(ev[2], s));
    CK(cudaStreamSynchronize(s));
    cudaFreeAsync(tabs, s);
    // long-range h term: lr = 1 - F^-1[chi q phi_L(k)]  (refresh, c_ref = 0)
    CK(cudaEventRecord(ev[3], s));
    if ((rc = refresh<P>(c, true))) return rc;
    cudaEvent_t ev4;
    CK(cudaEventCreate(&ev4));
    CK(cudaEventRecord(ev4, s));
    CK(cudaEventSynchronize(ev4));
    float t01 = 0, t12 = 0, t34 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    cudaEventElapsedTime(&t34, ev[3], ev4);
    c->setup_ms[0] = t01;
    c->setup_ms[1] = t12;
    c->setup_ms[2] = t34;
    for (auto &e : ev) cudaEventDestroy(e);
    cudaEventDestroy(ev4);
  }
  // control block and descriptor
  {
    Ctl h{};
    h.status = RUNNING;
    h.maxstep = p.maxstep;
    h.tol = p.convergence;
    h.count_left = p.count;
    CK(copy_h2d(c, c->ctl, &h, sizeof(Ctl), s));
    CK(copy_h2d(c, c->ddesc, &d, sizeof(Desc), s));
    if ((rc = autotune_x<P>(c))) return rc;
    // every IX variant writes one row of partials per CTA
    if (std::max(iter_ix_ctas(c->geo), c->geo.dot_ctas) > c->npart)
      return fail(c, R3D_ECUDA, "internal: partials rows for the chosen IX variant");
    const std::vector<int> pre = make_prefix(c->geo, 1);
    CK(copy_h2d(c, c->dprefix, pre.data(), pre.size() * sizeof(int), s));
    CK(cudaStreamSynchronize(s));
  }
  // the attribute is a per-function limit shared by every context: always
  // allow the largest tile any context may choose (set before any capture)
  kernels_set_smem(c->fp64, kSmemMax);
  kernels_set_smem(true, kSmemMax);
  CK(cudaGetLastError());
  return R3D_OK;
}

extern "C" int r3d_initialize(r3d_ctx *c) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (c->initialized) return fail(c, R3D_ESTATE, "already initialized");
  if (!c->prob.has_solute) return fail(c, R3D_ESTATE, "no solute/control loaded");
  if (!c->prob.has_solvent) return fail(c, R3D_ESTATE, "no solvent loaded");
  if (c->prob.natv > kMaxSites) return fail(c, R3D_EINVAL, "too many solvent sites");
  if (c->prob.maxstep < 1) return fail(c, R3D_EINVAL, "maxstep must be >= 1");
  if (c->opts.device < 0) return fail(c, R3D_ESTATE, "host-only context (device < 0)");
  CK(cudaSetDevice(c->opts.device));
  Desc d{};
  int rc = plan_geometry(c, d);
  if (rc) return rc;
  ShellTable st;
  std::string m = build_shells(c->prob, st);
  if (!m.empty()) return fail(c, R3D_EINVAL, m);
  c->nshell = st.nshell;
  size_t need = plan_bytes(c, d, st.nshell);
  if (c->opts.hbm_budget && need > c->opts.hbm_budget)
    return fail(c, R3D_EBUDGET, "problem needs " + std::to_string(need) +
                                    " device bytes, budget " +
                                    std::to_string(c->opts.hbm_budget));
  size_t fre = 0, tot = 0;
  CK(cudaMemGetInfo(&fre, &tot));
  fre += pool_spare(c->opts.device);  // held by the pool for the next solve
  if (need > fre) return fail(c, R3D_ENOMEM, "problem needs " + std::to_string(need) +
                                                 " device bytes, " + std::to_string(fre) + " free");
  c->desc = d;
  const auto t0 = std::chrono::steady_clock::now();
  rc = c->fp64 ? init_typed<P64>(c, st) : init_typed<PMix>(c, st);
  if (rc) {
    free_all(c);
    return rc;
  }
  c->setup_ms[3] =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  c->initialized = true;
  return R3D_OK;
}

extern "C" int r3d_refresh_timing(const r3d_ctx *c, int *count, double *ms) {
  if (!c || !count || !ms) return fail(nullptr, R3D_EINVAL, "bad arguments");
  *count = c->refreshes;
  *ms = c->refresh_ms;
  return R3D_OK;
}

extern "C" int r3d_setup_timing(const r3d_ctx *c, double *ms) {
  if (!c || !ms) return fail(nullptr, R3D_EINVAL, "bad arguments");
  if (!c->initialized) return fail(nullptr, R3D_ESTATE, "setup timing before initialize");
  for (int i = 0; i < 4; ++i) ms[i] = c->setup_ms[i];
  return R3D_OK;
}

// --------------------------------------------------------------- iterate
// Solves of one geometry whose iteration kernels are launched together.
struct Group {
  Desc rep;          // host descriptor of the first solve (shape fields)
  Geo geo;           // geometry of one solve
  const Desc *ddescs;  // device descriptors [ns]
  const int *dpf;    // device prefix block (make_prefix)
  int ns;
  int mixer;
};
static Group single_group(const r3d_ctx *c) {
  return Group{c->desc, c->geo, c->ddesc, c->dprefix, 1, c->mixer};
}

// stage: 0 = full iteration (evaluate, decide, mix), 1 = evaluate only
// (calculate), 2 = mix only (anderson).  Returns the kernels launched.
template <typename P>
static int enqueue_group(const Group &G, cudaStream_t s, int stage) {
  const int ns = G.ns;
  const Geo g = scaled(G.geo, ns);
  const Desc &d = G.rep;
  auto B = [&](int k) { return Batch{G.ddescs, G.dpf + pf_off(ns, k), ns}; };
  const int *ixc = G.dpf + pf_off(ns, PF_IXC), *dotc = G.dpf + pf_off(ns, PF_DOTC);
  int k = 0;
  if (stage != 2) {
    pass_fx<P>(d, g, B(PF_X), s, 1, nullptr, stage == 0 ? 1 : 0);
    pass_fy_iter<P>(d, g, B(PF_Y), s, -1);
    pass_zoz_iter<P>(d, g, B(PF_Z), s);
    pass_fy_iter<P>(d, g, B(PF_Y), s, 1);
    pass_ix<P>(d, g, B(PF_IX), s, 1, nullptr);
    k += 5;
    if (G.mixer == MIX_ANM) {
      launch_anm<P>(B(PF_DOT), g.dot_ctas, G.ddescs, dotc, ns, s, 0);
      ++k;
    }
    launch_reduce(G.ddescs, ixc, ns, stage == 0 ? 0 : 2, s);
    ++k;
  } else {
    launch_reduce(G.ddescs, ixc, ns, 1, s);
    ++k;
  }
  if (stage != 1) {
    if (G.mixer == MIX_AN2) {
      // (with the mix-fused FX the iteration's mix runs at the start of the
      // next iteration's FX)
      if (!(stage == 0 && g.mfx)) {
        launch_mix_an2<P>(B(PF_MIX), g.mix_ctas, s);
        ++k;
      }
    } else {
      launch_anm<P>(B(PF_MIX), g.mix_ctas, G.ddescs, dotc, ns, s, 1);
      launch_anm<P>(B(PF_MIX), g.mix_ctas, G.ddescs, dotc, ns, s, 2);
      k += 2;
    }
  }
  return k;
}
template <typename P>
static void enqueue(r3d_ctx *c, int stage) {
  const int k = enqueue_group<P>(single_group(c), c->stream, stage);
  if (stage == 0) c->kernels_per_iter = k;
}

static int read_ctl(r3d_ctx *c, Ctl &h) {
  CK(copy_d2h(c, &h, c->ctl, sizeof(Ctl), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (h.err & 2) return fail(c, R3D_ECUDA, "a kernel's index check failed (debug build)");
  if (h.err) return fail(c, R3D_ECUDA, "a kernel's bounded wait for a staged copy ran out");
  return R3D_OK;
}
static int set_running(r3d_ctx *c) {
  int st = RUNNING;
  CK(copy_h2d(c, &c->ctl->status, &st, sizeof(int), c->stream));
  return R3D_OK;
}

extern "C" int r3d_calculate(r3d_ctx *c, double *rms) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "calculate before initialize");
  CK(cudaSetDevice(c->opts.device));
  int rc = set_running(c);
  if (rc) return rc;
  if (c->fp64)
    enqueue<P64>(c, 1);
  else
    enqueue<PMix>(c, 1);
  CK(cudaGetLastError());
  Ctl h;
  if ((rc = read_ctl(c, h))) return rc;
  if (rms) *rms = h.rms;
  return R3D_OK;
}

extern "C" int r3d_anderson(r3d_ctx *c) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "anderson before initialize");
  CK(cudaSetDevice(c->opts.device));
  int rc = set_running(c);
  if (rc) return rc;
  if (c->fp64)
    enqueue<P64>(c, 2);
  else
    enqueue<PMix>(c, 2);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return R3D_OK;
}

// One iteration captured once as a CUDA graph (pointers never change).
static int ensure_graph(r3d_ctx *c) {
  if (c->gexec) return R3D_OK;
  cudaStream_t s = c->stream;
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  if (c->fp64)
    enqueue<P64>(c, 0);
  else
    enqueue<PMix>(c, 0);
  CK(cudaStreamEndCapture(s, &g));
  cudaError_t e = cudaGraphInstantiate(&c->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return fail(c, R3D_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  return R3D_OK;
}

static int reset_mixer(r3d_ctx *c) {
  Ctl h{};
  h.status = RUNNING;
  h.maxstep = c->prob.maxstep;
  h.tol = c->prob.convergence;
  h.count_left = c->prob.count;
  CK(copy_h2d(c, c->ctl, &h, sizeof(Ctl), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return R3D_OK;
}

extern "C" int r3d_step(r3d_ctx *c, int nsteps, double *ms) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "step before initialize");
  if (nsteps < 0) return fail(c, R3D_EINVAL, "nsteps < 0");
  CK(cudaSetDevice(c->opts.device));
  int rc = ensure_graph(c);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  for (int i = 0; i < nsteps; ++i) CK(cudaGraphLaunch(c->gexec, c->stream));
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaEventSynchronize(e1));
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t;
  return R3D_OK;
}

template <typename P>
static int profile_typed(r3d_ctx *c, int reps, std::string &names, double *ms,
                         double *bytes, int *nk) {
  using R = typename P::R;
  using T = typename P::T;
  const Desc &d = c->desc;
  cudaStream_t s = c->stream;
  const int *pf = c->dprefix;
  const double n = d.n, N = (double)d.N, rs = sizeof(R), ts = sizeof(T);
  Batch bx{c->ddesc, pf + pf_off(1, PF_X), 1}, by{c->ddesc, pf + pf_off(1, PF_Y), 1},
      bz{c->ddesc, pf + pf_off(1, PF_Z), 1}, bix{c->ddesc, pf + pf_off(1, PF_IX), 1},
      bmx{c->ddesc, pf + pf_off(1, PF_MIX), 1}, bdot{c->ddesc, pf + pf_off(1, PF_DOT), 1};
  const int *ixc = pf + pf_off(1, PF_IXC), *dotc = pf + pf_off(1, PF_DOTC);
  // keep t: the kernels below run out of sequence and overwrite it
  void *tsave = nullptr;
  const size_t tb = (size_t)d.n * d.Ns * sizeof(T);
  CK(pool_alloc(c->opts.device, &tsave, tb, s));
  CK(cudaMemcpyAsync(tsave, c->t, tb, cudaMemcpyDeviceToDevice, s));
  Ctl h;
  int rc = read_ctl(c, h);
  if (rc) return rc;
  const bool dots = c->mixer == MIX_AN2 && h.count_left <= 0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int k = 0;
  auto timed = [&](const char *name, double b, auto &&launch) -> int {
    launch();  // warm
    CK(cudaEventRecord(e0, s));
    for (int i = 0; i < reps; ++i) launch();
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    if (k < 16) {
      ms[k] = t / reps;
      bytes[k] = b;
      names += (k ? "," : "") + std::string(name);
    }
    ++k;
    return R3D_OK;
  };
  const double cref = d.cref ? rs : 0.0;
  if (c->geo.mfx) {
    // the mix fused into FX: t, u, c_ref, and (mixing) the residual and the
    // four history rows in; t, its two history entries, g and w out
    const bool mixing = h.mix_flag != 0, picard = h.coef[2] < 0;
    const double mixb = !mixing ? 0.0 : picard ? rs + ts + 2 * rs : 5 * rs + ts + 2 * rs;
    timed("mix_fx", n * N * (ts + rs + cref + rs + ts + mixb),
          [&] { pass_fx<P>(d, c->geo, bx, s, 1, nullptr, 1); });
  } else {
    // FX: t, u, c_ref in; w (half spectrum: one grid value per voxel) and g out
    timed("fwd_x", n * N * (ts + rs + cref + rs + ts),
          [&] { pass_fx<P>(d, c->geo, bx, s, 1, nullptr); });
  }
  timed("fft_y_fwd", n * N * 2 * rs,
        [&] { pass_fy_iter<P>(d, c->geo, by, s, -1); });
  timed("zoz", n * N * 2 * rs + (double)d.Nh * 4,
        [&] { pass_zoz_iter<P>(d, c->geo, bz, s); });
  timed("fft_y_inv", n * N * 2 * rs,
        [&] { pass_fy_iter<P>(d, c->geo, by, s, 1); });
  // IX: w, g, lr (and the two AN2 residual slots) in; R out
  timed("inv_x", n * N * (rs + ts + rs + rs + (dots ? 2 * rs : 0)),
        [&] { pass_ix<P>(d, c->geo, bix, s, 1, nullptr); });
  if (c->mixer == MIX_AN2) {
    timed("reduce", (double)iter_ix_ctas(c->geo) * kPartials * 8,
          [&] { launch_reduce(c->ddesc, ixc, 1, 1, s); });
    const bool picard = h.count_left > 0;
    const bool diffs = rs < ts;  // mixed: FP32 t differences in the slots
    if (!c->geo.mfx)
      timed("mix_an2", picard ? n * N * (diffs ? 2 * ts + 3 * rs : 3 * ts + 2 * rs)
                              : n * N * (diffs ? 2 * ts + 7 * rs : 5 * ts + 4 * rs),
            [&] { launch_mix_an2<P>(bmx, c->geo.mix_ctas, s); });
  } else {
    timed("anm_dots", n * N * rs * (h.hcount + 1),
          [&] { launch_anm<P>(bdot, c->geo.dot_ctas, c->ddesc, dotc, 1, s, 0); });
    timed("reduce", (double)iter_ix_ctas(c->geo) * kPartials * 8,
          [&] { launch_reduce(c->ddesc, ixc, 1, 1, s); });
    timed("anm_coef", 0, [&] { launch_anm<P>(bmx, c->geo.mix_ctas, c->ddesc, dotc, 1, s, 1); });
    const int m = std::min(h.hcount, c->history);
    // FP64: R_k, t_k, m z entries in; R_k, z_k, t out.  Mixed: R_k, t_k, the
    // last t difference, R_{k-1}, m - 1 z differences in; R_k, the new z
    // difference, the t difference and t out
    timed("mix_anm", rs < ts ? n * N * (rs + ts + rs + rs + (m - 1) * rs + rs + rs + rs + ts)
                             : n * N * (rs + ts + m * ts + rs + ts + ts),
          [&] { launch_anm<P>(bmx, c->geo.mix_ctas, c->ddesc, dotc, 1, s, 2); });
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->t, tsave, tb, cudaMemcpyDeviceToDevice, s));
  CK(cudaStreamSynchronize(s));
  cudaFreeAsync(tsave, s);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *nk = std::min(k, 16);
  return reset_mixer(c);
}

extern "C" int r3d_profile_kernels(r3d_ctx *c, int reps, char *names, int len,
                                   double *ms, double *bytes, int *nk) {
  if (!c || !ms || !bytes || !nk || reps < 1) return fail(c, R3D_EINVAL, "bad arguments");
  if (!c->initialized) return fail(c, R3D_ESTATE, "profile before initialize");
  CK(cudaSetDevice(c->opts.device));
  std::string nm;
  int rc = c->fp64 ? profile_typed<P64>(c, reps, nm, ms, bytes, nk)
                   : profile_typed<PMix>(c, reps, nm, ms, bytes, nk);
  if (names && len > 0) {
    std::strncpy(names, nm.c_str(), (size_t)len - 1);
    names[len - 1] = 0;
  }
  return rc;
}

extern "C" int r3d_status(r3d_ctx *c, int *steps, double *rms, int *status) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "status before initialize");
  CK(cudaSetDevice(c->opts.device));
  Ctl h;
  int rc = read_ctl(c, h);
  if (rc) return rc;
  if (steps) *steps = h.step;
  if (rms) *rms = h.rms;
  if (status)
    *status = h.status == RUNNING ? -1
              : h.status == CONVERGED ? R3D_CONVERGED
              : h.status == DIVERGED ? R3D_DIVERGED : R3D_MAXSTEP;
  return R3D_OK;
}

extern "C" int r3d_transfer_bytes(const r3d_ctx *c, unsigned long long *h2d,
                                  unsigned long long *d2h) {
  if (!c) return R3D_EINVAL;
  if (h2d) *h2d = c->h2d;
  if (d2h) *d2h = c->d2h;
  return R3D_OK;
}

extern "C" int r3d_write_tuv(r3d_ctx *c, const char *path);

extern "C" int r3d_iterate(r3d_ctx *c, int *steps, double *rms, int *status) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "iterate before initialize");
  CK(cudaSetDevice(c->opts.device));
  cudaStream_t s = c->stream;
  // AN2::initialize inside iterate (iterate.cu:39): fresh mixer state
  {
    Ctl h{};
    h.status = RUNNING;
    h.maxstep = c->prob.maxstep;
    h.tol = c->prob.convergence;
    h.count_left = c->prob.count;
    CK(copy_h2d(c, c->ctl, &h, sizeof(Ctl), s));
  }
  int grc = ensure_graph(c);
  if (grc) return grc;
  if (c->opts.verbose) std::printf("relaxing 3D UV RISM:\n");
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, s));
  Ctl h{};
  int printed = 0;
  std::vector<double> log;
  c->next_refresh = c->refresh_first;
  const int ksave = c->prob.ksave;  // iterate.cu:63-70: save t every ksave steps / at the end
  for (;;) {
    // chunks end on the multiples of ksave, where t is saved
    const int chunk = ksave > 0 ? std::min(8, ksave - h.step % ksave) : 8;
    for (int i = 0; i < chunk; ++i) CK(cudaGraphLaunch(c->gexec, s));
    int rc = read_ctl(c, h);
    if (rc) return rc;
    if (ksave > 0 && h.status == RUNNING && h.step % ksave == 0 &&
        (rc = r3d_write_tuv(c, nullptr)))
      return rc;
    if (!c->fp64 && h.status == RUNNING && h.rms < c->next_refresh) {
      // mixed path: move the converged part of c into the FP64 reference
      if ((rc = refresh<PMix>(c, false))) return rc;
      c->next_refresh *= c->refresh_factor;
    }
    if (c->opts.verbose && h.step > printed) {
      log.resize(h.step);
      CK(copy_d2h(c, log.data(), c->desc.rmslog, sizeof(double) * h.step, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      for (int i = printed; i < h.step; ++i)
        std::printf(" Step = %d Reside = %g\n", i + 1, log[i]);
      printed = h.step;
    }
    if (h.status != RUNNING) break;
  }
  CK(cudaEventRecord(e1, s));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->ms_per_iter = h.step > 0 ? ms / h.step : 0;
  int st = h.status == CONVERGED ? R3D_CONVERGED
                                 : (h.status == DIVERGED ? R3D_DIVERGED : R3D_MAXSTEP);
  if (ksave != 0 && st == R3D_CONVERGED) {
    int rc = r3d_write_tuv(c, nullptr);
    if (rc) return rc;
  }
  if (c->opts.verbose) {
    if (st == R3D_DIVERGED)
      std::printf("Calculation diverged.\n");
    else if (st == R3D_MAXSTEP)
      std::printf("3D UV RISM: reached limit # of relaxation steps: %d\n", c->prob.maxstep);
  }
  if (steps) *steps = h.step;
  if (rms) *rms = h.rms;
  if (status) *status = st;
  return R3D_OK;
}

// ------------------------------------------------------------ read-back
// Grid of t that produced the last residual: t itself, unless the last step
// also mixed (maxstep reached), in which case AN2 left the old t in its
// history slot (anderson_cuda.cu:11-22) -- in the mixed path as the FP32
// difference to the new t, so the old t is rebuilt into a buffer of its own.
static int t_of_residual(r3d_ctx *c, const Ctl &h, const void **out) {
  *out = c->t;
  if (h.status == MAXSTEP && h.mix_flag && c->mixer == MIX_AN2) {
    const long long niv = (long long)c->desc.n * c->desc.Ns;
    if (c->fp64) {
      *out = (const char *)c->hist_a + (size_t)h.coef[3] * niv * sizeof(double);
      return R3D_OK;
    }
    if (!c->tbuf) {
      int rc = dalloc(c, &c->tbuf, (size_t)niv * sizeof(double));
      if (rc) return rc;
    }
    launch_t_restore(c->t, (const char *)c->hist_a + (size_t)h.coef[3] * niv * sizeof(float),
                     c->tbuf, niv, c->stream);
    CK(cudaGetLastError());
    *out = c->tbuf;
  }
  return R3D_OK;
}

// Device -> caller host memory (pageable, as a numpy array is) through two
// pinned staging chunks: the DMA of chunk i + 1 runs while chunk i is copied
// from its staging buffer to the destination, split over several host
// threads (which also share the first-touch page faults of a fresh
// destination).  A direct pageable copy of a 256^3 x 4-site FP64 grid went
// through the driver's own staging at a fraction of the link's rate.
constexpr size_t kPinChunk = 32u << 20;
static int copy_out(r3d_ctx *c, void *host, const void *dsrc, size_t bytes, cudaStream_t s) {
  if (bytes < (4u << 20)) {  // small: one ordinary copy
    CK(copy_d2h(c, host, dsrc, bytes, s));
    CK(cudaStreamSynchronize(s));
    return R3D_OK;
  }
  for (int k = 0; k < 2; ++k) {
    if (!c->pin[k]) CK(cudaMallocHost(&c->pin[k], kPinChunk));
    if (!c->pin_ev[k]) CK(cudaEventCreateWithFlags(&c->pin_ev[k], cudaEventDisableTiming));
  }
  const size_t n = (bytes + kPinChunk - 1) / kPinChunk;
  const int nt = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  auto dma = [&](size_t i) -> cudaError_t {
    const size_t off = i * kPinChunk, len = std::min(kPinChunk, bytes - off);
    cudaError_t e = cudaMemcpyAsync(c->pin[i & 1], (const char *)dsrc + off, len,
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(c->pin_ev[i & 1], s);
    return e;
  };
  CK(dma(0));
  for (size_t i = 0; i < n; ++i) {
    // chunk i + 1 into the other buffer, whose previous chunk (i - 1) has
    // already been copied out
    if (i + 1 < n) CK(dma(i + 1));
    CK(cudaEventSynchronize(c->pin_ev[i & 1]));
    const size_t off = i * kPinChunk, len = std::min(kPinChunk, bytes - off);
    const char *src = (const char *)c->pin[i & 1];
    char *dst = (char *)host + off;
    const size_t part = (len / nt + 63) / 64 * 64;
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) {
      const size_t a = std::min(len, t * part), b = std::min(len, (t + 1) * part);
      if (a < b) th.emplace_back([=] { std::memcpy(dst + a, src + a, b - a); });
    }
    std::memcpy(dst, src, std::min(len, part));
    for (auto &x : th) x.join();
  }
  c->d2h += bytes;
  return R3D_OK;
}

static int ensure_scratch(r3d_ctx *c, size_t bytes) {
  if (c->scratch_bytes >= bytes) return R3D_OK;
  if (c->scratch) {
    cudaFreeAsync(c->scratch, c->stream);
    c->allocs.erase(std::find(c->allocs.begin(), c->allocs.end(), (void *)c->scratch));
    c->bytes -= c->scratch_bytes;
  }
  c->scratch = nullptr;
  c->scratch_bytes = 0;
  int rc = dalloc(c, (void **)&c->scratch, bytes);
  if (rc) return rc;
  c->scratch_bytes = bytes;
  return R3D_OK;
}

extern "C" int r3d_thermo(r3d_ctx *c, double *xmu, double *xmu2, double *pmv,
                          double *pressure) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "thermo before initialize");
  CK(cudaSetDevice(c->opts.device));
  const Desc &d = c->desc;
  const int ctas = 2 * kNumSM;
  int rc = ensure_scratch(c, (size_t)ctas * d.n * 4 * 8);
  if (rc) return rc;
  Ctl h;
  if ((rc = read_ctl(c, h))) return rc;
  const void *tg = nullptr;
  if ((rc = t_of_residual(c, h, &tg))) return rc;
  if (c->fp64)
    launch_thermo<P64>(d, tg, c->scratch, ctas, c->stream);
  else
    launch_thermo<PMix>(d, tg, c->scratch, ctas, c->stream);
  CK(cudaGetLastError());
  std::vector<double> part((size_t)ctas * d.n * 4);
  CK(copy_d2h(c, part.data(), c->scratch, part.size() * 8, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const Problem &p = c->prob;
  const double dv = p.box[0] * p.box[1] * p.box[2] / (double)d.N;
  double cuv = 0;
  for (int v = 0; v < d.n; ++v) {
    double s[4] = {0, 0, 0, 0};
    for (int k = 0; k < ctas; ++k)
      for (int j = 0; j < 4; ++j) s[j] += part[((size_t)k * d.n + v) * 4 + j];
    if (xmu) {
      xmu[v] = s[0] * p.rhov[v] * dv;
      xmu[d.n + v] = s[2] * p.rhov[v] * dv;
    }
    if (xmu2) xmu2[v] = s[1] * p.rhov[v] * dv;
    cuv += s[3] * p.rhov[v];
  }
  cuv *= dv;
  const double ibeta = phys::avogadro * phys::boltzmann * p.temper;
  if (pmv) *pmv = p.xt * (1.0 - cuv) * ibeta;  // cal_pmv.cu:19-23
  double pr = 0;
  for (int v = 0; v < d.n; ++v) pr += p.rhov[v];  // cal_pressure.cu:8-19
  pr *= 1.0e30 / phys::avogadro;
  if (pressure) *pressure = 0.5 * (pr + 1.0 / (p.xt * ibeta));
  return R3D_OK;
}

extern "C" int r3d_write_xmu(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  const int n = c->prob.natv;
  std::vector<double> xmu(2 * n), xmu2(n);
  double pmv, pr;
  int rc = r3d_thermo(c, xmu.data(), xmu2.data(), &pmv, &pr);
  if (rc) return rc;
  std::string out = path ? path : c->prob.fname + (c->prob.zero ? ".xmu0" : ".xmu");
  std::string m = write_xmu(c->prob, xmu.data(), xmu2.data(), pmv, pr, out);
  if (!m.empty()) return fail(c, R3D_EIO, m);
  return R3D_OK;
}

extern "C" int r3d_get_grid(r3d_ctx *c, int which, double *host) {
  if (!c || !host) return fail(c, R3D_EINVAL, "ctx or host is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "get_grid before initialize");
  CK(cudaSetDevice(c->opts.device));
  const Desc &d = c->desc;
  const long long niv = (long long)d.n * d.N;
  cudaStream_t s = c->stream;
  long long count = 0;
  int rc;
  Ctl h;
  if ((rc = read_ctl(c, h))) return rc;
  switch (which) {
    case R3D_GRID_U: case R3D_GRID_T: {  // short-range part + q_v phi_L(r)
      const void *src = which == R3D_GRID_U ? c->u : c->t;
      count = niv;
      if ((rc = ensure_scratch(c, count * 8))) return rc;
      const int x = which == R3D_GRID_T ? 1 : 0;
      if (c->fp64)
        launch_shift_qfr<P64>(d, src, c->scratch, 1.0, x, s);
      else
        launch_shift_qfr<PMix>(d, src, c->scratch, 1.0, x, s);
      break;
    }
    case R3D_GRID_R: {  // site-strided -> dense
      count = niv;
      if ((rc = ensure_scratch(c, count * 8))) return rc;
      if (c->fp64)
        launch_shift_qfr<P64>(d, c->res, c->scratch, 0.0, 0, s);
      else
        launch_shift_qfr<PMix>(d, c->res, c->scratch, 0.0, 0, s);
      break;
    }
    case R3D_GRID_FR: {
      count = d.N;
      if ((rc = ensure_scratch(c, count * 8))) return rc;
      if (c->fp64)
        launch_to_double<P64>(c->fr, c->scratch, count, 0, s);
      else
        launch_to_double<PMix>(c->fr, c->scratch, count, 0, s);
      break;
    }
    case R3D_GRID_G: case R3D_GRID_H: {
      count = niv;
      if ((rc = ensure_scratch(c, count * 8))) return rc;
      const void *tg = nullptr;
  if ((rc = t_of_residual(c, h, &tg))) return rc;
      double *g = which == R3D_GRID_G ? c->scratch : nullptr;
      double *hh = which == R3D_GRID_H ? c->scratch : nullptr;
      if (c->fp64)
        launch_gh<P64>(d, tg, g, hh, s);
      else
        launch_gh<PMix>(d, tg, g, hh, s);
      break;
    }
    case R3D_GRID_FK: case R3D_GRID_FKT: {
      count = 2 * d.Nh;
      if ((rc = ensure_scratch(c, count * 8))) return rc;
      launch_to_double<P64>(c->fk, c->scratch, count, 0, s);  // FP64 always
      break;
    }
    case R3D_GRID_CHI: {  // the shell table (FP64, times 2/N) through each point's shell
      const int n = d.n, chis = d.chis;
      std::vector<uint32_t> kidx((size_t)d.Nh);
      std::vector<double> tab((size_t)c->nshell * chis);
      CK(copy_d2h(c, kidx.data(), c->kidx, kidx.size() * 4, s));
      CK(copy_d2h(c, tab.data(), c->chi64, tab.size() * 8, s));
      CK(cudaStreamSynchronize(s));
      const double un = (double)d.N / 2.0;
      for (int q = 0; q < n * n; ++q)
        for (long long i = 0; i < d.Nh; ++i)
          host[(size_t)q * d.Nh + i] = tab[(size_t)kidx[i] * chis + q] * un;
      return R3D_OK;
    }
    default:
      return fail(c, R3D_EINVAL, "unknown grid");
  }
  CK(cudaGetLastError());
  if ((rc = copy_out(c, host, c->scratch, count * 8, s))) return rc;
  if (which == R3D_GRID_FK) {  // transform units -> physical beta phi_L(k)
    const Problem &p = c->prob;
    const double dv = p.box[0] * p.box[1] * p.box[2] / (double)d.N;
    const int par0 = ((d.nx + d.ny + d.nz) / 2) & 1;
    for (long long i = 0; i < d.Nh; ++i) {
      int pp = (int)(i % d.hx), y = (int)((i / d.hx) % d.ny), z = (int)(i / ((long long)d.hx * d.ny));
      double sg = ((2 * pp + y + z + par0) & 1) ? -1.0 : 1.0;
      double a = host[2 * i], b = host[2 * i + 1];
      // F = dv * C * raw, C = -i sigma:  (a + ib)(-i) = b - i a
      host[2 * i] = dv * sg * b;
      host[2 * i + 1] = -dv * sg * a;
    }
  }
  return R3D_OK;
}

extern "C" int r3d_set_t(r3d_ctx *c, const double *host) {
  if (!c || !host) return fail(c, R3D_EINVAL, "ctx or host is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "set_t before initialize");
  CK(cudaSetDevice(c->opts.device));
  const long long niv = (long long)c->desc.n * c->desc.N;
  int rc = ensure_scratch(c, niv * 8);
  if (rc) return rc;
  CK(copy_h2d(c, c->scratch, host, niv * 8, c->stream));
  if (c->fp64)
    launch_set_short<P64>(c->desc, c->scratch, c->t, c->stream);
  else
    launch_set_short<PMix>(c->desc, c->scratch, c->t, c->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return R3D_OK;
}

// ------------------------------------------------------------ grid files
static int grid_host(r3d_ctx *c, int which, std::vector<double> &v) {
  v.resize((size_t)c->desc.n * c->desc.N);
  return r3d_get_grid(c, which, v.data());
}
static std::string out_path(const r3d_ctx *c, const char *path, const char *ext) {
  return path ? std::string(path) : c->prob.fname + ext;
}

extern "C" int r3d_write_guv(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> g;
  int rc = grid_host(c, R3D_GRID_G, g);
  if (rc) return rc;
  std::string m = write_guv(c->prob, g.data(), out_path(c, path, ".guv"));
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_write_huv(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> h;
  int rc = grid_host(c, R3D_GRID_H, h);
  if (rc) return rc;
  std::string m = write_grid_text(c->prob, h.data(), out_path(c, path, ".huv0"));
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_write_cuv(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> h, t;
  int rc = grid_host(c, R3D_GRID_H, h);
  if (!rc) rc = grid_host(c, R3D_GRID_T, t);
  if (rc) return rc;
  for (size_t i = 0; i < h.size(); ++i) h[i] -= t[i];  // c = h - t
  std::string m = write_grid_text(c->prob, h.data(), out_path(c, path, ".cuv0"));
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_write_tuv(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> t;
  int rc = grid_host(c, R3D_GRID_T, t);
  if (rc) return rc;
  std::string m = write_tuv(c->prob, t.data(), out_path(c, path, ".tuv"));
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_read_tuv(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "read_tuv before initialize");
  std::vector<double> t((size_t)c->desc.n * c->desc.N);
  std::string m = read_tuv(c->prob, t.data(), out_path(c, path, ".tuv"));
  if (!m.empty()) return fail(c, R3D_EIO, m);
  return r3d_set_t(c, t.data());
}

// ------------------------------------------------ per-atom integrals
// cal_grad.cu, cal_euv.cu, cal_ad1.cu / cal_ad2.cu over g of the solve, in
// the units of their files: grad [nu][3] kcal/(mol A), euv [nu][natv] J/mol,
// ad [nu] kcal/mol (ad: the LJ lambda derivative after set_ad(lambda, 1),
// else the Coulomb one).  Any output may be NULL.
extern "C" int r3d_atom_integrals(r3d_ctx *c, double *grad, double *euv, double *ad) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  if (!c->initialized) return fail(c, R3D_ESTATE, "atom integrals before initialize");
  CK(cudaSetDevice(c->opts.device));
  const Problem &p = c->prob;
  const Desc &d = c->desc;
  const int nu = (int)p.q.size(), n = p.natv;
  const long long N = d.N, niv = (long long)n * N;
  cudaStream_t s = c->stream;
  Ctl h;
  int rc = read_ctl(c, h);
  if (rc) return rc;
  if ((rc = ensure_scratch(c, niv * 8))) return rc;  // g, FP64
  const void *tg = nullptr;
  if ((rc = t_of_residual(c, h, &tg))) return rc;
  if (c->fp64)
    launch_gh<P64>(d, tg, c->scratch, nullptr, s);
  else
    launch_gh<PMix>(d, tg, c->scratch, nullptr, s);
  const double lambda1 = p.adswitch == 1 ? p.lambda : 1.0;
  std::vector<double> tab((size_t)nu * (4 + 2 * n));
  for (int a = 0; a < nu; ++a) {
    tab[a] = p.r[3 * a];
    tab[nu + a] = p.r[3 * a + 1];
    tab[2 * nu + a] = p.r[3 * a + 2];
    tab[3 * nu + a] = p.q[a];
    for (int v = 0; v < n; ++v) {  // cal_LJ.cu:30-40
      tab[(size_t)(4 + v) * nu + a] = (p.sig[a] + p.sigv[v]) * 0.5 * lambda1;
      tab[(size_t)(4 + n + v) * nu + a] = std::sqrt(p.eps[a] * p.epsv[v]);
    }
  }
  const int nchunk = (int)std::max<long long>(1, std::min<long long>(256, N / 4096));
  const long long nk = (long long)nu * (4 + n);
  double *buf = nullptr;
  const size_t bytes = (tab.size() + (size_t)nchunk * nk + nk) * sizeof(double);
  CK(pool_alloc(c->opts.device, (void **)&buf, std::max<size_t>(bytes, 16), s));
  double *dtab = buf, *part = buf + tab.size(), *out = part + (size_t)nchunk * nk;
  int rcc = R3D_OK;
  std::vector<double> host(nk);
  if (nu > 0) {
    cudaError_t e = cudaMemcpyAsync(dtab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, s);
    IntAtoms at{};
    at.x = dtab;
    at.y = dtab + nu;
    at.z = dtab + 2 * nu;
    at.q = dtab + 3 * nu;
    at.sig = dtab + 4 * (size_t)nu;
    at.eps = dtab + (size_t)(4 + n) * nu;
    for (int v = 0; v < n; ++v) {
      at.qv[v] = p.qv[v];
      at.rhov[v] = p.rhov[v];
    }
    at.nu = nu;
    at.n = n;
    at.ad1 = p.adswitch == 1;
    at.lambda = p.lambda;
    at.cc = phys::hartree * phys::bohr * phys::avogadro;
    const double dr[3] = {p.box[0] / d.nx, p.box[1] / d.ny, p.box[2] / d.nz};
    if (e == cudaSuccess) {
      launch_atom_integrals(at, c->scratch, N, p.grid, dr, part, nchunk, out, s);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), out, nk * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rcc = fail(c, R3D_ECUDA, cudaGetErrorString(e));
    c->d2h += nk * 8;
    c->h2d += tab.size() * 8;
  }
  cudaFreeAsync(buf, s);
  if (rcc) return rcc;
  const double dv = p.box[0] * p.box[1] * p.box[2] / (double)N, kcal2J = 4184.0;
  for (int a = 0; a < nu; ++a) {
    const double *o = host.data() + (size_t)a * (4 + n);
    if (grad)
      for (int k = 0; k < 3; ++k) grad[3 * a + k] = o[k] * dv / kcal2J;
    if (ad) ad[a] = o[3] * dv / kcal2J;
    if (euv)
      for (int v = 0; v < n; ++v) euv[(size_t)a * n + v] = o[4 + v] * dv;
  }
  return R3D_OK;
}

extern "C" int r3d_write_gra(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> g(3 * c->prob.q.size());
  int rc = r3d_atom_integrals(c, g.data(), nullptr, nullptr);
  if (rc) return rc;
  std::string m = write_atom_file(c->prob, 'd', g.data(), out_path(c, path, ".gra"));
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_write_euv(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> e(c->prob.q.size() * c->prob.natv);
  int rc = r3d_atom_integrals(c, nullptr, e.data(), nullptr);
  if (rc) return rc;
  std::string m = write_atom_file(c->prob, 'b', e.data(), out_path(c, path, ".euv"));
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_write_ad(r3d_ctx *c, const char *path) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::vector<double> v(c->prob.q.size());
  int rc = r3d_atom_integrals(c, nullptr, nullptr, v.data());
  if (rc) return rc;
  std::ostringstream nm;  // output_ad.cu: <stem>-<adswitch>-<lambda>
  nm << c->prob.fname << "-" << c->prob.adswitch << "-" << c->prob.lambda;
  std::string m = write_atom_file(c->prob, 'a', v.data(), path ? std::string(path) : nm.str());
  return m.empty() ? R3D_OK : fail(c, R3D_EIO, m);
}

extern "C" int r3d_output(r3d_ctx *c, const char *outlist) {
  if (!c) return fail(c, R3D_EINVAL, "ctx is NULL");
  std::string ol = outlist ? outlist : c->prob.outlist;
  std::transform(ol.begin(), ol.end(), ol.begin(), ::tolower);
  int rc = R3D_OK;  // output.cu's order: m, d, c, g, h, a, b
  if (ol.find('m') != std::string::npos) rc = r3d_write_xmu(c, nullptr);
  if (!rc && ol.find('d') != std::string::npos) rc = r3d_write_gra(c, nullptr);
  if (!rc && ol.find('c') != std::string::npos) rc = r3d_write_cuv(c, nullptr);
  if (!rc && ol.find('g') != std::string::npos) rc = r3d_write_guv(c, nullptr);
  if (!rc && ol.find('h') != std::string::npos) rc = r3d_write_huv(c, nullptr);
  if (!rc && ol.find('a') != std::string::npos) rc = r3d_write_ad(c, nullptr);
  if (!rc && ol.find('b') != std::string::npos) rc = r3d_write_euv(c, nullptr);
  return rc;
}

extern "C" int r3d_info(const r3d_ctx *c, int *grid3, int *natv, long long *ngrid, int *nu) {
  if (!c) return R3D_EINVAL;
  if (grid3)
    for (int d = 0; d < 3; ++d) grid3[d] = c->prob.grid[d];
  if (natv) *natv = c->prob.natv;
  if (ngrid) *ngrid = (long long)c->prob.grid[0] * c->prob.grid[1] * c->prob.grid[2];
  if (nu) *nu = (int)c->prob.q.size();
  return R3D_OK;
}

extern "C" int r3d_solvent_sites(const r3d_ctx *c, double *qv, double *rhov) {
  if (!c || !qv || !rhov) return fail(nullptr, R3D_EINVAL, "bad arguments");
  if (!c->prob.has_solvent) return fail(nullptr, R3D_ESTATE, "no solvent loaded");
  for (int v = 0; v < c->prob.natv; ++v) {
    qv[v] = c->prob.qv[v];
    rhov[v] = c->prob.rhov[v];
  }
  return R3D_OK;
}

extern "C" int r3d_device_bytes(const r3d_ctx *c, unsigned long long *bytes) {
  if (!c || !bytes) return R3D_EINVAL;
  if (c->initialized) {
    *bytes = c->bytes;
    return R3D_OK;
  }
  r3d_ctx tmp = *c;
  tmp.allocs.clear();
  Desc d{};
  if (plan_geometry(&tmp, d)) return R3D_EINVAL;
  long long smax = 3LL * (d.nx - 1) * (d.nx - 1);
  int nshell = (int)std::min<long long>((smax - 3) / 8 + 1, d.Nh);
  *bytes = plan_bytes(&tmp, d, nshell);
  return R3D_OK;
}

extern "C" int r3d_iter_timing(const r3d_ctx *c, double *ms, int *kernels) {
  if (!c) return R3D_EINVAL;
  if (ms) *ms = c->ms_per_iter;
  if (kernels) *kernels = c->kernels_per_iter;
  return R3D_OK;
}

// ---------------------------------------------------------- fft3d seam
template <typename P>
static int fft_typed(r3d_ctx *c, int nx, int ny, int nz, const double *box, int dir,
                     const double *in, double *out) {
  using R = typename P::R;
  Desc &d = c->desc;
  cudaStream_t s = c->stream;
  const long long N = d.N, Nh = d.Nh;
  int rc;
  void *src, *w, *ctl, *ddesc, *pre, *hbuf;
  if ((rc = dalloc(c, &src, N * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &w, Nh * 2 * sizeof(R)))) return rc;
  if ((rc = dalloc(c, &ctl, sizeof(Ctl)))) return rc;
  if ((rc = dalloc(c, &ddesc, sizeof(Desc)))) return rc;
  if ((rc = dalloc(c, &pre, 16 * sizeof(int)))) return rc;
  if ((rc = dalloc(c, &hbuf, std::max(N, 2 * Nh) * 8))) return rc;
  CK(cudaMemsetAsync(ctl, 0, sizeof(Ctl), s));
  d.w = w;
  d.ctl = (Ctl *)ctl;
  void *t64 = nullptr, *t32 = nullptr;
  if ((rc = make_twiddles(c, d, c->fp64, &t64, &t32))) return rc;
  CK(copy_h2d(c, ddesc, &d, sizeof(Desc), s));
  int pf[16] = {0, c->geo.tiles_x, 0, c->geo.tiles_y, 0, c->geo.tiles_z, 0, c->geo.ix_ctas};
  CK(copy_h2d(c, pre, pf, sizeof(pf), s));
  const int *dp = (const int *)pre;
  Batch bx{(Desc *)ddesc, dp, 1}, by{(Desc *)ddesc, dp + 2, 1}, bz{(Desc *)ddesc, dp + 4, 1},
      bix{(Desc *)ddesc, dp + 6, 1};
  kernels_set_smem(c->fp64, kSmemMax);
  const double dv = box[0] * box[1] * box[2] / (double)N;
  const int par0 = ((nx + ny + nz) / 2) & 1;
  std::vector<double> tmp(std::max(N, 2 * Nh));
  if (dir < 0) {
    CK(copy_h2d(c, hbuf, in, N * 8, s));
    launch_from_double<P>((const double *)hbuf, src, N, 0, s);
    pass_fx<P>(d, c->geo, bx, s, 0, src);
    pass_fy<P>(d, c->geo, by, s, -1, 0);
    pass_zoz<P>(d, c->geo, bz, s, 0, 0);
    launch_to_double<P>(w, (double *)hbuf, 2 * Nh, 0, s);
    CK(cudaGetLastError());
    CK(copy_d2h(c, out, hbuf, 2 * Nh * 8, s));
    CK(cudaStreamSynchronize(s));
    for (long long i = 0; i < Nh; ++i) {
      int pp = (int)(i % d.hx), y = (int)((i / d.hx) % ny), z = (int)(i / ((long long)d.hx * ny));
      double sg = ((2 * pp + y + z + par0) & 1) ? -1.0 : 1.0;
      double a = out[2 * i], b = out[2 * i + 1];
      out[2 * i] = dv * sg * b;  // dv * (-i sigma) * (a + i b)
      out[2 * i + 1] = -dv * sg * a;
    }
  } else {
    for (long long i = 0; i < Nh; ++i) {
      int pp = (int)(i % d.hx), y = (int)((i / d.hx) % ny), z = (int)(i / ((long long)d.hx * ny));
      double sg = ((2 * pp + y + z + par0) & 1) ? -1.0 : 1.0;
      double a = in[2 * i], b = in[2 * i + 1];
      // raw = F conj(C) / dv = F (i sigma) / dv
      tmp[2 * i] = -b * sg / dv;
      tmp[2 * i + 1] = a * sg / dv;
    }
    CK(copy_h2d(c, hbuf, tmp.data(), 2 * Nh * 8, s));
    launch_from_double<P>((const double *)hbuf, w, 2 * Nh, 0, s);
    pass_zoz<P>(d, c->geo, bz, s, 1, 0);
    pass_fy<P>(d, c->geo, by, s, 1, 0);
    pass_ix<P>(d, c->geo, bix, s, 0, src);
    launch_to_double<P>(src, (double *)hbuf, N, 0, s);
    CK(cudaGetLastError());
    CK(copy_d2h(c, out, hbuf, N * 8, s));
    CK(cudaStreamSynchronize(s));
    const double sc = 2.0 / (double)N;
    for (long long i = 0; i < N; ++i) out[i] *= sc;
  }
  return R3D_OK;
}

extern "C" int r3d_fft3d(int device, int precision, int nx, int ny, int nz,
                         const double *box, int dir, const double *in, double *out) {
  if (!box || !in || !out || (dir != -1 && dir != 1))
    return fail(nullptr, R3D_EINVAL, "bad fft3d arguments");
  r3d_opts o{};
  o.device = device;
  o.precision = precision;
  r3d_ctx *c = nullptr;
  int rc = r3d_create(&o, &c);
  if (rc) return rc;
  c->prob.grid[0] = nx;
  c->prob.grid[1] = ny;
  c->prob.grid[2] = nz;
  c->prob.natv = 1;
  if (nx < 4 || ny < 2 || nz < 2 || (nx & 1)) {
    r3d_destroy(c);
    return fail(nullptr, R3D_EINVAL, "fft3d: nx must be even >= 4");
  }
  Desc d{};
  rc = plan_geometry(c, d);
  if (!rc) {
    c->desc = d;
    rc = c->fp64 ? fft_typed<P64>(c, nx, ny, nz, box, dir, in, out)
                 : fft_typed<PMix>(c, nx, ny, nz, box, dir, in, out);
  }
  if (rc) g_last_error = c->err;
  r3d_destroy(c);
  return rc;
}

// ----------------------------------------------------------------- batches
// Independent solves iterated together: the solves of one geometry (grid,
// sites, mixer) form a group, each kernel of an iteration covers every solve
// of its group (a CTA finds its solve in the group's prefix block), and one
// CUDA graph holds one iteration of all groups.  Solves that have converged,
// diverged or hit maxstep are skipped by every kernel while the others run.
struct r3d_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<r3d_ctx *> ctxs;
  std::vector<Group> groups;
  std::vector<void *> gmem;    // device blocks of the groups
  std::vector<int> order;      // gathered index -> ctxs index
  std::vector<std::vector<int>> members;  // per group: ctxs indices
  double *dsum = nullptr, *hsum = nullptr;  // gathered control words
  cudaGraphExec_t gexec = nullptr;
  bool dirty = true;
  int kernels_per_iter = 0;
};

static int bfail(int code, const std::string &m) {
  g_last_error = "batch: " + m;
  return code;
}
#define BCK(x)                                                              \
  do {                                                                      \
    cudaError_t e_ = (x);                                                   \
    if (e_ != cudaSuccess) return bfail(R3D_ECUDA, cudaGetErrorString(e_)); \
  } while (0)

static void batch_release(r3d_batch *b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  for (void *p : b->gmem) cudaFree(p);
  b->gmem.clear();
  b->groups.clear();
  if (b->dsum) cudaFree(b->dsum);
  if (b->hsum) cudaFreeHost(b->hsum);
  b->dsum = b->hsum = nullptr;
}

extern "C" int r3d_batch_create(int device, r3d_batch **out) {
  if (!out) return bfail(R3D_EINVAL, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return bfail(R3D_EINVAL, "no such device");
  BCK(cudaSetDevice(device));
  r3d_batch *b = new r3d_batch;
  b->device = device;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return bfail(R3D_ECUDA, "stream");
  }
  *out = b;
  return R3D_OK;
}

extern "C" int r3d_batch_add(r3d_batch *b, r3d_ctx *c) {
  if (!b || !c) return bfail(R3D_EINVAL, "NULL argument");
  if (!c->initialized) return bfail(R3D_ESTATE, "context not initialized");
  if (c->opts.device != b->device) return bfail(R3D_EINVAL, "context on another device");
  if (!b->ctxs.empty() && b->ctxs[0]->fp64 != c->fp64)
    return bfail(R3D_EINVAL, "contexts of one batch must share the precision");
  if (std::find(b->ctxs.begin(), b->ctxs.end(), c) != b->ctxs.end())
    return bfail(R3D_EINVAL, "context already in the batch");
  b->ctxs.push_back(c);
  b->dirty = true;
  return R3D_OK;
}

extern "C" int r3d_batch_destroy(r3d_batch *b) {
  if (!b) return R3D_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_release(b);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return R3D_OK;
}

// Groups, their device blocks and the graph of one iteration.
template <typename P>
static int batch_build(r3d_batch *b) {
  batch_release(b);
  std::vector<std::vector<int>> members;
  std::vector<std::array<long long, 6>> keys;
  for (int i = 0; i < (int)b->ctxs.size(); ++i) {
    const r3d_ctx *c = b->ctxs[i];
    const std::array<long long, 6> key{c->desc.nx, c->desc.ny, c->desc.nz, c->desc.n,
                                       c->mixer, c->mixer == MIX_ANM ? c->history : 0};
    size_t g = std::find(keys.begin(), keys.end(), key) - keys.begin();
    if (g == keys.size()) {
      keys.push_back(key);
      members.emplace_back();
    }
    members[g].push_back(i);
  }
  cudaStream_t s = b->stream;
  b->order.clear();
  b->members = members;
  for (auto &m : members) {
    const int ns = (int)m.size();
    const r3d_ctx *c0 = b->ctxs[m[0]];
    std::vector<Desc> ds(ns);
    for (int i = 0; i < ns; ++i) ds[i] = b->ctxs[m[i]]->desc;
    const std::vector<int> pre = make_prefix(c0->geo, ns);
    const size_t db = ((ns * sizeof(Desc) + 255) / 256) * 256;
    void *mem = nullptr;
    BCK(cudaMalloc(&mem, db + pre.size() * sizeof(int)));
    b->gmem.push_back(mem);
    BCK(cudaMemcpyAsync(mem, ds.data(), ns * sizeof(Desc), cudaMemcpyHostToDevice, s));
    BCK(cudaMemcpyAsync((char *)mem + db, pre.data(), pre.size() * sizeof(int),
                        cudaMemcpyHostToDevice, s));
    b->groups.push_back(Group{c0->desc, c0->geo, (const Desc *)mem,
                              (const int *)((char *)mem + db), ns, c0->mixer});
    for (int i : m) b->order.push_back(i);
  }
  const size_t nsol = b->ctxs.size();
  BCK(cudaMalloc((void **)&b->dsum, nsol * 4 * sizeof(double)));
  BCK(cudaMallocHost((void **)&b->hsum, nsol * 4 * sizeof(double)));
  BCK(cudaStreamSynchronize(s));
  cudaGraph_t g;
  BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int k = 0;
  for (const Group &G : b->groups) k += enqueue_group<P>(G, s, 0);
  BCK(cudaStreamEndCapture(s, &g));
  cudaError_t e = cudaGraphInstantiate(&b->gexec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return bfail(R3D_ECUDA, std::string("graph: ") + cudaGetErrorString(e));
  b->kernels_per_iter = k;
  b->dirty = false;
  return R3D_OK;
}

template <typename P>
static int batch_run(r3d_batch *b, int *iterations, double *ms_out) {
  cudaStream_t s = b->stream;
  // fresh mixer state of every solve (AN2::initialize inside iterate)
  for (r3d_ctx *c : b->ctxs) {
    int rc = reset_mixer(c);
    if (rc) return bfail(rc, c->err);
    c->next_refresh = c->refresh_first;
  }
  if (b->dirty) {
    int rc = batch_build<P>(b);
    if (rc) return rc;
  } else {  // closures and controls may have changed since the last run
    for (size_t g = 0; g < b->groups.size(); ++g) {
      std::vector<Desc> ds;
      for (int i : b->members[g]) ds.push_back(b->ctxs[i]->desc);
      BCK(cudaMemcpyAsync((void *)b->groups[g].ddescs, ds.data(), ds.size() * sizeof(Desc),
                          cudaMemcpyHostToDevice, s));
    }
    BCK(cudaStreamSynchronize(s));
  }
  const int nsol = (int)b->ctxs.size();
  int maxstep = 0;
  for (r3d_ctx *c : b->ctxs) maxstep = std::max(maxstep, c->prob.maxstep);
  cudaEvent_t e0, e1;
  BCK(cudaEventCreate(&e0));
  BCK(cudaEventCreate(&e1));
  BCK(cudaEventRecord(e0, s));
  const int chunk = 8;
  int iters = 0;
  for (;;) {
    for (int i = 0; i < chunk; ++i) BCK(cudaGraphLaunch(b->gexec, s));
    iters += chunk;
    int off = 0;
    for (const Group &G : b->groups) {
      launch_ctl_gather(G.ddescs, G.ns, b->dsum + 4 * off, s);
      off += G.ns;
    }
    BCK(cudaMemcpyAsync(b->hsum, b->dsum, nsol * 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    bool running = false;
    for (int j = 0; j < nsol; ++j) {
      r3d_ctx *c = b->ctxs[b->order[j]];
      const double *w = b->hsum + 4 * j;
      if (w[3] != 0) return bfail(R3D_ECUDA, "a kernel's bounded wait for a staged copy ran out");
      if ((int)w[0] != RUNNING) continue;
      running = true;
      if (!c->fp64 && w[2] < c->next_refresh) {
        // mixed path: move the converged part of c into the FP64 reference
        int rc = refresh<PMix>(c, false);
        if (rc) return bfail(rc, c->err);
        c->next_refresh *= c->refresh_factor;
      }
    }
    if (!running || iters > maxstep + chunk) break;
  }
  BCK(cudaEventRecord(e1, s));
  BCK(cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int most = 0;
  for (int j = 0; j < nsol; ++j) most = std::max(most, (int)b->hsum[4 * j + 1]);
  for (r3d_ctx *c : b->ctxs) c->ms_per_iter = most > 0 ? ms / most : 0;
  if (iterations) *iterations = most;
  if (ms_out) *ms_out = ms;
  return R3D_OK;
}

extern "C" int r3d_batch_iterate(r3d_batch *b, int *iterations, double *ms) {
  if (!b) return bfail(R3D_EINVAL, "batch is NULL");
  if (b->ctxs.empty()) return bfail(R3D_ESTATE, "empty batch");
  BCK(cudaSetDevice(b->device));
  for (r3d_ctx *c : b->ctxs) BCK(cudaStreamSynchronize(c->stream));
  return b->ctxs[0]->fp64 ? batch_run<P64>(b, iterations, ms) : batch_run<PMix>(b, iterations, ms);
}

extern "C" int r3d_batch_info(const r3d_batch *b, int *solves, int *groups, int *kernels_per_iter) {
  if (!b) return bfail(R3D_EINVAL, "batch is NULL");
  if (solves) *solves = (int)b->ctxs.size();
  if (groups) *groups = (int)b->groups.size();
  if (kernels_per_iter) *kernels_per_iter = b->kernels_per_iter;
  return R3D_OK;
}
#include "r3d_server.inc"
