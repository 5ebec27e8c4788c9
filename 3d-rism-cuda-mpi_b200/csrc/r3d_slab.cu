// r3d_slab.cu -- the stages of the shifted 3D transform on one rank's slab
// of a grid split over several GPUs (r3d_slab_transform).
//
// The reference distributes its transform over MPI ranks as 1D cuFFT passes
// and Alltoall transposes of pencils (fft3d.cu:81-163, the decomposition of
// cell.cc:30-48).  Here a grid split over P GPUs is cut in z-slabs (rank r
// owns z-planes [r nz/P, (r+1) nz/P)) for the x and y passes and in y-slabs
// for the z pass; one all-to-all per direction moves the half spectrum
// between the two (slabs.py drives it with NCCL).  This file runs one
// rank's stages on its own device buffers:
//   stage 0  z-slab real grid [nzl][ny][nx] -> packed x and y transforms ->
//            half spectrum [nzl][ny][nx/2]          (d_real in, d_spec out)
//   stage 1  y-slab half spectrum [nz][nyl][nx/2] -> z transform (in place)
//   stage 2  y-slab inverse z transform (in place)
//   stage 3  z-slab half spectrum -> inverse y and x transforms -> real grid
//            (d_spec in, destroyed; d_real out)
// in the transform units of the iteration's passes: unnormalised, the
// checkerboard and half-sample factors inside, the constant phase dv C(k)
// outside (the full-grid seam r3d_fft3d applies it).  The checkerboard sign
// (-1)^(x+y+z) uses the slab's local z, which equals the global z's parity
// when every slab starts on an even plane (the caller's partition).
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/rism3d_b200.h"
#include "r3d_common.cuh"

namespace r3d {
size_t smem_x(int hx, int n, int S, size_t csz);
size_t smem_y(int ny, int P, size_t csz);
size_t smem_z(int nz, int n, int P, size_t csz);
void kernels_set_smem(bool fp64, size_t maxbytes);
template <typename P>
void launch_fwd_x(Batch, int, size_t, cudaStream_t, int, const void *);
template <typename P>
void launch_fft_y(Batch, int, size_t, cudaStream_t, int, int);
template <typename P>
void launch_zoz(Batch, int, size_t, cudaStream_t, int, int);
template <typename P>
void launch_inv_x(Batch, int, size_t, cudaStream_t, int, void *, int);
void set_last_error(const std::string &m);
}  // namespace r3d

using namespace r3d;

namespace {
// per device: a descriptor, a control block and launch prefixes
struct SlabBlock {
  Desc *desc = nullptr;
  Ctl *ctl = nullptr;
  int *pre = nullptr;
};
SlabBlock g_slab[64];
std::mutex g_slab_mu;

int slab_fail(int code, const std::string &m) {
  set_last_error("r3d_slab_transform: " + m);
  return code;
}
}  // namespace

extern "C" int r3d_slab_transform_sites(int device, int stage, int nsites, int nx, int ny,
                                        int nz, double *d_spec, double *d_real, void *stream) {
  if (stage < 0 || stage > 3 || !d_spec || ((stage == 0 || stage == 3) && !d_real) ||
      nsites < 1 || nsites > kMaxSites)
    return slab_fail(R3D_EINVAL, "bad arguments");
  if (nx < 4 || (nx & 1) || ny < 1 || nz < 1 || device < 0 || device >= 64)
    return slab_fail(R3D_EINVAL, "nx must be even and >= 4, ny and nz >= 1");
  const int hx = nx / 2;
  Desc d{};
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.n = nsites;  // sites one after another: [site][slab]
  d.hx = hx;
  d.N = d.Ns = (long long)nx * ny * nz;
  d.Nh = d.Nhs = (long long)hx * ny * nz;
  d.nrad_x = factor_length(hx, d.rad_x);
  d.nrad_y = factor_length(ny, d.rad_y);
  d.nrad_z = factor_length(nz, d.rad_z);
  if (d.nrad_x < 0 || d.nrad_y < 0 || d.nrad_z < 0)
    return slab_fail(R3D_EINVAL, "grid sizes must factor into primes <= 13");
  const size_t cs = sizeof(double2), budget = 100 * 1024;
  // an x tile and a z tile hold every site (their shared memory grows with
  // nsites); a y tile holds one site
  int S = 16;
  while (S > 1 && ((ny * nz) % S || smem_x(hx, nsites, S, cs) > budget)) S >>= 1;
  int Py = 8;
  while (Py > 1 && (hx % Py || smem_y(ny, Py, cs) > budget)) Py >>= 1;
  int Pz = 4;
  while (Pz > 1 && (hx % Pz || smem_z(nz, nsites, Pz, cs) > budget)) Pz >>= 1;
  const size_t smx = smem_x(hx, nsites, S, cs), smy = smem_y(ny, Py, cs),
               smz = smem_z(nz, nsites, Pz, cs);
  if (smx > 220 * 1024 || smy > 220 * 1024 || smz > 220 * 1024)
    return slab_fail(R3D_EINVAL, "slab too large for one CTA's shared memory");
  d.rows = S;
  d.ycols = Py;
  d.zcols = Pz;
  d.tiles_x = (ny * nz) / S;
  d.tiles_y = nsites * nz * (hx / Py);
  d.tiles_z = ny * (hx / Pz);
  d.w = d_spec;

  int caller = -1;
  cudaError_t e = cudaGetDevice(&caller);
  if (e != cudaSuccess) return slab_fail(R3D_ECUDA, cudaGetErrorString(e));
  struct Restore {
    int dev;
    ~Restore() { cudaSetDevice(dev); }
  } restore{caller};
  if ((e = cudaSetDevice(device)) != cudaSuccess) return slab_fail(R3D_ECUDA, cudaGetErrorString(e));
  SlabBlock blk;
  {
    std::lock_guard<std::mutex> lk(g_slab_mu);
    SlabBlock &b = g_slab[device];
    if (!b.desc) {
      void *p = nullptr;
      if ((e = cudaMalloc(&p, sizeof(Desc) + sizeof(Ctl) + 64)) != cudaSuccess)
        return slab_fail(R3D_ENOMEM, cudaGetErrorString(e));
      b.desc = (Desc *)p;
      b.ctl = (Ctl *)((char *)p + sizeof(Desc));
      b.pre = (int *)((char *)p + sizeof(Desc) + sizeof(Ctl));
      kernels_set_smem(true, 220 * 1024);
    }
    blk = b;
  }
  d.ctl = blk.ctl;
  cudaStream_t s = (cudaStream_t)stream;
  const int pf[8] = {0, d.tiles_x, 0, d.tiles_y, 0, d.tiles_z, 0, d.tiles_x};
  Ctl hctl{};
  if ((e = cudaMemcpyAsync(blk.desc, &d, sizeof(Desc), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(blk.ctl, &hctl, sizeof(Ctl), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(blk.pre, pf, sizeof(pf), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return slab_fail(R3D_ECUDA, cudaGetErrorString(e));
  const int *pre = blk.pre;
  Batch bx{blk.desc, pre, 1}, by{blk.desc, pre + 2, 1}, bz{blk.desc, pre + 4, 1},
      bix{blk.desc, pre + 6, 1};
  switch (stage) {
    case 0:
      launch_fwd_x<P64>(bx, d.tiles_x, smx, s, 0, d_real);
      launch_fft_y<P64>(by, d.tiles_y, smy, s, -1, 0);
      break;
    case 1:
      launch_zoz<P64>(bz, d.tiles_z, smz, s, 0, 0);
      break;
    case 2:
      launch_zoz<P64>(bz, d.tiles_z, smz, s, 1, 0);
      break;
    default:
      launch_fft_y<P64>(by, d.tiles_y, smy, s, 1, 0);
      launch_inv_x<P64>(bix, d.tiles_x, smx, s, 0, d_real, 1);
      break;
  }
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return slab_fail(R3D_ECUDA, cudaGetErrorString(e));
  return R3D_OK;
}

extern "C" int r3d_slab_transform(int device, int stage, int nx, int ny, int nz, double *d_spec,
                                  double *d_real, void *stream) {
  return r3d_slab_transform_sites(device, stage, 1, nx, ny, nz, d_spec, d_real, stream);
}
