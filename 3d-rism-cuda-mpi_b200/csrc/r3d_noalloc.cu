// r3d_noalloc.cu -- r3d_fft3d_noalloc: the shifted 3D transform of
// r3d_fft3d on caller-owned device buffers, with no device allocation.
//
// Who needs this: callers that cannot call cudaMalloc -- code that runs
// while another framework owns the device's memory pool (and forbids or
// cannot afford foreign allocations), and real-time loops that must not
// take the allocator's locks or risk an out-of-memory failure in mid-run.
// They pass device pointers for the input and the output; the only working
// storage is the fixed array below, which every GPU that loads this library
// holds until the process exits.
//
// Sharing rules: all calls on a device use the same array and it keeps the
// contents of the last call.  Calls that overlap on the GPU (concurrent
// streams or threads) race on it and must be serialised by the caller.  The
// first call on each device looks up the array's device address (with that
// device current); make that first call before any stream capture.  That
// look-up is made under a lock, so host threads whose first calls coincide
// do not race on it.  The caller's current device is restored on return.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
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
}  // namespace r3d

using namespace r3d;

// The working storage: control words, then the half spectrum.
constexpr size_t kNoallocBytes = (size_t)R3D_NOALLOC_SCRATCH_BYTES;
constexpr size_t round256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kOffCtl = round256(sizeof(Desc));
constexpr size_t kOffPre = kOffCtl + round256(sizeof(Ctl));
constexpr size_t kNoallocHead = 16384;  // Desc + Ctl + launch prefixes
static_assert(kOffPre + 64 <= kNoallocHead, "control words overflow the head");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

namespace r3d {
void set_last_error(const std::string &m);  // r3d_last_error(NULL) reports it
}
// device address of the array, per ordinal (set once, under g_noalloc_mu)
static std::atomic<void *> g_noalloc_ptr[64];
static std::mutex g_noalloc_mu;

static int noalloc_fail(int code, const std::string &m) {
  set_last_error("r3d_fft3d_noalloc: " + m);
  return code;
}

// transform units <-> physical F(k): F = dv * C(k) * raw, C = -i sigma(k)
__global__ void k_noalloc_scale_fwd(const double2 *raw, double *out, long long nh, int hx,
                                    int ny, int par0, double dv) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nh;
       i += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(i % hx), y = (int)((i / hx) % ny), z = (int)(i / ((long long)hx * ny));
    const double sg = ((2 * p + y + z + par0) & 1) ? -1.0 : 1.0;
    const double2 a = raw[i];
    out[2 * i] = dv * sg * a.y;
    out[2 * i + 1] = -dv * sg * a.x;
  }
}
__global__ void k_noalloc_scale_inv_in(const double *in, double2 *raw, long long nh, int hx,
                                       int ny, int par0, double dv) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nh;
       i += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(i % hx), y = (int)((i / hx) % ny), z = (int)(i / ((long long)hx * ny));
    const double sg = ((2 * p + y + z + par0) & 1) ? -1.0 : 1.0;
    raw[i] = make_double2(-in[2 * i + 1] * sg / dv, in[2 * i] * sg / dv);
  }
}
// The descriptor (as plain 8-byte words), a cleared control block and the
// launch prefixes, written from kernel parameters (no host staging buffer is
// involved).
static_assert(sizeof(Desc) % 8 == 0, "descriptor words");
struct DescWords {
  unsigned long long w[sizeof(Desc) / 8];
};
__global__ void k_noalloc_setup(DescWords d, Desc *dd, Ctl *ctl, int4 pa, int4 pb, int *pre) {
  for (int i = threadIdx.x; i < (int)(sizeof(Desc) / 8); i += blockDim.x)
    ((unsigned long long *)dd)[i] = d.w[i];
  for (int i = threadIdx.x; i < (int)(sizeof(Ctl) / sizeof(int)); i += blockDim.x)
    ((int *)ctl)[i] = 0;
  if (threadIdx.x == 0) {
    pre[0] = pa.x, pre[1] = pa.y, pre[2] = pa.z, pre[3] = pa.w;
    pre[4] = pb.x, pre[5] = pb.y, pre[6] = pb.z, pre[7] = pb.w;
  }
}
__global__ void k_noalloc_scale(double *x, long long n, double s) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] *= s;
}

extern "C" int r3d_fft3d_noalloc(int device, int nx, int ny, int nz, const double *box,
                                 int dir, const double *d_in, double *d_out, void *stream) {
  if (!box || !d_in || !d_out || (dir != -1 && dir != 1))
    return noalloc_fail(R3D_EINVAL, "bad arguments");
  if (nx < 4 || (nx & 1) || ny < 2 || nz < 2)
    return noalloc_fail(R3D_EINVAL, "nx must be even and >= 4, ny and nz >= 2");
  if (device < 0 || device >= 64) return noalloc_fail(R3D_EINVAL, "device ordinal out of range");
  const int hx = nx / 2;
  const long long N = (long long)nx * ny * nz, Nh = (long long)hx * ny * nz;
  if ((size_t)Nh * sizeof(double2) > kNoallocBytes - kNoallocHead)
    return noalloc_fail(R3D_EBUDGET,
                        "grid too large for the fixed work array: nx/2*ny*nz must not exceed " +
                            std::to_string((kNoallocBytes - kNoallocHead) / sizeof(double2)) +
                            " points");
  Desc d{};
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.n = 1;
  d.hx = hx;
  d.N = d.Ns = N;
  d.Nh = d.Nhs = Nh;
  d.nrad_x = factor_length(hx, d.rad_x);
  d.nrad_y = factor_length(ny, d.rad_y);
  d.nrad_z = factor_length(nz, d.rad_z);
  if (d.nrad_x < 0 || d.nrad_y < 0 || d.nrad_z < 0)
    return noalloc_fail(R3D_EINVAL, "grid sizes must factor into primes <= 13");
  // tiles of the runtime-length passes (FP64), as small as divisibility allows
  const size_t cs = sizeof(double2), budget = 100 * 1024;
  int S = 16;
  while (S > 1 && ((ny * nz) % S || smem_x(hx, 1, S, cs) > budget)) S >>= 1;
  int Py = 8;
  while (Py > 1 && (hx % Py || smem_y(ny, Py, cs) > budget)) Py >>= 1;
  int Pz = 4;
  while (Pz > 1 && (hx % Pz || smem_z(nz, 1, Pz, cs) > budget)) Pz >>= 1;
  const size_t smx = smem_x(hx, 1, S, cs), smy = smem_y(ny, Py, cs), smz = smem_z(nz, 1, Pz, cs);
  if (smx > 220 * 1024 || smy > 220 * 1024 || smz > 220 * 1024)
    return noalloc_fail(R3D_EINVAL, "grid too large for one CTA's shared memory");
  d.rows = S;
  d.ycols = Py;
  d.zcols = Pz;
  d.tiles_x = (ny * nz) / S;
  d.tiles_y = nz * (hx / Py);
  d.tiles_z = ny * (hx / Pz);

  // an error left pending by earlier work of the process is not this call's:
  // report it without clearing it
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return noalloc_fail(R3D_ECUDA, std::string("a CUDA error was pending before the call: ") +
                                       cudaGetErrorString(e));
  int caller = -1;
  if ((e = cudaGetDevice(&caller)) != cudaSuccess)
    return noalloc_fail(R3D_ECUDA, cudaGetErrorString(e));
  struct Restore {  // the caller's current device, on every return path
    int dev;
    ~Restore() { cudaSetDevice(dev); }
  } restore{caller};
  if ((e = cudaSetDevice(device)) != cudaSuccess)
    return noalloc_fail(R3D_ECUDA, cudaGetErrorString(e));
  if (!g_noalloc_ptr[device].load()) {  // first call on this device: find the array
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[device].load()) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return noalloc_fail(R3D_ECUDA,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      kernels_set_smem(true, 220 * 1024);
      g_noalloc_ptr[device].store(p);
    }
  }
  unsigned char *base = (unsigned char *)g_noalloc_ptr[device].load();
  Desc *dd = (Desc *)base;
  Ctl *ctl = (Ctl *)(base + kOffCtl);
  int *pre = (int *)(base + kOffPre);
  double2 *w = (double2 *)(base + kNoallocHead);
  d.w = w;
  d.ctl = ctl;
  const int ix_ctas = d.tiles_x;
  cudaStream_t s = (cudaStream_t)stream;
  // control block cleared each call: nothing of the previous call is reused
  DescWords dw;
  std::memcpy(dw.w, &d, sizeof(Desc));
  k_noalloc_setup<<<1, 128, 0, s>>>(dw, dd, ctl, make_int4(0, d.tiles_x, 0, d.tiles_y),
                                    make_int4(0, d.tiles_z, 0, ix_ctas), pre);
  const double dv = box[0] * box[1] * box[2] / (double)N;
  const int par0 = ((nx + ny + nz) / 2) & 1;
  Batch bx{dd, pre, 1}, by{dd, pre + 2, 1}, bz{dd, pre + 4, 1}, bix{dd, pre + 6, 1};
  if (dir < 0) {
    launch_fwd_x<P64>(bx, d.tiles_x, smx, s, 0, d_in);
    launch_fft_y<P64>(by, d.tiles_y, smy, s, -1, 0);
    launch_zoz<P64>(bz, d.tiles_z, smz, s, 0, 0);
    k_noalloc_scale_fwd<<<1184, kThreads, 0, s>>>(w, d_out, Nh, hx, ny, par0, dv);
  } else {
    k_noalloc_scale_inv_in<<<1184, kThreads, 0, s>>>(d_in, w, Nh, hx, ny, par0, dv);
    launch_zoz<P64>(bz, d.tiles_z, smz, s, 1, 0);
    launch_fft_y<P64>(by, d.tiles_y, smy, s, 1, 0);
    launch_inv_x<P64>(bix, ix_ctas, smx, s, 0, d_out, 1);
    k_noalloc_scale<<<1184, kThreads, 0, s>>>(d_out, N, 2.0 / (double)N);
  }
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return noalloc_fail(R3D_ECUDA, cudaGetErrorString(e));
  return R3D_OK;
}
