// r3d_passes_tma.cu -- the iteration's y and z passes on the tensor copy
// engine.  A persistent CTA cycles NST shared-memory stages: the copy engine
// brings a tile (PC x-columns by one y or z column, from a tensor map of the
// half spectrum) into a stage while the CTA transforms the tiles already
// there in place, and stores each finished tile back from its stage.
//
// The transforms run in place on the natural-order tile, so the forward y
// transform is decimation in frequency (its spectrum stays in digit-reversed
// ky order in global memory), the z pass transforms forward by decimation in
// frequency, applies the Ornstein-Zernike contraction in digit-reversed kz
// order and transforms back by decimation in time (natural z again), and the
// inverse y transform takes the digit-reversed rows by decimation in time.
// Only these three kernels see the digit-reversed ky layout; the result of
// the three is the same as that of k_fy_ct / k_zoz_ct / k_fy_ct.
// Compiled once per precision like r3d_passes_ct.cu.
#include "r3d_async.cuh"
#include "r3d_common.cuh"
#include "r3d_fft_ct.cuh"

#ifndef R3D_CT_FP64
#define R3D_CT_FP64 1
#endif

namespace r3d {

#if R3D_CT_FP64
using PTM = P64;
#else
using PTM = PMix;
#endif

constexpr int kMaxStages = 4;

// natural index of digit-reversed position P (inverse of digit_rev<L>)
template <int L>
__device__ __forceinline__ int digit_rev_inv(int P) {
  constexpr Fac f = factorize(L);
  int I = 0, M = L, scale = 1;
#pragma unroll
  for (int k = 0; k < f.n; ++k) {
    M /= f.r[k];
    const int dk = P / M;
    P -= dk * M;
    I += dk * scale;
    scale *= f.r[k];
  }
  return I;
}

// Drain after a wait that ran out: flag the solve and wait (bounded) for the
// loads still in flight, then for this thread's stores.
__device__ __forceinline__ void tma_abort(const Desc &d, uint64_t *bar, int nst,
                                          uint32_t pending, uint32_t phase) {
  if (threadIdx.x != 0) return;
  atomicExch(&d.ctl->err, 1);
  for (int s = 0; s < nst; ++s)
    if ((pending >> s) & 1) mbar_wait(&bar[s], (phase >> s) & 1);
  bulk_wait_all();
}

// ------------------------------------------------------------------ FY
// tile = PC x-columns of one (site, z) plane, all ny rows; smem [y][PC].
template <typename P, int L, int PC, int DIR>
__global__ void __launch_bounds__(kThreads)
    k_fy_tma(Batch b, int per, int nst) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr int E8 = sizeof(C) / 8;           // 8-byte elements per complex
  constexpr int RB = L > 256 ? 256 : L;       // rows per tensor copy
  constexpr uint32_t SB = PC * L * sizeof(C);  // stage bytes
  extern __shared__ __align__(1024) char smem[];
  __shared__ __align__(8) uint64_t bar[kMaxStages];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int ptiles = d.hx / PC, nz = d.nz, ntile = d.n * nz * ptiles;
  const int first = cta * per, count = min(per, ntile - first);
  if (count <= 0) return;
  const void *tm = &d.tm_y;
  const C *pw = (const C *)d.pwy, *tw = (const C *)d.twy;
  char *const stages = smem;
  uint64_t *const bars = bar;
  auto issue = [=](int tile, int st) {  // thread 0
    const int pt = tile % ptiles, rest = tile / ptiles, z = rest % nz, v = rest / nz;
    uint64_t *br = bars + st;
    mbar_expect_tx(br, SB);
#pragma unroll
    for (int r0 = 0; r0 < L; r0 += RB)
      tma_load_4d(stages + st * SB + r0 * PC * sizeof(C), tm, pt * PC * E8, r0, z, v, br);
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) mbar_init(&bar[s]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t pending = 0, phase = 0;  // per stage: load in flight, parity of its next wait
  if (threadIdx.x == 0)
    for (int s = 0; s < nst && s < count; ++s) issue(first + s, s);
  for (int s = 0; s < nst && s < count; ++s) pending |= 1u << s;
  for (int it = 0; it < count; ++it) {
    const int st = it % nst, tile = first + it;
    const bool ok = mbar_wait(&bar[st], (phase >> st) & 1, d.wait_polls);
    if (__syncthreads_or(!ok)) {
      tma_abort(d, bar, nst, pending, phase);
      return;
    }
    phase ^= 1u << st;
    pending &= ~(1u << st);
    C *buf = (C *)(smem + st * SB);
    if (DIR < 0) {
#pragma unroll 4
      for (int e = threadIdx.x; e < PC * L; e += kThreads) buf[e] = cmul(buf[e], pw[e / PC]);
      __syncthreads();
      ct_fft_dif<L, PC, PC, -1>(buf, tw);
    } else {
      ct_fft_dit<L, PC, PC, 1>(buf, tw);
#pragma unroll 4
      for (int e = threadIdx.x; e < PC * L; e += kThreads)
        buf[e] = cmul(buf[e], cconj(pw[e / PC]));
    }
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      const int pt = tile % ptiles, rest = tile / ptiles, z = rest % nz, v = rest / nz;
#pragma unroll
      for (int r0 = 0; r0 < L; r0 += RB)
        tma_store_4d(tm, pt * PC * E8, r0, z, v, buf + r0 * PC);
      bulk_commit();
      if (it + nst < count) {
        bulk_wait_read();  // the stage is read out: refill it
        issue(tile + nst, st);
      }
    }
    if (it + nst < count) pending |= 1u << st;
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// ------------------------------------------------------------------ ZOZ
// tile = PC x-columns at one (digit-reversed) ky row, all nz rows, all n
// sites; smem [site][z][PC].  Forward z (DIF), Ornstein-Zernike on the
// digit-reversed kz rows, inverse z (DIT).
template <typename P, int L, int PC, int NS>
__device__ __forceinline__ void tma_oz(typename Cx<typename P::R>::T *buf, const Desc &d,
                                       int ky, int pt) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr int M = NS > 0 ? NS : kMaxSites;
  const int n = NS > 0 ? NS : d.n;
  const long long zs = (long long)d.ny * d.hx;
  const long long off = (long long)ky * d.hx + pt * PC;
  const R *chi = (const R *)d.chi;
  const double2 *fk = (const double2 *)d.fk;
  const long long ay = 2 * ky - d.ny + 1;
#pragma unroll 2
  for (int e = threadIdx.x; e < PC * L; e += kThreads) {
    const int p = e % PC, row = e / PC;
    const int kz = digit_rev_inv<L>(row);
    const long long gi = kz * zs + off + p;
    size_t shell;
    if (d.cubic) {
      const long long ax = 4 * (pt * PC + p) - d.nx + 1, az = 2 * kz - d.nz + 1;
      shell = (size_t)((ax * ax + ay * ay + az * az - 3) / 8);
    } else {
      shell = d.kidx[gi];
    }
    const R *ch = chi + shell * d.chis;
    R x[M * M];
    if constexpr (NS > 0 && (NS * NS) % 4 == 0 && sizeof(R) == 4) {  // 16-byte rows
#pragma unroll
      for (int q = 0; q < NS * NS / 4; ++q) {
        const float4 v4 = reinterpret_cast<const float4 *>(ch)[q];
        x[4 * q] = v4.x;
        x[4 * q + 1] = v4.y;
        x[4 * q + 2] = v4.z;
        x[4 * q + 3] = v4.w;
      }
    } else if constexpr (NS > 0 && (NS * NS) % 2 == 0 && sizeof(R) == 8) {
#pragma unroll
      for (int q = 0; q < NS * NS / 2; ++q) {
        const double2 v2 = reinterpret_cast<const double2 *>(ch)[q];
        x[2 * q] = v2.x;
        x[2 * q + 1] = v2.y;
      }
    } else {
#pragma unroll
      for (int q = 0; q < M * M; ++q)
        if (q < n * n) x[q] = ch[q];
    }
    C c[M];
#pragma unroll
    for (int q = 0; q < M; ++q)
      if (q < n) c[q] = buf[(q * L + row) * PC + p];
    if (fk) {  // mqvfk
      const double2 f = fk[gi];
#pragma unroll
      for (int q = 0; q < M; ++q)
        if (q < n) {
          c[q].x -= (R)(d.qv[q] * f.x);
          c[q].y -= (R)(d.qv[q] * f.y);
        }
    }
#pragma unroll
    for (int a = 0; a < M; ++a) {
      if (a < n) {
        R hr = 0, hi = 0;
#pragma unroll
        for (int q = 0; q < M; ++q) {
          if (q < n) {
            const R xq = x[a * n + q];
            hr += c[q].x * xq;
            hi += c[q].y * xq;
          }
        }
        buf[(a * L + row) * PC + p] = C{hr, hi};
      }
    }
  }
}

template <typename P, int L, int PC>
__global__ void __launch_bounds__(kThreads)
    k_zoz_tma(Batch b, int per, int nst) {
  using R = typename P::R;
  using C = typename Cx<R>::T;
  constexpr int E8 = sizeof(C) / 8;
  constexpr int RB = L > 256 ? 256 : L;
  extern __shared__ __align__(1024) char smem[];
  __shared__ __align__(8) uint64_t bar[kMaxStages];
  const int si = find_solve(b, blockIdx.x);
  const Desc &d = b.d[si];
  if (d.ctl->status != RUNNING) return;
  const int cta = blockIdx.x - b.prefix[si];
  const int n = d.n, ptiles = d.hx / PC, ntile = d.ny * ptiles;
  const int first = cta * per, count = min(per, ntile - first);
  if (count <= 0) return;
  const uint32_t SB = PC * L * n * sizeof(C);
  const void *tm = &d.tm_z;
  const C *pw = (const C *)d.pwz, *tw = (const C *)d.twz;
  char *const stages = smem;
  uint64_t *const bars = bar;
  auto issue = [=](int tile, int st) {  // thread 0
    const int pt = tile % ptiles, y = tile / ptiles;
    uint64_t *br = bars + st;
    mbar_expect_tx(br, SB);
    for (int v = 0; v < n; ++v)
#pragma unroll
      for (int r0 = 0; r0 < L; r0 += RB)
        tma_load_4d(stages + st * SB + (v * L + r0) * PC * sizeof(C), tm, pt * PC * E8, y, r0,
                    v, br);
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < nst; ++s) mbar_init(&bar[s]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t pending = 0, phase = 0;
  if (threadIdx.x == 0)
    for (int s = 0; s < nst && s < count; ++s) issue(first + s, s);
  for (int s = 0; s < nst && s < count; ++s) pending |= 1u << s;
  for (int it = 0; it < count; ++it) {
    const int st = it % nst, tile = first + it;
    const int pt = tile % ptiles, y = tile / ptiles;
    const bool ok = mbar_wait(&bar[st], (phase >> st) & 1, d.wait_polls);
    if (__syncthreads_or(!ok)) {
      tma_abort(d, bar, nst, pending, phase);
      return;
    }
    phase ^= 1u << st;
    pending &= ~(1u << st);
    C *buf = (C *)(smem + st * SB);
    for (int e = threadIdx.x; e < n * PC * L; e += kThreads)
      buf[e] = cmul(buf[e], pw[(e / PC) % L]);
    __syncthreads();
    for (int v = 0; v < n; ++v) ct_fft_dif<L, PC, PC, -1>(buf + v * L * PC, tw);
    const int ky = d.yrev[y];
    switch (n) {
      case 1: tma_oz<P, L, PC, 1>(buf, d, ky, pt); break;
      case 2: tma_oz<P, L, PC, 2>(buf, d, ky, pt); break;
      case 3: tma_oz<P, L, PC, 3>(buf, d, ky, pt); break;
      case 4: tma_oz<P, L, PC, 4>(buf, d, ky, pt); break;
      default: tma_oz<P, L, PC, 0>(buf, d, ky, pt); break;
    }
    __syncthreads();
    for (int v = 0; v < n; ++v) ct_fft_dit<L, PC, PC, 1>(buf + v * L * PC, tw);
    for (int e = threadIdx.x; e < n * PC * L; e += kThreads)
      buf[e] = cmul(buf[e], cconj(pw[(e / PC) % L]));
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int v = 0; v < n; ++v)
#pragma unroll
        for (int r0 = 0; r0 < L; r0 += RB)
          tma_store_4d(tm, pt * PC * E8, y, r0, v, buf + (v * L + r0) * PC);
      bulk_commit();
      if (it + nst < count) {
        bulk_wait_read();
        issue(tile + nst, st);
      }
    }
    if (it + nst < count) pending |= 1u << st;
  }
  if (threadIdx.x == 0) bulk_wait_all();
}

// ------------------------------------------------------------ launchers
// x-columns per tile: FY 8 (FP32) / 4 (FP64), ZOZ 4 / 2 -- rows of 32 to
// 64 bytes; lengths up to 512 (two tensor copies per column beyond 256)
#define R3D_TMA_LENGTHS(X) X(16) X(24) X(32) X(40) X(48) X(64) X(72) X(80) X(96) X(128) X(144) X(160) X(192) X(256) X(512)

template <typename P>
constexpr int tma_pc_y() {
  return sizeof(typename P::R) == 4 ? 8 : 4;
}
template <typename P>
constexpr int tma_pc_z() {
  return sizeof(typename P::R) == 4 ? 4 : 2;
}

template <typename P>
bool tma_launch_fy(int L, int dir, Batch b, int grid, size_t smem, cudaStream_t s, int per,
                   int nst) {
  constexpr int PC = tma_pc_y<P>();
#define R3D_TFY(LL)                                                        \
  if (L == LL) {                                                           \
    if (dir < 0)                                                           \
      k_fy_tma<P, LL, PC, -1><<<grid, kThreads, smem, s>>>(b, per, nst);   \
    else                                                                   \
      k_fy_tma<P, LL, PC, 1><<<grid, kThreads, smem, s>>>(b, per, nst);    \
    return true;                                                           \
  }
  R3D_TMA_LENGTHS(R3D_TFY)
#undef R3D_TFY
  return false;
}

template <typename P>
bool tma_launch_zoz(int L, Batch b, int grid, size_t smem, cudaStream_t s, int per, int nst) {
  constexpr int PC = tma_pc_z<P>();
#define R3D_TZ(LL)                                                         \
  if (L == LL) {                                                           \
    k_zoz_tma<P, LL, PC><<<grid, kThreads, smem, s>>>(b, per, nst);        \
    return true;                                                           \
  }
  R3D_TMA_LENGTHS(R3D_TZ)
#undef R3D_TZ
  return false;
}

// resident CTAs per SM (which: 0 FY, 1 ZOZ)
template <typename P>
int tma_occupancy(int which, int L, size_t smem) {
  constexpr int PY = tma_pc_y<P>(), PZ = tma_pc_z<P>();
  int nb = 0;
#define R3D_TOCC(LL)                                                                        \
  if (L == LL) {                                                                            \
    if (which == 0)                                                                         \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_fy_tma<P, LL, PY, -1>, kThreads, \
                                                    smem);                                  \
    else                                                                                    \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_zoz_tma<P, LL, PZ>, kThreads,    \
                                                    smem);                                  \
    return nb;                                                                              \
  }
  R3D_TMA_LENGTHS(R3D_TOCC)
#undef R3D_TOCC
  return 0;
}

template <typename P>
void tma_allow_smem_all() {
  constexpr int PY = tma_pc_y<P>(), PZ = tma_pc_z<P>();
  auto allow = [](const void *f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
  };
#define R3D_TATTR(LL)                                  \
  allow((const void *)k_fy_tma<P, LL, PY, -1>);        \
  allow((const void *)k_fy_tma<P, LL, PY, 1>);         \
  allow((const void *)k_zoz_tma<P, LL, PZ>);
  R3D_TMA_LENGTHS(R3D_TATTR)
#undef R3D_TATTR
}

template bool tma_launch_fy<PTM>(int, int, Batch, int, size_t, cudaStream_t, int, int);
template bool tma_launch_zoz<PTM>(int, Batch, int, size_t, cudaStream_t, int, int);
template int tma_occupancy<PTM>(int, int, size_t);
template void tma_allow_smem_all<PTM>();

}  // namespace r3d
