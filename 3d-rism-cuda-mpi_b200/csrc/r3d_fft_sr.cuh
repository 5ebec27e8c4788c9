// r3d_fft_sr.cuh -- Stockham FFT with whole radix passes in registers.
//
// A length L = R_0 R_1 ... R_{P-1} (every R_s <= 16) is transformed in P
// passes.  In pass s (N_s = R_0 ... R_{s-1}, N_0 = 1) task j in [0, L/R_s)
// reads the R_s elements x[j + m L/R_s], multiplies element m by the
// twiddle W_{N_s R_s}^{(j mod N_s) m}, takes their R_s-point DFT in
// registers and writes output u to
//     y[(j / N_s) N_s R_s + (j mod N_s) + u N_s]
// (the self-sorting Stockham formulation: natural order in and out, no
// digit reversal).  Each pass costs one read and one write of the data, so a
// 256-point transform (16 x 16) touches shared memory twice per element
// where a radix-8/4 in-place transform of three stages touches it three
// times and also reads a twiddle from global memory per stage.
//
// The inverse transform runs the radices in reverse order: its first pass
// (radix R_{P-1}, N = 1) reads x[j + m L/R_{P-1}], exactly the elements the
// forward transform's last pass (N = L/R_{P-1}) leaves in task j's
// registers, so a kernel can apply a pointwise operation (the OZ step)
// between the two without a shared-memory round trip.
//
// Small DFTs are written out for radices 2, 3, 4, 5, 8 (r3d_fft.cuh) and
// composed for 6, 9, 10, 12, 16 (R = R1 R2: R1-point DFTs of stride-R1
// subsequences, constant twiddles W_R^{n1 k2}, R2... natural order out).
// Both directions are unnormalised; DIR -1 is e^{-2 pi i / R}.
#pragma once

#include "r3d_fft.cuh"

namespace r3d {

// ------------------------------------------------------------ radix plans
struct SrPlan {
  int n;     // passes
  int r[4];  // radices of the forward transform, pass 0 first
};
__host__ __device__ constexpr SrPlan sr_plan(int L) {
  switch (L) {
    case 16: return {1, {16, 0, 0, 0}};
    case 24: return {2, {6, 4, 0, 0}};
    case 32: return {2, {8, 4, 0, 0}};
    case 40: return {2, {8, 5, 0, 0}};
    case 48: return {2, {8, 6, 0, 0}};
    case 64: return {2, {8, 8, 0, 0}};
    case 72: return {2, {8, 9, 0, 0}};
    case 80: return {2, {16, 5, 0, 0}};
    case 96: return {2, {12, 8, 0, 0}};
    case 128: return {2, {16, 8, 0, 0}};
    case 144: return {2, {16, 9, 0, 0}};
    case 160: return {2, {16, 10, 0, 0}};
    case 192: return {2, {16, 12, 0, 0}};
    case 256: return {2, {16, 16, 0, 0}};
    case 512: return {3, {8, 8, 8, 0}};
    default: return {0, {0, 0, 0, 0}};
  }
}
__host__ __device__ constexpr bool sr_length_ok(int L) { return sr_plan(L).n > 0; }
// radix of pass s of the forward (INV = false) or inverse (reversed) plan
__host__ __device__ constexpr int sr_radix(int L, int s, bool inv) {
  return inv ? sr_plan(L).r[sr_plan(L).n - 1 - s] : sr_plan(L).r[s];
}
// N_s: product of the radices before pass s
__host__ __device__ constexpr int sr_ns(int L, int s, bool inv) {
  int p = 1;
  for (int i = 0; i < s; ++i) p *= sr_radix(L, i, inv);
  return p;
}
__host__ __device__ constexpr int sr_max_radix(int L) {
  int m = 0;
  for (int i = 0; i < sr_plan(L).n; ++i) m = sr_plan(L).r[i] > m ? sr_plan(L).r[i] : m;
  return m;
}

// ---------------------------------------------------- constant roots W_R^e
// cos and sin of 2 pi e / R for the composite radices' inner twiddles
template <int R>
__device__ __forceinline__ constexpr double rcos(int e);
template <int R>
__device__ __forceinline__ constexpr double rsin(int e);

#define R3D_ROOTS(R, ...)                                                        \
  template <>                                                                    \
  __device__ __forceinline__ constexpr double rcos<R>(int e) {                   \
    constexpr double c[R] = {__VA_ARGS__};                                       \
    return c[e % R];                                                             \
  }                                                                              \
  template <>                                                                    \
  __device__ __forceinline__ constexpr double rsin<R>(int e) {                   \
    /* sin(2 pi e / R) = cos(2 pi (e - R/4) / R) for R divisible by 4; the */    \
    /* other radices list their sines separately below */                        \
    return rsin_tab_##R(e % R);                                                  \
  }

// The values are cos(2 pi e / R) and sin(2 pi e / R), each computed from its
// first-octant angle (so that the tabulated value is the correctly rounded
// one and the symmetries hold exactly).
__device__ __forceinline__ constexpr double rsin_tab_6(int e) {
  constexpr double s[6] = {0.0, 0.86602540378443864676, 0.86602540378443864676, 0.0,
                           -0.86602540378443864676, -0.86602540378443864676};
  return s[e];
}
__device__ __forceinline__ constexpr double rsin_tab_9(int e) {
  constexpr double s[9] = {0.0,
                           0.64278760968653932632,
                           0.98480775301220805936,
                           0.86602540378443864676,
                           0.34202014332566873304,
                           -0.34202014332566873304,
                           -0.86602540378443864676,
                           -0.98480775301220805936,
                           -0.64278760968653932632};
  return s[e];
}
__device__ __forceinline__ constexpr double rsin_tab_10(int e) {
  constexpr double s[10] = {0.0,
                            0.58778525229247312917,
                            0.95105651629515357212,
                            0.95105651629515357212,
                            0.58778525229247312917,
                            0.0,
                            -0.58778525229247312917,
                            -0.95105651629515357212,
                            -0.95105651629515357212,
                            -0.58778525229247312917};
  return s[e];
}
__device__ __forceinline__ constexpr double rsin_tab_12(int e) {
  constexpr double s[12] = {0.0, 0.5, 0.86602540378443864676, 1.0, 0.86602540378443864676, 0.5,
                            0.0, -0.5, -0.86602540378443864676, -1.0, -0.86602540378443864676,
                            -0.5};
  return s[e];
}
__device__ __forceinline__ constexpr double rsin_tab_16(int e) {
  constexpr double s[16] = {0.0,
                            0.38268343236508977173,
                            0.70710678118654752440,
                            0.92387953251128675613,
                            1.0,
                            0.92387953251128675613,
                            0.70710678118654752440,
                            0.38268343236508977173,
                            0.0,
                            -0.38268343236508977173,
                            -0.70710678118654752440,
                            -0.92387953251128675613,
                            -1.0,
                            -0.92387953251128675613,
                            -0.70710678118654752440,
                            -0.38268343236508977173};
  return s[e];
}
__device__ __forceinline__ constexpr double rsin_tab_24(int e) {
  constexpr double s[24] = {
      0.0, 0.25881904510252076235, 0.5, 0.70710678118654752440, 0.86602540378443864676,
      0.96592582628906828675, 1.0, 0.96592582628906828675, 0.86602540378443864676,
      0.70710678118654752440, 0.5, 0.25881904510252076235, 0.0, -0.25881904510252076235, -0.5,
      -0.70710678118654752440, -0.86602540378443864676, -0.96592582628906828675, -1.0,
      -0.96592582628906828675, -0.86602540378443864676, -0.70710678118654752440, -0.5,
      -0.25881904510252076235};
  return s[e];
}
__device__ __forceinline__ constexpr double rsin_tab_32(int e) {
  constexpr double s[32] = {
      0.0, 0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
      0.70710678118654752440, 0.83146961230254523708, 0.92387953251128675613,
      0.98078528040323044913, 1.0, 0.98078528040323044913, 0.92387953251128675613,
      0.83146961230254523708, 0.70710678118654752440, 0.55557023301960222474,
      0.38268343236508977173, 0.19509032201612826785, 0.0, -0.19509032201612826785,
      -0.38268343236508977173, -0.55557023301960222474, -0.70710678118654752440,
      -0.83146961230254523708, -0.92387953251128675613, -0.98078528040323044913, -1.0,
      -0.98078528040323044913, -0.92387953251128675613, -0.83146961230254523708,
      -0.70710678118654752440, -0.55557023301960222474, -0.38268343236508977173,
      -0.19509032201612826785};
  return s[e];
}
R3D_ROOTS(6, 1.0, 0.5, -0.5, -1.0, -0.5, 0.5)
R3D_ROOTS(9, 1.0, 0.76604444311897803520, 0.17364817766693034885, -0.5,
          -0.93969262078590838405, -0.93969262078590838405, -0.5, 0.17364817766693034885,
          0.76604444311897803520)
R3D_ROOTS(10, 1.0, 0.80901699437494742410, 0.30901699437494742410, -0.30901699437494742410,
          -0.80901699437494742410, -1.0, -0.80901699437494742410, -0.30901699437494742410,
          0.30901699437494742410, 0.80901699437494742410)
R3D_ROOTS(12, 1.0, 0.86602540378443864676, 0.5, 0.0, -0.5, -0.86602540378443864676, -1.0,
          -0.86602540378443864676, -0.5, 0.0, 0.5, 0.86602540378443864676)
R3D_ROOTS(16, 1.0, 0.92387953251128675613, 0.70710678118654752440, 0.38268343236508977173, 0.0,
          -0.38268343236508977173, -0.70710678118654752440, -0.92387953251128675613, -1.0,
          -0.92387953251128675613, -0.70710678118654752440, -0.38268343236508977173, 0.0,
          0.38268343236508977173, 0.70710678118654752440, 0.92387953251128675613)
R3D_ROOTS(24, 1.0, 0.96592582628906828675, 0.86602540378443864676, 0.70710678118654752440, 0.5,
          0.25881904510252076235, 0.0, -0.25881904510252076235, -0.5, -0.70710678118654752440,
          -0.86602540378443864676, -0.96592582628906828675, -1.0, -0.96592582628906828675,
          -0.86602540378443864676, -0.70710678118654752440, -0.5, -0.25881904510252076235, 0.0,
          0.25881904510252076235, 0.5, 0.70710678118654752440, 0.86602540378443864676,
          0.96592582628906828675)
R3D_ROOTS(32, 1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
          0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
          0.19509032201612826785, 0.0, -0.19509032201612826785, -0.38268343236508977173,
          -0.55557023301960222474, -0.70710678118654752440, -0.83146961230254523708,
          -0.92387953251128675613, -0.98078528040323044913, -1.0, -0.98078528040323044913,
          -0.92387953251128675613, -0.83146961230254523708, -0.70710678118654752440,
          -0.55557023301960222474, -0.38268343236508977173, -0.19509032201612826785, 0.0,
          0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
          0.70710678118654752440, 0.83146961230254523708, 0.92387953251128675613,
          0.98078528040323044913)
#undef R3D_ROOTS

// The half-sample twiddle over the R elements z = j + m L / R of a task of
// a first forward (last inverse) pass: e^{-i pi z / L} = e^{-i pi j / L}
// times the constant e^{-i pi m / R} = W_{2R}^m, so a task reads one table
// entry (for j) instead of R.  Returns that twiddle from the entry for j.
template <int R, typename C>
__device__ __forceinline__ C sr_half_twiddle(C pj, int m) {
  using Rt = decltype(pj.x);
  if (m == 0) return pj;
  const Rt c = (Rt)rcos<2 * R>(m), sn = (Rt)-rsin<2 * R>(m);
  return C{pj.x * c - pj.y * sn, pj.x * sn + pj.y * c};
}

// ------------------------------------------------------------ small DFTs
// In place, natural order in and out.
template <int R, int DIR, typename C>
__device__ __forceinline__ void sr_dft(C *a);

// R = R1 * R2 (R1 outer): sub-DFTs of length R2 over n2 for each n1
// (elements n1 + R1 n2), twiddles W_R^{n1 k2}, then R1-point DFTs over n1;
// output k = k2 + R2 k1.
template <int R1, int R2, int DIR, typename C>
__device__ __forceinline__ void sr_dft_composite(C *a) {
  using Rt = decltype(a[0].x);
  constexpr int R = R1 * R2;
  C b[R];
#pragma unroll
  for (int n1 = 0; n1 < R1; ++n1) {
    C s[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) s[n2] = a[n1 + R1 * n2];
    sr_dft<R2, DIR>(s);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      C v = s[k2];
      const int e = (n1 * k2) % R;
      if (e != 0) {
        const Rt c = (Rt)rcos<R>(e), sn = (Rt)(DIR < 0 ? -rsin<R>(e) : rsin<R>(e));
        v = C{v.x * c - v.y * sn, v.x * sn + v.y * c};
      }
      b[n1 * R2 + k2] = v;
    }
  }
#pragma unroll
  for (int k2 = 0; k2 < R2; ++k2) {
    C s[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) s[n1] = b[n1 * R2 + k2];
    sr_dft<R1, DIR>(s);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) a[k2 + R2 * k1] = s[k1];
  }
}

template <int R, int DIR, typename C>
__device__ __forceinline__ void sr_dft(C *a) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<DIR>(a[0], a[1]);
  } else if constexpr (R == 3) {
    dft3<DIR>(a[0], a[1], a[2]);
  } else if constexpr (R == 4) {
    dft4<DIR>(a[0], a[1], a[2], a[3]);
  } else if constexpr (R == 5) {
    dft5<DIR>(a[0], a[1], a[2], a[3], a[4]);
  } else if constexpr (R == 8) {
    dft8<DIR>(a);
  } else if constexpr (R == 6) {
    sr_dft_composite<2, 3, DIR>(a);
  } else if constexpr (R == 9) {
    sr_dft_composite<3, 3, DIR>(a);
  } else if constexpr (R == 10) {
    sr_dft_composite<2, 5, DIR>(a);
  } else if constexpr (R == 12) {
    sr_dft_composite<4, 3, DIR>(a);
  } else if constexpr (R == 16) {
    sr_dft_composite<4, 4, DIR>(a);
  } else {
    static_assert(R == 1, "radix without a register DFT");
  }
}

// Twiddle of element m of task j in a pass with N_s = NS, radix R, length
// L: W_L^{e}, e = (j mod NS) m L / (NS R), from tw[e] = e^{-2 pi i e / L}
// (conjugated for DIR +1).
template <int L, int R, int NS, int DIR, typename C>
__device__ __forceinline__ C sr_twiddle(const C *tw, int j, int m) {
  constexpr int step = L / (NS * R);
  const int e = ((j % NS) * m * step) % L;
  const C w = tw[e];
  return DIR < 0 ? w : cconj(w);
}

// One Stockham pass on registers: twiddles (when NS > 1) and the R-point
// DFT of task j's elements a[0..R).
template <int L, int R, int NS, int DIR, typename C>
__device__ __forceinline__ void sr_pass(C *a, const C *tw, int j) {
  if constexpr (NS > 1) {
#pragma unroll
    for (int m = 1; m < R; ++m) a[m] = cmul(a[m], sr_twiddle<L, R, NS, DIR>(tw, j, m));
  }
  sr_dft<R, DIR>(a);
}
// input and output positions of element m of task j
template <int L, int R>
__device__ __forceinline__ constexpr int sr_in(int j, int m) {
  return j + m * (L / R);
}
template <int R, int NS>
__device__ __forceinline__ constexpr int sr_out(int j, int m) {
  return (j / NS) * NS * R + (j % NS) + m * NS;
}

}  // namespace r3d
