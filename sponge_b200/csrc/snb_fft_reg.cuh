// Line transforms held in registers, for the short axes of a batch's PME
// grids (at most kRegFftMax points, multiples of 4 with factors 2, 3, 5, 7).
// One thread transforms one line: its N points stay in registers through
// every stage, and the compile-time length makes every index a constant.
//
// The stages are the Stockham autosort FFT of Govindaraju et al. (SC 2008),
// as in snb_fft.cuh: per stage of radix R, butterfly j reads the points
// j + r N / R, multiplies them by exp(-+2 pi i (j mod Ns) r / (Ns R)), takes
// their R-point DFT and writes them to (j / Ns) Ns R + (j mod Ns) + r Ns.
// Radices in stage order: 4s, then 2, 3, 5, 7.  The twiddles come from a
// table in constant memory (made in double on the host); every lane of a
// warp reads the same entry at the same time, which the constant cache
// broadcasts.
//
// This header defines a __constant__ array: include it from one translation
// unit only.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "snb_fft.cuh"

namespace snb {

// The lengths: X(n) for each.
#define SNB_REG_FFT_SIZES(X) \
  X(4) X(8) X(12) X(16) X(20) X(24) X(28) X(32) X(36) X(40) X(48) X(56) X(60) X(64)
constexpr int kRegFftMax = 64;

__host__ __device__ constexpr bool reg_fft_size(int n) {
  return n == 4 || n == 8 || n == 12 || n == 16 || n == 20 || n == 24 || n == 28 ||
         n == 32 || n == 36 || n == 40 || n == 48 || n == 56 || n == 60 || n == 64;
}

// First twiddle of length n in the table: the lengths below it, summed.
__host__ __device__ constexpr int reg_tw_offset(int n) {
  int o = 0;
  for (int k = 4; k < n; k += 4)
    if (reg_fft_size(k)) o += k;
  return o;
}
constexpr int kRegTwTotal = reg_tw_offset(kRegFftMax) + kRegFftMax;

__constant__ float2 c_reg_tw[kRegTwTotal];  // exp(-2 pi i k / n) per length n

__host__ __device__ constexpr int reg_nstages(int n) {
  int s = 0;
  while (n % 4 == 0) { n /= 4; ++s; }
  while (n % 2 == 0) { n /= 2; ++s; }
  while (n % 3 == 0) { n /= 3; ++s; }
  while (n % 5 == 0) { n /= 5; ++s; }
  while (n % 7 == 0) { n /= 7; ++s; }
  return s;
}

// Radix of stage s of a length-n transform.
__host__ __device__ constexpr int reg_radix(int n, int s) {
  while (n % 4 == 0) { if (s == 0) return 4; n /= 4; --s; }
  while (n % 2 == 0) { if (s == 0) return 2; n /= 2; --s; }
  while (n % 3 == 0) { if (s == 0) return 3; n /= 3; --s; }
  while (n % 5 == 0) { if (s == 0) return 5; n /= 5; --s; }
  while (n % 7 == 0) { if (s == 0) return 7; n /= 7; --s; }
  return 0;
}

// In-place transform of v (DIR < 0 forward, > 0 inverse; unnormalised).
template <int N, int DIR, int S = 0, int NS = 1>
__device__ __forceinline__ void fft_reg(float2 (&v)[N]) {
  if constexpr (S < reg_nstages(N)) {
    constexpr int R = reg_radix(N, S);
    constexpr int NR = N / R;
    constexpr int TW = reg_tw_offset(N);
    constexpr int TSTRIDE = N / (NS * R);
    float2 w[N];
#pragma unroll
    for (int j = 0; j < NR; ++j) {
      const int k = j % NS;
      float2 a[R];
#pragma unroll
      for (int r = 0; r < R; ++r) a[r] = v[j + r * NR];
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 t = c_reg_tw[TW + k * r * TSTRIDE];  // k r TSTRIDE < N
          if (DIR > 0) t.y = -t.y;
          a[r] = cmul(a[r], t);
        }
      }
      dft<R, DIR>(a);
      const int idxD = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) w[idxD + r * NS] = a[r];
    }
#pragma unroll
    for (int q = 0; q < N; ++q) v[q] = w[q];
    fft_reg<N, DIR, S + 1, NS * R>(v);
  }
}

// Host: the twiddle table (double precision, rounded once), and whether a
// length can be transformed here.
inline void reg_fft_twiddles(float2* out) {
  for (int n = 4; n <= kRegFftMax; n += 4) {
    if (!reg_fft_size(n)) continue;
    for (int k = 0; k < n; ++k) {
      const double a = 2.0 * M_PI * (double)k / (double)n;
      out[reg_tw_offset(n) + k] = make_float2((float)std::cos(a), (float)-std::sin(a));
    }
  }
}

}  // namespace snb
