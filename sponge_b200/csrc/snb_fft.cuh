// Mixed-radix FFT passes for the PME convolution of one box: the 3D
// real-to-complex transform of the charge grid and its inverse as passes
// over lines of one axis, each line held in shared memory while it is
// transformed.
//
// Each 1D transform is the Stockham autosort FFT in the formulation of
// Govindaraju, Lloyd, Dotsenko, Smith and Manferdelli, "High performance
// discrete Fourier transforms on graphics processors" (SC 2008): per stage of
// radix R, butterfly j reads the R points j + r N/R, multiplies them by the
// twiddles exp(-+2 pi i (j mod Ns) r / (Ns R)), takes their R-point DFT and
// writes them to (j / Ns) Ns R + (j mod Ns) + r Ns; Ns grows by R per stage.
// Radices 4, 2, 3, 5, 7 (the grid sizes are products of 2, 3, 5 and 7).
// Lines are interleaved in shared memory ([point][line], the point stride
// one word pair longer than the lines so that a warp writing one line's
// points spreads over the banks) so that the lanes of a warp touch
// consecutive words.
//
// Real rows are transformed two at a time as one complex row a + i b, then
// separated: A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = (Z[k] - conj Z[N-k]) / 2i;
// the inverse forms Z = A + i B from the two half spectra and keeps the real
// and imaginary parts.  Both directions are unnormalised, as cuFFT's.
#pragma once
#include <cuda_runtime.h>

#include "snb_internal.h"

namespace snb {

constexpr int kFftThreads = 256;

// Row pairs per block of the z passes (shared memory under 48 KB).
__host__ __device__ __forceinline__ int fft_row_pairs(int N) { return N <= 128 ? 16 : 8; }

// Lines per block of the y and x passes.
__host__ __device__ __forceinline__ int fft_lines_per_block(int N) {
  return N <= 128 ? 16 : 8;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// cos and sin of 2 pi k / R for the odd radices.
template <int R>
__device__ __forceinline__ float root_cos(int k);
template <int R>
__device__ __forceinline__ float root_sin(int k);
template <>
__device__ __forceinline__ float root_cos<3>(int k) {
  return k == 0 ? 1.0f : -0.5f;
}
template <>
__device__ __forceinline__ float root_sin<3>(int k) {
  return k == 0 ? 0.0f : (k == 1 ? 0.8660254037844387f : -0.8660254037844387f);
}
template <>
__device__ __forceinline__ float root_cos<5>(int k) {
  return k == 0 ? 1.0f
       : (k == 1 || k == 4) ? 0.30901699437494745f
                            : -0.8090169943749473f;
}
template <>
__device__ __forceinline__ float root_sin<5>(int k) {
  return k == 0 ? 0.0f
       : k == 1 ? 0.9510565162951535f
       : k == 2 ? 0.5877852522924732f
       : k == 3 ? -0.5877852522924732f
                : -0.9510565162951535f;
}
template <>
__device__ __forceinline__ float root_cos<7>(int k) {
  return k == 0 ? 1.0f
       : (k == 1 || k == 6) ? 0.6234898018587336f
       : (k == 2 || k == 5) ? -0.22252093395631434f
                            : -0.900968867902419f;
}
template <>
__device__ __forceinline__ float root_sin<7>(int k) {
  return k == 0 ? 0.0f
       : k == 1 ? 0.7818314824680298f
       : k == 2 ? 0.9749279121818236f
       : k == 3 ? 0.43388373911755823f
       : k == 4 ? -0.43388373911755823f
       : k == 5 ? -0.9749279121818236f
                : -0.7818314824680298f;
}

// R-point DFT in place: X[m] = sum_r v[r] exp(S 2 pi i m r / R), S = -1
// forward (DIR < 0), +1 inverse.
template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (R == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    const float2 t0 = make_float2(v[0].x + v[2].x, v[0].y + v[2].y);
    const float2 t1 = make_float2(v[0].x - v[2].x, v[0].y - v[2].y);
    const float2 t2 = make_float2(v[1].x + v[3].x, v[1].y + v[3].y);
    const float2 d = make_float2(v[1].x - v[3].x, v[1].y - v[3].y);
    // (v1 - v3) times -i (forward) or +i (inverse)
    const float2 t3 = DIR < 0 ? make_float2(d.y, -d.x) : make_float2(-d.y, d.x);
    v[0] = make_float2(t0.x + t2.x, t0.y + t2.y);
    v[2] = make_float2(t0.x - t2.x, t0.y - t2.y);
    v[1] = make_float2(t1.x + t3.x, t1.y + t3.y);
    v[3] = make_float2(t1.x - t3.x, t1.y - t3.y);
  } else {
    // odd R: pairs r, R - r share cos and mirror sin
    constexpr int H = (R - 1) / 2;
    constexpr float S = DIR < 0 ? -1.0f : 1.0f;
    float2 sp[H], sm[H];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      sp[r - 1] = make_float2(v[r].x + v[R - r].x, v[r].y + v[R - r].y);
      sm[r - 1] = make_float2(v[r].x - v[R - r].x, v[r].y - v[R - r].y);
    }
    float2 out[R];
    out[0] = v[0];
#pragma unroll
    for (int r = 0; r < H; ++r) {
      out[0].x += sp[r].x;
      out[0].y += sp[r].y;
    }
#pragma unroll
    for (int m = 1; m < R; ++m) {
      float re = v[0].x, im = v[0].y;
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const int k = (m * r) % R;
        const float c = root_cos<R>(k), s = root_sin<R>(k);
        re += sp[r - 1].x * c - S * sm[r - 1].y * s;
        im += sp[r - 1].y * c + S * sm[r - 1].x * s;
      }
      out[m] = make_float2(re, im);
    }
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = out[m];
  }
}

// One Stockham stage over L interleaved lines (point stride L + 1): A -> B.
template <int R, int DIR>
__device__ __forceinline__ void fft_stage(const float2* __restrict__ A, float2* __restrict__ B,
                                          const float2* __restrict__ tw, int N, int Ns,
                                          int L) {
  const int NR = N / R;
  const int tstride = N / (Ns * R);
  const int S = L + 1;
  for (int b = threadIdx.x; b < L * NR; b += blockDim.x) {
    const int line = b % L, j = b / L;
    const int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = A[(j + r * NR) * S + line];
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 t = tw[k * r * tstride];  // k r tstride < N
        if (DIR > 0) t.y = -t.y;
        v[r] = cmul(v[r], t);
      }
    }
    dft<R, DIR>(v);
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) B[(idxD + r * Ns) * S + line] = v[r];
  }
}

// All stages of the axis over L lines held in A (B is scratch of the same
// size); returns the buffer that holds the transform.  Block-wide: every
// thread of the block calls it.
template <int DIR>
__device__ float2* fft_lines(float2* A, float2* B, const float2* tw, const FftAxis& ax,
                             int L) {
  int Ns = 1;
  for (int s = 0; s < ax.nst; ++s) {
    const int R = ax.R[s];
    if (R == 4)
      fft_stage<4, DIR>(A, B, tw, ax.N, Ns, L);
    else if (R == 2)
      fft_stage<2, DIR>(A, B, tw, ax.N, Ns, L);
    else if (R == 3)
      fft_stage<3, DIR>(A, B, tw, ax.N, Ns, L);
    else if (R == 5)
      fft_stage<5, DIR>(A, B, tw, ax.N, Ns, L);
    else
      fft_stage<7, DIR>(A, B, tw, ax.N, Ns, L);
    __syncthreads();
    float2* t = A;
    A = B;
    B = t;
    Ns *= R;
  }
  return A;
}

// Forward z pass: rows of N reals (row r at Q + r N) to their half spectra
// (nc = N / 2 + 1 complex at FQ + r nc), P pairs of rows per block.
// Shared: twiddles [N], two buffers [N][P + 1].
template <int P>
__global__ void __launch_bounds__(kFftThreads)
k_fft_r2c_z(const float* __restrict__ Q, float2* __restrict__ FQ, int nrows, FftAxis ax,
            int nc, const float2* __restrict__ tw_g) {
  extern __shared__ float2 fsm[];
  const int N = ax.N;
  constexpr int S = P + 1;
  float2* tw = fsm;
  float2* A = fsm + N;
  float2* B = A + N * S;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = tw_g[k];
  const int pair0 = blockIdx.x * P;
  for (int t = threadIdx.x; t < N * P; t += blockDim.x) {
    const int n = t % N, p = t / N;
    const int ra = 2 * (pair0 + p), rb = ra + 1;
    const float a = ra < nrows ? Q[(size_t)ra * N + n] : 0.f;
    const float b = rb < nrows ? Q[(size_t)rb * N + n] : 0.f;
    A[n * S + p] = make_float2(a, b);
  }
  __syncthreads();
  const float2* Z = fft_lines<-1>(A, B, tw, ax, P);
  for (int t = threadIdx.x; t < nc * P; t += blockDim.x) {
    const int k = t % nc, p = t / nc;
    const int ra = 2 * (pair0 + p), rb = ra + 1;
    const float2 zk = Z[k * S + p];
    const float2 zm = Z[((N - k) % N) * S + p];
    if (ra < nrows)
      FQ[(size_t)ra * nc + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    if (rb < nrows)
      FQ[(size_t)rb * nc + k] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
  }
}

// Inverse z pass: half spectra (nc complex per row) to rows of N reals,
// pairs of rows at once.  The imaginary parts of the points 0 and N / 2 of
// a half spectrum are dropped (a real row's spectrum has none).
template <int P>
__global__ void __launch_bounds__(kFftThreads)
k_fft_c2r_z(const float2* __restrict__ FQ, float* __restrict__ out, int nrows, FftAxis ax,
            int nc, const float2* __restrict__ tw_g) {
  extern __shared__ float2 fsm[];
  const int N = ax.N;
  constexpr int S = P + 1;
  float2* tw = fsm;
  float2* A = fsm + N;
  float2* B = A + N * S;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = tw_g[k];
  const int pair0 = blockIdx.x * P;
  for (int t = threadIdx.x; t < N * P; t += blockDim.x) {
    const int k = t % N, p = t / N;
    const int ra = 2 * (pair0 + p), rb = ra + 1;
    float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
    if (k < nc) {
      if (ra < nrows) a = FQ[(size_t)ra * nc + k];
      if (rb < nrows) b = FQ[(size_t)rb * nc + k];
      if (k == 0 || 2 * k == N) {
        a.y = 0.f;
        b.y = 0.f;
      }
    } else {
      if (ra < nrows) a = FQ[(size_t)ra * nc + (N - k)];
      if (rb < nrows) b = FQ[(size_t)rb * nc + (N - k)];
      a.y = -a.y;
      b.y = -b.y;
    }
    A[k * S + p] = make_float2(a.x - b.y, a.y + b.x);
  }
  __syncthreads();
  const float2* Z = fft_lines<1>(A, B, tw, ax, P);
  for (int t = threadIdx.x; t < N * P; t += blockDim.x) {
    const int n = t % N, p = t / N;
    const int ra = 2 * (pair0 + p), rb = ra + 1;
    const float2 z = Z[n * S + p];
    if (ra < nrows) out[(size_t)ra * N + n] = z.x;
    if (rb < nrows) out[(size_t)rb * N + n] = z.y;
  }
}

// y pass over the half-spectrum grid [K0][K1][nc]: for each x plane, lines
// of K1 points, L consecutive kz per block.
template <int DIR>
__global__ void __launch_bounds__(kFftThreads)
k_fft_y(float2* __restrict__ FQ, int K1, int nc, FftAxis ax, const float2* __restrict__ tw_g) {
  extern __shared__ float2 fsm[];
  const int N = ax.N;  // == K1
  const int L = fft_lines_per_block(N), S = L + 1;
  float2* tw = fsm;
  float2* A = fsm + N;
  float2* B = A + N * S;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = tw_g[k];
  const int ngrp = (nc + L - 1) / L;
  const int x = blockIdx.x / ngrp, kz0 = (blockIdx.x % ngrp) * L;
  float2* plane = FQ + (size_t)x * K1 * nc;
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int line = t % L, n = t / L, kz = kz0 + line;
    A[n * S + line] = kz < nc ? plane[(size_t)n * nc + kz] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* Z = fft_lines<DIR>(A, B, tw, ax, L);
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int line = t % L, n = t / L, kz = kz0 + line;
    if (kz < nc) plane[(size_t)n * nc + kz] = Z[n * S + line];
  }
}

// Host: the radices of N (4s first, then 2, 3, 5, 7); false when N has
// another prime factor, is longer than kFftMaxN or needs too many stages.
inline bool fft_axis(int N, FftAxis& ax) {
  ax = FftAxis();
  ax.N = N;
  if (N < 2 || N > kFftMaxN) return false;
  int m = N;
  for (int r : {4, 2, 3, 5, 7})
    while (m % r == 0) {
      if (ax.nst == kFftMaxStages) return false;
      ax.R[ax.nst++] = r;
      m /= r;
    }
  return m == 1;
}

// Shared bytes of the z passes and of the y / x passes for an axis of N.
inline size_t fft_smem_rows(int N) {
  return sizeof(float2) * (size_t)(N + 2 * N * (fft_row_pairs(N) + 1));
}
inline size_t fft_smem_lines(int N) {
  return sizeof(float2) * (size_t)(N + 2 * N * (fft_lines_per_block(N) + 1));
}

}  // namespace snb
