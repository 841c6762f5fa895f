// Smooth PME reciprocal part (Particle_Mesh, PM_force.cpp) and the
// excluded-pair correction, re-designed for sm_100a.
//
// Method (unchanged from the reference): order-4 cardinal B-spline spreading
// of charges to a K0 x K1 x K2 grid from the fractional coordinates
// (PME_Atom_Near :699-762, weights PME_Ma..PME_Md :20-23), R2C FFT, multiply
// by BC(m) = |b(m)|^2 exp(-pi^2 m^2/beta^2)/(pi m^2 V) (tables :541-612),
// C2R, then force F = -q sum_g phi(g) grad W(g) (PME_Final :829-893).
// Energy E = 1/2 sum_m BC(m)|FQ(m)|^2 (equal to 1/2 sum_g Q phi, :896-919,
// :1142-1147) and the virial over the half spectrum with the reference's
// weights (PME_Sum_Virial :1024-1068), both reduced in FP64.
//
// What changes is how the grid is written.  Atoms are counting-sorted by the
// 8x8x8 grid tile of their base point every step; one CTA owns one tile and
// pulls the contributions of the atoms binned in the (at most 3 per axis)
// tiles whose stencils reach it, accumulating in shared memory in int32 fixed
// point (2^22 per charge unit).  The tile is then stored once: no global
// atomics, and the grid is the same bit pattern for any atom order.
#include <algorithm>
#include <cmath>
#include <set>
#include <tuple>
#include <type_traits>
#include <vector>

#include "snb_fft.cuh"
#include "snb_fft_reg.cuh"
#include "snb_internal.h"

namespace snb {

// ---------------------------------------------------------------------------
// Host helpers.
int fft_size(float length) {  // Get_Fft_Patameter (common.cpp:639-659)
  int t = ((int)ceil(length + 3)) >> 2 << 2;
  if (t >= 60 && t <= 68)
    t = 64;
  else if (t >= 120 && t <= 136)
    t = 128;
  else if (t >= 240 && t <= 272)
    t = 256;
  else if (t >= 480 && t <= 544)
    t = 512;
  else if (t >= 960 && t <= 1088)
    t = 1024;
  for (;;) {
    int m = t;
    for (int p : {2, 3, 5, 7})
      while (m > 1 && m % p == 0) m /= p;
    if (m == 1) return t;
    t += 4;
  }
}

// Ewald beta with erfc(beta rc) / rc = tolerance, found the way the
// reference finds it (Get_Beta, PM_force.cpp:246-274), since beta must come
// out bit-identical: the smallest power of two h with a screened value at or
// below the tolerance, then (doublings + 50) halvings of [0, h] in float, each
// keeping the half whose lower end still screens at or above the tolerance;
// the result is the last midpoint (lo + hi) / 2.
float get_beta(float cutoff, float tolerance) {
  const auto screened = [cutoff](float b) { return erfcf(b * cutoff) / cutoff; };
  float hi = 1.0f;
  int doublings = 0;
  while (screened(hi) > tolerance) {
    hi *= 2;
    ++doublings;
  }
  float lo = 0.0f, mid = 0.0f;
  for (int halving = 0; halving < doublings + 50; ++halving) {
    mid = (lo + hi) / 2;
    (screened(mid) >= tolerance ? lo : hi) = mid;
  }
  return mid;
}

// |b(k)|^2 of the order-4 Euler exponential spline (getb, PM_force.cpp:40-64),
// evaluated in double: 1/|sum_{j=0..2} M4(j+1) e^{2 pi i k j/K}|^2.
static double bspline_mod2(int k, int K) {
  const double two_pi = 6.283185307179586476925286766559;
  const double m4[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
  double re = 0, im = 0;
  for (int j = 0; j < 3; ++j) {
    double ang = two_pi * k * j / K;
    re += m4[j] * cos(ang);
    im += m4[j] * sin(ang);
  }
  return 1.0 / (re * re + im * im);
}

// ---------------------------------------------------------------------------
// Per-step binning by grid tile.
struct TileGeom {
  int K0, K1, K2;
  int T;
  int nt0, nt1, nt2;
  Cell rcell;
};
constexpr int kTileEdge = 8;  // grid tiles are kTileEdge^3 points

// Fractional coordinate, base point u and fraction as PME_Atom_Near
// (PM_force.cpp:707-733).
__device__ __forceinline__ void pme_base(float3 r, const Cell& rc, int K0, int K1,
                                         int K2, int& ux, int& uy, int& uz,
                                         float& fx, float& fy, float& fz) {
  float sx = r.x * rc.a11 + r.y * rc.a21 + r.z * rc.a31;
  float sy = r.y * rc.a22 + r.z * rc.a32;
  float sz = r.z * rc.a33;
  sx -= floorf(sx);
  sy -= floorf(sy);
  sz -= floorf(sz);
  if (!isfinite(sx) || !isfinite(sy) || !isfinite(sz)) sx = sy = sz = 0.f;
  sx *= K0;
  sy *= K1;
  sz *= K2;
  ux = (int)sx;
  uy = (int)sy;
  uz = (int)sz;
  ux = ux < 0 ? 0 : (ux < K0 ? ux : K0 - 1);
  uy = uy < 0 ? 0 : (uy < K1 ? uy : K1 - 1);
  uz = uz < 0 ? 0 : (uz < K2 ? uz : K2 - 1);
  fx = sx - ux;
  fx -= floorf(fx);
  fy = sy - uy;
  fy -= floorf(fy);
  fz = sz - uz;
  fz -= floorf(fz);
}

__device__ __forceinline__ int pack_u(int ux, int uy, int uz) {
  return (ux << 20) | (uy << 10) | uz;
}

__global__ void k_pme_bin(int n, const float4* __restrict__ pos, TileGeom g,
                          int* __restrict__ atom_tile, int* __restrict__ atom_slot,
                          int* __restrict__ tile_count, float4* __restrict__ frq,
                          int* __restrict__ upk) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 p = pos[i];
  int ux, uy, uz;
  float fx, fy, fz;
  pme_base(make_float3(p.x, p.y, p.z), g.rcell, g.K0, g.K1, g.K2, ux, uy, uz, fx,
           fy, fz);
  int t = ((ux / g.T) * g.nt1 + (uy / g.T)) * g.nt2 + (uz / g.T);
  atom_tile[i] = t;
  atom_slot[i] = atomicAdd(&tile_count[t], 1);
  frq[i] = make_float4(fx, fy, fz, p.w);
  upk[i] = pack_u(ux, uy, uz);
}

// Pack and bin in one pass: pos[s] = (crd[perm[s]], charge[perm[s]]) for the
// pair kernel, and the PME base point / fraction / tile of the same atom.
// The tile geometry of one system of a batch.
__device__ __forceinline__ TileGeom sys_tiles(const SysGeom& s) {
  TileGeom g;
  g.K0 = s.K0;
  g.K1 = s.K1;
  g.K2 = s.K2;
  g.T = kTileEdge;
  g.nt0 = s.nt0;
  g.nt1 = s.nt1;
  g.nt2 = s.nt2;
  g.rcell = s.rcell;
  return g;
}

template <bool BATCH>
__global__ void k_pack_pme_bin(int n, const float3* __restrict__ crd,
                               const float* __restrict__ charge,
                               const int* __restrict__ type, const int* __restrict__ perm,
                               float4* __restrict__ pos, int* __restrict__ type_sorted,
                               TileGeom g, int* __restrict__ atom_tile,
                               int* __restrict__ atom_slot, int* __restrict__ tile_count,
                               float4* __restrict__ frq, int* __restrict__ upk,
                               BatchView bv, const float3* __restrict__ img_off) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = s < n;
  int t = 0;
  float4 fr4;
  int up = 0;
  if (active) {
    int i = perm ? perm[s] : s;
    float3 r = crd[i];
    float q = charge[i];
    if (img_off) {
      const float3 o = img_off[s];
      pos[s] = make_float4(r.x - o.x, r.y - o.y, r.z - o.z, q);
    } else {
      pos[s] = make_float4(r.x, r.y, r.z, q);
    }
    if (type_sorted) type_sorted[s] = type[i];
    int tile_begin = 0;
    if (BATCH) {
      const SysGeom& sg = bv.sys[bv.sys_of[s]];
      g = sys_tiles(sg);
      tile_begin = sg.tile_begin;
    }
    int ux, uy, uz;
    float fx, fy, fz;
    pme_base(r, g.rcell, g.K0, g.K1, g.K2, ux, uy, uz, fx, fy, fz);
    t = tile_begin + ((ux / g.T) * g.nt1 + (uy / g.T)) * g.nt2 + (uz / g.T);
    fr4 = make_float4(fx, fy, fz, q);
    up = pack_u(ux, uy, uz);
  }
  // sorted neighbours share tiles: one atomic per tile per warp (no tile
  // counts for the atomic spread: tile_count null, uniform over the warp)
  const int slot = tile_count ? warp_aggregated_inc(tile_count, t, active) : 0;
  if (!active) return;
  atom_tile[s] = t;
  atom_slot[s] = slot;
  frq[s] = fr4;
  upk[s] = up;
}

// Scatter into tile order; the tile counters are cleared for the next step.
__global__ void k_pme_scatter(int n, const int* __restrict__ atom_tile,
                              const int* __restrict__ atom_slot,
                              const int* __restrict__ tile_start,
                              const float4* __restrict__ frq,
                              const int* __restrict__ upk, float4* __restrict__ binned,
                              int* __restrict__ binned_u, int* __restrict__ tile_count,
                              int ntiles) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  for (int t = i; t < ntiles; t += gridDim.x * blockDim.x) tile_count[t] = 0;
  if (i >= n) return;
  int d = tile_start[atom_tile[i]] + atom_slot[i];
  binned[d] = frq[i];
  binned_u[d] = upk[i];
}

// B-spline weights of the points u, u-1, u-2, u-3 (power form of
// PME_Ma..PME_Md) and their derivatives (PME_dMa..PME_dMc).
__device__ __forceinline__ void bspline4(float x, float* w) {
  float x2 = x * x, x3 = x2 * x;
  w[0] = 0.16666667f * x3;
  w[1] = -0.5f * x3 + 0.5f * x2 + 0.5f * x + 0.16666667f;
  w[2] = 0.5f * x3 - x2 + 0.66666667f;
  w[3] = -0.16666667f * x3 + 0.5f * x2 - 0.5f * x + 0.16666667f;
}
__device__ __forceinline__ void dbspline4(float x, float* d) {
  float x2 = x * x;
  d[0] = 0.5f * x2;
  d[1] = -1.5f * x2 + x + 0.5f;
  d[2] = 1.5f * x2 - 2.0f * x;
  d[3] = -0.5f * x2 + x - 0.5f;
}

// Bitmask of stencil offsets o in {0..3} with (u - o) mod K in [lo, hi).
__device__ __forceinline__ int stencil_mask(int u, int K, int lo, int hi) {
  int m = 0;
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    int p = u - o;
    p += p < 0 ? K : 0;
    m |= (p >= lo && p < hi) ? (1 << o) : 0;
  }
  return m;
}

constexpr int kTile = kTileEdge;

// One block of W warps per T x T x T tile of the charge grid (T = 8, W = 2
// unless the engine's autotuner picks another shape: T in {8, 16}),
// accumulating in a shared-memory tile.  src{0,1,2}[t] = {count, b0, b1, b2}
// lists the bins along each axis whose atoms can reach tile t.  The warps
// take interleaved rounds of 32 atoms from those bins (one flat range of up
// to 27 bin slices); pass 1 tests whether the atom's 4x4x4 stencil meets the
// tile and appends the ones that do to the warp's list (ballot + popc);
// pass 2 gives one lane per listed atom, which adds its up-to-64 products
// (charge folded into the x weights) to the tile in int32 fixed point (2^22
// per charge unit).  Block barriers only after zeroing and before the single
// store of the tile: no global atomics, and the grid is the same bit pattern
// for any atom order.  A list that fills up is drained and refilled.
constexpr int kSpreadWarps = 2;   // W of the default shape
constexpr int kSpreadList = 256;  // per-warp list of contributing atoms

// Local index (p - lo) of the stencil point u - o on an axis of K points,
// or -1 when it falls outside [lo, hi); four offsets packed in bytes.
__device__ __forceinline__ void stencil_local(int u, int K, int lo, int hi, int* l) {
#pragma unroll
  for (int o = 0; o < 4; ++o) {
    int p = u - o;
    p += p < 0 ? K : 0;
    l[o] = (p >= lo && p < hi) ? p - lo : -1;
  }
}

// Bound on the int32 tile sums.  A point's sum is at most the sum, over the
// atoms whose stencils reach it, of |q| 2^22 (2/3)^3 (each B-spline weight is
// at most 2/3) plus 1/2 for the rounding; every such atom's stencil meets the
// (T/2)^3 octant of the tile that holds the point.  So each lane keeps, per
// octant, the bound of the atoms it spreads that meet the octant; when the
// block's sum of some octant could reach the int32 range the tile is taken
// again with int64 sums.  A liquid's octants stay below a tenth of the range.
constexpr float kPointWeightBound = 0.2963f * 1.0001f;  // (2/3)^3 and float slack
constexpr float kTileSumLimit = 0.99f * 2147483648.0f;

__device__ __forceinline__ void tile_add(int* p, int c) { atomicAdd(p, c); }
__device__ __forceinline__ void tile_add(long long* p, int c) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p),
            static_cast<unsigned long long>((long long)c));
}

// Bits of the T/2-point halves (local index / (T/2)) a stencil axis touches.
template <int T>
__device__ __forceinline__ int halves_of(const int* l) {
  int m = 0;
#pragma unroll
  for (int o = 0; o < 4; ++o) m |= l[o] >= 0 ? 1 << (l[o] / (T / 2)) : 0;
  return m;
}

// Spreads one atom into the tile's store sq (local x runs from lo0); with
// BOUND the atom's per-point bound is added to each octant its stencil meets.
template <int T, typename Acc, bool BOUND>
__device__ __forceinline__ void spread_atom(Acc* sq, float4 f, int up, const TileGeom& g,
                                            int lo0, int hi0, int lo1, int hi1, int lo2,
                                            int hi2, float* oct) {
  const int ux = up >> 20, uy = (up >> 10) & 1023, uz = up & 1023;
  int lx[4], ly[4], lz[4];
  stencil_local(ux, g.K0, lo0, hi0, lx);
  stencil_local(uy, g.K1, lo1, hi1, ly);
  stencil_local(uz, g.K2, lo2, hi2, lz);
  float wx[4], wy[4], wz[4];
  bspline4(f.x, wx);
  bspline4(f.y, wy);
  bspline4(f.z, wz);
  const float qs = f.w * kGridScale;
  if (BOUND) {
    const float b = fabsf(qs) * kPointWeightBound + 0.5f;
    const int mx = halves_of<T>(lx), my = halves_of<T>(ly), mz = halves_of<T>(lz);
#pragma unroll
    for (int o = 0; o < 8; ++o)
      if ((mx >> (o >> 2) & 1) && (my >> ((o >> 1) & 1) & 1) && (mz >> (o & 1) & 1))
        oct[o] += b;
  }
#pragma unroll
  for (int ox = 0; ox < 4; ++ox) {
    if (lx[ox] < 0) continue;
    const float wq = qs * wx[ox];
#pragma unroll
    for (int oy = 0; oy < 4; ++oy) {
      if (ly[oy] < 0) continue;
      const float wxy = wq * wy[oy];
      Acc* row = sq + (lx[ox] * T + ly[oy]) * T;
#pragma unroll
      for (int oz = 0; oz < 4; ++oz)
        if (lz[oz] >= 0) tile_add(row + lz[oz], __float2int_rn(wxy * wz[oz]));
    }
  }
}

// The contributors of one tile (pass 1 of k_pme_spread) spread into sq.
template <int T, int W, typename Acc, bool BOUND>
__device__ __forceinline__ void spread_contributors(
    Acc* sq, int* list, const TileGeom& g, const float4* __restrict__ binned,
    const int* __restrict__ binned_u, int lo0, int hi0, int lo1, int hi1, int lo2,
    int hi2, int nb, int beg, int cnt, int excl, int total, float* oct) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int n_list = 0, bin_cursor = 0;
  for (int base = 32 * w; base < total; base += 32 * W) {
    // atom of flat index base + lane: the bin whose range holds it
    const int fi = base + lane;
    int k = -1;
    for (int b = bin_cursor; b < nb; ++b) {  // warp-uniform walk over the bins
      const int eb = __shfl_sync(0xffffffffu, excl, b);
      const int cb = __shfl_sync(0xffffffffu, cnt, b);
      const int bb = __shfl_sync(0xffffffffu, beg, b);
      if (fi >= eb && fi < eb + cb) k = bb + (fi - eb);
      if (eb + cb >= base + 32) break;
      bin_cursor = b + 1;
    }
    bool in = false;
    if (k >= 0) {
      const int up = binned_u[k];
      const int ux = up >> 20, uy = (up >> 10) & 1023, uz = up & 1023;
      in = stencil_mask(ux, g.K0, lo0, hi0) && stencil_mask(uy, g.K1, lo1, hi1) &&
           stencil_mask(uz, g.K2, lo2, hi2);
    }
    const unsigned m = __ballot_sync(0xffffffffu, in);
    if (in) list[n_list + __popc(m & lt)] = k;
    n_list += __popc(m);
    if (n_list > kSpreadList - 32 || base + 32 * W >= total) {
      __syncwarp();
      for (int e = lane; e < n_list; e += 32) {
        const int ka = list[e];
        spread_atom<T, Acc, BOUND>(sq, binned[ka], binned_u[ka], g, lo0, hi0, lo1, hi1, lo2,
                                   hi2, oct);
      }
      __syncwarp();
      n_list = 0;
    }
  }
}

// wide_tiles (may be null): running count of tiles taken again with int64
// sums because an octant's bound could reach the int32 range.  At the
// default shape sixteen blocks of 64 threads at 64 registers fill an SM's
// register file.
template <bool BATCH, int T = kTile, int W = kSpreadWarps>
__global__ void __launch_bounds__(32 * W, 32 / W)
k_pme_spread(TileGeom g, const int* __restrict__ tile_start,
             const float4* __restrict__ binned, const int* __restrict__ binned_u,
             const int4* __restrict__ src0, const int4* __restrict__ src1,
             const int4* __restrict__ src2, float* __restrict__ Q, int ntiles,
             BatchView bv, int* __restrict__ wide_tiles) {
  // the tile's int32 sums; the same bytes hold half a tile of int64 sums
  constexpr int kTile3 = T * T * T;
  __shared__ __align__(8) int sq[kTile3];
  __shared__ int list_all[W][kSpreadList];
  __shared__ float oct_sum[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int t = blockIdx.x;
  int* list = list_all[w];
  if (BATCH) {  // tile of one system: its geometry, tables and grid
    const SysGeom& sg = bv.sys[bv.tile_sys[t]];
    g = sys_tiles(sg);
    t -= sg.tile_begin;
    tile_start += sg.tile_begin;
    src0 += sg.src_begin0;
    src1 += sg.src_begin1;
    src2 += sg.src_begin2;
    Q += sg.grid_begin;
  }
  const int t2 = t % g.nt2, t1 = (t / g.nt2) % g.nt1, t0 = t / (g.nt1 * g.nt2);
  const int lo0 = t0 * g.T, hi0 = min(lo0 + g.T, g.K0);
  const int lo1 = t1 * g.T, hi1 = min(lo1 + g.T, g.K1);
  const int lo2 = t2 * g.T, hi2 = min(lo2 + g.T, g.K2);
  for (int k = threadIdx.x; k < kTile3; k += blockDim.x) sq[k] = 0;
  if (threadIdx.x < 8) oct_sum[threadIdx.x] = 0.f;
  __syncthreads();
  // the (up to 27) source bins: lane b holds bin b's first atom and count
  const int4 s0 = src0[t0], s1 = src1[t1], s2 = src2[t2];
  const int nb = s0.x * s1.x * s2.x;
  int beg = 0, cnt = 0;
  if (lane < nb) {
    const int a = lane / (s1.x * s2.x), b = (lane / s2.x) % s1.x, c = lane % s2.x;
    const int b0 = a == 0 ? s0.y : (a == 1 ? s0.z : s0.w);
    const int b1 = b == 0 ? s1.y : (b == 1 ? s1.z : s1.w);
    const int b2 = c == 0 ? s2.y : (c == 1 ? s2.z : s2.w);
    const int bin = (b0 * g.nt1 + b1) * g.nt2 + b2;
    beg = tile_start[bin];
    cnt = tile_start[bin + 1] - beg;
  }
  int incl = cnt;  // inclusive prefix of the counts over the bins
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  const int excl = incl - cnt;
  __syncwarp();
  float oct[8];
#pragma unroll
  for (int o = 0; o < 8; ++o) oct[o] = 0.f;
  spread_contributors<T, W, int, true>(sq, list, g, binned, binned_u, lo0, hi0, lo1, hi1,
                                       lo2, hi2, nb, beg, cnt, excl, total, oct);
#pragma unroll
  for (int o = 0; o < 8; ++o) {
    const float v = warp_sum(oct[o]);
    if (lane == 0 && v != 0.f) atomicAdd(&oct_sum[o], v);
  }
  __syncthreads();
  bool wide = false;
#pragma unroll
  for (int o = 0; o < 8; ++o) wide |= !(oct_sum[o] < kTileSumLimit);
  const int w0 = hi0 - lo0, w1 = hi1 - lo1, w2 = hi2 - lo2;
  if (wide) {
    // some point's int32 sum could have wrapped: take the tile again in two
    // halves along x, each with int64 sums (exact and order-independent like
    // the int32 ones) in the same shared bytes; values that fit int32
    // convert to the same floats
    long long* sq64 = reinterpret_cast<long long*>(sq);
    constexpr int kHalf = kTile3 / 2;
    for (int h = 0; h < 2; ++h) {
      const int hlo = lo0 + (T / 2) * h, hhi = min(hlo + T / 2, hi0);
      __syncthreads();
      for (int k = threadIdx.x; k < kHalf; k += blockDim.x) sq64[k] = 0;
      __syncthreads();
      if (hlo < hhi)
        spread_contributors<T, W, long long, false>(sq64, list, g, binned, binned_u, hlo,
                                                    hhi, lo1, hi1, lo2, hi2, nb, beg, cnt,
                                                    excl, total, oct);
      __syncthreads();
      for (int k = threadIdx.x; k < kHalf; k += blockDim.x) {
        int x = k / (T * T), y = (k / T) % T, z = k % T;
        if (x < hhi - hlo && y < w1 && z < w2)
          Q[((size_t)(hlo + x) * g.K1 + (lo1 + y)) * g.K2 + (lo2 + z)] =
              (float)((double)sq64[k] * (double)kGridScaleInv);
      }
    }
    if (threadIdx.x == 0 && wide_tiles) atomicAdd(wide_tiles, 1);
    return;
  }
  for (int k = threadIdx.x; k < kTile3; k += blockDim.x) {
    int x = k / (T * T), y = (k / T) % T, z = k % T;
    if (x < w0 && y < w1 && z < w2)
      Q[((size_t)(lo0 + x) * g.K1 + (lo1 + y)) * g.K2 + (lo2 + z)] =
          (float)sq[k] * kGridScaleInv;
  }
}

// The same grid by global atomics: 16 lanes per atom, lane (ox, oy) adds
// the four points of its z line in int64 fixed point (the products formed
// in the tile path's order, so every point gets the same integers; integer
// sums do not depend on their order).  Atoms in the pair kernel's sorted
// order, so a warp's two atoms are neighbours.
__global__ void __launch_bounds__(256)
k_pme_spread_red(int n, const float4* __restrict__ frq, const int* __restrict__ upk,
                 TileGeom g, long long* __restrict__ Q64) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t >> 4, l = t & 15;
  if (i >= n) return;
  const float4 f = frq[i];
  const int up = upk[i];
  const int ux = up >> 20, uy = (up >> 10) & 1023, uz = up & 1023;
  const int ox = l >> 2, oy = l & 3;
  float wx[4], wy[4], wz[4];
  bspline4(f.x, wx);
  bspline4(f.y, wy);
  bspline4(f.z, wz);
  const float qs = f.w * kGridScale;
  const float wxy = qs * wx[ox] * wy[oy];
  int px = ux - ox;
  px += px < 0 ? g.K0 : 0;
  int py = uy - oy;
  py += py < 0 ? g.K1 : 0;
  unsigned long long* row =
      reinterpret_cast<unsigned long long*>(Q64) + ((size_t)px * g.K1 + py) * g.K2;
#pragma unroll
  for (int oz = 0; oz < 4; ++oz) {
    int pz = uz - oz;
    pz += pz < 0 ? g.K2 : 0;
    const long long c = __float2int_rn(wxy * wz[oz]);
    atomicAdd(row + pz, static_cast<unsigned long long>(c));
  }
}

// int64 fixed-point grid -> float grid for the transform; the sums are
// cleared for the next spread.  (float)v * 2^-22 equals the tile path's
// conversion of the same integer (an int32 one, or an int64 one scaled in
// double: the scale is a power of two).
__global__ void k_pme_grid_float(int nall, long long* __restrict__ Q64,
                                 float* __restrict__ Q) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nall; k += gridDim.x * blockDim.x) {
    Q[k] = (float)Q64[k] * kGridScaleInv;
    Q64[k] = 0;
  }
}

// Plain path: the reference's scheme, 64 global float atomics per atom.
__global__ void k_pme_spread_atomic(int n, const float4* __restrict__ frq,
                                    const int* __restrict__ upk, TileGeom g,
                                    float* __restrict__ Q) {
  int i = blockIdx.x * (blockDim.x >> 4) + (threadIdx.x >> 4);
  int l = threadIdx.x & 15;
  if (i >= n) return;
  float4 f = frq[i];
  int up = upk[i];
  int ux = up >> 20, uy = (up >> 10) & 1023, uz = up & 1023;
  float wx[4], wy[4], wz[4];
  bspline4(f.x, wx);
  bspline4(f.y, wy);
  bspline4(f.z, wz);
  int ox = l >> 2, oy = l & 3;
  int px = ux - ox;
  px += px < 0 ? g.K0 : 0;
  int py = uy - oy;
  py += py < 0 ? g.K1 : 0;
  float qxy = f.w * wx[ox] * wy[oy];
#pragma unroll
  for (int oz = 0; oz < 4; ++oz) {
    int pz = uz - oz;
    pz += pz < 0 ? g.K2 : 0;
    atomicAdd(&Q[((size_t)px * g.K1 + py) * g.K2 + pz], qxy * wz[oz]);
  }
}

// ---------------------------------------------------------------------------
// Influence function, energy and virial over the half spectrum.
struct SpecGeom {
  int K0, K1, K2, nc;
  Cell rcell;
  float mpre;       // pi^2/beta^2
  float inv_pi_v;   // 1/(pi V)
};

constexpr int kSpecBlock = 256;

// The influence BC(m) of the point (kx, ky, kz) of the half spectrum (0 at
// the origin), with m and |m|^2.
__device__ __forceinline__ float influence_bc(int kx, int ky, int kz, const SpecGeom& g,
                                              const float* __restrict__ B0,
                                              const float* __restrict__ B1,
                                              const float* __restrict__ B2, float& mx,
                                              float& my, float& mz, float& msq) {
  const bool origin = (kx | ky | kz) == 0;
  float kxr = kx > g.K0 / 2 ? kx - g.K0 : kx;
  float kyr = ky > g.K1 / 2 ? ky - g.K1 : ky;
  float kzr = kz;
  mx = kxr * g.rcell.a11;
  my = kxr * g.rcell.a21 + kyr * g.rcell.a22;
  mz = kxr * g.rcell.a31 + kyr * g.rcell.a32 + kzr * g.rcell.a33;
  msq = mx * mx + my * my + mz * mz;
  float bc = 0.f;
  if (!origin) bc = g.inv_pi_v / msq * expf(-g.mpre * msq) * B0[kx] * B1[ky] * B2[kz];
  return bc;
}

// One point (kx, ky, kz) of the half spectrum: its influence BC(m) (0 at the
// origin) scales c, and |c|^2 BC feeds the energy and virial sums.
// bc_given >= 0: BC taken from a table instead of computed (m is still
// computed for the virial).
template <bool VIRIAL>
__device__ __forceinline__ float2 influence_point(int kx, int ky, int kz, const SpecGeom& g,
                                                  const float* __restrict__ B0,
                                                  const float* __restrict__ B1,
                                                  const float* __restrict__ B2, float2 c,
                                                  bool energy, double& e, double* v,
                                                  float bc_given = -1.0f) {
  const bool origin = (kx | ky | kz) == 0;
  float mx, my, mz, msq;
  float bc = influence_bc(kx, ky, kz, g, B0, B1, B2, mx, my, mz, msq);
  if (bc_given >= 0.0f) bc = bc_given;
  float f2 = c.x * c.x + c.y * c.y;
  if (energy) {
    float we = (kz == 0 || (2 * kz == g.K2)) ? 0.5f : 1.0f;
    e += (double)(we * bc * f2);
  }
  if (VIRIAL && !origin) {
    float factor = (kz == 0 || kz == g.nc - 1) ? 0.5f : 1.0f;
    float s = factor * f2 * 0.5f * bc;
    float cc = 2.0f / msq * (1.0f + g.mpre * msq);
    v[0] -= (double)(s * (1.0f - cc * mx * mx));
    v[1] -= (double)(s * (0.0f - cc * my * mx));
    v[2] -= (double)(s * (1.0f - cc * my * my));
    v[3] -= (double)(s * (0.0f - cc * mz * mx));
    v[4] -= (double)(s * (0.0f - cc * mz * my));
    v[5] -= (double)(s * (1.0f - cc * mz * mz));
  }
  c.x *= bc;
  c.y *= bc;
  return c;
}

// Block sums of the energy and virial in FP64, fixed order, to
// partial[block][0..6].
__device__ __forceinline__ void influence_partials(double e, const double* v,
                                                   double* __restrict__ partial) {
  __shared__ double sh[kSpecBlock / 32][7];
  double vals[7] = {e, v[0], v[1], v[2], v[3], v[4], v[5]};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 7; ++c) {
    double x = warp_sum(vals[c]);
    if (lane == 0) sh[warp][c] = x;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w][threadIdx.x];
    partial[(size_t)blockIdx.x * 8 + threadIdx.x] = s;
  }
}

template <bool VIRIAL, bool BATCH>
__global__ void __launch_bounds__(kSpecBlock)
k_pme_influence(int nfft, SpecGeom g, const float* __restrict__ B0,
                const float* __restrict__ B1, const float* __restrict__ B2,
                cufftComplex* __restrict__ FQ, double* __restrict__ partial,
                bool energy, BatchView bv, const int4* __restrict__ blocks) {
  double e = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
  int first = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  if (BATCH) {  // block = {system, first, end} of one system's spectrum
    const int4 bk = blocks[blockIdx.x];
    const SysGeom& sg = bv.sys[bk.x];
    g.K0 = sg.K0;
    g.K1 = sg.K1;
    g.K2 = sg.K2;
    g.nc = sg.K2 / 2 + 1;
    g.rcell = sg.rcell;
    g.mpre = sg.mpre;
    g.inv_pi_v = sg.inv_pi_v;
    B0 += sg.b_begin0;
    B1 += sg.b_begin1;
    B2 += sg.b_begin2;
    FQ += sg.spec_begin;
    first = bk.y + threadIdx.x;
    stride = blockDim.x;
    nfft = bk.z;
  }
  for (int idx = first; idx < nfft; idx += stride) {
    int kz = idx % g.nc;
    int ky = (idx / g.nc) % g.K1;
    int kx = idx / (g.nc * g.K1);
    const cufftComplex c = FQ[idx];
    const float2 r = influence_point<VIRIAL>(kx, ky, kz, g, B0, B1, B2,
                                             make_float2(c.x, c.y), energy, e, v);
    FQ[idx] = make_cuComplex(r.x, r.y);
  }
  influence_partials(e, v, partial);
}

// x pass of the convolution: the forward x transform of L columns (ky, kz)
// of the half spectrum, the influence function with the energy / virial
// sums, and the inverse x transform, in one pass over the columns.
template <bool VIRIAL>
__global__ void __launch_bounds__(kFftThreads)
k_fft_x_influence(float2* __restrict__ FQ, int K1, int nc, FftAxis ax,
                  const float2* __restrict__ tw_g, SpecGeom g, const float* __restrict__ B0,
                  const float* __restrict__ B1, const float* __restrict__ B2,
                  double* __restrict__ partial, bool energy) {
  extern __shared__ float2 fsm[];
  const int N = ax.N;  // == K0
  const int L = fft_lines_per_block(N), S = L + 1;
  float2* tw = fsm;
  float2* A = fsm + N;
  float2* B = A + N * S;
  for (int k = threadIdx.x; k < N; k += blockDim.x) tw[k] = tw_g[k];
  const int ncol = K1 * nc, c0 = blockIdx.x * L;
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int line = t % L, n = t / L, c = c0 + line;
    A[n * S + line] = c < ncol ? FQ[(size_t)n * ncol + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* Z = fft_lines<-1>(A, B, tw, ax, L);
  double e = 0.0, v[6] = {0, 0, 0, 0, 0, 0};
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int line = t % L, kx = t / L, c = c0 + line;
    if (c < ncol)
      Z[kx * S + line] = influence_point<VIRIAL>(kx, c / nc, c % nc, g, B0, B1, B2,
                                                 Z[kx * S + line], energy, e, v);
  }
  __syncthreads();
  const float2* Y = fft_lines<1>(Z, Z == A ? B : A, tw, ax, L);
  for (int t = threadIdx.x; t < N * L; t += blockDim.x) {
    const int line = t % L, n = t / L, c = c0 + line;
    if (c < ncol) FQ[(size_t)n * ncol + c] = Y[n * S + line];
  }
  influence_partials(e, v, partial);
}

// ---------------------------------------------------------------------------
// The batch's convolution by the library's own passes: one launch per pass
// over all boxes, each block on one box's lines (job {box, first, count}),
// each thread on one line held in registers (snb_fft_reg.cuh).
constexpr int kRegZPairs = 64;   // row pairs (threads) per block of the z passes
constexpr int kRegLines = 128;   // lines (threads) per block of the y and x passes

// z, forward: `pairs` pairs of real rows of N points from src (contiguous)
// to their half spectra (NC = N / 2 + 1 complex per row) in dst, through
// shared memory both ways so that global accesses are coalesced.  A pair
// a + i b is one complex transform, separated as
// A[k] = (Z[k] + conj Z[N-k]) / 2, B[k] = (Z[k] - conj Z[N-k]) / 2i.
template <int N>
__device__ __forceinline__ void regz_r2c(const float* __restrict__ src,
                                         float2* __restrict__ dst, int pairs, float* sm) {
  constexpr int NC = N / 2 + 1, S = N + 1, SC = NC + 1;
  const int rows = 2 * pairs, p = threadIdx.x;
  // rows of N (a multiple of 4) floats from a 16-byte aligned start: float4
  // loads, eight in flight per thread
  {
    const float4* s4 = reinterpret_cast<const float4*>(src);
    const int n4 = rows * N / 4;
    for (int t0 = threadIdx.x; t0 < n4; t0 += 8 * blockDim.x) {
      float4 q[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int t = t0 + u * blockDim.x;
        if (t < n4) q[u] = s4[t];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int t = t0 + u * blockDim.x;
        if (t < n4) {
          float* d = sm + (4 * t / N) * S + (4 * t) % N;
          d[0] = q[u].x;
          d[1] = q[u].y;
          d[2] = q[u].z;
          d[3] = q[u].w;
        }
      }
    }
  }
  __syncthreads();
  float2 v[N];
  if (p < pairs) {
#pragma unroll
    for (int n = 0; n < N; ++n) v[n] = make_float2(sm[2 * p * S + n], sm[(2 * p + 1) * S + n]);
  }
  __syncthreads();
  float2* out = reinterpret_cast<float2*>(sm);
  if (p < pairs) {
    fft_reg<N, -1>(v);
#pragma unroll
    for (int k = 0; k < NC; ++k) {
      const float2 zk = v[k], zm = v[(N - k) % N];
      out[2 * p * SC + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
      out[(2 * p + 1) * SC + k] = make_float2(0.5f * (zk.y + zm.y), 0.5f * (zm.x - zk.x));
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < rows * NC; t += blockDim.x) dst[t] = out[(t / NC) * SC + t % NC];
}

// Eight float2 loads in flight per thread: src[0, count) into the padded
// rows of `in` (NC per row, stride SC).
template <int NC, int SC>
__device__ __forceinline__ void regz_load_spec(const float2* __restrict__ src, float2* in,
                                               int count) {
  for (int t0 = threadIdx.x; t0 < count; t0 += 8 * blockDim.x) {
    float2 q[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < count) q[u] = src[t];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int t = t0 + u * blockDim.x;
      if (t < count) in[(t / NC) * SC + t % NC] = q[u];
    }
  }
}

// z, inverse: half spectra back to pairs of real rows.  Z = A + i B over the
// full spectrum (A[N-k] = conj A[k]); the imaginary parts of the points 0
// and N / 2 of a half spectrum are dropped (a real row's spectrum has none).
template <int N>
__device__ __forceinline__ void regz_c2r(const float2* __restrict__ src,
                                         float* __restrict__ dst, int pairs, float* sm) {
  constexpr int NC = N / 2 + 1, S = N + 1, SC = NC + 1;
  const int rows = 2 * pairs, p = threadIdx.x;
  float2* in = reinterpret_cast<float2*>(sm);
  regz_load_spec<NC, SC>(src, in, rows * NC);
  __syncthreads();
  float2 v[N];
  if (p < pairs) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      float2 a, b;
      if (k < NC) {
        a = in[2 * p * SC + k];
        b = in[(2 * p + 1) * SC + k];
        if (k == 0 || 2 * k == N) {
          a.y = 0.f;
          b.y = 0.f;
        }
      } else {
        a = in[2 * p * SC + N - k];
        b = in[(2 * p + 1) * SC + N - k];
        a.y = -a.y;
        b.y = -b.y;
      }
      v[k] = make_float2(a.x - b.y, a.y + b.x);
    }
  }
  __syncthreads();
  if (p < pairs) {
    fft_reg<N, 1>(v);
#pragma unroll
    for (int n = 0; n < N; ++n) {
      sm[2 * p * S + n] = v[n].x;
      sm[(2 * p + 1) * S + n] = v[n].y;
    }
  }
  __syncthreads();
  float4* d4 = reinterpret_cast<float4*>(dst);  // 16-byte aligned rows of N floats
  for (int t = threadIdx.x; t < rows * N / 4; t += blockDim.x) {
    const float* q = sm + (4 * t / N) * S + (4 * t) % N;
    d4[t] = make_float4(q[0], q[1], q[2], q[3]);
  }
}

// Shared bytes of a z block for axes up to kmax.
inline size_t regz_smem(int kmax) {
  return sizeof(float) * 2 * kRegZPairs * (size_t)(kmax + 4);
}

// KMAX: the longest axis compiled in (the register count follows it).
template <bool R2C, int KMAX>
__global__ void __launch_bounds__(kRegZPairs)
k_fftb_z(float* __restrict__ Q, float2* __restrict__ FQ, const int4* __restrict__ jobs,
         BatchView bv) {
  extern __shared__ float regz_sm[];
  const int4 jb = jobs[blockIdx.x];  // {box, first row pair, pairs}
  const SysGeom& g = bv.sys[jb.x];
  const int N = g.K2, nc = N / 2 + 1;
  float* rows = Q + g.grid_begin + (size_t)(2 * jb.y) * N;
  float2* spec = FQ + g.spec_begin + (size_t)(2 * jb.y) * nc;
  switch (N) {
#define SNB_CASE(n)                                              \
  case n:                                                        \
    if constexpr (n <= KMAX) {                                   \
      if (R2C)                                                   \
        regz_r2c<n>(rows, spec, jb.z, regz_sm);                  \
      else                                                       \
        regz_c2r<n>(spec, rows, jb.z, regz_sm);                  \
    }                                                            \
    break;
    SNB_REG_FFT_SIZES(SNB_CASE)
#undef SNB_CASE
    default:
      break;
  }
}

// y pass: the line (x, kz) of a box's half spectrum [K0][K1][nc], K1 = N.
template <int N, int DIR>
__device__ __forceinline__ void regy(float2* __restrict__ box, int nc, int line) {
  const int x = line / nc, kz = line - x * nc;
  float2* base = box + (size_t)x * N * nc + kz;
  float2 v[N];
#pragma unroll
  for (int y = 0; y < N; ++y) v[y] = base[(size_t)y * nc];
  fft_reg<N, DIR>(v);
#pragma unroll
  for (int y = 0; y < N; ++y) base[(size_t)y * nc] = v[y];
}

template <int DIR, int KMAX>
__global__ void __launch_bounds__(kRegLines, KMAX <= 40 ? 4 : 1)
k_fftb_y(float2* __restrict__ FQ, const int4* __restrict__ jobs, BatchView bv) {
  const int4 jb = jobs[blockIdx.x];  // {box, first line, lines}
  if ((int)threadIdx.x >= jb.z) return;
  const SysGeom& g = bv.sys[jb.x];
  const int nc = g.K2 / 2 + 1, line = jb.y + threadIdx.x;
  switch (g.K1) {
#define SNB_CASE(n)                                              \
  case n:                                                        \
    if constexpr (n <= KMAX) regy<n, DIR>(FQ + g.spec_begin, nc, line); \
    break;
    SNB_REG_FFT_SIZES(SNB_CASE)
#undef SNB_CASE
    default:
      break;
  }
}

// x pass: the column (ky, kz) of a box's half spectrum, K0 = N: forward
// transform, influence function read from the box's table (in the
// spectrum's layout; with SUMS also the energy / virial sums), inverse.
// Every call takes BC from the table, so the forces do not depend on
// whether the sums are asked for.
template <int N, bool VIRIAL, bool SUMS>
__device__ __forceinline__ void regx(float2* __restrict__ box, int K1, int nc, int line,
                                     const SpecGeom& g, const float* __restrict__ B0,
                                     const float* __restrict__ B1,
                                     const float* __restrict__ B2,
                                     const float* __restrict__ bc_box, bool energy,
                                     double& e, double* vir) {
  const int ky = line / nc, kz = line - ky * nc;
  const size_t stride = (size_t)K1 * nc;
  float2* base = box + line;
  float2 v[N];
#pragma unroll
  for (int x = 0; x < N; ++x) v[x] = base[x * stride];
  fft_reg<N, -1>(v);
#pragma unroll
  for (int kx = 0; kx < N; ++kx) {
    const float bc = bc_box[line + kx * stride];
    if (SUMS) {
      v[kx] = influence_point<VIRIAL>(kx, ky, kz, g, B0, B1, B2, v[kx], energy, e, vir, bc);
    } else {
      v[kx].x *= bc;
      v[kx].y *= bc;
    }
  }
  fft_reg<N, 1>(v);
#pragma unroll
  for (int x = 0; x < N; ++x) base[x * stride] = v[x];
}

// SUMS: the energy / virial sums too (into partial).
template <bool VIRIAL, int KMAX, bool SUMS>
__global__ void __launch_bounds__(kRegLines, KMAX <= 40 ? 3 : 1)
k_fftb_x_influence(float2* __restrict__ FQ, const int4* __restrict__ jobs, BatchView bv,
                   const float* __restrict__ B0, const float* __restrict__ B1,
                   const float* __restrict__ B2, const float* __restrict__ bc,
                   double* __restrict__ partial, bool energy) {
  const int4 jb = jobs[blockIdx.x];  // {box, first column, columns}
  const SysGeom& sg = bv.sys[jb.x];
  SpecGeom g;
  g.K0 = sg.K0;
  g.K1 = sg.K1;
  g.K2 = sg.K2;
  g.nc = sg.K2 / 2 + 1;
  g.rcell = sg.rcell;
  g.mpre = sg.mpre;
  g.inv_pi_v = sg.inv_pi_v;
  double e = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};
  if ((int)threadIdx.x < jb.z) {
    const int line = jb.y + threadIdx.x;
    switch (sg.K0) {
#define SNB_CASE(n)                                                                     \
  case n:                                                                               \
    if constexpr (n <= KMAX)                                                            \
      regx<n, VIRIAL, SUMS>(FQ + sg.spec_begin, sg.K1, g.nc, line, g, B0 + sg.b_begin0,  \
                            B1 + sg.b_begin1, B2 + sg.b_begin2, bc + sg.spec_begin,     \
                            energy, e, vir);                                            \
    break;
      SNB_REG_FFT_SIZES(SNB_CASE)
#undef SNB_CASE
      default:
        break;
    }
  }
  if (SUMS) influence_partials(e, vir, partial);  // every thread of the block
}

// A batch's influence table: BC at every point of every box's half
// spectrum (the boxes of a batch do not change).
__global__ void __launch_bounds__(kSpecBlock)
k_pme_bc_table(BatchView bv, const int4* __restrict__ blocks, const float* __restrict__ B0,
               const float* __restrict__ B1, const float* __restrict__ B2,
               float* __restrict__ bc) {
  const int4 bk = blocks[blockIdx.x];  // {system, first, end} of one box's spectrum
  const SysGeom& sg = bv.sys[bk.x];
  SpecGeom g;
  g.K0 = sg.K0;
  g.K1 = sg.K1;
  g.K2 = sg.K2;
  g.nc = sg.K2 / 2 + 1;
  g.rcell = sg.rcell;
  g.mpre = sg.mpre;
  g.inv_pi_v = sg.inv_pi_v;
  for (int idx = bk.y + threadIdx.x; idx < bk.z; idx += blockDim.x) {
    const int kz = idx % g.nc, ky = (idx / g.nc) % g.K1, kx = idx / (g.nc * g.K1);
    float mx, my, mz, msq;
    bc[sg.spec_begin + idx] = influence_bc(kx, ky, kz, g, B0 + sg.b_begin0, B1 + sg.b_begin1,
                                           B2 + sg.b_begin2, mx, my, mz, msq);
  }
}

// Final FP64 sums of the block partials plus the self / neutralising energy:
// E_self = -beta/sqrt(pi) sum q^2 - pi/(2 beta^2 V) (sum q)^2
// (PM_force.cpp:1149-1162).
__global__ void k_pme_finish(int nblocks, const double* __restrict__ partial,
                             const float4* __restrict__ pos, int n, double beta,
                             double volume, double* __restrict__ sums, bool energy) {
  __shared__ double sh[32][3];
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  if (threadIdx.x < 7)
    for (int b = 0; b < nblocks; ++b) acc[0] += partial[(size_t)b * 8 + threadIdx.x];
  double q2 = 0.0, qs = 0.0;
  if (energy)
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      double q = pos[i].w;
      q2 += q * q;
      qs += q;
    }
  q2 = warp_sum(q2);
  qs = warp_sum(qs);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[warp][0] = q2;
    sh[warp][1] = qs;
  }
  __syncthreads();
  if (threadIdx.x < 7) sums[threadIdx.x] = acc[0];
  if (threadIdx.x == 0 && energy) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += sh[w][0];
      b += sh[w][1];
    }
    const double pi = 3.141592653589793238462643383;
    sums[7] = -beta / sqrt(pi) * a - 0.5 * pi / (beta * beta * volume) * b * b;
  }
}

// Batch: one block per system sums its influence blocks (a contiguous range)
// and its self / neutralising energy into sys_sums[s][8]; then one block adds
// the systems in order into sums[8].  Fixed orders: deterministic.
__global__ void k_pme_finish_batch(BatchView bv, const int* __restrict__ block_begin,
                                   const double* __restrict__ partial,
                                   const float4* __restrict__ frq, double beta,
                                   double* __restrict__ sys_sums, bool energy) {
  const int s = blockIdx.x;
  const SysGeom& sg = bv.sys[s];
  __shared__ double sh[32][2];
  if (threadIdx.x < 7) {
    double a = 0.0;
    for (int b = block_begin[s]; b < block_begin[s + 1]; ++b)
      a += partial[(size_t)b * 8 + threadIdx.x];
    sys_sums[(size_t)s * 8 + threadIdx.x] = a;
  }
  if (!energy) return;
  double q2 = 0.0, qs = 0.0;
  for (int i = sg.atom_begin + threadIdx.x; i < sg.atom_end; i += blockDim.x) {
    double q = frq[i].w;
    q2 += q * q;
    qs += q;
  }
  q2 = warp_sum(q2);
  qs = warp_sum(qs);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sh[warp][0] = q2;
    sh[warp][1] = qs;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += sh[w][0];
      b += sh[w][1];
    }
    const double pi = 3.141592653589793238462643383;
    sys_sums[(size_t)s * 8 + 7] =
        -beta / sqrt(pi) * a - 0.5 * pi / (beta * beta * sg.volume) * b * b;
  }
}

__global__ void k_pme_sum_systems(int nsys, const double* __restrict__ sys_sums,
                                  double* __restrict__ sums) {
  if (threadIdx.x >= 8) return;
  double a = 0.0;
  for (int s = 0; s < nsys; ++s) a += sys_sums[(size_t)s * 8 + threadIdx.x];
  sums[threadIdx.x] = a;
}

// ---------------------------------------------------------------------------
// Gather: four lanes per atom, lane o handles the 16 points of x offset o.
template <int ACCUM, bool BATCH>
__global__ void k_pme_gather(int n, const float4* __restrict__ frq,
                             const int* __restrict__ upk, TileGeom g,
                             const float* __restrict__ phi, float scale,
                             Accumulators acc, BatchView bv) {
  int i = blockIdx.x * (blockDim.x >> 2) + (threadIdx.x >> 2);
  int ox = threadIdx.x & 3;
  bool active = i < n;
  float ax = 0.f, ay = 0.f, az = 0.f;
  if (active) {
    if (BATCH) {
      const SysGeom& sg = bv.sys[bv.sys_of[i]];
      g = sys_tiles(sg);
      phi += sg.grid_begin;
    }
    float4 f = frq[i];
    int up = upk[i];
    int ux = up >> 20, uy = (up >> 10) & 1023, uz = up & 1023;
    float wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
    bspline4(f.x, wx);
    bspline4(f.y, wy);
    bspline4(f.z, wz);
    dbspline4(f.x, dx);
    dbspline4(f.y, dy);
    dbspline4(f.z, dz);
    int px = ux - ox;
    px += px < 0 ? g.K0 : 0;
    float gxs = 0.f, gys = 0.f, gzs = 0.f;
#pragma unroll
    for (int oy = 0; oy < 4; ++oy) {
      int py = uy - oy;
      py += py < 0 ? g.K1 : 0;
      const float* row = phi + ((size_t)px * g.K1 + py) * g.K2;
#pragma unroll
      for (int oz = 0; oz < 4; ++oz) {
        int pz = uz - oz;
        pz += pz < 0 ? g.K2 : 0;
        float p = row[pz];
        gxs += p * dx[ox] * wy[oy] * wz[oz];
        gys += p * wx[ox] * dy[oy] * wz[oz];
        gzs += p * wx[ox] * wy[oy] * dz[oz];
      }
    }
    // -q * grad, grad = (dW/du * K) transformed by rcell (MultiplyTranspose)
    float q = -f.w * scale;
    float t0 = gxs * g.K0, t1 = gys * g.K1, t2 = gzs * g.K2;
    ax = q * (t0 * g.rcell.a11);
    ay = q * (t0 * g.rcell.a21 + t1 * g.rcell.a22);
    az = q * (t0 * g.rcell.a31 + t1 * g.rcell.a32 + t2 * g.rcell.a33);
  }
  ax += __shfl_xor_sync(0xffffffffu, ax, 1);
  ay += __shfl_xor_sync(0xffffffffu, ay, 1);
  az += __shfl_xor_sync(0xffffffffu, az, 1);
  ax += __shfl_xor_sync(0xffffffffu, ax, 2);
  ay += __shfl_xor_sync(0xffffffffu, ay, 2);
  az += __shfl_xor_sync(0xffffffffu, az, 2);
  if (active && ox == 0) {
    const int N = acc.n;
    if (ACCUM == kAccumFixed) {
      red_add(acc.d_f + i, to_fixed_force(ax));
      red_add(acc.d_f + N + i, to_fixed_force(ay));
      red_add(acc.d_f + 2 * N + i, to_fixed_force(az));
    } else {
      atomicAdd(acc.d_ff + i, ax);
      atomicAdd(acc.d_ff + N + i, ay);
      atomicAdd(acc.d_ff + 2 * N + i, az);
    }
  }
}

// ---------------------------------------------------------------------------
// Source bins per tile along one axis of K points in tiles of T: the bins
// holding a base point u with some stencil point (u - o) mod K, o in 0..3,
// inside the tile.  Returns nonzero if a tile needs more than 3 bins.
static int source_bins(int K, int T, std::vector<int4>& src) {
  const int nt = ceil_div(K, T);
  src.assign(nt, make_int4(0, 0, 0, 0));
  for (int t = 0; t < nt; ++t) {
    int lo = t * T, hi = std::min(lo + T, K);
    std::set<int> bins;
    for (int u = 0; u < K; ++u)
      for (int o = 0; o < 4; ++o) {
        int q = ((u - o) % K + K) % K;
        if (q >= lo && q < hi) bins.insert(u / T);
      }
    if (bins.size() > 3) return 1;
    int4 s = make_int4((int)bins.size(), 0, 0, 0);
    int k = 0;
    for (int b : bins) {
      if (k == 0) s.y = b;
      if (k == 1) s.z = b;
      if (k == 2) s.w = b;
      ++k;
    }
    src[t] = s;
  }
  return 0;
}

// Particle_Mesh::Update_Box (PM_force.cpp:1171-1248): the influence
// function and the neutralising term follow the new cell and volume at the
// same grid size.  Both are formed from p.cell / p.rcell / p.volume at each
// call, so the update replaces those.  (The reference also moves its domain
// corners, which this one-domain path has none of.)
int pme_update_box(PME& p, const float* cell6) {
  if (p.bv.nsys > 0) return fail(kNotSupported, "PME: box change of a batch");
  if (cell6[1] != 0.f || cell6[3] != 0.f || cell6[4] != 0.f)
    return fail(kNotSupported, "PME: only rectangular boxes are supported");
  if (!(cell6[0] > 0.f && cell6[2] > 0.f && cell6[5] > 0.f))
    return fail(kBadInput, "PME: box lengths must be > 0");
  p.cell = make_cell(cell6);
  Cell rc{};
  rc.a11 = 1.0f / p.cell.a11;
  rc.a22 = 1.0f / p.cell.a22;
  rc.a33 = 1.0f / p.cell.a33;
  p.rcell = rc;
  p.volume = (double)p.cell.a11 * p.cell.a22 * p.cell.a33;
  return kOk;
}

int pme_init(PME& p, int n, const float* cell6, const float* box_length3,
             float cutoff, float tolerance, int fftx, int ffty, int fftz,
             float grid_spacing, int update_interval, bool reciprocal,
             bool excluded) {
  if (n <= 0) return fail(kBadInput, "PME: atom_numbers must be > 0");
  p.n = n;
  p.cutoff = cutoff;
  p.tolerance = tolerance;
  p.update_interval = update_interval > 0 ? update_interval : 1;
  p.reciprocal = reciprocal;
  p.excluded = excluded;
  p.cell = make_cell(cell6);
  if (!(p.cell.a11 > 0.f && p.cell.a22 > 0.f && p.cell.a33 > 0.f))
    return fail(kBadInput, "PME: the cell's diagonal must be positive");
  // fractional coordinates through the inverse of the lower-triangular cell
  // (Invert_Lower_Triangular_Cell, utils/boundary.h:61-72); the reciprocal
  // vectors m = rcell k of the influence function and the force chain rule
  // use all six entries
  Cell rc{};
  rc.a11 = 1.0f / p.cell.a11;
  rc.a22 = 1.0f / p.cell.a22;
  rc.a33 = 1.0f / p.cell.a33;
  rc.a21 = -p.cell.a21 / (p.cell.a11 * p.cell.a22);
  rc.a31 = (p.cell.a21 * p.cell.a32 - p.cell.a22 * p.cell.a31) /
           (p.cell.a11 * p.cell.a22 * p.cell.a33);
  rc.a32 = -p.cell.a32 / (p.cell.a22 * p.cell.a33);
  p.rcell = rc;
  p.volume = (double)p.cell.a11 * p.cell.a22 * p.cell.a33;
  if (grid_spacing <= 0.f) grid_spacing = 1.0f;
  p.K[0] = fftx > 0 ? fftx : fft_size(box_length3[0] / grid_spacing);
  p.K[1] = ffty > 0 ? ffty : fft_size(box_length3[1] / grid_spacing);
  p.K[2] = fftz > 0 ? fftz : fft_size(box_length3[2] / grid_spacing);
  for (int d = 0; d < 3; ++d)
    if (p.K[d] < 4 || p.K[d] > 1023)
      return fail(kBadInput, "PME: grid dimension must be in [4, 1023]");
  p.nall = p.K[0] * p.K[1] * p.K[2];
  p.nfft = p.K[0] * p.K[1] * (p.K[2] / 2 + 1);
  p.beta = get_beta(cutoff, tolerance);
  p.T = kTile;
  for (int d = 0; d < 3; ++d) p.nt[d] = ceil_div(p.K[d], p.T);
  p.ntiles = p.nt[0] * p.nt[1] * p.nt[2];
  for (int d = 0; d < 3; ++d) {
    std::vector<float> b(p.K[d]);
    for (int k = 0; k < p.K[d]; ++k) b[k] = (float)bspline_mod2(k, p.K[d]);
    SNB_CUDA_TRY(cudaMalloc(&p.d_B[d], sizeof(float) * p.K[d]));
    SNB_CUDA_TRY(cudaMemcpy(p.d_B[d], b.data(), sizeof(float) * p.K[d],
                            cudaMemcpyHostToDevice));
    std::vector<int4> src;
    if (source_bins(p.K[d], p.T, src)) return fail(kBadInput, "PME: tile geometry");
    SNB_CUDA_TRY(cudaMalloc(&p.d_src[d], sizeof(int4) * p.nt[d]));
    SNB_CUDA_TRY(cudaMemcpy(p.d_src[d], src.data(), sizeof(int4) * p.nt[d],
                            cudaMemcpyHostToDevice));
  }
  SNB_CUDA_TRY(cudaMalloc(&p.d_Q, sizeof(float) * p.nall));
  SNB_CUDA_TRY(cudaMalloc(&p.d_FQ, sizeof(cufftComplex) * p.nfft));
  SNB_CUDA_TRY(cudaMalloc(&p.d_phi, sizeof(float) * p.nall));
  SNB_CUDA_TRY(cudaMemset(p.d_phi, 0, sizeof(float) * p.nall));
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_count, sizeof(int) * p.ntiles));
  SNB_CUDA_TRY(cudaMemset(p.d_tile_count, 0, sizeof(int) * p.ntiles));
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_start, sizeof(int) * (p.ntiles + 1)));
  SNB_CUDA_TRY(cudaMalloc(&p.d_atom_tile, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_atom_slot, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_binned, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_binned_u, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_frq, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_upk, sizeof(int) * n));
  p.partial_blocks = std::min(ceil_div(p.nfft, kSpecBlock), 148 * 8);
  SNB_CUDA_TRY(cudaMalloc(&p.d_partial, sizeof(double) * 8 * p.partial_blocks));
  SNB_CUDA_TRY(cudaMalloc(&p.d_sums, sizeof(double) * 8));
  SNB_CUDA_TRY(cudaMemset(p.d_sums, 0, sizeof(double) * 8));
  SNB_CUDA_TRY(cudaMalloc(&p.d_wide_tiles, sizeof(int)));
  SNB_CUDA_TRY(cudaMemset(p.d_wide_tiles, 0, sizeof(int)));
  if (scan_reserve(p.scan, p.ntiles)) return kCudaError;
  if (cufftPlan3d(&p.plan_r2c, p.K[0], p.K[1], p.K[2], CUFFT_R2C) != CUFFT_SUCCESS ||
      cufftPlan3d(&p.plan_c2r, p.K[0], p.K[1], p.K[2], CUFFT_C2R) != CUFFT_SUCCESS)
    return fail(kCudaError, "PME: cuFFT plan creation failed");
  return kOk;
}

// Spread shape of a one-box PME: edge T (8 or 16 grid points) and W warps
// per tile (1, 2, 4 at T = 8; 4, 8 at T = 16), or T = 0 (W = 0): int64
// global atomics instead of tiles.  Redraws the tiles and their source bins;
// the grid, and so every result, is the same bit pattern for every shape.
int pme_set_spread_shape(PME& p, int T, int W) {
  if (p.bv.nsys > 0) return fail(kNotSupported, "PME: spread shape of a batch");
  const bool ok = (T == 8 && (W == 1 || W == 2 || W == 4)) ||
                  (T == 16 && (W == 4 || W == 8)) || (T == 0 && W == 0);
  if (!ok) return fail(kBadInput, "PME: spread shape must be T 8 with 1, 2, 4 warps, T 16 "
                                  "with 4, 8 warps, or T 0 (atomics)");
  if (T == 0) {
    if (!p.d_Q64) {
      SNB_CUDA_TRY(cudaMalloc(&p.d_Q64, sizeof(long long) * (size_t)p.nall));
      SNB_CUDA_TRY(cudaMemset(p.d_Q64, 0, sizeof(long long) * (size_t)p.nall));
    }
    if (!p.spread_atomic) {
      // the tile counts restart from zero when the tiles come back
      SNB_CUDA_TRY(cudaDeviceSynchronize());
      SNB_CUDA_TRY(cudaMemset(p.d_tile_count, 0, sizeof(int) * p.ntiles));
    }
    p.spread_atomic = true;
    return kOk;
  }
  p.spread_atomic = false;
  p.spread_warps = W;
  if (T == p.T) return kOk;
  int nt[3];
  std::vector<int4> src[3];
  for (int d = 0; d < 3; ++d) {
    nt[d] = ceil_div(p.K[d], T);
    if (source_bins(p.K[d], T, src[d])) return fail(kBadInput, "PME: tile geometry");
  }
  const int ntiles = nt[0] * nt[1] * nt[2];
  SNB_CUDA_TRY(cudaDeviceSynchronize());  // nothing in flight reads the old tiles
  for (int d = 0; d < 3; ++d) {
    cudaFree(p.d_src[d]);
    SNB_CUDA_TRY(cudaMalloc(&p.d_src[d], sizeof(int4) * nt[d]));
    SNB_CUDA_TRY(cudaMemcpy(p.d_src[d], src[d].data(), sizeof(int4) * nt[d],
                            cudaMemcpyHostToDevice));
    p.nt[d] = nt[d];
  }
  cudaFree(p.d_tile_count);
  cudaFree(p.d_tile_start);
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_count, sizeof(int) * ntiles));
  SNB_CUDA_TRY(cudaMemset(p.d_tile_count, 0, sizeof(int) * ntiles));
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_start, sizeof(int) * (ntiles + 1)));
  p.T = T;
  p.ntiles = ntiles;
  if (scan_reserve(p.scan, p.ntiles)) return kCudaError;
  return kOk;
}

// The convolution by the own FFT passes (one box): radices and twiddles of
// the three axes.  Refused when an axis is longer than kFftMaxN, the z axis
// is odd, or a length has a prime factor above 7.
// A batch: every axis of every box at most kRegFftMax points (factors 2, 3,
// 5, 7, a multiple of 4); job tables of the five passes.
static int pme_set_own_fft_batch(PME& p) {
  for (const SysGeom& g : p.h_sys)
    if (!reg_fft_size(g.K0) || !reg_fft_size(g.K1) || !reg_fft_size(g.K2))
      return fail(kNotSupported, "PME: the own FFT of a batch needs axes of 4-64 points, "
                                 "multiples of 4 with factors 2, 3, 5, 7");
  if (!p.d_zjobs) {
    std::vector<int4> zj, yj, xj;
    std::vector<int> xb;
    int kmax = 4;
    for (int s = 0; s < (int)p.h_sys.size(); ++s) {
      const SysGeom& g = p.h_sys[s];
      const int nc = g.K2 / 2 + 1;
      kmax = std::max({kmax, g.K0, g.K1, g.K2});
      const int pairs = g.K0 * g.K1 / 2;  // K0 K1 is even (multiples of 4)
      for (int a = 0; a < pairs; a += kRegZPairs)
        zj.push_back(make_int4(s, a, std::min(kRegZPairs, pairs - a), 0));
      const int ylines = g.K0 * nc;
      for (int a = 0; a < ylines; a += kRegLines)
        yj.push_back(make_int4(s, a, std::min(kRegLines, ylines - a), 0));
      xb.push_back((int)xj.size());
      const int xlines = g.K1 * nc;
      for (int a = 0; a < xlines; a += kRegLines)
        xj.push_back(make_int4(s, a, std::min(kRegLines, xlines - a), 0));
    }
    xb.push_back((int)xj.size());
    auto up = [](auto** d, const auto& h) -> int {
      SNB_CUDA_TRY(cudaMalloc(d, sizeof(h[0]) * h.size()));
      SNB_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(h[0]) * h.size(), cudaMemcpyHostToDevice));
      return kOk;
    };
    int rc = up(&p.d_zjobs, zj);
    if (!rc) rc = up(&p.d_yjobs, yj);
    if (!rc) rc = up(&p.d_xjobs, xj);
    if (!rc) rc = up(&p.d_xjob_begin, xb);
    if (rc) return rc;
    p.nzjobs = (int)zj.size();
    p.nyjobs = (int)yj.size();
    p.nxjobs = (int)xj.size();
    p.zsmem = regz_smem(kmax);
    p.reg_kmax = kmax;
    SNB_CUDA_TRY(cudaMalloc(&p.d_bc, sizeof(float) * (size_t)p.nfft));
    k_pme_bc_table<<<p.spec_blocks, kSpecBlock>>>(p.bv, p.d_spec_blocks, p.d_B[0], p.d_B[1],
                                                  p.d_B[2], p.d_bc);
    SNB_CUDA_TRY(cudaGetLastError());
    SNB_CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(p.d_xpartial);
    p.d_xpartial = nullptr;
    SNB_CUDA_TRY(cudaMalloc(&p.d_xpartial, sizeof(double) * 8 * (size_t)p.nxjobs));
  }
  std::vector<float2> tw(kRegTwTotal);
  reg_fft_twiddles(tw.data());
  SNB_CUDA_TRY(cudaMemcpyToSymbol(c_reg_tw, tw.data(), sizeof(float2) * kRegTwTotal));
  p.own_fft = true;
  return kOk;
}

int pme_set_own_fft(PME& p, bool own) {
  if (!own) {
    p.own_fft = false;
    return kOk;
  }
  if (p.bv.nsys > 0) return pme_set_own_fft_batch(p);
  if (!p.d_tw[0]) {
    FftAxis ax[3];
    for (int d = 0; d < 3; ++d)
      if (!fft_axis(p.K[d], ax[d]))
        return fail(kNotSupported, "PME: own FFT needs axes of at most 256 points with "
                                   "factors 2, 3, 5, 7");
    if (p.K[2] % 2) return fail(kNotSupported, "PME: own FFT needs an even z axis");
    for (int d = 0; d < 3; ++d) {
      const int N = p.K[d];
      std::vector<float2> tw(N);
      for (int k = 0; k < N; ++k) {
        const double a = 2.0 * M_PI * (double)k / (double)N;
        tw[k] = make_float2((float)std::cos(a), (float)-std::sin(a));
      }
      SNB_CUDA_TRY(cudaMalloc(&p.d_tw[d], sizeof(float2) * N));
      SNB_CUDA_TRY(cudaMemcpy(p.d_tw[d], tw.data(), sizeof(float2) * N,
                              cudaMemcpyHostToDevice));
      p.fax[d] = ax[d];
    }
    const int nc = p.K[2] / 2 + 1;
    p.xblocks = ceil_div(p.K[1] * nc, fft_lines_per_block(p.K[0]));
    SNB_CUDA_TRY(cudaMalloc(&p.d_xpartial, sizeof(double) * 8 * (size_t)p.xblocks));
  }
  p.own_fft = true;
  return kOk;
}

int pme_init_batch(PME& p, int n, std::vector<SysGeom>& sys, float cutoff,
                   float tolerance, float grid_spacing, bool reciprocal, bool excluded) {
  if (n <= 0 || sys.empty()) return fail(kBadInput, "PME: empty batch");
  const int nsys = (int)sys.size();
  p.n = n;
  p.cutoff = cutoff;
  p.tolerance = tolerance;
  p.update_interval = 1;
  p.reciprocal = reciprocal;
  p.excluded = excluded;
  p.cell = sys[0].cell;
  p.rcell = sys[0].rcell;
  p.beta = get_beta(cutoff, tolerance);
  p.T = kTile;
  if (grid_spacing <= 0.f) grid_spacing = 1.0f;
  const double mpre = M_PI * M_PI / ((double)p.beta * p.beta);
  for (auto& g : sys) {
    g.K0 = fft_size(g.cell.a11 / grid_spacing);
    g.K1 = fft_size(g.cell.a22 / grid_spacing);
    g.K2 = fft_size(g.cell.a33 / grid_spacing);
    if (g.K0 > 1023 || g.K1 > 1023 || g.K2 > 1023)
      return fail(kBadInput, "PME: grid dimension must be in [4, 1023]");
    g.nt0 = ceil_div(g.K0, p.T);
    g.nt1 = ceil_div(g.K1, p.T);
    g.nt2 = ceil_div(g.K2, p.T);
    g.volume = (double)g.cell.a11 * g.cell.a22 * g.cell.a33;
    g.mpre = (float)mpre;
    g.inv_pi_v = (float)(1.0 / (M_PI * g.volume));
  }
  // grids of the same size side by side (one batched FFT plan per size)
  std::vector<int> order(nsys);
  for (int s = 0; s < nsys; ++s) order[s] = s;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const SysGeom &x = sys[a], &y = sys[b];
    return std::make_tuple(x.K0, x.K1, x.K2) < std::make_tuple(y.K0, y.K1, y.K2);
  });
  long long grid = 0, spec = 0;
  for (int s : order) {
    SysGeom& g = sys[s];
    if (p.groups.empty() || p.groups.back().K[0] != g.K0 || p.groups.back().K[1] != g.K1 ||
        p.groups.back().K[2] != g.K2) {
      PME::FftGroup fg;
      fg.K[0] = g.K0;
      fg.K[1] = g.K1;
      fg.K[2] = g.K2;
      fg.count = 0;
      fg.grid_begin = (int)grid;
      fg.spec_begin = (int)spec;
      p.groups.push_back(fg);
    }
    p.groups.back().count++;
    g.grid_begin = (int)grid;
    g.spec_begin = (int)spec;
    grid += (long long)g.K0 * g.K1 * g.K2;
    spec += (long long)g.K0 * g.K1 * (g.K2 / 2 + 1);
  }
  if (spec > 2147483647LL) return fail(kBadInput, "PME: batch grids exceed 32-bit offsets");
  p.nall = (int)grid;
  p.nfft = (int)spec;
  // tiles, source bins and |b|^2 tables in system order
  std::vector<int4> src_all[3];
  std::vector<float> b_all[3];
  std::vector<int> tile_sys;
  std::vector<int4> blocks;
  std::vector<int> block_begin(nsys + 1, 0);
  int tiles = 0;
  const int per_block = kSpecBlock * 8;  // spectrum points per influence block
  for (int s = 0; s < nsys; ++s) {
    SysGeom& g = sys[s];
    g.tile_begin = tiles;
    const int nt = g.nt0 * g.nt1 * g.nt2;
    tiles += nt;
    tile_sys.insert(tile_sys.end(), nt, s);
    const int K[3] = {g.K0, g.K1, g.K2};
    int* src_begin[3] = {&g.src_begin0, &g.src_begin1, &g.src_begin2};
    int* b_begin[3] = {&g.b_begin0, &g.b_begin1, &g.b_begin2};
    for (int d = 0; d < 3; ++d) {
      std::vector<int4> src;
      if (source_bins(K[d], p.T, src)) return fail(kBadInput, "PME: tile geometry");
      *src_begin[d] = (int)src_all[d].size();
      src_all[d].insert(src_all[d].end(), src.begin(), src.end());
      *b_begin[d] = (int)b_all[d].size();
      for (int k = 0; k < K[d]; ++k) b_all[d].push_back((float)bspline_mod2(k, K[d]));
    }
    const int nfft_s = g.K0 * g.K1 * (g.K2 / 2 + 1);
    block_begin[s] = (int)blocks.size();
    for (int b0 = 0; b0 < nfft_s; b0 += per_block)
      blocks.push_back(make_int4(s, b0, std::min(b0 + per_block, nfft_s), 0));
  }
  block_begin[nsys] = (int)blocks.size();
  p.ntiles = tiles;
  p.spec_blocks = (int)blocks.size();
  for (int d = 0; d < 3; ++d) {
    SNB_CUDA_TRY(cudaMalloc(&p.d_B[d], sizeof(float) * b_all[d].size()));
    SNB_CUDA_TRY(cudaMemcpy(p.d_B[d], b_all[d].data(), sizeof(float) * b_all[d].size(),
                            cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMalloc(&p.d_src[d], sizeof(int4) * src_all[d].size()));
    SNB_CUDA_TRY(cudaMemcpy(p.d_src[d], src_all[d].data(), sizeof(int4) * src_all[d].size(),
                            cudaMemcpyHostToDevice));
  }
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_sys, sizeof(int) * tiles));
  SNB_CUDA_TRY(cudaMemcpy(p.d_tile_sys, tile_sys.data(), sizeof(int) * tiles,
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&p.d_spec_blocks, sizeof(int4) * blocks.size()));
  SNB_CUDA_TRY(cudaMemcpy(p.d_spec_blocks, blocks.data(), sizeof(int4) * blocks.size(),
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&p.d_sys_block_begin, sizeof(int) * (nsys + 1)));
  SNB_CUDA_TRY(cudaMemcpy(p.d_sys_block_begin, block_begin.data(), sizeof(int) * (nsys + 1),
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&p.d_sys_sums, sizeof(double) * 8 * nsys));
  SNB_CUDA_TRY(cudaMemset(p.d_sys_sums, 0, sizeof(double) * 8 * nsys));
  SNB_CUDA_TRY(cudaMalloc(&p.d_Q, sizeof(float) * p.nall));
  SNB_CUDA_TRY(cudaMalloc(&p.d_FQ, sizeof(cufftComplex) * p.nfft));
  SNB_CUDA_TRY(cudaMalloc(&p.d_phi, sizeof(float) * p.nall));
  SNB_CUDA_TRY(cudaMemset(p.d_phi, 0, sizeof(float) * p.nall));
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_count, sizeof(int) * p.ntiles));
  SNB_CUDA_TRY(cudaMemset(p.d_tile_count, 0, sizeof(int) * p.ntiles));
  SNB_CUDA_TRY(cudaMalloc(&p.d_tile_start, sizeof(int) * (p.ntiles + 1)));
  SNB_CUDA_TRY(cudaMalloc(&p.d_atom_tile, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_atom_slot, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_binned, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_binned_u, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_frq, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&p.d_upk, sizeof(int) * n));
  p.partial_blocks = p.spec_blocks;
  SNB_CUDA_TRY(cudaMalloc(&p.d_partial, sizeof(double) * 8 * p.partial_blocks));
  SNB_CUDA_TRY(cudaMalloc(&p.d_sums, sizeof(double) * 8));
  SNB_CUDA_TRY(cudaMemset(p.d_sums, 0, sizeof(double) * 8));
  SNB_CUDA_TRY(cudaMalloc(&p.d_wide_tiles, sizeof(int)));
  SNB_CUDA_TRY(cudaMemset(p.d_wide_tiles, 0, sizeof(int)));
  if (scan_reserve(p.scan, p.ntiles)) return kCudaError;
  p.h_sys = sys;
  for (auto& fg : p.groups) {
    int dims[3] = {fg.K[0], fg.K[1], fg.K[2]};
    if (cufftPlanMany(&fg.r2c, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C,
                      fg.count) != CUFFT_SUCCESS ||
        cufftPlanMany(&fg.c2r, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R,
                      fg.count) != CUFFT_SUCCESS)
      return fail(kCudaError, "PME: cuFFT batched plan creation failed");
  }
  return kOk;
}

int pme_wide_tiles(PME& p, int* count, cudaStream_t st) {
  int v = 0;
  if (p.d_wide_tiles) {
    SNB_CUDA_TRY(cudaMemcpyAsync(&v, p.d_wide_tiles, sizeof(int), cudaMemcpyDeviceToHost, st));
    SNB_CUDA_TRY(cudaStreamSynchronize(st));
  }
  *count = v;
  return kOk;
}

void pme_free(PME& p) {
  cudaFree(p.d_wide_tiles);
  cudaFree(p.d_Q64);
  for (int d = 0; d < 3; ++d) cudaFree(p.d_tw[d]);
  cudaFree(p.d_xpartial);
  cudaFree(p.d_zjobs);
  cudaFree(p.d_bc);
  cudaFree(p.d_yjobs);
  cudaFree(p.d_xjobs);
  cudaFree(p.d_xjob_begin);
  for (auto& fg : p.groups) {
    if (fg.r2c) cufftDestroy(fg.r2c);
    if (fg.c2r) cufftDestroy(fg.c2r);
  }
  cudaFree(p.d_spec_blocks);
  cudaFree(p.d_sys_block_begin);
  cudaFree(p.d_sys_sums);
  cudaFree(p.d_tile_sys);
  for (int d = 0; d < 3; ++d) cudaFree(p.d_src[d]);
  cudaFree(p.d_frq);
  cudaFree(p.d_upk);
  for (int d = 0; d < 3; ++d) cudaFree(p.d_B[d]);
  cudaFree(p.d_Q);
  cudaFree(p.d_FQ);
  cudaFree(p.d_phi);
  cudaFree(p.d_tile_count);
  cudaFree(p.d_tile_start);
  cudaFree(p.d_atom_tile);
  cudaFree(p.d_atom_slot);
  cudaFree(p.d_binned);
  cudaFree(p.d_binned_u);
  cudaFree(p.d_partial);
  cudaFree(p.d_sums);
  cudaFree(p.scan.block_sums);
  if (p.plan_r2c) cufftDestroy(p.plan_r2c);
  if (p.plan_c2r) cufftDestroy(p.plan_c2r);
  p = PME();
}

// Binning from caller-frame coordinates through a permutation, fused with
// the pack of the pair kernel's input (pos, type_sorted may be null).
int pme_pack_bin(PME& p, int n, const float3* crd, const float* charge, const int* type,
                 const int* perm, float4* pos, int* type_sorted, cudaStream_t st,
                 const float3* img_off) {
  if (n != p.n) return fail(kBadInput, "PME: atom count differs from Initial");
  TileGeom g{p.K[0], p.K[1], p.K[2], p.T, p.nt[0], p.nt[1], p.nt[2], p.rcell};
  if (p.bv.nsys > 0)
    k_pack_pme_bin<true><<<ceil_div(n, 256), 256, 0, st>>>(
        n, crd, charge, type, perm, pos, type_sorted, g, p.d_atom_tile, p.d_atom_slot,
        p.d_tile_count, p.d_frq, p.d_upk, p.bv, img_off);
  else
    k_pack_pme_bin<false><<<ceil_div(n, 256), 256, 0, st>>>(
        n, crd, charge, type, perm, pos, type_sorted, g, p.d_atom_tile, p.d_atom_slot,
        p.spread_atomic ? nullptr : p.d_tile_count, p.d_frq, p.d_upk, p.bv, img_off);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Everything after binning: spread, FFT, influence / energy / virial, FFT,
// gather into acc (index = the frame the atoms were binned in).
int pme_after_bin(PME& p, int n, Accumulators& acc, int accum, bool need_energy,
                  bool need_virial, cudaStream_t st) {
  TileGeom g{p.K[0], p.K[1], p.K[2], p.T, p.nt[0], p.nt[1], p.nt[2], p.rcell};
  const bool batch = p.bv.nsys > 0;
  if (batch) {
    for (auto& fg : p.groups)
      if (cufftSetStream(fg.r2c, st) != CUFFT_SUCCESS ||
          cufftSetStream(fg.c2r, st) != CUFFT_SUCCESS)
        return fail(kCudaError, "PME: cufftSetStream failed");
  } else if (cufftSetStream(p.plan_r2c, st) != CUFFT_SUCCESS ||
             cufftSetStream(p.plan_c2r, st) != CUFFT_SUCCESS) {
    return fail(kCudaError, "PME: cufftSetStream failed");
  }
  if (accum == kAccumFixed && !batch && p.spread_atomic) {
    k_pme_spread_red<<<ceil_div(n, 16), 256, 0, st>>>(n, p.d_frq, p.d_upk, g, p.d_Q64);
    k_pme_grid_float<<<ceil_div(p.nall, 256 * 4), 256, 0, st>>>(p.nall, p.d_Q64, p.d_Q);
  } else if (accum == kAccumFixed) {
    int rc = scan_exclusive(p.d_tile_count, p.d_tile_start, p.ntiles, nullptr, p.scan,
                            st);
    if (rc) return rc;
    k_pme_scatter<<<ceil_div(n, 256), 256, 0, st>>>(
        n, p.d_atom_tile, p.d_atom_slot, p.d_tile_start, p.d_frq, p.d_upk, p.d_binned,
        p.d_binned_u, p.d_tile_count, p.ntiles);
    const int sblocks = p.ntiles;  // one block per tile
#define SNB_SPREAD(B, T, W)                                                              \
  k_pme_spread<B, T, W><<<sblocks, 32 * (W), 0, st>>>(                                    \
      g, p.d_tile_start, p.d_binned, p.d_binned_u, p.d_src[0], p.d_src[1], p.d_src[2],   \
      p.d_Q, p.ntiles, p.bv, p.d_wide_tiles)
    if (batch)
      SNB_SPREAD(true, kTile, kSpreadWarps);
    else if (p.T == 16 && p.spread_warps == 8)
      SNB_SPREAD(false, 16, 8);
    else if (p.T == 16)
      SNB_SPREAD(false, 16, 4);
    else if (p.spread_warps == 4)
      SNB_SPREAD(false, kTile, 4);
    else if (p.spread_warps == 1)
      SNB_SPREAD(false, kTile, 1);
    else
      SNB_SPREAD(false, kTile, kSpreadWarps);
#undef SNB_SPREAD
  } else {
    if (batch) return fail(kNotSupported, "PME batch: fixed-point accumulation only");
    SNB_CUDA_TRY(cudaMemsetAsync(p.d_Q, 0, sizeof(float) * p.nall, st));
    SNB_CUDA_TRY(cudaMemsetAsync(p.d_tile_count, 0, sizeof(int) * p.ntiles, st));
    k_pme_spread_atomic<<<ceil_div(n, 16), 256, 0, st>>>(n, p.d_frq, p.d_upk, g, p.d_Q);
  }
  SpecGeom sg;
  sg.K0 = p.K[0];
  sg.K1 = p.K[1];
  sg.K2 = p.K[2];
  sg.nc = p.K[2] / 2 + 1;
  sg.rcell = p.rcell;
  sg.mpre = (float)(M_PI * M_PI / ((double)p.beta * p.beta));
  sg.inv_pi_v = (float)(1.0 / (M_PI * p.volume));
  if (batch && p.own_fft) {
    // z, y, then x with the influence function and back, then y and z, one
    // launch per pass over all boxes
    float2* FQ = reinterpret_cast<float2*>(p.d_FQ);
    auto passes = [&](auto kmax) {
      constexpr int KM = decltype(kmax)::value;
      k_fftb_z<true, KM><<<p.nzjobs, kRegZPairs, p.zsmem, st>>>(p.d_Q, FQ, p.d_zjobs, p.bv);
      k_fftb_y<-1, KM><<<p.nyjobs, kRegLines, 0, st>>>(FQ, p.d_yjobs, p.bv);
      if (need_virial)
        k_fftb_x_influence<true, KM, true><<<p.nxjobs, kRegLines, 0, st>>>(
            FQ, p.d_xjobs, p.bv, p.d_B[0], p.d_B[1], p.d_B[2], p.d_bc, p.d_xpartial,
            need_energy);
      else if (need_energy)
        k_fftb_x_influence<false, KM, true><<<p.nxjobs, kRegLines, 0, st>>>(
            FQ, p.d_xjobs, p.bv, p.d_B[0], p.d_B[1], p.d_B[2], p.d_bc, p.d_xpartial,
            need_energy);
      else  // forces only: no sums
        k_fftb_x_influence<false, KM, false><<<p.nxjobs, kRegLines, 0, st>>>(
            FQ, p.d_xjobs, p.bv, p.d_B[0], p.d_B[1], p.d_B[2], p.d_bc, nullptr, false);
      if (need_energy || need_virial) {
        k_pme_finish_batch<<<p.bv.nsys, 256, 0, st>>>(p.bv, p.d_xjob_begin, p.d_xpartial,
                                                      p.d_frq, (double)p.beta, p.d_sys_sums,
                                                      need_energy);
        k_pme_sum_systems<<<1, 32, 0, st>>>(p.bv.nsys, p.d_sys_sums, p.d_sums);
      }
      k_fftb_y<1, KM><<<p.nyjobs, kRegLines, 0, st>>>(FQ, p.d_yjobs, p.bv);
      k_fftb_z<false, KM><<<p.nzjobs, kRegZPairs, p.zsmem, st>>>(p.d_phi, FQ, p.d_zjobs,
                                                                 p.bv);
    };
    if (p.reg_kmax <= 32)
      passes(std::integral_constant<int, 32>());
    else if (p.reg_kmax <= 40)
      passes(std::integral_constant<int, 40>());
    else
      passes(std::integral_constant<int, kRegFftMax>());
    const int gt = p.gather_threads;  // 4 lanes per atom
    k_pme_gather<kAccumFixed, true><<<ceil_div(n, gt / 4), gt, 0, st>>>(
        n, p.d_frq, p.d_upk, g, p.d_phi, 1.0f, acc, p.bv);
    SNB_CUDA_TRY(cudaGetLastError());
    return kOk;
  }
  if (!batch && p.own_fft) {
    // z, y, then x with the influence function and back, then y and z
    float2* FQ = reinterpret_cast<float2*>(p.d_FQ);
    const int nrows = p.K[0] * p.K[1], nc = sg.nc;
    const int zp = fft_row_pairs(p.K[2]);
    const int zblocks = ceil_div(ceil_div(nrows, 2), zp);
    const int yblocks = p.K[0] * ceil_div(nc, fft_lines_per_block(p.K[1]));
    const size_t zs = fft_smem_rows(p.K[2]), ys = fft_smem_lines(p.K[1]);
    const size_t xs = fft_smem_lines(p.K[0]);
    if (zp == 16)
      k_fft_r2c_z<16><<<zblocks, kFftThreads, zs, st>>>(p.d_Q, FQ, nrows, p.fax[2], nc,
                                                        p.d_tw[2]);
    else
      k_fft_r2c_z<8><<<zblocks, kFftThreads, zs, st>>>(p.d_Q, FQ, nrows, p.fax[2], nc,
                                                       p.d_tw[2]);
    k_fft_y<-1><<<yblocks, kFftThreads, ys, st>>>(FQ, p.K[1], nc, p.fax[1], p.d_tw[1]);
    if (need_virial)
      k_fft_x_influence<true><<<p.xblocks, kFftThreads, xs, st>>>(
          FQ, p.K[1], nc, p.fax[0], p.d_tw[0], sg, p.d_B[0], p.d_B[1], p.d_B[2],
          p.d_xpartial, need_energy);
    else
      k_fft_x_influence<false><<<p.xblocks, kFftThreads, xs, st>>>(
          FQ, p.K[1], nc, p.fax[0], p.d_tw[0], sg, p.d_B[0], p.d_B[1], p.d_B[2],
          p.d_xpartial, need_energy);
    if (need_energy || need_virial)
      k_pme_finish<<<1, 1024, 0, st>>>(p.xblocks, p.d_xpartial, p.d_frq, n, (double)p.beta,
                                       p.volume, p.d_sums, need_energy);
    k_fft_y<1><<<yblocks, kFftThreads, ys, st>>>(FQ, p.K[1], nc, p.fax[1], p.d_tw[1]);
    if (zp == 16)
      k_fft_c2r_z<16><<<zblocks, kFftThreads, zs, st>>>(FQ, p.d_phi, nrows, p.fax[2], nc,
                                                        p.d_tw[2]);
    else
      k_fft_c2r_z<8><<<zblocks, kFftThreads, zs, st>>>(FQ, p.d_phi, nrows, p.fax[2], nc,
                                                       p.d_tw[2]);
  } else if (batch) {
    for (auto& fg : p.groups)
      if (cufftExecR2C(fg.r2c, p.d_Q + fg.grid_begin, p.d_FQ + fg.spec_begin) !=
          CUFFT_SUCCESS)
        return fail(kCudaError, "PME: cufftExecR2C failed");
  } else if (cufftExecR2C(p.plan_r2c, p.d_Q, p.d_FQ) != CUFFT_SUCCESS) {
    return fail(kCudaError, "PME: cufftExecR2C failed");
  }
  if (batch) {
    if (need_virial)
      k_pme_influence<true, true><<<p.spec_blocks, kSpecBlock, 0, st>>>(
          p.nfft, sg, p.d_B[0], p.d_B[1], p.d_B[2], p.d_FQ, p.d_partial, need_energy,
          p.bv, p.d_spec_blocks);
    else
      k_pme_influence<false, true><<<p.spec_blocks, kSpecBlock, 0, st>>>(
          p.nfft, sg, p.d_B[0], p.d_B[1], p.d_B[2], p.d_FQ, p.d_partial, need_energy,
          p.bv, p.d_spec_blocks);
    if (need_energy || need_virial) {
      k_pme_finish_batch<<<p.bv.nsys, 256, 0, st>>>(p.bv, p.d_sys_block_begin, p.d_partial,
                                                    p.d_frq, (double)p.beta, p.d_sys_sums,
                                                    need_energy);
      k_pme_sum_systems<<<1, 32, 0, st>>>(p.bv.nsys, p.d_sys_sums, p.d_sums);
    }
    for (auto& fg : p.groups)
      if (cufftExecC2R(fg.c2r, p.d_FQ + fg.spec_begin, p.d_phi + fg.grid_begin) !=
          CUFFT_SUCCESS)
        return fail(kCudaError, "PME: cufftExecC2R failed");
    const int gt = p.gather_threads;  // 4 lanes per atom
    k_pme_gather<kAccumFixed, true><<<ceil_div(n, gt / 4), gt, 0, st>>>(
        n, p.d_frq, p.d_upk, g, p.d_phi, 1.0f, acc, p.bv);
    SNB_CUDA_TRY(cudaGetLastError());
    return kOk;
  }
  if (!p.own_fft) {
    if (need_virial)
      k_pme_influence<true, false><<<p.partial_blocks, kSpecBlock, 0, st>>>(
          p.nfft, sg, p.d_B[0], p.d_B[1], p.d_B[2], p.d_FQ, p.d_partial, need_energy, p.bv,
          nullptr);
    else
      k_pme_influence<false, false><<<p.partial_blocks, kSpecBlock, 0, st>>>(
          p.nfft, sg, p.d_B[0], p.d_B[1], p.d_B[2], p.d_FQ, p.d_partial, need_energy, p.bv,
          nullptr);
    if (need_energy || need_virial)
      k_pme_finish<<<1, 1024, 0, st>>>(p.partial_blocks, p.d_partial, p.d_frq, n,
                                       (double)p.beta, p.volume, p.d_sums, need_energy);
    if (cufftExecC2R(p.plan_c2r, p.d_FQ, p.d_phi) != CUFFT_SUCCESS)
      return fail(kCudaError, "PME: cufftExecC2R failed");
  }
  const float scale = (float)p.update_interval;
  const int gt = p.gather_threads;  // 4 lanes per atom
  if (accum == kAccumFixed)
    k_pme_gather<kAccumFixed, false><<<ceil_div(n, gt / 4), gt, 0, st>>>(
        n, p.d_frq, p.d_upk, g, p.d_phi, scale, acc, p.bv);
  else
    k_pme_gather<kAccumFloat, false><<<ceil_div(n, gt / 4), gt, 0, st>>>(
        n, p.d_frq, p.d_upk, g, p.d_phi, scale, acc, p.bv);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int pme_reciprocal(PME& p, const float4* pos, int n, Accumulators& acc, int accum,
                   bool need_energy, bool need_virial, cudaStream_t st) {
  if (n != p.n) return fail(kBadInput, "PME: atom count differs from Initial");
  TileGeom g{p.K[0], p.K[1], p.K[2], p.T, p.nt[0], p.nt[1], p.nt[2], p.rcell};
  k_pme_bin<<<ceil_div(n, 256), 256, 0, st>>>(n, pos, g, p.d_atom_tile, p.d_atom_slot,
                                              p.d_tile_count, p.d_frq, p.d_upk);
  return pme_after_bin(p, n, acc, accum, need_energy, need_virial, st);
}

// ---------------------------------------------------------------------------
// Excluded-pair correction: removes the reciprocal-space interaction of the
// excluded pairs (MPI_PME_Excluded_Force_With_Atom_Energy_Correction,
// PM_force.cpp:1745-1817, factor 1 for one process):
//   F/r = -q_i q_j ((2 beta r/sqrt(pi) e^{-b^2r^2} + erfc(beta r)) - 1)/r^3,
//   E_i -= q_i q_j erf(beta r)/r, virial_i -= (F/r) dr (x) dr.
template <int ACCUM, bool ENERGY, bool VIRIAL, bool BATCH>
__global__ void k_excluded(int n, const float3* __restrict__ crd,
                           const float* __restrict__ charge, Cell cell, Cell rcell,
                           float beta, const int* __restrict__ excl_start,
                           const int* __restrict__ excl_list,
                           const int* __restrict__ excl_numbers,
                           const int* __restrict__ map, Accumulators acc, BatchView bv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int cnt = excl_numbers[i];
  if (cnt <= 0) return;
  if (BATCH) {  // excluded pairs never cross systems
    const SysGeom& sg = bv.sys[bv.sys_of[i]];
    cell = sg.cell;
    rcell = sg.rcell;
  }
  const int N = acc.n;
  int st = excl_start[i];
  float3 ri = crd[i];
  float qi = charge[i];
  float fx = 0.f, fy = 0.f, fz = 0.f, e = 0.f;
  float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int k = st; k < st + cnt; ++k) {
    int j = excl_list[k];
    if ((unsigned)j >= (unsigned)n) continue;  // malformed list entry
    float3 d = min_image_fast<false>(crd[j], ri, cell, rcell);
    float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
    float r = sqrtf(r2);
    float br = beta * r;
    float fs = br * 1.1283791670955126f * expf(-br * br) + erfcf(br);
    fs = -qi * charge[j] * ((fs - 1.0f) / r2 / r);
    float gx = fs * d.x, gy = fs * d.y, gz = fs * d.z;
    fx += gx;
    fy += gy;
    fz += gz;
    int sj = map ? map[j] : j;
    if (ACCUM == kAccumFixed) {
      red_add(acc.d_f + sj, -to_fixed_force(gx));
      red_add(acc.d_f + N + sj, -to_fixed_force(gy));
      red_add(acc.d_f + 2 * N + sj, -to_fixed_force(gz));
    } else {
      atomicAdd(acc.d_ff + sj, -gx);
      atomicAdd(acc.d_ff + N + sj, -gy);
      atomicAdd(acc.d_ff + 2 * N + sj, -gz);
    }
    if (ENERGY) e -= qi * charge[j] * erff(br) / r;
    if (VIRIAL) {
      v[0] -= gx * d.x;
      v[1] -= gx * d.y + gy * d.x;
      v[2] -= gy * d.y;
      v[3] -= gx * d.z + gz * d.x;
      v[4] -= gy * d.z + gz * d.y;
      v[5] -= gz * d.z;
    }
  }
  int si = map ? map[i] : i;
  if (ACCUM == kAccumFixed) {
    red_add(acc.d_f + si, to_fixed_force(fx));
    red_add(acc.d_f + N + si, to_fixed_force(fy));
    red_add(acc.d_f + 2 * N + si, to_fixed_force(fz));
    if (ENERGY) red_add(acc.d_e + si, to_fixed_energy(e));
    if (VIRIAL)
      for (int c = 0; c < 6; ++c) red_add(acc.d_v + c * N + si, to_fixed_energy(v[c]));
  } else {
    atomicAdd(acc.d_ff + si, fx);
    atomicAdd(acc.d_ff + N + si, fy);
    atomicAdd(acc.d_ff + 2 * N + si, fz);
    if (ENERGY) atomicAdd(acc.d_fe + si, e);
    if (VIRIAL)
      for (int c = 0; c < 6; ++c) atomicAdd(acc.d_fv + c * N + si, v[c]);
  }
}

template <int ACCUM, bool BATCH>
static void launch_excl2(int n, const float3* crd, const float* charge,
                         const Cell& cell, const Cell& rcell, float beta,
                         const int* es, const int* el, const int* en, const int* map,
                         Accumulators& acc, bool energy, bool virial, const BatchView& bv,
                         cudaStream_t st) {
  dim3 g(ceil_div(n, 256)), b(256);
  if (energy && virial)
    k_excluded<ACCUM, true, true, BATCH><<<g, b, 0, st>>>(n, crd, charge, cell, rcell, beta,
                                                         es, el, en, map, acc, bv);
  else if (energy)
    k_excluded<ACCUM, true, false, BATCH><<<g, b, 0, st>>>(n, crd, charge, cell, rcell,
                                                          beta, es, el, en, map, acc, bv);
  else if (virial)
    k_excluded<ACCUM, false, true, BATCH><<<g, b, 0, st>>>(n, crd, charge, cell, rcell,
                                                          beta, es, el, en, map, acc, bv);
  else
    k_excluded<ACCUM, false, false, BATCH><<<g, b, 0, st>>>(n, crd, charge, cell, rcell,
                                                           beta, es, el, en, map, acc, bv);
}

int launch_excluded(int n, const float3* crd, const float* charge, const Cell& cell,
                    const Cell& rcell, float beta, const int* excl_start,
                    const int* excl_list, const int* excl_numbers, const int* map,
                    Accumulators& acc, int accum, bool energy, bool virial,
                    cudaStream_t st, const BatchView& bv) {
  if (n <= 0 || !excl_numbers) return kOk;
  if (bv.nsys > 0) {
    if (accum != kAccumFixed) return fail(kNotSupported, "batch: fixed-point only");
    launch_excl2<kAccumFixed, true>(n, crd, charge, cell, rcell, beta, excl_start,
                                    excl_list, excl_numbers, map, acc, energy, virial, bv,
                                    st);
  } else if (accum == kAccumFixed) {
    launch_excl2<kAccumFixed, false>(n, crd, charge, cell, rcell, beta, excl_start,
                                     excl_list, excl_numbers, map, acc, energy, virial, bv,
                                     st);
  } else {
    launch_excl2<kAccumFloat, false>(n, crd, charge, cell, rcell, beta, excl_start,
                                     excl_list, excl_numbers, map, acc, energy, virial, bv,
                                     st);
  }
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace snb
