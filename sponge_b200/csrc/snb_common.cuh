// Shared device helpers for the sm_100a nonbonded kernels.
//
// Conventions (SPONGE internal units, SPONGE/common.h):
//   length Angstrom, energy kcal/mol, charge pre-scaled by 18.2223,
//   LJ pair tables A' = 12*A, B' = 6*B indexed by Get_LJ_Type
//   (Lennard_Jones_force.h:19-28), box and virial as LTMatrix3
//   {a11, a21, a22, a31, a32, a33} (utils/vector.hpp:249).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace snb {

// Fixed-point scales.  Forces: 2^40 units per kcal/mol/A (|F| < 8.4e6 per
// atom).  Energies and virials: 2^32 units per kcal/mol (|E| < 2.1e9 for the
// whole box), so per-atom values and box totals both fit in int64.
constexpr double kForceScale = 1099511627776.0;        // 2^40
constexpr double kForceScaleInv = 1.0 / 1099511627776.0;
constexpr double kEnergyScale = 4294967296.0;          // 2^32
constexpr double kEnergyScaleInv = 1.0 / 4294967296.0;
constexpr float kForceScaleF = 1099511627776.0f;
constexpr float kEnergyScaleF = 4294967296.0f;
// PME charge grid accumulated in int32 inside shared memory: 2^22 units per
// (charge unit), |Q(g)| must stay below 512 (18.2223-scaled charges).
constexpr float kGridScale = 4194304.0f;               // 2^22
constexpr float kGridScaleInv = 1.0f / 4194304.0f;

struct Cell {
  float a11, a21, a22, a31, a32, a33;
};

__host__ __device__ __forceinline__ Cell make_cell(const float* c) {
  Cell r;
  r.a11 = c[0]; r.a21 = c[1]; r.a22 = c[2];
  r.a31 = c[3]; r.a32 = c[4]; r.a33 = c[5];
  return r;
}

// Minimum image exactly as the reference writes it (utils/boundary.h:31),
// dr = a - b; dr - floorf(dr*rcell + 0.5f)*cell, every product and sum
// rounded separately (no FMA contraction).  Used where results must match
// the reference bit for bit: the neighbor-pair criterion.
__device__ __forceinline__ float3 min_image_exact(float3 a, float3 b,
                                                  const Cell& cell,
                                                  const Cell& rcell) {
  float dx = __fsub_rn(a.x, b.x);
  float dy = __fsub_rn(a.y, b.y);
  float dz = __fsub_rn(a.z, b.z);
  float sx = __fadd_rn(__fadd_rn(__fmul_rn(dx, rcell.a11), __fmul_rn(dy, rcell.a21)),
                       __fmul_rn(dz, rcell.a31));
  float sy = __fadd_rn(__fmul_rn(dy, rcell.a22), __fmul_rn(dz, rcell.a32));
  float sz = __fmul_rn(dz, rcell.a33);
  float fx = floorf(__fadd_rn(sx, 0.5f));
  float fy = floorf(__fadd_rn(sy, 0.5f));
  float fz = floorf(__fadd_rn(sz, 0.5f));
  float cx = __fadd_rn(__fadd_rn(__fmul_rn(fx, cell.a11), __fmul_rn(fy, cell.a21)),
                       __fmul_rn(fz, cell.a31));
  float cy = __fadd_rn(__fmul_rn(fy, cell.a22), __fmul_rn(fz, cell.a32));
  float cz = __fmul_rn(fz, cell.a33);
  return make_float3(__fsub_rn(dx, cx), __fsub_rn(dy, cy), __fsub_rn(dz, cz));
}

// min_image_exact for a rectangular box, given dr = a - b.  The off-diagonal
// entries of cell and rcell are zero, so the general form only adds signed
// zeros to each sum; that can turn a -0 into +0 but never changes floorf of
// (s + 0.5) or the square of any component, so |dr|^2 is bit-identical.
__device__ __forceinline__ float3 min_image_exact_rect(float dx, float dy, float dz,
                                                       const Cell& cell,
                                                       const Cell& rcell) {
  const float fx = floorf(__fadd_rn(__fmul_rn(dx, rcell.a11), 0.5f));
  const float fy = floorf(__fadd_rn(__fmul_rn(dy, rcell.a22), 0.5f));
  const float fz = floorf(__fadd_rn(__fmul_rn(dz, rcell.a33), 0.5f));
  return make_float3(__fsub_rn(dx, __fmul_rn(fx, cell.a11)),
                     __fsub_rn(dy, __fmul_rn(fy, cell.a22)),
                     __fsub_rn(dz, __fmul_rn(fz, cell.a33)));
}

// |dr|^2 in the reference's operator order ((x*x + y*y) + z*z), unfused.
__device__ __forceinline__ float norm2_exact(float3 d) {
  return __fadd_rn(__fadd_rn(__fmul_rn(d.x, d.x), __fmul_rn(d.y, d.y)),
                   __fmul_rn(d.z, d.z));
}

// Minimum image of a rectangular box for force evaluation, on the FMA pipe:
// k = round(d / L) by the 1.5*2^23 shift (exact for |d / L| < 2^22), then
// d - k L.  It differs from floor(s + 0.5) only when d is an odd multiple of
// half a box length: both images are then equally far, and with a cutoff
// below half the box (the condition for the minimum image to be the only
// image in range) the pair is beyond the cutoff.
__device__ __forceinline__ float min_image_axis(float d, float L, float rL) {
  const float k = __fsub_rn(__fmaf_rn(d, rL, 12582912.0f), 12582912.0f);
  return __fmaf_rn(-k, L, d);
}

// Fast minimum image for force evaluation, contraction allowed.  ORTHO: a
// rectangular box, rounded per axis by min_image_axis; otherwise the
// reference's floor(s + 0.5) on the full cell.
template <bool ORTHO>
__device__ __forceinline__ float3 min_image_fast(float3 a, float3 b,
                                                 const Cell& cell,
                                                 const Cell& rcell) {
  float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  if (ORTHO) {
    dx = min_image_axis(dx, cell.a11, rcell.a11);
    dy = min_image_axis(dy, cell.a22, rcell.a22);
    dz = min_image_axis(dz, cell.a33, rcell.a33);
  } else {
    float sx = dx * rcell.a11 + dy * rcell.a21 + dz * rcell.a31;
    float sy = dy * rcell.a22 + dz * rcell.a32;
    float sz = dz * rcell.a33;
    float fx = floorf(sx + 0.5f), fy = floorf(sy + 0.5f), fz = floorf(sz + 0.5f);
    dx -= fx * cell.a11 + fy * cell.a21 + fz * cell.a31;
    dy -= fy * cell.a22 + fz * cell.a32;
    dz -= fz * cell.a33;
  }
  return make_float3(dx, dy, dz);
}

// Start pulling [p, p + bytes) into L2 (bytes a multiple of 16, p 16-byte
// aligned); a hint with no completion to wait for.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes)
               : "memory");
}

// Triangular LJ pair index, Get_LJ_Type (Lennard_Jones_force.h:19-28).
__host__ __device__ __forceinline__ int lj_pair_index(int a, int b) {
  int hi = a > b ? a : b, lo = a > b ? b : a;
  return ((hi * (hi + 1)) >> 1) + lo;
}

__device__ __forceinline__ long long to_fixed_force(float f) {
  return __float2ll_rn(f * kForceScaleF);
}
__device__ __forceinline__ long long to_fixed_energy(float e) {
  return __float2ll_rn(e * kEnergyScaleF);
}
__device__ __forceinline__ void red_add(long long* p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long*>(p),
            static_cast<unsigned long long>(v));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// erfc(x) and exp(-x^2) together for x >= 0.  erfcx(x) = erfc(x) e^{x^2} is
// a degree-8 polynomial in t = 1/(1 + x/2) on [0, 4] (weighted least-squares
// fit against double-precision erfcx; max relative error 3.3e-7 in float32), so
// erfc(x) = P(t) * exp(-x^2).  exp uses the hardware exp2 (__expf: error
// 2 + 1.16|x^2| ulp; measured 8.9e-7 relative at most on [0, 3], the range
// beta r takes below the cutoff); t uses the fast hardware division (2 ulp;
// |t P'(t) / P(t)| <= 2.26 on the range, so P moves by at most 5.4e-7
// relative through it).  Together erfc is within 1.01e-6 of double
// precision on [0, 3] (measured on B200), CUDA's erfcf within 2.9e-7.
// Beyond x = 4 CUDA's erfcf and expf are used.
__device__ __forceinline__ float erfc_and_exp(float x, float* e_out) {
  if (x > 4.0f) {
    *e_out = expf(-x * x);
    return erfcf(x);
  }
  const float e = __expf(-x * x);
  *e_out = e;
  const float t = __fdividef(1.0f, 1.0f + 0.5f * x);
  float p = -0.049221702f;
  p = fmaf(p, t, 0.33589873f);
  p = fmaf(p, t, -0.88379663f);
  p = fmaf(p, t, 1.0076897f);
  p = fmaf(p, t, -0.39945206f);
  p = fmaf(p, t, 0.47237507f);
  p = fmaf(p, t, 0.22729602f);
  p = fmaf(p, t, 0.2896666f);
  p = fmaf(p, t, -0.00045567533f);
  return p * e;
}

// atomicAdd(&counter[key], 1) with the lanes of a warp that share the same
// key served by one atomic (leader adds the group size, ranks follow lane
// order).  Call with all lanes of the warp active.
__device__ __forceinline__ int warp_aggregated_inc(int* counter, int key, bool active) {
  const unsigned act = __ballot_sync(0xffffffffu, active);
  if (!active) return 0;
  const unsigned peers = __match_any_sync(act, key);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  const int rank = __popc(peers & ((1u << lane) - 1u));
  int base = 0;
  if (lane == leader) base = atomicAdd(&counter[key], __popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + rank;
}

// Ceiling division for launch shapes.
__host__ __device__ __forceinline__ int ceil_div(long long a, int b) {
  return static_cast<int>((a + b - 1) / b);
}

}  // namespace snb
