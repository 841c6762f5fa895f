// Kernels around the nonbonded path that the fused engine needs: harmonic
// bonds and angles, leap-frog integration straight from the fixed-point
// accumulator, energy / virial totals, and small scalar adds.
//
// Bonds follow BOND (bond.cpp:14-60): E = k (r - r0)^2, f_i = -2k(r-r0)/r dr,
// dr = r_i - r_j.  Angles follow ANGLE (angle.cpp:8-70): E = k (theta -
// theta0)^2.  Leap-frog follows MD_Iteration_Leap_Frog (MD_core/nve.hpp:3-16):
// v += dt F/m, x += dt v.
#include <algorithm>

#include "snb_internal.h"

namespace snb {

__device__ __forceinline__ void acc_force(Accumulators& acc, int s, float fx, float fy,
                                          float fz) {
  const int N = acc.n;
  red_add(acc.d_f + s, to_fixed_force(fx));
  red_add(acc.d_f + N + s, to_fixed_force(fy));
  red_add(acc.d_f + 2 * N + s, to_fixed_force(fz));
}

// Bonds and angles in one launch: the first ceil(nb/256) blocks take bonds.
template <bool BATCH>
__global__ void k_bonded(int nb, const int* __restrict__ ba, const int* __restrict__ bb,
                         const float* __restrict__ bk, const float* __restrict__ br0,
                         int na, const int* __restrict__ aa, const int* __restrict__ ab,
                         const int* __restrict__ ac, const float* __restrict__ ak,
                         const float* __restrict__ at0, const float3* __restrict__ crd,
                         Cell cell, Cell rcell, const int* __restrict__ map,
                         Accumulators acc, long long* __restrict__ e_total, bool energy,
                         int bond_blocks, BatchView bv) {
  if ((int)blockIdx.x < bond_blocks) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    int i = ba[t], j = bb[t];
    if (BATCH) {  // bonded terms never cross systems
      const SysGeom& sg = bv.sys[bv.sys_of[i]];
      cell = sg.cell;
      rcell = sg.rcell;
    }
    float3 d = min_image_fast<false>(crd[i], crd[j], cell, rcell);
    float r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
    float dr = r - br0[t];
    float s = -2.0f * dr * bk[t] / r;
    int si = map ? map[i] : i, sj = map ? map[j] : j;
    acc_force(acc, si, s * d.x, s * d.y, s * d.z);
    acc_force(acc, sj, -s * d.x, -s * d.y, -s * d.z);
    if (energy) red_add(e_total, to_fixed_energy(bk[t] * dr * dr));
    return;
  }
  int t = (blockIdx.x - bond_blocks) * blockDim.x + threadIdx.x;
  if (t >= na) return;
  int i = aa[t], j = ab[t], l = ac[t];
  if (BATCH) {
    const SysGeom& sg = bv.sys[bv.sys_of[j]];
    cell = sg.cell;
    rcell = sg.rcell;
  }
  float3 dij = min_image_fast<false>(crd[i], crd[j], cell, rcell);
  float3 dkj = min_image_fast<false>(crd[l], crd[j], cell, rcell);
  float rij2 = 1.0f / (dij.x * dij.x + dij.y * dij.y + dij.z * dij.z);
  float rkj2 = 1.0f / (dkj.x * dkj.x + dkj.y * dkj.y + dkj.z * dkj.z);
  float rr = sqrtf(rij2 * rkj2);
  float c = (dij.x * dkj.x + dij.y * dkj.y + dij.z * dkj.z) * rr;
  c = fmaxf(-0.999999f, fminf(c, 0.999999f));
  float th = acosf(c);
  float dth = th - at0[t];
  float kk = -2.0f * ak[t] * dth / sinf(th);
  float cross = kk * rr, self = kk * c;
  float3 fi = make_float3(self * rij2 * dij.x - cross * dkj.x,
                          self * rij2 * dij.y - cross * dkj.y,
                          self * rij2 * dij.z - cross * dkj.z);
  float3 fk = make_float3(self * rkj2 * dkj.x - cross * dij.x,
                          self * rkj2 * dkj.y - cross * dij.y,
                          self * rkj2 * dkj.z - cross * dij.z);
  int si = map ? map[i] : i, sj = map ? map[j] : j, sk = map ? map[l] : l;
  acc_force(acc, si, fi.x, fi.y, fi.z);
  acc_force(acc, sk, fk.x, fk.y, fk.z);
  acc_force(acc, sj, -fi.x - fk.x, -fi.y - fk.y, -fi.z - fk.z);
  if (energy) red_add(e_total, to_fixed_energy(ak[t] * dth * dth));
}

int launch_bonded(int nb, const int* ba, const int* bb, const float* bk,
                  const float* br0, int na, const int* aa, const int* ab,
                  const int* ac, const float* ak, const float* at0,
                  const float3* crd, const Cell& cell, const Cell& rcell,
                  const int* map, Accumulators& acc, long long* e_total,
                  bool energy, cudaStream_t st, const BatchView& bv) {
  const int bblocks = nb > 0 ? ceil_div(nb, 256) : 0;
  const int ablocks = na > 0 ? ceil_div(na, 256) : 0;
  if (bblocks + ablocks == 0) return kOk;
  if (bv.nsys > 0)
    k_bonded<true><<<bblocks + ablocks, 256, 0, st>>>(nb, ba, bb, bk, br0, na, aa, ab, ac,
                                                     ak, at0, crd, cell, rcell, map, acc,
                                                     e_total, energy, bblocks, bv);
  else
    k_bonded<false><<<bblocks + ablocks, 256, 0, st>>>(nb, ba, bb, bk, br0, na, aa, ab, ac,
                                                      ak, at0, crd, cell, rcell, map, acc,
                                                      e_total, energy, bblocks, bv);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Leap-frog from the fixed-point accumulator (sorted frame via map); the
// launch then clears the accumulator for the next step.
// When old_crd is given, also performs the refresh check of the next step
// (Check_Refresh, neighbor_list.cpp:307-321) on the new coordinates and
// raises flags[0] if any atom moved more than sqrt(permit2) since the build;
// with pc.ref, the pruned rows' check likewise.
template <bool BATCH>
__global__ void k_leap_frog(int n, const int* __restrict__ map, Accumulators acc,
                            float3* __restrict__ crd, float3* __restrict__ vel,
                            const float* __restrict__ inv_mass, float dt,
                            const float3* __restrict__ old_crd, Cell cell, Cell rcell,
                            float permit2, int* __restrict__ flags, BatchView bv,
                            PruneCheck pc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // every load is issued before the first store: the force reads wait on the
  // permutation, the rest do not
  const int s = map[i];
  const float im = inv_mass[i];
  float3 v = vel[i];
  float3 r = crd[i];
  float3 r_old = make_float3(0.f, 0.f, 0.f);
  if (old_crd) r_old = old_crd[i];
  const int N = acc.n;
  const long long* __restrict__ f = acc.d_f;
  const long long fx_i = f[s], fy_i = f[N + s], fz_i = f[2 * N + s];
  const float fx = (float)((double)fx_i * kForceScaleInv);
  const float fy = (float)((double)fy_i * kForceScaleInv);
  const float fz = (float)((double)fz_i * kForceScaleInv);
  v.x += dt * (im * fx);
  v.y += dt * (im * fy);
  v.z += dt * (im * fz);
  vel[i] = v;
  r.x += dt * v.x;
  r.y += dt * v.y;
  r.z += dt * v.z;
  crd[i] = r;
  if (BATCH && (old_crd || pc.ref)) {  // the atom's own box
    const SysGeom& sg = bv.sys[bv.sys_of[i]];
    cell = sg.cell;
    rcell = sg.rcell;
  }
  if (old_crd) {
    float3 d = min_image_fast<false>(r, r_old, cell, rcell);
    const float d2 = d.x * d.x + d.y * d.y + d.z * d.z;
    bool moved = d2 > permit2;
    if (BATCH && bv.box_need) box_mark(bv.box_need, bv.sys_of[i], d2, permit2);
    if (__any_sync(__activemask(), moved) && moved) atomicExch(&flags[0], 1);
  }
  if (pc.ref) {
    const float4 q = pc.ref[s];
    const float3 d = min_image_fast<false>(r, make_float3(q.x, q.y, q.z), cell, rcell);
    const bool far = d.x * d.x + d.y * d.y + d.z * d.z > pc.permit2;
    if (__any_sync(__activemask(), far) && far) atomicExch(pc.flag, 1);
  }
}

template <bool BATCH>
__global__ void k_prune_check(int n, const float3* __restrict__ crd,
                              const int* __restrict__ map, PruneCheck pc, Cell cell,
                              Cell rcell, BatchView bv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (BATCH) {
    const SysGeom& sg = bv.sys[bv.sys_of[i]];
    cell = sg.cell;
    rcell = sg.rcell;
  }
  const float4 q = pc.ref[map[i]];
  const float3 d = min_image_fast<false>(crd[i], make_float3(q.x, q.y, q.z), cell, rcell);
  const bool far = d.x * d.x + d.y * d.y + d.z * d.z > pc.permit2;
  if (__any_sync(__activemask(), far) && far) atomicExch(pc.flag, 1);
}

int launch_prune_check(int n, const float3* crd, const int* map, const PruneCheck& pc,
                       const Cell& cell, const Cell& rcell, cudaStream_t st,
                       const BatchView& bv) {
  if (!pc.ref) return kOk;
  if (bv.nsys > 0)
    k_prune_check<true><<<ceil_div(n, 256), 256, 0, st>>>(n, crd, map, pc, cell, rcell, bv);
  else
    k_prune_check<false><<<ceil_div(n, 256), 256, 0, st>>>(n, crd, map, pc, cell, rcell, bv);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int launch_leap_frog(int n, const int* map, Accumulators& acc, float3* crd,
                     float3* vel, const float* inv_mass, float dt,
                     const float3* old_crd, const Cell& cell, const Cell& rcell,
                     float permit2, int* flags, cudaStream_t st, const BatchView& bv,
                     const PruneCheck& pc) {
  if (bv.nsys > 0)
    k_leap_frog<true><<<ceil_div(n, 256), 256, 0, st>>>(n, map, acc, crd, vel, inv_mass, dt,
                                                      old_crd, cell, rcell, permit2, flags,
                                                      bv, pc);
  else
    k_leap_frog<false><<<ceil_div(n, 256), 256, 0, st>>>(n, map, acc, crd, vel, inv_mass,
                                                       dt, old_crd, cell, rcell, permit2,
                                                       flags, bv, pc);
  SNB_CUDA_TRY(cudaGetLastError());
  // the accumulator starts the next step at zero: one coalesced clear
  // instead of scattered stores through the permutation
  SNB_CUDA_TRY(cudaMemsetAsync(acc.d_f, 0, sizeof(long long) * 3 * (size_t)acc.n, st));
  return kOk;
}

// Sum per-atom fixed-point energies / virials: out[0..2] = e, elj, ec,
// out[3..8] = virial.  int64 adds are order-independent.
__global__ void k_sum_acc(int n, Accumulators acc, long long* __restrict__ out,
                          bool energy, bool virial) {
  long long v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int N = acc.n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    if (energy) {
      v[0] += acc.d_e[i];
      v[1] += acc.d_elj[i];
      v[2] += acc.d_ec[i];
    }
    if (virial)
      for (int c = 0; c < 6; ++c) v[3 + c] += acc.d_v[c * N + i];
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    long long x = v[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x != 0) red_add(out + c, x);
  }
}

// totals[0..13] from the integer sums, the PME sums and the tail correction.
__global__ void k_totals(const long long* __restrict__ isum,
                         const long long* __restrict__ bonded,
                         const double* __restrict__ pme_sums, double lrc_energy,
                         double lrc_virial, double* __restrict__ totals, bool energy,
                         bool virial, bool have_pme) {
  if (threadIdx.x != 0) return;
  const double s = kEnergyScaleInv;
  if (energy) {
    double e = isum[0] * s, elj = isum[1] * s, ec = isum[2] * s;
    totals[0] = elj;
    totals[1] = lrc_energy;
    totals[2] = ec;
    totals[3] = e - elj - ec;
    totals[4] = have_pme ? pme_sums[0] : 0.0;
    totals[5] = have_pme ? pme_sums[7] : 0.0;
    totals[6] = bonded ? bonded[0] * s : 0.0;
    totals[7] = totals[0] + totals[1] + totals[2] + totals[3] + totals[4] + totals[5] +
                totals[6];
  }
  if (virial) {
    for (int c = 0; c < 6; ++c)
      totals[8 + c] = isum[3 + c] * s + (have_pme ? pme_sums[1 + c] : 0.0);
    totals[8] += lrc_virial;
    totals[10] += lrc_virial;
    totals[13] += lrc_virial;
  }
}

int launch_totals(int n, Accumulators& acc, long long* isum, const long long* bonded,
                  const double* pme_sums, double lrc_energy, double lrc_virial,
                  double* totals, bool energy, bool virial, bool have_pme,
                  cudaStream_t st) {
  SNB_CUDA_TRY(cudaMemsetAsync(isum, 0, sizeof(long long) * 9, st));
  k_sum_acc<<<std::min(ceil_div(n, 256), 148 * 4), 256, 0, st>>>(n, acc, isum, energy,
                                                                 virial);
  k_totals<<<1, 32, 0, st>>>(isum, bonded, pme_sums, lrc_energy, lrc_virial, totals,
                             energy, virial, have_pme);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Stress and pressure (MD_INFORMATION::Get_pressure, MD_core.cpp:1080-1107,
// with Get_Stress_Potential_Contribution / Get_Stress_Kinetic_Contribution,
// MD_core/sys.hpp:14-85): stress = (virial + sum_i m_i v_i (x) v_i) / V,
// LTMatrix3 order with the off-diagonal pairs summed; pressure = trace / 3.
// out[0..5] = stress (kcal/mol/A^3), out[6] = pressure in bar.
__global__ void k_kinetic_stress(int n, const float3* __restrict__ vel,
                                 const float* __restrict__ mass, double* __restrict__ acc) {
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float3 v = vel[i];
    const double m = mass[i];
    s[0] += m * v.x * v.x;
    s[1] += m * 2.0 * v.x * v.y;
    s[2] += m * v.y * v.y;
    s[3] += m * 2.0 * v.x * v.z;
    s[4] += m * 2.0 * v.y * v.z;
    s[5] += m * v.z * v.z;
  }
  __shared__ double sh[6][32];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double x = warp_sum(s[c]);
    if ((threadIdx.x & 31) == 0) sh[c][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double x = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += sh[threadIdx.x][w];
    atomicAdd(acc + threadIdx.x, x);
  }
}

__global__ void k_pressure(const double* __restrict__ kin, const double* __restrict__ virial,
                           const long long* __restrict__ constraint_virial, double inv_v,
                           double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double tr = 0.0;
  for (int c = 0; c < 6; ++c) {
    double w = virial ? virial[c] : 0.0;
    if (constraint_virial) w += (double)constraint_virial[c] * kEnergyScaleInv;
    out[c] = (w + kin[c]) * inv_v;
  }
  tr = out[0] + out[2] + out[5];
  out[6] = tr / 3.0 * 6.946827162543585e4;  // kcal/mol/A^3 -> bar
}

int launch_pressure(int n, const float3* vel, const float* mass, const double* virial,
                    const long long* constraint_virial, double inv_v, double* scratch6,
                    double* out, cudaStream_t st) {
  SNB_CUDA_TRY(cudaMemsetAsync(scratch6, 0, sizeof(double) * 6, st));
  k_kinetic_stress<<<std::max(1, std::min(ceil_div(n, 256), 148 * 4)), 256, 0, st>>>(
      n, vel, mass, scratch6);
  k_pressure<<<1, 32, 0, st>>>(scratch6, virial, constraint_virial, inv_v, out);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// d_potential[0] += e; d_virial[0..5] += v (reference folds global terms into
// slot 0 of the per-atom arrays, main.cpp:1473-1483,1541-1544).
__global__ void k_add_scalars(float* d_potential, float* d_virial,
                              const double* __restrict__ sums, float lrc_e,
                              float lrc_v, int mode) {
  if (threadIdx.x != 0) return;
  if (mode == 0) {  // PME: sums[0] recip, sums[7] self, sums[1..6] virial
    if (d_potential) d_potential[0] += (float)(sums[0] + sums[7]);
    if (d_virial)
      for (int c = 0; c < 6; ++c) d_virial[c] += (float)sums[1 + c];
  } else {  // LJ tail correction
    if (d_potential) d_potential[0] += lrc_e;
    if (d_virial) {
      d_virial[0] += lrc_v;
      d_virial[2] += lrc_v;
      d_virial[5] += lrc_v;
    }
  }
}

int launch_add_scalars(float* d_potential, float* d_virial, const double* sums,
                       float lrc_e, float lrc_v, int mode, cudaStream_t st) {
  k_add_scalars<<<1, 32, 0, st>>>(d_potential, d_virial, sums, lrc_e, lrc_v, mode);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// Sum of a float array in FP64 (Step_Print sums).
__global__ void k_sum_float(int n, const float* __restrict__ x, double* out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
  s = warp_sum(s);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    *out = t;
  }
}

int launch_sum_float(int n, const float* x, double* out, cudaStream_t st) {
  k_sum_float<<<1, 1024, 0, st>>>(n, x, out);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

__global__ void k_gather_type(int n, const int* __restrict__ src,
                              const int* __restrict__ atom_local, int* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[atom_local ? atom_local[i] : i];
}

int launch_gather_type(int n, const int* src, const int* atom_local, int* dst,
                       cudaStream_t st) {
  k_gather_type<<<ceil_div(n, 256), 256, 0, st>>>(n, src, atom_local, dst);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace snb
