// 1-4 nonbonded terms (NON_BOND_14, nb14/nb14.h, nb14/nb14.cpp:8-103):
// for each listed pair (a, b), r = |r_b - r_a| (minimum image),
//   F/r = -A' r^-14 + B' r^-8 - c q_a q_b r^-3,
//   E_LJ = A'/12 r^-12 - B'/6 r^-6,  E_CF = c q_a q_b / r,
// with A', B' the pair's scaled LJ table entries and c its Coulomb scale;
// a charge below 1e-10 in magnitude is taken as 1e-10, as the reference
// does.  Energy and virial go to atom a.  One thread per pair; forces,
// energies and virials accumulate in the fixed-point accumulators (at
// map[atom] when a frame map is given).  sums, when given, receives the
// totals {LJ + Coulomb, Coulomb}.
#include <vector>

#include "snb_internal.h"

namespace snb {

template <bool ENERGY, bool VIRIAL>
__global__ void k_nb14(int m, const int* __restrict__ ia, const int* __restrict__ ib,
                       const float* __restrict__ A, const float* __restrict__ B,
                       const float* __restrict__ cf, const float3* __restrict__ crd,
                       const float* __restrict__ charge, Cell cell, Cell rcell,
                       const int* __restrict__ map, Accumulators acc, bool per_atom,
                       long long* __restrict__ sums) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const int a0 = ia[t], b0 = ib[t];
  const int a = map ? map[a0] : a0, b = map ? map[b0] : b0;
  const float3 d = min_image_fast<false>(crd[b0], crd[a0], cell, rcell);
  const float r2 = d.x * d.x + d.y * d.y + d.z * d.z;
  const float ir2 = 1.0f / r2;
  const float ir4 = ir2 * ir2, ir8 = ir4 * ir4, ir14 = ir8 * ir4 * ir2;
  const float ir = rsqrtf(r2);
  float qa = charge[a0], qb = charge[b0];
  if (fabsf(qa) < 1e-10f) qa = 1e-10f;
  if (fabsf(qb) < 1e-10f) qb = 1e-10f;
  const float fs = -A[t] * ir14 + B[t] * ir8 - cf[t] * ir2 * ir * qa * qb;
  const float gx = fs * d.x, gy = fs * d.y, gz = fs * d.z;
  const int N = acc.n;
  red_add(acc.d_f + a, to_fixed_force(gx));
  red_add(acc.d_f + N + a, to_fixed_force(gy));
  red_add(acc.d_f + 2 * N + a, to_fixed_force(gz));
  red_add(acc.d_f + b, to_fixed_force(-gx));
  red_add(acc.d_f + N + b, to_fixed_force(-gy));
  red_add(acc.d_f + 2 * N + b, to_fixed_force(-gz));
  if (ENERGY) {
    const float ec = cf[t] * ir * qa * qb;
    // the reference's constants 0.08333333 and 0.1666666 (nb14.cpp:83-85)
    const float el = 0.08333333f * A[t] * ir4 * ir8 - 0.1666666f * B[t] * ir4 * ir2;
    if (per_atom) {
      red_add(acc.d_e + a, to_fixed_energy(ec + el));
      red_add(acc.d_elj + a, to_fixed_energy(el));
      red_add(acc.d_ec + a, to_fixed_energy(ec));
    }
    if (sums) {
      red_add(sums, to_fixed_energy(el + ec));
      red_add(sums + 1, to_fixed_energy(ec));
    }
  }
  if (VIRIAL) {  // -(F (x) dr) with summed off-diagonals, on atom a
    red_add(acc.d_v + a, to_fixed_energy(-(gx * d.x)));
    red_add(acc.d_v + N + a, to_fixed_energy(-(gx * d.y + gy * d.x)));
    red_add(acc.d_v + 2 * N + a, to_fixed_energy(-(gy * d.y)));
    red_add(acc.d_v + 3 * N + a, to_fixed_energy(-(gx * d.z + gz * d.x)));
    red_add(acc.d_v + 4 * N + a, to_fixed_energy(-(gy * d.z + gz * d.y)));
    red_add(acc.d_v + 5 * N + a, to_fixed_energy(-(gz * d.z)));
  }
}

int launch_nb14(const NB14& p, const float3* crd, const float* charge, const Cell& cell,
                const Cell& rcell, const int* map, Accumulators& acc, bool energy,
                bool virial, bool per_atom, long long* sums, cudaStream_t st) {
  if (p.m <= 0) return kOk;
  const int blocks = ceil_div(p.m, 256);
  if (energy && virial)
    k_nb14<true, true><<<blocks, 256, 0, st>>>(p.m, p.d_a, p.d_b, p.d_A, p.d_B, p.d_cf, crd,
                                               charge, cell, rcell, map, acc, per_atom, sums);
  else if (energy)
    k_nb14<true, false><<<blocks, 256, 0, st>>>(p.m, p.d_a, p.d_b, p.d_A, p.d_B, p.d_cf,
                                                crd, charge, cell, rcell, map, acc, per_atom,
                                                sums);
  else if (virial)
    k_nb14<false, true><<<blocks, 256, 0, st>>>(p.m, p.d_a, p.d_b, p.d_A, p.d_B, p.d_cf,
                                                crd, charge, cell, rcell, map, acc, per_atom,
                                                sums);
  else
    k_nb14<false, false><<<blocks, 256, 0, st>>>(p.m, p.d_a, p.d_b, p.d_A, p.d_B, p.d_cf,
                                                 crd, charge, cell, rcell, map, acc, per_atom,
                                                 sums);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int nb14_init(NB14& p, int m, const int* a, const int* b, const float* A, const float* B,
              const float* cf, int atom_numbers) {
  if (m < 0 || (m > 0 && (!a || !b || !A || !B || !cf)))
    return fail(kBadInput, "NON_BOND_14::Initial: bad argument");
  for (int t = 0; t < m; ++t)
    if (a[t] < 0 || a[t] >= atom_numbers || b[t] < 0 || b[t] >= atom_numbers)
      return fail(kBadInput, "NON_BOND_14::Initial: atom index out of range");
  p.m = m;
  const size_t k = m > 0 ? m : 1;
  SNB_CUDA_TRY(cudaMalloc(&p.d_a, sizeof(int) * k));
  SNB_CUDA_TRY(cudaMalloc(&p.d_b, sizeof(int) * k));
  SNB_CUDA_TRY(cudaMalloc(&p.d_A, sizeof(float) * k));
  SNB_CUDA_TRY(cudaMalloc(&p.d_B, sizeof(float) * k));
  SNB_CUDA_TRY(cudaMalloc(&p.d_cf, sizeof(float) * k));
  if (m > 0) {
    SNB_CUDA_TRY(cudaMemcpy(p.d_a, a, sizeof(int) * m, cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(p.d_b, b, sizeof(int) * m, cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(p.d_A, A, sizeof(float) * m, cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(p.d_B, B, sizeof(float) * m, cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(p.d_cf, cf, sizeof(float) * m, cudaMemcpyHostToDevice));
  }
  return kOk;
}

void nb14_free(NB14& p) {
  cudaFree(p.d_a);
  cudaFree(p.d_b);
  cudaFree(p.d_A);
  cudaFree(p.d_B);
  cudaFree(p.d_cf);
  p = NB14();
}

}  // namespace snb
