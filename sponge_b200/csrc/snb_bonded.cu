// Harmonic bonds and angles as modules: the BOND (bond/bond.h,
// bond/bond.cpp) and ANGLE (angle/angle.h, angle/angle.cpp) boundary.
//
// Bond t of atoms (i, j), dr = r_i - r_j (minimum image), r = |dr|:
//   E = k (r - r0)^2,  f_i = -2 k (r - r0) / r dr,  f_j = -f_i;
//   energy and virial f_i (x) dr on atom i (bond.cpp:15-60).
// Angle t of atoms (i, j, k) with vertex j, a = r_i - r_j, b = r_k - r_j:
//   cos = a.b / (|a||b|) clamped to +-0.999999, theta = acos(cos),
//   E = K (theta - theta0)^2, c = -2 K (theta - theta0) / sin(theta),
//   f_i = c (cos a / |a|^2 - b / (|a||b|)), f_k likewise with a and b
//   swapped, f_j = -f_i - f_k; energy and virial f_i (x) a + f_k (x) b on
//   atom i (angle.cpp:6-80).
// One thread per term; forces, per-atom energies and virials accumulate in
// the 64-bit fixed-point accumulators (order-independent), then are added
// to the caller's float arrays, and the energy sum of Step_Print is kept in
// fixed point.
#include <cstring>

#include "../../include/sponge_nb.h"
#include "snb_internal.h"

namespace snb {

__device__ __forceinline__ void bonded_virial(Accumulators& acc, int s, float3 f, float3 d) {
  const int N = acc.n;
  red_add(acc.d_v + s, to_fixed_energy(f.x * d.x));
  red_add(acc.d_v + N + s, to_fixed_energy(f.x * d.y + f.y * d.x));
  red_add(acc.d_v + 2 * N + s, to_fixed_energy(f.y * d.y));
  red_add(acc.d_v + 3 * N + s, to_fixed_energy(f.x * d.z + f.z * d.x));
  red_add(acc.d_v + 4 * N + s, to_fixed_energy(f.y * d.z + f.z * d.y));
  red_add(acc.d_v + 5 * N + s, to_fixed_energy(f.z * d.z));
}

__device__ __forceinline__ void bonded_force(Accumulators& acc, int s, float3 f) {
  const int N = acc.n;
  red_add(acc.d_f + s, to_fixed_force(f.x));
  red_add(acc.d_f + N + s, to_fixed_force(f.y));
  red_add(acc.d_f + 2 * N + s, to_fixed_force(f.z));
}

template <bool ENERGY, bool VIRIAL>
__global__ void k_bond_terms(int m, const int* __restrict__ ia, const int* __restrict__ ib,
                             const float* __restrict__ bk, const float* __restrict__ br0,
                             const float3* __restrict__ crd, Cell cell, Cell rcell,
                             Accumulators acc, long long* __restrict__ sum) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const int i = ia[t], j = ib[t];
  const float3 d = min_image_fast<false>(crd[i], crd[j], cell, rcell);
  const float r = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  const float dev = r - br0[t];
  const float s = -2.0f * dev * bk[t] / r;
  const float3 f = make_float3(s * d.x, s * d.y, s * d.z);
  bonded_force(acc, i, f);
  bonded_force(acc, j, make_float3(-f.x, -f.y, -f.z));
  if (ENERGY) {
    const long long e = to_fixed_energy(bk[t] * dev * dev);
    red_add(acc.d_e + i, e);
    red_add(sum, e);
  }
  if (VIRIAL) bonded_virial(acc, i, f, d);
}

template <bool ENERGY, bool VIRIAL>
__global__ void k_angle_terms(int m, const int* __restrict__ ia, const int* __restrict__ ib,
                              const int* __restrict__ ic, const float* __restrict__ ak,
                              const float* __restrict__ at0, const float3* __restrict__ crd,
                              Cell cell, Cell rcell, Accumulators acc,
                              long long* __restrict__ sum) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m) return;
  const int i = ia[t], j = ib[t], l = ic[t];
  const float3 a = min_image_fast<false>(crd[i], crd[j], cell, rcell);
  const float3 b = min_image_fast<false>(crd[l], crd[j], cell, rcell);
  const float ia2 = 1.0f / (a.x * a.x + a.y * a.y + a.z * a.z);
  const float ib2 = 1.0f / (b.x * b.x + b.y * b.y + b.z * b.z);
  const float iab = sqrtf(ia2 * ib2);
  float cs = (a.x * b.x + a.y * b.y + a.z * b.z) * iab;
  cs = fmaxf(-0.999999f, fminf(cs, 0.999999f));
  const float th = acosf(cs);
  const float dth = th - at0[t];
  const float c = -2.0f * ak[t] * dth / sinf(th);
  const float self_a = c * cs * ia2, self_b = c * cs * ib2, cross = c * iab;
  const float3 fi = make_float3(self_a * a.x - cross * b.x, self_a * a.y - cross * b.y,
                                self_a * a.z - cross * b.z);
  const float3 fk = make_float3(self_b * b.x - cross * a.x, self_b * b.y - cross * a.y,
                                self_b * b.z - cross * a.z);
  bonded_force(acc, i, fi);
  bonded_force(acc, l, fk);
  bonded_force(acc, j, make_float3(-fi.x - fk.x, -fi.y - fk.y, -fi.z - fk.z));
  if (ENERGY) {
    const long long e = to_fixed_energy(ak[t] * dth * dth);
    red_add(acc.d_e + i, e);
    red_add(sum, e);
  }
  if (VIRIAL) {
    bonded_virial(acc, i, fi, a);
    bonded_virial(acc, i, fk, b);
  }
}

// A term list on the device: up to three atom columns and two parameters.
struct TermList {
  int n = 0, m = 0;
  int* d_a = nullptr;
  int* d_b = nullptr;
  int* d_c = nullptr;
  float* d_p0 = nullptr;
  float* d_p1 = nullptr;
  Accumulators acc;
  long long* d_sum = nullptr;
};

static void terms_free(TermList& t) {
  cudaFree(t.d_a);
  cudaFree(t.d_b);
  cudaFree(t.d_c);
  cudaFree(t.d_p0);
  cudaFree(t.d_p1);
  cudaFree(t.d_sum);
  acc_free(t.acc);
  t = TermList();
}

static int terms_init(TermList& t, int atom_numbers, int m, const int* a, const int* b,
                      const int* c, const float* p0, const float* p1, const char* who) {
  if (atom_numbers <= 0) return fail(kBadInput, std::string(who) + ": atom_numbers must be > 0");
  if (m < 0 || (m > 0 && (!a || !b || !p0 || !p1)))
    return fail(kBadInput, std::string(who) + ": bad argument");
  for (int k = 0; k < m; ++k) {
    const bool bad = a[k] < 0 || a[k] >= atom_numbers || b[k] < 0 || b[k] >= atom_numbers ||
                     (c && (c[k] < 0 || c[k] >= atom_numbers));
    if (bad) return fail(kBadInput, std::string(who) + ": atom index out of range");
  }
  t.n = atom_numbers;
  t.m = m;
  const size_t w = m > 0 ? m : 1;
  auto up_i = [&](int** d, const int* h) -> int {
    SNB_CUDA_TRY(cudaMalloc(d, sizeof(int) * w));
    if (m > 0) SNB_CUDA_TRY(cudaMemcpy(*d, h, sizeof(int) * m, cudaMemcpyHostToDevice));
    return kOk;
  };
  auto up_f = [&](float** d, const float* h) -> int {
    SNB_CUDA_TRY(cudaMalloc(d, sizeof(float) * w));
    if (m > 0) SNB_CUDA_TRY(cudaMemcpy(*d, h, sizeof(float) * m, cudaMemcpyHostToDevice));
    return kOk;
  };
  int rc = up_i(&t.d_a, a);
  if (!rc) rc = up_i(&t.d_b, b);
  if (!rc && c) rc = up_i(&t.d_c, c);
  if (!rc) rc = up_f(&t.d_p0, p0);
  if (!rc) rc = up_f(&t.d_p1, p1);
  if (!rc) rc = acc_init(t.acc, atom_numbers);
  if (!rc) {
    SNB_CUDA_TRY(cudaMalloc(&t.d_sum, sizeof(long long)));
    SNB_CUDA_TRY(cudaMemset(t.d_sum, 0, sizeof(long long)));
  }
  return rc;
}

template <bool ANGLE>
static int terms_force(TermList& t, const float* crd, const snb_boundary& bd, float* frc,
                       bool en, bool vi, float* atom_energy, float* atom_virial,
                       cudaStream_t st) {
  const Cell cell = make_cell(bd.cell), rcell = make_cell(bd.rcell);
  const float3* x = reinterpret_cast<const float3*>(crd);
  if (en) SNB_CUDA_TRY(cudaMemsetAsync(t.d_sum, 0, sizeof(long long), st));
  if (t.m > 0) {
    const int blocks = ceil_div(t.m, 256);
#define SNB_TERMS(E, V)                                                                    \
  if (ANGLE)                                                                               \
    k_angle_terms<E, V><<<blocks, 256, 0, st>>>(t.m, t.d_a, t.d_b, t.d_c, t.d_p0, t.d_p1, \
                                                x, cell, rcell, t.acc, t.d_sum);           \
  else                                                                                     \
    k_bond_terms<E, V><<<blocks, 256, 0, st>>>(t.m, t.d_a, t.d_b, t.d_p0, t.d_p1, x, cell, \
                                               rcell, t.acc, t.d_sum);
    if (en && vi) {
      SNB_TERMS(true, true)
    } else if (en) {
      SNB_TERMS(true, false)
    } else if (vi) {
      SNB_TERMS(false, true)
    } else {
      SNB_TERMS(false, false)
    }
#undef SNB_TERMS
    SNB_CUDA_TRY(cudaGetLastError());
  }
  return launch_unpack(t.n, nullptr, t.acc, kAccumFixed, reinterpret_cast<float3*>(frc),
                       en ? atom_energy : nullptr, nullptr, nullptr,
                       vi ? atom_virial : nullptr, en, vi, st);
}

static int terms_energy(TermList& t, float* out, cudaStream_t st) {
  long long v = 0;
  SNB_CUDA_TRY(cudaMemcpyAsync(&v, t.d_sum, sizeof(v), cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  *out = (float)((double)v * kEnergyScaleInv);
  return kOk;
}

}  // namespace snb

using namespace snb;

struct snb_bond {
  TermList t;
};
struct snb_angle {
  TermList t;
};

static cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" int snb_bond_create(int atom_numbers, int bond_numbers, const int* h_atom_a,
                               const int* h_atom_b, const float* h_k, const float* h_r0,
                               snb_bond** out) {
  if (!out) return fail(kBadInput, "bond_create: null out");
  *out = nullptr;
  snb_bond* h = new snb_bond();
  int rc = terms_init(h->t, atom_numbers, bond_numbers, h_atom_a, h_atom_b, nullptr, h_k,
                      h_r0, "BOND::Initial");
  if (rc) {
    terms_free(h->t);
    delete h;
    return rc;
  }
  *out = h;
  return kOk;
}

extern "C" int snb_bond_force(snb_bond* h, const float* crd, snb_boundary boundary, float* frc,
                              int need_atom_energy, float* atom_energy, int need_virial,
                              float* atom_virial, void* stream) {
  if (!h || !crd || !frc) return fail(kBadInput, "bond_force: bad argument");
  if ((need_atom_energy && !atom_energy) || (need_virial && !atom_virial))
    return fail(kBadInput, "bond_force: missing energy or virial array");
  return terms_force<false>(h->t, crd, boundary, frc, need_atom_energy != 0,
                            need_virial != 0, atom_energy, atom_virial, as_stream(stream));
}

extern "C" int snb_bond_energy(snb_bond* h, float* h_energy, void* stream) {
  if (!h || !h_energy) return fail(kBadInput, "bond_energy: null argument");
  return terms_energy(h->t, h_energy, as_stream(stream));
}

extern "C" int snb_bond_destroy(snb_bond* h) {
  if (!h) return kOk;
  terms_free(h->t);
  delete h;
  return kOk;
}

extern "C" int snb_angle_create(int atom_numbers, int angle_numbers, const int* h_atom_a,
                                const int* h_atom_b, const int* h_atom_c, const float* h_k,
                                const float* h_theta0, snb_angle** out) {
  if (!out) return fail(kBadInput, "angle_create: null out");
  *out = nullptr;
  if (angle_numbers > 0 && !h_atom_c) return fail(kBadInput, "ANGLE::Initial: bad argument");
  snb_angle* h = new snb_angle();
  int rc = terms_init(h->t, atom_numbers, angle_numbers, h_atom_a, h_atom_b,
                      angle_numbers > 0 ? h_atom_c : nullptr, h_k, h_theta0,
                      "ANGLE::Initial");
  if (rc) {
    terms_free(h->t);
    delete h;
    return rc;
  }
  *out = h;
  return kOk;
}

extern "C" int snb_angle_force(snb_angle* h, const float* crd, snb_boundary boundary,
                               float* frc, int need_atom_energy, float* atom_energy,
                               int need_virial, float* atom_virial, void* stream) {
  if (!h || !crd || !frc) return fail(kBadInput, "angle_force: bad argument");
  if ((need_atom_energy && !atom_energy) || (need_virial && !atom_virial))
    return fail(kBadInput, "angle_force: missing energy or virial array");
  return terms_force<true>(h->t, crd, boundary, frc, need_atom_energy != 0, need_virial != 0,
                           atom_energy, atom_virial, as_stream(stream));
}

extern "C" int snb_angle_energy(snb_angle* h, float* h_energy, void* stream) {
  if (!h || !h_energy) return fail(kBadInput, "angle_energy: null argument");
  return terms_energy(h->t, h_energy, as_stream(stream));
}

extern "C" int snb_angle_destroy(snb_angle* h) {
  if (!h) return kOk;
  terms_free(h->t);
  delete h;
  return kOk;
}
