// Virtual atoms: the VIRTUAL_INFORMATION boundary (virtual_atoms/
// virtual_atoms.h, virtual_atoms.cpp) for types 0-3, re-designed for sm_100a.
//
// Each record places a massless site from one to three source atoms (r_ij is
// the minimum-image r_i - r_j):
//   0: x_v = x_1, y_v = y_1, z_v = 2h - z_1;   F_1 += (Fx, Fy, -Fz)
//   1: r_v = r_1 + a r_21;                     F_1 += (1-a) F, F_2 += a F
//   2: r_v = r_1 + a r_21 + b r_31;            F_1 += (1-a-b) F, F_2 += a F,
//                                              F_3 += b F
//   3: q = r_21 + k r_32, u = q/|q|, r_v = r_1 + d u, g = d/|q| (F - (F.u)u),
//      F_1 += F - g, F_2 += (1-k) g, F_3 += k g; |d| <= 1e-6 puts the site
//      on atom 1 with all its force, |q|^2 <= 1e-12 is an invalid geometry
// (virtual_atom_math.h).  A site may be built from other sites: its level
// is one more than the highest level of its sources (real atoms are level
// 0), positions are refreshed level by level upwards and forces moved down
// level by level, one launch per level for all types (a type switch per
// thread), as the reference's layers do with one launch per type per layer.
// Forces given as floats are moved with plain adds when no two sites of a
// level share a source (the order is then fixed) and with float atomics
// otherwise, as the reference does; the engine moves them inside its 64-bit
// fixed-point accumulator, order-independent.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/sponge_nb.h"
#include "snb_internal.h"

namespace snb {

struct VRecord {
  int type, v, a, b, c;
  float p, q;
};

constexpr float kVGeomEps = 1.0e-6f;

__device__ __forceinline__ float3 v_add(float3 x, float3 y) {
  return make_float3(x.x + y.x, x.y + y.y, x.z + y.z);
}
__device__ __forceinline__ float3 v_scale(float s, float3 x) {
  return make_float3(s * x.x, s * x.y, s * x.z);
}

// Position of the site of record r from crd; false for an invalid type-3
// geometry (the site is then put on atom 1).
__device__ __forceinline__ bool v_position(const VRecord& r, const float3* crd,
                                           const Cell& cell, const Cell& rcell,
                                           float3* out) {
  const float3 x1 = crd[r.a];
  if (r.type == 0) {
    *out = make_float3(x1.x, x1.y, 2.0f * r.p - x1.z);
    return true;
  }
  const float3 r21 = min_image_exact(crd[r.b], x1, cell, rcell);
  if (r.type == 1) {
    *out = v_add(x1, v_scale(r.p, r21));
    return true;
  }
  if (r.type == 2) {
    const float3 r31 = min_image_exact(crd[r.c], x1, cell, rcell);
    *out = v_add(v_add(x1, v_scale(r.p, r21)), v_scale(r.q, r31));
    return true;
  }
  const float3 r32 = min_image_exact(crd[r.c], crd[r.b], cell, rcell);
  const float3 w = v_add(r21, v_scale(r.q, r32));
  const float n2 = w.x * w.x + w.y * w.y + w.z * w.z;
  if (fabsf(r.p) <= kVGeomEps) {
    *out = x1;
    return true;
  }
  if (n2 <= kVGeomEps * kVGeomEps) {
    *out = x1;
    return false;
  }
  *out = v_add(x1, v_scale(r.p / sqrtf(n2), w));
  return true;
}

// The parts of the site force F that go to atoms a, b, c.
__device__ __forceinline__ bool v_split(const VRecord& r, float3 F, const float3* crd,
                                        const Cell& cell, const Cell& rcell, float3* fa,
                                        float3* fb, float3* fc) {
  const float3 zero = make_float3(0.f, 0.f, 0.f);
  *fb = zero;
  *fc = zero;
  if (r.type == 0) {
    *fa = make_float3(F.x, F.y, -F.z);
    return true;
  }
  if (r.type == 1) {
    *fa = v_scale(1.0f - r.p, F);
    *fb = v_scale(r.p, F);
    return true;
  }
  if (r.type == 2) {
    *fa = v_scale(1.0f - r.p - r.q, F);
    *fb = v_scale(r.p, F);
    *fc = v_scale(r.q, F);
    return true;
  }
  if (fabsf(r.p) <= kVGeomEps) {
    *fa = F;
    return true;
  }
  const float3 r21 = min_image_exact(crd[r.b], crd[r.a], cell, rcell);
  const float3 r32 = min_image_exact(crd[r.c], crd[r.b], cell, rcell);
  const float3 w = v_add(r21, v_scale(r.q, r32));
  const float n2 = w.x * w.x + w.y * w.y + w.z * w.z;
  if (n2 <= kVGeomEps * kVGeomEps) {
    *fa = zero;
    return false;
  }
  const float in = 1.0f / sqrtf(n2);
  const float3 u = v_scale(in, w);
  const float fu = F.x * u.x + F.y * u.y + F.z * u.z;
  const float3 g = v_scale(r.p * in, make_float3(F.x - fu * u.x, F.y - fu * u.y,
                                                  F.z - fu * u.z));
  *fa = make_float3(F.x - g.x, F.y - g.y, F.z - g.z);
  *fb = v_scale(1.0f - r.q, g);
  *fc = v_scale(r.q, g);
  return true;
}

__global__ void k_vatom_refresh(int begin, int end, const VRecord* __restrict__ rec,
                                float3* __restrict__ crd, Cell cell, Cell rcell,
                                int* __restrict__ err) {
  const int t = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= end) return;
  const VRecord r = rec[t];
  float3 x;
  if (!v_position(r, crd, cell, rcell, &x)) atomicCAS(err, 0, 1 + t);
  crd[r.v] = x;
}

__device__ __forceinline__ void f3_add(float3* p, float3 v, bool atomic) {
  if (atomic) {
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
  } else {
    *p = v_add(*p, v);
  }
}

__global__ void k_vatom_spread_float(int begin, int end, const VRecord* __restrict__ rec,
                                     const float3* __restrict__ crd, Cell cell, Cell rcell,
                                     float3* __restrict__ frc, bool atomic,
                                     int* __restrict__ err) {
  const int t = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= end) return;
  const VRecord r = rec[t];
  const float3 F = frc[r.v];
  float3 fa, fb, fc;
  if (!v_split(r, F, crd, cell, rcell, &fa, &fb, &fc)) atomicCAS(err, 0, 1 + t);
  f3_add(frc + r.a, fa, atomic);
  if (r.type >= 1) f3_add(frc + r.b, fb, atomic);
  if (r.type >= 2) f3_add(frc + r.c, fc, atomic);
  frc[r.v] = make_float3(0.f, 0.f, 0.f);
}

// The engine's form: site forces in the fixed-point accumulator at map[atom]
// (caller index -> sorted slot); the parts are rounded to fixed point from
// the double value of the site force, so the result is order-independent.
__global__ void k_vatom_spread_fixed(int begin, int end, const VRecord* __restrict__ rec,
                                     const float3* __restrict__ crd, Cell cell, Cell rcell,
                                     const int* __restrict__ map, Accumulators acc,
                                     int* __restrict__ err) {
  const int t = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= end) return;
  const VRecord r = rec[t];
  const int N = acc.n;
  const int sv = map ? map[r.v] : r.v;
  const float3 F = make_float3((float)((double)acc.d_f[sv] * kForceScaleInv),
                               (float)((double)acc.d_f[N + sv] * kForceScaleInv),
                               (float)((double)acc.d_f[2 * N + sv] * kForceScaleInv));
  float3 fa, fb, fc;
  if (!v_split(r, F, crd, cell, rcell, &fa, &fb, &fc)) atomicCAS(err, 0, 1 + t);
  auto add = [&](int atom, float3 v) {
    const int s = map ? map[atom] : atom;
    red_add(acc.d_f + s, to_fixed_force(v.x));
    red_add(acc.d_f + N + s, to_fixed_force(v.y));
    red_add(acc.d_f + 2 * N + s, to_fixed_force(v.z));
  };
  add(r.a, fa);
  if (r.type >= 1) add(r.b, fb);
  if (r.type >= 2) add(r.c, fc);
  acc.d_f[sv] = 0;
  acc.d_f[N + sv] = 0;
  acc.d_f[2 * N + sv] = 0;
}

}  // namespace snb

using namespace snb;

struct snb_vatom {
  int n = 0, m = 0;
  std::vector<int> level_begin;    // records of level L: [level_begin[L-1], level_begin[L])
  std::vector<char> level_shared;  // a source shared by two sites of the level
  VRecord* d_rec = nullptr;
  int* d_err = nullptr;            // 1 + record of an invalid type-3 geometry, else 0
};

namespace snb {

int vatom_refresh(snb_vatom* h, float* crd, const Cell& cell, const Cell& rcell,
                  cudaStream_t st) {
  for (size_t L = 1; L < h->level_begin.size(); ++L) {
    const int b = h->level_begin[L - 1], e = h->level_begin[L];
    if (e > b)
      k_vatom_refresh<<<ceil_div(e - b, 256), 256, 0, st>>>(
          b, e, h->d_rec, reinterpret_cast<float3*>(crd), cell, rcell, h->d_err);
  }
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int vatom_spread_fixed(snb_vatom* h, const float* crd, const Cell& cell, const Cell& rcell,
                       const int* map, Accumulators& acc, cudaStream_t st) {
  for (size_t L = h->level_begin.size() - 1; L >= 1; --L) {
    const int b = h->level_begin[L - 1], e = h->level_begin[L];
    if (e > b)
      k_vatom_spread_fixed<<<ceil_div(e - b, 256), 256, 0, st>>>(
          b, e, h->d_rec, reinterpret_cast<const float3*>(crd), cell, rcell, map, acc,
          h->d_err);
  }
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int vatom_status(snb_vatom* h, int* bad, cudaStream_t st) {
  SNB_CUDA_TRY(cudaMemcpyAsync(bad, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  return kOk;
}

int vatom_atoms(snb_vatom* h) { return h ? h->n : 0; }

}  // namespace snb

extern "C" int snb_vatom_create(int atom_numbers, int record_numbers, const int* h_type,
                                const int* h_virtual_atom, const int* h_from,
                                const float* h_parameter, snb_vatom** out) {
  if (!out) return fail(kBadInput, "vatom_create: null out");
  *out = nullptr;
  const int n = atom_numbers, m = record_numbers;
  if (n <= 0 || m < 0 || (m > 0 && (!h_type || !h_virtual_atom || !h_from || !h_parameter)))
    return fail(kBadInput, "VIRTUAL_INFORMATION::Initial: bad argument");
  std::vector<int> rec_of(n, -1);
  for (int t = 0; t < m; ++t) {
    const int v = h_virtual_atom[t], ty = h_type[t];
    if (ty < 0 || ty > 3)
      return fail(kBadInput, "VIRTUAL_INFORMATION::Initial: virtual atom type " +
                                 std::to_string(ty) + " is not built (types 0-3 are)");
    if (v < 0 || v >= n) return fail(kBadInput, "VIRTUAL_INFORMATION::Initial: atom index out of range");
    if (rec_of[v] >= 0)
      return fail(kBadInput, "VIRTUAL_INFORMATION::Initial: atom " + std::to_string(v) +
                                 " is defined as a virtual atom twice");
    rec_of[v] = t;
    const int ns = ty == 0 ? 1 : (ty == 1 ? 2 : 3);
    for (int k = 0; k < ns; ++k) {
      const int s = h_from[3 * t + k];
      if (s < 0 || s >= n)
        return fail(kBadInput, "VIRTUAL_INFORMATION::Initial: atom index out of range");
    }
  }
  // levels by repeated relaxation; a chain longer than the record count is
  // a cycle (a site that is its own source)
  std::vector<int> level(n, 0);
  for (int t = 0; t < m; ++t) level[h_virtual_atom[t]] = 1;
  bool changed = true;
  for (int pass = 0; changed; ++pass) {
    if (pass > m + 1)
      return fail(kBadInput,
                  "VIRTUAL_INFORMATION::Initial: the virtual atoms depend on themselves");
    changed = false;
    for (int t = 0; t < m; ++t) {
      const int ty = h_type[t], ns = ty == 0 ? 1 : (ty == 1 ? 2 : 3);
      int lv = 1;
      for (int k = 0; k < ns; ++k) lv = std::max(lv, 1 + level[h_from[3 * t + k]]);
      if (lv != level[h_virtual_atom[t]]) {
        level[h_virtual_atom[t]] = lv;
        changed = true;
      }
    }
  }
  std::vector<int> order(m);
  for (int t = 0; t < m; ++t) order[t] = t;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return level[h_virtual_atom[x]] < level[h_virtual_atom[y]];
  });
  snb_vatom* h = new snb_vatom();
  h->n = n;
  h->m = m;
  std::vector<VRecord> recs(m);
  int max_level = 0;
  for (int k = 0; k < m; ++k) {
    const int t = order[k];
    recs[k] = VRecord{h_type[t], h_virtual_atom[t], h_from[3 * t], h_from[3 * t + 1],
                      h_from[3 * t + 2], h_parameter[2 * t], h_parameter[2 * t + 1]};
    max_level = std::max(max_level, level[h_virtual_atom[t]]);
  }
  h->level_begin.assign(max_level + 1, 0);
  for (int k = 0; k < m; ++k) h->level_begin[level[recs[k].v]] = k + 1;
  for (int L = 1; L <= max_level; ++L)
    h->level_begin[L] = std::max(h->level_begin[L], h->level_begin[L - 1]);
  h->level_shared.assign(max_level + 1, 0);
  {
    std::vector<int> seen(n, -1);
    for (int L = 1; L <= max_level; ++L)
      for (int k = h->level_begin[L - 1]; k < h->level_begin[L]; ++k) {
        const int ns = recs[k].type == 0 ? 1 : (recs[k].type == 1 ? 2 : 3);
        const int src[3] = {recs[k].a, recs[k].b, recs[k].c};
        for (int q = 0; q < ns; ++q) {
          if (seen[src[q]] == L) h->level_shared[L] = 1;
          seen[src[q]] = L;
        }
      }
  }
  cudaError_t ce = cudaMalloc(&h->d_rec, sizeof(VRecord) * std::max(m, 1));
  if (ce == cudaSuccess && m > 0)
    ce = cudaMemcpy(h->d_rec, recs.data(), sizeof(VRecord) * m, cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_err, sizeof(int));
  if (ce == cudaSuccess) ce = cudaMemset(h->d_err, 0, sizeof(int));
  if (ce != cudaSuccess) {
    cudaFree(h->d_rec);
    cudaFree(h->d_err);
    delete h;
    return fail(kCudaError, std::string("vatom_create: ") + cudaGetErrorString(ce));
  }
  *out = h;
  return kOk;
}

extern "C" int snb_vatom_levels(snb_vatom* h, int* levels) {
  if (!h || !levels) return fail(kBadInput, "vatom_levels: null argument");
  *levels = (int)h->level_begin.size() - 1;
  return kOk;
}

extern "C" int snb_vatom_coordinate_refresh(snb_vatom* h, float* crd, snb_boundary boundary,
                                            void* stream) {
  if (!h || !crd) return fail(kBadInput, "vatom_coordinate_refresh: bad argument");
  return vatom_refresh(h, crd, make_cell(boundary.cell), make_cell(boundary.rcell),
                       reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int snb_vatom_force_redistribute(snb_vatom* h, const float* crd,
                                            snb_boundary boundary, float* frc, void* stream) {
  if (!h || !crd || !frc) return fail(kBadInput, "vatom_force_redistribute: bad argument");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  const Cell cell = make_cell(boundary.cell), rcell = make_cell(boundary.rcell);
  for (size_t L = h->level_begin.size() - 1; L >= 1; --L) {
    const int b = h->level_begin[L - 1], e = h->level_begin[L];
    if (e > b)
      k_vatom_spread_float<<<ceil_div(e - b, 256), 256, 0, st>>>(
          b, e, h->d_rec, reinterpret_cast<const float3*>(crd), cell, rcell,
          reinterpret_cast<float3*>(frc), h->level_shared[L] != 0, h->d_err);
  }
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

extern "C" int snb_vatom_status(snb_vatom* h, int* bad_record, void* stream) {
  if (!h || !bad_record) return fail(kBadInput, "vatom_status: null argument");
  int v = 0;
  int rc = vatom_status(h, &v, reinterpret_cast<cudaStream_t>(stream));
  if (rc) return rc;
  *bad_record = v - 1;
  return kOk;
}

extern "C" int snb_vatom_destroy(snb_vatom* h) {
  if (!h) return kOk;
  cudaFree(h->d_rec);
  cudaFree(h->d_err);
  delete h;
  return kOk;
}
