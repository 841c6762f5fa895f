// Rigid triangles and rigid pairs (SETTLE, constrain/settle.cpp).
//
// The constraint pairs are sorted on the host into rigid triangles (three
// atoms with exactly two constraints each, closing a triangle: water), rigid
// pairs (two atoms constrained only to each other) and the rest, which
// SETTLE leaves to SHAKE (SETTLE::Initial, settle.cpp:483-712).  Each
// triangle keeps its canonical frame: with the centre of mass at the origin
// A sits at (0, ra), B at (rc, rb), C at (rd, re), with (B - A) x (C - A)
// pointing along +z.
//
// Per step (main.cpp:1705,1772): the displacements B - A and C - A (pairs:
// j - i) are remembered before the coordinate update; after it, one thread
// per triangle or pair puts the atoms back on the rigid geometry and adds
// the change divided by dt to the velocities:
//  - triangles: the analytical solution of Miyamoto and Kollman (SETTLE,
//    J. Comput. Chem. 13, 952 (1992)) in the frame of the old plane
//    (settle.cpp:109-214);
//  - pairs: the displacement along the old bond that restores the length,
//    a root of a quadratic (settle.cpp:366-448), in double precision when
//    the discriminant is within rounding of zero.  A pair without a real
//    solution is left unchanged and its index recorded for the host (the
//    reference stops the run there).
// The constraint virial, sum of F (x) r_old over the constrained atoms with
// F = m (r_new - r_unconstrained) / (dt^2 x_factor), is accumulated in fixed
// point (reset by the remember kernel, so it holds the last step's) and, on
// request, added as virial / V to the caller's stress
// (Sum_Virial_Tensor_To_Stress, settle.cpp:450-481).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "snb_internal.h"

namespace snb {
namespace {

__device__ __forceinline__ float3 operator+(float3 a, float3 b) {
  return make_float3(a.x + b.x, a.y + b.y, a.z + b.z);
}
__device__ __forceinline__ float3 operator-(float3 a, float3 b) {
  return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ float3 operator*(float s, float3 a) {
  return make_float3(s * a.x, s * a.y, s * a.z);
}
__device__ __forceinline__ float dot(float3 a, float3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 unit(float3 a) { return rsqrtf(dot(a, a)) * a; }

// F (x) d with the off-diagonal pairs summed, LTMatrix3 order
__device__ __forceinline__ void add_virial(float* v, float3 f, float3 d) {
  v[0] += f.x * d.x;
  v[1] += f.x * d.y + f.y * d.x;
  v[2] += f.y * d.y;
  v[3] += f.x * d.z + f.z * d.x;
  v[4] += f.y * d.z + f.z * d.y;
  v[5] += f.z * d.z;
}

// one thread per triangle, then one per pair
__global__ void k_settle_remember(int nt, const SettleTri* __restrict__ tri, int np,
                                  const SettlePair* __restrict__ pair,
                                  const float3* __restrict__ crd, Cell cell, Cell rcell,
                                  float3* __restrict__ last_ba, float3* __restrict__ last_ca,
                                  float3* __restrict__ last_ab, long long* __restrict__ vir_sum) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 6) vir_sum[t] = 0;  // the step's constraint virial starts here
  if (t < nt) {
    const SettleTri g = tri[t];
    const float3 a = crd[g.a];
    last_ba[t] = min_image_fast<false>(crd[g.b], a, cell, rcell);
    last_ca[t] = min_image_fast<false>(crd[g.c], a, cell, rcell);
  } else if (t < nt + np) {
    const SettlePair p = pair[t - nt];
    last_ab[t - nt] = min_image_fast<false>(crd[p.j], crd[p.i], cell, rcell);
  }
}

__global__ void k_settle(int nt, const SettleTri* __restrict__ tri, int np,
                         const SettlePair* __restrict__ pair, float3* __restrict__ crd,
                         float3* __restrict__ vel, Cell cell, Cell rcell,
                         const float3* __restrict__ last_ba, const float3* __restrict__ last_ca,
                         const float3* __restrict__ last_ab, float dt, float v_factor,
                         float x_factor, long long* __restrict__ vir_sum,
                         int* __restrict__ err) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float v[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const float vscale = v_factor / dt / x_factor;    // position change -> velocity change
  const float fscale = 1.0f / (dt * dt * x_factor);  // position change * m -> force
  if (t < nt) {
    const SettleTri g = tri[t];
    // unconstrained positions relative to the centre of mass
    const float3 a = crd[g.a];
    float3 b1 = min_image_fast<false>(crd[g.b], a, cell, rcell);
    float3 c1 = min_image_fast<false>(crd[g.c], a, cell, rcell);
    const float3 com = (1.0f / (g.ma + g.mb + g.mc)) * (g.mb * b1 + g.mc * c1) + a;
    const float3 a1 = a - com;
    b1 = b1 + a1;
    c1 = c1 + a1;
    const float3 b0 = last_ba[t], c0 = last_ca[t];
    // frame of the old plane: z normal to it, x normal to z and to A now
    const float3 ez0 = cross(b0, c0);
    const float3 ex0 = cross(a1, ez0);
    const float3 ey = unit(cross(ez0, ex0));
    const float3 ex = unit(ex0), ez = unit(ez0);
    const float b0x = dot(ex, b0), b0y = dot(ey, b0);
    const float c0x = dot(ex, c0), c0y = dot(ey, c0);
    const float a1z = dot(ez, a1);
    const float b1x = dot(ex, b1), b1y = dot(ey, b1), b1z = dot(ez, b1);
    const float c1x = dot(ex, c1), c1y = dot(ey, c1), c1z = dot(ez, c1);
    // tilt of the template out of the plane: phi about x, psi about y
    const float sphi = a1z / g.ra;
    const float cphi = sqrtf(1.0f - sphi * sphi);
    const float spsi = (b1z - c1z - (g.rb - g.re) * sphi) / ((g.rd - g.rc) * cphi);
    const float cpsi = sqrtf(1.0f - spsi * spsi);
    const float a2y = g.ra * cphi;
    const float b2x = g.rc * cpsi, b2y = g.rb * cphi + g.rc * spsi * sphi;
    const float c2x = g.rd * cpsi, c2y = g.re * cphi + g.rd * spsi * sphi;
    // in-plane turn theta that conserves angular momentum about z
    const float al = b2x * b0x + c2x * c0x + b2y * b0y + c2y * c0y;
    const float be = b2y * b0x + c2y * c0x - b2x * b0y - c2x * c0y;
    const float ga = b1y * b0x - b1x * b0y + c1y * c0x - c1x * c0y;
    const float q = al * al + be * be;
    const float sth = (al * ga - be * sqrtf(q - ga * ga)) / q;
    const float cth = sqrtf(1.0f - sth * sth);
    // back to the box frame (z components are unchanged by the turn)
    const float3 a3 = (-a2y * sth) * ex + (a2y * cth) * ey + a1z * ez;
    const float3 b3 = (b2x * cth - b2y * sth) * ex + (b2x * sth + b2y * cth) * ey + b1z * ez;
    const float3 c3 = (c2x * cth - c2y * sth) * ex + (c2x * sth + c2y * cth) * ey + c1z * ez;
    const float3 da = a3 - a1, db = b3 - b1, dc = c3 - c1;
    vel[g.a] = vel[g.a] + vscale * da;
    vel[g.b] = vel[g.b] + vscale * db;
    vel[g.c] = vel[g.c] + vscale * dc;
    add_virial(v, (fscale * g.mb) * db, b0);
    add_virial(v, (fscale * g.mc) * dc, c0);
    crd[g.a] = a3 + com;
    crd[g.b] = b3 + com;
    crd[g.c] = c3 + com;
  } else if (t < nt + np) {
    const int k = t - nt;
    const SettlePair p = pair[k];
    const float3 r1 = min_image_fast<false>(crd[p.j], crd[p.i], cell, rcell);
    const float3 r2 = last_ab[k];
    // |r1 + s r2| = r0:  s = (sqrt(D) - r1.r2) / r2.r2,
    // D = (r1.r2)^2 - r1.r1 r2.r2 + r2.r2 r0^2
    const float r12 = dot(r1, r2), r11 = dot(r1, r1), r22 = dot(r2, r2);
    const float t0 = r12 * r12, t1 = r11 * r22, t2 = r22 * p.r0 * p.r0;
    const float D = t0 - t1 + t2;
    float s = 0.f;
    bool ok = false;
    if (isfinite(D) && isfinite(r22) && r22 > 0.f) {
      if (D > 8.0f * FLT_EPSILON * (t0 + t1 + t2)) {
        s = (sqrtf(D) - r12) / r22;
        ok = isfinite(s);
      } else {
        // discriminant within rounding of zero: D = r2.r2 r0^2 - |r1 x r2|^2 in double
        const double x1 = r1.x, y1 = r1.y, z1 = r1.z, x2 = r2.x, y2 = r2.y, z2 = r2.z;
        const double cx = y1 * z2 - z1 * y2, cy = z1 * x2 - x1 * z2, cz = x1 * y2 - y1 * x2;
        const double r22d = x2 * x2 + y2 * y2 + z2 * z2;
        const double Dd = r22d * (double)p.r0 * (double)p.r0 - (cx * cx + cy * cy + cz * cz);
        if (Dd >= 0.0 && isfinite(Dd)) {
          const double sd = (sqrt(Dd) - (x1 * x2 + y1 * y2 + z1 * z2)) / r22d;
          s = (float)sd;
          ok = isfinite(s);
        }
      }
    }
    if (!ok) {
      atomicExch(err, k + 1);  // left unchanged; the host reports it
    } else {
      const float3 sr2 = s * r2;
      const float3 di = (-p.mj * p.k) * sr2, dj = (p.mi * p.k) * sr2;
      crd[p.i] = crd[p.i] + di;
      crd[p.j] = crd[p.j] + dj;
      vel[p.i] = vel[p.i] + vscale * di;
      vel[p.j] = vel[p.j] + vscale * dj;
      add_virial(v, (fscale * p.mj) * dj, r2);
    }
  }
  if (vir_sum) {
    // warp sum, then one red.add per warp and component
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      float x = v[c];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      if ((threadIdx.x & 31) == 0 && x != 0.f) red_add(vir_sum + c, to_fixed_energy(x));
    }
  }
}

// stress += virial / V (V from the diagonal of rcell)
__global__ void k_settle_stress(const long long* __restrict__ vir_sum, Cell rcell,
                                float* __restrict__ stress) {
  const int c = threadIdx.x;
  if (c >= 6) return;
  const double inv_v = (double)rcell.a11 * rcell.a22 * rcell.a33;
  stress[c] += (float)((double)vir_sum[c] * kEnergyScaleInv * inv_v);
}

}  // namespace

// Canonical frame of a rigid triangle with sides rAB, rAC, rBC and masses
// mA, mB, mC (the role of Get_Rabcde_From_SSS, settle.cpp:53-107), worked
// out in double: any planar placement, shifted to the centre of mass, then
// expressed in the orthonormal in-plane basis whose y axis points at A.
static void triangle_frame(double rAB, double rAC, double rBC, double mA, double mB,
                           double mC, SettleTri& t) {
  // A at the origin, B on +x, C above the x axis
  const double cx = (rAB * rAB + rAC * rAC - rBC * rBC) / (2.0 * rAB);
  const double cy = std::sqrt(std::fmax(rAC * rAC - cx * cx, 0.0));
  const double M = mA + mB + mC;
  const double ox = (mB * rAB + mC * cx) / M, oy = mC * cy / M;
  const double P[3][2] = {{-ox, -oy}, {rAB - ox, -oy}, {cx - ox, cy - oy}};
  const double ra = std::hypot(P[0][0], P[0][1]);
  const double uy[2] = {P[0][0] / ra, P[0][1] / ra};  // y axis: centre of mass -> A
  const double ux[2] = {uy[1], -uy[0]};               // x axis: y turned by -90 degrees
  double x[3], y[3];
  for (int k = 0; k < 3; ++k) {
    x[k] = P[k][0] * ux[0] + P[k][1] * ux[1];
    y[k] = P[k][0] * uy[0] + P[k][1] * uy[1];
  }
  // keep (B - A) x (C - A) along +z (a proper rotation already does)
  if ((x[1] - x[0]) * (y[2] - y[0]) - (y[1] - y[0]) * (x[2] - x[0]) < 0)
    for (double& v : x) v = -v;
  t.ra = (float)ra;
  t.rb = (float)y[1];
  t.rc = (float)x[1];
  t.rd = (float)x[2];
  t.re = (float)y[2];
}

// The host side of SETTLE::Initial: groups and the left-over pair indices.
int settle_group(int n, int m, const int* ai, const int* aj, const float* r0,
                 const float* mass, std::vector<SettleTri>& tri,
                 std::vector<SettlePair>& pair, std::vector<int>& remaining) {
  if (n <= 0 || m < 0 || (m > 0 && (!ai || !aj || !r0)) || !mass)
    return fail(kBadInput, "SETTLE::Initial: bad argument");
  for (int p = 0; p < m; ++p)
    if (ai[p] < 0 || ai[p] >= n || aj[p] < 0 || aj[p] >= n || ai[p] == aj[p])
      return fail(kBadInput, "SETTLE::Initial: constraint atom index out of range");
  // links per atom (up to two kept), 3 = part of something SETTLE cannot take
  std::vector<int> links(n, 0), partner(2 * (size_t)n, -1);
  std::vector<float> len(3 * (size_t)n, 0.f);
  for (int p = 0; p < m; ++p) {
    const int i = ai[p], j = aj[p];
    if (links[i] < 2 && links[j] < 2) {
      partner[2 * i + links[i]] = j;
      partner[2 * j + links[j]] = i;
      len[3 * i + links[i]] = r0[p];
      len[3 * j + links[j]] = r0[p];
      ++links[i];
      ++links[j];
    } else {
      links[i] = 3;
      links[j] = 3;
    }
  }
  // classify: a closed triangle of three two-link atoms, or two one-link
  // atoms linked to each other; the first atom met in index order is A
  // (i for pairs) and marks its partners taken
  std::vector<int> role(n, 0);  // 2 / 1: first atom of a triangle / pair; -1 taken; 3 left
  for (int i = 0; i < n; ++i) role[i] = links[i];
  for (int i = 0; i < n; ++i) {
    if (role[i] == 2) {
      const int b = partner[2 * i], c = partner[2 * i + 1];
      const bool closed = role[b] == 2 && role[c] == 2 &&
                          ((partner[2 * b] == i && partner[2 * b + 1] == c) ||
                           (partner[2 * b + 1] == i && partner[2 * b] == c));
      if (closed) {
        role[b] = -2;
        role[c] = -2;
        len[3 * i + 2] = partner[2 * b + 1] == c ? len[3 * b + 1] : len[3 * b];
      } else {
        role[i] = role[b] = role[c] = 3;
      }
    } else if (role[i] == 1) {
      const int j = partner[2 * i];
      if (role[j] == 1) {
        role[j] = -1;
      } else {
        role[i] = role[j] = 3;
      }
    }
  }
  tri.clear();
  pair.clear();
  for (int i = 0; i < n; ++i) {
    if (role[i] == 2) {
      SettleTri g;
      g.a = i;
      g.b = partner[2 * i];
      g.c = partner[2 * i + 1];
      g.ma = mass[g.a];
      g.mb = mass[g.b];
      g.mc = mass[g.c];
      triangle_frame(len[3 * i], len[3 * i + 1], len[3 * i + 2], g.ma, g.mb, g.mc, g);
      tri.push_back(g);
    } else if (role[i] == 1) {
      SettlePair p;
      p.i = i;
      p.j = partner[2 * i];
      p.r0 = len[3 * i];
      p.mi = mass[p.i];
      p.mj = mass[p.j];
      p.k = 1.0f / (p.mi + p.mj);
      pair.push_back(p);
    }
  }
  remaining.clear();
  for (int p = 0; p < m; ++p)
    if (role[ai[p]] == 3) remaining.push_back(p);
  return kOk;
}

int settle_init(Settle& s, int n, int m, const int* ai, const int* aj, const float* r0,
                const float* mass) {
  std::vector<SettleTri> tri;
  std::vector<SettlePair> pair;
  int rc = settle_group(n, m, ai, aj, r0, mass, tri, pair, s.remaining);
  if (rc) return rc;
  s.n = n;
  s.nt = (int)tri.size();
  s.np = (int)pair.size();
  const size_t kt = std::max(s.nt, 1), kp = std::max(s.np, 1);
  SNB_CUDA_TRY(cudaMalloc(&s.d_tri, sizeof(SettleTri) * kt));
  SNB_CUDA_TRY(cudaMalloc(&s.d_pair, sizeof(SettlePair) * kp));
  SNB_CUDA_TRY(cudaMalloc(&s.d_last_ba, sizeof(float3) * kt));
  SNB_CUDA_TRY(cudaMalloc(&s.d_last_ca, sizeof(float3) * kt));
  SNB_CUDA_TRY(cudaMalloc(&s.d_last_ab, sizeof(float3) * kp));
  SNB_CUDA_TRY(cudaMalloc(&s.d_vir, sizeof(long long) * 6));
  SNB_CUDA_TRY(cudaMalloc(&s.d_err, sizeof(int)));
  SNB_CUDA_TRY(cudaMemset(s.d_err, 0, sizeof(int)));
  SNB_CUDA_TRY(cudaMemset(s.d_last_ba, 0, sizeof(float3) * kt));
  SNB_CUDA_TRY(cudaMemset(s.d_last_ca, 0, sizeof(float3) * kt));
  SNB_CUDA_TRY(cudaMemset(s.d_last_ab, 0, sizeof(float3) * kp));
  if (s.nt)
    SNB_CUDA_TRY(cudaMemcpy(s.d_tri, tri.data(), sizeof(SettleTri) * s.nt,
                            cudaMemcpyHostToDevice));
  if (s.np)
    SNB_CUDA_TRY(cudaMemcpy(s.d_pair, pair.data(), sizeof(SettlePair) * s.np,
                            cudaMemcpyHostToDevice));
  return kOk;
}

void settle_free(Settle& s) {
  cudaFree(s.d_tri);
  cudaFree(s.d_pair);
  cudaFree(s.d_last_ba);
  cudaFree(s.d_last_ca);
  cudaFree(s.d_last_ab);
  cudaFree(s.d_vir);
  cudaFree(s.d_err);
  s = Settle();
}

int launch_settle_remember(const Settle& s, const float3* crd, const Cell& cell,
                           const Cell& rcell, cudaStream_t st) {
  const int w = s.nt + s.np;
  if (w == 0) return kOk;
  k_settle_remember<<<ceil_div(std::max(w, 6), 256), 256, 0, st>>>(
      s.nt, s.d_tri, s.np, s.d_pair, crd, cell, rcell, s.d_last_ba, s.d_last_ca, s.d_last_ab,
      s.d_vir);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int launch_settle(const Settle& s, float3* crd, float3* vel, const Cell& cell,
                  const Cell& rcell, float dt, float v_factor, float x_factor, float* stress,
                  cudaStream_t st) {
  const int w = s.nt + s.np;
  if (w == 0) return kOk;
  k_settle<<<ceil_div(w, 128), 128, 0, st>>>(s.nt, s.d_tri, s.np, s.d_pair, crd, vel, cell,
                                             rcell, s.d_last_ba, s.d_last_ca, s.d_last_ab, dt,
                                             v_factor, x_factor, s.d_vir, s.d_err);
  SNB_CUDA_TRY(cudaGetLastError());
  if (stress) {
    k_settle_stress<<<1, 32, 0, st>>>(s.d_vir, rcell, stress);
    SNB_CUDA_TRY(cudaGetLastError());
  }
  return kOk;
}

}  // namespace snb
