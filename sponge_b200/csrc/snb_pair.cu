// Direct-space Lennard-Jones + erfc-screened Coulomb over the sorted half list:
// the Lennard_Jones_And_Direct_Coulomb_Device path
// (Lennard_Jones_force.cpp:45-137, pair terms Lennard_Jones_force.h:45-75)
// re-designed for sm_100a.
//
// Per listed pair (i, j) with r = |r_j - r_i| (minimum image) below cutoff:
//   F/r = (B' - A' r^-6) r^-8 - q_i q_j r^-3 (2 beta r/sqrt(pi) e^{-beta^2 r^2}
//         + erfc(beta r))
//   f_i += (F/r) dr, f_j -= (F/r) dr
//   E_LJ = (A'/12 r^-6 - B'/6) r^-6, E_C = q_i q_j erfc(beta r)/r
//   virial -= (F/r) dr (x) dr   (LTMatrix3 with summed off-diagonals)
// Energy and virial of a pair go to the atom with the smaller global id, as
// the reference's half list (global_j > global_i) assigns them.
//
// Layout: one warp per sorted atom i, lanes stride its CSR row (coalesced
// 4-byte index loads, 16-byte float4 {x,y,z,q} gathers that hit L1/L2 since
// the rows of neighbouring i are spatial neighbours).  The i force stays in
// registers and is reduced with warp shuffles; j forces go straight to the
// accumulators: 64-bit fixed point (deterministic, order-independent) or
// float atomics (the plain path).
#include <algorithm>
#include <cfloat>

#include <mutex>
#include <utility>
#include <vector>

#include "snb_internal.h"

namespace snb {

constexpr float kTwoOverSqrtPi = 1.1283791670955126f;

template <int ACCUM>
__device__ __forceinline__ void add_force(Accumulators& acc, int s, float fx,
                                          float fy, float fz) {
  const int N = acc.n;
  if (ACCUM == kAccumFixed) {
    red_add(acc.d_f + s, to_fixed_force(fx));
    red_add(acc.d_f + N + s, to_fixed_force(fy));
    red_add(acc.d_f + 2 * N + s, to_fixed_force(fz));
  } else {
    atomicAdd(acc.d_ff + s, fx);
    atomicAdd(acc.d_ff + N + s, fy);
    atomicAdd(acc.d_ff + 2 * N + s, fz);
  }
}

template <int ACCUM>
__device__ __forceinline__ void add_energy(Accumulators& acc, int s, float e,
                                           float elj, float ec) {
  const int N = acc.n;
  if (ACCUM == kAccumFixed) {
    red_add(acc.d_e + s, to_fixed_energy(e));
    red_add(acc.d_elj + s, to_fixed_energy(elj));
    red_add(acc.d_ec + s, to_fixed_energy(ec));
  } else {
    atomicAdd(acc.d_fe + s, e);
    atomicAdd(acc.d_fe + N + s, elj);
    atomicAdd(acc.d_fe + 2 * N + s, ec);
  }
}

template <int ACCUM>
__device__ __forceinline__ void add_virial(Accumulators& acc, int s, const float* v) {
  const int N = acc.n;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    if (ACCUM == kAccumFixed)
      red_add(acc.d_v + c * N + s, to_fixed_energy(v[c]));
    else
      atomicAdd(acc.d_fv + c * N + s, v[c]);
  }
}

// Each warp owns one row at a time and takes it in two phases.  Phase 1
// scans the listed candidates, four per lane in flight (index loads, then
// float4 gathers), and appends the j inside the cutoff to a per-warp list in
// shared memory (ballot + popc).  Phase 2 runs the pair terms over that list
// 32 pairs at a time, so every lane of the expensive part does useful work
// and the scan carries no force state.  A row with more hits than the list
// holds is taken in several rounds.
constexpr int kWarps = 8;      // rows in flight per block (warps per block)
constexpr int kHitCap = 512;   // per-warp hit list (entries)
// STASH: phase 1 keeps, per hit, the displacement and charge (float4) and
// the atom and LJ type-pair index (int2) in dynamic shared memory, so that
// phase 2 gathers nothing from global memory; the displacement is the one
// the cutoff test used, so the results are bitwise those of the plain list.
constexpr int kStashCap = 256;
// candidates per lane per scan round: a template parameter (2, 4 or 8), and
// rows in flight per block (4, 8 or 16 warps), that the engine's autotuner
// picks; 4 and 8 elsewhere

// The pair terms of i and j with the LJ coefficients A' = 12 A, B' = 6 B of
// their type pair.  COUL_ONLY: atom i's type has A' = B' = 0 with every
// type, so the LJ terms are exact zeros and are not formed (the results are
// bitwise the same).
template <int ACCUM, bool ENERGY, bool VIRIAL, bool COUL_ONLY = false, typename Args>
__device__ __forceinline__ void lj_pair_ab(const Args& a, Accumulators& acc, float A,
                                           float B, float qi, int gi, float4 e, int j,
                                           float& fx, float& fy, float& fz, float& e_lj,
                                           float& e_c, float* vir) {
  const float r2 = e.x * e.x + e.y * e.y + e.z * e.z;
  const float rinv = rsqrtf(r2);
  const float r = r2 * rinv;
  const float ir2 = rinv * rinv;
  const float ir6 = ir2 * ir2 * ir2;
  const float flj = COUL_ONLY ? 0.f : (B - A * ir6) * ir6 * ir2;
  const float qq = qi * e.w;
  const float br = a.beta * r;
  float ex;
  const float erfc_br = erfc_and_exp(br, &ex);
  const float fc = qq * rinv * ir2 * (br * kTwoOverSqrtPi * ex + erfc_br);
  const float fs = flj - fc;
  const float gx = fs * e.x, gy = fs * e.y, gz = fs * e.z;
  fx += gx;
  fy += gy;
  fz += gz;
  add_force<ACCUM>(acc, j, -gx, -gy, -gz);
  if (ENERGY || VIRIAL) {
    const bool own_i = gi < a.global[j];
    if (ENERGY) {
      const float elj = COUL_ONLY ? 0.f : (0.083333333f * A * ir6 - 0.166666667f * B) * ir6;
      const float ec = qq * erfc_br * rinv;
      if (own_i) {
        e_lj += elj;
        e_c += ec;
      } else {
        add_energy<ACCUM>(acc, j, elj + ec, elj, ec);
      }
    }
    if (VIRIAL) {
      float v[6];
      v[0] = -(gx * e.x);
      v[1] = -(gx * e.y + gy * e.x);
      v[2] = -(gy * e.y);
      v[3] = -(gx * e.z + gz * e.x);
      v[4] = -(gy * e.z + gz * e.y);
      v[5] = -(gz * e.z);
      if (own_i) {
#pragma unroll
        for (int c = 0; c < 6; ++c) vir[c] += v[c];
      } else {
        add_virial<ACCUM>(acc, j, v);
      }
    }
  }
}

// The same with the coefficients looked up from the types' pair index.
template <int ACCUM, bool ENERGY, bool VIRIAL, bool COUL_ONLY = false, typename Args>
__device__ __forceinline__ void lj_pair(const Args& a, Accumulators& acc,
                                        const float* sA, const float* sB, int ti,
                                        float qi, int gi, float4 e, int j, int tj,
                                        float& fx, float& fy, float& fz, float& e_lj,
                                        float& e_c, float* vir) {
  float A = 0.f, B = 0.f;
  if (!COUL_ONLY) {
    const int p = lj_pair_index(ti, tj);
    A = sA[p];
    B = sB[p];
  }
  lj_pair_ab<ACCUM, ENERGY, VIRIAL, COUL_ONLY>(a, acc, A, B, qi, gi, e, j, fx, fy, fz, e_lj,
                                               e_c, vir);
}

// SOLV 1 / 2: the solvent split of PairArgs::solvent_mode (pairs with both
// global ids >= solvent_begin left out / taken alone); 0: every pair.
template <int ACCUM, bool ENERGY, bool VIRIAL, bool ORTHO, bool BATCH, int kScanU,
          int SOLV = 0, int WARPS = kWarps, bool STASH = false>
__global__ void __launch_bounds__(32 * WARPS, 32 / WARPS)
k_lj_direct(PairArgs a, Accumulators acc) {
  constexpr int kCap = STASH ? kStashCap : kHitCap;
  static_assert(kScanU >= 1 && 32 * kScanU < kCap, "scan round exceeds the hit list");
  extern __shared__ float4 sh_dyn[];
  __shared__ int hits_all[STASH ? 1 : WARPS][STASH ? 1 : kHitCap];
  const int npair = a.n_types * (a.n_types + 1) / 2;
  // dynamic shared memory: [stash e: WARPS][kCap] float4, [stash jt] int2,
  // then the LJ tables
  float4* stash_e = sh_dyn;
  int2* stash_jt = reinterpret_cast<int2*>(sh_dyn + (STASH ? WARPS * kCap : 0));
  float* sA = reinterpret_cast<float*>(stash_jt + (STASH ? WARPS * kCap : 0));
  float* sB = sA + npair;
  for (int k = threadIdx.x; k < npair; k += blockDim.x) {
    sA[k] = a.A[k];
    sB[k] = a.B[k];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  int* hits = hits_all[STASH ? 0 : w];
  float4* se = stash_e + (STASH ? w * kCap : 0);
  int2* sjt = stash_jt + (STASH ? w * kCap : 0);
  if (a.nl_flags && a.nl_flags[1]) return;  // list overflowed: rows not written
  // Pruned rows: a prune pass scans the full rows and keeps the candidates
  // within cutoff + margin; the steps between scan only those.
  constexpr bool kPrunable = SOLV == 0;
  const bool prune_pass = kPrunable && a.prune != nullptr && a.prune[0] != 0;
  const bool use_inner = kPrunable && a.prune != nullptr && !prune_pass;
  const int* __restrict__ cols = use_inner ? a.cols_in : a.cols;
  const int* __restrict__ rcount = use_inner ? a.row_in_count : a.row_count;
  // Each block owns a contiguous range of sorted atoms, so the neighbours its
  // warps gather overlap and stay in this SM's L1.
  const int per_block = (a.n + gridDim.x - 1) / gridDim.x;
  const int i_begin = blockIdx.x * per_block;
  const int i_end = min(a.n, i_begin + per_block);
  const unsigned lt = (1u << lane) - 1u;
  for (int i = i_begin + w; i < i_end; i += WARPS) {
  const float4 pi = a.pos[i];
  const float3 ri = make_float3(pi.x, pi.y, pi.z);
  const int ti = a.type[i];
  const int gi = ENERGY || VIRIAL || SOLV ? a.global[i] : 0;
  const bool i_solvent = SOLV && gi >= a.solvent_begin;
  // box of atom i (and of all its pairs)
  const SysGeom* gs = BATCH ? a.bv.sys + a.bv.sys_of[i] : nullptr;
  const Cell& cell = BATCH ? gs->cell : a.cell;
  const Cell& rcell = BATCH ? gs->rcell : a.rcell;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  float e_lj = 0.f, e_c = 0.f;
  float vir[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const int k0 = a.row_start[i], k1 = k0 + rcount[i];
  int kept = 0;  // prune pass: entries kept so far
  // a type without LJ against every type (water H): Coulomb-only row
  bool coul_only = true;
  for (int t = lane; t < a.n_types; t += 32) {
    const int p = lj_pair_index(ti, t);
    coul_only = coul_only && sA[p] == 0.f && sB[p] == 0.f;
  }
  coul_only = __all_sync(0xffffffffu, coul_only);
  {
    // the warp's next row: start pulling its indices from HBM into L2 now
    // (row starts are multiples of 8 entries, so 16-byte aligned)
    const int inext = i + WARPS;
    if (lane == 0 && inext < i_end) {
      const int cn = rcount[inext];
      if (cn > 0)
        prefetch_l2(cols + a.row_start[inext], (unsigned)(cn * 4 + 15) & ~15u);
    }
  }
  // hits of the row taken in earlier rounds: lane l takes the row's hits
  // l, l + 32, ... in order whatever the rounds, so the float sums of i's
  // force are the same for every hit-list capacity and scan width
  int done = 0;
  // with up to 4 candidates per lane, each round's indices are loaded one
  // round ahead, so the gathers of a round wait only on their own load (at 8
  // the extra registers spill).  The index stream is read once: loaded
  // evict-first (__ldcs) so that L1 keeps the positions the rows share.
  constexpr bool kAhead = kScanU <= 4;
  int jn[kScanU];
#pragma unroll
  for (int u = 0; u < kScanU; ++u) {
    const int k = k0 + 32 * u + lane;
    jn[u] = kAhead && k < k1 ? __ldcs(cols + k) : -1;
  }
  for (int base = k0; base < k1;) {
    // phase 1: candidates -> hit list
    int count = 0;
    for (; base < k1 && count <= kCap - 32 * kScanU; base += 32 * kScanU) {
      int jj[kScanU];
#pragma unroll
      for (int u = 0; u < kScanU; ++u) {
        if (kAhead) {
          jj[u] = jn[u];
          const int k = base + 32 * (kScanU + u) + lane;
          jn[u] = k < k1 ? __ldcs(cols + k) : -1;
        } else {
          const int k = base + 32 * u + lane;
          jj[u] = k < k1 ? __ldcs(cols + k) : -1;
        }
      }
      float4 pp[kScanU];
      int tt[kScanU];
#pragma unroll
      for (int u = 0; u < kScanU; ++u) {
        if (jj[u] >= 0) pp[u] = a.pos[jj[u]];
        tt[u] = STASH && !coul_only && jj[u] >= 0 ? a.type[jj[u]] : 0;
      }
#pragma unroll
      for (int u = 0; u < kScanU; ++u) {
        bool in = false, keep = false;
        if (jj[u] >= 0) {
          const float3 dr = min_image_fast<ORTHO>(make_float3(pp[u].x, pp[u].y, pp[u].z),
                                                  ri, cell, rcell);
          const float d2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
          in = d2 < a.cutoff2;
          keep = kPrunable && d2 < a.prune2;
          if (SOLV && in) {
            const bool both = i_solvent && a.global[jj[u]] >= a.solvent_begin;
            in = SOLV == 1 ? !both : both;
          }
        }
        if (kPrunable && prune_pass) {  // warp-uniform
          const unsigned mk = __ballot_sync(0xffffffffu, keep);
          if (keep) a.cols_in[k0 + kept + __popc(mk & lt)] = jj[u];
          kept += __popc(mk);
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) {
          const int slot = count + __popc(m & lt);
          if (STASH) {
            const float3 dr = min_image_fast<ORTHO>(make_float3(pp[u].x, pp[u].y, pp[u].z),
                                                    ri, cell, rcell);
            se[slot] = make_float4(dr.x, dr.y, dr.z, pp[u].w);
            sjt[slot] = make_int2(jj[u], coul_only ? 0 : lj_pair_index(ti, tt[u]));
          } else {
            hits[slot] = jj[u];
          }
        }
        count += __popc(m);
      }
    }
    __syncwarp();
    // phase 2: pair terms over the hit list
    const int h0 = (lane - done) & 31;
    if (STASH && coul_only) {
      for (int h = h0; h < count; h += 32) {
        const int2 jt = sjt[h];
        lj_pair_ab<ACCUM, ENERGY, VIRIAL, true>(a, acc, 0.f, 0.f, pi.w, gi, se[h], jt.x, fx,
                                                fy, fz, e_lj, e_c, vir);
      }
    } else if (STASH) {
      for (int h = h0; h < count; h += 32) {
        const int2 jt = sjt[h];
        lj_pair_ab<ACCUM, ENERGY, VIRIAL>(a, acc, sA[jt.y], sB[jt.y], pi.w, gi, se[h], jt.x,
                                          fx, fy, fz, e_lj, e_c, vir);
      }
    } else if (coul_only) {
      for (int h = h0; h < count; h += 32) {
        const int j = hits[h];
        const float4 pj = a.pos[j];
        const float3 dr = min_image_fast<ORTHO>(make_float3(pj.x, pj.y, pj.z), ri, cell,
                                                rcell);
        lj_pair<ACCUM, ENERGY, VIRIAL, true>(a, acc, sA, sB, ti, pi.w, gi,
                                             make_float4(dr.x, dr.y, dr.z, pj.w), j, 0, fx,
                                             fy, fz, e_lj, e_c, vir);
      }
    } else {
      for (int h = h0; h < count; h += 32) {
        const int j = hits[h];
        const float4 pj = a.pos[j];
        const int tj = a.type[j];
        const float3 dr = min_image_fast<ORTHO>(make_float3(pj.x, pj.y, pj.z), ri, cell,
                                                rcell);
        lj_pair<ACCUM, ENERGY, VIRIAL>(a, acc, sA, sB, ti, pi.w, gi,
                                       make_float4(dr.x, dr.y, dr.z, pj.w), j, tj, fx, fy,
                                       fz, e_lj, e_c, vir);
      }
    }
    done += count;
    __syncwarp();
  }
  if (kPrunable && prune_pass && lane == 0) {
    a.row_in_count[i] = kept;
    a.prune_ref[i] = pi;
  }
  fx = warp_sum(fx);
  fy = warp_sum(fy);
  fz = warp_sum(fz);
  if (ENERGY) {
    e_lj = warp_sum(e_lj);
    e_c = warp_sum(e_c);
  }
  if (VIRIAL) {
#pragma unroll
    for (int c = 0; c < 6; ++c) vir[c] = warp_sum(vir[c]);
  }
  if (lane == 0) {
    add_force<ACCUM>(acc, i, fx, fy, fz);
    if (ENERGY) add_energy<ACCUM>(acc, i, e_lj + e_c, e_lj, e_c);
    if (VIRIAL) add_virial<ACCUM>(acc, i, vir);
  }
  }
}

using RowKern = void (*)(PairArgs, Accumulators);

// The plain single-box row kernel of W warps per block with or without the
// hit stash (which needs at most 4 candidates per lane per round).
template <int ACCUM, bool ENERGY, bool VIRIAL, int W, bool S>
static RowKern row_kernel(int u) {
  if constexpr (S)
    return u == 2 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 2, 0, W, true>
                  : k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 4, 0, W, true>;
  else
    return u == 2 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 2, 0, W>
         : u == 8 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 8, 0, W>
                  : k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 4, 0, W>;
}

// Raises a kernel's dynamic shared memory limit once, when it needs more
// than the default 48 KB.
static void allow_smem(RowKern k, size_t smem) {
  static std::mutex mu;
  static std::vector<std::pair<RowKern, size_t>> done;
  if (smem <= 48 * 1024) return;
  std::lock_guard<std::mutex> lock(mu);
  for (auto& d : done)
    if (d.first == k && d.second >= smem) return;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  done.push_back({k, smem});
}

template <int ACCUM, bool ENERGY, bool VIRIAL>
static void launch3(const PairArgs& a, Accumulators& acc, bool ortho, cudaStream_t st) {
  size_t smem = sizeof(float) * a.n_types * (a.n_types + 1);
  RowKern kern;
  // the launch-shape choices apply to the MD step's variant (fixed point,
  // force only, rectangular, one box, no solvent split); the others take 4
  // candidates per lane and 8 warps without the stash
  constexpr bool kTunable = ACCUM == kAccumFixed && !ENERGY && !VIRIAL;
  const bool tunable = kTunable && ortho;
  const bool single = a.bv.nsys == 0 && a.solvent_mode == 0;
  const int u = tunable ? a.unroll : 4;
  // rows in flight per block: 4, 8 or 16 warps for one box, 8 or 16 for a
  // batch; 8 for the other variants
  int wb = kWarps;
  if (tunable && a.solvent_mode == 0)
    wb = a.bv.nsys == 0 ? a.warps : (a.warps == 16 ? 16 : kWarps);
  const bool stash = tunable && single && a.stash;
  if (a.solvent_mode != 0 && a.bv.nsys == 0)
    kern = ortho ? (a.solvent_mode == 1 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 4, 1>
                                        : k_lj_direct<ACCUM, ENERGY, VIRIAL, true, false, 4, 2>)
                 : (a.solvent_mode == 1 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, false, false, 4, 1>
                                        : k_lj_direct<ACCUM, ENERGY, VIRIAL, false, false, 4, 2>);
  else if (a.bv.nsys > 0 && kTunable && wb == 16)
    kern = u == 2 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, true, 2, 0, 16>
         : u == 8 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, true, 8, 0, 16>
                  : k_lj_direct<ACCUM, ENERGY, VIRIAL, true, true, 4, 0, 16>;
  else if (a.bv.nsys > 0)
    kern = u == 2 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, true, 2>
         : u == 8 ? k_lj_direct<ACCUM, ENERGY, VIRIAL, true, true, 8>
                  : k_lj_direct<ACCUM, ENERGY, VIRIAL, true, true, 4>;
  else if (ortho) {
    if constexpr (kTunable) {
      if (wb == 4)
        kern = stash ? row_kernel<ACCUM, ENERGY, VIRIAL, 4, true>(u)
                     : row_kernel<ACCUM, ENERGY, VIRIAL, 4, false>(u);
      else if (wb == 16)
        kern = stash ? row_kernel<ACCUM, ENERGY, VIRIAL, 16, true>(u)
                     : row_kernel<ACCUM, ENERGY, VIRIAL, 16, false>(u);
      else
        kern = stash ? row_kernel<ACCUM, ENERGY, VIRIAL, kWarps, true>(u)
                     : row_kernel<ACCUM, ENERGY, VIRIAL, kWarps, false>(u);
    } else {
      kern = row_kernel<ACCUM, ENERGY, VIRIAL, kWarps, false>(u);
    }
  } else {
    kern = k_lj_direct<ACCUM, ENERGY, VIRIAL, false, false, 4>;
  }
  if (stash) smem += (sizeof(float4) + sizeof(int2)) * (size_t)wb * kStashCap;
  allow_smem(kern, smem);
  // persistent grid: as many blocks as fit at once, or the tuned count
  static int sms = 0;
  if (!sms) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const int threads = 32 * wb;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
  per_sm = std::max(per_sm, 1);
  if (a.blocks_per_sm > 0) per_sm = std::min(per_sm, a.blocks_per_sm);
  int blocks = std::max(1, std::min(sms * per_sm, ceil_div(a.n, threads / 32)));
  kern<<<blocks, threads, smem, st>>>(a, acc);
}

template <int ACCUM>
static void launch2(const PairArgs& a, Accumulators& acc, bool energy, bool virial,
                    bool ortho, cudaStream_t st) {
  if (energy && virial)
    launch3<ACCUM, true, true>(a, acc, ortho, st);
  else if (energy)
    launch3<ACCUM, true, false>(a, acc, ortho, st);
  else if (virial)
    launch3<ACCUM, false, true>(a, acc, ortho, st);
  else
    launch3<ACCUM, false, false>(a, acc, ortho, st);
}

int launch_pair(const PairArgs& a, Accumulators& acc, int accum, bool energy,
                bool virial, bool ortho, cudaStream_t st) {
  if (a.n <= 0) return kOk;
  if (accum == kAccumFixed)
    launch2<kAccumFixed>(a, acc, energy, virial, ortho, st);
  else
    launch2<kAccumFloat>(a, acc, energy, virial, ortho, st);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// The same pair terms over the cluster form of the list.  One warp per
// i-cluster (up to four sorted atoms, held in every lane's registers) at a
// time.  Phase 1 scans the row eight entries per round: lane l takes entry
// l/4 and its j atom l%4 (one 16-byte load, the entry's periodic image
// added), tests it against the four i atoms under the entry's mask and the
// cutoff, and appends each hit to the list of its i atom (ballot + popc):
// no index load per candidate, and the j atoms of an entry are contiguous.
// Phase 2 runs the pair terms of each i atom's list 32 at a time as the row
// kernel does, i force in registers, j forces to the accumulators.
// Coordinates are in the pair frame (each atom in its cell's image), so the
// displacement is (x_j + shift) - x_i with no rounding to an image.
constexpr int kCWarps = 8;
constexpr int kSubCap = 256;  // per i atom list of hits
constexpr int kCScanU = 2;    // rounds of eight entries in flight in phase 1

template <int ACCUM, bool ENERGY, bool VIRIAL>
__global__ void __launch_bounds__(32 * kCWarps, 3)
k_lj_clusters(ClusterPairArgs a, Accumulators acc) {
  extern __shared__ float sh_tab[];
  __shared__ int hits_all[kCWarps][kClusterSize][kSubCap];
  __shared__ float4 shift_tab[27];
  float* sA = sh_tab;
  float* sB = sh_tab + a.n_types * (a.n_types + 1) / 2;
  const int npair = a.n_types * (a.n_types + 1) / 2;
  for (int k = threadIdx.x; k < npair; k += blockDim.x) {
    sA[k] = a.A[k];
    sB[k] = a.B[k];
  }
  if (threadIdx.x < 27) {
    const int k = threadIdx.x;
    shift_tab[k] = make_float4((float)(k / 9 - 1) * a.box.x, (float)((k / 3) % 3 - 1) * a.box.y,
                               (float)(k % 3 - 1) * a.box.z, 0.f);
  }
  __syncthreads();
  if (a.nl_flags && a.nl_flags[1]) return;  // list overflowed: rows not written
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int nclus = *a.nclus;
  const int per_block = (nclus + gridDim.x - 1) / gridDim.x;
  const int c_end = min(nclus, (int)blockIdx.x * per_block + per_block);
  for (int c = blockIdx.x * per_block + w; c < c_end; c += kCWarps) {
    const int2 ci = a.clus[c];
    // the i atoms, broadcast from lanes 0..3
    const bool own = lane < ci.y;
    const float4 pl = own ? a.pos[ci.x + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int tl = own ? a.type[ci.x + lane] : 0;
    const int gl = (ENERGY || VIRIAL) && own ? a.global[ci.x + lane] : 0;
    float4 p_i[kClusterSize];
    int t_i[kClusterSize], g_i[kClusterSize];
    bool coul_only[kClusterSize];
#pragma unroll
    for (int ii = 0; ii < kClusterSize; ++ii) {
      p_i[ii] = make_float4(__shfl_sync(0xffffffffu, pl.x, ii), __shfl_sync(0xffffffffu, pl.y, ii),
                            __shfl_sync(0xffffffffu, pl.z, ii), __shfl_sync(0xffffffffu, pl.w, ii));
      t_i[ii] = __shfl_sync(0xffffffffu, tl, ii);
      g_i[ii] = __shfl_sync(0xffffffffu, gl, ii);
      // a type without LJ against every type (water H): Coulomb-only terms
      bool co = true;
      for (int t = lane; t < a.n_types; t += 32) {
        const int p = lj_pair_index(t_i[ii], t);
        co = co && sA[p] == 0.f && sB[p] == 0.f;
      }
      coul_only[ii] = __all_sync(0xffffffffu, co);
    }
    float f_i[kClusterSize][3];
    float elj_i[kClusterSize], ec_i[kClusterSize], vir_i[kClusterSize][6];
#pragma unroll
    for (int ii = 0; ii < kClusterSize; ++ii) {
      f_i[ii][0] = f_i[ii][1] = f_i[ii][2] = 0.f;
      elj_i[ii] = ec_i[ii] = 0.f;
#pragma unroll
      for (int q = 0; q < 6; ++q) vir_i[ii][q] = 0.f;
    }
    const int n_ent = min(a.crow_count[c], a.ccap);
    const int2* row = a.centry + (size_t)c * a.ccap;
    {
      // the warp's next row: start pulling its entries into L2 now (rows
      // start on 32-byte boundaries)
      const int cn = c + kCWarps;
      if (lane == 0 && cn < c_end) {
        const int m = min(a.crow_count[cn], a.ccap);
        if (m > 0)
          prefetch_l2(a.centry + (size_t)cn * a.ccap, (unsigned)(m * 8 + 15) & ~15u);
      }
    }
    const int jl = lane & 3, eo = lane >> 2;
    for (int base = 0; base < n_ent;) {
      // phase 1: candidates -> per-i hit lists, kCScanU rounds of eight
      // entries in flight per pass
      int cnt[kClusterSize] = {0, 0, 0, 0};
      for (; base < n_ent &&
             max(max(cnt[0], cnt[1]), max(cnt[2], cnt[3])) <= kSubCap - 32 * kCScanU;
           base += 8 * kCScanU) {
        int2 en[kCScanU];
#pragma unroll
        for (int u = 0; u < kCScanU; ++u) {
          const int e = base + 8 * u + eo;
          en[u] = e < n_ent ? row[e] : make_int2(0, 0);
        }
        float4 pp[kCScanU];
#pragma unroll
        for (int u = 0; u < kCScanU; ++u)
          if (((unsigned)en[u].y >> jl) & 0x1111u) pp[u] = a.pos[en[u].x + jl];
#pragma unroll
        for (int u = 0; u < kCScanU; ++u) {
          const unsigned col = ((unsigned)en[u].y >> jl) & 0x1111u;
          const unsigned code = ((unsigned)en[u].y >> 16) & 31u;
          float3 pj = make_float3(0.f, 0.f, 0.f);
          if (col) {
            const float4 sh = shift_tab[code];
            pj = make_float3(pp[u].x + sh.x, pp[u].y + sh.y, pp[u].z + sh.z);
          }
          const int hcode = (en[u].x + jl) | (int)(code << 27);
#pragma unroll
          for (int ii = 0; ii < kClusterSize; ++ii) {
            bool hit = false;
            if ((col >> (4 * ii)) & 1u) {
              const float dx = pj.x - p_i[ii].x, dy = pj.y - p_i[ii].y, dz = pj.z - p_i[ii].z;
              hit = dx * dx + dy * dy + dz * dz < a.cutoff2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) hits_all[w][ii][cnt[ii] + __popc(m & lt)] = hcode;
            cnt[ii] += __popc(m);
          }
        }
      }
      __syncwarp();
      // phase 2: pair terms of each i atom's hits
#pragma unroll
      for (int ii = 0; ii < kClusterSize; ++ii) {
        const int* hits = hits_all[w][ii];
        if (coul_only[ii]) {
          for (int h = lane; h < cnt[ii]; h += 32) {
            const int hc = hits[h];
            const int jj = hc & 0x7FFFFFF;
            const float4 pj = a.pos[jj];
            const float4 sh = shift_tab[(unsigned)hc >> 27];
            lj_pair<ACCUM, ENERGY, VIRIAL, true>(
                a, acc, sA, sB, t_i[ii], p_i[ii].w, g_i[ii],
                make_float4(pj.x + sh.x - p_i[ii].x, pj.y + sh.y - p_i[ii].y,
                            pj.z + sh.z - p_i[ii].z, pj.w),
                jj, 0, f_i[ii][0], f_i[ii][1], f_i[ii][2], elj_i[ii], ec_i[ii], vir_i[ii]);
          }
        } else {
          for (int h = lane; h < cnt[ii]; h += 32) {
            const int hc = hits[h];
            const int jj = hc & 0x7FFFFFF;
            const float4 pj = a.pos[jj];
            const int tj = a.type[jj];
            const float4 sh = shift_tab[(unsigned)hc >> 27];
            lj_pair<ACCUM, ENERGY, VIRIAL>(
                a, acc, sA, sB, t_i[ii], p_i[ii].w, g_i[ii],
                make_float4(pj.x + sh.x - p_i[ii].x, pj.y + sh.y - p_i[ii].y,
                            pj.z + sh.z - p_i[ii].z, pj.w),
                jj, tj, f_i[ii][0], f_i[ii][1], f_i[ii][2], elj_i[ii], ec_i[ii], vir_i[ii]);
          }
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int ii = 0; ii < kClusterSize; ++ii) {
      if (ii >= ci.y) break;  // warp-uniform
      const float fx = warp_sum(f_i[ii][0]), fy = warp_sum(f_i[ii][1]),
                  fz = warp_sum(f_i[ii][2]);
      float el = 0.f, ec = 0.f;
      if (ENERGY) {
        el = warp_sum(elj_i[ii]);
        ec = warp_sum(ec_i[ii]);
      }
      if (VIRIAL) {
#pragma unroll
        for (int q = 0; q < 6; ++q) vir_i[ii][q] = warp_sum(vir_i[ii][q]);
      }
      if (lane == 0) {
        add_force<ACCUM>(acc, ci.x + ii, fx, fy, fz);
        if (ENERGY) add_energy<ACCUM>(acc, ci.x + ii, el + ec, el, ec);
        if (VIRIAL) add_virial<ACCUM>(acc, ci.x + ii, vir_i[ii]);
      }
    }
  }
}

template <int ACCUM, bool ENERGY, bool VIRIAL>
static int launch_clusters3(const ClusterPairArgs& a, Accumulators& acc, cudaStream_t st) {
  const size_t smem = sizeof(float) * a.n_types * (a.n_types + 1);
  auto kern = k_lj_clusters<ACCUM, ENERGY, VIRIAL>;
  static int sms = 0;
  if (!sms) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kCWarps, smem);
  per_sm = std::max(per_sm, 1);
  if (a.blocks_per_sm > 0) per_sm = std::min(per_sm, a.blocks_per_sm);
  kern<<<sms * per_sm, 32 * kCWarps, smem, st>>>(a, acc);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

template <int ACCUM>
static int launch_clusters2(const ClusterPairArgs& a, Accumulators& acc, bool energy,
                            bool virial, cudaStream_t st) {
  if (energy && virial) return launch_clusters3<ACCUM, true, true>(a, acc, st);
  if (energy) return launch_clusters3<ACCUM, true, false>(a, acc, st);
  if (virial) return launch_clusters3<ACCUM, false, true>(a, acc, st);
  return launch_clusters3<ACCUM, false, false>(a, acc, st);
}

int launch_pair_clusters(const ClusterPairArgs& a, Accumulators& acc, int accum,
                         bool energy, bool virial, cudaStream_t st) {
  return accum == kAccumFixed ? launch_clusters2<kAccumFixed>(a, acc, energy, virial, st)
                              : launch_clusters2<kAccumFloat>(a, acc, energy, virial, st);
}

// ---------------------------------------------------------------------------
// Soft-core variant: Lennard_Jones_And_Direct_Coulomb_Soft_Core_CUDA
// (LJ_soft_core.cpp:196-461; pair terms LJ_soft_core.h:33-149).
// A pair whose end states both have LJ (A'_A * A'_B != 0), or neither has
// (A'_A + A'_B == 0), mixes the hard-core forms linearly in lambda; any other
// pair uses the soft-core radius r_sc = (r^6 + alpha lambda^p sigma^6)^(1/6)
// for state A and (r^6 + alpha (1-lambda)^p sigma^6)^(1/6) for state B, with
// sigma^6 = max(A'/(2B'), sigma_min^6), or the input sigma^6 when A' or B' is 0.
__device__ __forceinline__ float lj_e(float A, float B, float ir6) {
  return (0.083333333f * A * ir6 - 0.166666667f * B) * ir6;
}
__device__ __forceinline__ float sc_sigma(float A, float B, float s6, float s6min) {
  return (A == 0.f || B == 0.f) ? s6 : fmaxf(0.5f * A / B, s6min);
}
// dU/dlambda chain term (Get_Soft_Core_dU_dlambda, LJ_soft_core.h:142-149)
__device__ __forceinline__ float sc_dudl(float F, float sigma, float rsc, float alpha,
                                         float p, float lambda) {
  float rsc2 = rsc * rsc;
  return 0.16666667f * p * alpha * (1.0f - lambda) * powf(lambda + FLT_MIN, p - 1.0f) *
         F / (rsc2 * rsc2) * sigma;
}
__device__ __forceinline__ float coul_e(float qq, float beta, float r) {
  return qq * erfcf(beta * r) / r;
}
__device__ __forceinline__ float coul_f(float qq, float beta, float r) {
  float br = beta * r;
  return qq / (r * r * r) * (br * kTwoOverSqrtPi * expf(-br * br) + erfcf(br));
}

template <int ACCUM, bool ENERGY, bool VIRIAL, bool DUDL>
__global__ void __launch_bounds__(256)
k_lj_soft(SoftArgs a, Accumulators acc, long long* dudl_total) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= a.n) return;
  if (a.nl_flags && a.nl_flags[1]) return;  // list overflowed: rows not written
  const float lam = a.lambda, lam_ = 1.0f - a.lambda;
  const float alp_A = a.alpha * powf(lam, a.p);
  const float alp_B = a.alpha * powf(lam_, a.p);
  const float4 pi = a.pos[i];
  const float3 ri = make_float3(pi.x, pi.y, pi.z);
  const int2 pri = a.par[i];
  const int tAi = pri.x & 0xffff, tBi = pri.x >> 16;
  const float dqi = DUDL && a.dq ? a.dq[i] : 0.f;
  const int gi = ENERGY || VIRIAL ? a.global[i] : 0;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  float e_lj = 0.f, e_c = 0.f, e_inter = 0.f, e_intra = 0.f;
  float du_lj = 0.f, du_c = 0.f;
  float vir[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  const int k0 = a.row_start[i], k1 = k0 + a.row_count[i];
  for (int k = k0 + lane; k < k1; k += 32) {
    const int j = a.cols[k];
    const float4 pj = a.pos[j];
    const float3 dr = min_image_fast<false>(make_float3(pj.x, pj.y, pj.z), ri, a.cell,
                                            a.rcell);
    const float r2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
    if (!(r2 < a.cutoff2)) continue;
    const int2 prj = a.par[j];
    const int tAj = prj.x & 0xffff, tBj = prj.x >> 16;
    const int pA = lj_pair_index(tAi, tAj), pB = lj_pair_index(tBi, tBj);
    const float AA = a.AA[pA], AB = a.AB[pA], BA = a.BA[pB], BB = a.BB[pB];
    const float r = sqrtf(r2);
    const float qq = pi.w * pj.w;
    float fs, elj, ec, dl = 0.f, dc = 0.f;
    if (BA * AA != 0.f || BA + AA == 0.f) {
      const float ir2 = 1.0f / r2, ir6 = ir2 * ir2 * ir2;
      fs = lam_ * (AB - AA * ir6) * ir6 * ir2 + lam * (BB - BA * ir6) * ir6 * ir2 -
           coul_f(qq, a.beta, r);
      elj = lam_ * lj_e(AA, AB, ir6) + lam * lj_e(BA, BB, ir6);
      ec = coul_e(qq, a.beta, r);
      if (DUDL) {
        dl = lj_e(BA, BB, ir6) - lj_e(AA, AB, ir6);
        const float dqj = a.dq ? a.dq[j] : 0.f;
        dc = erfcf(a.beta * r) * (dqj * pi.w + pj.w * dqi) / r;
      }
    } else {
      const float sA = sc_sigma(AA, AB, a.sigma6, a.sigma6_min);
      const float sB = sc_sigma(BA, BB, a.sigma6, a.sigma6_min);
      const float r6 = r2 * r2 * r2;
      const float rA = powf(r6 + alp_A * sA, 0.16666667f);
      const float rB = powf(r6 + alp_B * sB, 0.16666667f);
      const float r4 = r2 * r2;
      const float iA2 = 1.0f / (rA * rA), iA6 = iA2 * iA2 * iA2;
      const float iB2 = 1.0f / (rB * rB), iB6 = iB2 * iB2 * iB2;
      const float flA = r4 * (AB - AA * iA6) * iA6 * iA6;
      const float flB = r4 * (BB - BA * iB6) * iB6 * iB6;
      const float bA = a.beta * rA, bB = a.beta * rB;
      const float fcA = qq * r4 *
                        (expf(-bA * bA) * kTwoOverSqrtPi * a.beta + erfcf(bA) / rA) * iA6;
      const float fcB = qq * r4 *
                        (expf(-bB * bB) * kTwoOverSqrtPi * a.beta + erfcf(bB) / rB) * iB6;
      fs = lam_ * flA + lam * flB - (lam_ * fcA + lam * fcB);
      ec = lam_ * coul_e(qq, a.beta, rA) + lam * coul_e(qq, a.beta, rB);
      elj = lam_ * lj_e(AA, AB, iA6) + lam * lj_e(BA, BB, iB6);
      if (DUDL) {
        dl = lj_e(BA, BB, iB6) - lj_e(AA, AB, iA6);
        dl += sc_dudl((AB - AA * iA6) * iA6 * iA2, sA, rA, a.alpha, a.p, lam) -
              sc_dudl((BB - BA * iB6) * iB6 * iB2, sB, rB, a.alpha, a.p, lam_);
        const float dqj = a.dq ? a.dq[j] : 0.f;
        const float qd = dqj * pi.w + pj.w * dqi;
        dc = coul_e(qq, a.beta, rB) - coul_e(qq, a.beta, rA);
        dc += sc_dudl(coul_f(qq, a.beta, rB), sB, rB, a.alpha, a.p, lam_) -
              sc_dudl(coul_f(qq, a.beta, rA), sA, rA, a.alpha, a.p, lam);
        dc += lam * erfcf(a.beta * rB) * qd / rB + lam_ * erfcf(a.beta * rA) * qd / rA;
      }
    }
    const float gx = fs * dr.x, gy = fs * dr.y, gz = fs * dr.z;
    if (!DUDL) {
      fx += gx;
      fy += gy;
      fz += gz;
      add_force<ACCUM>(acc, j, -gx, -gy, -gz);
    }
    if (DUDL) {
      du_lj += dl;
      du_c += dc;
    }
    if (ENERGY || VIRIAL) {
      const bool own_i = gi < a.global[j];
      const bool intra = pri.y == prj.y;
      if (ENERGY) {
        if (own_i) {
          e_lj += elj;
          e_c += ec;
          if (intra) e_intra += elj; else e_inter += elj;
        } else {
          add_energy<ACCUM>(acc, j, elj + ec, elj, ec);
          const int N = acc.n;
          if (ACCUM == kAccumFixed)
            red_add(acc.d_eaux + (intra ? N : 0) + j, to_fixed_energy(elj));
          else
            atomicAdd(acc.d_feaux + (intra ? N : 0) + j, elj);
        }
      }
      if (VIRIAL) {
        float v[6];
        v[0] = -(gx * dr.x);
        v[1] = -(gx * dr.y + gy * dr.x);
        v[2] = -(gy * dr.y);
        v[3] = -(gx * dr.z + gz * dr.x);
        v[4] = -(gy * dr.z + gz * dr.y);
        v[5] = -(gz * dr.z);
        if (own_i) {
#pragma unroll
          for (int c = 0; c < 6; ++c) vir[c] += v[c];
        } else {
          add_virial<ACCUM>(acc, j, v);
        }
      }
    }
  }
  if (DUDL) {
    du_lj = warp_sum(du_lj);
    du_c = warp_sum(du_c);
    if (lane == 0) {
      red_add(dudl_total, to_fixed_energy(du_lj));
      red_add(dudl_total + 1, to_fixed_energy(du_c));
    }
    return;
  }
  fx = warp_sum(fx);
  fy = warp_sum(fy);
  fz = warp_sum(fz);
  if (ENERGY) {
    e_lj = warp_sum(e_lj);
    e_c = warp_sum(e_c);
    e_inter = warp_sum(e_inter);
    e_intra = warp_sum(e_intra);
  }
  if (VIRIAL) {
#pragma unroll
    for (int c = 0; c < 6; ++c) vir[c] = warp_sum(vir[c]);
  }
  if (lane == 0) {
    add_force<ACCUM>(acc, i, fx, fy, fz);
    if (ENERGY) {
      add_energy<ACCUM>(acc, i, e_lj + e_c, e_lj, e_c);
      const int N = acc.n;
      if (ACCUM == kAccumFixed) {
        red_add(acc.d_eaux + i, to_fixed_energy(e_inter));
        red_add(acc.d_eaux + N + i, to_fixed_energy(e_intra));
      } else {
        atomicAdd(acc.d_feaux + i, e_inter);
        atomicAdd(acc.d_feaux + N + i, e_intra);
      }
    }
    if (VIRIAL) add_virial<ACCUM>(acc, i, vir);
  }
}

// Soft-core pair terms without dU/dlambda (the forms of k_lj_soft): force
// over r, LJ and Coulomb energies.  alp_A = alpha lambda^p, alp_B = alpha
// (1 - lambda)^p.
__device__ __forceinline__ void soft_pair(const SoftArgs& a, float AA, float AB, float BA,
                                          float BB, float r2, float qq, float alp_A,
                                          float alp_B, float& fs, float& elj, float& ec) {
  const float lam = a.lambda, lam_ = 1.0f - a.lambda;
  const float r = sqrtf(r2);
  if (BA * AA != 0.f || BA + AA == 0.f) {
    const float ir2 = 1.0f / r2, ir6 = ir2 * ir2 * ir2;
    fs = lam_ * (AB - AA * ir6) * ir6 * ir2 + lam * (BB - BA * ir6) * ir6 * ir2 -
         coul_f(qq, a.beta, r);
    elj = lam_ * lj_e(AA, AB, ir6) + lam * lj_e(BA, BB, ir6);
    ec = coul_e(qq, a.beta, r);
  } else {
    const float sA = sc_sigma(AA, AB, a.sigma6, a.sigma6_min);
    const float sB = sc_sigma(BA, BB, a.sigma6, a.sigma6_min);
    const float r6 = r2 * r2 * r2;
    const float rA = powf(r6 + alp_A * sA, 0.16666667f);
    const float rB = powf(r6 + alp_B * sB, 0.16666667f);
    const float r4 = r2 * r2;
    const float iA2 = 1.0f / (rA * rA), iA6 = iA2 * iA2 * iA2;
    const float iB2 = 1.0f / (rB * rB), iB6 = iB2 * iB2 * iB2;
    const float flA = r4 * (AB - AA * iA6) * iA6 * iA6;
    const float flB = r4 * (BB - BA * iB6) * iB6 * iB6;
    const float bA = a.beta * rA, bB = a.beta * rB;
    const float fcA =
        qq * r4 * (expf(-bA * bA) * kTwoOverSqrtPi * a.beta + erfcf(bA) / rA) * iA6;
    const float fcB =
        qq * r4 * (expf(-bB * bB) * kTwoOverSqrtPi * a.beta + erfcf(bB) / rB) * iB6;
    fs = lam_ * flA + lam * flB - (lam_ * fcA + lam * fcB);
    ec = lam_ * coul_e(qq, a.beta, rA) + lam * coul_e(qq, a.beta, rB);
    elj = lam_ * lj_e(AA, AB, iA6) + lam * lj_e(BA, BB, iB6);
  }
}

// Soft-core LJ + direct Coulomb for the fused engine, in the two-phase row
// scheme of k_lj_direct (scan to a shared hit list, then dense batches of
// pair terms).  A pair whose end states carry the same LJ parameters
// (A'_A == A'_B and B'_A == B'_B, as between unperturbed atoms) takes the
// plain pair terms of lj_pair, to which the lambda mix of the two equal
// forms reduces; the other pairs take soft_pair.  Energies and virial split
// by global id as in k_lj_direct; no inter/intra split and no dU/dlambda
// (the module's k_lj_soft provides those).
template <int ACCUM, bool ENERGY, bool VIRIAL>
__global__ void __launch_bounds__(256, 4)
k_lj_soft_rows(SoftArgs a, Accumulators acc) {
  constexpr int kScanU = 4;
  extern __shared__ float sh_soft[];
  __shared__ int hits_all[kWarps][kHitCap];
  const int pA_n = a.n_types_A * (a.n_types_A + 1) / 2;
  const int pB_n = a.n_types_B * (a.n_types_B + 1) / 2;
  float* sAA = sh_soft;
  float* sAB = sAA + pA_n;
  float* sBA = sAB + pA_n;
  float* sBB = sBA + pB_n;
  for (int k = threadIdx.x; k < pA_n; k += blockDim.x) {
    sAA[k] = a.AA[k];
    sAB[k] = a.AB[k];
  }
  for (int k = threadIdx.x; k < pB_n; k += blockDim.x) {
    sBA[k] = a.BA[k];
    sBB[k] = a.BB[k];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  int* hits = hits_all[w];
  if (a.nl_flags && a.nl_flags[1]) return;  // list overflowed: rows not written
  // pruned rows, as in k_lj_direct
  const bool prune_pass = a.prune != nullptr && a.prune[0] != 0;
  const bool use_inner = a.prune != nullptr && !prune_pass;
  const int* __restrict__ cols = use_inner ? a.cols_in : a.cols;
  const int* __restrict__ rcount = use_inner ? a.row_in_count : a.row_count;
  const float alp_A = a.alpha * powf(a.lambda, a.p);
  const float alp_B = a.alpha * powf(1.0f - a.lambda, a.p);
  const int per_block = (a.n + gridDim.x - 1) / gridDim.x;
  const int i_begin = blockIdx.x * per_block;
  const int i_end = min(a.n, i_begin + per_block);
  const unsigned lt = (1u << lane) - 1u;
  // the plain-path constants of lj_pair
  PairArgs pa;
  pa.beta = a.beta;
  pa.global = a.global;
  for (int i = i_begin + w; i < i_end; i += kWarps) {
    const float4 pi = a.pos[i];
    const float3 ri = make_float3(pi.x, pi.y, pi.z);
    const int2 pri = a.par[i];
    const int tAi = pri.x & 0xffff, tBi = pri.x >> 16;
    const int gi = ENERGY || VIRIAL ? a.global[i] : 0;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    float e_lj = 0.f, e_c = 0.f;
    float vir[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int k0 = a.row_start[i], k1 = k0 + rcount[i];
    int kept = 0;  // prune pass: entries kept so far
    for (int base = k0; base < k1;) {
      int count = 0;
      for (; base < k1 && count <= kHitCap - 32 * kScanU; base += 32 * kScanU) {
        int jj[kScanU];
#pragma unroll
        for (int u = 0; u < kScanU; ++u) {
          const int k = base + 32 * u + lane;
          jj[u] = k < k1 ? cols[k] : -1;
        }
        float4 pp[kScanU];
#pragma unroll
        for (int u = 0; u < kScanU; ++u)
          if (jj[u] >= 0) pp[u] = a.pos[jj[u]];
#pragma unroll
        for (int u = 0; u < kScanU; ++u) {
          bool in = false, keep = false;
          if (jj[u] >= 0) {
            const float3 dr = min_image_fast<true>(make_float3(pp[u].x, pp[u].y, pp[u].z),
                                                   ri, a.cell, a.rcell);
            const float d2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
            in = d2 < a.cutoff2;
            keep = d2 < a.prune2;
          }
          if (prune_pass) {  // warp-uniform
            const unsigned mk = __ballot_sync(0xffffffffu, keep);
            if (keep) a.cols_in[k0 + kept + __popc(mk & lt)] = jj[u];
            kept += __popc(mk);
          }
          const unsigned m = __ballot_sync(0xffffffffu, in);
          if (in) hits[count + __popc(m & lt)] = jj[u];
          count += __popc(m);
        }
      }
      __syncwarp();
      for (int h = lane; h < count; h += 32) {
        const int j = hits[h];
        const float4 pj = a.pos[j];
        const int2 prj = a.par[j];
        const float3 dr = min_image_fast<true>(make_float3(pj.x, pj.y, pj.z), ri, a.cell,
                                               a.rcell);
        const int pA = lj_pair_index(tAi, prj.x & 0xffff);
        const int pB = lj_pair_index(tBi, prj.x >> 16);
        const float AA = sAA[pA], AB = sAB[pA], BA = sBA[pB], BB = sBB[pB];
        if (AA == BA && AB == BB) {
          // one table entry carries the pair's (equal) end-state parameters
          lj_pair<ACCUM, ENERGY, VIRIAL>(pa, acc, sAA, sAB, tAi, pi.w, gi,
                                         make_float4(dr.x, dr.y, dr.z, pj.w), j,
                                         prj.x & 0xffff, fx, fy, fz, e_lj, e_c, vir);
          continue;
        }
        const float r2 = dr.x * dr.x + dr.y * dr.y + dr.z * dr.z;
        float fs, elj, ec;
        soft_pair(a, AA, AB, BA, BB, r2, pi.w * pj.w, alp_A, alp_B, fs, elj, ec);
        const float gx = fs * dr.x, gy = fs * dr.y, gz = fs * dr.z;
        fx += gx;
        fy += gy;
        fz += gz;
        add_force<ACCUM>(acc, j, -gx, -gy, -gz);
        if (ENERGY || VIRIAL) {
          const bool own_i = gi < a.global[j];
          if (ENERGY) {
            if (own_i) {
              e_lj += elj;
              e_c += ec;
            } else {
              add_energy<ACCUM>(acc, j, elj + ec, elj, ec);
            }
          }
          if (VIRIAL) {
            float v[6];
            v[0] = -(gx * dr.x);
            v[1] = -(gx * dr.y + gy * dr.x);
            v[2] = -(gy * dr.y);
            v[3] = -(gx * dr.z + gz * dr.x);
            v[4] = -(gy * dr.z + gz * dr.y);
            v[5] = -(gz * dr.z);
            if (own_i) {
#pragma unroll
              for (int c = 0; c < 6; ++c) vir[c] += v[c];
            } else {
              add_virial<ACCUM>(acc, j, v);
            }
          }
        }
      }
      __syncwarp();
    }
    if (prune_pass && lane == 0) {
      a.row_in_count[i] = kept;
      a.prune_ref[i] = pi;
    }
    fx = warp_sum(fx);
    fy = warp_sum(fy);
    fz = warp_sum(fz);
    if (ENERGY) {
      e_lj = warp_sum(e_lj);
      e_c = warp_sum(e_c);
    }
    if (VIRIAL) {
#pragma unroll
      for (int c = 0; c < 6; ++c) vir[c] = warp_sum(vir[c]);
    }
    if (lane == 0) {
      add_force<ACCUM>(acc, i, fx, fy, fz);
      if (ENERGY) add_energy<ACCUM>(acc, i, e_lj + e_c, e_lj, e_c);
      if (VIRIAL) add_virial<ACCUM>(acc, i, vir);
    }
  }
}

int launch_soft_rows(const SoftArgs& a, Accumulators& acc, bool energy, bool virial,
                     cudaStream_t st) {
  if (a.n <= 0) return kOk;
  const size_t smem = sizeof(float) * (a.n_types_A * (a.n_types_A + 1) +
                                       a.n_types_B * (a.n_types_B + 1));
  using Kern = void (*)(SoftArgs, Accumulators);
  Kern kern = energy && virial ? k_lj_soft_rows<kAccumFixed, true, true>
              : energy         ? k_lj_soft_rows<kAccumFixed, true, false>
              : virial         ? k_lj_soft_rows<kAccumFixed, false, true>
                               : k_lj_soft_rows<kAccumFixed, false, false>;
  if (smem > 48 * 1024) return fail(kNotSupported, "soft-core rows: type tables too large");
  static int sms = 0;
  if (!sms) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kWarps, smem);
  per_sm = std::max(per_sm, 1);
  const int blocks = std::max(1, std::min(sms * per_sm, ceil_div(a.n, kWarps)));
  kern<<<blocks, 32 * kWarps, smem, st>>>(a, acc);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

template <int ACCUM>
static void launch_soft2(const SoftArgs& a, Accumulators& acc, bool energy, bool virial,
                         bool dudl, long long* dt, cudaStream_t st) {
  dim3 grid(ceil_div(a.n, 8)), block(256);
  if (dudl)
    k_lj_soft<ACCUM, false, false, true><<<grid, block, 0, st>>>(a, acc, dt);
  else if (energy && virial)
    k_lj_soft<ACCUM, true, true, false><<<grid, block, 0, st>>>(a, acc, dt);
  else if (energy)
    k_lj_soft<ACCUM, true, false, false><<<grid, block, 0, st>>>(a, acc, dt);
  else if (virial)
    k_lj_soft<ACCUM, false, true, false><<<grid, block, 0, st>>>(a, acc, dt);
  else
    k_lj_soft<ACCUM, false, false, false><<<grid, block, 0, st>>>(a, acc, dt);
}

int launch_soft(const SoftArgs& a, Accumulators& acc, int accum, bool energy,
                bool virial, bool dudl, long long* dudl_total, cudaStream_t st) {
  if (a.n <= 0) return kOk;
  if (accum == kAccumFixed)
    launch_soft2<kAccumFixed>(a, acc, energy, virial, dudl, dudl_total, st);
  else
    launch_soft2<kAccumFloat>(a, acc, energy, virial, dudl, dudl_total, st);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace snb
