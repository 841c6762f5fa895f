// Neighbor list build: the NEIGHBOR_LIST path (neighbor_list.cpp) re-designed
// for sm_100a.
//
// The pair criterion is the reference's, bit for bit: pair (i, j) with global
// ids gi < gj is listed when |Get_Displacement(crd_i, crd_j)|^2 < rl2, with
// rl2 = (0.5*(cutoff+skin))^2*4 and the minimum image and square evaluated in
// the reference's operation order without FMA contraction
// (neighbor_list.cpp:509-517, 847; utils/boundary.h:31); excluded pairs are
// dropped when gj is in the exclusion list of gi (:744-803).
//
// The layout is different.  Atoms are counting-sorted into cells of side
// L/floor(L/((cutoff+skin)/2)) with a stable order inside each cell (caller
// index), so the sorted order and the list are deterministic.  One warp scans,
// for one sorted atom i, the atoms after i in its own cell and the neighbor
// cells its cell owns (+-2 cells), walked as runs of consecutive cells along
// z: each run is one contiguous slice of the sorted coordinate array, read
// with coalesced 16-byte loads, and is trimmed to the cells whose box comes
// within rl of atom i.  Hits go in one pass into rows of fixed capacity;
// a row that would overflow raises a flag and the host regrows the rows.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <map>
#include <vector>

#include "snb_internal.h"

namespace snb {

// ---------------------------------------------------------------------------
// Refresh decision (Check_Refresh, neighbor_list.cpp:307-321): any atom moved
// more than skin*skin_permit since the last build.
template <bool BATCH>
__global__ void k_check_refresh(int n, const float3* __restrict__ crd,
                                const float3* __restrict__ old_crd, Cell cell,
                                Cell rcell, float permit2, int* flags, BatchView bv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool moved = false;
  if (i < n) {
    if (BATCH) {
      const SysGeom& g = bv.sys[bv.sys_of[i]];
      cell = g.cell;
      rcell = g.rcell;
    }
    float3 d = min_image_fast<false>(crd[i], old_crd[i], cell, rcell);
    const float d2 = d.x * d.x + d.y * d.y + d.z * d.z;
    moved = d2 > permit2;
    if (BATCH && bv.box_need) box_mark(bv.box_need, bv.sys_of[i], d2, permit2);
  }
  if (__any_sync(0xffffffffu, moved) && (threadIdx.x & 31) == 0)
    atomicExch(&flags[kFlagNeed], 1);
}

__global__ void k_set_need(int* flags, int v) { flags[kFlagNeed] = v; }

// A rebuild of every system: the need flag, the full flag and each system's
// flag of a batch (nsys 0: one box).
__global__ void k_set_need_all(int* flags, unsigned char* box_need, int nsys) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    flags[kFlagNeed] = 1;
    flags[kFlagFull] = 1;
  }
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nsys; s += gridDim.x * blockDim.x)
    box_need[s] = 1;
}

// ---------------------------------------------------------------------------
// Binning.  Cell of the wrapped coordinate with uniform cells of side a_ii/N.
// The coordinate is wrapped into the brick [0, a11) x [0, a22) x [0, a33),
// which tiles space under the lattice of the lower-triangular cell (the
// reduction of Put_Atom_In_Grids, neighbor_list.cpp:365-373; for a
// rectangular box it is x - floor(x / L) L per axis).
__device__ __forceinline__ int wrapped_cell(float3 r, const Cell& cell, int Nx,
                                            int Ny, int Nz) {
  float z = r.z, y = r.y, x = r.x;
  const float k3 = floorf(z / cell.a33);
  z -= k3 * cell.a33;
  y -= k3 * cell.a32;
  const float k2 = floorf(y / cell.a22);
  y -= k2 * cell.a22;
  x -= k3 * cell.a31 + k2 * cell.a21;
  x -= floorf(x / cell.a11) * cell.a11;
  int nx = (int)(x / cell.a11 * Nx);
  int ny = (int)(y / cell.a22 * Ny);
  int nz = (int)(z / cell.a33 * Nz);
  nx = nx < 0 ? 0 : (nx < Nx ? nx : Nx - 1);
  ny = ny < 0 ? 0 : (ny < Ny ? ny : Ny - 1);
  nz = nz < 0 ? 0 : (nz < Nz ? nz : Nz - 1);
  return (nx * Ny + ny) * Nz + nz;
}

// Order key of an atom inside its cell for the cluster form: the cell's four
// xy quarter columns in the order (0,0) (0,1) (1,1) (1,0), z rising in the
// first and third and falling in the second and fourth, so that consecutive
// atoms stay close across the turns; z in 2^-22 steps of the cell height.
__device__ __forceinline__ int cell_order_key(float3 r, const Cell& cell, int Nx, int Ny,
                                              int Nz, int c) {
  const float x = r.x - floorf(r.x / cell.a11) * cell.a11;
  const float y = r.y - floorf(r.y / cell.a22) * cell.a22;
  const float z = r.z - floorf(r.z / cell.a33) * cell.a33;
  const int cz = c % Nz, cy = (c / Nz) % Ny, cx = c / (Nz * Ny);
  const bool hx = x / cell.a11 * Nx - (float)cx >= 0.5f;
  const bool hy = y / cell.a22 * Ny - (float)cy >= 0.5f;
  const int q = hx ? (hy ? 2 : 3) : (hy ? 1 : 0);
  int zq = (int)((z / cell.a33 * Nz - (float)cz) * 4194304.0f);
  zq = zq < 0 ? 0 : (zq > 4194303 ? 4194303 : zq);
  if (q & 1) zq = 4194303 - zq;
  return (q << 22) | zq;
}

template <bool BATCH>
__global__ void k_bin_count(int n, const float3* __restrict__ crd, Cell cell,
                            int Nx, int Ny, int Nz, int* __restrict__ atom_cell,
                            int* __restrict__ atom_slot, int* __restrict__ cell_count,
                            int* __restrict__ excl_count, const int* flags,
                            BatchView bv, int* __restrict__ atom_key) {
  if (flags[kFlagNeed] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (BATCH && !box_rebuilds(bv.box_need, bv.sys_of, i)) return;
  int c;
  if (BATCH) {
    const SysGeom& g = bv.sys[bv.sys_of[i]];
    c = g.cell_begin + wrapped_cell(crd[i], g.cell, g.Nx, g.Ny, g.Nz);
  } else {
    c = wrapped_cell(crd[i], cell, Nx, Ny, Nz);
    if (atom_key) atom_key[i] = cell_order_key(crd[i], cell, Nx, Ny, Nz, c);
  }
  atom_cell[i] = c;
  atom_slot[i] = atomicAdd(&cell_count[c], 1);
  if (excl_count) excl_count[i] = 0;
}

// Excluded partners per atom, E(x) = {y : the pair (x, y) is removed}: the
// reference removes a pair when the larger id is in the exclusion list of
// the smaller one, so an entry y of list(x) counts only when y > x and then
// excludes the pair for both ends.  Up to kExclCap partners are kept per
// atom; the count is exact, and atoms with more use the list lookup.
constexpr int kExclCap = 16;

__global__ void k_bin_scatter(int n, const int* __restrict__ atom_cell,
                              const int* __restrict__ atom_slot,
                              const int* __restrict__ cell_start,
                              int* __restrict__ unsorted, const int* __restrict__ excl_start,
                              const int* __restrict__ excl_list,
                              const int* __restrict__ excl_numbers,
                              int* __restrict__ excl_count, int* __restrict__ excl_partner,
                              const int* flags, const unsigned char* __restrict__ box_need,
                              const int* __restrict__ sys_of) {
  if (flags[kFlagNeed] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (!box_rebuilds(box_need, sys_of, i)) return;
  unsorted[cell_start[atom_cell[i]] + atom_slot[i]] = i;
  if (!excl_count) return;
  const int cnt = excl_numbers[i];
  const int s = cnt > 0 ? excl_start[i] : 0;
  for (int k = 0; k < cnt; ++k) {
    const int y = excl_list[s + k];
    if (y <= i || y >= n) continue;
    const int a = atomicAdd(&excl_count[i], 1);
    if (a < kExclCap) excl_partner[i * kExclCap + a] = y;
    const int b = atomicAdd(&excl_count[y], 1);
    if (b < kExclCap) excl_partner[y * kExclCap + b] = i;
  }
}

// One warp per cell: order inside the cell by caller index (rank sort), or
// by (key, caller index) when keys are given.
__global__ void k_cell_order(int ncell, const int* __restrict__ cell_start,
                             const int* __restrict__ unsorted,
                             int* __restrict__ perm, const int* flags,
                             const int* __restrict__ key,
                             const unsigned char* __restrict__ box_need,
                             const int* __restrict__ cell_sys) {
  if (flags[kFlagNeed] == 0) return;
  int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (c >= ncell) return;
  if (!box_rebuilds(box_need, cell_sys, c)) return;
  int a = cell_start[c], b = cell_start[c + 1];
  for (int k = a + lane; k < b; k += 32) {
    int v = unsorted[k];
    int rank = 0;
    if (key) {
      const int kv = key[v];
      for (int m = a; m < b; ++m) {
        const int u = unsorted[m];
        const int ku = key[u];
        rank += ku < kv || (ku == kv && u < v);
      }
    } else {
      for (int m = a; m < b; ++m) rank += unsorted[m] < v;
    }
    perm[a + rank] = v;
  }
}

// img_off (may be null, single rectangular box): the offset that wraps the
// atom into the box at this build, floor(r / L) L per axis, which the pair
// frame subtracts until the next build.
__global__ void k_fill_sorted(int n, const int* __restrict__ perm,
                              const float3* __restrict__ crd,
                              const int* __restrict__ atom_local,
                              int* __restrict__ inv_perm, int* __restrict__ global,
                              float4* __restrict__ pos, float3* __restrict__ old_crd,
                              const int* flags, float3* __restrict__ img_off, Cell cell,
                              const unsigned char* __restrict__ box_need,
                              const int* __restrict__ sys_of) {
  if (flags[kFlagNeed] == 0) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  if (!box_rebuilds(box_need, sys_of, s)) return;
  int i = perm[s];
  inv_perm[i] = s;
  const int g = atom_local ? atom_local[i] : i;
  global[s] = g;
  float3 r = crd[i];
  pos[s] = make_float4(r.x, r.y, r.z, __int_as_float(g));  // w: global id bits
  old_crd[i] = r;
  if (img_off)
    img_off[s] = make_float3(floorf(r.x / cell.a11) * cell.a11,
                             floorf(r.y / cell.a22) * cell.a22,
                             floorf(r.z / cell.a33) * cell.a33);
}

// ---------------------------------------------------------------------------
// Is gh in the exclusion list of gl?  (Delete_Excluded_Atoms_Serial_In_
// Neighbor_List, neighbor_list.cpp:744-773, single domain.)
__device__ __forceinline__ bool excluded_pair(int gl, int gh,
                                              const int* __restrict__ excl_start,
                                              const int* __restrict__ excl_list,
                                              const int* __restrict__ excl_numbers) {
  if (!excl_numbers) return false;
  int cnt = excl_numbers[gl];
  if (cnt <= 0) return false;
  int st = excl_start[gl];
  for (int k = 0; k < cnt; ++k)
    if (excl_list[st + k] == gh) return true;
  return false;
}

// Arguments of the pair search.
struct SearchArgs {
  int n;
  const float4* pos;        // sorted (x, y, z, global id bits)
  const int* sorted_cell;
  const int* cell_start;
  const int2* runs;         // [ncell][max_runs] {first cell, last cell}
  const char4* geom;        // [ncell][max_runs] {dx, dy, dz of first, dz of last}
  const int* run_count;
  int max_runs;
  int Nx, Ny, Nz;
  Cell cell, rcell;
  float rl2;
  float rl2_lo, rl2_hi;     // rl2 (1 -+ 2e-5): outside, the fast |dr|^2 decides
  bool ortho;               // rectangular; otherwise every candidate is decided
                            // by the exact criterion on the full cell
  bool trim;                // cell offsets are unique (>= 5 cells per axis)
  float reach2;             // (rl + margin)^2 for trimming runs
  float wx, wy, iwz;        // cell widths x, y and 1/width z
  const int* excl_start;
  const int* excl_list;
  const int* excl_numbers;
  const int* excl_count;    // E(x) sizes, or null: use the lists directly
  const int* excl_partner;  // [n][kExclCap]
  int* row_count;
  int row_cap;
  int* cols;
  int* flags;
  BatchView bv;             // per-system grids when BATCH
};

// Distance, in cell widths, from a point at fractional offset f inside its
// cell to the cell at integer offset o along one axis.
__device__ __forceinline__ float cell_gap(int o, float f) {
  const float g = o > 0 ? (float)o - f : (o < 0 ? f - (float)(o + 1) : 0.f);
  return fmaxf(g, 0.f);
}

// Pair search for sorted atom i (one warp), one pass: row i has room for
// row_cap entries at cols[i * row_cap]; hits beyond it are counted (the
// largest row is kept in flags[kFlagMaxRow]) and raise the overflow flag so
// the host can regrow the rows and repeat the build.
//
// Each run is cut down to the cells whose box is within rl (plus a margin)
// of atom i.  With at least 5 cells per axis a pair within rl sits at the
// run's cell offset in its minimum image, so a cut cell holds no hit.
constexpr int kSearchChunk = 32;

template <bool BATCH>
__global__ void __launch_bounds__(256)
k_pair_search(SearchArgs a) {
  if (a.flags[kFlagNeed] == 0) return;
  const int lane = threadIdx.x & 31;
  const int nw = blockDim.x >> 5;
  // One box: a contiguous range of sorted atoms per block (shared neighbour
  // cells in L1).  Batch: chunks of kSearchChunk sorted atoms dealt to the
  // blocks in turn, so that the few boxes of a partial rebuild spread over
  // every SM.  i grows with t, so the first i past the end ends the loop.
  const int per_block = BATCH ? kSearchChunk : (a.n + gridDim.x - 1) / gridDim.x;
  const int stride = BATCH ? (int)gridDim.x * kSearchChunk : 0;
  for (int t = threadIdx.x >> 5;; t += nw) {
  const int q = t / per_block, r = t - q * per_block;
  if (!BATCH && q > 0) break;
  const int i = (int)blockIdx.x * per_block + q * stride + r;
  if (i >= a.n) break;
  if (BATCH && !box_rebuilds(a.bv.box_need, a.bv.sys_of, i)) continue;  // warp-uniform
  const float4 pi4 = a.pos[i];
  const int gi = __float_as_int(pi4.w);
  const int c = a.sorted_cell[i];
  // grid of atom i's box
  int Nx = a.Nx, Ny = a.Ny, Nz = a.Nz, c_local = c;
  Cell cell = a.cell, rcell = a.rcell;
  bool trim = a.trim;
  float wx = a.wx, wy = a.wy, iwz = a.iwz;
  if (BATCH) {
    const SysGeom& g = a.bv.sys[a.bv.sys_of[i]];
    Nx = g.Nx;
    Ny = g.Ny;
    Nz = g.Nz;
    c_local = c - g.cell_begin;
    cell = g.cell;
    rcell = g.rcell;
    trim = g.trim != 0;
    wx = g.wx;
    wy = g.wy;
    iwz = g.iwz;
  }
  int* out_row = a.cols + (size_t)i * a.row_cap;
  int count = 0;
  const int nr = a.run_count[c];
  // excluded partners of gi held one per lane (warp-uniform count)
  int n_ex = 0, ex = -1;
  bool ex_lists = a.excl_numbers != nullptr;
  if (a.excl_count) {
    n_ex = a.excl_count[gi];
    if (n_ex <= kExclCap) {
      ex_lists = false;
      if (lane < n_ex) ex = a.excl_partner[gi * kExclCap + lane];
    } else {
      n_ex = 0;
    }
  }
  // the first two partners in every lane (a water atom has two)
  const int ex0 = __shfl_sync(0xffffffffu, ex, 0), ex1 = __shfl_sync(0xffffffffu, ex, 1);
  // position of i inside its cell, in cell widths (the binning's arithmetic)
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (trim) {
    const int cz = c_local % Nz, cy = (c_local / Nz) % Ny, cx = c_local / (Nz * Ny);
    const float x = pi4.x - floorf(pi4.x / cell.a11) * cell.a11;
    const float y = pi4.y - floorf(pi4.y / cell.a22) * cell.a22;
    const float z = pi4.z - floorf(pi4.z / cell.a33) * cell.a33;
    fx = x / cell.a11 * Nx - (float)cx;
    fy = y / cell.a22 * Ny - (float)cy;
    fz = z / cell.a33 * Nz - (float)cz;
  }
  // Range list: the own cell after i, then the owned runs, 32 ranges at a
  // time.  Lane r works out range r0 + r (its trimmed slice of the sorted
  // array); a prefix sum over the lanes lays the slices end to end, and the
  // candidates are taken 32 at a time across slice boundaries.
  const unsigned lt = (1u << lane) - 1u;
  for (int r0 = -1; r0 < nr; r0 += 32) {
    const int r = r0 + lane;
    int lo = 0, len = 0;
    if (r < 0) {
      lo = i + 1;
      len = a.cell_start[c + 1] - lo;
    } else if (r < nr) {
      int2 rr = a.runs[(size_t)c * a.max_runs + r];
      bool keep = true;
      if (trim) {
        const char4 g = a.geom[(size_t)c * a.max_runs + r];
        const float gx = cell_gap(g.x, fx) * wx, gy = cell_gap(g.y, fy) * wy;
        const float s2 = a.reach2 - gx * gx - gy * gy;
        keep = s2 >= 0.f;
        if (keep) {
          const float s = sqrtf(s2) * iwz;
          const int zmax = (int)floorf(fz + s), zmin = (int)ceilf(fz - 1.f - s);
          const int z0 = max((int)g.z, zmin), z1 = min((int)g.w, zmax);
          keep = z0 <= z1;
          rr.x += z0 - g.z;
          rr.y -= g.w - z1;
        }
      }
      if (keep) {
        lo = a.cell_start[rr.x];
        len = a.cell_start[rr.y + 1] - lo;
      }
    }
    int incl = len;  // inclusive prefix of the slice lengths
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - len;
    const int nq = min(32, nr - r0);  // ranges in this chunk
    int cursor = 0;                   // first slice not yet used up
    for (int base = 0; base < total; base += 32) {
      // candidate of flat index base + lane: its slice among those that meet
      // [base, base + 32)
      const int fi = base + lane;
      int j = -1;
      for (int q = cursor; q < nq; ++q) {  // warp-uniform
        const int eq = __shfl_sync(0xffffffffu, excl, q);
        const int lq = __shfl_sync(0xffffffffu, len, q);
        const int oq = __shfl_sync(0xffffffffu, lo, q);
        if (eq >= base + 32) break;
        if (fi >= eq && fi < eq + lq) j = oq + (fi - eq);
        if (eq + lq > base + 32) break;  // goes on into the next batch
        cursor = q + 1;
      }
      bool hit = false;
      int gj = -1;
      bool unsure = false;
      float4 pj4 = make_float4(0.f, 0.f, 0.f, 0.f);
      if (j >= 0) {
        pj4 = a.pos[j];
        gj = __float_as_int(pj4.w);
        if (a.ortho) {
          // fast |dr|^2 (contracted, FMA-pipe min image) first: it differs
          // from the exact one by far less than the band, so outside the
          // band it decides the criterion alone
          const float ex_ = min_image_axis(pj4.x - pi4.x, cell.a11, rcell.a11);
          const float ey_ = min_image_axis(pj4.y - pi4.y, cell.a22, rcell.a22);
          const float ez_ = min_image_axis(pj4.z - pi4.z, cell.a33, rcell.a33);
          const float r2f = ex_ * ex_ + ey_ * ey_ + ez_ * ez_;
          hit = r2f < a.rl2_lo;
          unsure = !hit && r2f <= a.rl2_hi;
        } else {
          // a skewed cell: the image choice of a rounded fractional
          // displacement can differ between two roundings, so no fast path
          unsure = true;
        }
      }
      if (__any_sync(0xffffffffu, unsure) && unsure) {
        // the exact criterion, dr = crd[lower id] - crd[higher id] as the
        // reference forms it, no contraction
        if (a.ortho) {
          float dx = __fsub_rn(pi4.x, pj4.x);
          float dy = __fsub_rn(pi4.y, pj4.y);
          float dz = __fsub_rn(pi4.z, pj4.z);
          if (gj < gi) {
            dx = -dx;
            dy = -dy;
            dz = -dz;
          }
          const float3 d = min_image_exact_rect(dx, dy, dz, cell, rcell);
          hit = norm2_exact(d) < a.rl2;
        } else {
          const float3 ri = make_float3(pi4.x, pi4.y, pi4.z);
          const float3 rj = make_float3(pj4.x, pj4.y, pj4.z);
          const float3 d = gi < gj ? min_image_exact(ri, rj, cell, rcell)
                                   : min_image_exact(rj, ri, cell, rcell);
          hit = norm2_exact(d) < a.rl2;
        }
      }
      if (n_ex > 0 && (gj == ex0 || gj == ex1)) hit = false;
      for (int k = 2; k < n_ex; ++k)  // warp-uniform
        if (__shfl_sync(0xffffffffu, ex, k) == gj) hit = false;
      if (hit && ex_lists)
        hit = !excluded_pair(min(gi, gj), max(gi, gj), a.excl_start, a.excl_list,
                             a.excl_numbers);
      const unsigned m = __ballot_sync(0xffffffffu, hit);
      if (hit) {
        const int slot = count + __popc(m & lt);
        if (slot < a.row_cap) out_row[slot] = j;
      }
      count += __popc(m);
    }
  }
  if (lane == 0) {
    // a partial batch rebuild replaces this row's share of the kept total
    const int prev = (BATCH && a.flags[kFlagFull] == 0) ? a.row_count[i] : 0;
    a.row_count[i] = count < a.row_cap ? count : a.row_cap;
    atomicAdd(&a.flags[kFlagTotal], count - prev);
    if (count > a.row_cap) {
      a.flags[kFlagListOverflow] = 1;
      atomicMax(&a.flags[kFlagMaxRow], count);
    }
  }
  }
}

// ---------------------------------------------------------------------------
// Cluster form.  Clusters of a cell: ceil(count / kClusterSize).
__global__ void k_clus_count(int ncell, const int* __restrict__ cell_start,
                             int* __restrict__ clus_count, const int* flags) {
  if (flags[kFlagNeed] == 0) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncell) return;
  clus_count[k] = (cell_start[k + 1] - cell_start[k] + kClusterSize - 1) / kClusterSize;
}

// One thread per cell: its clusters' atom ranges and bounding boxes (in the
// wrapped frame the binning used).
__global__ void k_clus_fill(int ncell, const int* __restrict__ cell_start,
                            const int* __restrict__ cell_clus,
                            const float4* __restrict__ pos, Cell cell,
                            int2* __restrict__ clus, float4* __restrict__ lo,
                            float4* __restrict__ hi, const int* flags) {
  if (flags[kFlagNeed] == 0) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ncell) return;
  const int a = cell_start[k], b = cell_start[k + 1];
  int cc = cell_clus[k];
  for (int s = a; s < b; s += kClusterSize, ++cc) {
    const int m = min(kClusterSize, b - s);
    float3 l = make_float3(FLT_MAX, FLT_MAX, FLT_MAX);
    float3 h = make_float3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (int t = 0; t < m; ++t) {
      const float4 p = pos[s + t];
      const float x = p.x - floorf(p.x / cell.a11) * cell.a11;
      const float y = p.y - floorf(p.y / cell.a22) * cell.a22;
      const float z = p.z - floorf(p.z / cell.a33) * cell.a33;
      l = make_float3(fminf(l.x, x), fminf(l.y, y), fminf(l.z, z));
      h = make_float3(fmaxf(h.x, x), fmaxf(h.y, y), fmaxf(h.z, z));
    }
    clus[cc] = make_int2(s, m);
    lo[cc] = make_float4(l.x, l.y, l.z, 0.f);
    hi[cc] = make_float4(h.x, h.y, h.z, 0.f);
  }
}

struct ClusterSearchArgs {
  const float4* pos;          // sorted build-time coordinates (x,y,z, global id bits)
  const int* sorted_cell;
  const int* cell_clus;
  const int2* clus;
  const float4* clus_lo;
  const float4* clus_hi;
  const int* nclus;
  const int2* runs;
  const char4* geom;
  const int* run_count;
  int max_runs;
  int Nx, Ny, Nz;
  Cell cell, rcell;
  float rl2, rl2_lo, rl2_hi;
  float reach2;               // (rl + margin)^2 for the box and run tests
  float wx, wy, wz;           // cell widths
  const int* excl_start;
  const int* excl_list;
  const int* excl_numbers;
  const int* excl_count;      // E(x) sizes, or null
  const int* excl_partner;
  int* crow_count;
  int ccap;
  int2* centry;
  int* flags;
};

// Distance, in cell widths, from the span [lo, hi] (fractions of the own
// cell) to the cell at integer offset o along one axis.
__device__ __forceinline__ float span_gap(int o, float lo, float hi) {
  const float g = o > 0 ? (float)o - hi : (o < 0 ? lo - (float)(o + 1) : 0.f);
  return fmaxf(g, 0.f);
}

// Gap between two boxes along an axis (centre distance minus half widths).
__device__ __forceinline__ float box_gap(float lo_a, float hi_a, float lo_b, float hi_b,
                                         float shift) {
  const float d = fabsf(0.5f * (lo_b + hi_b) + shift - 0.5f * (lo_a + hi_a));
  return fmaxf(d - 0.5f * (hi_a - lo_a) - 0.5f * (hi_b - lo_b), 0.f);
}

// One warp per i-cluster.  The candidates are the clusters of the own cell
// from this one on and those of the owned runs, each run cut to the cells
// within reach of the cluster's box; a candidate whose box (in the run's
// periodic image) is within reach has its pairs tested with the reference's
// exact criterion, eight candidates at a time (lane = 4 k + j: candidate k,
// its atom j against the four i atoms every lane holds), and is listed when
// any pair passes.  Exclusions and, inside one cluster, the order j > i are
// applied in the mask.  The box tests only drop clusters that hold no pair
// within r_l: box gaps bound the distances of the atoms inside from below,
// with a 0.01 A margin over the rounding.
__global__ void __launch_bounds__(256, 2) k_cluster_search(ClusterSearchArgs a) {
  if (a.flags[kFlagNeed] == 0) return;
  __shared__ int4 pass_all[8][32];  // {cluster, shift code, first atom, atoms}
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int nclus = *a.nclus;
  const int per_block = (nclus + gridDim.x - 1) / gridDim.x;
  const int c_end = min(nclus, (int)blockIdx.x * per_block + per_block);
  const float Lx = a.cell.a11, Ly = a.cell.a22, Lz = a.cell.a33;
  for (int c = blockIdx.x * per_block + w; c < c_end; c += nw) {
    const int2 ci = a.clus[c];
    const int cell = a.sorted_cell[ci.x];
    const int cz = cell % a.Nz, cy = (cell / a.Nz) % a.Ny, cx = cell / (a.Nz * a.Ny);
    const float4 blo = a.clus_lo[c], bhi = a.clus_hi[c];
    const float flx = blo.x / a.wx - (float)cx, fhx = bhi.x / a.wx - (float)cx;
    const float fly = blo.y / a.wy - (float)cy, fhy = bhi.y / a.wy - (float)cy;
    const float flz = blo.z / a.wz - (float)cz, fhz = bhi.z / a.wz - (float)cz;
    // the i atoms and their first two excluded partners, in every lane
    float4 p_i[kClusterSize];
    int g_i[kClusterSize], nex_i[kClusterSize], ex0_i[kClusterSize], ex1_i[kClusterSize];
    bool lists_i[kClusterSize];
    {
      const bool own = lane < ci.y;
      const float4 pl = a.pos[ci.x + (own ? lane : 0)];
      const int gl = __float_as_int(pl.w);
      int nl_ = 0, e0 = -1, e1 = -1;
      bool li = a.excl_numbers != nullptr;
      if (own && a.excl_count) {
        nl_ = a.excl_count[gl];
        if (nl_ <= kExclCap) {
          li = false;
          if (nl_ > 0) e0 = a.excl_partner[gl * kExclCap];
          if (nl_ > 1) e1 = a.excl_partner[gl * kExclCap + 1];
        } else {
          nl_ = 0;
        }
      }
#pragma unroll
      for (int ii = 0; ii < kClusterSize; ++ii) {
        p_i[ii] = make_float4(__shfl_sync(0xffffffffu, pl.x, ii),
                              __shfl_sync(0xffffffffu, pl.y, ii),
                              __shfl_sync(0xffffffffu, pl.z, ii), 0.f);
        g_i[ii] = __shfl_sync(0xffffffffu, gl, ii);
        nex_i[ii] = __shfl_sync(0xffffffffu, nl_, ii);
        ex0_i[ii] = __shfl_sync(0xffffffffu, e0, ii);
        ex1_i[ii] = __shfl_sync(0xffffffffu, e1, ii);
        lists_i[ii] = __shfl_sync(0xffffffffu, (int)li, ii) != 0;
      }
    }
    int count = 0, pairs = 0;
    int2* out = a.centry + (size_t)c * a.ccap;
    const int nr = a.run_count[cell];
    for (int r0 = -1; r0 < nr; r0 += 32) {
      const int r = r0 + lane;
      int lo = 0, len = 0, code = 13;
      if (r < 0) {
        lo = c;
        len = a.cell_clus[cell + 1] - c;
      } else if (r < nr) {
        const int2 rr = a.runs[(size_t)cell * a.max_runs + r];
        const char4 g = a.geom[(size_t)cell * a.max_runs + r];
        const float gx = span_gap(g.x, flx, fhx) * a.wx;
        const float gy = span_gap(g.y, fly, fhy) * a.wy;
        const float s2 = a.reach2 - gx * gx - gy * gy;
        if (s2 >= 0.f) {
          const float sz = sqrtf(s2) / a.wz;
          const int zmax = (int)floorf(fhz + sz), zmin = (int)ceilf(flz - 1.f - sz);
          const int z0 = max((int)g.z, zmin), z1 = min((int)g.w, zmax);
          if (z0 <= z1) {
            const int f = rr.x + (z0 - g.z), l = rr.y - (g.w - z1);
            lo = a.cell_clus[f];
            len = a.cell_clus[l + 1] - lo;
            // periodic image of the run's cells relative to the own cell
            const int ux = cx + g.x, uy = cy + g.y, uz = cz + g.z;
            const int sx = ux < 0 ? -1 : (ux >= a.Nx ? 1 : 0);
            const int sy = uy < 0 ? -1 : (uy >= a.Ny ? 1 : 0);
            const int szz = uz < 0 ? -1 : (uz >= a.Nz ? 1 : 0);
            code = (sx + 1) * 9 + (sy + 1) * 3 + (szz + 1);
          }
        }
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      const int excl = incl - len;
      const int nq = min(32, nr - r0);
      int cursor = 0;
      for (int base = 0; base < total; base += 32) {
        const int fi = base + lane;
        int jc = -1, jcode = 13;
        for (int q = cursor; q < nq; ++q) {  // warp-uniform
          const int eq = __shfl_sync(0xffffffffu, excl, q);
          const int lq = __shfl_sync(0xffffffffu, len, q);
          const int oq = __shfl_sync(0xffffffffu, lo, q);
          const int cq = __shfl_sync(0xffffffffu, code, q);
          if (eq >= base + 32) break;
          if (fi >= eq && fi < eq + lq) {
            jc = oq + (fi - eq);
            jcode = cq;
          }
          if (eq + lq > base + 32) break;
          cursor = q + 1;
        }
        bool pass = false;
        int2 cj = make_int2(0, 0);
        if (jc >= 0) {
          const float4 jl = a.clus_lo[jc], jh = a.clus_hi[jc];
          cj = a.clus[jc];
          const float shx = (float)(jcode / 9 - 1) * Lx;
          const float shy = (float)((jcode / 3) % 3 - 1) * Ly;
          const float shz = (float)(jcode % 3 - 1) * Lz;
          const float gx = box_gap(blo.x, bhi.x, jl.x, jh.x, shx);
          const float gy = box_gap(blo.y, bhi.y, jl.y, jh.y, shy);
          const float gz = box_gap(blo.z, bhi.z, jl.z, jh.z, shz);
          pass = gx * gx + gy * gy + gz * gz < a.reach2;
        }
        const unsigned pm = __ballot_sync(0xffffffffu, pass);
        if (pass) pass_all[w][__popc(pm & lt)] = make_int4(jc, jcode, cj.x, cj.y);
        __syncwarp();
        const int np = __popc(pm);
        const int kk = lane >> 2, jj = lane & 3;
        for (int k0 = 0; k0 < np; k0 += 8) {
          const bool have = k0 + kk < np;
          const int4 pj = pass_all[w][have ? k0 + kk : k0];
          const bool j_ok = have && jj < pj.w;
          const float4 pj4 = j_ok ? a.pos[pj.z + jj] : make_float4(0.f, 0.f, 0.f, 0.f);
          const int gj = __float_as_int(pj4.w);
          unsigned mask = 0;  // bits 4 ii + jj of this lane's candidate
#pragma unroll
          for (int ii = 0; ii < kClusterSize; ++ii) {
            bool hit = false, unsure = false;
            if (j_ok && ii < ci.y && (pj.x != c || jj > ii)) {
              const float ex_ = min_image_axis(pj4.x - p_i[ii].x, a.cell.a11, a.rcell.a11);
              const float ey_ = min_image_axis(pj4.y - p_i[ii].y, a.cell.a22, a.rcell.a22);
              const float ez_ = min_image_axis(pj4.z - p_i[ii].z, a.cell.a33, a.rcell.a33);
              const float r2f = ex_ * ex_ + ey_ * ey_ + ez_ * ez_;
              hit = r2f < a.rl2_lo;
              unsure = !hit && r2f <= a.rl2_hi;
            }
            if (__any_sync(0xffffffffu, unsure) && unsure) {
              // the band: the exact criterion, dr = crd[lower id] - crd[higher id]
              float dx = __fsub_rn(p_i[ii].x, pj4.x);
              float dy = __fsub_rn(p_i[ii].y, pj4.y);
              float dz = __fsub_rn(p_i[ii].z, pj4.z);
              if (gj < g_i[ii]) {
                dx = -dx;
                dy = -dy;
                dz = -dz;
              }
              const float3 d = min_image_exact_rect(dx, dy, dz, a.cell, a.rcell);
              hit = norm2_exact(d) < a.rl2;
            }
            if (hit && nex_i[ii] > 0) {
              if (gj == ex0_i[ii] || gj == ex1_i[ii]) hit = false;
              for (int q = 2; q < nex_i[ii] && hit; ++q)
                if (a.excl_partner[g_i[ii] * kExclCap + q] == gj) hit = false;
            }
            if (hit && lists_i[ii])
              hit = !excluded_pair(min(g_i[ii], gj), max(g_i[ii], gj), a.excl_start,
                                   a.excl_list, a.excl_numbers);
            mask |= hit ? 1u << (4 * ii + jj) : 0u;
          }
          // the candidate's mask: OR over its four lanes
          mask |= __shfl_xor_sync(0xffffffffu, mask, 1);
          mask |= __shfl_xor_sync(0xffffffffu, mask, 2);
          const bool lead = jj == 0 && mask != 0u;
          const unsigned lm = __ballot_sync(0xffffffffu, lead);
          if (lead) {
            const int slot = count + __popc(lm & lt);
            if (slot < a.ccap)
              out[slot] = make_int2(pj.z, (int)(mask | ((unsigned)pj.y << 16)));
          }
          count += __popc(lm);
          pairs += __popc(mask) * (jj == 0);
        }
        __syncwarp();
      }
    }
    pairs = __reduce_add_sync(0xffffffffu, pairs);
    if (lane == 0) {
      a.crow_count[c] = count < a.ccap ? count : a.ccap;
      atomicAdd(&a.flags[kFlagTotal], pairs);
      if (count > a.ccap) {
        a.flags[kFlagListOverflow] = 1;
        atomicMax(&a.flags[kFlagMaxRow], count);
      }
    }
  }
}

// batch: a rebuild of only some systems keeps the total of the others
__global__ void k_rebuild_begin(int* flags, bool batch) {
  if (flags[kFlagNeed] == 0) return;
  if (!batch || flags[kFlagFull] != 0) flags[kFlagTotal] = 0;
  flags[kFlagMaxRow] = 0;
}

__global__ void k_row_starts(int n, int row_cap, int* row_start) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= n) row_start[i] = i * row_cap;
}

__global__ void k_sorted_cell(int n, const int* __restrict__ perm,
                              const int* __restrict__ atom_cell, int* __restrict__ sc,
                              const int* flags, const unsigned char* __restrict__ box_need,
                              const int* __restrict__ sys_of) {
  if (flags[kFlagNeed] == 0) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < n && box_rebuilds(box_need, sys_of, s)) sc[s] = atom_cell[perm[s]];
}

// Zeroes the cell counts of the systems that rebuild (all cells for one
// box): the others keep the counts of their last build, so the scan gives
// their cells the same starts again.
__global__ void k_zero_cells(int ncell, int* __restrict__ cell_count, const int* flags,
                             const unsigned char* __restrict__ box_need,
                             const int* __restrict__ cell_sys) {
  if (flags[kFlagNeed] == 0) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncell && box_rebuilds(box_need, cell_sys, c)) cell_count[c] = 0;
}

__global__ void k_finish_build(int* flags) {
  if (flags[kFlagNeed] != 0) flags[kFlagGeneration] += 1;
  flags[kFlagNeed] = 0;
  flags[kFlagFull] = 0;
}

// Reads the rebuild flag into the graph's conditional handle (the IF node
// that holds the rebuild kernels).
// prune (may be null): the pruned rows' flags of an engine, decided here in
// the same launch: the step prunes when it rebuilds or when an atom moved
// past half the prune margin ({pass, moved, generation after this step,
// passes}).
__global__ void k_set_rebuild_condition(cudaGraphConditionalHandle h, const int* flags,
                                        int* prune) {
  const int need = flags[kFlagNeed] != 0 ? 1 : 0;
  cudaGraphSetConditional(h, need ? 1u : 0u);
  if (prune) {
    const int pass = (prune[1] != 0 || need) ? 1 : 0;
    prune[0] = pass;
    prune[1] = 0;
    prune[2] = flags[kFlagGeneration] + need;  // the rebuild adds one
    prune[3] += pass;
  }
}

int nl_set_condition(NeighborList& nl, cudaGraphConditionalHandle h, cudaStream_t st,
                     int* prune) {
  k_set_rebuild_condition<<<1, 1, 0, st>>>(h, nl.d_flags, prune);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int nl_check_moved(NeighborList& nl, const float* crd_f, cudaStream_t st) {
  const float permit = nl.skin * nl.skin_permit;
  if (nl.bv.nsys > 0)
    k_check_refresh<true><<<ceil_div(nl.n, 256), 256, 0, st>>>(
        nl.n, reinterpret_cast<const float3*>(crd_f), nl.d_old_crd, nl.cell, nl.rcell,
        permit * permit, nl.d_flags, nl.bv);
  else
    k_check_refresh<false><<<ceil_div(nl.n, 256), 256, 0, st>>>(
        nl.n, reinterpret_cast<const float3*>(crd_f), nl.d_old_crd, nl.cell, nl.rcell,
        permit * permit, nl.d_flags, nl.bv);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// The next rebuild covers every system.
static void nl_need_all(NeighborList& nl, cudaStream_t st) {
  const int nsys = (nl.bv.nsys > 0 && nl.bv.box_need) ? nl.bv.nsys : 0;
  k_set_need_all<<<std::max(1, std::min(ceil_div(nsys, 256), 64)), 256, 0, st>>>(
      nl.d_flags, nl.bv.box_need, nsys);
}

int nl_force_next(NeighborList& nl, cudaStream_t st) {
  nl_need_all(nl, st);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
// Owned neighbour runs of every cell of one Nx x Ny x Nz box whose cells are
// numbered from `offset` in the list's cell space; appended to per/per_geom.
static void box_runs(int Nx, int Ny, int Nz, int offset,
                     std::vector<std::vector<int2>>& per,
                     std::vector<std::vector<char4>>& per_geom) {
  for (int cx = 0; cx < Nx; ++cx)
    for (int cy = 0; cy < Ny; ++cy)
      for (int cz = 0; cz < Nz; ++cz) {
        int c = (cx * Ny + cy) * Nz + cz;
        // Which cell of a neighbouring pair searches the pair.  With at least
        // 5 cells per axis every neighbour has one offset (dx, dy, dz) in
        // [-2, 2]^3 and the pair belongs to the cell that sees the other at
        // a lexicographically positive offset: every cell owns 62 of its 124
        // neighbours, so rows have about the same length everywhere.  With
        // fewer cells an offset can alias (+2 and -2 meet), and the pair
        // belongs to the cell with the smaller index.
        const bool offset_rule = Nx >= 5 && Ny >= 5 && Nz >= 5;
        std::map<int, char4> nb;  // owned cell -> its offset
        for (int dx = -2; dx <= 2; ++dx)
          for (int dy = -2; dy <= 2; ++dy)
            for (int dz = -2; dz <= 2; ++dz) {
              int x = ((cx + dx) % Nx + Nx) % Nx;
              int y = ((cy + dy) % Ny + Ny) % Ny;
              int z = ((cz + dz) % Nz + Nz) % Nz;
              int o = (x * Ny + y) * Nz + z;
              bool own = offset_rule
                             ? (dx > 0 || (dx == 0 && (dy > 0 || (dy == 0 && dz > 0))))
                             : o > c;
              if (own && o != c && !nb.count(o))
                nb[o] = make_char4((signed char)dx, (signed char)dy, (signed char)dz,
                                   (signed char)dz);
            }
        // runs: consecutive cells of one z column (dz then rises by one)
        std::vector<int2> rr;
        std::vector<char4> gg;
        for (const auto& kv : nb) {
          const int o = kv.first;
          if (!rr.empty() && rr.back().y == offset + o - 1 && (o - 1) / Nz == o / Nz &&
              gg.back().w + 1 == kv.second.z) {
            rr.back().y = offset + o;
            gg.back().w = kv.second.z;
          } else {
            rr.push_back(make_int2(offset + o, offset + o));
            gg.push_back(kv.second);
          }
        }
        per[offset + c] = rr;
        per_geom[offset + c] = gg;
      }
}

// Neighbour cells of every cell of a box with a general lower-triangular
// cell (a = (a11,0,0), b = (a21,a22,0), c = (a31,a32,a33)), cells of the
// brick [0,a11) x [0,a22) x [0,a33) of side a_ii / N.  A pair within r_l
// has j's wrapped position at i's plus a displacement of length below r_l
// less a lattice vector; for every lattice vector that can occur the cells
// that i's cell plus the displacement box reach are taken (with 0.01 A over
// r_l for the rounding of the wrap), the same cell once.  Ownership as for
// small rectangular boxes: the cell with the smaller index scans the pair,
// the own cell holds its later atoms.  Runs are cut along z as in box_runs;
// the offsets are not used (no trimming for skewed cells).
static void skewed_runs(int Nx, int Ny, int Nz, const Cell& cl, float rl,
                        std::vector<std::vector<int2>>& per,
                        std::vector<std::vector<char4>>& per_geom) {
  const double a11 = cl.a11, a21 = cl.a21, a22 = cl.a22, a31 = cl.a31, a32 = cl.a32,
               a33 = cl.a33;
  const double wx = a11 / Nx, wy = a22 / Ny, wz = a33 / Nz;
  const double reach = (double)rl + 0.01;
  // lattice-vector counts that keep both wrapped points inside the brick
  const int nc_max = (int)std::ceil(1.0 + reach / a33);
  const int nb_max = (int)std::ceil(1.0 + (reach + std::fabs(a32) * nc_max) / a22);
  const int na_max = (int)std::ceil(
      1.0 + (reach + std::fabs(a21) * nb_max + std::fabs(a31) * nc_max) / a11);
  auto range = [](double lo, double hi, double w, int N, int* k0, int* k1) {
    *k0 = std::max(0, (int)std::floor(lo / w));
    *k1 = std::min(N - 1, (int)std::floor(hi / w));
    return *k0 <= *k1;
  };
  for (int cx = 0; cx < Nx; ++cx)
    for (int cy = 0; cy < Ny; ++cy)
      for (int cz = 0; cz < Nz; ++cz) {
        const int c = (cx * Ny + cy) * Nz + cz;
        std::map<int, char4> nb;
        for (int nc = -nc_max; nc <= nc_max; ++nc)
          for (int nbv = -nb_max; nbv <= nb_max; ++nbv)
            for (int na = -na_max; na <= na_max; ++na) {
              const double tx = na * a11 + nbv * a21 + nc * a31;
              const double ty = nbv * a22 + nc * a32;
              const double tz = nc * a33;
              int x0, x1, y0, y1, z0, z1;
              if (!range(cx * wx - reach - tx, (cx + 1) * wx + reach - tx, wx, Nx, &x0, &x1) ||
                  !range(cy * wy - reach - ty, (cy + 1) * wy + reach - ty, wy, Ny, &y0, &y1) ||
                  !range(cz * wz - reach - tz, (cz + 1) * wz + reach - tz, wz, Nz, &z0, &z1))
                continue;
              for (int x = x0; x <= x1; ++x)
                for (int y = y0; y <= y1; ++y)
                  for (int z = z0; z <= z1; ++z) {
                    const int o = (x * Ny + y) * Nz + z;
                    if (o > c) nb[o] = make_char4(0, 0, 0, 0);
                  }
            }
        std::vector<int2> rr;
        for (const auto& kv : nb) {
          const int o = kv.first;
          if (!rr.empty() && rr.back().y == o - 1 && (o - 1) / Nz == o / Nz)
            rr.back().y = o;
          else
            rr.push_back(make_int2(o, o));
        }
        per[c] = rr;
        per_geom[c].assign(rr.size(), make_char4(0, 0, 0, 0));
      }
}

// Inverse of a lower-triangular cell in Invert_Lower_Triangular_Cell's
// operation order (utils/boundary.h:61-72): the pair criterion reads it.
static Cell lower_rcell(const Cell& c) {
  Cell r{};
  r.a11 = 1.0f / c.a11;
  r.a22 = 1.0f / c.a22;
  r.a33 = 1.0f / c.a33;
  r.a21 = -c.a21 / (c.a11 * c.a22);
  r.a31 = (c.a21 * c.a32 - c.a22 * c.a31) / (c.a11 * c.a22 * c.a33);
  r.a32 = -c.a32 / (c.a22 * c.a33);
  return r;
}

// Per-cell run lists as fixed-width tables [ncell][max_runs].
static void pack_runs(const std::vector<std::vector<int2>>& per,
                      const std::vector<std::vector<char4>>& per_geom,
                      std::vector<int2>& runs, std::vector<char4>& geom,
                      std::vector<int>& counts, int& max_runs) {
  const int ncell = (int)per.size();
  max_runs = 1;
  for (const auto& r : per) max_runs = std::max(max_runs, (int)r.size());
  runs.assign((size_t)ncell * max_runs, make_int2(0, -1));
  geom.assign((size_t)ncell * max_runs, make_char4(0, 0, 0, -1));
  counts.assign(ncell, 0);
  for (int c = 0; c < ncell; ++c) {
    counts[c] = (int)per[c].size();
    for (size_t k = 0; k < per[c].size(); ++k) {
      runs[(size_t)c * max_runs + k] = per[c][k];
      geom[(size_t)c * max_runs + k] = per_geom[c][k];
    }
  }
}

// The reference's grid for one rectangular box (NEIGHBOR_LIST::Initial,
// neighbor_list.cpp:943-960): N = floor(L / ((cutoff + skin) / 2)) per axis.
static int box_grid(float grid_length, const Cell& cell, int* N) {
  N[0] = (int)floorf(cell.a11 / grid_length);
  N[1] = (int)floorf(cell.a22 / grid_length);
  N[2] = (int)floorf(cell.a33 / grid_length);
  if (N[0] <= 2 || N[1] <= 2 || N[2] <= 2)
    return fail(kBadInput, "NEIGHBOR_LIST::Initial: the box is too small.");
  return kOk;
}

static Cell rect_rcell(const Cell& c) {
  Cell r{};
  r.a11 = 1.0f / c.a11;
  r.a22 = 1.0f / c.a22;
  r.a33 = 1.0f / c.a33;
  return r;
}

static int nl_alloc(NeighborList& nl, int n, long long initial_capacity,
                    const std::vector<int2>& runs, const std::vector<char4>& geom,
                    const std::vector<int>& counts, double max_per_atom,
                    bool all_balanced);

static void nl_common(NeighborList& nl, int n, float cutoff, float skin,
                      int refresh_interval, float skin_permit, int max_neighbor_numbers) {
  nl.n = n;
  nl.cutoff = cutoff;
  nl.skin = skin;
  nl.grid_length = 0.5f * (cutoff + skin);
  nl.rl2 = nl.grid_length * nl.grid_length * 4.0f;
  nl.refresh_interval = refresh_interval;
  nl.skin_permit = skin_permit;
  nl.max_neighbor_numbers = max_neighbor_numbers;
  // margin of 0.01 A over rl for trimming runs: far above the float error
  // of the cell geometry (positions are wrapped with one rounding each)
  const double reach = sqrt((double)nl.rl2) + 0.01;
  nl.reach2 = (float)(reach * reach);
}

// Mean number of half-list entries per atom at density rho.
static double half_sphere(double rho, float rl2) {
  const double rl = sqrt((double)rl2);
  return 0.5 * rho * 4.18879020478639 * rl * rl * rl;
}

int nl_init(NeighborList& nl, int n, float cutoff, float skin, const float* cell6,
            int refresh_interval, float skin_permit, int max_neighbor_numbers,
            long long initial_capacity) {
  if (n <= 0) return fail(kBadInput, "neighbor list: atom_numbers must be > 0");
  nl_common(nl, n, cutoff, skin, refresh_interval, skin_permit, max_neighbor_numbers);
  nl.cell = make_cell(cell6);
  nl.ortho = cell6[1] == 0.f && cell6[3] == 0.f && cell6[4] == 0.f;
  nl.rcell = nl.ortho ? rect_rcell(nl.cell) : lower_rcell(nl.cell);
  if (!(nl.cell.a11 > 0.f && nl.cell.a22 > 0.f && nl.cell.a33 > 0.f))
    return fail(kBadInput, "neighbor list: the cell's diagonal must be positive");
  int N[3];
  int rc = box_grid(nl.grid_length, nl.cell, N);
  if (rc) return rc;
  nl.Nx = N[0];
  nl.Ny = N[1];
  nl.Nz = N[2];
  nl.ncell = nl.Nx * nl.Ny * nl.Nz;
  nl.trim = nl.ortho && nl.Nx >= 5 && nl.Ny >= 5 && nl.Nz >= 5;
  nl.wx = nl.cell.a11 / nl.Nx;
  nl.wy = nl.cell.a22 / nl.Ny;
  nl.iwz = nl.Nz / nl.cell.a33;
  std::vector<std::vector<int2>> per(nl.ncell);
  std::vector<std::vector<char4>> per_geom(nl.ncell);
  if (nl.ortho)
    box_runs(nl.Nx, nl.Ny, nl.Nz, 0, per, per_geom);
  else
    skewed_runs(nl.Nx, nl.Ny, nl.Nz, nl.cell, sqrtf(nl.rl2), per, per_geom);
  std::vector<int2> runs;
  std::vector<char4> geom;
  std::vector<int> counts;
  pack_runs(per, per_geom, runs, geom, counts, nl.max_runs);
  const double vol = (double)nl.cell.a11 * nl.cell.a22 * nl.cell.a33;
  return nl_alloc(nl, n, initial_capacity, runs, geom, counts,
                  half_sphere(n / vol, nl.rl2), nl.trim);
}

// A batch of independent rectangular boxes: each gets the reference's grid,
// its cells numbered after the previous box's; fills the neighbor-grid
// fields of sys.
int nl_init_batch(NeighborList& nl, int n, float cutoff, float skin,
                  std::vector<SysGeom>& sys, int refresh_interval, float skin_permit,
                  int max_neighbor_numbers) {
  if (n <= 0 || sys.empty()) return fail(kBadInput, "neighbor list: empty batch");
  nl_common(nl, n, cutoff, skin, refresh_interval, skin_permit, max_neighbor_numbers);
  int total = 0;
  double max_per = 0.0;
  bool all_balanced = true;
  for (auto& g : sys) {
    int N[3];
    int rc = box_grid(nl.grid_length, g.cell, N);
    if (rc) return rc;
    g.Nx = N[0];
    g.Ny = N[1];
    g.Nz = N[2];
    g.cell_begin = total;
    total += N[0] * N[1] * N[2];
    g.trim = N[0] >= 5 && N[1] >= 5 && N[2] >= 5;
    all_balanced = all_balanced && g.trim;
    g.wx = g.cell.a11 / N[0];
    g.wy = g.cell.a22 / N[1];
    g.iwz = N[2] / g.cell.a33;
    const double vol = (double)g.cell.a11 * g.cell.a22 * g.cell.a33;
    max_per = std::max(max_per, half_sphere((g.atom_end - g.atom_begin) / vol, nl.rl2));
  }
  nl.ncell = total;
  nl.cell = sys[0].cell;
  nl.rcell = sys[0].rcell;
  nl.ortho = true;
  std::vector<std::vector<int2>> per(total);
  std::vector<std::vector<char4>> per_geom(total);
  for (const auto& g : sys) box_runs(g.Nx, g.Ny, g.Nz, g.cell_begin, per, per_geom);
  std::vector<int2> runs;
  std::vector<char4> geom;
  std::vector<int> counts;
  pack_runs(per, per_geom, runs, geom, counts, nl.max_runs);
  return nl_alloc(nl, n, 0, runs, geom, counts, max_per, all_balanced);
}

static int nl_alloc(NeighborList& nl, int n, long long initial_capacity,
                    const std::vector<int2>& runs, const std::vector<char4>& geom,
                    const std::vector<int>& counts, double max_per_atom,
                    bool all_balanced) {
  SNB_CUDA_TRY(cudaMalloc(&nl.d_run_ranges, sizeof(int2) * runs.size()));
  SNB_CUDA_TRY(cudaMemcpy(nl.d_run_ranges, runs.data(), sizeof(int2) * runs.size(),
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_run_geom, sizeof(char4) * geom.size()));
  SNB_CUDA_TRY(cudaMemcpy(nl.d_run_geom, geom.data(), sizeof(char4) * geom.size(),
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_excl_count, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_excl_partner, sizeof(int) * kExclCap * (size_t)n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_run_count, sizeof(int) * nl.ncell));
  SNB_CUDA_TRY(cudaMemcpy(nl.d_run_count, counts.data(), sizeof(int) * nl.ncell,
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_cell_count, sizeof(int) * nl.ncell));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_cell_start, sizeof(int) * (nl.ncell + 1)));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_atom_cell, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_atom_slot, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_perm, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_inv_perm, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_global, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_pos, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_old_crd, sizeof(float3) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_row_count, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_row_start, sizeof(int) * (n + 1)));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_flags, sizeof(int) * kNumFlags));
  SNB_CUDA_TRY(cudaMemset(nl.d_flags, 0, sizeof(int) * kNumFlags));
  SNB_CUDA_TRY(cudaMallocHost(&nl.h_flags, sizeof(int) * kNumFlags));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_unsorted, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_sorted_cell, sizeof(int) * n));
  {
    // before the first build: identity frame and empty rows
    std::vector<int> iota(n);
    for (int i = 0; i < n; ++i) iota[i] = i;
    SNB_CUDA_TRY(cudaMemcpy(nl.d_perm, iota.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(nl.d_inv_perm, iota.data(), sizeof(int) * n,
                            cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(nl.d_global, iota.data(), sizeof(int) * n,
                            cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemset(nl.d_row_count, 0, sizeof(int) * n));
    SNB_CUDA_TRY(cudaMemset(nl.d_row_start, 0, sizeof(int) * (n + 1)));
    SNB_CUDA_TRY(cudaMemset(nl.d_sorted_cell, 0, sizeof(int) * n));
    SNB_CUDA_TRY(cudaMemset(nl.d_pos, 0, sizeof(float4) * n));
  }
  // Row capacity: 1.5x (2.5x where cell pairs are owned by index, which
  // balances rows less well) the mean half-sphere count plus a margin;
  // regrown on overflow by nl_check_overflow.
  if (initial_capacity <= 0)
    initial_capacity = (long long)((all_balanced ? 1.5 : 2.5) * max_per_atom) + 64;
  nl.row_cap = (int)std::min<long long>(initial_capacity, n);
  if (nl.row_cap < 32) nl.row_cap = 32;
  nl.row_cap = (nl.row_cap + 7) & ~7;  // rows start on 32-byte boundaries
  nl.cap = (long long)nl.row_cap * n;
  if (nl.cap + nl.row_cap > 2147483647LL)
    return fail(kBadInput, "neighbor list: rows exceed 32-bit offsets");
  SNB_CUDA_TRY(cudaMalloc(&nl.d_cols, sizeof(int) * nl.cap));
  k_row_starts<<<ceil_div(n + 1, 256), 256>>>(n, nl.row_cap, nl.d_row_start);
  SNB_CUDA_TRY(cudaGetLastError());
  return scan_reserve(nl.scan, std::max(nl.ncell, n));
}

static void clusters_free(NeighborList& nl) {
  cudaFree(nl.d_atom_key);
  cudaFree(nl.d_clus_count);
  cudaFree(nl.d_cell_clus);
  cudaFree(nl.d_clus);
  cudaFree(nl.d_clus_lo);
  cudaFree(nl.d_clus_hi);
  cudaFree(nl.d_nclus);
  cudaFree(nl.d_img_off);
  cudaFree(nl.d_crow_count);
  cudaFree(nl.d_centry);
  nl.d_atom_key = nl.d_clus_count = nl.d_cell_clus = nl.d_nclus = nl.d_crow_count = nullptr;
  nl.d_clus = nl.d_centry = nullptr;
  nl.d_clus_lo = nl.d_clus_hi = nullptr;
  nl.d_img_off = nullptr;
  nl.maxclus = 0;
}

// Storage of the cluster form for the current grid.  Row capacity: 1.5x the
// mean number of clusters in half a sphere of radius r_l + 3 A (a cluster's
// reach) plus a margin; regrown on overflow by nl_check_overflow.
static int clusters_alloc(NeighborList& nl) {
  clusters_free(nl);
  const int n = nl.n;
  nl.maxclus = (n + 3 * nl.ncell) / kClusterSize + 1;
  SNB_CUDA_TRY(cudaMalloc(&nl.d_atom_key, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_clus_count, sizeof(int) * nl.ncell));
  SNB_CUDA_TRY(cudaMemset(nl.d_clus_count, 0, sizeof(int) * nl.ncell));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_cell_clus, sizeof(int) * (nl.ncell + 1)));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_clus, sizeof(int2) * nl.maxclus));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_clus_lo, sizeof(float4) * nl.maxclus));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_clus_hi, sizeof(float4) * nl.maxclus));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_nclus, sizeof(int)));
  SNB_CUDA_TRY(cudaMemset(nl.d_nclus, 0, sizeof(int)));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_img_off, sizeof(float3) * n));
  SNB_CUDA_TRY(cudaMemset(nl.d_img_off, 0, sizeof(float3) * n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_crow_count, sizeof(int) * nl.maxclus));
  SNB_CUDA_TRY(cudaMemset(nl.d_crow_count, 0, sizeof(int) * nl.maxclus));
  if (nl.ccap <= 0) {
    const double vol = (double)nl.cell.a11 * nl.cell.a22 * nl.cell.a33;
    const double rho_c = (double)nl.maxclus / vol;
    const double R = sqrt((double)nl.rl2) + 3.0;
    const double mean = 0.5 * rho_c * 4.18879020478639 * R * R * R;
    nl.ccap = (int)std::min<double>(1.5 * mean + 32.0, (double)nl.maxclus);
    nl.ccap = std::max(nl.ccap, 32);
    nl.ccap = (nl.ccap + 3) & ~3;
  }
  SNB_CUDA_TRY(cudaMalloc(&nl.d_centry, sizeof(int2) * (size_t)nl.maxclus * nl.ccap));
  return kOk;
}

int nl_set_clusters(NeighborList& nl, bool on) {
  if (!on) {
    if (nl.clusters) {
      clusters_free(nl);
      nl.clusters = false;
      nl.generation = 0;
    }
    return kOk;
  }
  if (nl.bv.nsys > 0 || !nl.ortho || !nl.trim)
    return fail(kNotSupported,
                "neighbor list: the cluster form needs one rectangular box of at least "
                "five cells per axis");
  if (nl.n >= (1 << 27))  // the pair kernel packs a sorted index into 27 bits
    return fail(kNotSupported, "neighbor list: the cluster form holds up to 2^27 atoms");
  if (!nl.clusters || nl.maxclus == 0) {
    int rc = clusters_alloc(nl);
    if (rc) return rc;
  }
  nl.clusters = true;
  nl.generation = 0;
  return kOk;
}

// The pruned rows' storage (rows' layout; contents written by the pair
// kernel's prune passes).
int nl_enable_prune(NeighborList& nl) {
  if (nl.d_cols_in) return kOk;
  SNB_CUDA_TRY(cudaMalloc(&nl.d_cols_in, sizeof(int) * nl.cap));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_row_in_count, sizeof(int) * nl.n));
  SNB_CUDA_TRY(cudaMalloc(&nl.d_prune_ref, sizeof(float4) * nl.n));
  SNB_CUDA_TRY(cudaMemset(nl.d_row_in_count, 0, sizeof(int) * nl.n));
  return kOk;
}

void nl_free(NeighborList& nl) {
  clusters_free(nl);
  cudaFree(nl.d_cols_in);
  cudaFree(nl.d_row_in_count);
  cudaFree(nl.d_prune_ref);
  cudaFree(nl.d_unsorted);
  cudaFree(nl.d_sorted_cell);
  cudaFree(nl.d_run_ranges);
  cudaFree(nl.d_run_geom);
  cudaFree(nl.d_excl_count);
  cudaFree(nl.d_excl_partner);
  cudaFree(nl.d_run_count);
  cudaFree(nl.d_cell_count);
  cudaFree(nl.d_cell_start);
  cudaFree(nl.d_atom_cell);
  cudaFree(nl.d_atom_slot);
  cudaFree(nl.d_perm);
  cudaFree(nl.d_inv_perm);
  cudaFree(nl.d_global);
  cudaFree(nl.d_pos);
  cudaFree(nl.d_old_crd);
  cudaFree(nl.d_row_count);
  cudaFree(nl.d_row_start);
  cudaFree(nl.d_cols);
  cudaFree(nl.d_flags);
  if (nl.h_flags) cudaFreeHost(nl.h_flags);
  cudaFree(nl.scan.block_sums);
  nl = NeighborList();
}

// A new rectangular box for a single-box list (barostat box change): the
// reference's grid rule for the new lengths, its neighbour runs when the
// cell counts change, and a forced rebuild on the next update.  The pair
// criterion is exact in any grid whose cells are at least r_l / 2 wide, so
// the pair set is the exact one of the new box.
int nl_regrid(NeighborList& nl, const float* cell6) {
  if (nl.bv.nsys > 0) return fail(kNotSupported, "neighbor list: box change of a batch");
  if (cell6[1] != 0.f || cell6[3] != 0.f || cell6[4] != 0.f || !nl.ortho)
    return fail(kNotSupported,
                "neighbor list: a box change is supported for rectangular boxes");
  const Cell c = make_cell(cell6);
  int N[3];
  int rc = box_grid(nl.grid_length, c, N);
  if (rc) return rc;
  if (N[0] != nl.Nx || N[1] != nl.Ny || N[2] != nl.Nz) {
    const int ncell = N[0] * N[1] * N[2];
    std::vector<std::vector<int2>> per(ncell);
    std::vector<std::vector<char4>> per_geom(ncell);
    box_runs(N[0], N[1], N[2], 0, per, per_geom);
    std::vector<int2> runs;
    std::vector<char4> geom;
    std::vector<int> counts;
    int max_runs = 0;
    pack_runs(per, per_geom, runs, geom, counts, max_runs);
    int2* d_runs = nullptr;
    char4* d_geom = nullptr;
    int *d_run_count = nullptr, *d_cell_count = nullptr, *d_cell_start = nullptr;
    SNB_CUDA_TRY(cudaMalloc(&d_runs, sizeof(int2) * runs.size()));
    SNB_CUDA_TRY(cudaMalloc(&d_geom, sizeof(char4) * geom.size()));
    SNB_CUDA_TRY(cudaMalloc(&d_run_count, sizeof(int) * ncell));
    SNB_CUDA_TRY(cudaMalloc(&d_cell_count, sizeof(int) * ncell));
    SNB_CUDA_TRY(cudaMalloc(&d_cell_start, sizeof(int) * (ncell + 1)));
    SNB_CUDA_TRY(cudaMemcpy(d_runs, runs.data(), sizeof(int2) * runs.size(),
                            cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(d_geom, geom.data(), sizeof(char4) * geom.size(),
                            cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(d_run_count, counts.data(), sizeof(int) * ncell,
                            cudaMemcpyHostToDevice));
    rc = scan_reserve(nl.scan, std::max(ncell, nl.n));
    if (rc) return rc;
    // the old arrays may still be read by work queued before this call
    SNB_CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(nl.d_run_ranges);
    cudaFree(nl.d_run_geom);
    cudaFree(nl.d_run_count);
    cudaFree(nl.d_cell_count);
    cudaFree(nl.d_cell_start);
    nl.d_run_ranges = d_runs;
    nl.d_run_geom = d_geom;
    nl.d_run_count = d_run_count;
    nl.d_cell_count = d_cell_count;
    nl.d_cell_start = d_cell_start;
    nl.max_runs = max_runs;
    nl.Nx = N[0];
    nl.Ny = N[1];
    nl.Nz = N[2];
    nl.ncell = ncell;
    nl.trim = N[0] >= 5 && N[1] >= 5 && N[2] >= 5;
  }
  // cluster storage is sized by the cell count
  const bool regridded =
      nl.clusters && nl.maxclus != (nl.n + 3 * nl.ncell) / kClusterSize + 1;
  nl.cell = c;
  nl.rcell = rect_rcell(c);
  nl.wx = c.a11 / nl.Nx;
  nl.wy = c.a22 / nl.Ny;
  nl.iwz = nl.Nz / c.a33;
  nl.generation = 0;  // the next update rebuilds
  if (nl.clusters) {
    // the cluster form needs five cells per axis; below that the rows serve
    if (!nl.trim) {
      clusters_free(nl);
      nl.clusters = false;
    } else if (regridded) {
      SNB_CUDA_TRY(cudaDeviceSynchronize());
      return clusters_alloc(nl);
    }
  }
  return kOk;
}

int nl_update(NeighborList& nl, const float* crd_f, const int* atom_local,
              const float* cell6, int step, int forced, const int* excl_start,
              const int* excl_list, const int* excl_numbers, cudaStream_t st) {
  if (cell6) {
    Cell c = make_cell(cell6);
    if (c.a11 != nl.cell.a11 || c.a22 != nl.cell.a22 || c.a33 != nl.cell.a33 ||
        c.a21 != nl.cell.a21 || c.a31 != nl.cell.a31 || c.a32 != nl.cell.a32) {
      int rc = nl_regrid(nl, cell6);
      if (rc) return rc;
    }
  }
  const bool first = nl.generation == 0;
  int rc = nl_decide(nl, crd_f, step, forced, st);
  if (rc) return rc;
  rc = nl_rebuild(nl, crd_f, atom_local, excl_start, excl_list, excl_numbers, st);
  if (rc || !first) return rc;
  // The first build sizes the rows from the mean density of the box, which
  // a box with empty regions (a slab, a droplet) underestimates: check it
  // here, regrow and build again, so the first evaluation is complete.  (It
  // is never inside a stream capture: later overflows are caught by
  // nl_check_overflow at the caller's interval.)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  SNB_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  if (cs != cudaStreamCaptureStatusNone) return kOk;
  for (int tries = 0; tries < 4; ++tries) {
    bool regrown = false;
    if ((rc = nl_check_overflow(nl, &regrown, st))) return rc;
    if (!regrown) return kOk;
    if ((rc = nl_decide(nl, crd_f, step, 1, st))) return rc;
    if ((rc = nl_rebuild(nl, crd_f, atom_local, excl_start, excl_list, excl_numbers, st)))
      return rc;
  }
  return kOk;
}

// need_update decision of NEIGHBOR_LIST::Update (neighbor_list.cpp:983-999)
int nl_decide(NeighborList& nl, const float* crd_f, int step, int forced,
              cudaStream_t st) {
  const float3* crd = reinterpret_cast<const float3*>(crd_f);
  const int n = nl.n;
  if (nl.generation == 0) forced = 1;  // nothing built yet
  nl.generation += 1;
  if (forced) {
    nl_need_all(nl, st);
  } else if (nl.refresh_interval <= 0) {
    k_set_need<<<1, 1, 0, st>>>(nl.d_flags, 0);
    float permit = nl.skin * nl.skin_permit;
    if (nl.bv.nsys > 0)
      k_check_refresh<true><<<ceil_div(n, 256), 256, 0, st>>>(
          n, crd, nl.d_old_crd, nl.cell, nl.rcell, permit * permit, nl.d_flags, nl.bv);
    else
      k_check_refresh<false><<<ceil_div(n, 256), 256, 0, st>>>(
          n, crd, nl.d_old_crd, nl.cell, nl.rcell, permit * permit, nl.d_flags, nl.bv);
  } else {
    if ((step + 1) % nl.refresh_interval == 0)
      nl_need_all(nl, st);
    else
      k_set_need<<<1, 1, 0, st>>>(nl.d_flags, 0);
  }
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// The rebuild itself; every kernel returns at once unless the need flag is
// set, so it can also run unconditionally.
int nl_rebuild(NeighborList& nl, const float* crd_f, const int* atom_local,
               const int* excl_start, const int* excl_list, const int* excl_numbers,
               cudaStream_t st) {
  const float3* crd = reinterpret_cast<const float3*>(crd_f);
  const int n = nl.n;
  // Excluded-partner sets need global ids equal to the caller's indices.
  int* excl_count = (excl_numbers && !atom_local) ? nl.d_excl_count : nullptr;
  const unsigned char* need = nl.bv.nsys > 0 ? nl.bv.box_need : nullptr;
  const int* sys_of = nl.bv.nsys > 0 ? nl.bv.sys_of : nullptr;
  const int* cell_sys = nl.bv.nsys > 0 ? nl.bv.cell_sys : nullptr;
  if (need)
    k_zero_cells<<<ceil_div(nl.ncell, 256), 256, 0, st>>>(nl.ncell, nl.d_cell_count,
                                                          nl.d_flags, need, cell_sys);
  else
    SNB_CUDA_TRY(cudaMemsetAsync(nl.d_cell_count, 0, sizeof(int) * nl.ncell, st));
  k_rebuild_begin<<<1, 1, 0, st>>>(nl.d_flags, need != nullptr);
  const bool clus = nl.clusters;
  if (nl.bv.nsys > 0)
    k_bin_count<true><<<ceil_div(n, 256), 256, 0, st>>>(
        n, crd, nl.cell, nl.Nx, nl.Ny, nl.Nz, nl.d_atom_cell, nl.d_atom_slot,
        nl.d_cell_count, excl_count, nl.d_flags, nl.bv, nullptr);
  else
    k_bin_count<false><<<ceil_div(n, 256), 256, 0, st>>>(
        n, crd, nl.cell, nl.Nx, nl.Ny, nl.Nz, nl.d_atom_cell, nl.d_atom_slot,
        nl.d_cell_count, excl_count, nl.d_flags, nl.bv, clus ? nl.d_atom_key : nullptr);
  int rc = scan_exclusive(nl.d_cell_count, nl.d_cell_start, nl.ncell, nullptr,
                          nl.scan, st);
  if (rc) return rc;
  k_bin_scatter<<<ceil_div(n, 256), 256, 0, st>>>(
      n, nl.d_atom_cell, nl.d_atom_slot, nl.d_cell_start, nl.d_unsorted, excl_start,
      excl_list, excl_numbers, excl_count, nl.d_excl_partner, nl.d_flags, need, sys_of);
  k_cell_order<<<ceil_div(nl.ncell, 8), 256, 0, st>>>(nl.ncell, nl.d_cell_start,
                                                      nl.d_unsorted, nl.d_perm,
                                                      nl.d_flags,
                                                      clus ? nl.d_atom_key : nullptr, need,
                                                      cell_sys);
  k_fill_sorted<<<ceil_div(n, 256), 256, 0, st>>>(n, nl.d_perm, crd, atom_local,
                                                  nl.d_inv_perm, nl.d_global,
                                                  nl.d_pos, nl.d_old_crd, nl.d_flags,
                                                  clus ? nl.d_img_off : nullptr, nl.cell,
                                                  need, sys_of);
  k_sorted_cell<<<ceil_div(n, 256), 256, 0, st>>>(n, nl.d_perm, nl.d_atom_cell,
                                                  nl.d_sorted_cell, nl.d_flags, need, sys_of);
  static int sms = 0;
  if (!sms) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  if (clus) {
    k_clus_count<<<ceil_div(nl.ncell, 256), 256, 0, st>>>(nl.ncell, nl.d_cell_start,
                                                          nl.d_clus_count, nl.d_flags);
    rc = scan_exclusive(nl.d_clus_count, nl.d_cell_clus, nl.ncell, nl.d_nclus, nl.scan,
                        st);
    if (rc) return rc;
    k_clus_fill<<<ceil_div(nl.ncell, 128), 128, 0, st>>>(
        nl.ncell, nl.d_cell_start, nl.d_cell_clus, nl.d_pos, nl.cell, nl.d_clus,
        nl.d_clus_lo, nl.d_clus_hi, nl.d_flags);
    ClusterSearchArgs ca;
    ca.pos = nl.d_pos;
    ca.sorted_cell = nl.d_sorted_cell;
    ca.cell_clus = nl.d_cell_clus;
    ca.clus = nl.d_clus;
    ca.clus_lo = nl.d_clus_lo;
    ca.clus_hi = nl.d_clus_hi;
    ca.nclus = nl.d_nclus;
    ca.runs = nl.d_run_ranges;
    ca.geom = nl.d_run_geom;
    ca.run_count = nl.d_run_count;
    ca.max_runs = nl.max_runs;
    ca.Nx = nl.Nx;
    ca.Ny = nl.Ny;
    ca.Nz = nl.Nz;
    ca.cell = nl.cell;
    ca.rcell = nl.rcell;
    ca.rl2 = nl.rl2;
    ca.rl2_lo = nl.rl2 * (1.0f - 2e-5f);
    ca.rl2_hi = nl.rl2 * (1.0f + 2e-5f);
    ca.reach2 = nl.reach2;
    ca.wx = nl.cell.a11 / nl.Nx;
    ca.wy = nl.cell.a22 / nl.Ny;
    ca.wz = nl.cell.a33 / nl.Nz;
    ca.excl_start = excl_start;
    ca.excl_list = excl_list;
    ca.excl_numbers = excl_numbers;
    ca.excl_count = excl_count;
    ca.excl_partner = nl.d_excl_partner;
    ca.crow_count = nl.d_crow_count;
    ca.ccap = nl.ccap;
    ca.centry = nl.d_centry;
    ca.flags = nl.d_flags;
    const int cblocks = std::min(ceil_div(nl.maxclus, 8),
                                 sms * std::max(1, nl.search_blocks_per_sm));
    k_cluster_search<<<cblocks, 256, 0, st>>>(ca);
    k_finish_build<<<1, 1, 0, st>>>(nl.d_flags);
    SNB_CUDA_TRY(cudaGetLastError());
    return kOk;
  }
  SearchArgs sa;
  sa.n = n;
  sa.pos = nl.d_pos;
  sa.sorted_cell = nl.d_sorted_cell;
  sa.cell_start = nl.d_cell_start;
  sa.runs = nl.d_run_ranges;
  sa.geom = nl.d_run_geom;
  sa.run_count = nl.d_run_count;
  sa.max_runs = nl.max_runs;
  sa.Nx = nl.Nx;
  sa.Ny = nl.Ny;
  sa.Nz = nl.Nz;
  sa.cell = nl.cell;
  sa.rcell = nl.rcell;
  sa.rl2 = nl.rl2;
  sa.rl2_lo = nl.rl2 * (1.0f - 2e-5f);
  sa.rl2_hi = nl.rl2 * (1.0f + 2e-5f);
  sa.ortho = nl.ortho;
  sa.trim = nl.trim;
  sa.reach2 = nl.reach2;
  sa.wx = nl.wx;
  sa.wy = nl.wy;
  sa.iwz = nl.iwz;
  sa.excl_start = excl_start;
  sa.excl_list = excl_list;
  sa.excl_numbers = excl_numbers;
  sa.excl_count = excl_count;
  sa.excl_partner = nl.d_excl_partner;
  sa.row_count = nl.d_row_count;
  sa.row_cap = nl.row_cap;
  sa.cols = nl.d_cols;
  sa.flags = nl.d_flags;
  sa.bv = nl.bv;
  const int blocks = std::min(ceil_div(n, 8), sms * std::max(1, nl.search_blocks_per_sm));
  if (nl.bv.nsys > 0)
    k_pair_search<true><<<blocks, 256, 0, st>>>(sa);
  else
    k_pair_search<false><<<blocks, 256, 0, st>>>(sa);
  k_finish_build<<<1, 1, 0, st>>>(nl.d_flags);
  if (need)  // the systems' flags for the next decision
    SNB_CUDA_TRY(cudaMemsetAsync(nl.bv.box_need, 0, nl.bv.nsys, st));
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

int nl_check_overflow(NeighborList& nl, bool* regrown, cudaStream_t st) {
  *regrown = false;
  SNB_CUDA_TRY(cudaMemcpyAsync(nl.h_flags, nl.d_flags, sizeof(int) * kNumFlags,
                               cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  nl.last_total = nl.h_flags[kFlagTotal];
  if (nl.h_flags[kFlagListOverflow] && nl.clusters) {
    const long long need = nl.h_flags[kFlagMaxRow];
    int cap = (int)std::min<long long>(need + need / 5 + 16, nl.maxclus);
    cap = (std::max(cap, nl.ccap + 16) + 3) & ~3;
    SNB_CUDA_TRY(cudaStreamSynchronize(st));
    SNB_CUDA_TRY(cudaFree(nl.d_centry));
    nl.d_centry = nullptr;
    nl.ccap = cap;
    SNB_CUDA_TRY(cudaMalloc(&nl.d_centry, sizeof(int2) * (size_t)nl.maxclus * nl.ccap));
    int zero = 0;
    SNB_CUDA_TRY(cudaMemcpyAsync(nl.d_flags + kFlagListOverflow, &zero, sizeof(int),
                                 cudaMemcpyHostToDevice, st));
    SNB_CUDA_TRY(cudaStreamSynchronize(st));
    *regrown = true;
    return kOk;
  }
  if (nl.h_flags[kFlagListOverflow]) {
    long long need = nl.h_flags[kFlagMaxRow];
    int cap = (int)std::min<long long>(need + need / 5 + 32, nl.n);
    SNB_CUDA_TRY(cudaFree(nl.d_cols));
    nl.row_cap = (std::max(cap, nl.row_cap + 32) + 7) & ~7;
    nl.cap = (long long)nl.row_cap * nl.n;
    if (nl.cap + nl.row_cap > 2147483647LL)
      return fail(kOverflow, "neighbor list: rows exceed 32-bit offsets");
    SNB_CUDA_TRY(cudaMalloc(&nl.d_cols, sizeof(int) * nl.cap));
    if (nl.d_cols_in) {  // the pruned rows follow the rows' capacity
      SNB_CUDA_TRY(cudaFree(nl.d_cols_in));
      nl.d_cols_in = nullptr;
      SNB_CUDA_TRY(cudaMalloc(&nl.d_cols_in, sizeof(int) * nl.cap));
    }
    k_row_starts<<<ceil_div(nl.n + 1, 256), 256, 0, st>>>(nl.n, nl.row_cap, nl.d_row_start);
    int zero = 0;
    SNB_CUDA_TRY(cudaMemcpyAsync(nl.d_flags + kFlagListOverflow, &zero, sizeof(int),
                                 cudaMemcpyHostToDevice, st));
    SNB_CUDA_TRY(cudaStreamSynchronize(st));
    *regrown = true;
  }
  return kOk;
}

int nl_total_pairs(NeighborList& nl, long long* total, cudaStream_t st) {
  bool regrown;
  int rc = nl_check_overflow(nl, &regrown, st);
  if (rc) return rc;
  *total = nl.last_total;
  return kOk;
}

// ---------------------------------------------------------------------------
// Exports.
struct AtomGroupABI {  // layout of the reference's ATOM_GROUP (common.h:177-182)
  int atom_numbers;
  int ghost_numbers;
  int* atom_serial;
};

// pairs in global ids (lo, hi), in sorted-frame list order
__global__ void k_export_pairs(int n, const int* __restrict__ row_start,
                               const int* __restrict__ row_count,
                               const int* __restrict__ cols,
                               const long long* __restrict__ out_start,
                               const int* __restrict__ global, int* pi, int* pj,
                               long long cap) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (i >= n) return;
  int gi = global[i];
  const long long o = out_start[i];
  for (int q = lane; q < row_count[i]; q += 32) {
    if (o + q >= cap) break;
    int gj = global[cols[row_start[i] + q]];
    pi[o + q] = gi < gj ? gi : gj;
    pj[o + q] = gi < gj ? gj : gi;
  }
}

__global__ void k_export_groups_reset(int n, AtomGroupABI* groups, int* slab,
                                      int maxn, int* counts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  counts[i] = 0;
  groups[i].ghost_numbers = 0;
  groups[i].atom_serial = slab + (size_t)i * maxn;
}

// Reference row semantics: the row of local atom a holds local b with
// global(b) > global(a).  Local index = caller index here.
__global__ void k_export_groups_fill(int n, const int* __restrict__ row_start,
                                     const int* __restrict__ row_count,
                                     const int* __restrict__ cols,
                                     const int* __restrict__ global,
                                     const int* __restrict__ perm, int* slab, int maxn,
                                     int* counts, int* flags) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (i >= n) return;
  if (flags[kFlagListOverflow]) return;
  int gi = global[i];
  int li = perm[i];
  for (int k = row_start[i] + lane; k < row_start[i] + row_count[i]; k += 32) {
    int j = cols[k];
    int gj = global[j];
    int lj = perm[j];
    int owner = gi < gj ? li : lj;
    int other = gi < gj ? lj : li;
    int slot = atomicAdd(&counts[owner], 1);
    if (slot < maxn)
      slab[(size_t)owner * maxn + slot] = other;
    else
      flags[kFlagExportOverflow] = 1;
  }
}

__global__ void k_export_groups_counts(int n, AtomGroupABI* groups, const int* counts,
                                       int maxn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  groups[i].atom_numbers = counts[i] < maxn ? counts[i] : maxn;
}

int nl_export_atom_groups(NeighborList& nl, void* d_groups, int* d_slab,
                          int max_neighbor_numbers, cudaStream_t st) {
  if (nl.clusters)
    return fail(kNotSupported, "neighbor list export: ATOM_GROUP rows of the cluster form");
  const int n = nl.n;
  int* counts = nullptr;
  SNB_CUDA_TRY(cudaMallocAsync(&counts, sizeof(int) * n, st));
  AtomGroupABI* g = reinterpret_cast<AtomGroupABI*>(d_groups);
  k_export_groups_reset<<<ceil_div(n, 256), 256, 0, st>>>(n, g, d_slab,
                                                          max_neighbor_numbers, counts);
  k_export_groups_fill<<<ceil_div(n, 8), 256, 0, st>>>(
      n, nl.d_row_start, nl.d_row_count, nl.d_cols, nl.d_global, nl.d_perm, d_slab,
      max_neighbor_numbers, counts, nl.d_flags);
  k_export_groups_counts<<<ceil_div(n, 256), 256, 0, st>>>(n, g, counts,
                                                           max_neighbor_numbers);
  SNB_CUDA_TRY(cudaFreeAsync(counts, st));
  SNB_CUDA_TRY(cudaGetLastError());
  int flag = 0;
  SNB_CUDA_TRY(cudaMemcpyAsync(&flag, nl.d_flags + kFlagExportOverflow, sizeof(int),
                               cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  if (flag) {
    int zero = 0;
    cudaMemcpy(nl.d_flags + kFlagExportOverflow, &zero, sizeof(int),
               cudaMemcpyHostToDevice);
    return fail(kOverflow, "neighbor list export: max_neighbor_numbers exceeded");
  }
  return kOk;
}

// Pairs of the cluster form in global ids (lo, hi), in no particular order.
__global__ void k_export_cluster_pairs(const int* __restrict__ nclus,
                                       const int2* __restrict__ clus,
                                       const int* __restrict__ crow_count,
                                       const int2* __restrict__ centry, int ccap,
                                       const int* __restrict__ global, int* pi, int* pj,
                                       long long cap, unsigned long long* next) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= *nclus) return;
  const int si = clus[c].x;
  for (int e = lane; e < crow_count[c]; e += 32) {
    const int2 en = centry[(size_t)c * ccap + e];
    for (int b = 0; b < 16; ++b) {
      if (!((en.y >> b) & 1)) continue;
      const int gi = global[si + (b >> 2)], gj = global[en.x + (b & 3)];
      const unsigned long long o = atomicAdd(next, 1ull);
      if ((long long)o < cap) {
        pi[o] = gi < gj ? gi : gj;
        pj[o] = gi < gj ? gj : gi;
      }
    }
  }
}

int nl_export_pairs(NeighborList& nl, int* d_pi, int* d_pj, long long cap,
                    long long* count, cudaStream_t st) {
  long long total = 0;
  int rc = nl_total_pairs(nl, &total, st);
  if (rc) return rc;
  *count = total;
  if (total > cap) return fail(kOverflow, "export_pairs: capacity too small");
  if (nl.clusters) {
    unsigned long long* next = nullptr;
    SNB_CUDA_TRY(cudaMalloc(&next, sizeof(unsigned long long)));
    SNB_CUDA_TRY(cudaMemsetAsync(next, 0, sizeof(unsigned long long), st));
    k_export_cluster_pairs<<<ceil_div(nl.maxclus, 8), 256, 0, st>>>(
        nl.d_nclus, nl.d_clus, nl.d_crow_count, nl.d_centry, nl.ccap, nl.d_global, d_pi,
        d_pj, cap, next);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(next);
    if (e != cudaSuccess) return fail(kCudaError, cudaGetErrorString(e));
    SNB_CUDA_TRY(cudaGetLastError());
    return kOk;
  }
  // output offsets of the rows (host prefix sum of the row counts)
  std::vector<int> counts(nl.n);
  SNB_CUDA_TRY(cudaMemcpy(counts.data(), nl.d_row_count, sizeof(int) * nl.n,
                          cudaMemcpyDeviceToHost));
  std::vector<long long> starts(nl.n);
  long long acc = 0;
  for (int i = 0; i < nl.n; ++i) {
    starts[i] = acc;
    acc += counts[i];
  }
  long long* d_starts = nullptr;
  SNB_CUDA_TRY(cudaMalloc(&d_starts, sizeof(long long) * nl.n));
  SNB_CUDA_TRY(cudaMemcpy(d_starts, starts.data(), sizeof(long long) * nl.n,
                          cudaMemcpyHostToDevice));
  k_export_pairs<<<ceil_div(nl.n, 8), 256, 0, st>>>(nl.n, nl.d_row_start, nl.d_row_count,
                                                    nl.d_cols, d_starts, nl.d_global,
                                                    d_pi, d_pj, cap);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(d_starts);
  if (e != cudaSuccess) return fail(kCudaError, cudaGetErrorString(e));
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace snb
