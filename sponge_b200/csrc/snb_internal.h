// Internal state of the nonbonded engine and the launchers each .cu exposes.
// Not part of the public C-ABI (that is include/sponge_nb.h).
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "snb_common.cuh"

struct snb_vatom;  // virtual atoms (snb_vatom.cu)

namespace snb {

// ----------------------------------------------------------------------------
// Status codes (mirrored in include/sponge_nb.h)
enum Status {
  kOk = 0,
  kBadInput = 1,
  kCudaError = 2,
  kOverflow = 3,
  kTimeout = 4,
  kNotSupported = 5,
};

void set_error(const std::string& msg);
int fail(int code, const std::string& msg);

#define SNB_CUDA_TRY(expr)                                                   \
  do {                                                                       \
    cudaError_t e_ = (expr);                                                 \
    if (e_ != cudaSuccess)                                                   \
      return ::snb::fail(::snb::kCudaError,                                  \
                         std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Scratch for the device-wide exclusive scan (3-phase).
struct ScanScratch {
  int* block_sums = nullptr;
  int capacity_blocks = 0;
};
constexpr int kScanBlock = 1024;
int scan_exclusive(const int* in, int* out, int n, int* total_out,
                   ScanScratch& s, cudaStream_t st);
int scan_reserve(ScanScratch& s, int n);

// ----------------------------------------------------------------------------
// Independent periodic boxes advanced together (a batch).  The atoms of
// system s are [atom_begin, atom_end) in the caller's order; the counting
// sort keeps each system's cells together and in system order, so the same
// range holds in the sorted frame.  One SysGeom per system on the device;
// kernels compiled with BATCH = true read their atom's (or tile's) entry,
// the single-box kernels (BATCH = false) take the geometry as arguments.
struct SysGeom {
  Cell cell, rcell;             // rectangular box
  int atom_begin, atom_end;
  // neighbor grid: cells [cell_begin, cell_begin + Nx*Ny*Nz) of the batch
  int Nx, Ny, Nz, cell_begin;
  float wx, wy, iwz;            // cell widths (x, y) and 1/width (z)
  int trim;                     // cell offsets unique (>= 5 cells per axis)
  // PME: grid K0 x K1 x K2, 8^3 tiles [tile_begin, tile_begin + nt0*nt1*nt2)
  int K0, K1, K2;
  int nt0, nt1, nt2, tile_begin;
  int grid_begin;               // first point of the real grid (Q, phi)
  int spec_begin;               // first point of the half spectrum (FQ)
  int src_begin0, src_begin1, src_begin2;  // per-axis source-bin tables
  int b_begin0, b_begin1, b_begin2;        // per-axis |b|^2 tables
  float mpre, inv_pi_v;         // pi^2 / beta^2, 1 / (pi V)
  double volume;
};

struct BatchView {
  const SysGeom* sys = nullptr;  // [nsys]
  const int* sys_of = nullptr;   // [n] system of each atom
  const int* tile_sys = nullptr;  // [ntiles] system of each PME tile
  int nsys = 0;
  // per-system list rebuild: box_need[s] set when an atom of system s moved
  // past the skin allowance (cleared after each rebuild); cell_sys maps a
  // neighbor cell to its system
  unsigned char* box_need = nullptr;  // [nsys]
  const int* cell_sys = nullptr;      // [ncell]
};

// A batch rebuilds the lists of the systems that need it.  A system joins a
// rebuild once one of its atoms has moved more than kBatchEarly x the skin
// allowance; only a move past the full allowance starts one.  Systems near
// their own limit thus rebuild together, so fewer steps rebuild at all.
constexpr float kBatchEarly = 0.75f;

// Marks system s of a batch for the next rebuild after an atom of it moved
// by sqrt(d2) (permit2: the squared allowance).
__device__ __forceinline__ void box_mark(unsigned char* need, int s, float d2, float permit2) {
  if (d2 > permit2 * (kBatchEarly * kBatchEarly) && need[s] == 0) need[s] = 1;
}

// True unless i (an atom, or a sorted slot: a system's sorted slots are its
// own atom range) belongs to a system that keeps its list this rebuild.
__device__ __forceinline__ bool box_rebuilds(const unsigned char* need, const int* sys, int i) {
  return need == nullptr || need[sys[i]] != 0;
}

// Device flags of a neighbor list (NeighborList::d_flags).  kFlagFull: the
// pending rebuild covers every system of a batch (so the pair total restarts
// from zero instead of being corrected row by row).
enum { kFlagNeed = 0, kFlagListOverflow = 1, kFlagTotal = 2, kFlagGeneration = 3,
       kFlagExportOverflow = 4, kFlagMaxRow = 5, kFlagFull = 6, kNumFlags = 8 };

// ----------------------------------------------------------------------------
// Neighbor list: cell grid of side >= (cutoff+skin)/2 (neighbor_list.cpp:943),
// atoms counting-sorted by cell (stable: ties by caller index), half list in
// the sorted frame stored as CSR rows.
struct NeighborList {
  int n = 0;
  float cutoff = 10.f, skin = 2.f;
  float grid_length = 6.f;
  float rl2 = 144.f;           // (grid_length^2)*4, formed as the reference
  int refresh_interval = 0;    // neighbor_list_refresh_interval
  float skin_permit = 0.5f;    // neighbor_list_skin_permit
  int max_neighbor_numbers = 1200;  // capacity of the exported ATOM_GROUP slab
  int Nx = 0, Ny = 0, Nz = 0, ncell = 0;
  Cell cell{}, rcell{};
  bool ortho = true;
  // per-cell runs of forward neighbor cells (cell index > own), merged into
  // contiguous cell ranges [first, last]
  int max_runs = 0;
  int2* d_run_ranges = nullptr;  // [ncell][max_runs] {first_cell, last_cell}
  char4* d_run_geom = nullptr;   // [ncell][max_runs] {dx, dy, dz first, dz last}
  int* d_run_count = nullptr;  // [ncell]
  bool trim = false;           // runs are cut to the cells within reach of i
  float reach2 = 0.f;
  float wx = 0.f, wy = 0.f, iwz = 0.f;
  // excluded partners per atom (rebuilt with the list when ids are the
  // caller's indices): count [n] and up to 16 partners [n][16]
  int* d_excl_count = nullptr;
  int* d_excl_partner = nullptr;
  BatchView bv;                // nsys > 0: a batch of boxes (per-system grids)
  int search_blocks_per_sm = 8;  // persistent blocks of the pair search per SM
  // binning
  int* d_cell_count = nullptr;  // [ncell]
  int* d_cell_start = nullptr;  // [ncell + 1]
  int* d_atom_cell = nullptr;   // [n] cell of caller atom
  int* d_atom_slot = nullptr;   // [n]
  int* d_perm = nullptr;        // [n] sorted -> caller index
  int* d_inv_perm = nullptr;    // [n] caller -> sorted index
  int* d_global = nullptr;      // [n] sorted -> global id (atom_local)
  float4* d_pos = nullptr;      // [n] sorted build-time coordinates (x,y,z,-)
  float3* d_old_crd = nullptr;  // [n] caller-frame coordinates at last build
  // list
  int* d_row_count = nullptr;   // [n] entries in row i
  int* d_row_start = nullptr;   // [n + 1] = i * row_cap
  int* d_cols = nullptr;        // [n * row_cap] sorted-frame j of each pair
  int row_cap = 0;
  // pruned rows (engine, single box): the entries of each row within
  // cutoff + prune margin at the last prune pass, in the rows' layout, and
  // the sorted positions that pass saw (null until nl_enable_prune)
  int* d_cols_in = nullptr;     // [n * row_cap]
  int* d_row_in_count = nullptr;  // [n]
  float4* d_prune_ref = nullptr;  // [n]
  long long cap = 0;
  int* d_unsorted = nullptr;    // [n] cell-binned caller indices before ordering
  int* d_sorted_cell = nullptr;  // [n] cell of each sorted atom
  int* d_flags = nullptr;       // [0] need_update  [1] list overflow  [2] pair total
                                // [3] rebuild count  [4] export overflow
  int* h_flags = nullptr;       // pinned mirror
  ScanScratch scan;
  long long last_total = 0;
  int generation = 0;
  // Cluster form of the list (the engine's single-box step; needs at least
  // five cells per axis).  Inside a cell the atoms follow a path up and down
  // its four xy quarter columns, and every run of up to kClusterSize of them
  // is one cluster.  Row c lists the j-clusters with a pair within r_l of
  // i-cluster c: {first sorted atom of j, 4x4 pair mask | shift code << 16}.
  // Pair-frame coordinates are crd - img_off (each atom in its build-time
  // cell image); the shift code gives the periodic image of j's cell.
  bool clusters = false;
  int maxclus = 0;
  int* d_atom_key = nullptr;     // [n] caller frame: order key inside the cell
  int* d_clus_count = nullptr;   // [ncell] clusters of each cell
  int* d_cell_clus = nullptr;    // [ncell + 1] first cluster of each cell
  int2* d_clus = nullptr;        // [maxclus] {first sorted atom, atom count}
  float4* d_clus_lo = nullptr;   // [maxclus] bounding box in the wrapped frame
  float4* d_clus_hi = nullptr;
  int* d_nclus = nullptr;        // [1] clusters of the last build
  float3* d_img_off = nullptr;   // [n] sorted frame: box offset of the cell image
  int* d_crow_count = nullptr;   // [maxclus]
  int2* d_centry = nullptr;      // [maxclus * ccap]
  int ccap = 0;
};
constexpr int kClusterSize = 4;
// Turns the cluster form on or off (single box, rectangular, at least five
// cells per axis); the next update rebuilds.  Returns kNotSupported when the
// box does not allow it.
int nl_set_clusters(NeighborList& nl, bool on);

int nl_init(NeighborList& nl, int n, float cutoff, float skin, const float* cell6,
            int refresh_interval, float skin_permit, int max_neighbor_numbers,
            long long initial_capacity);
// A batch of rectangular boxes (sys[s].cell, rcell and atom ranges set);
// fills the neighbor-grid fields of sys.  The caller sets nl.bv once the
// SysGeom table is on the device.
int nl_init_batch(NeighborList& nl, int n, float cutoff, float skin,
                  std::vector<SysGeom>& sys, int refresh_interval, float skin_permit,
                  int max_neighbor_numbers);
void nl_free(NeighborList& nl);
// Allocates the pruned rows (NeighborList::d_cols_in and the rest).
int nl_enable_prune(NeighborList& nl);
// Update as NEIGHBOR_LIST::Update (neighbor_list.cpp:974-1025): forced, or
// conditional on the displacement check / refresh interval.  Device-side
// decision; no host sync.
int nl_update(NeighborList& nl, const float* crd, const int* atom_local,
              const float* cell6, int step, int forced, const int* excl_start,
              const int* excl_list, const int* excl_numbers, cudaStream_t st);
int nl_decide(NeighborList& nl, const float* crd, int step, int forced, cudaStream_t st);
int nl_rebuild(NeighborList& nl, const float* crd, const int* atom_local,
               const int* excl_start, const int* excl_list, const int* excl_numbers,
               cudaStream_t st);
// Sets the graph's rebuild condition from the need flag; with prune (an
// engine's pruned-row flags) also decides the step's prune pass.
int nl_set_condition(NeighborList& nl, cudaGraphConditionalHandle h, cudaStream_t st,
                     int* prune = nullptr);
// stress = (virial [6] (may be null) + constraint virial (fixed point, may be
// null) + sum m v (x) v) * inv_v into out[0..5], pressure in bar into out[6].
int launch_pressure(int n, const float3* vel, const float* mass, const double* virial,
                    const long long* constraint_virial, double inv_v, double* scratch6,
                    double* out, cudaStream_t st);
// Raises the need flag when an atom of crd is more than skin * skin_permit
// from where it was at the last build (single boxes).
int nl_check_moved(NeighborList& nl, const float* crd, cudaStream_t st);
int nl_force_next(NeighborList& nl, cudaStream_t st);
// A new rectangular box (single-box list): re-grid and force the next build.
int nl_regrid(NeighborList& nl, const float* cell6);
// Reads the overflow flag and regrows the pair storage if needed (host sync).
int nl_check_overflow(NeighborList& nl, bool* regrown, cudaStream_t st);
int nl_total_pairs(NeighborList& nl, long long* total, cudaStream_t st);
// Reference-format export (ATOM_GROUP {int n, int ghost_n, int* serial}).
int nl_export_atom_groups(NeighborList& nl, void* d_groups, int* d_slab,
                          int max_neighbor_numbers, cudaStream_t st);
int nl_export_pairs(NeighborList& nl, int* d_pi, int* d_pj, long long cap,
                    long long* count, cudaStream_t st);

// ----------------------------------------------------------------------------
// Accumulation mode.
enum Accum { kAccumFixed = 0, kAccumFloat = 1 };

// Per-atom accumulators in the sorted frame.
struct Accumulators {
  int n = 0;
  long long* d_f = nullptr;     // [3][n] fixed-point forces (2^40)
  long long* d_e = nullptr;     // [n] fixed-point energy (2^32)  (pair owner)
  long long* d_elj = nullptr;   // [n] LJ part
  long long* d_ec = nullptr;    // [n] direct Coulomb part
  long long* d_v = nullptr;     // [6][n] fixed-point virial (2^32)
  float* d_ff = nullptr;        // [3][n] float forces (plain path)
  float* d_fe = nullptr;        // [3][n] float energies e, elj, ec
  float* d_fv = nullptr;        // [6][n] float virial
  long long* d_eaux = nullptr;  // [2][n] soft-core LJ energy inter / intra subsystem
  float* d_feaux = nullptr;     // [2][n] float version
};
int acc_init(Accumulators& a, int n);
void acc_free(Accumulators& a);

// ----------------------------------------------------------------------------
// Lennard-Jones + direct Coulomb.
struct LJParams {
  int n_types = 0;
  int n_pairs = 0;
  float* d_A = nullptr;
  float* d_B = nullptr;
  int* d_type = nullptr;        // caller frame [n]
  int* d_type_local = nullptr;  // after Get_Local
  std::vector<int> h_type;
  std::vector<float> h_A, h_B;
  float cutoff = 10.f;
  float long_range_factor = 0.f;
};

struct PairArgs {
  int n;
  const float4* pos;            // sorted (x,y,z,q)
  const int* type;              // sorted LJ type
  const int* global;            // sorted -> global id (owner rule)
  const int* row_start;
  const int* row_count;
  const int* cols;
  const int* nl_flags;          // neighbor-list flags: skip when the list overflowed
  const float* A;
  const float* B;
  int n_types;
  Cell cell, rcell;
  float cutoff2;
  float beta;
  BatchView bv;                 // nsys > 0: per-system boxes (rectangular)
  int unroll = 4;               // scan candidates per lane per round (2, 4, 8)
  int blocks_per_sm = 0;        // persistent blocks per SM, 0: occupancy maximum
  int warps = 8;                // rows in flight per block (4, 8, 16)
  bool stash = false;           // hits keep displacement / pair index (row kernel)
  // solvent split (single box): the atoms with global id >= solvent_begin
  // are the trailing water block.  solvent_mode 1: every pair but the
  // solvent-solvent ones (LENNARD_JONES_INFORMATION with solvent_numbers);
  // 2: only those (SOLVENT_LENNARD_JONES); 0: every pair
  int solvent_mode = 0;
  int solvent_begin = 0;
  // pruned rows (solvent_mode 0; prune == null: full rows only).
  // prune[0] != 0: a prune pass scans the full rows and keeps the entries
  // within sqrt(prune2) in cols_in / row_in_count, with row i's position in
  // prune_ref[i]; otherwise the scan reads cols_in / row_in_count.
  const int* prune = nullptr;
  int* cols_in = nullptr;
  int* row_in_count = nullptr;
  float4* prune_ref = nullptr;
  float prune2 = 0.f;
};
int launch_pair(const PairArgs& a, Accumulators& acc, int accum, bool energy,
                bool virial, bool ortho, cudaStream_t st);

// The pruned rows' displacement check of the next step: flag[0] is raised
// when an atom lies more than sqrt(permit2) from ref[its sorted slot] (the
// position the last prune pass saw).  ref == null: no check.
struct PruneCheck {
  const float4* ref = nullptr;
  float permit2 = 0.f;
  int* flag = nullptr;
};
// The same check alone, on final coordinates (after constraints or sites).
int launch_prune_check(int n, const float3* crd, const int* map, const PruneCheck& pc,
                       const Cell& cell, const Cell& rcell, cudaStream_t st,
                       const BatchView& bv);

// The pair kernel over the cluster form of the list.
struct ClusterPairArgs {
  const int2* clus;             // {first sorted atom, atom count}
  const int* nclus;             // device count of clusters
  const int* crow_count;
  const int2* centry;           // {first atom of j, mask | shift code << 16}
  int ccap;
  const float4* pos;            // pair frame (x,y,z,q), sorted
  const int* type;              // sorted LJ type
  const int* global;            // sorted -> global id (owner rule)
  const int* nl_flags;          // skip when the list overflowed
  const float* A;
  const float* B;
  int n_types;
  float3 box;                   // rectangular box lengths (image shifts)
  float cutoff2;
  float beta;
  int blocks_per_sm = 0;        // persistent blocks per SM, 0: occupancy maximum
};
int launch_pair_clusters(const ClusterPairArgs& a, Accumulators& acc, int accum,
                         bool energy, bool virial, cudaStream_t st);

// Rigid triangle: atoms A, B, C, canonical frame (A at (0, ra), B at (rc, rb),
// C at (rd, re) about the centre of mass) and masses.
struct SettleTri {
  int a, b, c;
  float ra, rb, rc, rd, re;
  float ma, mb, mc;
};
// Rigid pair i-j of length r0; k = 1 / (m_i + m_j).
struct SettlePair {
  int i, j;
  float r0, k, mi, mj;
};
struct Settle {
  int n = 0, nt = 0, np = 0;
  std::vector<int> remaining;  // constraint pairs SETTLE leaves to SHAKE
  SettleTri* d_tri = nullptr;
  SettlePair* d_pair = nullptr;
  float3* d_last_ba = nullptr;
  float3* d_last_ca = nullptr;
  float3* d_last_ab = nullptr;
  long long* d_vir = nullptr;  // [6] constraint virial since the last remember, fixed point
  int* d_err = nullptr;        // 1 + index of a pair without a real solution, else 0
};
int settle_group(int n, int m, const int* ai, const int* aj, const float* r0,
                 const float* mass, std::vector<SettleTri>& tri,
                 std::vector<SettlePair>& pair, std::vector<int>& remaining);
int settle_init(Settle& s, int n, int m, const int* ai, const int* aj, const float* r0,
                const float* mass);
void settle_free(Settle& s);
int launch_settle_remember(const Settle& s, const float3* crd, const Cell& cell,
                           const Cell& rcell, cudaStream_t st);
// stress (may be null): += constraint virial / V.
int launch_settle(const Settle& s, float3* crd, float3* vel, const Cell& cell,
                  const Cell& rcell, float dt, float v_factor, float x_factor, float* stress,
                  cudaStream_t st);

// 1-4 terms (NON_BOND_14): pairs with their scaled A', B' and Coulomb scale.
struct NB14 {
  int m = 0;
  int* d_a = nullptr;
  int* d_b = nullptr;
  float* d_A = nullptr;
  float* d_B = nullptr;
  float* d_cf = nullptr;
};
int nb14_init(NB14& p, int m, const int* a, const int* b, const float* A, const float* B,
              const float* cf, int atom_numbers);
void nb14_free(NB14& p);
// map (may be null): caller index -> accumulator slot; per_atom: per-atom
// energies into acc; sums (may be null): fixed-point {LJ + Coulomb, Coulomb}
int launch_nb14(const NB14& p, const float3* crd, const float* charge, const Cell& cell,
                const Cell& rcell, const int* map, Accumulators& acc, bool energy,
                bool virial, bool per_atom, long long* sums, cudaStream_t st);

// Soft-core LJ + direct Coulomb (LJ_SOFT_CORE).
struct SoftArgs {
  int n;
  const float4* pos;            // sorted (x,y,z,q)
  const int2* par;              // sorted {typeA | typeB << 16, mask}
  const float* dq;              // sorted charge_B - charge_A (may be null)
  const int* global;
  const int* row_start;
  const int* row_count;
  const int* cols;
  const int* nl_flags;
  const float* AA;              // A' of state A, per pair of A types
  const float* AB;              // B' of state A
  const float* BA;              // A' of state B, per pair of B types
  const float* BB;              // B' of state B
  int n_types_A, n_types_B;
  Cell cell, rcell;
  float cutoff2;
  float beta;
  float lambda, alpha, p;
  float sigma6, sigma6_min;
  // pruned rows of the engine's row kernel, as PairArgs::prune
  const int* prune = nullptr;
  int* cols_in = nullptr;
  int* row_in_count = nullptr;
  float4* prune_ref = nullptr;
  float prune2 = 0.f;
};
int launch_soft(const SoftArgs& a, Accumulators& acc, int accum, bool energy,
                bool virial, bool dudl, long long* dudl_total, cudaStream_t st);
// The engine's soft-core pair kernel (fixed point, rectangular box).
int launch_soft_rows(const SoftArgs& a, Accumulators& acc, bool energy, bool virial,
                     cudaStream_t st);

// ----------------------------------------------------------------------------
// One axis of the convolution's own FFT passes (snb_fft.cuh): length and
// radices in stage order.
constexpr int kFftMaxN = 256;   // longest axis the passes take
constexpr int kFftMaxStages = 8;
struct FftAxis {
  int N = 0;
  int nst = 0;
  int R[kFftMaxStages] = {};
};

// Particle mesh Ewald (reciprocal part).
struct PME {
  int n = 0;
  int K[3] = {0, 0, 0};
  int nall = 0, nfft = 0;
  float beta = 0.f;
  float cutoff = 10.f;
  float tolerance = 1e-5f;
  int update_interval = 1;
  bool reciprocal = true, excluded = true;
  Cell cell{}, rcell{};
  double volume = 0.0;
  // tiles of the charge grid owned by spread CTAs: edge T, warps per tile
  int T = 8;
  int spread_warps = 2;
  // spread by int64 fixed-point atomics into d_Q64 instead of the tiles
  // (one box; the same grid bit for bit)
  bool spread_atomic = false;
  long long* d_Q64 = nullptr;   // [nall], zero between steps
  // the convolution by the own FFT passes instead of cuFFT (one box)
  bool own_fft = false;
  FftAxis fax[3];
  float2* d_tw[3] = {nullptr, nullptr, nullptr};  // exp(-2 pi i k / K) per axis
  double* d_xpartial = nullptr;  // [xblocks][8] sums of the x pass
  int xblocks = 0;
  // a batch's own passes (snb_fft_reg.cuh): jobs {box, first, count} of the
  // z passes (row pairs), y passes and x pass (lines), and the x jobs'
  // first block per box
  int4* d_zjobs = nullptr;
  int4* d_yjobs = nullptr;
  int4* d_xjobs = nullptr;
  int* d_xjob_begin = nullptr;    // [nsys + 1]
  int nzjobs = 0, nyjobs = 0, nxjobs = 0;
  size_t zsmem = 0;
  int reg_kmax = 0;               // longest axis of the batch's grids
  float* d_bc = nullptr;          // [nfft] a batch's influence BC, spectrum layout
  std::vector<SysGeom> h_sys;     // a batch's boxes (host copy)
  int nt[3] = {0, 0, 0};
  int ntiles = 0;
  float* d_B[3] = {nullptr, nullptr, nullptr};  // |b(k)|^2 per axis
  float* d_Q = nullptr;         // [nall]
  cufftComplex* d_FQ = nullptr;  // [nfft]
  float* d_phi = nullptr;       // [nall]
  int* d_tile_count = nullptr;  // [ntiles]
  int* d_tile_start = nullptr;  // [ntiles + 1]
  int* d_atom_tile = nullptr;   // [n]
  int* d_atom_slot = nullptr;   // [n]
  float4* d_binned = nullptr;   // [n] (frx, fry, frz, q) in tile order
  int* d_binned_u = nullptr;    // [n] packed base point in tile order
  double* d_partial = nullptr;  // [nblocks][8] energy + virial partial sums
  double* d_sums = nullptr;     // [8]: e_recip, virial[6], spare
  int partial_blocks = 0;
  int4* d_src[3] = {nullptr, nullptr, nullptr};  // per-axis source bins of a tile
  float4* d_frq = nullptr;      // [n] (frx, fry, frz, q) in input order
  int* d_upk = nullptr;         // [n] packed base point in input order
  cufftHandle plan_r2c = 0, plan_c2r = 0;
  ScanScratch scan;
  // batch of boxes (bv.nsys > 0): grids of equal size are stored next to
  // each other and transformed by one batched plan per size
  BatchView bv;
  struct FftGroup {
    int K[3];
    int count;
    int grid_begin, spec_begin;
    cufftHandle r2c = 0, c2r = 0;
  };
  std::vector<FftGroup> groups;
  int4* d_spec_blocks = nullptr;   // [spec_blocks] {system, first, end}
  int spec_blocks = 0;
  int* d_sys_block_begin = nullptr;  // [nsys + 1]
  double* d_sys_sums = nullptr;    // [nsys][8]
  int* d_tile_sys = nullptr;       // [ntiles]
  int gather_threads = 256;        // threads per block of the force gather
  // running count of spread tiles whose int32 fixed-point sums could have
  // left the int32 range (an octant bound of 512 charge units or more at a
  // point) and were taken again in int64
  int* d_wide_tiles = nullptr;
};
int pme_init(PME& p, int n, const float* cell6, const float* box_length3,
             float cutoff, float tolerance, int fftx, int ffty, int fftz,
             float grid_spacing, int update_interval, bool reciprocal,
             bool excluded);
// A batch of rectangular boxes (sys[s].cell, rcell, atom ranges set): one
// grid per box by the reference's size rule; fills the PME fields of sys.
// Particle_Mesh::Update_Box: a new rectangular box at the same grid size.
int pme_update_box(PME& p, const float* cell6);
int pme_set_spread_shape(PME& p, int T, int W);
int pme_set_own_fft(PME& p, bool own);
int pme_init_batch(PME& p, int n, std::vector<SysGeom>& sys, float cutoff,
                   float tolerance, float grid_spacing, bool reciprocal, bool excluded);
void pme_free(PME& p);
float get_beta(float cutoff, float tolerance);
int fft_size(float length);

// Reciprocal forces for atoms given as pos (x,y,z,q), accumulated into acc at
// index i (the frame of pos).  Energy/virial sums land in p.d_sums (FP64).
int pme_reciprocal(PME& p, const float4* pos, int n, Accumulators& acc,
                   int accum, bool need_energy, bool need_virial,
                   cudaStream_t st);
// img_off (may be null): sorted-frame offsets subtracted from the pair
// frame's coordinates (pos) only; the PME binning takes crd as given.
int pme_pack_bin(PME& p, int n, const float3* crd, const float* charge, const int* type,
                 const int* perm, float4* pos, int* type_sorted, cudaStream_t st,
                 const float3* img_off = nullptr);
int pme_after_bin(PME& p, int n, Accumulators& acc, int accum, bool need_energy,
                  bool need_virial, cudaStream_t st);
// Virtual atoms for the engine: positions refreshed in crd (caller frame),
// site forces moved onto their sources inside the fixed-point accumulator
// (at map[atom]); status = 1 + the first record of an invalid type-3
// geometry since creation, else 0 (host sync).
int vatom_refresh(snb_vatom* h, float* crd, const Cell& cell, const Cell& rcell,
                  cudaStream_t st);
int vatom_spread_fixed(snb_vatom* h, const float* crd, const Cell& cell, const Cell& rcell,
                       const int* map, Accumulators& acc, cudaStream_t st);
int vatom_status(snb_vatom* h, int* bad, cudaStream_t st);
int vatom_atoms(snb_vatom* h);

// Reads the count of spread tiles redone with int64 sums (host sync).
int pme_wide_tiles(PME& p, int* count, cudaStream_t st);

// Excluded-pair correction (PM_force.cpp:1745-1817).  Caller-frame inputs;
// forces land in acc at map[i] (map = inv_perm, or nullptr for identity).
int launch_excluded(int n, const float3* crd, const float* charge,
                    const Cell& cell, const Cell& rcell, float beta,
                    const int* excl_start, const int* excl_list,
                    const int* excl_numbers, const int* map, Accumulators& acc,
                    int accum, bool energy, bool virial, cudaStream_t st,
                    const BatchView& bv = BatchView());

// ----------------------------------------------------------------------------
// Frame conversion kernels.
// pos[s] = (crd[perm[s]] - img_off[s] (when given), charge[perm[s]]).
int launch_pack(int n, const float3* crd, const float* charge, const int* type,
                const int* perm, float4* pos, int* type_sorted, cudaStream_t st,
                const float3* img_off = nullptr);
// frc[caller i] += acc[map[i]] (converted), optional energies/virials, then
// zero the accumulators.
int launch_unpack(int n, const int* map, Accumulators& acc, int accum,
                  float3* frc, float* atom_energy, float* lj_energy,
                  float* coul_energy, float* atom_virial, bool energy,
                  bool virial, cudaStream_t st);
int launch_zero_acc(Accumulators& acc, int accum, bool energy, bool virial,
                    cudaStream_t st);

}  // namespace snb
