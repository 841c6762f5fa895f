// C ABI (include/sponge_nb.h): module handles that mirror SPONGE's
// NEIGHBOR_LIST, LENNARD_JONES_INFORMATION, Particle_Mesh and the fused
// engine.  Host-side logic only; kernels live in the other .cu files.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sponge_nb.h"
#include "snb_internal.h"

namespace snb {
std::string last_error();
int launch_bonded(int nb, const int* ba, const int* bb, const float* bk,
                  const float* br0, int na, const int* aa, const int* ab,
                  const int* ac, const float* ak, const float* at0,
                  const float3* crd, const Cell& cell, const Cell& rcell,
                  const int* map, Accumulators& acc, long long* e_total,
                  bool energy, cudaStream_t st, const BatchView& bv);
int launch_leap_frog(int n, const int* map, Accumulators& acc, float3* crd,
                     float3* vel, const float* inv_mass, float dt,
                     const float3* old_crd, const Cell& cell, const Cell& rcell,
                     float permit2, int* flags, cudaStream_t st, const BatchView& bv,
                     const PruneCheck& pc);
int launch_totals(int n, Accumulators& acc, long long* isum, const long long* bonded,
                  const double* pme_sums, double lrc_energy, double lrc_virial,
                  double* totals, bool energy, bool virial, bool have_pme,
                  cudaStream_t st);
int launch_add_scalars(float* d_potential, float* d_virial, const double* sums,
                       float lrc_e, float lrc_v, int mode, cudaStream_t st);
int launch_sum_float(int n, const float* x, double* out, cudaStream_t st);
int launch_gather_type(int n, const int* src, const int* atom_local, int* dst,
                       cudaStream_t st);
}  // namespace snb

using namespace snb;

static inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

static Cell cell_of(const snb_boundary& b) { return make_cell(b.cell); }
static Cell rcell_of(const snb_boundary& b) { return make_cell(b.rcell); }

// Tail-correction factor as LENNARD_JONES_INFORMATION::Initial forms it
// (Lennard_Jones_force.cpp:212-237): type histogram, double C6 sum, float
// scaling by -2/3 pi / rc^3 / 6.
static float lrc_factor(const std::vector<int>& type, int n_types,
                        const std::vector<float>& B, float cutoff) {
  std::vector<long long> cnt(n_types, 0);
  for (int t : type) cnt[t] += 1;
  double c6 = 0.0;
  for (int a = 0; a < n_types; ++a) {
    if (!cnt[a]) continue;
    double inner = 0.0;
    for (int b = 0; b < n_types; ++b) {
      if (!cnt[b]) continue;
      inner += (double)cnt[b] * (double)B[lj_pair_index(a, b)];
    }
    c6 += (double)cnt[a] * inner;
  }
  float f = (float)c6;
  f *= -2.0f / 3.0f * 3.1415926535897932f / cutoff / cutoff / cutoff / 6.0f;
  return f;
}

// ============================================================== handles
struct snb_nl {
  NeighborList nl;
  snb_options opt;
};

struct snb_lj {
  LJParams p;
  Accumulators acc;
  int n = 0;
  int accum = kAccumFixed;
  float4* d_pos = nullptr;
  int* d_type_sorted = nullptr;
  float* d_lj_energy = nullptr;  // d_LJ_energy_atom
  double* d_sum = nullptr;
  float h_long_energy = 0.f;
};

struct snb_pme {
  PME p;
  Accumulators acc;
  int accum = kAccumFixed;
  float4* d_pos = nullptr;
};

struct snb_nb14 {
  NB14 p;
  int n = 0;
  int accum = kAccumFixed;
  Accumulators acc;
  long long* d_sums = nullptr;  // [2] {LJ + Coulomb, Coulomb} of the last energy call
};

struct snb_settle {
  Settle s;
};

struct snb_engine {
  snb_options opt;
  int n = 0;
  int accum = kAccumFixed;
  Cell cell{}, rcell{};
  NeighborList nl;
  LJParams lj;
  PME pme;
  Accumulators acc;
  float4* d_pos = nullptr;
  int* d_type_sorted = nullptr;
  float* d_charge = nullptr;
  int* d_excl_start = nullptr;
  int* d_excl_numbers = nullptr;
  int* d_excl_list = nullptr;
  long long* d_isum = nullptr;    // [9]
  long long* d_bonded_e = nullptr;  // [1]
  double* d_totals_scratch = nullptr;
  // bonded terms
  int nb = 0, na = 0;
  int *d_ba = nullptr, *d_bb = nullptr, *d_aa = nullptr, *d_ab = nullptr, *d_ac = nullptr;
  float *d_bk = nullptr, *d_br0 = nullptr, *d_ak = nullptr, *d_at0 = nullptr;
  // graph of one MD step
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraph_t graph = nullptr;
  float* g_crd = nullptr;
  float* g_vel = nullptr;
  const float* g_invm = nullptr;
  float g_dt = 0.f;
  cudaStream_t g_stream = nullptr;
  bool g_vel_wait = false;  // the graph waits on ev_vel_in before the update
  // host-buffer steps: the velocities cross the link on `io` while the
  // forces are computed; the update waits on ev_vel_in (recorded after that
  // copy and the velocity snapshot)
  cudaStream_t io = nullptr;
  cudaEvent_t ev_crd_in = nullptr, ev_vel_in = nullptr;
  bool vel_wait = false;      // steps of this call wait on ev_vel_in
  bool vel_snapped = false;   // the first chunk's velocity snapshot is taken
  // a batch of independent boxes (nsys > 0)
  int nsys = 0;
  std::vector<SysGeom> h_sys;
  SysGeom* d_sys = nullptr;
  int* d_sys_of = nullptr;
  int* d_cell_sys = nullptr;          // [ncell] system of each neighbor cell
  unsigned char* d_box_need = nullptr;  // [nsys] systems whose list is rebuilt
  BatchView bv;
  double lrc_energy = 0.0;   // tail energy summed over the boxes
  double lrc_virial = 0.0;   // tail virial (diagonal) summed over the boxes
  double lrc_energy_lj = 0.0, lrc_virial_lj = 0.0;  // the plain LJ module's
  snb_lj_soft* soft = nullptr;  // soft-core pair terms in place of plain LJ
  snb_nb14* nb14 = nullptr;     // 1-4 terms beside the excluded correction
  snb_settle* settle = nullptr;  // rigid triangles / pairs after the coordinate update
  snb_vatom* vatom = nullptr;    // massless sites: forces moved, positions refreshed
  long long* d_nb14_sums = nullptr;  // [2]
  double* d_kin = nullptr;           // [6] scratch of the pressure call
  // launch shapes picked by snb_engine_autotune
  int pair_unroll = 4;
  int pair_blocks_per_sm = 0;
  int pair_warps = 16;  // measured on the 100k box: 4 candidates x 16 rows is the fastest
  bool pair_stash = false;
  // pruned rows (single box, plain LJ rows): between prune passes the pair
  // kernel scans only the entries within cutoff + prune_margin (0: off).
  // d_prune = {pass this step, an atom moved more than half the margin since
  // the last pass, list generation at the last pass, passes so far}
  float prune_margin = 0.f;
  int* d_prune = nullptr;
  cudaStream_t side = nullptr;  // captures the conditional rebuild body
  // second branch of a step: excluded correction, bonded terms and PME run
  // on `branch` while the pair kernel runs on the step's stream; both add
  // into the same fixed-point accumulator (integer adds commute)
  cudaStream_t branch = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // third branch: the excluded correction and bonded terms, beside PME
  cudaStream_t branch2 = nullptr;
  cudaEvent_t ev_join2 = nullptr;
  int body_kernels = 0;         // kernel nodes inside the rebuild body
  // recovery snapshot for neighbor-list overflow
  float* d_snap_crd = nullptr;
  float* d_snap_vel = nullptr;
  long long steps_done = 0;
  // per-phase CUDA events (profiling pass only)
  bool prof_on = false;
  cudaEvent_t prof_ev[8] = {};
  double prof_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

static void prof_mark(snb_engine* e, int k, cudaStream_t st) {
  if (e->prof_on) cudaEventRecord(e->prof_ev[k], st);
}

// The step runs a prune pass when an atom moved more than half the margin
// since the last one, or when the list was rebuilt since (one thread; runs
// after the list update and before the pair kernel).
__global__ void k_prune_decide(int* prune, const int* nl_flags) {
  const int gen = nl_flags[kFlagGeneration];
  const int pass = (prune[1] != 0 || gen != prune[2]) ? 1 : 0;
  prune[0] = pass;
  prune[1] = 0;
  prune[2] = gen;
  prune[3] += pass;
}

constexpr float kDefaultPruneMargin = 0.8f;  // A
constexpr int kPruneMinAtoms = 20000;        // single boxes below: full rows

static bool engine_prunes(const snb_engine* e) {
  return e->prune_margin > 0.f && e->d_prune && !(e->nl.clusters && !e->soft);
}

// The check that follows an update: displacements above half the margin
// (less a relative 1e-3 for the rounding of the distances) force a pass.
static PruneCheck engine_prune_check(const snb_engine* e) {
  PruneCheck pc;
  if (!engine_prunes(e)) return pc;
  const float h = 0.5f * e->prune_margin * (1.0f - 1e-3f);
  pc.ref = e->nl.d_prune_ref;
  pc.permit2 = h * h;
  pc.flag = e->d_prune + 1;
  return pc;
}

// The next prune-capable pair launch runs a full pass (its kept rows are
// stale: coordinates from outside the MD loop, or another pair kernel ran).
static int engine_prune_invalidate(snb_engine* e, cudaStream_t st) {
  if (e->d_prune) SNB_CUDA_TRY(cudaMemsetAsync(e->d_prune + 1, 1, 1, st));
  return kOk;
}

// ============================================================ options
extern "C" int snb_version(void) { return SNB_VERSION; }

extern "C" const char* snb_last_error(void) {
  static thread_local std::string s;
  s = last_error();
  return s.c_str();
}

extern "C" void snb_options_default(snb_options* o) {
  memset(o, 0, sizeof(*o));
  o->cutoff = 10.0f;
  o->skin = 2.0f;
  o->nl_refresh_interval = 0;
  o->nl_skin_permit = 0.5f;
  o->nl_max_neighbor_numbers = 1200;
  o->nl_max_atom_in_grid_numbers = 150;
  o->nl_max_ghost_in_grid_numbers = 150;
  o->nl_check_overflow_interval = 150;
  o->nl_throw_error_when_overflow = 0;
  o->pm_fftx = o->pm_ffty = o->pm_fftz = -1;
  o->pm_grid_spacing = 1.0f;
  o->pm_direct_tolerance = 0.00001f;
  o->pme_update_interval = 1;
  o->pme_calculate_reciprocal_part = 1;
  o->pme_calculate_excluded_part = 1;
  o->lambda_lj = 0.0f;
  o->soft_core_alpha = 0.5f;
  o->soft_core_powfer = 1.0f;
  o->soft_core_sigma = 3.0f;
  o->soft_core_sigma_min = 0.0f;
  o->accumulation = SNB_ACCUM_FIXED64;
  o->dom_dec_update_interval = 100;
}

static bool parse_bool(const char* v) {
  std::string s(v);
  for (auto& c : s) c = (char)tolower(c);
  return s == "1" || s == "true" || s == "yes" || s == "on";
}

extern "C" int snb_options_set(snb_options* o, const char* key, const char* value) {
  if (!o || !key || !value) return fail(kBadInput, "options_set: null argument");
  std::string k(key);
  auto F = [&]() { return (float)atof(value); };
  auto I = [&]() { return atoi(value); };
  if (k == "cutoff") o->cutoff = F();
  else if (k == "skin") o->skin = F();
  else if (k == "neighbor_list_refresh_interval") o->nl_refresh_interval = I();
  else if (k == "neighbor_list_skin_permit") o->nl_skin_permit = F();
  else if (k == "neighbor_list_max_neighbor_numbers") o->nl_max_neighbor_numbers = I();
  else if (k == "neighbor_list_max_atom_in_grid_numbers") o->nl_max_atom_in_grid_numbers = I();
  else if (k == "neighbor_list_max_ghost_in_grid_numbers") o->nl_max_ghost_in_grid_numbers = I();
  else if (k == "neighbor_list_check_overflow_interval") o->nl_check_overflow_interval = I();
  else if (k == "neighbor_list_throw_error_when_overflow") o->nl_throw_error_when_overflow = parse_bool(value);
  else if (k == "PM_fftx") o->pm_fftx = I();
  else if (k == "PM_ffty") o->pm_ffty = I();
  else if (k == "PM_fftz") o->pm_fftz = I();
  else if (k == "PM_grid_spacing") o->pm_grid_spacing = F();
  else if (k == "PM_Direct_Tolerance") o->pm_direct_tolerance = F();
  else if (k == "PME_update_interval") o->pme_update_interval = I();
  else if (k == "PME_calculate_reciprocal_part") o->pme_calculate_reciprocal_part = parse_bool(value);
  else if (k == "PME_calculate_excluded_part") o->pme_calculate_excluded_part = parse_bool(value);
  else if (k == "lambda_lj") o->lambda_lj = F();
  else if (k == "soft_core_alpha") o->soft_core_alpha = F();
  else if (k == "soft_core_powfer") o->soft_core_powfer = F();
  else if (k == "soft_core_sigma") o->soft_core_sigma = F();
  else if (k == "soft_core_sigma_min") o->soft_core_sigma_min = F();
  else if (k == "DOM_DEC_update_interval") o->dom_dec_update_interval = I();
  else if (k == "accumulation") {
    std::string v(value);
    if (v == "fixed64" || v == "fixed") o->accumulation = SNB_ACCUM_FIXED64;
    else if (v == "float") o->accumulation = SNB_ACCUM_FLOAT;
    else return fail(kBadInput, "accumulation must be fixed64 or float");
  } else {
    return fail(kBadInput, "unknown key " + k);
  }
  return kOk;
}

static snb_options opts_or_default(const snb_options* o) {
  snb_options d;
  if (o) return *o;
  snb_options_default(&d);
  return d;
}

// ========================================================= NEIGHBOR_LIST
extern "C" int snb_nl_create(const snb_options* opt, int atom_numbers, float cutoff,
                             float skin, snb_boundary boundary, snb_nl** out) {
  if (!out) return fail(kBadInput, "nl_create: null out");
  *out = nullptr;
  if (boundary.policy != 1)
    return fail(kNotSupported, "neighbor list: periodic boundary required");
  snb_nl* h = new snb_nl();
  h->opt = opts_or_default(opt);
  int rc = nl_init(h->nl, atom_numbers, cutoff, skin, boundary.cell,
                   h->opt.nl_refresh_interval, h->opt.nl_skin_permit,
                   h->opt.nl_max_neighbor_numbers, 0);
  if (rc) {
    nl_free(h->nl);
    delete h;
    return rc;
  }
  *out = h;
  return kOk;
}

extern "C" int snb_nl_update(snb_nl* h, const int* atom_local, int local_atom_numbers,
                             int ghost_numbers, const float* crd, snb_boundary boundary,
                             int step, int update, const int* excluded_list_start,
                             const int* excluded_list, const int* excluded_numbers,
                             void* stream) {
  if (!h) return fail(kBadInput, "nl_update: null handle");
  if (local_atom_numbers <= 0 && ghost_numbers <= 0) return kOk;
  if (ghost_numbers != 0)
    return fail(kNotSupported, "nl_update: ghost atoms (domain decomposition) are "
                               "not supported");
  if (local_atom_numbers != h->nl.n)
    return fail(kBadInput, "nl_update: local_atom_numbers differs from Initial");
  return nl_update(h->nl, crd, atom_local, boundary.cell, step,
                   update == SNB_FORCED_UPDATE, excluded_list_start, excluded_list,
                   excluded_numbers, S(stream));
}

extern "C" int snb_nl_check_overflow(snb_nl* h, int* regrown, void* stream) {
  if (!h) return fail(kBadInput, "nl_check_overflow: null handle");
  bool r = false;
  int rc = nl_check_overflow(h->nl, &r, S(stream));
  if (regrown) *regrown = r ? 1 : 0;
  if (!rc && r && h->opt.nl_throw_error_when_overflow)
    return fail(kOverflow, "NEIGHBOR_LIST::Check_Overflow: overflow occured in "
                           "neighbor searching");
  return rc;
}

extern "C" int snb_nl_pair_count(snb_nl* h, long long* count, void* stream) {
  if (!h || !count) return fail(kBadInput, "nl_pair_count: null argument");
  return nl_total_pairs(h->nl, count, S(stream));
}

extern "C" int snb_nl_export_pairs(snb_nl* h, int* d_pi, int* d_pj, long long cap,
                                   long long* count, void* stream) {
  if (!h || !count) return fail(kBadInput, "nl_export_pairs: null argument");
  int rc = nl_export_pairs(h->nl, d_pi, d_pj, cap, count, S(stream));
  if (rc) return rc;
  SNB_CUDA_TRY(cudaStreamSynchronize(S(stream)));
  return kOk;
}

extern "C" int snb_nl_export_atom_groups(snb_nl* h, void* d_nl, int* d_slab, int maxn,
                                         void* stream) {
  if (!h || !d_nl || !d_slab || maxn <= 0)
    return fail(kBadInput, "nl_export_atom_groups: bad argument");
  return nl_export_atom_groups(h->nl, d_nl, d_slab, maxn, S(stream));
}

extern "C" int snb_nl_destroy(snb_nl* h) {
  if (!h) return kOk;
  nl_free(h->nl);
  delete h;
  return kOk;
}

// ============================================= LENNARD_JONES_INFORMATION
extern "C" int snb_lj_create(const snb_options* opt, int atom_numbers,
                             int atom_type_numbers, const int* h_type, const float* h_A,
                             const float* h_B, float cutoff, snb_lj** out) {
  if (!out) return fail(kBadInput, "lj_create: null out");
  *out = nullptr;
  if (atom_numbers <= 0 || atom_type_numbers <= 0 || !h_type || !h_A || !h_B)
    return fail(kBadInput, "lj_create: bad argument");
  snb_options o = opts_or_default(opt);
  snb_lj* h = new snb_lj();
  h->n = atom_numbers;
  h->accum = o.accumulation;
  LJParams& p = h->p;
  p.n_types = atom_type_numbers;
  p.n_pairs = atom_type_numbers * (atom_type_numbers + 1) / 2;
  p.h_type.assign(h_type, h_type + atom_numbers);
  for (int t : p.h_type)
    if (t < 0 || t >= atom_type_numbers) {
      delete h;
      return fail(kBadInput, "lj_create: LJ type out of range");
    }
  p.h_A.assign(h_A, h_A + p.n_pairs);
  p.h_B.assign(h_B, h_B + p.n_pairs);
  p.cutoff = cutoff;
  p.long_range_factor = lrc_factor(p.h_type, p.n_types, p.h_B, cutoff);
  SNB_CUDA_TRY(cudaMalloc(&p.d_A, sizeof(float) * p.n_pairs));
  SNB_CUDA_TRY(cudaMalloc(&p.d_B, sizeof(float) * p.n_pairs));
  SNB_CUDA_TRY(cudaMemcpy(p.d_A, h_A, sizeof(float) * p.n_pairs, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMemcpy(p.d_B, h_B, sizeof(float) * p.n_pairs, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&p.d_type, sizeof(int) * atom_numbers));
  SNB_CUDA_TRY(cudaMemcpy(p.d_type, h_type, sizeof(int) * atom_numbers,
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&p.d_type_local, sizeof(int) * atom_numbers));
  SNB_CUDA_TRY(cudaMemcpy(p.d_type_local, h_type, sizeof(int) * atom_numbers,
                          cudaMemcpyHostToDevice));
  int rc = acc_init(h->acc, atom_numbers);
  if (rc) return rc;
  SNB_CUDA_TRY(cudaMalloc(&h->d_pos, sizeof(float4) * atom_numbers));
  SNB_CUDA_TRY(cudaMalloc(&h->d_type_sorted, sizeof(int) * atom_numbers));
  SNB_CUDA_TRY(cudaMalloc(&h->d_lj_energy, sizeof(float) * atom_numbers));
  SNB_CUDA_TRY(cudaMemset(h->d_lj_energy, 0, sizeof(float) * atom_numbers));
  SNB_CUDA_TRY(cudaMalloc(&h->d_sum, sizeof(double)));
  *out = h;
  return kOk;
}

extern "C" int snb_lj_get_local(snb_lj* h, const int* atom_local, int local_n,
                                int ghost_n, void* stream) {
  if (!h) return fail(kBadInput, "lj_get_local: null handle");
  if (ghost_n != 0) return fail(kNotSupported, "lj_get_local: ghost atoms");
  if (local_n != h->n) return fail(kBadInput, "lj_get_local: atom count");
  return launch_gather_type(local_n, h->p.d_type, atom_local, h->p.d_type_local,
                            S(stream));
}

// Direct-space pairs of the LJ module over the list: solvent_mode 0 every
// pair, 1 all but the solvent-solvent ones, 2 only those (see PairArgs).
static int lj_direct(snb_lj* h, snb_nl* nl, const float* crd, const float* charge,
                     float* frc, snb_boundary boundary, float pme_beta, bool en, bool vi,
                     float* atom_energy, float* atom_virial, float* atom_direct_pme_energy,
                     int solvent_mode, int solvent_begin, cudaStream_t st) {
  int rc = launch_pack(h->n, reinterpret_cast<const float3*>(crd), charge,
                       h->p.d_type_local, nl->nl.d_perm, h->d_pos, h->d_type_sorted, st);
  if (rc) return rc;
  PairArgs a;
  a.n = h->n;
  a.pos = h->d_pos;
  a.type = h->d_type_sorted;
  a.global = nl->nl.d_global;
  a.row_start = nl->nl.d_row_start;
  a.row_count = nl->nl.d_row_count;
  a.cols = nl->nl.d_cols;
  a.nl_flags = nl->nl.d_flags;
  a.A = h->p.d_A;
  a.B = h->p.d_B;
  a.n_types = h->p.n_types;
  a.cell = cell_of(boundary);
  a.rcell = rcell_of(boundary);
  a.cutoff2 = h->p.cutoff * h->p.cutoff;
  a.beta = pme_beta;
  a.solvent_mode = solvent_mode;
  a.solvent_begin = solvent_begin;
  bool ortho = a.cell.a21 == 0.f && a.cell.a31 == 0.f && a.cell.a32 == 0.f;
  rc = launch_pair(a, h->acc, h->accum, en, vi, ortho, st);
  if (rc) return rc;
  return launch_unpack(h->n, nl->nl.d_inv_perm, h->acc, h->accum,
                       reinterpret_cast<float3*>(frc), en ? atom_energy : nullptr,
                       en ? h->d_lj_energy : nullptr,
                       en ? atom_direct_pme_energy : nullptr,
                       vi ? atom_virial : nullptr, en, vi, st);
}

extern "C" int snb_lj_pme_direct_force(snb_lj* h, int atom_numbers, int local_n,
                                       int solvent_n, int ghost_n, const float* crd,
                                       const float* charge, float* frc,
                                       snb_boundary boundary, snb_nl* nl,
                                       float pme_beta, int need_atom_energy,
                                       float* atom_energy, int need_virial,
                                       float* atom_virial,
                                       float* atom_direct_pme_energy, void* stream) {
  if (!h || !nl) return fail(kBadInput, "lj_pme_direct_force: null handle");
  cudaStream_t st = S(stream);
  if (need_atom_energy) {
    if (atom_direct_pme_energy)
      SNB_CUDA_TRY(cudaMemsetAsync(atom_direct_pme_energy, 0, sizeof(float) * h->n, st));
    SNB_CUDA_TRY(cudaMemsetAsync(h->d_lj_energy, 0, sizeof(float) * h->n, st));
  }
  if (atom_numbers == 0 || local_n == 0) return kOk;
  if (ghost_n != 0) return fail(kNotSupported, "lj_pme_direct_force: ghost atoms");
  if (local_n != h->n || nl->nl.n != h->n)
    return fail(kBadInput, "lj_pme_direct_force: atom count mismatch");
  if (solvent_n < 0 || solvent_n > local_n)
    return fail(kBadInput, "lj_pme_direct_force: solvent_numbers out of range");
  if (solvent_n > 0 && nl->nl.bv.nsys > 0)
    return fail(kNotSupported, "lj_pme_direct_force: solvent split of a batch");
  return lj_direct(h, nl, crd, charge, frc, boundary, pme_beta, need_atom_energy != 0,
                   need_virial != 0, atom_energy, atom_virial, atom_direct_pme_energy,
                   solvent_n > 0 ? 1 : 0, local_n - solvent_n, st);
}

extern "C" int snb_solvent_lj_pme_direct_force(snb_lj* h, snb_nl* nl, int atom_numbers,
                                               int solvent_numbers, const float* crd,
                                               const float* charge, float* frc,
                                               snb_boundary boundary, float pme_beta,
                                               int need_atom_energy, float* atom_energy,
                                               int need_virial, float* atom_virial,
                                               float* atom_direct_pme_energy,
                                               void* stream) {
  if (!h || !nl) return fail(kBadInput, "solvent_lj_pme_direct_force: null handle");
  if (atom_numbers != h->n || nl->nl.n != h->n)
    return fail(kBadInput, "solvent_lj_pme_direct_force: atom count mismatch");
  if (solvent_numbers < 0 || solvent_numbers > atom_numbers)
    return fail(kBadInput, "solvent_lj_pme_direct_force: solvent_numbers out of range");
  if (nl->nl.bv.nsys > 0)
    return fail(kNotSupported, "solvent_lj_pme_direct_force: batch lists");
  if (solvent_numbers == 0) return kOk;
  return lj_direct(h, nl, crd, charge, frc, boundary, pme_beta, need_atom_energy != 0,
                   need_virial != 0, atom_energy, atom_virial, atom_direct_pme_energy, 2,
                   atom_numbers - solvent_numbers, S(stream));
}

extern "C" int snb_lj_long_range_correction(snb_lj* h, int need_pressure,
                                            float* d_virial, int need_potential,
                                            float* d_potential, float volume,
                                            void* stream) {
  if (!h) return fail(kBadInput, "lj_long_range_correction: null handle");
  float e = h->p.long_range_factor / volume;
  float v = 2 * h->p.long_range_factor / volume;
  if (need_potential) h->h_long_energy = e;
  return launch_add_scalars(need_potential ? d_potential : nullptr,
                            need_pressure ? d_virial : nullptr, nullptr, e, v, 1,
                            S(stream));
}

extern "C" int snb_lj_energy_sum(snb_lj* h, float* out, void* stream) {
  if (!h || !out) return fail(kBadInput, "lj_energy_sum: null argument");
  int rc = launch_sum_float(h->n, h->d_lj_energy, h->d_sum, S(stream));
  if (rc) return rc;
  double v = 0;
  SNB_CUDA_TRY(cudaMemcpyAsync(&v, h->d_sum, sizeof(double), cudaMemcpyDeviceToHost,
                               S(stream)));
  SNB_CUDA_TRY(cudaStreamSynchronize(S(stream)));
  *out = (float)v;
  return kOk;
}

extern "C" float snb_lj_long_range_factor(snb_lj* h) {
  return h ? h->p.long_range_factor : 0.f;
}

extern "C" int snb_lj_destroy(snb_lj* h) {
  if (!h) return kOk;
  cudaFree(h->p.d_A);
  cudaFree(h->p.d_B);
  cudaFree(h->p.d_type);
  cudaFree(h->p.d_type_local);
  acc_free(h->acc);
  cudaFree(h->d_pos);
  cudaFree(h->d_type_sorted);
  cudaFree(h->d_lj_energy);
  cudaFree(h->d_sum);
  delete h;
  return kOk;
}

// ========================================================== LJ_SOFT_CORE
struct snb_lj_soft {
  int n = 0;
  int accum = kAccumFixed;
  int nA = 0, nB = 0;
  float *d_AA = nullptr, *d_AB = nullptr, *d_BA = nullptr, *d_BB = nullptr;
  int2* d_par = nullptr;         // caller frame {typeA | typeB << 16, mask}
  int2* d_par_local = nullptr;   // after Get_Local
  int2* d_par_sorted = nullptr;
  float4* d_pos = nullptr;
  float* d_dq_sorted = nullptr;
  float* d_lj_energy = nullptr;  // d_LJ_energy_atom
  float* d_inter = nullptr;      // d_LJ_energy_atom_intersys
  float* d_intra = nullptr;      // d_LJ_energy_atom_intrasys
  long long* d_dudl = nullptr;   // [2] fixed point: LJ, direct Coulomb
  Accumulators acc;
  float lambda = 0.f, alpha = 0.5f, p = 1.f, sigma6 = 729.f, sigma6_min = 0.f;
  float cutoff = 10.f;
  float lrc = 0.f, lrc_ti = 0.f;
  float lrc_energy = 0.f;        // h_LJ_long_energy of the last tail call
  double* d_sums = nullptr;      // [3] scratch for Step_Print sums
};

__global__ void k_pack_soft(int n, const int* __restrict__ perm,
                            const int2* __restrict__ par, const float* __restrict__ dq,
                            int2* __restrict__ par_sorted, float* __restrict__ dq_sorted) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i = perm[s];
  par_sorted[s] = par[i];
  if (dq_sorted) dq_sorted[s] = dq ? dq[i] : 0.f;
}

__global__ void k_gather_par(int n, const int2* __restrict__ src,
                             const int* __restrict__ atom_local, int2* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[atom_local ? atom_local[i] : i];
}

// inter/intra LJ energies (sorted accumulators) -> caller-frame arrays
__global__ void k_unpack_aux(int n, const int* __restrict__ map, Accumulators a,
                             float* inter, float* intra, int accum) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = map[i];
  const int N = a.n;
  if (accum == kAccumFixed) {
    inter[i] += (float)((double)a.d_eaux[s] * kEnergyScaleInv);
    intra[i] += (float)((double)a.d_eaux[N + s] * kEnergyScaleInv);
    a.d_eaux[s] = 0;
    a.d_eaux[N + s] = 0;
  } else {
    inter[i] += a.d_feaux[s];
    intra[i] += a.d_feaux[N + s];
    a.d_feaux[s] = 0.f;
    a.d_feaux[N + s] = 0.f;
  }
}

// Tail correction of LJ_SOFT_CORE::Initial (LJ_soft_core.cpp:640-672): the
// O(N^2) Total_C6_Get / Total_C6_B_A_Get sums depend only on the type
// histograms of each end state, so they are formed from those.
static void soft_lrc(const std::vector<int>& tA, const std::vector<int>& tB, int nA,
                     int nB, const float* AB, const float* BB, float lambda,
                     float cutoff, float* lrc, float* lrc_ti) {
  std::vector<double> cA(nA, 0.0), cB(nB, 0.0);
  for (int t : tA) cA[t] += 1;
  for (int t : tB) cB[t] += 1;
  double sA = 0.0, sB = 0.0;
  for (int a = 0; a < nA; ++a)
    for (int b = 0; b < nA; ++b) sA += cA[a] * cA[b] * (double)AB[lj_pair_index(a, b)];
  for (int a = 0; a < nB; ++a)
    for (int b = 0; b < nB; ++b) sB += cB[a] * cB[b] * (double)BB[lj_pair_index(a, b)];
  float f = (float)((double)(1.0f - lambda) * sA + (double)lambda * sB);
  float fti = (float)(sB - sA);
  const float k = -2.0f / 3.0f * 3.1415926535897932f / cutoff / cutoff / cutoff / 6.0f;
  *lrc = f * k;
  *lrc_ti = fti * k;
}

extern "C" int snb_lj_soft_create(const snb_options* opt, int n, int nA, int nB,
                                  const int* h_tA, const int* h_tB, const float* h_AA,
                                  const float* h_AB, const float* h_BA,
                                  const float* h_BB, const int* h_mask, float cutoff,
                                  snb_lj_soft** out) {
  if (!out) return fail(kBadInput, "lj_soft_create: null out");
  *out = nullptr;
  if (n <= 0 || nA <= 0 || nB <= 0 || !h_tA || !h_tB || !h_AA || !h_AB || !h_BA || !h_BB)
    return fail(kBadInput, "lj_soft_create: bad argument");
  if (nA > 0xffff || nB > 0x7fff) return fail(kBadInput, "lj_soft_create: too many types");
  snb_options o = opts_or_default(opt);
  snb_lj_soft* h = new snb_lj_soft();
  h->n = n;
  h->accum = o.accumulation;
  h->nA = nA;
  h->nB = nB;
  h->lambda = o.lambda_lj;
  h->alpha = o.soft_core_alpha;
  h->p = o.soft_core_powfer;
  h->sigma6 = powf(o.soft_core_sigma, 6);
  h->sigma6_min = powf(o.soft_core_sigma_min, 6);
  h->cutoff = cutoff;
  int pA = nA * (nA + 1) / 2, pB = nB * (nB + 1) / 2;
  std::vector<int> tA(h_tA, h_tA + n), tB(h_tB, h_tB + n);
  std::vector<int2> par(n);
  for (int i = 0; i < n; ++i) {
    if (tA[i] < 0 || tA[i] >= nA || tB[i] < 0 || tB[i] >= nB) {
      delete h;
      return fail(kBadInput, "lj_soft_create: LJ type out of range");
    }
    par[i] = make_int2(tA[i] | (tB[i] << 16), h_mask ? h_mask[i] : 0);
  }
  soft_lrc(tA, tB, nA, nB, h_AB, h_BB, h->lambda, cutoff, &h->lrc, &h->lrc_ti);
  auto up = [](float** d, const float* src, int m) -> int {
    SNB_CUDA_TRY(cudaMalloc(d, sizeof(float) * m));
    SNB_CUDA_TRY(cudaMemcpy(*d, src, sizeof(float) * m, cudaMemcpyHostToDevice));
    return kOk;
  };
  if (up(&h->d_AA, h_AA, pA) || up(&h->d_AB, h_AB, pA) || up(&h->d_BA, h_BA, pB) ||
      up(&h->d_BB, h_BB, pB))
    return fail(kCudaError, "lj_soft_create: upload failed");
  SNB_CUDA_TRY(cudaMalloc(&h->d_par, sizeof(int2) * n));
  SNB_CUDA_TRY(cudaMemcpy(h->d_par, par.data(), sizeof(int2) * n, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&h->d_par_local, sizeof(int2) * n));
  SNB_CUDA_TRY(cudaMemcpy(h->d_par_local, par.data(), sizeof(int2) * n,
                          cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&h->d_par_sorted, sizeof(int2) * n));
  SNB_CUDA_TRY(cudaMalloc(&h->d_pos, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&h->d_dq_sorted, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMalloc(&h->d_lj_energy, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMalloc(&h->d_inter, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMalloc(&h->d_intra, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMemset(h->d_lj_energy, 0, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMemset(h->d_inter, 0, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMemset(h->d_intra, 0, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMalloc(&h->d_dudl, sizeof(long long) * 2));
  int rc = acc_init(h->acc, n);
  if (rc) return rc;
  *out = h;
  return kOk;
}

static SoftArgs soft_args(snb_lj_soft* h, snb_nl* nl, const snb_boundary& b, float beta) {
  SoftArgs a;
  a.n = h->n;
  a.pos = h->d_pos;
  a.par = h->d_par_sorted;
  a.dq = h->d_dq_sorted;
  a.global = nl->nl.d_global;
  a.row_start = nl->nl.d_row_start;
  a.row_count = nl->nl.d_row_count;
  a.cols = nl->nl.d_cols;
  a.nl_flags = nl->nl.d_flags;
  a.AA = h->d_AA;
  a.AB = h->d_AB;
  a.BA = h->d_BA;
  a.BB = h->d_BB;
  a.n_types_A = h->nA;
  a.n_types_B = h->nB;
  a.cell = cell_of(b);
  a.rcell = rcell_of(b);
  a.cutoff2 = h->cutoff * h->cutoff;
  a.beta = beta;
  a.lambda = h->lambda;
  a.alpha = h->alpha;
  a.p = h->p;
  a.sigma6 = h->sigma6;
  a.sigma6_min = h->sigma6_min;
  return a;
}

extern "C" int snb_lj_soft_pme_direct_force(snb_lj_soft* h, int atom_numbers, int local_n,
                                            int ghost_n, const float* crd,
                                            const float* charge, const float* charge_B_A,
                                            float* frc, snb_boundary boundary,
                                            snb_nl* nl, float pme_beta,
                                            int need_atom_energy, float* atom_energy,
                                            int need_virial, float* atom_virial,
                                            float* atom_direct_pme_energy, void* stream) {
  if (!h || !nl) return fail(kBadInput, "lj_soft_pme_direct_force: null handle");
  cudaStream_t st = S(stream);
  if (need_atom_energy) {
    SNB_CUDA_TRY(cudaMemsetAsync(h->d_lj_energy, 0, sizeof(float) * h->n, st));
    SNB_CUDA_TRY(cudaMemsetAsync(h->d_inter, 0, sizeof(float) * h->n, st));
    SNB_CUDA_TRY(cudaMemsetAsync(h->d_intra, 0, sizeof(float) * h->n, st));
    if (atom_direct_pme_energy)
      SNB_CUDA_TRY(cudaMemsetAsync(atom_direct_pme_energy, 0, sizeof(float) * h->n, st));
  }
  if (atom_numbers == 0 || local_n == 0) return kOk;
  if (ghost_n != 0) return fail(kNotSupported, "lj_soft: ghost atoms");
  if (local_n != h->n || nl->nl.n != h->n) return fail(kBadInput, "lj_soft: atom count");
  int rc = launch_pack(h->n, reinterpret_cast<const float3*>(crd), charge, nullptr,
                       nl->nl.d_perm, h->d_pos, nullptr, st);
  if (rc) return rc;
  k_pack_soft<<<ceil_div(h->n, 256), 256, 0, st>>>(h->n, nl->nl.d_perm, h->d_par_local,
                                                  charge_B_A, h->d_par_sorted,
                                                  h->d_dq_sorted);
  SoftArgs a = soft_args(h, nl, boundary, pme_beta);
  bool en = need_atom_energy != 0, vi = need_virial != 0;
  rc = launch_soft(a, h->acc, h->accum, en, vi, false, nullptr, st);
  if (rc) return rc;
  if (en)
    k_unpack_aux<<<ceil_div(h->n, 256), 256, 0, st>>>(h->n, nl->nl.d_inv_perm, h->acc,
                                                     h->d_inter, h->d_intra, h->accum);
  return launch_unpack(h->n, nl->nl.d_inv_perm, h->acc, h->accum,
                       reinterpret_cast<float3*>(frc), en ? atom_energy : nullptr,
                       en ? h->d_lj_energy : nullptr, en ? atom_direct_pme_energy : nullptr,
                       vi ? atom_virial : nullptr, en, vi, st);
}

extern "C" int snb_lj_soft_dh_dlambda(snb_lj_soft* h, const float* crd,
                                      const float* charge, const float* charge_B_A,
                                      snb_boundary boundary, snb_nl* nl, float pme_beta,
                                      int charge_perturbated, double* out, void* stream) {
  (void)charge_perturbated;
  if (!h || !nl || !out) return fail(kBadInput, "lj_soft_dh_dlambda: bad argument");
  cudaStream_t st = S(stream);
  int rc = launch_pack(h->n, reinterpret_cast<const float3*>(crd), charge, nullptr,
                       nl->nl.d_perm, h->d_pos, nullptr, st);
  if (rc) return rc;
  k_pack_soft<<<ceil_div(h->n, 256), 256, 0, st>>>(h->n, nl->nl.d_perm, h->d_par_local,
                                                  charge_B_A, h->d_par_sorted,
                                                  h->d_dq_sorted);
  SNB_CUDA_TRY(cudaMemsetAsync(h->d_dudl, 0, sizeof(long long) * 2, st));
  SoftArgs a = soft_args(h, nl, boundary, pme_beta);
  rc = launch_soft(a, h->acc, h->accum, false, false, true, h->d_dudl, st);
  if (rc) return rc;
  long long v[2];
  SNB_CUDA_TRY(cudaMemcpyAsync(v, h->d_dudl, sizeof(v), cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  // the reference returns the LJ part plus the tail term (LJ_soft_core.cpp:883-885)
  double vol = (double)boundary.cell[0] * boundary.cell[2] * boundary.cell[5];
  *out = (double)v[0] * kEnergyScaleInv + (double)h->lrc_ti / vol;
  return kOk;
}

extern "C" int snb_lj_soft_long_range_correction(snb_lj_soft* h, int need_pressure,
                                                 float* d_virial, int need_potential,
                                                 float* d_potential, float volume,
                                                 void* stream) {
  if (!h) return fail(kBadInput, "lj_soft_long_range_correction: null handle");
  if (need_potential > 0) h->lrc_energy = h->lrc / volume;
  return launch_add_scalars(need_potential > 0 ? d_potential : nullptr,
                            need_pressure > 0 ? d_virial : nullptr, nullptr,
                            h->lrc / volume, 2 * h->lrc / volume, 1, S(stream));
}

extern "C" int snb_lj_soft_energy_sums(snb_lj_soft* h, float* out, void* stream) {
  if (!h || !out) return fail(kBadInput, "lj_soft_energy_sums: null argument");
  cudaStream_t st = S(stream);
  if (!h->d_sums) SNB_CUDA_TRY(cudaMalloc(&h->d_sums, sizeof(double) * 3));
  int rc = launch_sum_float(h->n, h->d_lj_energy, h->d_sums, st);
  if (!rc) rc = launch_sum_float(h->n, h->d_inter, h->d_sums + 1, st);
  if (!rc) rc = launch_sum_float(h->n, h->d_intra, h->d_sums + 2, st);
  if (rc) return rc;
  double v[3];
  SNB_CUDA_TRY(cudaMemcpyAsync(v, h->d_sums, sizeof(v), cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  out[0] = (float)v[0];
  out[1] = (float)v[1];
  out[2] = (float)v[2];
  out[3] = h->lrc_energy;
  return kOk;
}

extern "C" int snb_lj_soft_destroy(snb_lj_soft* h) {
  if (!h) return kOk;
  for (void* p : {(void*)h->d_AA, (void*)h->d_AB, (void*)h->d_BA, (void*)h->d_BB,
                  (void*)h->d_par, (void*)h->d_par_local, (void*)h->d_par_sorted,
                  (void*)h->d_pos, (void*)h->d_dq_sorted, (void*)h->d_lj_energy,
                  (void*)h->d_inter, (void*)h->d_intra, (void*)h->d_dudl,
                  (void*)h->d_sums})
    cudaFree(p);
  acc_free(h->acc);
  delete h;
  return kOk;
}

// ========================================================= Particle_Mesh
extern "C" int snb_pme_create(const snb_options* opt, int atom_numbers,
                              snb_boundary boundary, const float* box_length,
                              float cutoff, snb_pme** out) {
  if (!out) return fail(kBadInput, "pme_create: null out");
  *out = nullptr;
  snb_options o = opts_or_default(opt);
  snb_pme* h = new snb_pme();
  h->accum = o.accumulation;
  float box[3] = {boundary.cell[0], boundary.cell[2], boundary.cell[5]};
  if (box_length) memcpy(box, box_length, sizeof(box));
  int rc = pme_init(h->p, atom_numbers, boundary.cell, box, cutoff,
                    o.pm_direct_tolerance, o.pm_fftx, o.pm_ffty, o.pm_fftz,
                    o.pm_grid_spacing, o.pme_update_interval,
                    o.pme_calculate_reciprocal_part != 0,
                    o.pme_calculate_excluded_part != 0);
  if (rc) {
    pme_free(h->p);
    delete h;
    return rc;
  }
  rc = acc_init(h->acc, atom_numbers);
  if (rc) return rc;
  SNB_CUDA_TRY(cudaMalloc(&h->d_pos, sizeof(float4) * atom_numbers));
  *out = h;
  return kOk;
}

extern "C" float snb_pme_beta(snb_pme* h) { return h ? h->p.beta : 0.f; }

extern "C" int snb_pme_grid(snb_pme* h, int* fft3) {
  if (!h || !fft3) return fail(kBadInput, "pme_grid: null argument");
  for (int d = 0; d < 3; ++d) fft3[d] = h->p.K[d];
  return kOk;
}

extern "C" int snb_pme_reciprocal_force(snb_pme* h, const float* crd,
                                        snb_boundary boundary, const float* charge,
                                        float* force, int need_virial, int need_energy,
                                        float* d_virial, float* d_potential, int step,
                                        void* stream) {
  if (!h) return fail(kBadInput, "pme_reciprocal_force: null handle");
  if (!h->p.reciprocal) return kOk;
  cudaStream_t st = S(stream);
  if (step % h->p.update_interval == 0) {
    int rc = launch_pack(h->p.n, reinterpret_cast<const float3*>(crd), charge, nullptr,
                         nullptr, h->d_pos, nullptr, st);
    if (rc) return rc;
    rc = pme_reciprocal(h->p, h->d_pos, h->p.n, h->acc, h->accum, need_energy != 0,
                        need_virial != 0, st);
    if (rc) return rc;
    rc = launch_unpack(h->p.n, nullptr, h->acc, h->accum,
                       reinterpret_cast<float3*>(force), nullptr, nullptr, nullptr,
                       nullptr, false, false, st);
    if (rc) return rc;
  }
  if (need_energy || need_virial)
    return launch_add_scalars(need_energy ? d_potential : nullptr,
                              need_virial ? d_virial : nullptr, h->p.d_sums, 0.f, 0.f, 0,
                              st);
  return kOk;
}

extern "C" int snb_pme_excluded_force(snb_pme* h, int atom_numbers,
                                      const int* atom_local, const int* atom_local_id,
                                      const float* crd, snb_boundary boundary,
                                      const float* charge, const int* es,
                                      const int* el, const int* en, float* frc,
                                      int need_energy, float* atom_ene, int need_virial,
                                      float* atom_virial, void* stream) {
  (void)atom_local;
  (void)atom_local_id;
  if (!h) return fail(kBadInput, "pme_excluded_force: null handle");
  if (!h->p.excluded) return kOk;
  if (atom_numbers != h->p.n) return fail(kBadInput, "pme_excluded_force: atom count");
  cudaStream_t st = S(stream);
  int rc = launch_excluded(atom_numbers, reinterpret_cast<const float3*>(crd), charge,
                           cell_of(boundary), rcell_of(boundary), h->p.beta, es, el, en,
                           nullptr, h->acc, h->accum, need_energy != 0,
                           need_virial != 0, st);
  if (rc) return rc;
  return launch_unpack(atom_numbers, nullptr, h->acc, h->accum,
                       reinterpret_cast<float3*>(frc), need_energy ? atom_ene : nullptr,
                       nullptr, nullptr, need_virial ? atom_virial : nullptr,
                       need_energy != 0, need_virial != 0, st);
}

extern "C" int snb_pme_spread_wide_tiles(snb_pme* h, int* count, void* stream) {
  if (!h || !count) return fail(kBadInput, "pme_spread_wide_tiles: null argument");
  return pme_wide_tiles(h->p, count, S(stream));
}

extern "C" int snb_pme_energies(snb_pme* h, double* rec, double* self, double* vir,
                                void* stream) {
  if (!h) return fail(kBadInput, "pme_energies: null handle");
  double s[8];
  SNB_CUDA_TRY(cudaMemcpyAsync(s, h->p.d_sums, sizeof(s), cudaMemcpyDeviceToHost,
                               S(stream)));
  SNB_CUDA_TRY(cudaStreamSynchronize(S(stream)));
  if (rec) *rec = s[0];
  if (self) *self = s[7];
  if (vir)
    for (int c = 0; c < 6; ++c) vir[c] = s[1 + c];
  return kOk;
}

extern "C" int snb_pme_update_box(snb_pme* h, snb_boundary boundary, const float* g,
                                  float dt) {
  (void)g;   // the box-change rate and time step only move the reference's
  (void)dt;  // domain corners; the new cell is in `boundary`
  if (!h) return fail(kBadInput, "pme_update_box: null handle");
  return pme_update_box(h->p, boundary.cell);
}

extern "C" int snb_pme_destroy(snb_pme* h) {
  if (!h) return kOk;
  pme_free(h->p);
  acc_free(h->acc);
  cudaFree(h->d_pos);
  delete h;
  return kOk;
}

// ============================================================= engine
// Everything of engine creation after the neighbor list and PME: LJ tables,
// charges, exclusions, accumulators and the step scratch.
static int engine_finish_create(snb_engine* e, int n, int n_types, const int* h_type,
                                const float* h_A, const float* h_B, const float* h_charge,
                                const int* h_es, const int* h_en, const int* h_el,
                                int n_excl) {
  int rc = acc_init(e->acc, n);
  if (rc) return rc;
  LJParams& p = e->lj;
  p.n_types = n_types;
  p.n_pairs = n_types * (n_types + 1) / 2;
  p.h_type.assign(h_type, h_type + n);
  p.h_A.assign(h_A, h_A + p.n_pairs);
  p.h_B.assign(h_B, h_B + p.n_pairs);
  p.cutoff = e->opt.cutoff;
  for (int i = 0; i < n; ++i)
    if (h_type[i] < 0 || h_type[i] >= n_types)
      return fail(kBadInput, "engine_create: LJ type out of range");
  if (e->nsys > 0) {
    // tail correction per box (its own type histogram and volume)
    e->lrc_energy = e->lrc_virial = 0.0;
    for (const auto& g : e->h_sys) {
      std::vector<int> ts(h_type + g.atom_begin, h_type + g.atom_end);
      const double f = lrc_factor(ts, n_types, p.h_B, p.cutoff);
      e->lrc_energy += f / g.volume;
      e->lrc_virial += 2.0 * f / g.volume;
    }
  } else {
    p.long_range_factor = lrc_factor(p.h_type, n_types, p.h_B, p.cutoff);
    const double vol = (double)e->cell.a11 * e->cell.a22 * e->cell.a33;
    e->lrc_energy = p.long_range_factor / vol;
    e->lrc_virial = 2.0 * p.long_range_factor / vol;
  }
  e->lrc_energy_lj = e->lrc_energy;
  e->lrc_virial_lj = e->lrc_virial;
  SNB_CUDA_TRY(cudaMalloc(&p.d_A, sizeof(float) * p.n_pairs));
  SNB_CUDA_TRY(cudaMalloc(&p.d_B, sizeof(float) * p.n_pairs));
  SNB_CUDA_TRY(cudaMemcpy(p.d_A, h_A, sizeof(float) * p.n_pairs, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMemcpy(p.d_B, h_B, sizeof(float) * p.n_pairs, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&p.d_type, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMemcpy(p.d_type, h_type, sizeof(int) * n, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&e->d_charge, sizeof(float) * n));
  SNB_CUDA_TRY(cudaMemcpy(e->d_charge, h_charge, sizeof(float) * n, cudaMemcpyHostToDevice));
  SNB_CUDA_TRY(cudaMalloc(&e->d_pos, sizeof(float4) * n));
  SNB_CUDA_TRY(cudaMalloc(&e->d_type_sorted, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&e->d_excl_start, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&e->d_excl_numbers, sizeof(int) * n));
  SNB_CUDA_TRY(cudaMalloc(&e->d_excl_list, sizeof(int) * std::max(n_excl, 1)));
  if (h_es && h_en) {
    for (int i = 0; i < n; ++i) {
      if (h_en[i] < 0 || (h_en[i] > 0 && (h_es[i] < 0 || h_es[i] + h_en[i] > n_excl)))
        return fail(kBadInput, "engine_create: exclusion list out of range");
      for (int k = 0; k < h_en[i]; ++k) {
        const int j = h_el[h_es[i] + k];
        if (j < 0 || j >= n)
          return fail(kBadInput, "engine_create: excluded atom index out of range");
        if (e->nsys > 0) {  // an exclusion must stay inside its box
          int si = 0, sj = 0;
          while (i >= e->h_sys[si].atom_end) ++si;
          while (j >= e->h_sys[sj].atom_end) ++sj;
          if (si != sj)
            return fail(kBadInput, "batch_create: exclusion between two systems");
        }
      }
    }
    SNB_CUDA_TRY(cudaMemcpy(e->d_excl_start, h_es, sizeof(int) * n, cudaMemcpyHostToDevice));
    SNB_CUDA_TRY(cudaMemcpy(e->d_excl_numbers, h_en, sizeof(int) * n, cudaMemcpyHostToDevice));
    if (n_excl > 0)
      SNB_CUDA_TRY(cudaMemcpy(e->d_excl_list, h_el, sizeof(int) * n_excl,
                              cudaMemcpyHostToDevice));
  } else {
    SNB_CUDA_TRY(cudaMemset(e->d_excl_start, 0, sizeof(int) * n));
    SNB_CUDA_TRY(cudaMemset(e->d_excl_numbers, 0, sizeof(int) * n));
  }
  SNB_CUDA_TRY(cudaMalloc(&e->d_isum, sizeof(long long) * 9));
  SNB_CUDA_TRY(cudaMalloc(&e->d_bonded_e, sizeof(long long)));
  SNB_CUDA_TRY(cudaMemset(e->d_bonded_e, 0, sizeof(long long)));
  SNB_CUDA_TRY(cudaMalloc(&e->d_totals_scratch, sizeof(double) * 16));
  SNB_CUDA_TRY(cudaMalloc(&e->d_snap_crd, sizeof(float) * 3 * n));
  SNB_CUDA_TRY(cudaMalloc(&e->d_snap_vel, sizeof(float) * 3 * n));
  SNB_CUDA_TRY(cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking));
  {
    // the branch's short kernels take SMs ahead of the persistent pair kernel
    int lo = 0, hi = 0;
    SNB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    SNB_CUDA_TRY(cudaStreamCreateWithPriority(&e->branch, cudaStreamNonBlocking, hi));
    SNB_CUDA_TRY(cudaStreamCreateWithPriority(&e->branch2, cudaStreamNonBlocking, hi));
  }
  SNB_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming));
  SNB_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming));
  SNB_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_join2, cudaEventDisableTiming));
  SNB_CUDA_TRY(cudaStreamCreateWithFlags(&e->io, cudaStreamNonBlocking));
  SNB_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_crd_in, cudaEventDisableTiming));
  SNB_CUDA_TRY(cudaEventCreateWithFlags(&e->ev_vel_in, cudaEventDisableTiming));
  SNB_CUDA_TRY(cudaEventRecord(e->ev_vel_in, e->io));  // a completed record
  return kOk;
}

extern "C" int snb_engine_create(const snb_options* opt, int n, snb_boundary boundary,
                                 int n_types, const int* h_type, const float* h_A,
                                 const float* h_B, const float* h_charge,
                                 const int* h_es, const int* h_en, const int* h_el,
                                 int n_excl, snb_engine** out) {
  if (!out) return fail(kBadInput, "engine_create: null out");
  *out = nullptr;
  if (n <= 0 || n_types <= 0 || !h_type || !h_A || !h_B || !h_charge)
    return fail(kBadInput, "engine_create: bad argument");
  if (boundary.policy != 1) return fail(kNotSupported, "engine: periodic box required");
  if (boundary.cell[1] != 0.f || boundary.cell[3] != 0.f || boundary.cell[4] != 0.f)
    return fail(kNotSupported,
                "engine: rectangular boxes (skewed cells run through the modules: "
                "snb_nl, snb_lj, snb_pme)");
  snb_engine* e = new snb_engine();
  e->opt = opts_or_default(opt);
  e->n = n;
  e->accum = e->opt.accumulation;
  e->cell = cell_of(boundary);
  e->rcell = rcell_of(boundary);
  int rc = nl_init(e->nl, n, e->opt.cutoff, e->opt.skin, boundary.cell,
                   e->opt.nl_refresh_interval, e->opt.nl_skin_permit,
                   e->opt.nl_max_neighbor_numbers, 0);
  float box[3] = {boundary.cell[0], boundary.cell[2], boundary.cell[5]};
  if (!rc)
    rc = pme_init(e->pme, n, boundary.cell, box, e->opt.cutoff, e->opt.pm_direct_tolerance,
                  e->opt.pm_fftx, e->opt.pm_ffty, e->opt.pm_fftz, e->opt.pm_grid_spacing,
                  e->opt.pme_update_interval, e->opt.pme_calculate_reciprocal_part != 0,
                  e->opt.pme_calculate_excluded_part != 0);
  // the engine spreads by int64 atomics up to half a million atoms unless a
  // launch shape says otherwise (the same grid as the tiles): on the 100k box
  // the step is 14 us shorter than with the tiles; on the 1M box the 64 M
  // reductions of the atomic spread made it 0.16 ms longer
  if (!rc && n <= 500000) rc = pme_set_spread_shape(e->pme, 0, 0);
  if (!rc)
    rc = engine_finish_create(e, n, n_types, h_type, h_A, h_B, h_charge, h_es, h_en, h_el,
                              n_excl);
  // pruned rows at 0.8 A: on the 100k box (cutoff 10 A, skin 2 A) a prune
  // pass every 7-8 steps and the MD step 4 % shorter than with full rows
  // (0.3 A: 269-275 us, 0.5: 271-272, 0.8: 268-271, 1.2: 273-275; off:
  // 276-285).  On the 9,000-atom box the extra launch and the passes cost
  // more than they save (631 against 680 ns/day), so small boxes keep the
  // full rows.
  if (!rc && n >= kPruneMinAtoms) rc = snb_engine_set_prune_margin(e, kDefaultPruneMargin);
  if (rc) {
    snb_engine_destroy(e);
    return rc;
  }
  *out = e;
  return kOk;
}

extern "C" int snb_batch_create(const snb_options* opt, int n_systems,
                                const int* atoms_per_system, const float* box_lengths,
                                int n_types, const int* h_type, const float* h_A,
                                const float* h_B, const float* h_charge,
                                const int* h_es, const int* h_en, const int* h_el,
                                int n_excl, snb_engine** out) {
  if (!out) return fail(kBadInput, "batch_create: null out");
  *out = nullptr;
  if (n_systems <= 0 || !atoms_per_system || !box_lengths || n_types <= 0 || !h_type ||
      !h_A || !h_B || !h_charge)
    return fail(kBadInput, "batch_create: bad argument");
  snb_engine* e = new snb_engine();
  e->opt = opts_or_default(opt);
  if (e->opt.pm_fftx > 0 || e->opt.pm_ffty > 0 || e->opt.pm_fftz > 0 ||
      e->opt.pme_update_interval != 1 || e->opt.nl_refresh_interval > 0 ||
      e->opt.accumulation != kAccumFixed) {
    delete e;
    return fail(kNotSupported,
                "batch_create: per-box grids from PM_grid_spacing, PME every step, "
                "displacement-triggered lists and fixed-point accumulation only");
  }
  long long total = 0;
  e->nsys = n_systems;
  e->h_sys.resize(n_systems);
  for (int s = 0; s < n_systems; ++s) {
    SysGeom& g = e->h_sys[s];
    memset(&g, 0, sizeof(g));
    const float* L = box_lengths + 3 * s;
    if (atoms_per_system[s] <= 0 || !(L[0] > 0.f && L[1] > 0.f && L[2] > 0.f)) {
      delete e;
      return fail(kBadInput, "batch_create: empty system or bad box");
    }
    g.atom_begin = (int)total;
    total += atoms_per_system[s];
    g.atom_end = (int)total;
    g.cell.a11 = L[0];
    g.cell.a22 = L[1];
    g.cell.a33 = L[2];
    g.rcell.a11 = 1.0f / L[0];
    g.rcell.a22 = 1.0f / L[1];
    g.rcell.a33 = 1.0f / L[2];
    g.volume = (double)L[0] * L[1] * L[2];
  }
  if (total > 2147483647LL / 16) {
    delete e;
    return fail(kBadInput, "batch_create: too many atoms");
  }
  const int n = (int)total;
  e->n = n;
  e->accum = kAccumFixed;
  e->cell = e->h_sys[0].cell;
  e->rcell = e->h_sys[0].rcell;
  int rc = nl_init_batch(e->nl, n, e->opt.cutoff, e->opt.skin, e->h_sys,
                         e->opt.nl_refresh_interval, e->opt.nl_skin_permit,
                         e->opt.nl_max_neighbor_numbers);
  if (!rc)
    rc = pme_init_batch(e->pme, n, e->h_sys, e->opt.cutoff, e->opt.pm_direct_tolerance,
                        e->opt.pm_grid_spacing, e->opt.pme_calculate_reciprocal_part != 0,
                        e->opt.pme_calculate_excluded_part != 0);
  if (!rc) {
    std::vector<int> sys_of(n);
    for (int s = 0; s < n_systems; ++s)
      for (int i = e->h_sys[s].atom_begin; i < e->h_sys[s].atom_end; ++i) sys_of[i] = s;
    if (cudaMalloc(&e->d_sys, sizeof(SysGeom) * n_systems) != cudaSuccess ||
        cudaMemcpy(e->d_sys, e->h_sys.data(), sizeof(SysGeom) * n_systems,
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&e->d_sys_of, sizeof(int) * n) != cudaSuccess ||
        cudaMemcpy(e->d_sys_of, sys_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice) !=
            cudaSuccess)
      rc = fail(kCudaError, "batch_create: system table upload failed");
  }
  if (!rc) {
    // each system rebuilds its list when its own atoms moved past the skin
    // allowance: cell -> system map and the per-system flags
    std::vector<int> cell_sys(e->nl.ncell, 0);
    for (int s = 0; s < n_systems; ++s) {
      const SysGeom& g = e->h_sys[s];
      for (int c = g.cell_begin; c < g.cell_begin + g.Nx * g.Ny * g.Nz; ++c) cell_sys[c] = s;
    }
    if (cudaMalloc(&e->d_cell_sys, sizeof(int) * cell_sys.size()) != cudaSuccess ||
        cudaMemcpy(e->d_cell_sys, cell_sys.data(), sizeof(int) * cell_sys.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&e->d_box_need, n_systems) != cudaSuccess ||
        cudaMemset(e->d_box_need, 0, n_systems) != cudaSuccess)
      rc = fail(kCudaError, "batch_create: per-system rebuild tables failed");
  }
  if (!rc) {
    e->bv.sys = e->d_sys;
    e->bv.sys_of = e->d_sys_of;
    e->bv.tile_sys = e->pme.d_tile_sys;
    e->bv.nsys = n_systems;
    e->bv.box_need = e->d_box_need;
    e->bv.cell_sys = e->d_cell_sys;
    e->nl.bv = e->bv;
    e->pme.bv = e->bv;
    rc = engine_finish_create(e, n, n_types, h_type, h_A, h_B, h_charge, h_es, h_en, h_el,
                              n_excl);
  }
  if (!rc) rc = snb_engine_set_prune_margin(e, kDefaultPruneMargin);
  // the batch's own FFT passes where every grid allows them: on the 256-box
  // batch (grids 20^3-40^3) the PME chain takes 467 us against 636 us with
  // the batched cuFFT plans, the step 1.65 ms against 1.77 ms
  if (!rc && e->pme.reciprocal && pme_set_own_fft(e->pme, true)) set_error("");
  if (rc) {
    snb_engine_destroy(e);
    return rc;
  }
  *out = e;
  return kOk;
}

// Inside a stream capture: an IF node whose body is the neighbor-list
// rebuild, taken when the rebuild flag is set (by the previous step's
// leap-frog check, or by a forced update).  Non-rebuild steps then cost one
// tiny kernel instead of the ~15 early-exit launches of the rebuild.
static int capture_conditional_rebuild(snb_engine* e, const float* crd, cudaStream_t st) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  SNB_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) return fail(kCudaError, "capture not active");
  cudaGraphConditionalHandle hc;
  SNB_CUDA_TRY(cudaGraphConditionalHandleCreate(&hc, cg, 0, cudaGraphCondAssignDefault));
  int rc = nl_set_condition(e->nl, hc, st, engine_prunes(e) ? e->d_prune : nullptr);
  if (rc) return rc;
  SNB_CUDA_TRY(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd));
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeIf;
  cp.conditional.size = 1;
  cudaGraphNode_t cn;
  SNB_CUDA_TRY(cudaGraphAddNode(&cn, cg, deps, nd, &cp));
  SNB_CUDA_TRY(cudaStreamUpdateCaptureDependencies(st, &cn, 1,
                                                   cudaStreamSetCaptureDependencies));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  SNB_CUDA_TRY(cudaStreamBeginCaptureToGraph(e->side, body, nullptr, nullptr, 0,
                                             cudaStreamCaptureModeThreadLocal));
  rc = nl_rebuild(e->nl, crd, nullptr, e->d_excl_start, e->d_excl_list,
                  e->d_excl_numbers, e->side);
  cudaGraph_t b2 = nullptr;
  cudaError_t ce = cudaStreamEndCapture(e->side, &b2);
  if (rc) return rc;
  if (ce != cudaSuccess)
    return fail(kCudaError, std::string("rebuild body capture: ") + cudaGetErrorString(ce));
  size_t nn = 0;
  SNB_CUDA_TRY(cudaGraphGetNodes(body, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  SNB_CUDA_TRY(cudaGraphGetNodes(body, nodes.data(), &nn));
  e->body_kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    e->body_kernels += t == cudaGraphNodeTypeKernel;
  }
  return kOk;
}

// nonbonded forces of one step into e->acc (sorted frame), no unpack.
// in_graph: called while capturing the replayed step (conditional rebuild,
// refresh check done by the previous step's leap-frog).
static int engine_bonded(snb_engine* e, const float* crd, cudaStream_t st) {
  return launch_bonded(e->nb, e->d_ba, e->d_bb, e->d_bk, e->d_br0, e->na, e->d_aa, e->d_ab,
                       e->d_ac, e->d_ak, e->d_at0, reinterpret_cast<const float3*>(crd),
                       e->cell, e->rcell, e->nl.d_inv_perm, e->acc, nullptr, false, st,
                       e->bv);
}

// with_bonded: also the water bonds and angles (MD steps).  Outside the
// per-phase profiling pass the excluded correction, the bonded terms and the
// PME chain run on a second stream, concurrently with the pair kernel.
static int engine_forces(snb_engine* e, const float* crd, int step, bool energy,
                         bool virial, bool forced_nl, cudaStream_t st,
                         bool in_graph = false, bool with_bonded = false) {
  prof_mark(e, 0, st);
  int rc;
  if (in_graph) {
    rc = capture_conditional_rebuild(e, crd, st);
  } else {
    rc = nl_update(e->nl, crd, nullptr, nullptr, step, forced_nl ? 1 : 0,
                   e->d_excl_start, e->d_excl_list, e->d_excl_numbers, st);
  }
  if (rc) return rc;
  prof_mark(e, 1, st);
  const bool do_pme = e->pme.reciprocal && step % e->pme.update_interval == 0;
  // cluster form: the pair frame holds each atom in its cell's image
  const bool clus = e->nl.clusters && !e->soft;
  const float3* img = clus ? e->nl.d_img_off : nullptr;
  if (do_pme)
    rc = pme_pack_bin(e->pme, e->n, reinterpret_cast<const float3*>(crd), e->d_charge,
                      e->lj.d_type, e->nl.d_perm, e->d_pos, e->d_type_sorted, st, img);
  else
    rc = launch_pack(e->n, reinterpret_cast<const float3*>(crd), e->d_charge,
                     e->lj.d_type, e->nl.d_perm, e->d_pos, e->d_type_sorted, st, img);
  if (rc) return rc;
  if (e->soft)
    k_pack_soft<<<ceil_div(e->n, 256), 256, 0, st>>>(e->n, e->nl.d_perm, e->soft->d_par_local,
                                                    nullptr, e->soft->d_par_sorted, nullptr);
  prof_mark(e, 2, st);
  const bool fork = !e->prof_on;
  cudaStream_t sb = fork ? e->branch : st;
  if (fork) {
    // PME on `branch`, the excluded correction and bonded terms on `branch2`,
    // the pair kernel on the step's stream
    cudaStream_t sb2 = e->branch2;
    SNB_CUDA_TRY(cudaEventRecord(e->ev_fork, st));
    SNB_CUDA_TRY(cudaStreamWaitEvent(sb, e->ev_fork, 0));
    SNB_CUDA_TRY(cudaStreamWaitEvent(sb2, e->ev_fork, 0));
    if (with_bonded && (rc = engine_bonded(e, crd, sb2))) return rc;
    if (e->pme.excluded &&
        (rc = launch_excluded(e->n, reinterpret_cast<const float3*>(crd), e->d_charge,
                              e->cell, e->rcell, e->pme.beta, e->d_excl_start,
                              e->d_excl_list, e->d_excl_numbers, e->nl.d_inv_perm, e->acc,
                              e->accum, energy, virial, sb2, e->bv)))
      return rc;
    if (e->nb14 &&
        (rc = launch_nb14(e->nb14->p, reinterpret_cast<const float3*>(crd), e->d_charge,
                          e->cell, e->rcell, e->nl.d_inv_perm, e->acc, energy, virial, false,
                          energy ? e->d_nb14_sums : nullptr, sb2)))
      return rc;
    SNB_CUDA_TRY(cudaEventRecord(e->ev_join2, sb2));
    if (do_pme && (rc = pme_after_bin(e->pme, e->n, e->acc, e->accum, energy, virial, sb)))
      return rc;
    SNB_CUDA_TRY(cudaEventRecord(e->ev_join, sb));
  }
  PairArgs a;
  a.n = e->n;
  a.pos = e->d_pos;
  a.type = e->d_type_sorted;
  a.global = e->nl.d_global;
  a.row_start = e->nl.d_row_start;
  a.row_count = e->nl.d_row_count;
  a.cols = e->nl.d_cols;
  a.nl_flags = e->nl.d_flags;
  a.A = e->lj.d_A;
  a.B = e->lj.d_B;
  a.n_types = e->lj.n_types;
  a.cell = e->cell;
  a.rcell = e->rcell;
  a.cutoff2 = e->opt.cutoff * e->opt.cutoff;
  a.beta = e->pme.beta;
  a.bv = e->bv;
  a.unroll = e->pair_unroll;
  a.blocks_per_sm = e->pair_blocks_per_sm;
  a.warps = e->pair_warps;
  a.stash = e->pair_stash;
  if (engine_prunes(e)) {
    if (!in_graph) {  // (in the graph the rebuild condition's kernel decides)
      k_prune_decide<<<1, 1, 0, st>>>(e->d_prune, e->nl.d_flags);
      SNB_CUDA_TRY(cudaGetLastError());
    }
    const float rp = e->opt.cutoff + e->prune_margin;
    a.prune = e->d_prune;
    a.cols_in = e->nl.d_cols_in;
    a.row_in_count = e->nl.d_row_in_count;
    a.prune_ref = e->nl.d_prune_ref;
    a.prune2 = rp * rp;
  } else if ((rc = engine_prune_invalidate(e, st))) {
    return rc;
  }
  if (e->soft) {
    SoftArgs sa;
    sa.n = e->n;
    sa.pos = e->d_pos;
    sa.par = e->soft->d_par_sorted;
    sa.dq = nullptr;
    sa.global = e->nl.d_global;
    sa.row_start = e->nl.d_row_start;
    sa.row_count = e->nl.d_row_count;
    sa.cols = e->nl.d_cols;
    sa.nl_flags = e->nl.d_flags;
    sa.AA = e->soft->d_AA;
    sa.AB = e->soft->d_AB;
    sa.BA = e->soft->d_BA;
    sa.BB = e->soft->d_BB;
    sa.n_types_A = e->soft->nA;
    sa.n_types_B = e->soft->nB;
    sa.cell = e->cell;
    sa.rcell = e->rcell;
    sa.cutoff2 = a.cutoff2;
    sa.beta = a.beta;
    sa.lambda = e->soft->lambda;
    sa.alpha = e->soft->alpha;
    sa.p = e->soft->p;
    sa.sigma6 = e->soft->sigma6;
    sa.sigma6_min = e->soft->sigma6_min;
    sa.prune = a.prune;
    sa.cols_in = a.cols_in;
    sa.row_in_count = a.row_in_count;
    sa.prune_ref = a.prune_ref;
    sa.prune2 = a.prune2;
    rc = launch_soft_rows(sa, e->acc, energy, virial, st);
  } else if (clus) {
    ClusterPairArgs ca;
    ca.clus = e->nl.d_clus;
    ca.nclus = e->nl.d_nclus;
    ca.crow_count = e->nl.d_crow_count;
    ca.centry = e->nl.d_centry;
    ca.ccap = e->nl.ccap;
    ca.pos = e->d_pos;
    ca.type = e->d_type_sorted;
    ca.global = e->nl.d_global;
    ca.nl_flags = e->nl.d_flags;
    ca.A = e->lj.d_A;
    ca.B = e->lj.d_B;
    ca.n_types = e->lj.n_types;
    ca.box = make_float3(e->cell.a11, e->cell.a22, e->cell.a33);
    ca.cutoff2 = a.cutoff2;
    ca.beta = a.beta;
    ca.blocks_per_sm = e->pair_blocks_per_sm;
    rc = launch_pair_clusters(ca, e->acc, e->accum, energy, virial, st);
  } else {
    rc = launch_pair(a, e->acc, e->accum, energy, virial, true, st);
  }
  if (rc) return rc;
  if (fork) {
    SNB_CUDA_TRY(cudaStreamWaitEvent(st, e->ev_join, 0));
    SNB_CUDA_TRY(cudaStreamWaitEvent(st, e->ev_join2, 0));
    return kOk;
  }
  prof_mark(e, 3, st);
  if (e->pme.excluded) {
    rc = launch_excluded(e->n, reinterpret_cast<const float3*>(crd), e->d_charge, e->cell,
                         e->rcell, e->pme.beta, e->d_excl_start, e->d_excl_list,
                         e->d_excl_numbers, e->nl.d_inv_perm, e->acc, e->accum, energy,
                         virial, st, e->bv);
    if (rc) return rc;
  }
  if (e->nb14 &&
      (rc = launch_nb14(e->nb14->p, reinterpret_cast<const float3*>(crd), e->d_charge, e->cell,
                        e->rcell, e->nl.d_inv_perm, e->acc, energy, virial, false,
                        energy ? e->d_nb14_sums : nullptr, st)))
    return rc;
  prof_mark(e, 4, st);
  if (do_pme) {
    rc = pme_after_bin(e->pme, e->n, e->acc, e->accum, energy, virial, st);
    if (rc) return rc;
  }
  prof_mark(e, 5, st);
  if (with_bonded && (rc = engine_bonded(e, crd, st))) return rc;
  prof_mark(e, 6, st);
  return kOk;
}

extern "C" int snb_engine_force(snb_engine* e, const float* crd, float* frc, int step,
                                int need_energy, int need_virial, double* d_totals,
                                void* stream) {
  if (!e) return fail(kBadInput, "engine_force: null handle");
  cudaStream_t st = S(stream);
  bool en = need_energy != 0, vi = need_virial != 0;
  if ((en || vi) && !d_totals) return fail(kBadInput, "engine_force: d_totals required");
  if (en || vi) SNB_CUDA_TRY(cudaMemsetAsync(e->d_bonded_e, 0, sizeof(long long), st));
  if (en && e->nb14)
    SNB_CUDA_TRY(cudaMemsetAsync(e->d_nb14_sums, 0, sizeof(long long) * 2, st));
  // any coordinates: the pruned rows are made again from the full rows
  int rc = engine_prune_invalidate(e, st);
  if (rc) return rc;
  rc = engine_forces(e, crd, step, en, vi, e->steps_done == 0, st);
  if (rc) return rc;
  e->steps_done++;
  if (en || vi) {
    rc = launch_totals(e->n, e->acc, e->d_isum, e->nb14 ? e->d_nb14_sums : nullptr,
                       e->pme.d_sums, e->lrc_energy,
                       e->lrc_virial, d_totals, en, vi, e->pme.reciprocal, st);
    if (rc) return rc;
  }
  if (e->vatom && (rc = vatom_spread_fixed(e->vatom, crd, e->cell, e->rcell,
                                           e->nl.d_inv_perm, e->acc, st)))
    return rc;
  return launch_unpack(e->n, e->nl.d_inv_perm, e->acc, e->accum,
                       reinterpret_cast<float3*>(frc), nullptr, nullptr, nullptr, nullptr,
                       en, vi, st);
}

extern "C" int snb_nb14_create(int atom_numbers, int nb14_numbers, const int* h_atom_a,
                               const int* h_atom_b, const float* h_A, const float* h_B,
                               const float* h_cf_scale_factor, snb_nb14** out) {
  if (!out) return fail(kBadInput, "nb14_create: null out");
  *out = nullptr;
  if (atom_numbers <= 0) return fail(kBadInput, "nb14_create: atom_numbers must be > 0");
  snb_nb14* h = new snb_nb14();
  h->n = atom_numbers;
  int rc = nb14_init(h->p, nb14_numbers, h_atom_a, h_atom_b, h_A, h_B, h_cf_scale_factor,
                     atom_numbers);
  if (!rc) rc = acc_init(h->acc, atom_numbers);
  if (!rc) {
    cudaError_t ce = cudaMalloc(&h->d_sums, sizeof(long long) * 2);
    if (ce == cudaSuccess) ce = cudaMemset(h->d_sums, 0, sizeof(long long) * 2);
    if (ce != cudaSuccess) rc = fail(kCudaError, cudaGetErrorString(ce));
  }
  if (rc) {
    nb14_free(h->p);
    delete h;
    return rc;
  }
  *out = h;
  return kOk;
}

extern "C" int snb_nb14_force(snb_nb14* h, const float* crd, const float* charge,
                              snb_boundary boundary, float* frc, int need_atom_energy,
                              float* atom_energy, int need_virial, float* atom_virial,
                              void* stream) {
  if (!h || !crd || !charge || !frc) return fail(kBadInput, "nb14_force: bad argument");
  cudaStream_t st = S(stream);
  const bool en = need_atom_energy != 0, vi = need_virial != 0;
  if (en) SNB_CUDA_TRY(cudaMemsetAsync(h->d_sums, 0, sizeof(long long) * 2, st));
  int rc = launch_nb14(h->p, reinterpret_cast<const float3*>(crd), charge, cell_of(boundary),
                       rcell_of(boundary), nullptr, h->acc, en, vi, true,
                       en ? h->d_sums : nullptr, st);
  if (rc) return rc;
  return launch_unpack(h->n, nullptr, h->acc, h->accum, reinterpret_cast<float3*>(frc),
                       en ? atom_energy : nullptr, nullptr, nullptr, vi ? atom_virial : nullptr,
                       en, vi, st);
}

extern "C" int snb_nb14_energy_sums(snb_nb14* h, float* h_lj, float* h_ee, void* stream) {
  if (!h || !h_lj || !h_ee) return fail(kBadInput, "nb14_energy_sums: null argument");
  long long v[2];
  cudaStream_t st = S(stream);
  SNB_CUDA_TRY(cudaMemcpyAsync(v, h->d_sums, sizeof(v), cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  *h_ee = (float)((double)v[1] * kEnergyScaleInv);
  *h_lj = (float)((double)(v[0] - v[1]) * kEnergyScaleInv);
  return kOk;
}

extern "C" int snb_nb14_destroy(snb_nb14* h) {
  if (!h) return kOk;
  nb14_free(h->p);
  acc_free(h->acc);
  cudaFree(h->d_sums);
  delete h;
  return kOk;
}

extern "C" int snb_engine_set_nb14(snb_engine* e, snb_nb14* nb14) {
  if (!e) return fail(kBadInput, "engine_set_nb14: null handle");
  if (nb14) {
    if (e->nsys > 0) return fail(kNotSupported, "engine_set_nb14: batch engines");
    if (e->accum != kAccumFixed)
      return fail(kNotSupported, "engine_set_nb14: fixed-point accumulation required");
    if (nb14->n != e->n) return fail(kBadInput, "engine_set_nb14: atom count differs");
    if (!e->d_nb14_sums) {
      SNB_CUDA_TRY(cudaMalloc(&e->d_nb14_sums, sizeof(long long) * 2));
      SNB_CUDA_TRY(cudaMemset(e->d_nb14_sums, 0, sizeof(long long) * 2));
    }
  }
  e->nb14 = nb14;
  if (e->graph_exec) {  // the captured step holds the previous set of terms
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
  }
  return kOk;
}

extern "C" int snb_settle_create(int atom_numbers, int constrain_pair_numbers,
                                 const int* h_atom_i, const int* h_atom_j,
                                 const float* h_constant_r, const float* h_mass,
                                 snb_settle** out) {
  if (!out) return fail(kBadInput, "settle_create: null out");
  *out = nullptr;
  snb_settle* h = new snb_settle();
  int rc = settle_init(h->s, atom_numbers, constrain_pair_numbers, h_atom_i, h_atom_j,
                       h_constant_r, h_mass);
  if (rc) {
    settle_free(h->s);
    delete h;
    return rc;
  }
  *out = h;
  return kOk;
}

extern "C" int snb_settle_group(int atom_numbers, int constrain_pair_numbers,
                                const int* h_atom_i, const int* h_atom_j,
                                const float* h_constant_r, const float* h_mass,
                                int* counts, int* h_remaining_pairs) {
  if (!counts) return fail(kBadInput, "settle_group: null counts");
  std::vector<SettleTri> tri;
  std::vector<SettlePair> pair;
  std::vector<int> rem;
  int rc = settle_group(atom_numbers, constrain_pair_numbers, h_atom_i, h_atom_j,
                        h_constant_r, h_mass, tri, pair, rem);
  if (rc) return rc;
  counts[0] = (int)tri.size();
  counts[1] = (int)pair.size();
  counts[2] = (int)rem.size();
  if (h_remaining_pairs)
    for (size_t k = 0; k < rem.size(); ++k) h_remaining_pairs[k] = rem[k];
  return kOk;
}

extern "C" int snb_settle_counts(snb_settle* h, int* triangle_numbers, int* pair_numbers,
                                 int* remaining_pair_numbers, int* h_remaining_pairs) {
  if (!h) return fail(kBadInput, "settle_counts: null handle");
  if (triangle_numbers) *triangle_numbers = h->s.nt;
  if (pair_numbers) *pair_numbers = h->s.np;
  if (remaining_pair_numbers) *remaining_pair_numbers = (int)h->s.remaining.size();
  if (h_remaining_pairs)
    for (size_t k = 0; k < h->s.remaining.size(); ++k) h_remaining_pairs[k] = h->s.remaining[k];
  return kOk;
}

extern "C" int snb_settle_remember_last_coordinates(snb_settle* h, const float* crd,
                                                    snb_boundary boundary, void* stream) {
  if (!h || !crd) return fail(kBadInput, "settle_remember: bad argument");
  return launch_settle_remember(h->s, reinterpret_cast<const float3*>(crd), cell_of(boundary),
                                rcell_of(boundary), S(stream));
}

extern "C" int snb_settle_do(snb_settle* h, float* crd, snb_boundary boundary, float* vel,
                             float dt, float v_factor, float x_factor, int need_pressure,
                             float* d_stress, void* stream) {
  if (!h || !crd || !vel || !(dt > 0.f) || (need_pressure && !d_stress))
    return fail(kBadInput, "settle_do: bad argument");
  return launch_settle(h->s, reinterpret_cast<float3*>(crd), reinterpret_cast<float3*>(vel),
                       cell_of(boundary), rcell_of(boundary), dt, v_factor, x_factor,
                       need_pressure ? d_stress : nullptr, S(stream));
}

extern "C" int snb_settle_status(snb_settle* h, int* invalid_pair, void* stream) {
  if (!h || !invalid_pair) return fail(kBadInput, "settle_status: bad argument");
  int v = 0;
  cudaStream_t st = S(stream);
  SNB_CUDA_TRY(cudaMemcpyAsync(&v, h->s.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaMemsetAsync(h->s.d_err, 0, sizeof(int), st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  *invalid_pair = v - 1;
  return v ? fail(kBadInput, "SETTLE: rigid pair " + std::to_string(v - 1) +
                                 " has no real position update")
           : kOk;
}

extern "C" int snb_settle_destroy(snb_settle* h) {
  if (!h) return kOk;
  settle_free(h->s);
  delete h;
  return kOk;
}

extern "C" int snb_engine_pressure(snb_engine* e, const float* vel, const float* mass,
                                   const double* d_totals, double* d_out, void* stream) {
  if (!e || !vel || !mass || !d_out) return fail(kBadInput, "engine_pressure: bad argument");
  if (e->nsys > 0) return fail(kNotSupported, "engine_pressure: batch engines");
  if (!e->d_kin) SNB_CUDA_TRY(cudaMalloc(&e->d_kin, sizeof(double) * 6));
  // 1 / V of the cell, as Get_Volume gives it (MD_core/sys.hpp:493-525)
  const double inv_v = 1.0 / ((double)e->cell.a11 * e->cell.a22 * e->cell.a33);
  return launch_pressure(e->n, reinterpret_cast<const float3*>(vel), mass,
                         d_totals ? d_totals + 8 : nullptr,
                         e->settle ? e->settle->s.d_vir : nullptr, inv_v, e->d_kin, d_out,
                         S(stream));
}

extern "C" int snb_engine_set_settle(snb_engine* e, snb_settle* settle) {
  if (!e) return fail(kBadInput, "engine_set_settle: null handle");
  if (settle) {
    if (e->nsys > 0) return fail(kNotSupported, "engine_set_settle: batch engines");
    if (settle->s.n != e->n) return fail(kBadInput, "engine_set_settle: atom count differs");
  }
  e->settle = settle;
  if (e->graph_exec) {  // the captured step holds the previous integration
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
  }
  return kOk;
}

extern "C" int snb_engine_update_box(snb_engine* e, snb_boundary boundary) {
  if (!e) return fail(kBadInput, "engine_update_box: null handle");
  if (e->nsys > 0) return fail(kNotSupported, "engine_update_box: batch engines");
  const float* c6 = boundary.cell;
  if (c6[1] != 0.f || c6[3] != 0.f || c6[4] != 0.f)
    return fail(kNotSupported, "engine_update_box: only rectangular boxes are supported");
  if (!(c6[0] > 0.f && c6[2] > 0.f && c6[5] > 0.f))
    return fail(kBadInput, "engine_update_box: box lengths must be > 0");
  int rc = nl_regrid(e->nl, c6);
  if (rc) return rc;
  if ((rc = pme_update_box(e->pme, c6))) return rc;
  e->cell = make_cell(c6);
  Cell r{};
  r.a11 = 1.0f / e->cell.a11;
  r.a22 = 1.0f / e->cell.a22;
  r.a33 = 1.0f / e->cell.a33;
  e->rcell = r;
  // tail terms at the new volume
  const double vol = (double)e->cell.a11 * e->cell.a22 * e->cell.a33;
  e->lrc_energy_lj = e->lj.long_range_factor / vol;
  e->lrc_virial_lj = 2.0 * e->lj.long_range_factor / vol;
  if (e->soft) {
    e->lrc_energy = e->soft->lrc / vol;
    e->lrc_virial = 2.0 * e->soft->lrc / vol;
  } else {
    e->lrc_energy = e->lrc_energy_lj;
    e->lrc_virial = e->lrc_virial_lj;
  }
  if (e->graph_exec) {  // the captured step holds the old box and list arrays
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
  }
  e->steps_done = 0;  // the next step rebuilds the list, as after Initial
  return kOk;
}

extern "C" int snb_engine_set_virtual_atoms(snb_engine* e, snb_vatom* vatom) {
  if (!e) return fail(kBadInput, "engine_set_virtual_atoms: null handle");
  if (vatom) {
    if (e->nsys > 0) return fail(kNotSupported, "engine_set_virtual_atoms: batch engines");
    if (e->accum != kAccumFixed)
      return fail(kNotSupported, "engine_set_virtual_atoms: fixed-point accumulation only");
    if (vatom_atoms(vatom) != e->n)
      return fail(kBadInput, "engine_set_virtual_atoms: atom count differs");
  }
  e->vatom = vatom;
  if (e->graph_exec) {  // the captured step holds the previous step shape
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
  }
  return kOk;
}

extern "C" int snb_engine_set_soft_core(snb_engine* e, snb_lj_soft* soft) {
  if (!e) return fail(kBadInput, "engine_set_soft_core: null handle");
  if (soft) {
    if (e->nsys > 0) return fail(kNotSupported, "engine_set_soft_core: batch engines");
    if (e->accum != kAccumFixed || soft->accum != kAccumFixed)
      return fail(kNotSupported, "engine_set_soft_core: fixed-point accumulation only");
    if (soft->n != e->n) return fail(kBadInput, "engine_set_soft_core: atom count differs");
  }
  e->soft = soft;
  // the soft-core pair kernel reads the rows
  if (soft && e->nl.clusters) {
    int rc = nl_set_clusters(e->nl, false);
    if (rc) return rc;
    e->steps_done = 0;  // the next step rebuilds the list in its new form
  }
  if (soft) {
    const double vol = (double)e->cell.a11 * e->cell.a22 * e->cell.a33;
    e->lrc_energy = soft->lrc / vol;
    e->lrc_virial = 2.0 * soft->lrc / vol;
  } else {
    e->lrc_energy = e->lrc_energy_lj;
    e->lrc_virial = e->lrc_virial_lj;
  }
  if (e->graph_exec) {  // the captured step holds the previous pair kernel
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
  }
  return kOk;
}

extern "C" int snb_engine_set_bonded(snb_engine* e, int nb, const int* ba, const int* bb,
                                     const float* bk, const float* br0, int na,
                                     const int* aa, const int* ab, const int* ac,
                                     const float* ak, const float* at0) {
  if (!e) return fail(kBadInput, "engine_set_bonded: null handle");
  for (int t = 0; t < nb; ++t)
    if (ba[t] < 0 || ba[t] >= e->n || bb[t] < 0 || bb[t] >= e->n)
      return fail(kBadInput, "engine_set_bonded: bond atom index out of range");
  for (int t = 0; t < na; ++t)
    if (aa[t] < 0 || aa[t] >= e->n || ab[t] < 0 || ab[t] >= e->n || ac[t] < 0 ||
        ac[t] >= e->n)
      return fail(kBadInput, "engine_set_bonded: angle atom index out of range");
  auto up_i = [](int** d, const int* h, int m) -> int {
    cudaFree(*d);
    *d = nullptr;
    if (m <= 0) return kOk;
    SNB_CUDA_TRY(cudaMalloc(d, sizeof(int) * m));
    SNB_CUDA_TRY(cudaMemcpy(*d, h, sizeof(int) * m, cudaMemcpyHostToDevice));
    return kOk;
  };
  auto up_f = [](float** d, const float* h, int m) -> int {
    cudaFree(*d);
    *d = nullptr;
    if (m <= 0) return kOk;
    SNB_CUDA_TRY(cudaMalloc(d, sizeof(float) * m));
    SNB_CUDA_TRY(cudaMemcpy(*d, h, sizeof(float) * m, cudaMemcpyHostToDevice));
    return kOk;
  };
  int rc = up_i(&e->d_ba, ba, nb) | up_i(&e->d_bb, bb, nb) | up_f(&e->d_bk, bk, nb) |
           up_f(&e->d_br0, br0, nb) | up_i(&e->d_aa, aa, na) | up_i(&e->d_ab, ab, na) |
           up_i(&e->d_ac, ac, na) | up_f(&e->d_ak, ak, na) | up_f(&e->d_at0, at0, na);
  if (rc) return fail(kCudaError, "engine_set_bonded: upload failed");
  e->nb = nb;
  e->na = na;
  if (e->graph_exec) {
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
  }
  return kOk;
}

static int engine_md_step(snb_engine* e, float* crd, float* vel, const float* invm,
                          float dt, int step, bool forced_nl, cudaStream_t st,
                          bool in_graph = false) {
  if (e->accum != kAccumFixed)
    return fail(kNotSupported, "md steps need the fixed-point accumulation");
  int rc = engine_forces(e, crd, step, false, false, forced_nl, st, in_graph, true);
  if (rc) return rc;
  // the sites' forces onto their atoms before the update (Force_Redistribute)
  if (e->vatom && (rc = vatom_spread_fixed(e->vatom, crd, e->cell, e->rcell,
                                           e->nl.d_inv_perm, e->acc, st)))
    return rc;
  // the next step's refresh check rides on the coordinate update
  const bool check = e->opt.nl_refresh_interval <= 0;
  const float permit = e->opt.skin * e->opt.nl_skin_permit;
  if (e->settle && (rc = launch_settle_remember(e->settle->s,
                                                reinterpret_cast<const float3*>(crd), e->cell,
                                                e->rcell, st)))
    return rc;
  // with SETTLE or virtual sites the check waits for the final positions
  const bool fused = check && !e->settle && !e->vatom;
  // host-buffer steps: the velocities copied in beside the force phase
  if (e->vel_wait)
    SNB_CUDA_TRY(cudaStreamWaitEvent(st, e->ev_vel_in,
                                     in_graph ? cudaEventWaitExternal : cudaEventWaitDefault));
  const PruneCheck pc = engine_prune_check(e);
  const bool late = e->settle || e->vatom;  // the checks wait for the final positions
  rc = launch_leap_frog(e->n, e->nl.d_inv_perm, e->acc, reinterpret_cast<float3*>(crd),
                        reinterpret_cast<float3*>(vel), invm, dt,
                        fused ? e->nl.d_old_crd : nullptr, e->cell, e->rcell,
                        permit * permit, e->nl.d_flags, st, e->bv,
                        late ? PruneCheck() : pc);
  if (rc) return rc;
  if (e->settle) {
    rc = launch_settle(e->settle->s, reinterpret_cast<float3*>(crd),
                       reinterpret_cast<float3*>(vel), e->cell, e->rcell, dt, 1.0f, 1.0f,
                       nullptr, st);
    if (!rc && check && !e->vatom) rc = nl_check_moved(e->nl, crd, st);
    if (rc) return rc;
  }
  if (e->vatom) {  // the sites follow their atoms (Coordinate_Refresh)
    rc = vatom_refresh(e->vatom, crd, e->cell, e->rcell, st);
    if (!rc && check) rc = nl_check_moved(e->nl, crd, st);
    if (rc) return rc;
  }
  if (late && (rc = launch_prune_check(e->n, reinterpret_cast<const float3*>(crd),
                                       e->nl.d_inv_perm, pc, e->cell, e->rcell, st, e->bv)))
    return rc;
  prof_mark(e, 7, st);
  return rc;
}

// Runs `steps` steps; every check_overflow_interval steps reads the list
// overflow flag and, on overflow, regrows the list, restores the snapshot
// and repeats the steps since it (the recovery loop Check_Overflow was meant
// to provide, neighbor_list.cpp:1027-1103).
// h_crd_out / h_vel_out (host, may be null): the final crd / vel are copied
// there before the last overflow check, so that one synchronisation serves
// both (a repeat after an overflow copies them again).
static int engine_run(snb_engine* e, float* crd, float* vel, const float* invm, float dt,
                      int first, int steps, cudaStream_t st, bool use_graph,
                      float* h_crd_out = nullptr, float* h_vel_out = nullptr) {
  const int chk = std::max(1, e->opt.nl_check_overflow_interval);
  int s = 0;
  int retries = 0;
  // sites placed from the given atoms before the first force
  if (e->vatom && e->steps_done == 0) {
    int rc = vatom_refresh(e->vatom, crd, e->cell, e->rcell, st);
    if (rc) return rc;
  }
  while (s < steps) {
    int chunk = std::min(chk, steps - s);
    SNB_CUDA_TRY(cudaMemcpyAsync(e->d_snap_crd, crd, sizeof(float) * 3 * e->n,
                                 cudaMemcpyDeviceToDevice, st));
    if (!e->vel_snapped)
      SNB_CUDA_TRY(cudaMemcpyAsync(e->d_snap_vel, vel, sizeof(float) * 3 * e->n,
                                   cudaMemcpyDeviceToDevice, st));
    e->vel_snapped = false;  // later chunks start from velocities on the device
    for (int k = 0; k < chunk; ++k) {
      int step = first + s + k;
      // forced rebuild on the first step and every DOM_DEC_update_interval
      // steps, as the reference MD loop does (main.cpp:1805-1822)
      const int ui = e->opt.dom_dec_update_interval;
      bool forced = e->steps_done == 0 || (ui > 0 && step > 0 && step % ui == 0);
      if (use_graph && !forced) {
        if (!e->graph_exec || e->g_crd != crd || e->g_vel != vel || e->g_invm != invm ||
            e->g_dt != dt || e->g_stream != st || e->g_vel_wait != e->vel_wait) {
          if (e->graph_exec) {
            cudaGraphExecDestroy(e->graph_exec);
            cudaGraphDestroy(e->graph);
            e->graph_exec = nullptr;
          }
          SNB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
          int rc = engine_md_step(e, crd, vel, invm, dt, step, false, st, true);
          cudaGraph_t g = nullptr;
          cudaError_t ce = cudaStreamEndCapture(st, &g);
          if (rc) return rc;
          if (ce != cudaSuccess)
            return fail(kCudaError, std::string("graph capture: ") + cudaGetErrorString(ce));
          e->graph = g;
          SNB_CUDA_TRY(cudaGraphInstantiate(&e->graph_exec, g, 0));
          e->g_crd = crd;
          e->g_vel = vel;
          e->g_invm = invm;
          e->g_dt = dt;
          e->g_stream = st;
          e->g_vel_wait = e->vel_wait;
        }
        SNB_CUDA_TRY(cudaGraphLaunch(e->graph_exec, st));
      } else {
        int rc = engine_md_step(e, crd, vel, invm, dt, step, forced, st);
        if (rc) return rc;
      }
      e->steps_done++;
    }
    if (s + chunk == steps) {
      const size_t b3 = sizeof(float) * 3 * e->n;
      if (h_crd_out && h_vel_out == h_crd_out + 3 * (size_t)e->n && vel == crd + 3 * (size_t)e->n) {
        SNB_CUDA_TRY(cudaMemcpyAsync(h_crd_out, crd, 2 * b3, cudaMemcpyDeviceToHost, st));
      } else {
        if (h_crd_out)
          SNB_CUDA_TRY(cudaMemcpyAsync(h_crd_out, crd, b3, cudaMemcpyDeviceToHost, st));
        if (h_vel_out)
          SNB_CUDA_TRY(cudaMemcpyAsync(h_vel_out, vel, b3, cudaMemcpyDeviceToHost, st));
      }
    }
    bool regrown = false;
    int rc = nl_check_overflow(e->nl, &regrown, st);
    if (rc) return rc;
    if (e->vatom) {
      int bad = 0;
      if ((rc = vatom_status(e->vatom, &bad, st))) return rc;
      if (bad)
        return fail(kBadInput, "virtual atom record " + std::to_string(bad - 1) +
                                   ": the direction of a type-3 site has zero length");
    }
    if (e->settle) {
      int bad = 0;
      SNB_CUDA_TRY(cudaMemcpyAsync(&bad, e->settle->s.d_err, sizeof(int),
                                   cudaMemcpyDeviceToHost, st));
      SNB_CUDA_TRY(cudaStreamSynchronize(st));
      if (bad)
        return fail(kBadInput, "SETTLE: rigid pair " + std::to_string(bad - 1) +
                                   " has no real position update; reduce the time step or "
                                   "minimise the input");
    }
    if (regrown) {
      if (e->opt.nl_throw_error_when_overflow)
        return fail(kOverflow, "neighbor list overflow");
      if (++retries > 8) return fail(kOverflow, "neighbor list overflow persists");
      if (e->graph_exec) {  // the graph holds the old list pointer
        cudaGraphExecDestroy(e->graph_exec);
        cudaGraphDestroy(e->graph);
        e->graph_exec = nullptr;
      }
      SNB_CUDA_TRY(cudaMemcpyAsync(crd, e->d_snap_crd, sizeof(float) * 3 * e->n,
                                   cudaMemcpyDeviceToDevice, st));
      SNB_CUDA_TRY(cudaMemcpyAsync(vel, e->d_snap_vel, sizeof(float) * 3 * e->n,
                                   cudaMemcpyDeviceToDevice, st));
      e->steps_done = 0;  // forces a rebuild on the next step
      continue;
    }
    s += chunk;
  }
  return kOk;
}

extern "C" int snb_engine_md_steps(snb_engine* e, float* crd, float* vel,
                                   const float* invm, float dt, int first, int steps,
                                   void* stream) {
  if (!e || !crd || !vel || !invm) return fail(kBadInput, "engine_md_steps: bad argument");
  return engine_run(e, crd, vel, invm, dt, first, steps, S(stream), false);
}

extern "C" int snb_engine_md_steps_graph(snb_engine* e, float* crd, float* vel,
                                         const float* invm, float dt, int first,
                                         int steps, void* stream) {
  if (!e || !crd || !vel || !invm) return fail(kBadInput, "engine_md_steps: bad argument");
  if (S(stream) == nullptr)
    return fail(kBadInput, "graph replay needs a non-default stream");
  bool graphable = e->opt.nl_refresh_interval <= 0 && e->pme.update_interval == 1;
  return engine_run(e, crd, vel, invm, dt, first, steps, S(stream), graphable);
}

extern "C" int snb_engine_md_steps_host(snb_engine* e, float* h_crd, float* h_vel,
                                        float* crd, float* vel, const float* invm, float dt,
                                        int first, int steps, void* stream) {
  if (!e || !h_crd || !h_vel || !crd || !vel || !invm || steps < 0)
    return fail(kBadInput, "engine_md_steps_host: bad argument");
  cudaStream_t st = S(stream);
  if (st == nullptr) return fail(kBadInput, "engine_md_steps_host: needs a non-default stream");
  const size_t bytes = sizeof(float) * 3 * (size_t)e->n;
  if (steps == 0) {
    SNB_CUDA_TRY(cudaMemcpyAsync(crd, h_crd, bytes, cudaMemcpyHostToDevice, st));
    SNB_CUDA_TRY(cudaMemcpyAsync(vel, h_vel, bytes, cudaMemcpyHostToDevice, st));
    return kOk;
  }
  // the coordinates first: the forces need them.  The velocities follow on
  // the link while the forces are computed (the copies are issued one after
  // the other, so the coordinates get the link's full bandwidth), and the
  // first update waits for them.
  SNB_CUDA_TRY(cudaMemcpyAsync(crd, h_crd, bytes, cudaMemcpyHostToDevice, st));
  SNB_CUDA_TRY(cudaEventRecord(e->ev_crd_in, st));
  SNB_CUDA_TRY(cudaStreamWaitEvent(e->io, e->ev_crd_in, 0));
  SNB_CUDA_TRY(cudaMemcpyAsync(vel, h_vel, bytes, cudaMemcpyHostToDevice, e->io));
  SNB_CUDA_TRY(cudaMemcpyAsync(e->d_snap_vel, vel, bytes, cudaMemcpyDeviceToDevice, e->io));
  SNB_CUDA_TRY(cudaEventRecord(e->ev_vel_in, e->io));
  bool graphable = e->opt.nl_refresh_interval <= 0 && e->pme.update_interval == 1;
  e->vel_wait = true;
  e->vel_snapped = true;
  int rc = engine_run(e, crd, vel, invm, dt, first, steps, st, graphable, h_crd, h_vel);
  e->vel_wait = false;
  e->vel_snapped = false;
  if (rc) {
    cudaStreamSynchronize(e->io);
    return rc;
  }
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  return kOk;
}

// Stream-launched steps with CUDA events between phases; h_phase_ms gets the
// mean per step of {neighbor update, pack, pair kernel, excluded correction,
// PME reciprocal, bonded, integration}.  Synchronises after every step.
extern "C" int snb_engine_profile_steps(snb_engine* e, float* crd, float* vel,
                                        const float* invm, float dt, int first,
                                        int steps, double* h_phase_ms, void* stream) {
  if (!e || !crd || !vel || !invm || !h_phase_ms || steps <= 0)
    return fail(kBadInput, "engine_profile_steps: bad argument");
  cudaStream_t st = S(stream);
  for (int k = 0; k < 8; ++k)
    if (!e->prof_ev[k]) SNB_CUDA_TRY(cudaEventCreate(&e->prof_ev[k]));
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  e->prof_on = true;
  for (int s = 0; s < steps; ++s) {
    bool forced = e->steps_done == 0;
    int rc = engine_md_step(e, crd, vel, invm, dt, first + s, forced, st);
    if (rc) {
      e->prof_on = false;
      return rc;
    }
    e->steps_done++;
    SNB_CUDA_TRY(cudaEventSynchronize(e->prof_ev[7]));
    for (int k = 0; k < 7; ++k) {
      float ms = 0.f;
      SNB_CUDA_TRY(cudaEventElapsedTime(&ms, e->prof_ev[k], e->prof_ev[k + 1]));
      acc[k] += ms;
    }
  }
  e->prof_on = false;
  for (int k = 0; k < 7; ++k) h_phase_ms[k] = acc[k] / steps;
  return kOk;
}

// Times `steps` stream-launched steps from the same starting coordinates for
// each candidate launch shape and keeps the fastest: the pair kernel's scan
// unroll (2, 4, 8) and blocks per SM (occupancy maximum, 2, 3) by the whole
// step (the PME branch shares the SMs with it), the pair
// search's blocks per SM (4, 8, 16; a rebuild is forced every step), and the
// gather's threads per block (128, 256, 512).  crd / vel are restored.
extern "C" int snb_engine_autotune(snb_engine* e, float* crd, float* vel,
                                   const float* invm, float dt, int steps, int* h_choice,
                                   void* stream) {
  if (!e || !crd || !vel || !invm || steps <= 0)
    return fail(kBadInput, "engine_autotune: bad argument");
  if (e->accum != kAccumFixed) return fail(kNotSupported, "autotune: fixed point only");
  cudaStream_t st = S(stream);
  const size_t bytes = sizeof(float) * 3 * e->n;
  float *c0 = nullptr, *v0 = nullptr;
  SNB_CUDA_TRY(cudaMalloc(&c0, bytes));
  SNB_CUDA_TRY(cudaMalloc(&v0, bytes));
  SNB_CUDA_TRY(cudaMemcpyAsync(c0, crd, bytes, cudaMemcpyDeviceToDevice, st));
  SNB_CUDA_TRY(cudaMemcpyAsync(v0, vel, bytes, cudaMemcpyDeviceToDevice, st));
  for (int k = 0; k < 8; ++k)
    if (!e->prof_ev[k]) SNB_CUDA_TRY(cudaEventCreate(&e->prof_ev[k]));
  // mean ms over the steps, from the saved coordinates, of phase `ph`
  // (between prof_ev[ph] and prof_ev[ph + 1], phases run one after another),
  // or with ph < 0 of the whole step as the MD loop runs it (branches
  // concurrent); force_nl: rebuild every step
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  SNB_CUDA_TRY(cudaEventCreate(&t0));
  SNB_CUDA_TRY(cudaEventCreate(&t1));
  // Every step starts from the saved frame, so that each measures the same
  // work and no list rebuild falls into a window by chance (one costs about
  // two steps).
  auto measure = [&](int ph, bool force_nl, double* ms) -> int {
    double acc = 0.0;
    e->prof_on = ph >= 0;
    for (int s = -1; s < steps; ++s) {  // s = -1: untimed warm-up step
      SNB_CUDA_TRY(cudaMemcpyAsync(crd, c0, bytes, cudaMemcpyDeviceToDevice, st));
      SNB_CUDA_TRY(cudaMemcpyAsync(vel, v0, bytes, cudaMemcpyDeviceToDevice, st));
      SNB_CUDA_TRY(cudaEventRecord(t0, st));
      int rc = engine_md_step(e, crd, vel, invm, dt, 1 + s, force_nl || s < 0, st);
      if (rc) {
        e->prof_on = false;
        return rc;
      }
      SNB_CUDA_TRY(cudaEventRecord(t1, st));
      SNB_CUDA_TRY(cudaEventSynchronize(t1));
      float m = 0.f;
      if (ph >= 0)
        SNB_CUDA_TRY(cudaEventElapsedTime(&m, e->prof_ev[ph], e->prof_ev[ph + 1]));
      else
        SNB_CUDA_TRY(cudaEventElapsedTime(&m, t0, t1));
      if (s >= 0) acc += m;
    }
    e->prof_on = false;
    *ms = acc / steps;
    return kOk;
  };
  // the whole step as the MD loop runs it: one step graph captured for the
  // candidate and replayed, each replay from the saved frame
  // (stream-launched steps where the stream cannot be captured)
  auto measure_step = [&](double* ms) -> int {
    if (st == nullptr) return measure(-1, false, ms);
    SNB_CUDA_TRY(cudaMemcpyAsync(crd, c0, bytes, cudaMemcpyDeviceToDevice, st));
    SNB_CUDA_TRY(cudaMemcpyAsync(vel, v0, bytes, cudaMemcpyDeviceToDevice, st));
    int rc = engine_md_step(e, crd, vel, invm, dt, 0, true, st);  // list from the frame
    if (rc) return rc;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    SNB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = engine_md_step(e, crd, vel, invm, dt, 1, false, st, true);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (!rc && ce == cudaSuccess) ce = cudaGraphInstantiate(&x, g, 0);
    if (rc || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return rc ? rc : fail(kCudaError, std::string("autotune capture: ") +
                                            cudaGetErrorString(ce));
    }
    double acc = 0.0;
    for (int s = -1; s < steps && !rc; ++s) {  // s = -1: untimed replay
      if (cudaMemcpyAsync(crd, c0, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
          cudaMemcpyAsync(vel, v0, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
          cudaEventRecord(t0, st) != cudaSuccess || cudaGraphLaunch(x, st) != cudaSuccess ||
          cudaEventRecord(t1, st) != cudaSuccess || cudaEventSynchronize(t1) != cudaSuccess) {
        rc = fail(kCudaError, "autotune: graph replay failed");
        break;
      }
      float m = 0.f;
      cudaEventElapsedTime(&m, t0, t1);
      if (s >= 0) acc += m;
    }
    cudaGraphExecDestroy(x);
    cudaGraphDestroy(g);
    *ms = acc / steps;
    return rc;
  };
  int rc = kOk;
  double best = 1e30, ms = 0.0;
  int bu = e->pair_unroll, bb = e->pair_blocks_per_sm;
  const bool rows = !(e->nl.clusters && !e->soft);
  // candidates per lane per round and rows in flight per block (the row
  // kernel of the plain single box) together, then blocks per SM
  int bw = e->pair_warps;
  const bool warps_knob = rows && !e->soft;
  for (int u : {2, 4, 8})
    for (int w : {4, 8, 16}) {
      if (rc) break;
      if (!rows && u != bu) continue;  // the cluster kernel has no unroll choice
      if ((!warps_knob && w != bw) || (e->nsys > 0 && w == 4)) continue;
      e->pair_unroll = u;
      e->pair_warps = w;
      e->pair_blocks_per_sm = 0;
      if ((rc = measure_step(&ms))) break;  // the step, PME branch alongside
      if (ms < best) {
        best = ms;
        bu = u;
        bw = w;
      }
    }
  e->pair_unroll = bu;
  e->pair_warps = bw;
  bb = 0;  // the joint search above ran at the occupancy maximum
  for (int b : {2, 3}) {
    if (rc) break;
    e->pair_blocks_per_sm = b;
    if ((rc = measure_step(&ms))) break;
    if (ms < best) {
      best = ms;
      bb = b;
    }
  }
  e->pair_blocks_per_sm = bb;
  // the hit stash (phase 2 without gathers), same kernel otherwise
  bool bst = e->pair_stash;
  if (!rc && rows && !e->soft && e->nsys == 0) {
    best = 1e30;
    for (bool sx : {false, true}) {
      e->pair_stash = sx;
      if ((rc = measure_step(&ms))) break;
      if (ms < best) {
        best = ms;
        bst = sx;
      }
    }
  }
  e->pair_stash = bst;
  int bs = e->nl.search_blocks_per_sm;
  best = 1e30;
  for (int b : {4, 8, 16}) {
    if (rc) break;
    e->nl.search_blocks_per_sm = b;
    if ((rc = measure(0, true, &ms))) break;
    if (ms < best) {
      best = ms;
      bs = b;
    }
  }
  e->nl.search_blocks_per_sm = bs;
  int bg = e->pme.gather_threads;
  best = 1e30;
  for (int gt : {128, 256, 512}) {
    if (rc) break;
    e->pme.gather_threads = gt;
    if ((rc = measure_step(&ms))) break;
    if (ms < best) {
      best = ms;
      bg = gt;
    }
  }
  e->pme.gather_threads = bg;
  // spread tile shape: edge and warps per tile (one box), timed as the whole
  // step with the PME chain beside the pair kernel
  int bt = e->pme.spread_atomic ? 0 : e->pme.T;
  int bsw = e->pme.spread_atomic ? 0 : e->pme.spread_warps;
  if (!rc && e->nsys == 0 && e->pme.reciprocal) {
    best = 1e30;
    // (edge 16 is left out: its 8^3 octants' bound on the int32 sums sits
    // near the range in a liquid, so whether tiles are taken again with
    // int64 sums depends on the frame)
    const int shapes[4][2] = {{8, 1}, {8, 2}, {8, 4}, {0, 0}};
    for (const auto& sh : shapes) {
      if ((rc = pme_set_spread_shape(e->pme, sh[0], sh[1]))) break;
      if ((rc = measure_step(&ms))) break;
      if (ms < best) {
        best = ms;
        bt = sh[0];
        bsw = sh[1];
      }
    }
    if (!rc) rc = pme_set_spread_shape(e->pme, bt, bsw);
  }
  // the convolution's FFT: cuFFT or the own passes (where the grid allows)
  bool bfft = e->pme.own_fft;
  if (!rc && e->pme.reciprocal) {
    best = 1e30;
    for (bool own : {false, true}) {
      if (pme_set_own_fft(e->pme, own)) {  // grid not supported: cuFFT only
        set_error("");
        continue;
      }
      if ((rc = measure_step(&ms))) break;
      if (ms < best) {
        best = ms;
        bfft = own;
      }
    }
    if (!rc) rc = pme_set_own_fft(e->pme, bfft);
  }
  cudaMemcpyAsync(crd, c0, bytes, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(vel, v0, bytes, cudaMemcpyDeviceToDevice, st);
  cudaStreamSynchronize(st);
  cudaFree(c0);
  cudaFree(v0);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (rc) return rc;
  e->steps_done = 0;  // the next step rebuilds the list for the restored frame
  if (e->graph_exec) {  // recapture with the chosen shapes
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
  }
  if (h_choice) {
    h_choice[0] = e->pair_unroll;
    h_choice[1] = e->pair_blocks_per_sm;
    h_choice[2] = e->nl.search_blocks_per_sm;
    h_choice[3] = e->pme.gather_threads;
    h_choice[4] = e->pair_warps;
    h_choice[5] = e->pme.spread_atomic ? 0 : e->pme.T;
    h_choice[6] = e->pme.spread_atomic ? 0 : e->pme.spread_warps;
    h_choice[7] = e->pair_stash ? 1 : 0;
    h_choice[8] = e->pme.own_fft ? 1 : 0;
  }
  return kOk;
}

extern "C" int snb_engine_set_launch_shapes(snb_engine* e, const int* h_choice) {
  if (!e || !h_choice) return fail(kBadInput, "engine_set_launch_shapes: bad argument");
  const int u = h_choice[0], b = h_choice[1], sb = h_choice[2], gt = h_choice[3];
  const int w = h_choice[4], T = h_choice[5], sw = h_choice[6], sx = h_choice[7];
  const int ff = h_choice[8];
  if ((u != 2 && u != 4 && u != 8) || b < 0 || b > 32 || (sb != 4 && sb != 8 && sb != 16) ||
      (gt != 128 && gt != 256 && gt != 512) || (w != 4 && w != 8 && w != 16) ||
      (sx != 0 && sx != 1) || (ff != 0 && ff != 1))
    return fail(kBadInput, "engine_set_launch_shapes: a shape outside the tuned set");
  if (e->nsys == 0) {
    int rc = pme_set_spread_shape(e->pme, T, sw);
    if (!rc) rc = pme_set_own_fft(e->pme, ff != 0);
    if (rc) return rc;
  } else if (T != e->pme.T || sw != e->pme.spread_warps || e->pme.spread_atomic) {
    return fail(kNotSupported,
                "engine_set_launch_shapes: the spread shape of a batch is fixed");
  } else {
    int rc = pme_set_own_fft(e->pme, ff != 0);
    if (rc) return rc;
  }
  e->pair_unroll = u;
  e->pair_blocks_per_sm = b;
  e->nl.search_blocks_per_sm = sb;
  e->pme.gather_threads = gt;
  e->pair_warps = w;
  e->pair_stash = sx != 0;
  if (e->graph_exec) {  // recapture with these shapes
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
  }
  return kOk;
}

// Kernel nodes in the captured one-step graph: all, and those that belong to
// cuFFT (counted from a graph holding only the two transforms).
extern "C" int snb_engine_graph_info(snb_engine* e, int* kernel_nodes,
                                     int* library_kernel_nodes, int* rebuild_kernel_nodes,
                                     void* stream) {
  if (!e || !kernel_nodes || !library_kernel_nodes)
    return fail(kBadInput, "engine_graph_info: bad argument");
  if (rebuild_kernel_nodes) *rebuild_kernel_nodes = e->body_kernels;
  auto count = [](cudaGraph_t g, int* out) -> int {
    size_t nn = 0;
    SNB_CUDA_TRY(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    SNB_CUDA_TRY(cudaGraphGetNodes(g, nodes.data(), &nn));
    int k = 0;
    for (auto nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) {
        cudaGetLastError();  // node types this runtime cannot name: not kernels
        continue;
      }
      k += t == cudaGraphNodeTypeKernel;
    }
    *out = k;
    return kOk;
  };
  if (!e->graph) return fail(kBadInput, "engine_graph_info: no graph captured yet");
  int rc = count(e->graph, kernel_nodes);
  if (rc) return rc;
  cudaStream_t st = S(stream);
  cudaGraph_t g = nullptr;
  PME& p = e->pme;
  if (p.own_fft || !p.reciprocal) {  // no cuFFT kernel in the step
    *library_kernel_nodes = 0;
    return kOk;
  }
  if (p.bv.nsys > 0) {  // a batch: one plan pair per grid size
    for (auto& fg : p.groups) {
      cufftSetStream(fg.r2c, st);
      cufftSetStream(fg.c2r, st);
    }
    SNB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (auto& fg : p.groups) {
      cufftExecR2C(fg.r2c, p.d_Q + fg.grid_begin, p.d_FQ + fg.spec_begin);
      cufftExecC2R(fg.c2r, p.d_FQ + fg.spec_begin, p.d_phi + fg.grid_begin);
    }
  } else {
    cufftSetStream(p.plan_r2c, st);
    cufftSetStream(p.plan_c2r, st);
    SNB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cufftExecR2C(p.plan_r2c, p.d_Q, p.d_FQ);
    cufftExecC2R(p.plan_c2r, p.d_FQ, p.d_phi);
  }
  SNB_CUDA_TRY(cudaStreamEndCapture(st, &g));
  rc = count(g, library_kernel_nodes);
  cudaGraphDestroy(g);
  return rc;
}

extern "C" int snb_engine_set_list_form(snb_engine* e, int clusters) {
  if (!e) return fail(kBadInput, "engine_set_list_form: null handle");
  if (clusters && e->soft)
    return fail(kNotSupported, "engine_set_list_form: the soft-core kernel reads rows");
  int rc = nl_set_clusters(e->nl, clusters != 0);
  if (rc) return rc;
  if (e->graph_exec) {  // the captured step holds the previous list form
    cudaGraphExecDestroy(e->graph_exec);
    cudaGraphDestroy(e->graph);
    e->graph_exec = nullptr;
    e->graph = nullptr;
  }
  e->steps_done = 0;
  return kOk;
}

extern "C" int snb_engine_set_prune_margin(snb_engine* e, float margin) {
  if (!e) return fail(kBadInput, "engine_set_prune_margin: null handle");
  if (!(margin >= 0.f) || margin > 100.f)
    return fail(kBadInput, "engine_set_prune_margin: margin must be in [0, 100] A");
  if (margin > 0.f) {
    int rc = nl_enable_prune(e->nl);
    if (rc) return rc;
    if (!e->d_prune) {
      SNB_CUDA_TRY(cudaMalloc(&e->d_prune, sizeof(int) * 4));
      const int init[4] = {0, 1, -1, 0};  // the first step prunes
      SNB_CUDA_TRY(cudaMemcpy(e->d_prune, init, sizeof(init), cudaMemcpyHostToDevice));
    }
  }
  if (margin != e->prune_margin) {
    if (e->d_prune) {
      const int one = 1;  // rows kept at another margin are redone
      SNB_CUDA_TRY(cudaMemcpy(e->d_prune + 1, &one, sizeof(int), cudaMemcpyHostToDevice));
    }
    if (e->graph_exec) {  // the captured step holds the previous choice
      cudaGraphExecDestroy(e->graph_exec);
      cudaGraphDestroy(e->graph);
      e->graph_exec = nullptr;
      e->graph = nullptr;
    }
  }
  e->prune_margin = margin;
  return kOk;
}

extern "C" int snb_engine_prune_passes(snb_engine* e, int* passes, long long* kept_entries,
                                       void* stream) {
  if (!e || !passes) return fail(kBadInput, "engine_prune_passes: null argument");
  *passes = 0;
  if (kept_entries) *kept_entries = 0;
  if (!e->d_prune) return kOk;
  cudaStream_t st = S(stream);
  SNB_CUDA_TRY(cudaMemcpyAsync(passes, e->d_prune + 3, sizeof(int), cudaMemcpyDeviceToHost,
                               st));
  std::vector<int> kept;
  if (kept_entries) {
    kept.resize(e->n);
    SNB_CUDA_TRY(cudaMemcpyAsync(kept.data(), e->nl.d_row_in_count, sizeof(int) * e->n,
                                 cudaMemcpyDeviceToHost, st));
  }
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  if (kept_entries)
    for (int c : kept) *kept_entries += c;
  return kOk;
}

extern "C" int snb_engine_list_form(snb_engine* e, int* clusters) {
  if (!e || !clusters) return fail(kBadInput, "engine_list_form: null argument");
  *clusters = e->nl.clusters && !e->soft ? 1 : 0;
  return kOk;
}

extern "C" int snb_engine_export_pairs(snb_engine* e, int* d_pi, int* d_pj, long long cap,
                                       long long* count, void* stream) {
  if (!e || !count) return fail(kBadInput, "engine_export_pairs: null argument");
  return nl_export_pairs(e->nl, d_pi, d_pj, cap, count, S(stream));
}

extern "C" int snb_engine_spread_wide_tiles(snb_engine* e, int* count, void* stream) {
  if (!e || !count) return fail(kBadInput, "engine_spread_wide_tiles: null argument");
  return pme_wide_tiles(e->pme, count, S(stream));
}

extern "C" int snb_engine_stats(snb_engine* e, long long* rebuilds, long long* pairs,
                                void* stream) {
  if (!e) return fail(kBadInput, "engine_stats: null handle");
  bool regrown;
  int rc = nl_check_overflow(e->nl, &regrown, S(stream));
  if (rc) return rc;
  if (rebuilds) *rebuilds = e->nl.h_flags[3];
  if (pairs) *pairs = e->nl.last_total;
  return kOk;
}

extern "C" int snb_engine_destroy(snb_engine* e) {
  if (!e) return kOk;
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  for (int k = 0; k < 8; ++k)
    if (e->prof_ev[k]) cudaEventDestroy(e->prof_ev[k]);
  if (e->side) cudaStreamDestroy(e->side);
  if (e->branch) cudaStreamDestroy(e->branch);
  if (e->ev_fork) cudaEventDestroy(e->ev_fork);
  if (e->ev_join) cudaEventDestroy(e->ev_join);
  if (e->branch2) cudaStreamDestroy(e->branch2);
  if (e->ev_join2) cudaEventDestroy(e->ev_join2);
  if (e->io) cudaStreamDestroy(e->io);
  if (e->ev_crd_in) cudaEventDestroy(e->ev_crd_in);
  if (e->ev_vel_in) cudaEventDestroy(e->ev_vel_in);
  nl_free(e->nl);
  pme_free(e->pme);
  acc_free(e->acc);
  cudaFree(e->lj.d_A);
  cudaFree(e->lj.d_B);
  cudaFree(e->lj.d_type);
  cudaFree(e->d_pos);
  cudaFree(e->d_type_sorted);
  cudaFree(e->d_charge);
  cudaFree(e->d_excl_start);
  cudaFree(e->d_excl_numbers);
  cudaFree(e->d_excl_list);
  cudaFree(e->d_isum);
  cudaFree(e->d_bonded_e);
  cudaFree(e->d_nb14_sums);
  cudaFree(e->d_kin);
  cudaFree(e->d_totals_scratch);
  cudaFree(e->d_snap_crd);
  cudaFree(e->d_snap_vel);
  cudaFree(e->d_sys);
  cudaFree(e->d_sys_of);
  cudaFree(e->d_cell_sys);
  cudaFree(e->d_box_need);
  cudaFree(e->d_prune);
  for (void* p : {(void*)e->d_ba, (void*)e->d_bb, (void*)e->d_bk, (void*)e->d_br0,
                  (void*)e->d_aa, (void*)e->d_ab, (void*)e->d_ac, (void*)e->d_ak,
                  (void*)e->d_at0})
    cudaFree(p);
  delete e;
  return kOk;
}
