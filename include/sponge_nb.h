/* sponge_nb.h -- C ABI of the B200 (sm_100a) nonbonded hot path.
 *
 * Drop-in boundary for SPONGE's NEIGHBOR_LIST, LENNARD_JONES_INFORMATION,
 * LJ_SOFT_CORE and Particle_Mesh modules.  Every module entry point below
 * replaces one member function of those structs (file:line in the SPONGE
 * source tree given beside it); arguments keep the reference's meaning and
 * order.  Differences that follow from being a C ABI:
 *   - `Boundary` is passed as snb_boundary (same fields: policy, cell, rcell);
 *   - VECTOR* / LTMatrix3* are float* with 3 / 6 floats per atom;
 *   - each call takes the CUDA stream to run on (NULL = legacy default
 *     stream, what the reference uses) and returns a status code instead of
 *     calling Throw_SPONGE_Error; snb_last_error() gives the message;
 *   - the input keys the modules read from CONTROLLER are set on an
 *     snb_options with snb_options_set() using the same key names.
 * All pointer arguments of compute calls are device pointers unless named
 * h_*.  Compute calls neither allocate nor synchronise, so they can be
 * captured in a CUDA graph, except where a comment says otherwise.
 *
 * Accumulation: compute calls add (+=) into frc / atom_energy / atom_virial
 * like the reference.  Internally each module accumulates in 64-bit fixed
 * point (forces 2^40 per kcal/mol/A, energies and virials 2^32 per kcal/mol)
 * so results do not depend on thread order, or, with
 * accumulation = SNB_ACCUM_FLOAT, with float atomics (the plain path).
 */
#ifndef SPONGE_NB_H
#define SPONGE_NB_H
#ifdef __cplusplus
extern "C" {
#endif

#define SNB_VERSION 1

/* status codes */
#define SNB_OK 0
#define SNB_ERR_BAD_INPUT 1
#define SNB_ERR_CUDA 2
#define SNB_ERR_OVERFLOW 3
#define SNB_ERR_TIMEOUT 4
#define SNB_ERR_NOT_SUPPORTED 5

#define SNB_ACCUM_FIXED64 0
#define SNB_ACCUM_FLOAT 1

/* NEIGHBOR_LIST::Update `update` argument (neighbor_list.h:112-116) */
#define SNB_CONDITIONAL_UPDATE 0
#define SNB_FORCED_UPDATE 1

/* Boundary (utils/boundary.h:15-20): policy 0 open, 1 periodic; cell and
 * rcell as LTMatrix3 {a11, a21, a22, a31, a32, a33}. */
typedef struct snb_boundary {
    int policy;
    float cell[6];
    float rcell[6];
} snb_boundary;

/* Input keys of the hot-path modules (docs/input-reference; defaults as the
 * reference).  snb_options_set() accepts the reference key names:
 *   cutoff, skin                                   (MD_core/nb.hpp:5-27)
 *   neighbor_list_refresh_interval, neighbor_list_skin_permit,
 *   neighbor_list_max_neighbor_numbers, neighbor_list_max_atom_in_grid_numbers,
 *   neighbor_list_max_ghost_in_grid_numbers,
 *   neighbor_list_check_overflow_interval,
 *   neighbor_list_throw_error_when_overflow        (neighbor_list.cpp:276-305,
 *                                                   885-940)
 *   PM_fftx, PM_ffty, PM_fftz, PM_grid_spacing, PM_Direct_Tolerance,
 *   PME_update_interval, PME_calculate_reciprocal_part,
 *   PME_calculate_excluded_part                    (PM_force.cpp:315-503)
 *   lambda_lj, soft_core_alpha, soft_core_powfer, soft_core_sigma,
 *   soft_core_sigma_min                            (LJ_soft_core.cpp:496-558)
 *   DOM_DEC_update_interval: the MD loop's forced neighbor rebuild period
 *                                                  (Domain_decomposition.cpp:33-39,
 *                                                   main.cpp:1805-1822)
 * plus this library's own key `accumulation` = fixed64 | float. */
typedef struct snb_options {
    float cutoff;
    float skin;
    int nl_refresh_interval;
    float nl_skin_permit;
    int nl_max_neighbor_numbers;
    int nl_max_atom_in_grid_numbers;
    int nl_max_ghost_in_grid_numbers;
    int nl_check_overflow_interval;
    int nl_throw_error_when_overflow;
    int pm_fftx, pm_ffty, pm_fftz;
    float pm_grid_spacing;
    float pm_direct_tolerance;
    int pme_update_interval;
    int pme_calculate_reciprocal_part;
    int pme_calculate_excluded_part;
    float lambda_lj;
    float soft_core_alpha;
    float soft_core_powfer;
    float soft_core_sigma;
    float soft_core_sigma_min;
    int accumulation;
    int dom_dec_update_interval;
} snb_options;

typedef struct snb_nl snb_nl;
typedef struct snb_lj snb_lj;
typedef struct snb_lj_soft snb_lj_soft;
typedef struct snb_pme snb_pme;
typedef struct snb_engine snb_engine;
typedef struct snb_nb14 snb_nb14;
typedef struct snb_settle snb_settle;
typedef struct snb_bond snb_bond;
typedef struct snb_angle snb_angle;
typedef struct snb_vatom snb_vatom;

/* ---------------------------------------------------------------- misc */
int snb_version(void);
/* No counterpart in the reference: a self-check of the pair kernels'
 * screened-Coulomb factors.  For each x = d_x[i] >= 0 writes d_out[4i..4i+3]
 * = {erfc(x), exp(-x^2)} as the pair kernels form them (erfc from a
 * polynomial in 1/(1 + x/2) times exp(-x^2) for x <= 4) and CUDA's
 * {erfcf(x), expf(-x^2)}, so tests can hold the two against each other and
 * against double precision. */
int snb_check_erfc_exp(int n, const float* d_x, float* d_out, void* stream);
const char* snb_last_error(void);
void snb_options_default(snb_options* opt);
int snb_options_set(snb_options* opt, const char* key, const char* value);

/* ------------------------------------------------------- NEIGHBOR_LIST */
/* NEIGHBOR_LIST::Initial (neighbor_list.h:17-18, neighbor_list.cpp:871-972) */
int snb_nl_create(const snb_options* opt, int atom_numbers, float cutoff,
                  float skin, snb_boundary boundary, snb_nl** out);
/* NEIGHBOR_LIST::Update (neighbor_list.h:19-22, neighbor_list.cpp:974-1025).
 * crd: float[3*N].  ghost_numbers must be 0 (one domain).  A rectangular
 * box that differs from the last one redraws the cell grid by the
 * reference's rule and forces the rebuild (a barostat's box change; the
 * reference re-initialises the list for a large change, main.cpp:2092). */
int snb_nl_update(snb_nl* nl, const int* atom_local, int local_atom_numbers,
                  int ghost_numbers, const float* crd, snb_boundary boundary,
                  int step, int update, const int* excluded_list_start,
                  const int* excluded_list, const int* excluded_numbers,
                  void* stream);
/* NEIGHBOR_LIST::Check_Overflow (neighbor_list.cpp:1027-1103): reads the
 * overflow flag (host sync) and regrows the pair storage; *regrown = 1 when
 * the last build overflowed and must be repeated (forced update). */
int snb_nl_check_overflow(snb_nl* nl, int* regrown, void* stream);
/* Number of listed pairs of the last build (host sync). */
int snb_nl_pair_count(snb_nl* nl, long long* count, void* stream);
/* The pair set as (global_i < global_j) pairs, unsorted (host sync). */
int snb_nl_export_pairs(snb_nl* nl, int* d_pair_i, int* d_pair_j,
                        long long capacity, long long* count, void* stream);
/* NEIGHBOR_LIST::d_nl in the reference layout (neighbor_list.h:42-44,
 * ATOM_GROUP {int atom_numbers; int ghost_numbers; int* atom_serial;},
 * common.h:177-182): d_nl[N] rows point into d_serial_slab[N*max]; row i
 * lists local j with atom_local[j] > atom_local[i].  Host sync. */
int snb_nl_export_atom_groups(snb_nl* nl, void* d_nl, int* d_serial_slab,
                              int max_neighbor_numbers, void* stream);
/* NEIGHBOR_LIST::Clear (neighbor_list.cpp:1105-1119) */
int snb_nl_destroy(snb_nl* nl);

/* ------------------------------------------- LENNARD_JONES_INFORMATION */
/* LENNARD_JONES_INFORMATION::Initial (Lennard_Jones_force.h:118-119,
 * Lennard_Jones_force.cpp:147-250).  The type table replaces the Xponge
 * LennardJones record: h_LJ_A/h_LJ_B are A'=12A, B'=6B per triangular pair
 * index, as Xponge leaves them. */
int snb_lj_create(const snb_options* opt, int atom_numbers,
                  int atom_type_numbers, const int* h_atom_LJ_type,
                  const float* h_LJ_A, const float* h_LJ_B, float cutoff,
                  snb_lj** out);
/* LENNARD_JONES_INFORMATION::Get_Local (Lennard_Jones_force.h:135-136) */
int snb_lj_get_local(snb_lj* lj, const int* atom_local, int local_atom_numbers,
                     int ghost_numbers, void* stream);
/* LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (Lennard_Jones_force.h:139-145, Lennard_Jones_force.cpp:326-384).  `nl` is
 * the neighbor list handle whose d_nl the reference would pass.  With
 * solvent_numbers > 0 the pairs of two atoms of the trailing water block
 * (the last solvent_numbers atoms) are left to
 * snb_solvent_lj_pme_direct_force, as the reference leaves the rows of those
 * atoms to SOLVENT_LENNARD_JONES.  ghost_numbers must be 0. */
int snb_lj_pme_direct_force(snb_lj* lj, int atom_numbers,
                            int local_atom_numbers, int solvent_numbers,
                            int ghost_numbers, const float* crd,
                            const float* charge, float* frc,
                            snb_boundary boundary, snb_nl* nl, float pme_beta,
                            int need_atom_energy, float* atom_energy,
                            int need_virial, float* atom_virial,
                            float* atom_direct_pme_energy, void* stream);
/* SOLVENT_LENNARD_JONES::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (solvent_LJ.h:23-42, solvent_LJ.cpp:256-432): the pairs between atoms of
 * the trailing water block (the last solvent_numbers atoms), which
 * snb_lj_pme_direct_force leaves out when given the same solvent_numbers
 * (main.cpp runs the two one after the other, 1453-1467).  It uses the LJ
 * handle's tables and the same list, and adds to frc, atom_energy,
 * atom_virial and atom_direct_pme_energy without clearing them. */
int snb_solvent_lj_pme_direct_force(snb_lj* lj, snb_nl* nl, int atom_numbers,
                                    int solvent_numbers, const float* crd,
                                    const float* charge, float* frc, snb_boundary boundary,
                                    float pme_beta, int need_atom_energy,
                                    float* atom_energy, int need_virial, float* atom_virial,
                                    float* atom_direct_pme_energy, void* stream);
/* LENNARD_JONES_INFORMATION::Long_Range_Correction (:168-170, .cpp:287-308) */
int snb_lj_long_range_correction(snb_lj* lj, int need_pressure, float* d_virial,
                                 int need_potential, float* d_potential,
                                 float volume, void* stream);
/* Step_Print's LJ_short sum (Lennard_Jones_force.cpp:386-400), host sync */
int snb_lj_energy_sum(snb_lj* lj, float* h_LJ_energy_sum, void* stream);
float snb_lj_long_range_factor(snb_lj* lj);
int snb_lj_destroy(snb_lj* lj);

/* -------------------------------------------------------- LJ_SOFT_CORE */
/* LJ_SOFT_CORE::Initial (LJ_soft_core.h:238-239, LJ_soft_core.cpp:463-688):
 * A/B end-state type tables and per-atom types, perturbation mask and the
 * soft-core parameters (lambda_lj, soft_core_alpha, soft_core_powfer,
 * soft_core_sigma, soft_core_sigma_min from opt). */
int snb_lj_soft_create(const snb_options* opt, int atom_numbers,
                       int atom_type_numbers_A, int atom_type_numbers_B,
                       const int* h_LJ_type_A, const int* h_LJ_type_B,
                       const float* h_LJ_AA, const float* h_LJ_AB,
                       const float* h_LJ_BA, const float* h_LJ_BB,
                       const int* h_subsys_mask, float cutoff,
                       snb_lj_soft** out);
/* LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial
 * (LJ_soft_core.h:247-254, LJ_soft_core.cpp:757-825).  charge_B_A is
 * charge_B - charge_A per atom (NULL if charges are not perturbed). */
int snb_lj_soft_pme_direct_force(snb_lj_soft* lj, int atom_numbers,
                                 int local_atom_numbers, int ghost_numbers,
                                 const float* crd, const float* charge,
                                 const float* charge_B_A, float* frc,
                                 snb_boundary boundary, snb_nl* nl,
                                 float pme_beta, int need_atom_energy,
                                 float* atom_energy, int need_virial,
                                 float* atom_virial,
                                 float* atom_direct_pme_energy, void* stream);
/* LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct
 * (LJ_soft_core.h:256-260, .cpp:827-888): dH/dlambda of the pair terms,
 * host sync. */
int snb_lj_soft_dh_dlambda(snb_lj_soft* lj, const float* crd,
                           const float* charge, const float* charge_B_A,
                           snb_boundary boundary, snb_nl* nl, float pme_beta,
                           int charge_perturbated, double* h_dH_dlambda,
                           void* stream);
/* LJ_SOFT_CORE::Long_Range_Correction (LJ_soft_core.h:262-264) */
int snb_lj_soft_long_range_correction(snb_lj_soft* lj, int need_pressure,
                                      float* d_virial, int need_potential,
                                      float* d_potential, float volume,
                                      void* stream);
/* LJ_SOFT_CORE::Step_Print sums (LJ_soft_core.cpp:890-921): h_sums[0..3] =
 * {LJ_soft_short, LJ_soft_inter, LJ_soft_intra, LJ_soft_long} from the last
 * energy evaluation and the last tail correction (host sync). */
int snb_lj_soft_energy_sums(snb_lj_soft* lj, float* h_sums, void* stream);
int snb_lj_soft_destroy(snb_lj_soft* lj);

/* ------------------------------------------------------- Particle_Mesh */
/* Particle_Mesh::Initial (PM_force.h:153-156, PM_force.cpp:295-654) */
int snb_pme_create(const snb_options* opt, int atom_numbers,
                   snb_boundary boundary, const float* box_length,
                   float cutoff, snb_pme** out);
float snb_pme_beta(snb_pme* pme);
int snb_pme_grid(snb_pme* pme, int* fft3);
/* Particle_Mesh::PME_Reciprocal_Force_With_Energy_And_Virial
 * (PM_force.h:175-178, PM_force.cpp:1070-1168): forces += into force;
 * self + reciprocal energy added to d_potential[0]; the reciprocal virial
 * added to d_virial[0..5]. */
int snb_pme_reciprocal_force(snb_pme* pme, const float* crd,
                             snb_boundary boundary, const float* charge,
                             float* force, int need_virial, int need_energy,
                             float* d_virial, float* d_potential, int step,
                             void* stream);
/* Particle_Mesh::MPI_PME_Excluded_Force_With_Atom_Energy
 * (PM_force.h:185-190, PM_force.cpp:1819-1842) */
int snb_pme_excluded_force(snb_pme* pme, int atom_numbers,
                           const int* atom_local, const int* atom_local_id,
                           const float* crd, snb_boundary boundary,
                           const float* charge, const int* excluded_list_start,
                           const int* excluded_list,
                           const int* excluded_atom_numbers, float* frc,
                           int need_energy, float* atom_ene, int need_virial,
                           float* atom_virial, void* stream);
/* Step_Print detail: reciprocal and self energies and the reciprocal virial
 * of the last energy/virial evaluation, FP64 (host sync). */
int snb_pme_energies(snb_pme* pme, double* h_reciprocal, double* h_self,
                     double* h_virial6, void* stream);
/* The spread step of PME_Q_Spread (PM_force.cpp:765-814) sums each grid
 * point's charge in int32 fixed point (2^22 per 18.2223-scaled charge unit,
 * so |Q| < 512 at a point) inside its 8x8x8 tile.  A bound on every point's
 * sum is kept per 4x4x4 octant of the tile (the atoms' |q| times the largest
 * B-spline weight product); a tile where it could reach the int32 range (far
 * above any dense liquid) is taken again with int64 sums, so the grid stays
 * exact.  *count = how many tiles were taken again since the handle was made
 * (host sync). */
int snb_pme_spread_wide_tiles(snb_pme* pme, int* count, void* stream);
/* Particle_Mesh::Update_Box (PM_force.h:180, PM_force.cpp:1171-1248): the
 * reciprocal part follows the new rectangular box in `boundary` at the same
 * grid size (the influence function and the neutralising term are formed
 * from the new cell and volume).  g (LTMatrix3 box-change rate) and dt only
 * move the reference's domain corners and are not used.  A box change large
 * enough to move the grid (main.cpp:2092-2124) re-creates the handle. */
int snb_pme_update_box(snb_pme* pme, snb_boundary boundary, const float* g, float dt);
int snb_pme_destroy(snb_pme* pme);

/* No counterpart in the reference.  The excluded-pair correction of
 * snb_pme_excluded_force (fixed-point accumulation, same results) for
 * callers that cannot allocate device memory while they run -- a loop
 * sharing the GPU with a caching allocator that holds the rest of HBM, or
 * one that must avoid the device-wide synchronisation of cudaMalloc/cudaFree
 * -- and that keep no snb_pme handle (pme_beta comes from the caller).  It
 * allocates nothing: its accumulator is a static device array of
 * SNB_NOALLOC_MAX_ATOMS atoms (6 MiB per device), and larger atom_numbers
 * are rejected with SNB_ERR_BAD_INPUT.  The array is shared by every call
 * on a device, so calls that may overlap in time (unordered streams,
 * concurrent threads) race and give wrong results: order them.  The array
 * must start at zero; the first call on each device clears it and each
 * completed call leaves it zero.  Every call looks up the array's address
 * in the current context; the first call on a device (which may load the
 * module) also enqueues the clear, so make it before any stream capture
 * begins.  After cudaDeviceReset, or in another context on the same device,
 * the array is a fresh one and a changed address is cleared again. */
#define SNB_NOALLOC_MAX_ATOMS 65536
int snb_pme_excluded_force_noalloc(int atom_numbers, const float* crd,
                                   snb_boundary boundary, const float* charge,
                                   float pme_beta,
                                   const int* excluded_list_start,
                                   const int* excluded_list,
                                   const int* excluded_atom_numbers, float* frc,
                                   int need_energy, float* atom_ene,
                                   int need_virial, float* atom_virial,
                                   void* stream);

/* ------------------------------------------------ fused force engine */
/* The whole nonbonded force of Main_Calculate_Force (main.cpp:1389-1544:
 * neighbor update, excluded correction, LJ + direct Coulomb, long-range LJ
 * correction, PME reciprocal) for one box, in one stream, one fixed-point
 * accumulator and one sorted frame: no host synchronisation, capturable in a
 * CUDA graph.  Host arrays are copied at creation. */
int snb_engine_create(const snb_options* opt, int atom_numbers,
                      snb_boundary boundary, int atom_type_numbers,
                      const int* h_atom_LJ_type, const float* h_LJ_A,
                      const float* h_LJ_B, const float* h_charge,
                      const int* h_excluded_list_start,
                      const int* h_excluded_numbers, const int* h_excluded_list,
                      int excluded_list_length, snb_engine** out);
/* No counterpart in the reference (it runs one system per process).  A batch
 * of n_systems independent rectangular boxes advanced together: the atoms of
 * system s are the next atoms_per_system[s] atoms of every per-atom array (all
 * systems share one LJ type table), box_lengths[3s..3s+2] is its box, and
 * exclusion indices are global atom indices that stay inside their system.
 * Every engine call below then acts on all systems at once, each step being
 * one launch per phase over all boxes (one neighbor list, one pair kernel,
 * one PME spread / gather with a grid per box, and for the convolution the
 * library's own passes, one launch per pass over all grids, where every
 * grid axis has 4-64 points (multiples of 4), else one batched cuFFT plan
 * per grid size).  Each box gets the single-box defaults: its own cell grid and
 * PME grid (by PM_grid_spacing); PME every step, displacement-triggered list
 * updates and fixed-point accumulation are required.  A list update starts
 * when an atom of some box moved more than half the skin since that box's
 * last build; it rebuilds that box's list and those of the boxes with an
 * atom past three quarters of that allowance, and keeps the others.
 * Energies and virials from snb_engine_force are sums over the systems. */
int snb_batch_create(const snb_options* opt, int n_systems,
                     const int* atoms_per_system, const float* box_lengths,
                     int atom_type_numbers, const int* h_atom_LJ_type,
                     const float* h_LJ_A, const float* h_LJ_B, const float* h_charge,
                     const int* h_excluded_list_start, const int* h_excluded_numbers,
                     const int* h_excluded_list, int excluded_list_length,
                     snb_engine** out);
/* frc (float[3N]) += nonbonded force at crd (float[3N]).  When need_energy /
 * need_virial, the FP64 totals are written to d_totals[0..7] =
 * {LJ, LJ long-range, direct Coulomb, excluded correction, PME reciprocal,
 *  PME self, (spare), potential sum} and d_totals[8..13] = virial tensor. */
int snb_engine_force(snb_engine* e, const float* crd, float* frc, int step,
                     int need_energy, int need_virial, double* d_totals,
                     void* stream);
/* Leap-frog NVE steps (MD_core/nve.hpp:3-16) of the same box with harmonic
 * bonds E = k(r-r0)^2 and angles E = k(theta-theta0)^2 (bond.cpp:14-60,
 * angle.cpp) on top of the nonbonded force: crd, vel updated in place. */
int snb_engine_set_bonded(snb_engine* e, int bond_numbers, const int* h_bond_a,
                          const int* h_bond_b, const float* h_bond_k,
                          const float* h_bond_r0, int angle_numbers,
                          const int* h_angle_a, const int* h_angle_b,
                          const int* h_angle_c, const float* h_angle_k,
                          const float* h_angle_theta0);
/* Box change of the engine's box (Main_Box_Change, main.cpp:2055-2090, for a
 * barostat): the neighbor grid is redrawn for the new lengths by the
 * reference's rule and the list is rebuilt at the next step; PME follows
 * Update_Box at the same grid size; the tail terms follow the new volume.
 * The caller scales the coordinates.  Single rectangular boxes. */
int snb_engine_update_box(snb_engine* e, snb_boundary boundary);
/* Soft-core LJ in the engine (main.cpp:1460-1465 runs LJ_SOFT_CORE in place
 * of the plain LJ module when it is initialised): the engine's pair step
 * takes the end-state tables, types, perturbation mask and lambda / alpha /
 * p / sigma of `soft` (created for the same atom count), and its tail
 * correction.  `soft` must outlive the engine's use of it; NULL turns the
 * plain LJ back on.  Single boxes, fixed-point accumulation. */
int snb_engine_set_soft_core(snb_engine* e, snb_lj_soft* soft);
/* 1-4 terms in the engine (main.cpp runs NON_BOND_14 in the same force
 * pass): the pairs of `nb14` (created for the same atom count) are added to
 * every step's forces and virial; their energy (LJ + Coulomb) fills slot 6
 * of the totals.  `nb14` must outlive the engine's use of it; NULL removes
 * them.  Single boxes, fixed-point accumulation. */
int snb_engine_set_nb14(snb_engine* e, snb_nb14* nb14);
/* SETTLE in the engine's MD steps (main.cpp:1705,1772 around the NVE
 * leap-frog, v_factor = x_factor = 1): the rigid triangles and pairs of
 * `settle` (created for the same atom count) are remembered before each
 * coordinate update and put back on their geometry after it; the neighbor
 * refresh check runs on the constrained positions.  A rigid pair without a
 * real update makes the MD call return SNB_ERR_BAD_INPUT.  NULL removes it.
 * Single boxes. */
int snb_engine_set_settle(snb_engine* e, snb_settle* settle);
/* Stress and pressure (MD_INFORMATION::Get_pressure, MD_core.cpp:1080-1107;
 * MD_core/sys.hpp:14-85): d_out[0..5] = (W + sum_i m_i v_i (x) v_i) / V in
 * LTMatrix3 order (kcal/mol/A^3, off-diagonal pairs summed), d_out[6] =
 * their trace / 3 in bar (CONSTANT_PRES_CONVERTION).  W = the potential
 * virial in slots 8..13 of d_totals (from snb_engine_force with
 * need_virial; NULL leaves it out) plus, with SETTLE set, the constraint
 * virial of the last MD step.  vel and mass [N] on the device. */
int snb_engine_pressure(snb_engine* e, const float* vel, const float* mass,
                        const double* d_totals, double* d_out, void* stream);
int snb_engine_md_steps(snb_engine* e, float* crd, float* vel,
                        const float* inverse_mass, float dt, int first_step,
                        int steps, void* stream);
/* Same as snb_engine_md_steps but replays a CUDA graph of one step (captured
 * on first use). */
int snb_engine_md_steps_graph(snb_engine* e, float* crd, float* vel,
                              const float* inverse_mass, float dt,
                              int first_step, int steps, void* stream);
/* snb_engine_md_steps_graph for a caller that keeps the state in host
 * memory (no counterpart in the reference, whose state stays on the
 * device): h_crd and h_vel [N*3] (pinned for full speed) are copied into the
 * device work buffers crd and vel, the steps run, and the results are
 * copied back into h_crd and h_vel; the list-overflow check and the copy
 * back share one synchronisation, after which the call returns.  The
 * coordinates are copied in first; the velocities follow on a second stream
 * while the forces are computed, and the first coordinate update waits for
 * them.  When vel follows crd directly on both sides (one [2][N*3] state
 * array each), the copy back is one copy. */
int snb_engine_md_steps_host(snb_engine* e, float* h_crd, float* h_vel, float* crd,
                             float* vel, const float* inverse_mass, float dt,
                             int first_step, int steps, void* stream);
/* Tracing (the CUDA-event counterpart of the reference's TIME_RECORDER,
 * utils/control/time_recorder.hpp:9-43): runs `steps` stream-launched steps
 * with events between phases and writes the mean milliseconds per step of
 * {neighbor update, pack, pair kernel, excluded correction, PME reciprocal,
 *  bonded, integration} to h_phase_ms[0..6].  Host sync every step. */
int snb_engine_profile_steps(snb_engine* e, float* crd, float* vel,
                             const float* inverse_mass, float dt, int first_step,
                             int steps, double* h_phase_ms, void* stream);
/* Autotuner (no counterpart in the reference).  For each candidate launch
 * shape, times `steps` replays of the captured step graph (stream-launched
 * steps for the pair search's shape, or where the stream is the legacy
 * default one), each from the given coordinates, and keeps the fastest:
 * the pair kernel's candidates per lane per scan round (2, 4, 8) and
 * persistent blocks per SM (occupancy maximum, 2, 3), its rows in flight
 * per block (4, 8, 16 warps for one box, 8 or 16 for a batch; plain LJ),
 * whether its hit list keeps each hit's displacement, charge and LJ pair
 * index in shared memory (so that the pair terms gather nothing; plain
 * single box, at most 4 candidates per lane), the pair search's
 * blocks per SM (4, 8, 16), the PME gather's threads per block (128, 256,
 * 512), the PME spread's shape (tiles of edge 8 with 1, 2, 4 warps per
 * tile, or edge 0: int64 global atomics, no tiles; single box; edge 16 with
 * 4, 8 warps is only set by snb_engine_set_launch_shapes) and the PME
 * convolution's FFT (cuFFT, or this library's own
 * mixed-radix passes with the influence function fused between the forward
 * and inverse x transforms: for one box, axes of at most 256 points; for a
 * batch, axes of 4-64 points, multiples of 4, each line transformed in
 * registers, one launch per pass over all boxes).
 * Results are bitwise
 * the same for every shape but the FFT, whose two choices differ by float
 * rounding in the reciprocal part.  crd / vel are restored; the next step rebuilds the list and
 * recaptures the step graph.  h_choice[0..8] receives {unroll, blocks per
 * SM (0 = occupancy maximum), search blocks per SM, gather threads, pair
 * warps per block, spread tile edge, spread warps per tile, hit stash (0 /
 * 1), own FFT (0 / 1)}.  Allocates scratch. */
int snb_engine_autotune(snb_engine* e, float* crd, float* vel,
                        const float* inverse_mass, float dt, int steps,
                        int* h_choice, void* stream);
/* No counterpart in the reference: sets the launch shapes directly, in the
 * h_choice order of snb_engine_autotune (for instance to reuse a tuned
 * choice); values outside the tuned sets are refused, and so is the own FFT
 * where the grid does not allow it.  Results are bitwise the same for every
 * shape but the FFT choice. */
int snb_engine_set_launch_shapes(snb_engine* e, const int* h_choice);
/* Kernel nodes of the captured one-step graph: top level (a step without a
 * neighbor rebuild), cuFFT's share of them, and the kernels inside the
 * conditional rebuild node. */
int snb_engine_graph_info(snb_engine* e, int* kernel_nodes,
                          int* library_kernel_nodes, int* rebuild_kernel_nodes,
                          void* stream);
/* Number of neighbor-list rebuilds so far and current pair count (host sync). */
int snb_engine_stats(snb_engine* e, long long* rebuilds, long long* pairs,
                     void* stream);
/* snb_pme_spread_wide_tiles of the engine's PME (host sync).  A single-box
 * engine of up to 500,000 atoms spreads by int64 global atomics unless
 * snb_engine_set_launch_shapes or snb_engine_autotune picks a tile shape;
 * with the atomics no tile is taken again and the count stays 0. */
int snb_engine_spread_wide_tiles(snb_engine* e, int* count, void* stream);
/* The engine's neighbor list holds the pair set of NEIGHBOR_LIST::Update
 * (neighbor_list.cpp:974-1025) in one of two forms.  Rows (the default):
 * one row of partners per atom, as snb_nl keeps them.  Clusters (on request,
 * for one rectangular box of at least five cells per axis, not with the
 * soft-core kernel): runs of up to four atoms of a cell, and per cluster
 * the clusters with a pair within cutoff + skin, each with its 4x4 pair
 * mask; the pair kernel loads a neighbour cluster once for four atoms.
 * Both hold the same pairs.  clusters = 0 / 1 picks the form (1 is refused
 * where the box or the soft-core kernel does not allow it); the next step
 * rebuilds the list. */
int snb_engine_set_list_form(snb_engine* e, int clusters);
/* Virtual atoms in the engine (NULL to remove): every force evaluation moves
 * the sites' forces onto their atoms before the forces are returned or the
 * coordinates updated, and every MD step places the sites after the update
 * (and before the first step).  The sites' inverse masses must be 0. */
int snb_engine_set_virtual_atoms(snb_engine* e, snb_vatom* vatom);
int snb_engine_list_form(snb_engine* e, int* clusters);
/* No counterpart in the reference.  Pruned rows for the plain LJ rows of a
 * single box: a prune pass of the pair kernel scans the full rows (the
 * entries within cutoff + skin) and keeps those within cutoff + margin; the
 * steps after it scan only the kept entries, until an atom has moved more
 * than half the margin since the pass or the list is rebuilt.  A pair
 * outside cutoff + margin at the pass stays outside the cutoff until then,
 * so every step sees the same pairs within the cutoff as without pruning
 * and the forces are the same bit for bit.  snb_engine_create (for boxes of
 * at least 20,000 atoms) and snb_batch_create set a margin of 0.8 A;
 * margin 0 turns it off.  Force
 * calls outside the MD steps always scan the full rows.  Not used with the
 * cluster form. */
int snb_engine_set_prune_margin(snb_engine* e, float margin);
/* Prune passes run so far, and (kept_entries may be null) the entries the
 * last pass kept in all rows (host sync; 0 while pruning was never on). */
int snb_engine_prune_passes(snb_engine* e, int* passes, long long* kept_entries,
                            void* stream);
/* The engine's current pair set in global ids, lo < hi, in no particular
 * order (as snb_nl_export_pairs; host sync). */
int snb_engine_export_pairs(snb_engine* e, int* d_pi, int* d_pj, long long cap,
                            long long* count, void* stream);
int snb_engine_destroy(snb_engine* e);

/* ------------------------------------------------------ bonds, angles */
/* BOND (bond/bond.h, bond/bond.cpp).  Bond t of atoms (a, b), dr = r_a - r_b
 * (minimum image): E = k (|dr| - r0)^2, f_a = -2 k (|dr| - r0) / |dr| dr,
 * f_b = -f_a; its energy and virial f_a (x) dr go to atom a.
 * Initial (bond.cpp:65-156): host arrays of bond_numbers entries. */
int snb_bond_create(int atom_numbers, int bond_numbers, const int* h_atom_a,
                    const int* h_atom_b, const float* h_k, const float* h_r0,
                    snb_bond** out);
/* Bond_Force_With_Atom_Energy_And_Virial (bond.cpp:242-258, kernel
 * bond.cpp:15-60): adds to frc[N*3], atom_energy[N] and atom_virial[N*6]
 * (LTMatrix3 order) on `stream`. */
int snb_bond_force(snb_bond* h, const float* crd, snb_boundary boundary, float* frc,
                   int need_atom_energy, float* atom_energy, int need_virial,
                   float* atom_virial, void* stream);
/* Step_Print's sum of the bond energies (bond.cpp:260-274) of the last call
 * with energies (host sync). */
int snb_bond_energy(snb_bond* h, float* h_energy, void* stream);
int snb_bond_destroy(snb_bond* h);
/* ANGLE (angle/angle.h, angle/angle.cpp).  Angle t of atoms (a, b, c), b the
 * vertex: E = k (theta - theta0)^2 with cos(theta) clamped to +-0.999999;
 * its energy and the virial f_a (x) (r_a - r_b) + f_c (x) (r_c - r_b) go to
 * atom a.  Initial (angle.cpp:83-150): host arrays of angle_numbers
 * entries, theta0 in radians. */
int snb_angle_create(int atom_numbers, int angle_numbers, const int* h_atom_a,
                     const int* h_atom_b, const int* h_atom_c, const float* h_k,
                     const float* h_theta0, snb_angle** out);
/* Angle_Force_With_Atom_Energy_And_Virial (angle.cpp:253-269, kernel
 * angle.cpp:6-80): adds to frc[N*3], atom_energy[N] and atom_virial[N*6]. */
int snb_angle_force(snb_angle* h, const float* crd, snb_boundary boundary, float* frc,
                    int need_atom_energy, float* atom_energy, int need_virial,
                    float* atom_virial, void* stream);
/* Step_Print's sum of the angle energies (angle.cpp:271-289) (host sync). */
int snb_angle_energy(snb_angle* h, float* h_energy, void* stream);
int snb_angle_destroy(snb_angle* h);

/* ------------------------------------------------------- virtual atoms */
/* VIRTUAL_INFORMATION (virtual_atoms/virtual_atoms.h, virtual_atoms.cpp) for
 * the types 0-3 of virtual_atoms.h:8-105: massless sites placed from one to
 * three atoms (0: mirror z -> 2h - z; 1: r_1 + a r_21; 2: r_1 + a r_21 +
 * b r_31; 3: r_1 + d (r_21 + k r_32) / |r_21 + k r_32|), whose forces are
 * moved onto those atoms.  A site may be built from sites; they are
 * processed in dependency levels.  Initial (virtual_atoms.cpp:338-866) from
 * record_numbers records: h_type, h_virtual_atom, h_from [3 per record,
 * unused -1] and h_parameter [2 per record: h | a | a, b | d, k].  Refused:
 * other types, a site defined twice, a site that depends on itself. */
int snb_vatom_create(int atom_numbers, int record_numbers, const int* h_type,
                     const int* h_virtual_atom, const int* h_from, const float* h_parameter,
                     snb_vatom** out);
int snb_vatom_levels(snb_vatom* v, int* levels);
/* Coordinate_Refresh (virtual_atoms.cpp:867-932): crd [N*3] updated in place. */
int snb_vatom_coordinate_refresh(snb_vatom* v, float* crd, snb_boundary boundary,
                                 void* stream);
/* Force_Redistribute (virtual_atoms.cpp:934-1001): each site's force in
 * frc [N*3] added onto its atoms, then set to zero. */
int snb_vatom_force_redistribute(snb_vatom* v, const float* crd, snb_boundary boundary,
                                 float* frc, void* stream);
/* The first record whose type-3 direction had zero length since creation,
 * or -1 (the reference stops with a runtime error there; host sync). */
int snb_vatom_status(snb_vatom* v, int* bad_record, void* stream);
int snb_vatom_destroy(snb_vatom* v);

/* ----------------------------------------------------------- 1-4 terms */
/* NON_BOND_14 (nb14/nb14.h, nb14/nb14.cpp).  Pair t of atoms (a, b) at
 * distance r (minimum image) adds E = A'/12 r^-12 - B'/6 r^-6
 * + c q_a q_b / r with A', B' the pair's scaled LJ entries (A' = 12 A,
 * B' = 6 B) and c its Coulomb scale factor; charges below 1e-10 in
 * magnitude are taken as 1e-10.  Energy and virial go to atom a.
 * Initial (nb14.cpp:102-176) / Parameter_Host_To_Device: host arrays of
 * nb14_numbers entries. */
int snb_nb14_create(int atom_numbers, int nb14_numbers, const int* h_atom_a,
                    const int* h_atom_b, const float* h_A, const float* h_B,
                    const float* h_cf_scale_factor, snb_nb14** out);
/* Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial (nb14.cpp:292-305,
 * kernel nb14.cpp:8-103): adds to frc[N*3], atom_energy[N] and
 * atom_virial[N*6] (LTMatrix3 order) on `stream`. */
int snb_nb14_force(snb_nb14* h, const float* crd, const float* charge,
                   snb_boundary boundary, float* frc, int need_atom_energy,
                   float* atom_energy, int need_virial, float* atom_virial,
                   void* stream);
/* Step_Print's sums (nb14.cpp:307-324) of the last call with energies:
 * nb14_LJ and nb14_EE (host sync). */
int snb_nb14_energy_sums(snb_nb14* h, float* h_lj, float* h_ee, void* stream);
int snb_nb14_destroy(snb_nb14* h);

/* -------------------------------------------------------------- SETTLE */
/* SETTLE (constrain/settle.h, constrain/settle.cpp).  Initial
 * (settle.cpp:483-712): the constraint pairs (atom_i, atom_j, constant_r)
 * are sorted, as the reference does, into rigid triangles (three atoms with
 * two constraints each that close a triangle; A = the lowest index), rigid
 * pairs (two atoms constrained only to each other) and the remaining pairs,
 * which SETTLE leaves to SHAKE.  h_mass [atom_numbers] sets each group's
 * masses and canonical frame. */
int snb_settle_create(int atom_numbers, int constrain_pair_numbers, const int* h_atom_i,
                      const int* h_atom_j, const float* h_constant_r, const float* h_mass,
                      snb_settle** out);
/* The grouping of snb_settle_create alone, on the host (no device memory):
 * counts[3] = {rigid triangles, rigid pairs, pairs left over} and, when
 * h_remaining_pairs is not NULL, the indices of the left-over pairs.
 * h_remaining_pairs must hold counts[2] ints; constrain_pair_numbers ints
 * always suffice, or call once with NULL to read counts[2] first. */
int snb_settle_group(int atom_numbers, int constrain_pair_numbers, const int* h_atom_i,
                     const int* h_atom_j, const float* h_constant_r, const float* h_mass,
                     int* counts, int* h_remaining_pairs);
/* triangle_numbers, pair_numbers and the constraint pairs left over (their
 * indices in the creation order into h_remaining_pairs when not NULL). */
int snb_settle_counts(snb_settle* h, int* triangle_numbers, int* pair_numbers,
                      int* remaining_pair_numbers, int* h_remaining_pairs);
/* Remember_Last_Coordinates (settle.cpp:714-730): the displacements B - A,
 * C - A and j - i at the start of the step. */
int snb_settle_remember_last_coordinates(snb_settle* h, const float* crd,
                                         snb_boundary boundary, void* stream);
/* Do_SETTLE (settle.cpp:798-882) after the coordinate update: crd and vel
 * [N*3] are corrected in place with the step dt and the integrator's
 * v_factor / x_factor (1 and 1 for leap-frog NVE); with need_pressure the
 * constraint virial / V is added to d_stress[6] (LTMatrix3 order).  A rigid
 * pair without a real update is left unchanged and recorded: read it with
 * snb_settle_status. */
int snb_settle_do(snb_settle* h, float* crd, snb_boundary boundary, float* vel, float dt,
                  float v_factor, float x_factor, int need_pressure, float* d_stress,
                  void* stream);
/* SNB_ERR_BAD_INPUT, with *invalid_pair the pair's index, when a call since
 * the last status had a rigid pair without a real update; else SNB_OK and
 * -1 (host sync; clears the record). */
int snb_settle_status(snb_settle* h, int* invalid_pair, void* stream);
int snb_settle_destroy(snb_settle* h);

/* ------------------------------------------- native inputs and outputs */
/* SPONGE's native text inputs of this path, read on the host.  Each reader
 * reads the file's counts; called with NULL arrays it returns only those,
 * so the caller can size its buffers and call again.  Conversions are the
 * reference's (fscanf "%f" / "%d"; LJ tables stored as A' = 12 A,
 * B' = 6 B).  A file that does not parse returns SNB_ERR_BAD_INPUT with
 * the reference's "the format of ... is not right" message. */
/* Xponge::Native_Load_LJ (xponge/load/native/lj.hpp:9-67): "N T", then
 * T(T+1)/2 A, T(T+1)/2 B, N types.  A and B are [T(T+1)/2], type is [N]. */
int snb_read_lj_in_file(const char* path, int* atom_numbers, int* atom_type_numbers,
                        float* h_LJ_A, float* h_LJ_B, int* h_atom_LJ_type);
/* Xponge::Native_Load_LJ_Soft_Core (xponge/load/native/lj_soft.hpp:8-89):
 * "N TA TB", the AA, AB tables of state A, the BA, BB tables of state B,
 * then N pairs "typeA typeB". */
int snb_read_lj_soft_core_in_file(const char* path, int* atom_numbers,
                                  int* atom_type_numbers_A, int* atom_type_numbers_B,
                                  float* h_LJ_AA, float* h_LJ_AB, float* h_LJ_BA,
                                  float* h_LJ_BB, int* h_LJ_type_A, int* h_LJ_type_B);
/* subsys_division_in_file (xponge/load/native/lj_soft.hpp:91-124): "N", then
 * N ints. */
int snb_read_subsys_division_in_file(const char* path, int* atom_numbers,
                                     int* h_subsys_division);
/* Xponge::Native_Load_Charge / Native_Load_Mass
 * (xponge/load/native/md_core.hpp:9-103): "N", then N floats (charges in
 * the internal unit, already scaled by 18.2223). */
int snb_read_charge_in_file(const char* path, int* atom_numbers, float* h_charge);
int snb_read_mass_in_file(const char* path, int* atom_numbers, float* h_mass);
/* Xponge::Native_Load_Exclusions (xponge/load/native/md_core.hpp:259-313):
 * "N M", then per atom its count and excluded atoms; returned as the CSR
 * that MD_INFORMATION::non_bond_information::Initial builds from it
 * (MD_core/nb.hpp:32-76): start[N], numbers[N], list[M]. */
int snb_read_exclude_in_file(const char* path, int* atom_numbers,
                             int* excluded_atom_numbers, int* h_excluded_list_start,
                             int* h_excluded_numbers, int* h_excluded_list);
/* Xponge::Native_Load_NB14 (xponge/load/native/nb14.hpp:8-101): the rows
 * of extra_path ("M", then M rows "a b A B c", A and B stored times 12 and
 * 6) first, then those of path ("K", then K rows "a b lj_scale c", A' and
 * B' = lj_scale times the pair's h_LJ_A / h_LJ_B entry for the two atoms'
 * types).  Either path may be NULL.  nb14_numbers = M + K.  An atom index
 * outside [0, atom_numbers) returns SNB_ERR_BAD_INPUT. */
/* Xponge::Native_Load_Bonds (xponge/load/native/bond.hpp:9-42): "M", then
 * M rows "a b k r0". */
int snb_read_bond_in_file(const char* path, int* bond_numbers, int* h_atom_a,
                          int* h_atom_b, float* h_k, float* h_r0);
/* Xponge::Native_Load_Angles (xponge/load/native/angle.hpp:8-44): "M", then
 * M rows "a b c k theta0". */
int snb_read_angle_in_file(const char* path, int* angle_numbers, int* h_atom_a,
                           int* h_atom_b, int* h_atom_c, float* h_k, float* h_theta0);
/* Xponge::Native_Load_Virtual_Atoms (xponge/load/native/virtual_atoms.hpp:
 * 10-120): one record per line, "type virtual_atom" then the type's fields;
 * records in file order, from [3m] (unused -1) and parameter [2m]. */
int snb_read_virtual_atom_in_file(const char* path, int* record_numbers, int* h_type,
                                  int* h_virtual_atom, int* h_from, float* h_parameter);
int snb_read_nb14_in_file(const char* path, const char* extra_path, int atom_numbers,
                          const int* h_atom_LJ_type, const float* h_LJ_A,
                          const float* h_LJ_B, int* nb14_numbers, int* h_atom_a,
                          int* h_atom_b, float* h_A, float* h_B,
                          float* h_cf_scale_factor);
/* MD_INFORMATION::trajectory_output::Append_Frc_Traj_File
 * (MD_core/output.hpp:1691-1700): appends one frame, the N float3 forces of
 * device array d_frc, to the binary file at path (host sync). */
int snb_append_frc_traj(const char* path, const float* d_frc, int atom_numbers,
                        void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPONGE_NB_H */
