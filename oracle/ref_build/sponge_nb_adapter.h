/* The reference-side adapter: SPONGE's NEIGHBOR_LIST, LENNARD_JONES_INFORMATION,
 * LJ_SOFT_CORE and Particle_Mesh as structs whose hot-path members keep the
 * reference's signatures (neighbor_list.h:17-24, Lennard_Jones_force.h:118-172,
 * LJ_soft_core.h:238-274, PM_force.h:153-190) and forward to the C ABI of
 * include/sponge_nb.h.  A SPONGE build that links libsponge_nb.so includes
 * this header where main.cpp includes those four and brings the names into
 * the global namespace (using snb_adapter::NEIGHBOR_LIST; ...).
 * adapter_signatures.cpp compiles it beside the reference's own headers and
 * holds every member's type equal to the reference member it replaces.
 *
 * It is written against the reference's common.h and control.h and uses
 * their helpers (Device_Malloc_Safely, deviceMemset, deviceMemcpy,
 * Launch_Device_Kernel, CONTROLLER::Step_Print), so it compiles with the
 * reference's CPU and CUDA backends alike.
 *
 * Conventions: device pointers as in the reference; a non-zero status from
 * the library goes to CONTROLLER::Throw_SPONGE_Error with the library's
 * message.  The modules receive the neighbor list as the reference's
 * ATOM_GROUP* d_nl; the adapter finds the library handle of a list by that
 * pointer.  d_nl is filled in the reference's layout (each row's partners in
 * a slab of max_neighbor_numbers ints) only when the input key
 * neighbor_list_export_atom_groups is true, for readers of d_nl other than
 * these modules; otherwise its rows read as empty.
 *
 * Not covered: the members of the reference's domain decomposition
 * (Particle_Mesh::Domain_Decomposition, Get_Atoms, Send_Recv_*, g_crd/g_frc)
 * and the full neighbor list of the many-body potentials; one domain holds
 * every atom, as the library's calls require (ghost_numbers = 0). */
#pragma once
#include "common.h"
#include "control.h"
#include "sponge_nb.h"

namespace snb_adapter
{

snb_boundary to_snb(const Boundary& b);
// CONTROLLER::Throw_SPONGE_Error with the library's message unless rc is 0
void check(CONTROLLER* controller, int rc, const char* where);
// snb_options from the defaults, the cutoff and every key of the library's
// option set that the controller's command map holds
void options_from(CONTROLLER* controller, snb_options* opt, float cutoff);

struct NEIGHBOR_LIST
{
    enum NEIGHBOR_LIST_UPDATE_PARAMETER
    {
        CONDITIONAL_UPDATE = 0,
        FORCED_UPDATE = 1
    };
    bool is_initialized = 0;
    float cutoff = 10.0f;
    float skin = 2.0f;
    int atom_numbers = 0;
    int ghost_numbers = 0;
    int max_neighbor_numbers = 1200;
    int check_overflow_interval = 100;
    ATOM_GROUP* d_nl = NULL;
    int* d_slab = NULL;  // the rows of d_nl when they are exported
    bool export_atom_groups = false;
    bool force_next_update = false;  // the last build overflowed and regrew
    snb_nl* handle = NULL;
    CONTROLLER* controller = NULL;

    void Initial(CONTROLLER* controller, int atom_numbers, float cutoff,
                 float skin, const Boundary boundary);
    void Update(int* atom_local, int local_atom_numbers, int ghost_numbers,
                VECTOR* crd, const Boundary boundary, int step, int update,
                int* excluded_list_start = NULL, int* excluded_list = NULL,
                int* excluded_numbers = NULL);
    void Check_Overflow(CONTROLLER* controller, int steps,
                        const Boundary boundary, LTMatrix3* cell0);
    void Clear();
    // the library handle of the list whose d_nl this is, or NULL
    static snb_nl* Handle_Of(const ATOM_GROUP* nl);
};

struct LENNARD_JONES_INFORMATION
{
    char module_name[CHAR_LENGTH_MAX];
    int is_initialized = 0;
    int atom_numbers = 0;
    int atom_type_numbers = 0;
    int pair_type_numbers = 0;
    int* h_atom_LJ_type = NULL;
    float* h_LJ_A = NULL;
    float* h_LJ_B = NULL;
    float h_LJ_energy_sum = 0;
    float h_LJ_long_energy = 0;
    float cutoff = 10.0f;
    float long_range_factor = 0;
    int local_atom_numbers = 0;
    int ghost_numbers = 0;
    snb_lj* handle = NULL;
    CONTROLLER* controller = NULL;

    // tables from Xponge::system.classical_force_field.lj, or from the file
    // of the key <module_name>_in_file when a module name is given
    void Initial(CONTROLLER* controller, float cutoff,
                 const char* module_name = NULL);
    void LJ_Malloc();
    void Parameter_Host_To_Device();
    void Get_Local(int* atom_local, int local_atom_numbers, int ghost_numbers);
    void LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
        const int atom_numbers, const int local_atom_numbers,
        const int solvent_numbers, const int ghost_numbers, const VECTOR* crd,
        const float* charge, VECTOR* frc, const Boundary boundary,
        const ATOM_GROUP* nl, const float pme_beta, const int need_atom_energy,
        float* atom_energy, const int need_virial, LTMatrix3* atom_virial,
        float* atom_direct_pme_energy);
    void Long_Range_Correction(int need_pressure, LTMatrix3* d_virial,
                               int need_potential, float* d_potential,
                               const float volume);
    void Step_Print(CONTROLLER* controller);
    void Clear();
};

struct LJ_SOFT_CORE
{
    char module_name[CHAR_LENGTH_MAX];
    int is_initialized = 0;
    int atom_numbers = 0;
    int atom_type_numbers_A = 0;
    int atom_type_numbers_B = 0;
    int* h_LJ_type_A = NULL;
    int* h_LJ_type_B = NULL;
    int* h_subsys_division = NULL;
    float* h_LJ_AA = NULL;
    float* h_LJ_AB = NULL;
    float* h_LJ_BA = NULL;
    float* h_LJ_BB = NULL;
    float cutoff = 10.0f;
    float lambda = 0.0f;
    float h_LJ_energy_sum = 0;
    float h_LJ_energy_sum_intersys = 0;
    float h_LJ_energy_sum_intrasys = 0;
    float h_LJ_long_energy = 0;
    int local_atom_numbers = 0;
    int ghost_numbers = 0;
    snb_options options;
    snb_lj_soft* handle = NULL;
    CONTROLLER* controller = NULL;

    // tables from Xponge::system.classical_force_field.lj_soft_core, or from
    // the files of <module_name>_in_file and subsys_division_in_file
    void Initial(CONTROLLER* controller, float cutoff, char* module_name = NULL);
    void LJ_Soft_Core_Malloc();
    void Clear();
    void Parameter_Host_To_Device();
    void LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
        const int atom_numbers, const int local_atom_numbers,
        const int solvent_numbers, const int ghost_numbers, const VECTOR* crd,
        const float* charge, VECTOR* frc, const Boundary boundary,
        const ATOM_GROUP* nl, const float pme_beta, const int need_atom_energy,
        float* atom_energy, const int need_virial, LTMatrix3* atom_lj_virial,
        float* atom_direct_pme_energy);
    void Step_Print(CONTROLLER* controller);
    void Long_Range_Correction(int need_pressure, LTMatrix3* d_virial,
                               int need_potential, float* d_potential,
                               const float volume);
    float Get_Partial_H_Partial_Lambda_With_Columb_Direct(
        const int solvent_numbers, const VECTOR* crd, const Boundary boundary,
        const float* charge, const ATOM_GROUP* nl, const float* charge_B_A,
        const float pme_beta, const int charge_perturbated);
    void Get_Local(int* atom_local, int local_atom_numbers, int ghost_numbers);
};

struct Particle_Mesh
{
    char module_name[CHAR_LENGTH_MAX];
    int is_initialized = 0;
    int atom_numbers = 0;
    int fftx = 0, ffty = 0, fftz = 0;
    float beta = 0.0f;
    float cutoff = 10.0f;
    float exclude_factor = 1.0f;
    bool print_detail = false;
    // per-atom direct-space Coulomb energy (filled by the LJ modules through
    // their atom_direct_pme_energy argument) and excluded-pair correction
    float* d_direct_atom_energy = NULL;
    float* d_correction_atom_energy = NULL;
    float direct_ene = 0, correction_ene = 0, self_ene = 0, reciprocal_ene = 0;
    float ee_ene = 0;
    snb_pme* handle = NULL;
    CONTROLLER* controller = NULL;

    void Initial(CONTROLLER* controller, int atom_numbers,
                 const Boundary boundary, VECTOR box_length, float cutoff,
                 int no_direct_interaction_virtual_atom_numbers,
                 const char* module_name = NULL);
    void Clear();
    void PME_Excluded_Force_With_Atom_Energy(
        const VECTOR* crd, const Boundary boundary, const float* charge,
        const int* excluded_list_start, const int* excluded_list,
        const int* excluded_atom_numbers, VECTOR* frc, int need_energy,
        float* atom_ene, LTMatrix3* atom_virial);
    void PME_Reciprocal_Force_With_Energy_And_Virial(
        const VECTOR* crd, const Boundary boundary, const float* charge,
        VECTOR* force, int need_virial, int need_energy, LTMatrix3* d_virial,
        float* d_potential, int step);
    void Update_Box(const Boundary boundary, LTMatrix3 g, float dt);
    void Step_Print(CONTROLLER* controller);
    void MPI_PME_Excluded_Force_With_Atom_Energy(
        const int N, const int* id1, const int* id2, const VECTOR* crd,
        const Boundary boundary, const float* charge,
        const int* excluded_list_start, const int* excluded_list,
        const int* excluded_atom_numbers, VECTOR* frc, int need_energy,
        float* atom_ene, int need_virial, LTMatrix3* atom_virial);
};

}  // namespace snb_adapter
