/* The adapter's members: each forwards to the C ABI of include/sponge_nb.h in
 * the place of the reference member named beside it.  Device memory and
 * kernels of the adapter's own (two per-atom energy buffers of
 * Particle_Mesh, one list add) go through the reference's backend helpers,
 * so the file builds with its CPU or CUDA definitions. */
#include "sponge_nb_adapter.h"

#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "xponge/xponge.h"

namespace snb_adapter
{

namespace
{
std::mutex g_lists_mutex;
std::map<const ATOM_GROUP*, snb_nl*>& lists()
{
    static std::map<const ATOM_GROUP*, snb_nl*> m;
    return m;
}

bool truthy(const char* v)
{
    std::string s(v ? v : "");
    for (char& c : s) c = (char)tolower((unsigned char)c);
    return s == "1" || s == "true" || s == "yes" || s == "on";
}

// every key snb_options_set knows; the reference reads each of these from
// its command map under the same name
const char* const kOptionKeys[] = {
    "skin",
    "neighbor_list_refresh_interval",
    "neighbor_list_skin_permit",
    "neighbor_list_max_neighbor_numbers",
    "neighbor_list_max_atom_in_grid_numbers",
    "neighbor_list_max_ghost_in_grid_numbers",
    "neighbor_list_check_overflow_interval",
    "neighbor_list_throw_error_when_overflow",
    "PM_fftx",
    "PM_ffty",
    "PM_fftz",
    "PM_grid_spacing",
    "PM_Direct_Tolerance",
    "PME_update_interval",
    "PME_calculate_reciprocal_part",
    "PME_calculate_excluded_part",
    "lambda_lj",
    "soft_core_alpha",
    "soft_core_powfer",
    "soft_core_sigma",
    "soft_core_sigma_min",
    "DOM_DEC_update_interval",
    "accumulation",
};

snb_nl* list_of(CONTROLLER* controller, const ATOM_GROUP* nl, const char* where)
{
    snb_nl* h = NEIGHBOR_LIST::Handle_Of(nl);
    if (h == NULL)
        controller->Throw_SPONGE_Error(
            spongeErrorValueErrorCommand, where,
            "Reason:\n\tthe neighbor list was not made by this library's "
            "NEIGHBOR_LIST\n");
    return h;
}

template <typename T>
void host_array(T** p, size_t n)
{
    free(*p);
    *p = NULL;
    Malloc_Safely((void**)p, sizeof(T) * (n > 0 ? n : 1));
}

float device_sum(const float* d, int n)
{
    if (d == NULL || n <= 0) return 0.0f;
    std::vector<float> h(n);
    deviceMemcpy(h.data(), d, sizeof(float) * n, deviceMemcpyDeviceToHost);
    double s = 0.0;
    for (float v : h) s += v;
    return (float)s;
}
}  // namespace

static __global__ void Add_Atom_List(const int n, float* to, const float* from)
{
    SIMPLE_DEVICE_FOR(i, n) { to[i] += from[i]; }
}

snb_boundary to_snb(const Boundary& b)
{
    snb_boundary s;
    s.policy = b.policy == BoundaryPolicy::Periodic ? 1 : 0;
    const LTMatrix3* m[2] = {&b.cell, &b.rcell};
    float* o[2] = {s.cell, s.rcell};
    for (int k = 0; k < 2; ++k)
    {
        o[k][0] = m[k]->a11;
        o[k][1] = m[k]->a21;
        o[k][2] = m[k]->a22;
        o[k][3] = m[k]->a31;
        o[k][4] = m[k]->a32;
        o[k][5] = m[k]->a33;
    }
    return s;
}

void check(CONTROLLER* controller, int rc, const char* where)
{
    if (rc == SNB_OK) return;
    int code = rc == SNB_ERR_BAD_INPUT       ? spongeErrorValueErrorCommand
               : rc == SNB_ERR_OVERFLOW      ? spongeErrorOverflow
               : rc == SNB_ERR_NOT_SUPPORTED ? spongeErrorNotImplemented
                                             : spongeErrorMallocFailed;
    std::string why = std::string("Reason:\n\t") + snb_last_error() + "\n";
    controller->Throw_SPONGE_Error(code, where, why.c_str());
}

void options_from(CONTROLLER* controller, snb_options* opt, float cutoff)
{
    snb_options_default(opt);
    opt->cutoff = cutoff;
    for (const char* key : kOptionKeys)
        if (controller->Command_Exist(key))
            check(controller,
                  snb_options_set(opt, key, controller->Command(key)), key);
}

/* ------------------------------------------------------ NEIGHBOR_LIST */

// neighbor_list.cpp:871-972
void NEIGHBOR_LIST::Initial(CONTROLLER* controller, int atom_numbers,
                            float cutoff, float skin, const Boundary boundary)
{
    this->controller = controller;
    this->atom_numbers = atom_numbers;
    this->cutoff = cutoff;
    this->skin = skin;
    snb_options o;
    options_from(controller, &o, cutoff);
    o.skin = skin;
    max_neighbor_numbers = o.nl_max_neighbor_numbers;
    check_overflow_interval = o.nl_check_overflow_interval;
    check(controller,
          snb_nl_create(&o, atom_numbers, cutoff, skin, to_snb(boundary), &handle),
          "NEIGHBOR_LIST::Initial");
    export_atom_groups =
        controller->Command_Exist("neighbor_list_export_atom_groups") &&
        truthy(controller->Command("neighbor_list_export_atom_groups"));
    Device_Malloc_Safely((void**)&d_nl, sizeof(ATOM_GROUP) * atom_numbers);
    deviceMemset(d_nl, 0, sizeof(ATOM_GROUP) * atom_numbers);
    if (export_atom_groups)
        Device_Malloc_Safely((void**)&d_slab, sizeof(int) * (size_t)atom_numbers *
                                                  max_neighbor_numbers);
    {
        std::lock_guard<std::mutex> lock(g_lists_mutex);
        lists()[d_nl] = handle;
    }
    is_initialized = 1;
}

// neighbor_list.cpp:974-1025
void NEIGHBOR_LIST::Update(int* atom_local, int local_atom_numbers,
                           int ghost_numbers, VECTOR* crd,
                           const Boundary boundary, int step, int update,
                           int* excluded_list_start, int* excluded_list,
                           int* excluded_numbers)
{
    if (!is_initialized) return;
    if (local_atom_numbers <= 0 && ghost_numbers <= 0) return;
    this->ghost_numbers = ghost_numbers;
    int forced = update == FORCED_UPDATE || force_next_update;
    force_next_update = false;
    check(controller,
          snb_nl_update(handle, atom_local, local_atom_numbers, ghost_numbers,
                        (const float*)crd, to_snb(boundary), step, forced,
                        excluded_list_start, excluded_list, excluded_numbers,
                        NULL),
          "NEIGHBOR_LIST::Update");
    if (export_atom_groups)
        check(controller,
              snb_nl_export_atom_groups(handle, d_nl, d_slab,
                                        max_neighbor_numbers, NULL),
              "NEIGHBOR_LIST::Update");
}

// neighbor_list.cpp:1027-1103: the library regrows its storage itself; the
// list built with too little room is rebuilt at the next update
void NEIGHBOR_LIST::Check_Overflow(CONTROLLER* controller, int steps,
                                   const Boundary boundary, LTMatrix3* cell0)
{
    if (!is_initialized || (steps + 1) % check_overflow_interval != 0) return;
    int regrown = 0;
    check(controller, snb_nl_check_overflow(handle, &regrown, NULL),
          "NEIGHBOR_LIST::Check_Overflow");
    if (regrown) force_next_update = true;
}

// neighbor_list.cpp:1105-1119
void NEIGHBOR_LIST::Clear()
{
    if (!is_initialized) return;
    {
        std::lock_guard<std::mutex> lock(g_lists_mutex);
        lists().erase(d_nl);
    }
    snb_nl_destroy(handle);
    handle = NULL;
    deviceFree(d_nl);
    d_nl = NULL;
    if (d_slab) deviceFree(d_slab);
    d_slab = NULL;
    is_initialized = 0;
}

snb_nl* NEIGHBOR_LIST::Handle_Of(const ATOM_GROUP* nl)
{
    std::lock_guard<std::mutex> lock(g_lists_mutex);
    auto it = lists().find(nl);
    return it == lists().end() ? NULL : it->second;
}

/* ------------------------------------------ LENNARD_JONES_INFORMATION */

// Lennard_Jones_force.cpp:147-250
void LENNARD_JONES_INFORMATION::Initial(CONTROLLER* controller, float cutoff,
                                        const char* module_name)
{
    this->controller = controller;
    strcpy(this->module_name, module_name == NULL ? "LJ" : module_name);
    const Xponge::LennardJones* lj = NULL;
    Xponge::LennardJones local;
    if (module_name == NULL)
    {
        lj = &Xponge::system.classical_force_field.lj;
    }
    else if (controller->Command_Exist(this->module_name, "in_file"))
    {
        const char* path = controller->Command(this->module_name, "in_file");
        int n = 0, t = 0;
        check(controller,
              snb_read_lj_in_file(path, &n, &t, NULL, NULL, NULL),
              "LENNARD_JONES_INFORMATION::Initial");
        local.atom_type.resize(n);
        local.pair_A.resize(t * (t + 1) / 2);
        local.pair_B.resize(t * (t + 1) / 2);
        local.atom_type_numbers = t;
        check(controller,
              snb_read_lj_in_file(path, &n, &t, local.pair_A.data(),
                                  local.pair_B.data(), local.atom_type.data()),
              "LENNARD_JONES_INFORMATION::Initial");
        lj = &local;
    }
    if (lj == NULL || lj->atom_type.empty()) return;
    atom_numbers = (int)lj->atom_type.size();
    atom_type_numbers = lj->atom_type_numbers;
    pair_type_numbers = atom_type_numbers * (atom_type_numbers + 1) / 2;
    LJ_Malloc();
    for (int i = 0; i < pair_type_numbers; i++)
    {
        h_LJ_A[i] = lj->pair_A[i];
        h_LJ_B[i] = lj->pair_B[i];
    }
    for (int i = 0; i < atom_numbers; i++) h_atom_LJ_type[i] = lj->atom_type[i];
    this->cutoff = cutoff;
    Parameter_Host_To_Device();
    is_initialized = 1;
    controller->Step_Print_Initial("LJ_short", "%.2f");
    controller->Step_Print_Initial("LJ_long", "%.2f");
    controller->Step_Print_Initial("LJ", "%.2f");
}

void LENNARD_JONES_INFORMATION::LJ_Malloc()
{
    host_array(&h_atom_LJ_type, atom_numbers);
    host_array(&h_LJ_A, pair_type_numbers);
    host_array(&h_LJ_B, pair_type_numbers);
}

// the library's tables on the device, and the long-range factor it forms
// from them as Lennard_Jones_force.cpp:205-236 does
void LENNARD_JONES_INFORMATION::Parameter_Host_To_Device()
{
    snb_options o;
    options_from(controller, &o, cutoff);
    if (handle) snb_lj_destroy(handle);
    handle = NULL;
    check(controller,
          snb_lj_create(&o, atom_numbers, atom_type_numbers, h_atom_LJ_type,
                        h_LJ_A, h_LJ_B, cutoff, &handle),
          "LENNARD_JONES_INFORMATION::Parameter_Host_To_Device");
    long_range_factor = snb_lj_long_range_factor(handle);
}

// Lennard_Jones_force.cpp:263-285
void LENNARD_JONES_INFORMATION::Get_Local(int* atom_local,
                                          int local_atom_numbers,
                                          int ghost_numbers)
{
    if (!is_initialized) return;
    this->local_atom_numbers = local_atom_numbers;
    this->ghost_numbers = ghost_numbers;
    check(controller,
          snb_lj_get_local(handle, atom_local, local_atom_numbers, ghost_numbers,
                           NULL),
          "LENNARD_JONES_INFORMATION::Get_Local");
}

// Lennard_Jones_force.cpp:326-384
void LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
    const int atom_numbers, const int local_atom_numbers,
    const int solvent_numbers, const int ghost_numbers, const VECTOR* crd,
    const float* charge, VECTOR* frc, const Boundary boundary,
    const ATOM_GROUP* nl, const float pme_beta, const int need_atom_energy,
    float* atom_energy, const int need_virial, LTMatrix3* atom_virial,
    float* atom_direct_pme_energy)
{
    if (!is_initialized) return;
    const char* where =
        "LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_"
        "Virial";
    check(controller,
          snb_lj_pme_direct_force(
              handle, atom_numbers, local_atom_numbers, solvent_numbers,
              ghost_numbers, (const float*)crd, charge, (float*)frc,
              to_snb(boundary), list_of(controller, nl, where), pme_beta,
              need_atom_energy, atom_energy, need_virial, (float*)atom_virial,
              atom_direct_pme_energy, NULL),
          where);
}

// Lennard_Jones_force.cpp:287-308
void LENNARD_JONES_INFORMATION::Long_Range_Correction(int need_pressure,
                                                      LTMatrix3* d_virial,
                                                      int need_potential,
                                                      float* d_potential,
                                                      const float volume)
{
    if (!is_initialized) return;
    check(controller,
          snb_lj_long_range_correction(handle, need_pressure, (float*)d_virial,
                                       need_potential, d_potential, volume,
                                       NULL),
          "LENNARD_JONES_INFORMATION::Long_Range_Correction");
    if (need_potential) h_LJ_long_energy = long_range_factor / volume;
}

// Lennard_Jones_force.cpp:386-400
void LENNARD_JONES_INFORMATION::Step_Print(CONTROLLER* controller)
{
    if (!is_initialized) return;
    check(controller, snb_lj_energy_sum(handle, &h_LJ_energy_sum, NULL),
          "LENNARD_JONES_INFORMATION::Step_Print");
    controller->Step_Print("LJ_short", h_LJ_energy_sum);
    controller->Step_Print("LJ_long", h_LJ_long_energy);
    controller->Step_Print("LJ", h_LJ_energy_sum + h_LJ_long_energy, true);
}

void LENNARD_JONES_INFORMATION::Clear()
{
    if (handle) snb_lj_destroy(handle);
    handle = NULL;
    free(h_atom_LJ_type);
    free(h_LJ_A);
    free(h_LJ_B);
    h_atom_LJ_type = NULL;
    h_LJ_A = h_LJ_B = NULL;
    is_initialized = 0;
}

/* ------------------------------------------------------- LJ_SOFT_CORE */

// LJ_soft_core.cpp:463-688
void LJ_SOFT_CORE::Initial(CONTROLLER* controller, float cutoff,
                           char* module_name)
{
    this->controller = controller;
    strcpy(this->module_name, module_name == NULL ? "LJ_soft_core" : module_name);
    const Xponge::LJSoftCore* sc = NULL;
    Xponge::LJSoftCore local;
    if (module_name == NULL)
    {
        sc = &Xponge::system.classical_force_field.lj_soft_core;
    }
    else if (controller->Command_Exist(this->module_name, "in_file"))
    {
        const char* path = controller->Command(this->module_name, "in_file");
        const char* where = "LJ_SOFT_CORE::Initial";
        int n = 0, ta = 0, tb = 0;
        check(controller,
              snb_read_lj_soft_core_in_file(path, &n, &ta, &tb, NULL, NULL, NULL,
                                            NULL, NULL, NULL),
              where);
        local.atom_numbers = n;
        local.atom_type_numbers_A = ta;
        local.atom_type_numbers_B = tb;
        local.LJ_AA.resize(ta * (ta + 1) / 2);
        local.LJ_AB.resize(ta * (ta + 1) / 2);
        local.LJ_BA.resize(tb * (tb + 1) / 2);
        local.LJ_BB.resize(tb * (tb + 1) / 2);
        local.atom_LJ_type_A.resize(n);
        local.atom_LJ_type_B.resize(n);
        check(controller,
              snb_read_lj_soft_core_in_file(
                  path, &n, &ta, &tb, local.LJ_AA.data(), local.LJ_AB.data(),
                  local.LJ_BA.data(), local.LJ_BB.data(),
                  local.atom_LJ_type_A.data(), local.atom_LJ_type_B.data()),
              where);
        if (controller->Command_Exist("subsys_division_in_file"))
        {
            const char* sub = controller->Command("subsys_division_in_file");
            int m = 0;
            check(controller, snb_read_subsys_division_in_file(sub, &m, NULL), where);
            if (m != n)
                controller->Throw_SPONGE_Error(
                    spongeErrorConflictingCommand, where,
                    "Reason:\n\tthe atom numbers of subsys_division_in_file "
                    "and LJ_soft_core_in_file differ\n");
            local.subsystem_division.resize(n);
            check(controller,
                  snb_read_subsys_division_in_file(sub, &m,
                                                   local.subsystem_division.data()),
                  where);
        }
        sc = &local;
    }
    if (sc == NULL || sc->atom_numbers <= 0) return;
    if (!controller->Command_Exist("lambda_lj"))
        controller->Throw_SPONGE_Error(
            spongeErrorMissingCommand, "LJ_SOFT_CORE::Initial",
            "Reason:\n\t'lambda_lj' is required for the calculation of "
            "LJ_soft_core\n");
    this->cutoff = cutoff;
    options_from(controller, &options, cutoff);
    lambda = options.lambda_lj;
    atom_numbers = sc->atom_numbers;
    atom_type_numbers_A = sc->atom_type_numbers_A;
    atom_type_numbers_B = sc->atom_type_numbers_B;
    LJ_Soft_Core_Malloc();
    memcpy(h_LJ_AA, sc->LJ_AA.data(), sizeof(float) * sc->LJ_AA.size());
    memcpy(h_LJ_AB, sc->LJ_AB.data(), sizeof(float) * sc->LJ_AB.size());
    memcpy(h_LJ_BA, sc->LJ_BA.data(), sizeof(float) * sc->LJ_BA.size());
    memcpy(h_LJ_BB, sc->LJ_BB.data(), sizeof(float) * sc->LJ_BB.size());
    memcpy(h_LJ_type_A, sc->atom_LJ_type_A.data(), sizeof(int) * atom_numbers);
    memcpy(h_LJ_type_B, sc->atom_LJ_type_B.data(), sizeof(int) * atom_numbers);
    for (int i = 0; i < atom_numbers; i++)
        h_subsys_division[i] = sc->subsystem_division.empty()
                                   ? 0
                                   : sc->subsystem_division[i];
    Parameter_Host_To_Device();
    is_initialized = 1;
    controller->Step_Print_Initial("LJ_soft", "%.2f");
    controller->Step_Print_Initial("LJ_soft_inter", "%.2f");
    controller->Step_Print_Initial("LJ_soft_intra", "%.2f");
    controller->Step_Print_Initial("LJ_soft_short", "%.2f");
    controller->Step_Print_Initial("LJ_soft_long", "%.2f");
}

void LJ_SOFT_CORE::LJ_Soft_Core_Malloc()
{
    int pa = atom_type_numbers_A * (atom_type_numbers_A + 1) / 2;
    int pb = atom_type_numbers_B * (atom_type_numbers_B + 1) / 2;
    host_array(&h_LJ_type_A, atom_numbers);
    host_array(&h_LJ_type_B, atom_numbers);
    host_array(&h_subsys_division, atom_numbers);
    host_array(&h_LJ_AA, pa);
    host_array(&h_LJ_AB, pa);
    host_array(&h_LJ_BA, pb);
    host_array(&h_LJ_BB, pb);
}

void LJ_SOFT_CORE::Clear()
{
    if (handle) snb_lj_soft_destroy(handle);
    handle = NULL;
    int** ints[3] = {&h_LJ_type_A, &h_LJ_type_B, &h_subsys_division};
    float** floats[4] = {&h_LJ_AA, &h_LJ_AB, &h_LJ_BA, &h_LJ_BB};
    for (int** p : ints)
    {
        free(*p);
        *p = NULL;
    }
    for (float** p : floats)
    {
        free(*p);
        *p = NULL;
    }
    is_initialized = 0;
}

void LJ_SOFT_CORE::Parameter_Host_To_Device()
{
    if (handle) snb_lj_soft_destroy(handle);
    handle = NULL;
    check(controller,
          snb_lj_soft_create(&options, atom_numbers, atom_type_numbers_A,
                             atom_type_numbers_B, h_LJ_type_A, h_LJ_type_B,
                             h_LJ_AA, h_LJ_AB, h_LJ_BA, h_LJ_BB,
                             h_subsys_division, cutoff, &handle),
          "LJ_SOFT_CORE::Parameter_Host_To_Device");
}

// LJ_soft_core.cpp:757-825.  The reference leaves the pairs of the trailing
// water block to SOLVENT_LENNARD_JONES when solvent_numbers > 0; the
// library's soft-core call takes every pair, so that split is refused.
void LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
    const int atom_numbers, const int local_atom_numbers,
    const int solvent_numbers, const int ghost_numbers, const VECTOR* crd,
    const float* charge, VECTOR* frc, const Boundary boundary,
    const ATOM_GROUP* nl, const float pme_beta, const int need_atom_energy,
    float* atom_energy, const int need_virial, LTMatrix3* atom_lj_virial,
    float* atom_direct_pme_energy)
{
    if (!is_initialized) return;
    const char* where =
        "LJ_SOFT_CORE::LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_"
        "Virial";
    if (solvent_numbers > 0)
        controller->Throw_SPONGE_Error(
            spongeErrorNotImplemented, where,
            "Reason:\n\tthe soft-core pair terms of this library take the "
            "solvent pairs too; run without SOLVENT_LENNARD_JONES\n");
    check(controller,
          snb_lj_soft_pme_direct_force(
              handle, atom_numbers, local_atom_numbers, ghost_numbers,
              (const float*)crd, charge, NULL, (float*)frc, to_snb(boundary),
              list_of(controller, nl, where), pme_beta, need_atom_energy,
              atom_energy, need_virial, (float*)atom_lj_virial,
              atom_direct_pme_energy, NULL),
          where);
}

// LJ_soft_core.cpp:890-921
void LJ_SOFT_CORE::Step_Print(CONTROLLER* controller)
{
    if (!is_initialized) return;
    float sums[4];
    check(controller, snb_lj_soft_energy_sums(handle, sums, NULL),
          "LJ_SOFT_CORE::Step_Print");
    h_LJ_energy_sum = sums[0];
    h_LJ_energy_sum_intersys = sums[1];
    h_LJ_energy_sum_intrasys = sums[2];
    h_LJ_long_energy = sums[3];
    controller->Step_Print("LJ_soft_inter", h_LJ_energy_sum_intersys);
    controller->Step_Print("LJ_soft_intra", h_LJ_energy_sum_intrasys);
    controller->Step_Print("LJ_soft_short", h_LJ_energy_sum);
    controller->Step_Print("LJ_soft_long", h_LJ_long_energy);
    controller->Step_Print("LJ_soft", h_LJ_energy_sum + h_LJ_long_energy, true);
}

void LJ_SOFT_CORE::Long_Range_Correction(int need_pressure, LTMatrix3* d_virial,
                                         int need_potential, float* d_potential,
                                         const float volume)
{
    if (!is_initialized) return;
    check(controller,
          snb_lj_soft_long_range_correction(handle, need_pressure,
                                            (float*)d_virial, need_potential,
                                            d_potential, volume, NULL),
          "LJ_SOFT_CORE::Long_Range_Correction");
}

// LJ_soft_core.cpp:827-888 (solvent_numbers: see the force call above)
float LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct(
    const int solvent_numbers, const VECTOR* crd, const Boundary boundary,
    const float* charge, const ATOM_GROUP* nl, const float* charge_B_A,
    const float pme_beta, const int charge_perturbated)
{
    if (!is_initialized) return 0.0f;
    const char* where =
        "LJ_SOFT_CORE::Get_Partial_H_Partial_Lambda_With_Columb_Direct";
    double dh = 0.0;
    check(controller,
          snb_lj_soft_dh_dlambda(handle, (const float*)crd, charge, charge_B_A,
                                 to_snb(boundary), list_of(controller, nl, where),
                                 pme_beta, charge_perturbated, &dh, NULL),
          where);
    return (float)dh;
}

// LJ_soft_core.cpp:962-980: one domain, so only the counts are kept
void LJ_SOFT_CORE::Get_Local(int* atom_local, int local_atom_numbers,
                             int ghost_numbers)
{
    this->local_atom_numbers = local_atom_numbers;
    this->ghost_numbers = ghost_numbers;
}

/* ------------------------------------------------------ Particle_Mesh */

// PM_force.cpp:295-654.  no_direct_interaction_virtual_atom_numbers sizes
// the reference's domain-decomposition buffers only.
void Particle_Mesh::Initial(CONTROLLER* controller, int atom_numbers,
                            const Boundary boundary, VECTOR box_length,
                            float cutoff,
                            int no_direct_interaction_virtual_atom_numbers,
                            const char* module_name)
{
    this->controller = controller;
    strcpy(this->module_name, module_name == NULL ? "PM" : module_name);
    this->atom_numbers = atom_numbers;
    this->cutoff = cutoff;
    snb_options o;
    options_from(controller, &o, cutoff);
    float lengths[3] = {box_length.x, box_length.y, box_length.z};
    check(controller,
          snb_pme_create(&o, atom_numbers, to_snb(boundary), lengths, cutoff,
                         &handle),
          "Particle_Mesh::Initial");
    beta = snb_pme_beta(handle);
    int fft3[3];
    check(controller, snb_pme_grid(handle, fft3), "Particle_Mesh::Initial");
    fftx = fft3[0];
    ffty = fft3[1];
    fftz = fft3[2];
    Device_Malloc_Safely((void**)&d_direct_atom_energy, sizeof(float) * atom_numbers);
    Device_Malloc_Safely((void**)&d_correction_atom_energy,
                         sizeof(float) * atom_numbers);
    deviceMemset(d_direct_atom_energy, 0, sizeof(float) * atom_numbers);
    deviceMemset(d_correction_atom_energy, 0, sizeof(float) * atom_numbers);
    is_initialized = 1;
    controller->Step_Print_Initial(this->module_name, "%.2f");
    if (controller->Command_Exist(this->module_name, "print_detail"))
        print_detail = truthy(controller->Command(this->module_name, "print_detail"));
    if (print_detail)
    {
        controller->Step_Print_Initial("PM_direct", "%.2f");
        controller->Step_Print_Initial("PM_reciprocal", "%.2f");
        controller->Step_Print_Initial("PM_self", "%.2f");
        controller->Step_Print_Initial("PM_correction", "%.2f");
    }
}

void Particle_Mesh::Clear()
{
    if (!is_initialized) return;
    snb_pme_destroy(handle);
    handle = NULL;
    deviceFree(d_direct_atom_energy);
    deviceFree(d_correction_atom_energy);
    d_direct_atom_energy = d_correction_atom_energy = NULL;
    is_initialized = 0;
}

// PM_force.cpp:984-1005: the correction's per-atom energy goes to atom_ene
// and to this module's own buffer, which Step_Print sums
void Particle_Mesh::PME_Excluded_Force_With_Atom_Energy(
    const VECTOR* crd, const Boundary boundary, const float* charge,
    const int* excluded_list_start, const int* excluded_list,
    const int* excluded_atom_numbers, VECTOR* frc, int need_energy,
    float* atom_ene, LTMatrix3* atom_virial)
{
    MPI_PME_Excluded_Force_With_Atom_Energy(
        atom_numbers, NULL, NULL, crd, boundary, charge, excluded_list_start,
        excluded_list, excluded_atom_numbers, frc, need_energy, atom_ene,
        atom_virial != NULL, atom_virial);
}

// PM_force.cpp:1070-1168
void Particle_Mesh::PME_Reciprocal_Force_With_Energy_And_Virial(
    const VECTOR* crd, const Boundary boundary, const float* charge,
    VECTOR* force, int need_virial, int need_energy, LTMatrix3* d_virial,
    float* d_potential, int step)
{
    if (!is_initialized) return;
    check(controller,
          snb_pme_reciprocal_force(handle, (const float*)crd, to_snb(boundary),
                                   charge, (float*)force, need_virial,
                                   need_energy, (float*)d_virial, d_potential,
                                   step, NULL),
          "Particle_Mesh::PME_Reciprocal_Force_With_Energy_And_Virial");
}

// PM_force.cpp:1254-1266
void Particle_Mesh::Update_Box(const Boundary boundary, LTMatrix3 g, float dt)
{
    if (!is_initialized) return;
    float g6[6] = {g.a11, g.a21, g.a22, g.a31, g.a32, g.a33};
    check(controller, snb_pme_update_box(handle, to_snb(boundary), g6, dt),
          "Particle_Mesh::Update_Box");
}

// PM_force.cpp:1844-1869 (one process)
void Particle_Mesh::Step_Print(CONTROLLER* controller)
{
    if (!is_initialized) return;
    double rec = 0.0, self = 0.0, vir[6];
    check(controller, snb_pme_energies(handle, &rec, &self, vir, NULL),
          "Particle_Mesh::Step_Print");
    reciprocal_ene = (float)rec;
    self_ene = (float)self;
    direct_ene = device_sum(d_direct_atom_energy, atom_numbers);
    correction_ene = device_sum(d_correction_atom_energy, atom_numbers);
    ee_ene = direct_ene + reciprocal_ene + self_ene + correction_ene;
    controller->Step_Print(module_name, ee_ene, true);
    if (print_detail)
    {
        controller->Step_Print("PM_direct", direct_ene);
        controller->Step_Print("PM_reciprocal", reciprocal_ene);
        controller->Step_Print("PM_self", self_ene);
        controller->Step_Print("PM_correction", correction_ene);
    }
}

// PM_force.cpp:1819-1842.  One domain: id1/id2 (the local-global maps) are
// the identity and are not read.
void Particle_Mesh::MPI_PME_Excluded_Force_With_Atom_Energy(
    const int N, const int* id1, const int* id2, const VECTOR* crd,
    const Boundary boundary, const float* charge,
    const int* excluded_list_start, const int* excluded_list,
    const int* excluded_atom_numbers, VECTOR* frc, int need_energy,
    float* atom_ene, int need_virial, LTMatrix3* atom_virial)
{
    if (!is_initialized) return;
    if (need_energy)
        deviceMemset(d_correction_atom_energy, 0, sizeof(float) * N);
    check(controller,
          snb_pme_excluded_force(handle, N, id1, id2, (const float*)crd,
                                 to_snb(boundary), charge, excluded_list_start,
                                 excluded_list, excluded_atom_numbers,
                                 (float*)frc, need_energy,
                                 d_correction_atom_energy, need_virial,
                                 (float*)atom_virial, NULL),
          "Particle_Mesh::MPI_PME_Excluded_Force_With_Atom_Energy");
    if (need_energy && atom_ene != NULL)
        Launch_Device_Kernel(Add_Atom_List,
                             (N + CONTROLLER::device_max_thread - 1) /
                                 CONTROLLER::device_max_thread,
                             CONTROLLER::device_max_thread, 0, NULL, N,
                             atom_ene, d_correction_atom_energy);
}

}  // namespace snb_adapter
