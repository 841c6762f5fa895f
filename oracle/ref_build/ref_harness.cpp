/* TEST INFRASTRUCTURE ONLY -- builds the reference's own CPU implementation
 * of the nonbonded hot path (its unmodified neighbor_list.cpp,
 * Lennard_Jones_force.cpp, LJ_soft_core.cpp, PM_force.cpp, nb14.cpp,
 * settle.cpp and common.cpp,
 * compiled from the reference tree by oracle/Makefile) into oracle/_ref/.
 *
 * The reference's MD_core, Domain_decomposition, Xponge loaders and CONTROLLER
 * implementation need HDF5 / toml++ and are not compiled.  This file supplies
 * what the hot-path modules use of them: the CONTROLLER command map, printing
 * and error entry points, the global Xponge::system, plus C entry points that
 * let Python drive the modules on a synthetic system (host pointers: the CPU
 * backend's "device" memory is host memory).  Nothing here re-implements the
 * path itself; every force, list and energy comes from the reference code. */
#include <omp.h>

#include <stdexcept>
#include <string>

#include "Lennard_Jones_force/LJ_soft_core.h"
#include "angle/angle.h"
#include "bond/bond.h"
#include "virtual_atoms/virtual_atom_math.h"
#include "Lennard_Jones_force/Lennard_Jones_force.h"
#include "PM_force/PM_force.h"
#include "constrain/settle.h"
#include "nb14/nb14.h"
#include "neighbor_list/neighbor_list.h"
#include "ref_controller.h"
#include "xponge/load/native/angle.hpp"
#include "xponge/load/native/bond.hpp"
#include "xponge/load/native/lj.hpp"
#include "xponge/load/native/lj_soft.hpp"
#include "xponge/load/native/md_core.hpp"
#include "xponge/load/native/nb14.hpp"
#include "xponge/load/native/virtual_atoms.hpp"

/* --------------------------- the system --------------------------- */
namespace
{
struct RefContext
{
    int n = 0;
    Boundary boundary;
    VECTOR box;
    float cutoff = 10.0f, skin = 2.0f;
    std::vector<int> atom_local;
    std::vector<int> excl_start, excl_numbers, excl_list;
    std::vector<float> charge;
    NEIGHBOR_LIST nl;
    LENNARD_JONES_INFORMATION lj;
    Particle_Mesh pm;
    LJ_SOFT_CORE lj_soft;
    bool soft_ready = false;
    bool ready = false;
};
RefContext* g = NULL;
Xponge::System g_native;
std::string g_err;
}  // namespace

#define REF_TRY(...)                       \
    try                                    \
    {                                      \
        __VA_ARGS__;                       \
    }                                      \
    catch (const std::exception& e)        \
    {                                      \
        g_err = e.what();                  \
        fprintf(stderr, "%s\n", e.what()); \
        return -1;                         \
    }

extern "C"
{
    const char* ref_last_error() { return g_err.c_str(); }
    void ref_set_threads(int t)
    {
        if (t > 0) omp_set_num_threads(t);
    }
    int ref_max_threads() { return omp_get_max_threads(); }

    /* commands: "key=value;key=value" in the reference's mdin key naming */
    int ref_init(int n, const float* crd, const float* charge,
                 const int* lj_type, int n_types, const float* lj_A,
                 const float* lj_B, const int* excl_start,
                 const int* excl_numbers, const int* excl_list, int n_excl,
                 const float* cell6, float cutoff, float skin,
                 const char* commands, float* beta_out)
    {
        REF_TRY({
            delete g;
            g = new RefContext();
            g->n = n;
            g->cutoff = cutoff;
            g->skin = skin;
            controller.commands.clear();
            std::string c = commands ? commands : "";
            size_t pos = 0;
            while (pos < c.size())
            {
                size_t end = c.find(';', pos);
                if (end == std::string::npos) end = c.size();
                std::string kv = c.substr(pos, end - pos);
                size_t eq = kv.find('=');
                if (eq != std::string::npos)
                    controller.commands[kv.substr(0, eq)] = kv.substr(eq + 1);
                pos = end + 1;
            }
            g->boundary.policy = BoundaryPolicy::Periodic;
            g->boundary.cell = LTMatrix3(cell6[0], cell6[1], cell6[2],
                                         cell6[3], cell6[4], cell6[5]);
            g->boundary.rcell = Invert_Lower_Triangular_Cell(g->boundary.cell);
            g->box = VECTOR(cell6[0], cell6[2], cell6[5]);
            g->atom_local.resize(n);
            for (int i = 0; i < n; ++i) g->atom_local[i] = i;
            g->excl_start.assign(excl_start, excl_start + n);
            g->excl_numbers.assign(excl_numbers, excl_numbers + n);
            g->excl_list.assign(excl_list, excl_list + (n_excl > 0 ? n_excl : 0));
            g->excl_list.push_back(0);
            g->charge.assign(charge, charge + n);

            auto& ljff = Xponge::system.classical_force_field.lj;
            ljff.atom_type.assign(lj_type, lj_type + n);
            int npair = n_types * (n_types + 1) / 2;
            ljff.pair_A.assign(lj_A, lj_A + npair);
            ljff.pair_B.assign(lj_B, lj_B + npair);
            ljff.atom_type_numbers = n_types;

            g->lj.Initial(&controller, cutoff);
            g->pm.Initial(&controller, n, g->boundary, g->box, cutoff, 0);
            g->nl.Initial(&controller, n, cutoff, skin, g->boundary);
            g->lj.Get_Local(g->atom_local.data(), n, 0);
            if (beta_out) *beta_out = g->pm.beta;
            g->ready = true;
        });
        return 0;
    }

    int ref_grid(int* fft3)
    {
        if (!g) return -1;
        fft3[0] = g->pm.fftx;
        fft3[1] = g->pm.ffty;
        fft3[2] = g->pm.fftz;
        return 0;
    }

    /* Runs NEIGHBOR_LIST::Update on crd (forced when forced != 0) and copies
     * the half list out: counts[n] and, when serial != NULL, the rows packed
     * back to back in list order (row i starts at sum of counts before it). */
    int ref_nl_update(const float* crd, int forced, int step, int* counts,
                      int* serial, long long cap, int* overflow)
    {
        if (!g) return -1;
        REF_TRY({
            g->nl.Update(g->atom_local.data(), g->n, 0, (VECTOR*)crd,
                         g->boundary, step, forced ? 1 : 0,
                         g->excl_start.data(), g->excl_list.data(),
                         g->excl_numbers.data());
            long long off = 0;
            for (int i = 0; i < g->n; ++i)
            {
                ATOM_GROUP a = g->nl.d_nl[i];
                counts[i] = a.atom_numbers;
                if (serial && off + a.atom_numbers <= cap)
                    memcpy(serial + off, a.atom_serial,
                           sizeof(int) * a.atom_numbers);
                off += a.atom_numbers;
            }
            if (overflow)
            {
                overflow[0] = g->nl.d_neighbor_list_overflow[0];
                overflow[1] = g->nl.d_neighbor_grid_overflow[0];
            }
        });
        return 0;
    }

    /* NEIGHBOR_LIST::Update alone (no copy-out): for timing the reference. */
    int ref_nl_update_only(const float* crd, int forced, int step)
    {
        if (!g) return -1;
        REF_TRY({
            g->nl.Update(g->atom_local.data(), g->n, 0, (VECTOR*)crd,
                         g->boundary, step, forced ? 1 : 0,
                         g->excl_start.data(), g->excl_list.data(),
                         g->excl_numbers.data());
        });
        return 0;
    }

    /* LJ_PME_Direct_Force_With_Atom_Energy_And_Virial with energy and virial.
     * frc/atom_energy/atom_virial are accumulated into; lj_energy and
     * coulomb_energy receive the module's per-atom arrays. */
    int ref_lj_direct(const float* crd, float* frc, float* atom_energy,
                      float* atom_virial, float* lj_energy,
                      float* coulomb_energy, int need_energy, int need_virial)
    {
        if (!g) return -1;
        REF_TRY({
            std::vector<float> direct(g->n, 0.0f);
            g->lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
                g->n, g->n, 0, 0, (const VECTOR*)crd, g->charge.data(),
                (VECTOR*)frc, g->boundary, g->nl.d_nl, g->pm.beta, need_energy,
                atom_energy, need_virial, (LTMatrix3*)atom_virial,
                direct.data());
            if (lj_energy)
                memcpy(lj_energy, g->lj.d_LJ_energy_atom, sizeof(float) * g->n);
            if (coulomb_energy)
                memcpy(coulomb_energy, direct.data(), sizeof(float) * g->n);
        });
        return 0;
    }

    /* PME_Reciprocal_Force_With_Energy_And_Virial: reciprocal forces into frc,
     * self+reciprocal energy into potential[0], virial into virial6. */
    int ref_pme_reciprocal(const float* crd, float* frc, float* virial6,
                           float* potential, float* parts, int need_energy,
                           int need_virial, int step)
    {
        if (!g) return -1;
        REF_TRY({
            g->pm.PME_Reciprocal_Force_With_Energy_And_Virial(
                (const VECTOR*)crd, g->boundary, g->charge.data(),
                (VECTOR*)frc, need_virial, need_energy, (LTMatrix3*)virial6,
                potential, step);
            if (parts)
            {
                parts[0] = g->pm.d_reciprocal_ene[0];
                parts[1] = g->pm.d_self_ene[0];
            }
        });
        return 0;
    }

    int ref_pme_excluded(const float* crd, float* frc, float* atom_energy,
                         float* atom_virial, int need_energy, int need_virial)
    {
        if (!g) return -1;
        REF_TRY({
            g->pm.MPI_PME_Excluded_Force_With_Atom_Energy(
                g->n, g->atom_local.data(), g->atom_local.data(),
                (const VECTOR*)crd, g->boundary, g->charge.data(),
                g->excl_start.data(), g->excl_list.data(),
                g->excl_numbers.data(), (VECTOR*)frc, need_energy,
                atom_energy, need_virial, (LTMatrix3*)atom_virial);
        });
        return 0;
    }

    int ref_lj_long_range(float* virial6, float* potential, float volume)
    {
        if (!g) return -1;
        REF_TRY({
            g->lj.Long_Range_Correction(1, (LTMatrix3*)virial6, 1, potential,
                                        volume);
        });
        return 0;
    }

    float ref_lj_long_range_factor() { return g ? g->lj.long_range_factor : 0; }

    /* A barostat's box change as main.cpp's Main_Box_Change makes it for a
     * small change (main.cpp:2055-2090): the new rectangular cell becomes the
     * boundary every later call uses, and Particle_Mesh::Update_Box
     * recomputes the influence function at the same grid size.  The
     * neighbor list keeps its Initial grid, as there. */
    int ref_box_change(const float* cell6)
    {
        if (!g) return -1;
        REF_TRY({
            g->boundary.cell = LTMatrix3(cell6[0], cell6[1], cell6[2],
                                         cell6[3], cell6[4], cell6[5]);
            g->boundary.rcell = Invert_Lower_Triangular_Cell(g->boundary.cell);
            g->box = VECTOR(cell6[0], cell6[2], cell6[5]);
            LTMatrix3 rate = LTMatrix3(0, 0, 0, 0, 0, 0);
            g->pm.Update_Box(g->boundary, rate, 0.0f);
        });
        return 0;
    }

    /* LJ_SOFT_CORE::Initial on the current system (after ref_init): end
     * state types and tables, subsystem masks; lambda_lj and soft_core_*
     * come from `commands` ("key=value;..."). */
    int ref_soft_init(const int* type_A, const int* type_B, int nA, int nB,
                      const float* AA, const float* AB, const float* BA,
                      const float* BB, const int* mask, const char* commands)
    {
        if (!g) return -1;
        REF_TRY({
            std::string c = commands ? commands : "";
            size_t pos = 0;
            while (pos < c.size())
            {
                size_t end = c.find(';', pos);
                if (end == std::string::npos) end = c.size();
                std::string kv = c.substr(pos, end - pos);
                size_t eq = kv.find('=');
                if (eq != std::string::npos)
                    controller.commands[kv.substr(0, eq)] = kv.substr(eq + 1);
                pos = end + 1;
            }
            auto& sc = Xponge::system.classical_force_field.lj_soft_core;
            const int n = g->n;
            sc.atom_numbers = n;
            sc.atom_type_numbers_A = nA;
            sc.atom_type_numbers_B = nB;
            const int pA = nA * (nA + 1) / 2;
            const int pB = nB * (nB + 1) / 2;
            sc.LJ_AA.assign(AA, AA + pA);
            sc.LJ_AB.assign(AB, AB + pA);
            sc.LJ_BA.assign(BA, BA + pB);
            sc.LJ_BB.assign(BB, BB + pB);
            sc.atom_LJ_type_A.assign(type_A, type_A + n);
            sc.atom_LJ_type_B.assign(type_B, type_B + n);
            sc.subsystem_division.assign(mask, mask + n);
            g->lj_soft.Initial(&controller, g->cutoff);
            g->lj_soft.Get_Local(g->atom_local.data(), n, 0);
            g->soft_ready = true;
        });
        return 0;
    }

    /* LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial on the
     * current half list; per-atom LJ, inter/intra LJ and direct Coulomb
     * energies are copied out of the module. */
    int ref_soft_direct(const float* crd, float* frc, float* atom_energy,
                        float* atom_virial, float* lj_energy, float* inter,
                        float* intra, float* coulomb_energy, int need_energy,
                        int need_virial)
    {
        if (!g || !g->soft_ready) return -1;
        REF_TRY({
            std::vector<float> direct(g->n, 0.0f);
            g->lj_soft.LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial(
                g->n, g->n, 0, 0, (const VECTOR*)crd, g->charge.data(),
                (VECTOR*)frc, g->boundary, g->nl.d_nl, g->pm.beta, need_energy,
                atom_energy, need_virial, (LTMatrix3*)atom_virial,
                direct.data());
            const size_t b = sizeof(float) * g->n;
            if (lj_energy) memcpy(lj_energy, g->lj_soft.d_LJ_energy_atom, b);
            if (inter) memcpy(inter, g->lj_soft.d_LJ_energy_atom_intersys, b);
            if (intra) memcpy(intra, g->lj_soft.d_LJ_energy_atom_intrasys, b);
            if (coulomb_energy) memcpy(coulomb_energy, direct.data(), b);
        });
        return 0;
    }

    /* Get_Partial_H_Partial_Lambda_With_Columb_Direct: the module's return
     * value (LJ dU/dlambda plus the tail term).  The module evaluates it at
     * the coordinates of its last direct-force call. */
    int ref_soft_dhdl(const float* crd, const float* charge_B_A,
                      int charge_perturbated, float* out)
    {
        if (!g || !g->soft_ready) return -1;
        REF_TRY({
            *out = g->lj_soft.Get_Partial_H_Partial_Lambda_With_Columb_Direct(
                0, (const VECTOR*)crd, g->boundary, g->charge.data(),
                g->nl.d_nl, charge_B_A, g->pm.beta, charge_perturbated);
        });
        return 0;
    }

    int ref_soft_long_range(float* virial6, float* potential, float volume,
                            float* factors)
    {
        if (!g || !g->soft_ready) return -1;
        REF_TRY({
            g->lj_soft.Long_Range_Correction(1, (LTMatrix3*)virial6, 1,
                                             potential, volume);
            if (factors)
            {
                factors[0] = g->lj_soft.long_range_factor;
                factors[1] = g->lj_soft.long_range_factor_TI;
            }
        });
        return 0;
    }

    /* NON_BOND_14 on pairs given directly (the arrays Initial copies from
     * its loader, nb14.cpp:155-163), one call of
     * Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial after Get_Local
     * over all n atoms of a periodic box cell6.  frc [n*3], atom_energy [n]
     * and atom_virial [n*6] are added to; sums[0..1] = the per-pair LJ and
     * Coulomb energies that Step_Print sums, here summed in double. */
    int ref_nb14(int n, int m, const int* a, const int* b, const float* A,
                 const float* B, const float* cf, const float* crd,
                 const float* charge, const float* cell6, float* frc,
                 float* atom_energy, float* atom_virial, double* sums)
    {
        REF_TRY({
            NON_BOND_14 nb;
            nb.nb14_numbers = m;
            nb.Memory_Allocate();
            for (int t = 0; t < m; ++t)
            {
                nb.h_atom_a[t] = a[t];
                nb.h_atom_b[t] = b[t];
                nb.h_A[t] = A[t];
                nb.h_B[t] = B[t];
                nb.h_cf_scale_factor[t] = cf[t];
            }
            nb.Parameter_Host_To_Device();
            nb.is_initialized = 1;
            std::vector<char> label(n, 1);
            std::vector<int> id(n);
            for (int i = 0; i < n; ++i) id[i] = i;
            nb.Get_Local(id.data(), n, 0, label.data(), id.data());
            Boundary bd;
            bd.policy = BoundaryPolicy::Periodic;
            bd.cell = LTMatrix3(cell6[0], cell6[1], cell6[2], cell6[3], cell6[4],
                                cell6[5]);
            bd.rcell = Invert_Lower_Triangular_Cell(bd.cell);
            nb.Non_Bond_14_LJ_CF_Force_With_Atom_Energy_And_Virial(
                reinterpret_cast<const VECTOR*>(crd), charge, bd,
                reinterpret_cast<VECTOR*>(frc), 1, atom_energy, 1,
                reinterpret_cast<LTMatrix3*>(atom_virial));
            double lj = 0.0, ee = 0.0;
            for (int t = 0; t < m; ++t)
            {
                lj += nb.d_nb14_lj_energy[t];
                ee += nb.d_nb14_cf_energy[t];
            }
            sums[0] = lj;
            sums[1] = ee;
            void* host[] = {nb.h_atom_a, nb.h_atom_b, nb.h_A, nb.h_B,
                            nb.h_cf_scale_factor, nb.h_nb14_lj_energy_sum,
                            nb.h_nb14_cf_energy_sum};
            for (void* p : host) free(p);
            void* dev[] = {nb.d_atom_a, nb.d_atom_b, nb.d_A, nb.d_B,
                           nb.d_cf_scale_factor, nb.d_nb14_cf_energy,
                           nb.d_nb14_lj_energy, nb.d_nb14_lj_energy_sum,
                           nb.d_nb14_cf_energy_sum, nb.d_atom_a_local,
                           nb.d_atom_b_local, nb.d_A_local, nb.d_B_local,
                           nb.d_cf_scale_factor_local, nb.d_num_nb14_local};
            for (void* p : dev) deviceFree(p);
        });
        return 0;
    }

    /* BOND and ANGLE over terms given directly (Xponge::system's bond and
     * angle tables, which their Initial copies), Get_Local over all n atoms,
     * then one call each of Bond_Force_With_Atom_Energy_And_Virial and
     * Angle_Force_With_Atom_Energy_And_Virial in a periodic box cell6, each
     * into its own frc [n*3], atom_energy [n] and atom_virial [n*6] (added
     * to).  sums[0..1] = the per-term bond and angle energies that Step_Print
     * sums, here summed in double. */
    int ref_bonded(int n, int nb, const int* ba, const int* bb, const float* bk,
                   const float* br0, int na, const int* aa, const int* ab,
                   const int* ac, const float* ak, const float* at0, const float* crd,
                   const float* cell6, float* bond_frc, float* bond_energy,
                   float* bond_virial, float* angle_frc, float* angle_energy,
                   float* angle_virial, double* sums)
    {
        REF_TRY({
            auto& B = Xponge::system.classical_force_field.bonds;
            B.atom_a.assign(ba, ba + nb);
            B.atom_b.assign(bb, bb + nb);
            B.k.assign(bk, bk + nb);
            B.r0.assign(br0, br0 + nb);
            auto& A = Xponge::system.classical_force_field.angles;
            A.atom_a.assign(aa, aa + na);
            A.atom_b.assign(ab, ab + na);
            A.atom_c.assign(ac, ac + na);
            A.k.assign(ak, ak + na);
            A.theta0.assign(at0, at0 + na);
            std::vector<char> label(n, 1);
            std::vector<int> id(n);
            for (int i = 0; i < n; ++i) id[i] = i;
            Boundary bd;
            bd.policy = BoundaryPolicy::Periodic;
            bd.cell = LTMatrix3(cell6[0], cell6[1], cell6[2], cell6[3], cell6[4],
                                cell6[5]);
            bd.rcell = Invert_Lower_Triangular_Cell(bd.cell);
            sums[0] = sums[1] = 0.0;
            if (nb > 0)
            {
                BOND bond;
                bond.Initial(&controller, NULL, NULL);
                bond.Get_Local(id.data(), n, 0, label.data(), id.data());
                bond.Bond_Force_With_Atom_Energy_And_Virial(
                    reinterpret_cast<const VECTOR*>(crd), bd,
                    reinterpret_cast<VECTOR*>(bond_frc), 1, bond_energy, 1,
                    reinterpret_cast<LTMatrix3*>(bond_virial));
                for (int t = 0; t < nb; ++t) sums[0] += bond.d_bond_ene[t];
            }
            if (na > 0)
            {
                ANGLE angle;
                angle.Initial(&controller);
                angle.Get_Local(id.data(), n, 0, label.data(), id.data());
                angle.Angle_Force_With_Atom_Energy_And_Virial(
                    reinterpret_cast<const VECTOR*>(crd), bd,
                    reinterpret_cast<VECTOR*>(angle_frc), 1, angle_energy, 1,
                    reinterpret_cast<LTMatrix3*>(angle_virial));
                for (int t = 0; t < na; ++t) sums[1] += angle.d_angle_ene[t];
            }
            B = Xponge::Bonds();
            A = Xponge::Angles();
        });
        return 0;
    }

    /* Virtual atoms of types 0-3 through the reference's own position and
     * force formulas (virtual_atoms/virtual_atom_math.h), record by record:
     * positions in the given order (each record after the ones it depends
     * on), then the force of each virtual atom moved onto its sources in
     * the reverse order and set to zero (Force_Redistribute).  from [3m]
     * (unused slots ignored), param [2m]; crd [n*3] and frc [n*3] are
     * updated in place.  Returns 1 + the record of a type 3 geometry the
     * reference rejects, else 0. */
    int ref_vatom(int n, int m, const int* type, const int* virt, const int* from,
                  const float* param, const float* cell6, float* crd, float* frc)
    {
        Boundary bd;
        bd.policy = BoundaryPolicy::Periodic;
        bd.cell = LTMatrix3(cell6[0], cell6[1], cell6[2], cell6[3], cell6[4], cell6[5]);
        bd.rcell = Invert_Lower_Triangular_Cell(bd.cell);
        VECTOR* x = reinterpret_cast<VECTOR*>(crd);
        VECTOR* f = reinterpret_cast<VECTOR*>(frc);
        int bad = 0;
        for (int t = 0; t < m; ++t)
        {
            const int v = virt[t], a = from[3 * t], b = from[3 * t + 1],
                      c = from[3 * t + 2];
            const float p = param[2 * t], q = param[2 * t + 1];
            if (type[t] == 0) x[v] = Virtual_Atom_Type_0_Position(x[a], p);
            else if (type[t] == 1) x[v] = Virtual_Atom_Type_1_Position(x[a], x[b], p, bd);
            else if (type[t] == 2)
                x[v] = Virtual_Atom_Type_2_Position(x[a], x[b], x[c], p, q, bd);
            else if (!Virtual_Atom_Type_3_Position(x[a], x[b], x[c], p, q, bd, &x[v]) &&
                     !bad)
                bad = 1 + t;
        }
        for (int t = m - 1; t >= 0; --t)
        {
            const int v = virt[t], a = from[3 * t], b = from[3 * t + 1],
                      c = from[3 * t + 2];
            const float p = param[2 * t], q = param[2 * t + 1];
            const VECTOR fv = f[v];
            VECTOR f1, f2, f3;
            if (type[t] == 0)
            {
                f[a] = f[a] + Virtual_Atom_Type_0_Source_Force(fv);
            }
            else if (type[t] == 1)
            {
                Virtual_Atom_Type_1_Source_Forces(fv, p, &f1, &f2);
                f[a] = f[a] + f1;
                f[b] = f[b] + f2;
            }
            else if (type[t] == 2)
            {
                Virtual_Atom_Type_2_Source_Forces(fv, p, q, &f1, &f2, &f3);
                f[a] = f[a] + f1;
                f[b] = f[b] + f2;
                f[c] = f[c] + f3;
            }
            else
            {
                if (!Virtual_Atom_Type_3_Source_Forces(x[a], x[b], x[c], fv, p, q, bd, &f1,
                                                       &f2, &f3) &&
                    !bad)
                    bad = 1 + t;
                f[a] = f[a] + f1;
                f[b] = f[b] + f2;
                f[c] = f[c] + f3;
            }
            f[v] = VECTOR(0.0f);
        }
        return bad;
    }

    /* SETTLE on one step: Initial from the constraint pairs (atom_i,
     * atom_j, constant_r) and masses, Get_Local over all n atoms,
     * Remember_Last_Coordinates on crd_old, then Do_SETTLE with the step
     * dt (v_factor = x_factor = 1) on crd / vel, which are updated in place;
     * stress[6] receives the constraint virial / V.  counts = {triangles,
     * rigid pairs, constraint pairs left over}; left [2 m] receives the
     * atoms (i, j) of the pairs left over. */
    int ref_settle(int n, int m, const int* ai, const int* aj, const float* r0,
                   const float* mass, const float* cell6, const float* crd_old,
                   float* crd, float* vel, float dt, float* stress, int* counts,
                   int* left)
    {
        REF_TRY({
            CONSTRAIN c;
            c.atom_numbers = n;
            c.dt = dt;
            c.constrain_pair_numbers = m;
            c.h_constrain_pair = (CONSTRAIN_PAIR*)malloc(sizeof(CONSTRAIN_PAIR) * (m > 0 ? m : 1));
            c.d_constrain_pair = (CONSTRAIN_PAIR*)malloc(sizeof(CONSTRAIN_PAIR) * (m > 0 ? m : 1));
            for (int p = 0; p < m; ++p)
            {
                c.h_constrain_pair[p].atom_i_serial = ai[p];
                c.h_constrain_pair[p].atom_j_serial = aj[p];
                c.h_constrain_pair[p].constant_r = r0[p];
                c.h_constrain_pair[p].constrain_k =
                    mass[ai[p]] * mass[aj[p]] / (mass[ai[p]] + mass[aj[p]]);
            }
            std::vector<float> h_mass(mass, mass + n);
            SETTLE s;
            s.Initial(&controller, &c, h_mass.data());
            counts[0] = s.triangle_numbers;
            counts[1] = s.pair_numbers;
            counts[2] = c.constrain_pair_numbers;
            for (int p = 0; p < c.constrain_pair_numbers; ++p)
            {
                left[2 * p] = c.h_constrain_pair[p].atom_i_serial;
                left[2 * p + 1] = c.h_constrain_pair[p].atom_j_serial;
            }
            if (s.is_initialized)
            {
                std::vector<char> label(n, 1);
                std::vector<int> id(n);
                for (int i = 0; i < n; ++i) id[i] = i;
                s.Get_Local(id.data(), label.data(), n);
                Boundary bd;
                bd.policy = BoundaryPolicy::Periodic;
                bd.cell = LTMatrix3(cell6[0], cell6[1], cell6[2], cell6[3],
                                    cell6[4], cell6[5]);
                bd.rcell = Invert_Lower_Triangular_Cell(bd.cell);
                s.Remember_Last_Coordinates(
                    reinterpret_cast<const VECTOR*>(crd_old), bd);
                LTMatrix3 st = {0, 0, 0, 0, 0, 0};
                s.Do_SETTLE(&controller, id.data(), h_mass.data(),
                            reinterpret_cast<VECTOR*>(crd), bd,
                            reinterpret_cast<VECTOR*>(vel), 1, &st);
                stress[0] = st.a11;
                stress[1] = st.a21;
                stress[2] = st.a22;
                stress[3] = st.a31;
                stress[4] = st.a32;
                stress[5] = st.a33;
            }
        });
        return 0;
    }

    /* The reference's native-input loaders (xponge/load/native/*.hpp) on
     * the files named in `commands` ("key=path;..."): mass_in_file,
     * charge_in_file, exclude_in_file, LJ_in_file, LJ_soft_core_in_file,
     * subsys_division_in_file, nb14_in_file and nb14_extra_in_file, each
     * only when given.  The results stay in a
     * System of their own; ref_native_get copies one field out. */
    int ref_native_load(const char* commands)
    {
        REF_TRY({
            controller.commands.clear();
            std::string c = commands ? commands : "";
            size_t pos = 0;
            while (pos < c.size())
            {
                size_t end = c.find(';', pos);
                if (end == std::string::npos) end = c.size();
                std::string kv = c.substr(pos, end - pos);
                size_t eq = kv.find('=');
                if (eq != std::string::npos)
                    controller.commands[kv.substr(0, eq)] = kv.substr(eq + 1);
                pos = end + 1;
            }
            g_native = Xponge::System();
            if (controller.Command_Exist("mass_in_file"))
                Xponge::Native_Load_Mass(&g_native, &controller);
            if (controller.Command_Exist("charge_in_file"))
                Xponge::Native_Load_Charge(&g_native, &controller);
            if (controller.Command_Exist("exclude_in_file"))
                Xponge::Native_Load_Exclusions(&g_native, &controller);
            Xponge::Native_Load_LJ(&g_native, &controller);
            Xponge::Native_Load_LJ_Soft_Core(&g_native, &controller);
            Xponge::Native_Load_NB14(&g_native, &controller);
            if (controller.Command_Exist("virtual_atom_in_file"))
                Xponge::Native_Load_Virtual_Atoms(&g_native.virtual_atoms, &controller);
            if (controller.Command_Exist("bond_in_file"))
                Xponge::Native_Load_Bonds(&g_native.classical_force_field.bonds,
                                          &controller, "bond");
            if (controller.Command_Exist("angle_in_file"))
                Xponge::Native_Load_Angles(&g_native.classical_force_field.angles,
                                           &controller, "angle");
        });
        return 0;
    }

    /* Copies field `name` of the loaded System into out (when not NULL) and
     * returns its length, or -1 for an unknown name. */
    long long ref_native_get(const char* name, void* out)
    {
        const auto& ff = g_native.classical_force_field;
        const auto& sc = ff.lj_soft_core;
        std::string n = name ? name : "";
        auto put_f = [&](const std::vector<float>& v) -> long long {
            if (out) memcpy(out, v.data(), sizeof(float) * v.size());
            return (long long)v.size();
        };
        auto put_i = [&](const std::vector<int>& v) -> long long {
            if (out) memcpy(out, v.data(), sizeof(int) * v.size());
            return (long long)v.size();
        };
        if (n == "mass") return put_f(g_native.atoms.mass);
        if (n == "charge") return put_f(g_native.atoms.charge);
        if (n == "lj_A") return put_f(ff.lj.pair_A);
        if (n == "lj_B") return put_f(ff.lj.pair_B);
        if (n == "lj_type") return put_i(ff.lj.atom_type);
        if (n == "lj_type_numbers") return ff.lj.atom_type_numbers;
        if (n == "AA") return put_f(sc.LJ_AA);
        if (n == "AB") return put_f(sc.LJ_AB);
        if (n == "BA") return put_f(sc.LJ_BA);
        if (n == "BB") return put_f(sc.LJ_BB);
        if (n == "type_A") return put_i(sc.atom_LJ_type_A);
        if (n == "type_B") return put_i(sc.atom_LJ_type_B);
        if (n == "subsys") return put_i(sc.subsystem_division);
        if (n == "nb14_a") return put_i(ff.nb14.atom_a);
        if (n == "nb14_b") return put_i(ff.nb14.atom_b);
        if (n == "nb14_A") return put_f(ff.nb14.A);
        if (n == "nb14_B") return put_f(ff.nb14.B);
        if (n == "nb14_cf") return put_f(ff.nb14.cf_scale_factor);
        if (n == "vatom_type" || n == "vatom_virtual" || n == "vatom_from" ||
            n == "vatom_param")
        {
            // one entry per record; three sources and two parameters per
            // record, unused slots -1 / 0
            std::vector<int> vi;
            std::vector<float> vf;
            for (const auto& r : g_native.virtual_atoms.records)
            {
                if (n == "vatom_type") vi.push_back(r.type);
                if (n == "vatom_virtual") vi.push_back(r.virtual_atom);
                for (int k = 0; k < 3 && n == "vatom_from"; ++k)
                    vi.push_back(k < (int)r.from.size() ? r.from[k] : -1);
                for (int k = 0; k < 2 && n == "vatom_param"; ++k)
                    vf.push_back(k < (int)r.parameter.size() ? r.parameter[k] : 0.0f);
            }
            return n == "vatom_param" ? put_f(vf) : put_i(vi);
        }
        if (n == "bond_a") return put_i(ff.bonds.atom_a);
        if (n == "bond_b") return put_i(ff.bonds.atom_b);
        if (n == "bond_k") return put_f(ff.bonds.k);
        if (n == "bond_r0") return put_f(ff.bonds.r0);
        if (n == "angle_a") return put_i(ff.angles.atom_a);
        if (n == "angle_b") return put_i(ff.angles.atom_b);
        if (n == "angle_c") return put_i(ff.angles.atom_c);
        if (n == "angle_k") return put_f(ff.angles.k);
        if (n == "angle_theta0") return put_f(ff.angles.theta0);
        if (n == "excl_numbers" || n == "excl_list")
        {
            std::vector<int> num, list;
            for (const auto& e : g_native.exclusions.excluded_atoms)
            {
                num.push_back((int)e.size());
                list.insert(list.end(), e.begin(), e.end());
            }
            return put_i(n == "excl_numbers" ? num : list);
        }
        return -1;
    }
}
