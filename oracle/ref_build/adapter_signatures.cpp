/* TEST INFRASTRUCTURE ONLY -- compiles the adapter header beside the
 * reference's own module headers and holds the type of every adapter member
 * equal to the type of the reference member it replaces (the class part of
 * the member-function pointer taken off).  A mismatch stops the build at
 * the static_assert that names it.  Nothing here runs. */
#include <type_traits>

#include "Lennard_Jones_force/LJ_soft_core.h"
#include "Lennard_Jones_force/Lennard_Jones_force.h"
#include "PM_force/PM_force.h"
#include "neighbor_list/neighbor_list.h"
#include "sponge_nb_adapter.h"

namespace
{
template <typename M>
struct member_type;
template <typename C, typename R, typename... A>
struct member_type<R (C::*)(A...)>
{
    using type = R(A...);
};

#define SAME_MEMBER(REF, NAME)                                                 \
    static_assert(                                                             \
        std::is_same<member_type<decltype(&::REF::NAME)>::type,                \
                     member_type<decltype(&snb_adapter::REF::NAME)>::type>::value, \
        #REF "::" #NAME " differs from the reference")

// neighbor_list.h:17-24
SAME_MEMBER(NEIGHBOR_LIST, Initial);
SAME_MEMBER(NEIGHBOR_LIST, Update);
SAME_MEMBER(NEIGHBOR_LIST, Check_Overflow);
SAME_MEMBER(NEIGHBOR_LIST, Clear);

// Lennard_Jones_force.h:118-172
SAME_MEMBER(LENNARD_JONES_INFORMATION, Initial);
SAME_MEMBER(LENNARD_JONES_INFORMATION, LJ_Malloc);
SAME_MEMBER(LENNARD_JONES_INFORMATION, Parameter_Host_To_Device);
SAME_MEMBER(LENNARD_JONES_INFORMATION, Get_Local);
SAME_MEMBER(LENNARD_JONES_INFORMATION,
            LJ_PME_Direct_Force_With_Atom_Energy_And_Virial);
SAME_MEMBER(LENNARD_JONES_INFORMATION, Long_Range_Correction);
SAME_MEMBER(LENNARD_JONES_INFORMATION, Step_Print);

// LJ_soft_core.h:238-274
SAME_MEMBER(LJ_SOFT_CORE, Initial);
SAME_MEMBER(LJ_SOFT_CORE, LJ_Soft_Core_Malloc);
SAME_MEMBER(LJ_SOFT_CORE, Clear);
SAME_MEMBER(LJ_SOFT_CORE, Parameter_Host_To_Device);
SAME_MEMBER(LJ_SOFT_CORE,
            LJ_Soft_Core_PME_Direct_Force_With_Atom_Energy_And_Virial);
SAME_MEMBER(LJ_SOFT_CORE, Step_Print);
SAME_MEMBER(LJ_SOFT_CORE, Long_Range_Correction);
SAME_MEMBER(LJ_SOFT_CORE, Get_Partial_H_Partial_Lambda_With_Columb_Direct);
SAME_MEMBER(LJ_SOFT_CORE, Get_Local);

// PM_force.h:153-190
SAME_MEMBER(Particle_Mesh, Initial);
SAME_MEMBER(Particle_Mesh, Clear);
SAME_MEMBER(Particle_Mesh, PME_Excluded_Force_With_Atom_Energy);
SAME_MEMBER(Particle_Mesh, PME_Reciprocal_Force_With_Energy_And_Virial);
SAME_MEMBER(Particle_Mesh, Update_Box);
SAME_MEMBER(Particle_Mesh, Step_Print);
SAME_MEMBER(Particle_Mesh, MPI_PME_Excluded_Force_With_Atom_Energy);

// the fields main.cpp hands from one module to another
static_assert(std::is_same<decltype(::NEIGHBOR_LIST::d_nl),
                           decltype(snb_adapter::NEIGHBOR_LIST::d_nl)>::value,
              "NEIGHBOR_LIST::d_nl");
static_assert(std::is_same<decltype(::Particle_Mesh::beta),
                           decltype(snb_adapter::Particle_Mesh::beta)>::value,
              "Particle_Mesh::beta");
static_assert(
    std::is_same<decltype(::Particle_Mesh::d_direct_atom_energy),
                 decltype(snb_adapter::Particle_Mesh::d_direct_atom_energy)>::value,
    "Particle_Mesh::d_direct_atom_energy");
static_assert(int(::NEIGHBOR_LIST::FORCED_UPDATE) ==
                      int(snb_adapter::NEIGHBOR_LIST::FORCED_UPDATE) &&
                  int(::NEIGHBOR_LIST::CONDITIONAL_UPDATE) ==
                      int(snb_adapter::NEIGHBOR_LIST::CONDITIONAL_UPDATE),
              "NEIGHBOR_LIST update modes");
}  // namespace
