/* TEST INFRASTRUCTURE ONLY -- drives one force evaluation through the
 * reference-side adapter (sponge_nb_adapter.h) the way main.cpp drives the
 * reference's modules for one rank and one step (main.cpp:1385-1544:
 * forced list update, excluded PME correction, LJ + direct Coulomb,
 * long-range LJ correction, PME reciprocal; then Step_Print), with the LJ
 * tables placed in Xponge::system as the reference's loaders leave them.
 * Built with the reference's CUDA definitions by oracle/Makefile into
 * oracle/_ref/libsponge_nb_adapter.so, linked to libsponge_nb.so; the
 * -m gpu test compares what it returns with the same calls made on the C ABI
 * directly. */
#include <cuda_runtime.h>

#include <vector>

#include "ref_controller.h"
#include "sponge_nb_adapter.h"

namespace
{
template <typename T>
T* to_device(const T* h, size_t n)
{
    T* d = NULL;
    Device_Malloc_Safely((void**)&d, sizeof(T) * (n > 0 ? n : 1));
    if (n > 0) deviceMemcpy(d, h, sizeof(T) * n, deviceMemcpyHostToDevice);
    return d;
}
template <typename T>
T* zeros(size_t n)
{
    T* d = NULL;
    Device_Malloc_Safely((void**)&d, sizeof(T) * (n > 0 ? n : 1));
    deviceMemset(d, 0, sizeof(T) * (n > 0 ? n : 1));
    return d;
}
}  // namespace

extern "C"
{
/* One force evaluation of n atoms in the periodic cell {a11..a33} (its
 * inverse rcell6), lengths (a11, a22, a33) for the PME grid.  Outputs (host):
 *   frc[3n], atom_energy[n], atom_virial[6n]  (the arrays main.cpp sums)
 *   virial6: the box virial the LJ tail and PME reciprocal add to
 *   potential: the potential the LJ tail and PME reciprocal add to
 *   prints[9]: LJ_short, LJ_long, LJ, PM, PM_direct, PM_reciprocal, PM_self,
 *              PM_correction, pme beta
 * Returns 0; an error inside exits the process through
 * CONTROLLER::Throw_SPONGE_Error, as the reference does. */
int adapter_force(int n, const float* h_crd, const float* h_charge, int n_types,
                  const int* h_type, const float* h_A, const float* h_B,
                  const int* h_excl_start, const int* h_excl_numbers, int n_excl,
                  const int* h_excl_list, const float* cell6, const float* rcell6,
                  float cutoff, float skin, float* frc, float* atom_energy,
                  float* atom_virial, float* virial6, float* potential,
                  float* prints)
{
    auto& lj_in = Xponge::system.classical_force_field.lj;
    lj_in.atom_type.assign(h_type, h_type + n);
    lj_in.pair_A.assign(h_A, h_A + n_types * (n_types + 1) / 2);
    lj_in.pair_B.assign(h_B, h_B + n_types * (n_types + 1) / 2);
    lj_in.atom_type_numbers = n_types;
    controller.commands["PM_print_detail"] = "1";

    Boundary boundary;
    boundary.policy = BoundaryPolicy::Periodic;
    boundary.cell = LTMatrix3(cell6[0], cell6[1], cell6[2], cell6[3], cell6[4],
                              cell6[5]);
    boundary.rcell = LTMatrix3(rcell6[0], rcell6[1], rcell6[2], rcell6[3],
                               rcell6[4], rcell6[5]);
    VECTOR box_length = {cell6[0], cell6[2], cell6[5]};
    float volume = cell6[0] * cell6[2] * cell6[5];

    std::vector<int> local(n);
    for (int i = 0; i < n; i++) local[i] = i;
    VECTOR* d_crd = to_device((const VECTOR*)h_crd, n);
    float* d_charge = to_device(h_charge, n);
    int* d_local = to_device(local.data(), n);
    int* d_es = to_device(h_excl_start, n);
    int* d_en = to_device(h_excl_numbers, n);
    int* d_el = to_device(h_excl_list, n_excl);
    VECTOR* d_frc = zeros<VECTOR>(n);
    float* d_energy = zeros<float>(n);
    LTMatrix3* d_atom_virial = zeros<LTMatrix3>(n);
    LTMatrix3* d_virial = zeros<LTMatrix3>(1);
    float* d_potential = zeros<float>(1);

    snb_adapter::NEIGHBOR_LIST neighbor_list;
    snb_adapter::LENNARD_JONES_INFORMATION lj;
    snb_adapter::Particle_Mesh pm;
    pm.Initial(&controller, n, boundary, box_length, cutoff, 0);
    lj.Initial(&controller, cutoff);
    neighbor_list.Initial(&controller, n, cutoff, skin, boundary);
    lj.Get_Local(d_local, n, 0);

    neighbor_list.Update(d_local, n, 0, d_crd, boundary, 0,
                         neighbor_list.FORCED_UPDATE, d_es, d_el, d_en);
    pm.MPI_PME_Excluded_Force_With_Atom_Energy(n, d_local, d_local, d_crd,
                                               boundary, d_charge, d_es, d_el,
                                               d_en, d_frc, 1, d_energy, 1,
                                               d_atom_virial);
    lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
        n, n, 0, 0, d_crd, d_charge, d_frc, boundary, neighbor_list.d_nl,
        pm.beta, 1, d_energy, 1, d_atom_virial, pm.d_direct_atom_energy);
    lj.Long_Range_Correction(1, d_virial, 1, d_potential, volume);
    pm.PME_Reciprocal_Force_With_Energy_And_Virial(d_crd, boundary, d_charge,
                                                   d_frc, 1, 1, d_virial,
                                                   d_potential, 0);
    neighbor_list.Check_Overflow(&controller, 99, boundary, &boundary.cell);
    cudaDeviceSynchronize();
    lj.Step_Print(&controller);
    pm.Step_Print(&controller);

    deviceMemcpy(frc, d_frc, sizeof(VECTOR) * n, deviceMemcpyDeviceToHost);
    deviceMemcpy(atom_energy, d_energy, sizeof(float) * n, deviceMemcpyDeviceToHost);
    deviceMemcpy(atom_virial, d_atom_virial, sizeof(LTMatrix3) * n,
                 deviceMemcpyDeviceToHost);
    deviceMemcpy(virial6, d_virial, sizeof(LTMatrix3), deviceMemcpyDeviceToHost);
    deviceMemcpy(potential, d_potential, sizeof(float), deviceMemcpyDeviceToHost);
    const float p[9] = {lj.h_LJ_energy_sum, lj.h_LJ_long_energy,
                        lj.h_LJ_energy_sum + lj.h_LJ_long_energy, pm.ee_ene,
                        pm.direct_ene, pm.reciprocal_ene, pm.self_ene,
                        pm.correction_ene, pm.beta};
    for (int k = 0; k < 9; k++) prints[k] = p[k];

    neighbor_list.Clear();
    lj.Clear();
    pm.Clear();
    void* bufs[] = {d_crd, d_charge, d_local, d_es, d_en, d_el, d_frc,
                    d_energy, d_atom_virial, d_virial, d_potential};
    for (void* b : bufs) deviceFree(b);
    return (int)cudaGetLastError();
}
}
