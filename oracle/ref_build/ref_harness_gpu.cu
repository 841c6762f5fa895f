/* TEST INFRASTRUCTURE ONLY -- the reference's own GPU implementation of the
 * nonbonded hot path, for comparison with the fixed-point kernels: its
 * unmodified neighbor_list.cpp, Lennard_Jones_force.cpp, PM_force.cpp,
 * bond.cpp, angle.cpp and common.cpp compiled as CUDA with the definitions
 * and flags of its CMake CUDA build (USE_GPU, USE_CUDA, --use_fast_math,
 * -O3; cmake/parallel/cuda.cmake, cmake/utils/common.cmake) by
 * oracle/Makefile into oracle/_ref/libsponge_ref_gpu.so.  This is the plain
 * FP32 float-atomic GPU path.
 *
 * main.cpp and MD_core need HDF5 and do not build, so this file drives the
 * modules itself, in the order main.cpp:1385-1544 calls them for one step
 * with one rank: force reset (Reset_Force_and_Virial), conditional neighbor
 * update, excluded PME correction, LJ + direct Coulomb, long-range LJ
 * correction, angle, bond, PME reciprocal.  The NVE leap-frog of
 * MD_core/nve.hpp:3-16 (v += dt f / m; x += dt v) is written out here, and
 * the forced list update that the one-rank domain refresh makes every 100
 * steps follows it (main.cpp:1802-1822).
 * Every launch goes to the legacy default stream, as in the reference.
 * Nothing here computes a force, list or energy of the path itself. */
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "Lennard_Jones_force/Lennard_Jones_force.h"
#include "PM_force/PM_force.h"
#include "angle/angle.h"
#include "bond/bond.h"
#include "neighbor_list/neighbor_list.h"
#include "ref_controller.h"

namespace
{
struct RefGpu
{
    int n = 0;
    int step = 0;
    Boundary boundary;
    VECTOR box;
    float cutoff = 10.0f, skin = 2.0f;
    int* d_atom_local = NULL;  // identity: one rank owns every atom
    char* d_local_label = NULL;
    int* d_excl_start = NULL;
    int* d_excl_numbers = NULL;
    int* d_excl_list = NULL;
    float* d_charge = NULL;
    float* d_inv_mass = NULL;
    VECTOR* d_crd = NULL;
    VECTOR* d_vel = NULL;
    VECTOR* d_frc = NULL;
    float* d_atom_energy = NULL;
    LTMatrix3* d_atom_virial = NULL;
    float* d_potential = NULL;
    LTMatrix3* d_virial = NULL;
    NEIGHBOR_LIST nl;
    LENNARD_JONES_INFORMATION lj;
    Particle_Mesh pm;
    BOND bond;
    ANGLE angle;
    bool bonded = false;
    // the next update is forced: the list's displacement reference (old_crd)
    // is only written by a rebuild, as after main.cpp's initial forced update
    bool need_forced = true;
};
RefGpu* g = NULL;
std::string g_err;

void check(cudaError_t e, const char* where)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(where) + ": " +
                                 cudaGetErrorString(e));
}

template <typename T>
T* device_copy(const T* h, size_t count)
{
    T* d = NULL;
    check(cudaMalloc((void**)&d, sizeof(T) * (count > 0 ? count : 1)),
          "cudaMalloc");
    if (h && count > 0)
        check(cudaMemcpy(d, h, sizeof(T) * count, cudaMemcpyHostToDevice),
              "cudaMemcpy");
    return d;
}

void parse_commands(const char* commands)
{
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
}

__global__ void leap_frog(int n, VECTOR* vel, VECTOR* crd, const VECTOR* frc,
                          const float* inv_mass, float dt)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float m = inv_mass[i];
    VECTOR v = vel[i];
    v.x += dt * (m * frc[i].x);
    v.y += dt * (m * frc[i].y);
    v.z += dt * (m * frc[i].z);
    vel[i] = v;
    VECTOR r = crd[i];
    r.x += dt * v.x;
    r.y += dt * v.y;
    r.z += dt * v.z;
    crd[i] = r;
}

/* One force evaluation in main.cpp's order (one rank, no ghosts). */
void forces(int forced, int need_energy, int need_virial, bool with_bonded)
{
    RefGpu& c = *g;
    const int n = c.n;
    cudaMemsetAsync(c.d_frc, 0, sizeof(VECTOR) * n, 0);
    if (need_energy)
    {
        cudaMemsetAsync(c.d_atom_energy, 0, sizeof(float) * n, 0);
        cudaMemsetAsync(c.d_potential, 0, sizeof(float), 0);
    }
    if (need_virial)
    {
        cudaMemsetAsync(c.d_atom_virial, 0, sizeof(LTMatrix3) * n, 0);
        cudaMemsetAsync(c.d_virial, 0, sizeof(LTMatrix3), 0);
    }
    c.nl.Update(c.d_atom_local, n, 0, c.d_crd, c.boundary, c.step,
                (forced || c.need_forced) ? 1 : 0, c.d_excl_start,
                c.d_excl_list, c.d_excl_numbers);
    c.need_forced = false;
    c.pm.MPI_PME_Excluded_Force_With_Atom_Energy(
        n, c.d_atom_local, c.d_atom_local, c.d_crd, c.boundary, c.d_charge,
        c.d_excl_start, c.d_excl_list, c.d_excl_numbers, c.d_frc, need_energy,
        c.d_atom_energy, need_virial, c.d_atom_virial);
    c.lj.LJ_PME_Direct_Force_With_Atom_Energy_And_Virial(
        n, n, 0, 0, c.d_crd, c.d_charge, c.d_frc, c.boundary, c.nl.d_nl,
        c.pm.beta, need_energy, c.d_atom_energy, need_virial, c.d_atom_virial,
        c.pm.d_direct_atom_energy);
    const float volume =
        c.boundary.cell.a11 * c.boundary.cell.a22 * c.boundary.cell.a33;
    c.lj.Long_Range_Correction(need_virial, c.d_virial, need_energy,
                               c.d_potential, volume);
    if (with_bonded && c.bonded)
    {
        c.angle.Angle_Force_With_Atom_Energy_And_Virial(
            c.d_crd, c.boundary, c.d_frc, need_energy, c.d_atom_energy,
            need_virial, c.d_atom_virial);
        c.bond.Bond_Force_With_Atom_Energy_And_Virial(
            c.d_crd, c.boundary, c.d_frc, need_energy, c.d_atom_energy,
            need_virial, c.d_atom_virial);
    }
    c.pm.PME_Reciprocal_Force_With_Energy_And_Virial(
        c.d_crd, c.boundary, c.d_charge, c.d_frc, need_virial, need_energy,
        c.d_virial, c.d_potential, c.step);
}
}  // namespace

#define REFG_TRY(...)                       \
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
    const char* refg_last_error() { return g_err.c_str(); }

    /* Same arguments as the CPU harness's ref_init (host arrays). */
    int refg_init(int n, const float* crd, const float* charge,
                  const int* lj_type, int n_types, const float* lj_A,
                  const float* lj_B, const int* excl_start,
                  const int* excl_numbers, const int* excl_list, int n_excl,
                  const float* cell6, float cutoff, float skin,
                  const char* commands, float* beta_out)
    {
        REFG_TRY({
            if (g) throw std::runtime_error("refg_init: already initialised");
            g = new RefGpu();
            g->n = n;
            g->cutoff = cutoff;
            g->skin = skin;
            controller.commands.clear();
            parse_commands(commands);
            g->boundary.policy = BoundaryPolicy::Periodic;
            g->boundary.cell = LTMatrix3(cell6[0], cell6[1], cell6[2],
                                         cell6[3], cell6[4], cell6[5]);
            g->boundary.rcell = Invert_Lower_Triangular_Cell(g->boundary.cell);
            g->box = VECTOR(cell6[0], cell6[2], cell6[5]);
            std::vector<int> ident(n);
            for (int i = 0; i < n; ++i) ident[i] = i;
            std::vector<char> label(n, 1);
            std::vector<int> el(excl_list, excl_list + (n_excl > 0 ? n_excl : 0));
            el.push_back(0);
            g->d_atom_local = device_copy(ident.data(), n);
            g->d_local_label = device_copy(label.data(), n);
            g->d_excl_start = device_copy(excl_start, n);
            g->d_excl_numbers = device_copy(excl_numbers, n);
            g->d_excl_list = device_copy(el.data(), el.size());
            g->d_charge = device_copy(charge, n);
            g->d_crd = device_copy((const VECTOR*)crd, n);
            g->d_vel = device_copy((const VECTOR*)NULL, n);
            g->d_frc = device_copy((const VECTOR*)NULL, n);
            g->d_inv_mass = device_copy((const float*)NULL, n);
            g->d_atom_energy = device_copy((const float*)NULL, n);
            g->d_atom_virial = device_copy((const LTMatrix3*)NULL, n);
            g->d_potential = device_copy((const float*)NULL, 1);
            g->d_virial = device_copy((const LTMatrix3*)NULL, 1);
            check(cudaMemset(g->d_vel, 0, sizeof(VECTOR) * n), "memset");

            auto& ljff = Xponge::system.classical_force_field.lj;
            ljff.atom_type.assign(lj_type, lj_type + n);
            const int npair = n_types * (n_types + 1) / 2;
            ljff.pair_A.assign(lj_A, lj_A + npair);
            ljff.pair_B.assign(lj_B, lj_B + npair);
            ljff.atom_type_numbers = n_types;

            g->lj.Initial(&controller, cutoff);
            g->pm.Initial(&controller, n, g->boundary, g->box, cutoff, 0);
            g->nl.Initial(&controller, n, cutoff, skin, g->boundary);
            g->lj.Get_Local(g->d_atom_local, n, 0);
            if (beta_out) *beta_out = g->pm.beta;
            check(cudaDeviceSynchronize(), "refg_init");
        });
        return 0;
    }

    int refg_grid(int* fft3)
    {
        if (!g) return -1;
        fft3[0] = g->pm.fftx;
        fft3[1] = g->pm.ffty;
        fft3[2] = g->pm.fftz;
        return 0;
    }

    /* The reference's BOND and ANGLE modules over the given terms
     * (Xponge::system's bond and angle tables, then Get_Local). */
    int refg_set_bonded(int nb, const int* ba, const int* bb, const float* bk,
                        const float* br0, int na, const int* aa, const int* ab,
                        const int* ac, const float* ak, const float* at0)
    {
        if (!g) return -1;
        REFG_TRY({
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
            g->bond.Initial(&controller, NULL, NULL);
            g->angle.Initial(&controller);
            g->bond.Get_Local(g->d_atom_local, g->n, 0, g->d_local_label,
                              g->d_atom_local);
            g->angle.Get_Local(g->d_atom_local, g->n, 0, g->d_local_label,
                               g->d_atom_local);
            g->bonded = true;
            check(cudaDeviceSynchronize(), "refg_set_bonded");
        });
        return 0;
    }

    /* crd, vel, inv_mass: host arrays (vel and inv_mass may be NULL). */
    int refg_set_state(const float* crd, const float* vel,
                       const float* inv_mass)
    {
        if (!g) return -1;
        REFG_TRY({
            const size_t b = sizeof(VECTOR) * g->n;
            check(cudaMemcpy(g->d_crd, crd, b, cudaMemcpyHostToDevice), "crd");
            if (vel)
                check(cudaMemcpy(g->d_vel, vel, b, cudaMemcpyHostToDevice),
                      "vel");
            if (inv_mass)
                check(cudaMemcpy(g->d_inv_mass, inv_mass, sizeof(float) * g->n,
                                 cudaMemcpyHostToDevice),
                      "inv_mass");
            g->need_forced = true;
        });
        return 0;
    }

    int refg_get_state(float* crd, float* vel)
    {
        if (!g) return -1;
        REFG_TRY({
            const size_t b = sizeof(VECTOR) * g->n;
            if (crd)
                check(cudaMemcpy(crd, g->d_crd, b, cudaMemcpyDeviceToHost),
                      "crd");
            if (vel)
                check(cudaMemcpy(vel, g->d_vel, b, cudaMemcpyDeviceToHost),
                      "vel");
        });
        return 0;
    }

    /* One nonbonded force evaluation on the current coordinates; copies out
     * (when non-NULL) frc[3n], atom_energy[n] (LJ + direct + excluded, per
     * atom), potential[1] (reciprocal + self + LRC: element 0 of the
     * caller's energy array) and virial6 (the box virial, element 0). */
    int refg_force(int forced, int need_energy, int need_virial, float* frc,
                   float* atom_energy, float* potential, float* virial6)
    {
        if (!g) return -1;
        REFG_TRY({
            forces(forced, need_energy, need_virial, false);
            check(cudaDeviceSynchronize(), "refg_force");
            const int n = g->n;
            if (frc)
                check(cudaMemcpy(frc, g->d_frc, sizeof(VECTOR) * n,
                                 cudaMemcpyDeviceToHost),
                      "frc");
            if (atom_energy && need_energy)
                check(cudaMemcpy(atom_energy, g->d_atom_energy,
                                 sizeof(float) * n, cudaMemcpyDeviceToHost),
                      "atom_energy");
            if (potential && need_energy)
                check(cudaMemcpy(potential, g->d_potential, sizeof(float),
                                 cudaMemcpyDeviceToHost),
                      "potential");
            if (virial6 && need_virial)
            {
                std::vector<LTMatrix3> v(n + 1);
                check(cudaMemcpy(v.data(), g->d_atom_virial,
                                 sizeof(LTMatrix3) * n, cudaMemcpyDeviceToHost),
                      "virial");
                check(cudaMemcpy(&v[n], g->d_virial, sizeof(LTMatrix3),
                                 cudaMemcpyDeviceToHost),
                      "virial");
                double s[6] = {0, 0, 0, 0, 0, 0};
                for (int i = 0; i <= n; ++i)
                {
                    s[0] += v[i].a11;
                    s[1] += v[i].a21;
                    s[2] += v[i].a22;
                    s[3] += v[i].a31;
                    s[4] += v[i].a32;
                    s[5] += v[i].a33;
                }
                for (int k = 0; k < 6; ++k) virial6[k] = (float)s[k];
            }
        });
        return 0;
    }

    /* `steps` NVE steps (forces with bonded terms, then leap-frog), no
     * energies or virials, as on the reference's non-print steps.  *ms gets
     * their device time from CUDA events on the legacy stream. */
    int refg_md_steps(int steps, float dt, float* ms)
    {
        if (!g) return -1;
        REFG_TRY({
            cudaEvent_t e0, e1;
            check(cudaEventCreate(&e0), "event");
            check(cudaEventCreate(&e1), "event");
            check(cudaDeviceSynchronize(), "refg_md_steps");
            check(cudaEventRecord(e0, 0), "record");
            const int blocks =
                (g->n + CONTROLLER::device_max_thread - 1) /
                CONTROLLER::device_max_thread;
            for (int s = 0; s < steps; ++s)
            {
                forces(0, 0, 0, true);
                leap_frog<<<blocks, CONTROLLER::device_max_thread>>>(
                    g->n, g->d_vel, g->d_crd, g->d_frc, g->d_inv_mass, dt);
                // one rank: the domain refresh every update_interval (100)
                // steps is a forced list update (main.cpp:1802-1822)
                if ((g->step + 1) % 100 == 0)
                    g->nl.Update(g->d_atom_local, g->n, 0, g->d_crd,
                                 g->boundary, g->step, 1, g->d_excl_start,
                                 g->d_excl_list, g->d_excl_numbers);
                g->step++;
            }
            check(cudaEventRecord(e1, 0), "record");
            check(cudaEventSynchronize(e1), "refg_md_steps");
            float t = 0.f;
            check(cudaEventElapsedTime(&t, e0, e1), "elapsed");
            if (ms) *ms = t;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            check(cudaGetLastError(), "refg_md_steps");
        });
        return 0;
    }

    /* Entries of the current half list and the list-overflow flag. */
    int refg_pair_count(long long* count, int* overflow)
    {
        if (!g) return -1;
        REFG_TRY({
            std::vector<ATOM_GROUP> h(g->n);
            check(cudaMemcpy(h.data(), g->nl.d_nl, sizeof(ATOM_GROUP) * g->n,
                             cudaMemcpyDeviceToHost),
                  "nl");
            long long t = 0;
            for (int i = 0; i < g->n; ++i) t += h[i].atom_numbers;
            *count = t;
            if (overflow)
                check(cudaMemcpy(overflow, g->nl.d_neighbor_list_overflow,
                                 sizeof(int), cudaMemcpyDeviceToHost),
                      "overflow");
        });
        return 0;
    }
}
