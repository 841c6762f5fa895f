// PME excluded-pair correction that allocates no device memory.
//
// snb_pme_excluded_force_noalloc computes what snb_pme_excluded_force
// computes with fixed-point accumulation (same kernels, same fixed-point
// sums), but it takes no snb_pme handle and never calls an allocator: the
// fixed-point accumulator it scatters into is the file-scope device array
// below, sized for SNB_NOALLOC_MAX_ATOMS atoms.  It exists for callers that
// cannot allocate device memory while they run -- for instance a simulation
// loop sharing the GPU with a caching allocator that has reserved the rest of
// HBM, or a host loop that must not take the device-wide synchronisation a
// cudaMalloc/cudaFree may imply -- and for callers that keep no handle.
//
// Rules the caller must follow (also stated in include/sponge_nb.h):
//  * The scratch is one per device and per process.  Two calls on the same
//    device that may run at the same time (different unordered streams, or
//    concurrent host threads each with their own stream) race on it and give
//    wrong forces.  Order the calls: one stream, or events between streams.
//  * The scratch must hold zeros when a call starts.  The first call on each
//    device clears it; every call that completes leaves every word it touched
//    at zero again (the unpack kernel resets what it reads).  A call that
//    returns an error after launching work marks the device's scratch for a
//    fresh clear on its next call.
//  * Every call looks the scratch address up with cudaGetSymbolAddress in
//    the context current on the calling thread; the first call on a device
//    (which may load the module) also enqueues the clear, so make that first
//    call before any stream capture begins.  The address is not kept between
//    calls as the truth: after cudaDeviceReset, or under another context on
//    the same device, the module is loaded again, possibly elsewhere, and a
//    changed address is cleared again before use.
#include <mutex>
#include <string>

#include "../../include/sponge_nb.h"
#include "snb_internal.h"

using namespace snb;

namespace {

// int64 words per atom: forces [3][n], energies (total, LJ, Coulomb) [3][n],
// virial [6][n] -- the layout of Accumulators with stride n.
constexpr int kWordsPerAtom = 12;
constexpr int kMaxDevices = 64;

std::mutex g_mutex;
// address seen by the last call on each device ordinal; a call that finds
// another address (a reset or another context loaded the module again)
// clears the array before using it
long long* g_scratch[kMaxDevices] = {};
bool g_needs_clear[kMaxDevices] = {};

}  // namespace

// 12 x 8 bytes x SNB_NOALLOC_MAX_ATOMS = 6 MiB of device memory per device,
// reserved when the module loads.
static __device__ __align__(256) long long
    g_excluded_scratch[kWordsPerAtom * SNB_NOALLOC_MAX_ATOMS];

extern "C" int snb_pme_excluded_force_noalloc(
    int atom_numbers, const float* crd, snb_boundary boundary, const float* charge,
    float pme_beta, const int* excluded_list_start, const int* excluded_list,
    const int* excluded_atom_numbers, float* frc, int need_energy, float* atom_ene,
    int need_virial, float* atom_virial, void* stream) {
  if (atom_numbers < 0 || atom_numbers > SNB_NOALLOC_MAX_ATOMS)
    return fail(kBadInput,
                "pme_excluded_force_noalloc: atom_numbers " +
                    std::to_string(atom_numbers) + " is outside 0.." +
                    std::to_string(SNB_NOALLOC_MAX_ATOMS) +
                    " (the size of its static scratch); use snb_pme_excluded_force");
  if (atom_numbers == 0) return kOk;
  if (!crd || !charge || !excluded_list_start || !excluded_list ||
      !excluded_atom_numbers || !frc)
    return fail(kBadInput, "pme_excluded_force_noalloc: null argument");
  if ((need_energy && !atom_ene) || (need_virial && !atom_virial))
    return fail(kBadInput, "pme_excluded_force_noalloc: energy/virial output missing");
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

  int dev = -1;
  SNB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(kNotSupported, "pme_excluded_force_noalloc: device ordinal " +
                                   std::to_string(dev) + " out of range");
  long long* scratch = nullptr;
  {
    // the address in the current context; cheap once the module is loaded
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_excluded_scratch);
    if (err != cudaSuccess)
      return fail(kCudaError,
                  std::string("pme_excluded_force_noalloc: cudaGetSymbolAddress: ") +
                      cudaGetErrorString(err));
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_scratch[dev] != static_cast<long long*>(p)) {
      g_scratch[dev] = static_cast<long long*>(p);
      g_needs_clear[dev] = true;
    }
    scratch = g_scratch[dev];
    if (g_needs_clear[dev]) {
      SNB_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(g_excluded_scratch), st));
      g_needs_clear[dev] = false;
    }
  }

  const long long n = atom_numbers;
  Accumulators acc;
  acc.n = atom_numbers;
  acc.d_f = scratch;
  acc.d_e = scratch + 3 * n;
  acc.d_elj = acc.d_e + n;
  acc.d_ec = acc.d_e + 2 * n;
  acc.d_v = scratch + 6 * n;

  Cell cell = make_cell(boundary.cell), rcell = make_cell(boundary.rcell);
  int rc = launch_excluded(atom_numbers, reinterpret_cast<const float3*>(crd), charge,
                           cell, rcell, pme_beta, excluded_list_start, excluded_list,
                           excluded_atom_numbers, nullptr, acc, kAccumFixed,
                           need_energy != 0, need_virial != 0, st);
  if (rc == kOk)
    rc = launch_unpack(atom_numbers, nullptr, acc, kAccumFixed,
                       reinterpret_cast<float3*>(frc), need_energy ? atom_ene : nullptr,
                       nullptr, nullptr, need_virial ? atom_virial : nullptr,
                       need_energy != 0, need_virial != 0, st);
  if (rc != kOk) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_needs_clear[dev] = true;
  }
  return rc;
}
