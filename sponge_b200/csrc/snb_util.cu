// Error state, device-wide scan, accumulators and frame conversion kernels.
#include <cstdio>
#include <mutex>

#include "snb_internal.h"

namespace snb {

static std::mutex g_err_mu;
static std::string g_err;

void set_error(const std::string& msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err = msg;
}
int fail(int code, const std::string& msg) {
  set_error(msg);
  return code;
}
std::string last_error() {
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_err;
}

// ---------------------------------------------------------------------------
// Exclusive scan: per-block scan + block sums, scan of block sums, add.
__device__ __forceinline__ int block_scan_exclusive(int v, int* sh, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int nw = blockDim.x >> 5;
    int w = lane < nw ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < nw) sh[lane] = w;
  }
  __syncthreads();
  int base = warp > 0 ? sh[warp - 1] : 0;
  if (total) *total = sh[(blockDim.x >> 5) - 1];
  return base + x - v;
}

__global__ void k_scan_blocks(const int* in, int* out, int n, int* block_sums) {
  __shared__ int sh[32];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int v = i < n ? in[i] : 0;
  int tot;
  int ex = block_scan_exclusive(v, sh, &tot);
  if (i < n) out[i] = ex;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// one block scans the block sums sequentially in chunks of blockDim
__global__ void k_scan_sums(int* block_sums, int nblocks, int* out, int n,
                            int* total_out) {
  __shared__ int sh[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nblocks; base += blockDim.x) {
    int i = base + threadIdx.x;
    int v = i < nblocks ? block_sums[i] : 0;
    int tot;
    int ex = block_scan_exclusive(v, sh, &tot);
    if (i < nblocks) block_sums[i] = ex + carry;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[n] = carry;
    if (total_out) *total_out = carry;
  }
}

__global__ void k_scan_add(int* out, int n, const int* block_sums) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += block_sums[blockIdx.x];
}

int scan_reserve(ScanScratch& s, int n) {
  int nb = ceil_div(n > 0 ? n : 1, kScanBlock);
  if (nb > s.capacity_blocks) {
    if (s.block_sums) cudaFree(s.block_sums);
    SNB_CUDA_TRY(cudaMalloc(&s.block_sums, sizeof(int) * nb));
    s.capacity_blocks = nb;
  }
  return kOk;
}

// One block for short arrays (n <= 16 * blockDim.x): each thread takes a
// contiguous chunk of up to 16 entries, so one block-wide scan covers all.
__global__ void k_scan_single(const int* in, int* out, int n, int* total_out) {
  __shared__ int sh[32];
  const int c = (n + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * c;
  int v[16];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = (k < c && b + k < n) ? in[b + k] : 0;
    sum += v[k];
  }
  int tot;
  int ex = block_scan_exclusive(sum, sh, &tot);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if (k < c && b + k < n) out[b + k] = ex;
    ex += v[k];
  }
  if (threadIdx.x == 0) {
    out[n] = tot;
    if (total_out) *total_out = tot;
  }
}

int scan_exclusive(const int* in, int* out, int n, int* total_out,
                   ScanScratch& s, cudaStream_t st) {
  if (n <= 16 * kScanBlock) {
    k_scan_single<<<1, kScanBlock, 0, st>>>(in, out, n, total_out);
    SNB_CUDA_TRY(cudaGetLastError());
    return kOk;
  }
  int nb = ceil_div(n > 0 ? n : 1, kScanBlock);
  if (nb > s.capacity_blocks) {
    if (s.block_sums) cudaFree(s.block_sums);
    SNB_CUDA_TRY(cudaMalloc(&s.block_sums, sizeof(int) * nb));
    s.capacity_blocks = nb;
  }
  k_scan_blocks<<<nb, kScanBlock, 0, st>>>(in, out, n, s.block_sums);
  k_scan_sums<<<1, kScanBlock, 0, st>>>(s.block_sums, nb, out, n, total_out);
  k_scan_add<<<nb, kScanBlock, 0, st>>>(out, n, s.block_sums);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// ---------------------------------------------------------------------------
int acc_init(Accumulators& a, int n) {
  a.n = n;
  size_t N = n > 0 ? n : 1;
  SNB_CUDA_TRY(cudaMalloc(&a.d_f, sizeof(long long) * 3 * N));
  SNB_CUDA_TRY(cudaMalloc(&a.d_e, sizeof(long long) * 3 * N));
  a.d_elj = a.d_e + N;
  a.d_ec = a.d_e + 2 * N;
  SNB_CUDA_TRY(cudaMalloc(&a.d_v, sizeof(long long) * 6 * N));
  SNB_CUDA_TRY(cudaMalloc(&a.d_ff, sizeof(float) * 3 * N));
  SNB_CUDA_TRY(cudaMalloc(&a.d_fe, sizeof(float) * 3 * N));
  SNB_CUDA_TRY(cudaMalloc(&a.d_fv, sizeof(float) * 6 * N));
  SNB_CUDA_TRY(cudaMalloc(&a.d_eaux, sizeof(long long) * 2 * N));
  SNB_CUDA_TRY(cudaMalloc(&a.d_feaux, sizeof(float) * 2 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_eaux, 0, sizeof(long long) * 2 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_feaux, 0, sizeof(float) * 2 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_f, 0, sizeof(long long) * 3 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_e, 0, sizeof(long long) * 3 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_v, 0, sizeof(long long) * 6 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_ff, 0, sizeof(float) * 3 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_fe, 0, sizeof(float) * 3 * N));
  SNB_CUDA_TRY(cudaMemset(a.d_fv, 0, sizeof(float) * 6 * N));
  return kOk;
}

void acc_free(Accumulators& a) {
  cudaFree(a.d_f);
  cudaFree(a.d_e);
  cudaFree(a.d_v);
  cudaFree(a.d_ff);
  cudaFree(a.d_fe);
  cudaFree(a.d_fv);
  cudaFree(a.d_eaux);
  cudaFree(a.d_feaux);
  a = Accumulators();
}

int launch_zero_acc(Accumulators& a, int accum, bool energy, bool virial,
                    cudaStream_t st) {
  size_t N = a.n > 0 ? a.n : 1;
  if (accum == kAccumFixed) {
    SNB_CUDA_TRY(cudaMemsetAsync(a.d_f, 0, sizeof(long long) * 3 * N, st));
    if (energy) SNB_CUDA_TRY(cudaMemsetAsync(a.d_e, 0, sizeof(long long) * 3 * N, st));
    if (virial) SNB_CUDA_TRY(cudaMemsetAsync(a.d_v, 0, sizeof(long long) * 6 * N, st));
  } else {
    SNB_CUDA_TRY(cudaMemsetAsync(a.d_ff, 0, sizeof(float) * 3 * N, st));
    if (energy) SNB_CUDA_TRY(cudaMemsetAsync(a.d_fe, 0, sizeof(float) * 3 * N, st));
    if (virial) SNB_CUDA_TRY(cudaMemsetAsync(a.d_fv, 0, sizeof(float) * 6 * N, st));
  }
  return kOk;
}

// ---------------------------------------------------------------------------
// pos[s] = (crd[perm[s]], charge[perm[s]]), type_sorted[s] = type[perm[s]]
__global__ void k_pack(int n, const float3* __restrict__ crd,
                       const float* __restrict__ charge,
                       const int* __restrict__ type, const int* __restrict__ perm,
                       float4* __restrict__ pos, int* __restrict__ type_sorted,
                       const float3* __restrict__ img_off) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i = perm ? perm[s] : s;
  float3 r = crd[i];
  if (img_off) {
    const float3 o = img_off[s];
    r = make_float3(r.x - o.x, r.y - o.y, r.z - o.z);
  }
  pos[s] = make_float4(r.x, r.y, r.z, charge[i]);
  if (type_sorted) type_sorted[s] = type[i];
}

int launch_pack(int n, const float3* crd, const float* charge, const int* type,
                const int* perm, float4* pos, int* type_sorted, cudaStream_t st,
                const float3* img_off) {
  if (n <= 0) return kOk;
  k_pack<<<ceil_div(n, 256), 256, 0, st>>>(n, crd, charge, type, perm, pos,
                                          type_sorted, img_off);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

// frc[i] += F[map[i]]; energies/virial likewise; accumulators zeroed after.
template <int ACCUM>
__global__ void k_unpack(int n, const int* __restrict__ map, Accumulators a,
                         float3* __restrict__ frc, float* atom_energy,
                         float* lj_energy, float* coul_energy, float* atom_virial,
                         bool energy, bool virial) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = map ? map[i] : i;
  const int N = a.n;
  float fx, fy, fz;
  if (ACCUM == kAccumFixed) {
    fx = (float)((double)a.d_f[s] * kForceScaleInv);
    fy = (float)((double)a.d_f[N + s] * kForceScaleInv);
    fz = (float)((double)a.d_f[2 * N + s] * kForceScaleInv);
    a.d_f[s] = 0;
    a.d_f[N + s] = 0;
    a.d_f[2 * N + s] = 0;
  } else {
    fx = a.d_ff[s];
    fy = a.d_ff[N + s];
    fz = a.d_ff[2 * N + s];
    a.d_ff[s] = 0.f;
    a.d_ff[N + s] = 0.f;
    a.d_ff[2 * N + s] = 0.f;
  }
  if (frc) {
    float3 f = frc[i];
    f.x += fx;
    f.y += fy;
    f.z += fz;
    frc[i] = f;
  }
  if (energy) {
    float e, elj, ec;
    if (ACCUM == kAccumFixed) {
      e = (float)((double)a.d_e[s] * kEnergyScaleInv);
      elj = (float)((double)a.d_elj[s] * kEnergyScaleInv);
      ec = (float)((double)a.d_ec[s] * kEnergyScaleInv);
      a.d_e[s] = 0;
      a.d_elj[s] = 0;
      a.d_ec[s] = 0;
    } else {
      e = a.d_fe[s];
      elj = a.d_fe[N + s];
      ec = a.d_fe[2 * N + s];
      a.d_fe[s] = 0.f;
      a.d_fe[N + s] = 0.f;
      a.d_fe[2 * N + s] = 0.f;
    }
    if (atom_energy) atom_energy[i] += e;
    if (lj_energy) lj_energy[i] += elj;
    if (coul_energy) coul_energy[i] += ec;
  }
  if (virial) {
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      float v;
      if (ACCUM == kAccumFixed) {
        v = (float)((double)a.d_v[c * N + s] * kEnergyScaleInv);
        a.d_v[c * N + s] = 0;
      } else {
        v = a.d_fv[c * N + s];
        a.d_fv[c * N + s] = 0.f;
      }
      if (atom_virial) atom_virial[6 * i + c] += v;
    }
  }
}

int launch_unpack(int n, const int* map, Accumulators& acc, int accum,
                  float3* frc, float* atom_energy, float* lj_energy,
                  float* coul_energy, float* atom_virial, bool energy,
                  bool virial, cudaStream_t st) {
  if (n <= 0) return kOk;
  if (accum == kAccumFixed)
    k_unpack<kAccumFixed><<<ceil_div(n, 256), 256, 0, st>>>(
        n, map, acc, frc, atom_energy, lj_energy, coul_energy, atom_virial,
        energy, virial);
  else
    k_unpack<kAccumFloat><<<ceil_div(n, 256), 256, 0, st>>>(
        n, map, acc, frc, atom_energy, lj_energy, coul_energy, atom_virial,
        energy, virial);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}

}  // namespace snb

// ---------------------------------------------------------------------------
// Self-check of the pair kernels' screened-Coulomb factors: erfc(x) and
// exp(-x^2) as erfc_and_exp forms them, beside CUDA's erfcf and expf.
__global__ void k_check_erfc(int n, const float* __restrict__ x, float* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = x[i];
  float e;
  const float c = snb::erfc_and_exp(v, &e);
  out[4 * i + 0] = c;
  out[4 * i + 1] = e;
  out[4 * i + 2] = erfcf(v);
  out[4 * i + 3] = expf(-v * v);
}

extern "C" int snb_check_erfc_exp(int n, const float* d_x, float* d_out, void* stream) {
  using namespace snb;
  if (n < 0 || (n > 0 && (!d_x || !d_out)))
    return fail(kBadInput, "check_erfc_exp: bad arguments");
  if (n == 0) return kOk;
  k_check_erfc<<<ceil_div(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      n, d_x, d_out);
  SNB_CUDA_TRY(cudaGetLastError());
  return kOk;
}
