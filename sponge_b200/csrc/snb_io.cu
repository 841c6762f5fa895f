// SPONGE's native text inputs of this path and its force trajectory output,
// on the host: the LJ and soft-core LJ tables (Xponge::Native_Load_LJ,
// xponge/load/native/lj.hpp:9-67; Native_Load_LJ_Soft_Core, lj_soft.hpp),
// the subsystem division, the exclusion lists, charges and masses
// (xponge/load/native/md_core.hpp), the 1-4 pair list
// (Xponge::Native_Load_NB14, xponge/load/native/nb14.hpp:8-101), and the
// binary frc trajectory
// (MD_core/output.hpp:1691-1700).
//
// Each reader reads the file's counts first.  Called with NULL arrays it
// returns only the counts, so a caller can size its buffers and call again.
// Values are read with the same conversions as the reference (fscanf "%f"
// and "%d"; A' = 12 A and B' = 6 B as the tables are stored).
#include <cstdio>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "snb_internal.h"

namespace snb {
namespace {

struct File {
  FILE* fp = nullptr;
  explicit File(const char* path) : fp(path ? fopen(path, "r") : nullptr) {}
  ~File() {
    if (fp) fclose(fp);
  }
};

int bad_format(const char* what) {
  return fail(kBadInput, std::string("the format of ") + what + " is not right");
}

int no_file(const char* what, const char* path) {
  return fail(kBadInput, std::string("cannot open ") + what + " '" + (path ? path : "") + "'");
}

// n floats into out (or skipped when out is NULL), each times scale
bool read_floats(FILE* fp, int n, float* out, float scale) {
  for (int i = 0; i < n; ++i) {
    float v;
    if (fscanf(fp, "%f", &v) != 1) return false;
    if (out) out[i] = v * scale;
  }
  return true;
}

bool read_ints(FILE* fp, int n, int* out) {
  for (int i = 0; i < n; ++i) {
    int v;
    if (fscanf(fp, "%d", &v) != 1) return false;
    if (out) out[i] = v;
  }
  return true;
}

}  // namespace
}  // namespace snb

using namespace snb;

extern "C" int snb_read_lj_in_file(const char* path, int* atom_numbers,
                                   int* atom_type_numbers, float* h_LJ_A, float* h_LJ_B,
                                   int* h_atom_LJ_type) {
  const char* what = "LJ_in_file";
  if (!atom_numbers || !atom_type_numbers) return fail(kBadInput, "read_lj_in_file: null count");
  File f(path);
  if (!f.fp) return no_file(what, path);
  int n = 0, t = 0;
  if (fscanf(f.fp, "%d %d", &n, &t) != 2 || n < 0 || t <= 0) return bad_format(what);
  *atom_numbers = n;
  *atom_type_numbers = t;
  if (!h_LJ_A && !h_LJ_B && !h_atom_LJ_type) return kOk;
  if (!h_LJ_A || !h_LJ_B || !h_atom_LJ_type)
    return fail(kBadInput, "read_lj_in_file: give all three arrays or none");
  const int pairs = t * (t + 1) / 2;
  if (!read_floats(f.fp, pairs, h_LJ_A, 12.0f) || !read_floats(f.fp, pairs, h_LJ_B, 6.0f) ||
      !read_ints(f.fp, n, h_atom_LJ_type))
    return bad_format(what);
  return kOk;
}

extern "C" int snb_read_lj_soft_core_in_file(const char* path, int* atom_numbers,
                                             int* atom_type_numbers_A,
                                             int* atom_type_numbers_B, float* h_LJ_AA,
                                             float* h_LJ_AB, float* h_LJ_BA, float* h_LJ_BB,
                                             int* h_LJ_type_A, int* h_LJ_type_B) {
  const char* what = "LJ_soft_core_in_file";
  if (!atom_numbers || !atom_type_numbers_A || !atom_type_numbers_B)
    return fail(kBadInput, "read_lj_soft_core_in_file: null count");
  File f(path);
  if (!f.fp) return no_file(what, path);
  int n = 0, ta = 0, tb = 0;
  if (fscanf(f.fp, "%d %d %d", &n, &ta, &tb) != 3 || n < 0 || ta <= 0 || tb <= 0)
    return bad_format(what);
  *atom_numbers = n;
  *atom_type_numbers_A = ta;
  *atom_type_numbers_B = tb;
  const bool any = h_LJ_AA || h_LJ_AB || h_LJ_BA || h_LJ_BB || h_LJ_type_A || h_LJ_type_B;
  if (!any) return kOk;
  if (!h_LJ_AA || !h_LJ_AB || !h_LJ_BA || !h_LJ_BB || !h_LJ_type_A || !h_LJ_type_B)
    return fail(kBadInput, "read_lj_soft_core_in_file: give all six arrays or none");
  const int pa = ta * (ta + 1) / 2, pb = tb * (tb + 1) / 2;
  if (!read_floats(f.fp, pa, h_LJ_AA, 12.0f) || !read_floats(f.fp, pa, h_LJ_AB, 6.0f) ||
      !read_floats(f.fp, pb, h_LJ_BA, 12.0f) || !read_floats(f.fp, pb, h_LJ_BB, 6.0f))
    return bad_format(what);
  for (int i = 0; i < n; ++i)
    if (fscanf(f.fp, "%d %d", h_LJ_type_A + i, h_LJ_type_B + i) != 2) return bad_format(what);
  return kOk;
}

// One count then one value per atom: subsys_division_in_file (int),
// charge_in_file and mass_in_file (float).
static int read_per_atom(const char* path, const char* what, int* atom_numbers, float* fv,
                         int* iv) {
  if (!atom_numbers) return fail(kBadInput, std::string("read ") + what + ": null count");
  File f(path);
  if (!f.fp) return no_file(what, path);
  int n = 0;
  if (fscanf(f.fp, "%d", &n) != 1 || n < 0) return bad_format(what);
  *atom_numbers = n;
  if (fv && !read_floats(f.fp, n, fv, 1.0f)) return bad_format(what);
  if (iv && !read_ints(f.fp, n, iv)) return bad_format(what);
  return kOk;
}

extern "C" int snb_read_subsys_division_in_file(const char* path, int* atom_numbers,
                                                int* h_subsys_division) {
  return read_per_atom(path, "subsys_division_in_file", atom_numbers, nullptr,
                       h_subsys_division);
}

extern "C" int snb_read_charge_in_file(const char* path, int* atom_numbers, float* h_charge) {
  return read_per_atom(path, "charge_in_file", atom_numbers, h_charge, nullptr);
}

extern "C" int snb_read_mass_in_file(const char* path, int* atom_numbers, float* h_mass) {
  return read_per_atom(path, "mass_in_file", atom_numbers, h_mass, nullptr);
}

extern "C" int snb_read_exclude_in_file(const char* path, int* atom_numbers,
                                        int* excluded_atom_numbers, int* h_excluded_list_start,
                                        int* h_excluded_numbers, int* h_excluded_list) {
  const char* what = "exclude_in_file";
  if (!atom_numbers || !excluded_atom_numbers)
    return fail(kBadInput, "read_exclude_in_file: null count");
  File f(path);
  if (!f.fp) return no_file(what, path);
  int n = 0, m = 0;
  if (fscanf(f.fp, "%d %d", &n, &m) != 2 || n < 0 || m < 0) return bad_format(what);
  *atom_numbers = n;
  *excluded_atom_numbers = m;
  const bool any = h_excluded_list_start || h_excluded_numbers || h_excluded_list;
  if (!any) return kOk;
  if (!h_excluded_list_start || !h_excluded_numbers || !h_excluded_list)
    return fail(kBadInput, "read_exclude_in_file: give all three arrays or none");
  int count = 0;
  for (int i = 0; i < n; ++i) {
    int k = 0;
    if (fscanf(f.fp, "%d", &k) != 1 || k < 0) return bad_format(what);
    h_excluded_list_start[i] = count;
    h_excluded_numbers[i] = k;
    for (int j = 0; j < k; ++j) {
      int v;
      if (fscanf(f.fp, "%d", &v) != 1) return bad_format(what);
      if (count >= m)
        return fail(kBadInput, "the format of exclude_in_file is not right "
                               "(excluded_atom_numbers is not right)");
      h_excluded_list[count++] = v;
    }
  }
  if (count != m)
    return fail(kBadInput, "the format of exclude_in_file is not right "
                           "(excluded_atom_numbers is not right)");
  return kOk;
}

extern "C" int snb_read_nb14_in_file(const char* path, const char* extra_path,
                                     int atom_numbers, const int* h_atom_LJ_type,
                                     const float* h_LJ_A, const float* h_LJ_B,
                                     int* nb14_numbers, int* h_atom_a, int* h_atom_b,
                                     float* h_A, float* h_B, float* h_cf_scale_factor) {
  if (!nb14_numbers) return fail(kBadInput, "read_nb14_in_file: null count");
  File f(path), fx(extra_path);
  if (path && !f.fp) return no_file("nb14_in_file", path);
  if (extra_path && !fx.fp) return no_file("nb14_extra_in_file", extra_path);
  int n = 0, nx = 0;
  if (f.fp && fscanf(f.fp, "%d", &n) != 1) return bad_format("nb14_in_file");
  if (fx.fp && fscanf(fx.fp, "%d", &nx) != 1) return bad_format("nb14_extra_in_file");
  if (n < 0) return bad_format("nb14_in_file");
  if (nx < 0) return bad_format("nb14_extra_in_file");
  *nb14_numbers = n + nx;
  const bool any = h_atom_a || h_atom_b || h_A || h_B || h_cf_scale_factor;
  if (!any) return kOk;
  if (!h_atom_a || !h_atom_b || !h_A || !h_B || !h_cf_scale_factor)
    return fail(kBadInput, "read_nb14_in_file: give all five arrays or none");
  if (n > 0 && (!h_atom_LJ_type || !h_LJ_A || !h_LJ_B))
    return fail(kBadInput, "'nb14_in_file' should be provided with initialized LJ parameters");
  auto in_range = [&](int a) { return a >= 0 && a < atom_numbers; };
  // the extra file's rows come first, with their own A, B (times 12 and 6)
  for (int i = 0; i < nx; ++i) {
    if (fscanf(fx.fp, "%d %d %f %f %f", &h_atom_a[i], &h_atom_b[i], &h_A[i], &h_B[i],
               &h_cf_scale_factor[i]) != 5)
      return bad_format("nb14_extra_in_file");
    if (!in_range(h_atom_a[i]) || !in_range(h_atom_b[i]))
      return fail(kBadInput, "nb14_extra_in_file: atom index out of range");
    h_A[i] *= 12.0f;
    h_B[i] *= 6.0f;
  }
  for (int i = nx; i < nx + n; ++i) {
    float lj_scale = 0.0f;
    if (fscanf(f.fp, "%d %d %f %f", &h_atom_a[i], &h_atom_b[i], &lj_scale,
               &h_cf_scale_factor[i]) != 4)
      return bad_format("nb14_in_file");
    if (!in_range(h_atom_a[i]) || !in_range(h_atom_b[i]))
      return fail(kBadInput, "nb14_in_file: atom index out of range");
    int lo = h_atom_LJ_type[h_atom_a[i]], hi = h_atom_LJ_type[h_atom_b[i]];
    if (lo > hi) std::swap(lo, hi);
    const int pair = hi * (hi + 1) / 2 + lo;
    h_A[i] = lj_scale * h_LJ_A[pair];
    h_B[i] = lj_scale * h_LJ_B[pair];
  }
  return kOk;
}

extern "C" int snb_append_frc_traj(const char* path, const float* d_frc, int atom_numbers,
                                   void* stream) {
  if (!path || !d_frc || atom_numbers <= 0) return fail(kBadInput, "append_frc_traj: bad argument");
  std::vector<float> h(3 * (size_t)atom_numbers);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  SNB_CUDA_TRY(cudaMemcpyAsync(h.data(), d_frc, sizeof(float) * h.size(),
                               cudaMemcpyDeviceToHost, st));
  SNB_CUDA_TRY(cudaStreamSynchronize(st));
  FILE* fp = fopen(path, "ab");
  if (!fp) return no_file("frc trajectory", path);
  const size_t w = fwrite(h.data(), sizeof(float) * 3, atom_numbers, fp);
  fclose(fp);
  if (w != (size_t)atom_numbers) return fail(kBadInput, "append_frc_traj: short write");
  return kOk;
}

// Xponge::Native_Load_Bonds (xponge/load/native/bond.hpp:9-42): "M", then M
// rows "a b k r0" (fscanf "%d %d %f %f").
extern "C" int snb_read_bond_in_file(const char* path, int* bond_numbers, int* h_atom_a,
                                     int* h_atom_b, float* h_k, float* h_r0) {
  using namespace snb;
  const char* what = "bond_in_file";
  if (!bond_numbers) return fail(kBadInput, "read_bond_in_file: null count");
  File f(path);
  if (!f.fp) return no_file(what, path);
  int m = 0;
  if (fscanf(f.fp, "%d", &m) != 1 || m < 0) return bad_format(what);
  *bond_numbers = m;
  const bool any = h_atom_a || h_atom_b || h_k || h_r0;
  if (!any) return kOk;
  if (!h_atom_a || !h_atom_b || !h_k || !h_r0)
    return fail(kBadInput, "read_bond_in_file: give all four arrays or none");
  for (int i = 0; i < m; ++i)
    if (fscanf(f.fp, "%d %d %f %f", &h_atom_a[i], &h_atom_b[i], &h_k[i], &h_r0[i]) != 4)
      return bad_format(what);
  return kOk;
}

// Xponge::Native_Load_Angles (xponge/load/native/angle.hpp:8-44): "M", then
// M rows "a b c k theta0" (fscanf "%d %d %d %f %f", theta0 in radians).
extern "C" int snb_read_angle_in_file(const char* path, int* angle_numbers, int* h_atom_a,
                                      int* h_atom_b, int* h_atom_c, float* h_k,
                                      float* h_theta0) {
  using namespace snb;
  const char* what = "angle_in_file";
  if (!angle_numbers) return fail(kBadInput, "read_angle_in_file: null count");
  File f(path);
  if (!f.fp) return no_file(what, path);
  int m = 0;
  if (fscanf(f.fp, "%d", &m) != 1 || m < 0) return bad_format(what);
  *angle_numbers = m;
  const bool any = h_atom_a || h_atom_b || h_atom_c || h_k || h_theta0;
  if (!any) return kOk;
  if (!h_atom_a || !h_atom_b || !h_atom_c || !h_k || !h_theta0)
    return fail(kBadInput, "read_angle_in_file: give all five arrays or none");
  for (int i = 0; i < m; ++i)
    if (fscanf(f.fp, "%d %d %d %f %f", &h_atom_a[i], &h_atom_b[i], &h_atom_c[i], &h_k[i],
               &h_theta0[i]) != 5)
      return bad_format(what);
  return kOk;
}

// Xponge::Native_Load_Virtual_Atoms (xponge/load/native/virtual_atoms.hpp:
// 10-120): one record per line, "type virtual_atom" then the type's fields
// (0: from h; 1: from1 from2 a; 2 and 3: from1 from2 from3 a b); lines
// without the two leading integers are skipped, an unknown type or missing
// fields are format errors, and trailing fields must start with '#'.
// Records come back in file order: from [3m] (unused slots -1) and
// parameter [2m] (unused 0).
extern "C" int snb_read_virtual_atom_in_file(const char* path, int* record_numbers,
                                             int* h_type, int* h_virtual_atom, int* h_from,
                                             float* h_parameter) {
  using namespace snb;
  const char* what = "virtual_atom_in_file";
  if (!record_numbers) return fail(kBadInput, "read_virtual_atom_in_file: null count");
  const bool any = h_type || h_virtual_atom || h_from || h_parameter;
  if (any && (!h_type || !h_virtual_atom || !h_from || !h_parameter))
    return fail(kBadInput, "read_virtual_atom_in_file: give all four arrays or none");
  File f(path);
  if (!f.fp) return no_file(what, path);
  char line[4096];
  int m = 0, line_no = 0;
  while (fgets(line, sizeof(line), f.fp)) {
    ++line_no;
    std::istringstream in(line);
    int type = -1, v = -1;
    if (!(in >> type >> v)) continue;
    int src[3] = {-1, -1, -1};
    float par[2] = {0.f, 0.f};
    bool ok = false;
    if (type == 0) {
      ok = static_cast<bool>(in >> src[0] >> par[0]);
    } else if (type == 1) {
      ok = static_cast<bool>(in >> src[0] >> src[1] >> par[0]);
    } else if (type == 2 || type == 3) {
      ok = static_cast<bool>(in >> src[0] >> src[1] >> src[2] >> par[0] >> par[1]);
    } else {
      return fail(kBadInput, "virtual_atom_in_file contains an unsupported virtual atom type");
    }
    if (!ok) return bad_format(what);
    std::string trailing;
    if (in >> trailing && (trailing.empty() || trailing[0] != '#'))
      return fail(kBadInput, "virtual_atom_in_file line " + std::to_string(line_no) +
                                 " contains unexpected trailing fields");
    if (any) {
      h_type[m] = type;
      h_virtual_atom[m] = v;
      for (int k = 0; k < 3; ++k) h_from[3 * m + k] = src[k];
      for (int k = 0; k < 2; ++k) h_parameter[2 * m + k] = par[k];
    }
    ++m;
  }
  *record_numbers = m;
  return kOk;
}
