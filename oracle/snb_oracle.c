/* TEST INFRASTRUCTURE ONLY -- the oracle.
 *
 * CPU restatement of SPONGE's nonbonded hot path, used only by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker of the
 * CUDA kernels.  The product (sponge_b200/) never links, loads or calls it.
 *
 * Two precisions on purpose:
 *  - snbo_nl_pairs() evaluates the neighbor criterion exactly as the reference
 *    does, in FP32 with no FMA contraction (build flag -ffp-contract=off), so
 *    the pair set it returns is the bit-exact contract for the GPU list;
 *  - everything else is an FP64 run of the same method (same formulas, same
 *    weighting and per-atom assignment), the accuracy yardstick.
 *
 * Reference files restated (paths inside the SPONGE source tree):
 *   utils/boundary.h:22-32           minimum image
 *   utils/vector.hpp:249-346          LTMatrix3 products, virial from force/dis
 *   neighbor_list/neighbor_list.cpp:504-548,637-733,736-807,847   half list
 *   Lennard_Jones_force/Lennard_Jones_force.h:45-75, .cpp:45-137  pair terms
 *   Lennard_Jones_force/Lennard_Jones_force.cpp:212-235,279-308  tail corr.
 *   PM_force/PM_force.cpp:20-64,246-274,541-612,699-919,1024-1068,1142-1166,
 *                         1745-1817                              PME
 *   Lennard_Jones_force/LJ_soft_core.h:86-149, LJ_soft_core.cpp:196-461
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fft_mixed.h"

#define SNBO_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* FP32 minimum image exactly as boundary.h:31 evaluates it:
 *   dr - floorf(dr * rcell + 0.5f) * cell
 * with VECTOR*LTMatrix3 = {x*a11 + y*a21 + z*a31, y*a22 + z*a32, z*a33}. */
static void min_image_f32(const float* a, const float* b, const float* cell,
                          const float* rcell, float* out)
{
    float dx = a[0] - b[0];
    float dy = a[1] - b[1];
    float dz = a[2] - b[2];
    float sx = dx * rcell[0];
    sx = sx + dy * rcell[1];
    sx = sx + dz * rcell[3];
    float sy = dy * rcell[2];
    sy = sy + dz * rcell[4];
    float sz = dz * rcell[5];
    float fx = floorf(sx + 0.5f);
    float fy = floorf(sy + 0.5f);
    float fz = floorf(sz + 0.5f);
    float cx = fx * cell[0];
    cx = cx + fy * cell[1];
    cx = cx + fz * cell[3];
    float cy = fy * cell[2];
    cy = cy + fz * cell[4];
    float cz = fz * cell[5];
    out[0] = dx - cx;
    out[1] = dy - cy;
    out[2] = dz - cz;
}

/* Same formula in double for the FP64 method runs. */
static void min_image_f64(const float* a, const float* b, const float* cell,
                          const float* rcell, double* out)
{
    double dx = (double)a[0] - b[0], dy = (double)a[1] - b[1],
           dz = (double)a[2] - b[2];
    double sx = dx * rcell[0] + dy * rcell[1] + dz * rcell[3];
    double sy = dy * rcell[2] + dz * rcell[4];
    double sz = dz * rcell[5];
    double fx = floor(sx + 0.5), fy = floor(sy + 0.5), fz = floor(sz + 0.5);
    out[0] = dx - (fx * cell[0] + fy * cell[1] + fz * cell[3]);
    out[1] = dy - (fy * cell[2] + fz * cell[4]);
    out[2] = dz - fz * cell[5];
}

/* LTMatrix3 += sign * Get_Virial_From_Force_Dis(f, d)   (vector.hpp:322-334) */
static void virial_add(double* v, const double* f, const double* d, double s)
{
    v[0] += s * (f[0] * d[0]);
    v[1] += s * (f[0] * d[1] + f[1] * d[0]);
    v[2] += s * (f[1] * d[1]);
    v[3] += s * (f[0] * d[2] + f[2] * d[0]);
    v[4] += s * (f[1] * d[2] + f[2] * d[1]);
    v[5] += s * (f[2] * d[2]);
}

/* ------------------------------------------------------------------ */
/* Ewald beta by bisection, PM_force.cpp:246-274.  `precision` selects which
 * erfc the comparison uses: 0 = float erfcf, 1 = double erfc.  All the
 * iteration variables are float as in the reference. */
SNBO_API float snbo_get_beta(float cutoff, float tolerance, int precision)
{
    float beta, low, high, tempf;
    int ilow, ihigh;
    high = 1.0f;
    ihigh = 1;
    for (;;)
    {
        tempf = precision ? (float)(erfc((double)(high * cutoff)) / cutoff)
                          : erfcf(high * cutoff) / cutoff;
        if (tempf <= tolerance) break;
        high *= 2;
        ihigh++;
    }
    ihigh += 50;
    low = 0.0f;
    beta = 0.0f;
    for (ilow = 1; ilow < ihigh; ilow++)
    {
        beta = (low + high) / 2;
        tempf = precision ? (float)(erfc((double)(beta * cutoff)) / cutoff)
                          : erfcf(beta * cutoff) / cutoff;
        if (tempf >= tolerance)
            low = beta;
        else
            high = beta;
    }
    return beta;
}

/* ------------------------------------------------------------------ */
/* Excluded test with the reference's semantics for a single domain
 * (neighbor_list.cpp:744-773): pair (i, j), i < j, is removed when j appears
 * in the exclusion list of i. */
static int is_excluded(int i, int j, const int* excl_start,
                       const int* excl_numbers, const int* excl_list)
{
    if (!excl_numbers) return 0;
    int n = excl_numbers[i];
    if (n <= 0) return 0;
    const int* l = excl_list + excl_start[i];
    for (int k = 0; k < n; ++k)
        if (l[k] == j) return 1;
    return 0;
}

typedef struct
{
    int* j;
    int n, cap;
} jlist;

static void jl_push(jlist* l, int j)
{
    if (l->n == l->cap)
    {
        l->cap = l->cap ? 2 * l->cap : 64;
        l->j = (int*)realloc(l->j, sizeof(int) * (size_t)l->cap);
    }
    l->j[l->n++] = j;
}

static int cmp_int(const void* a, const void* b)
{
    int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* Half neighbor list: all pairs i < j with dr.dr < rl2 (FP32, no contraction),
 * dr = crd[i] - crd[j] minimum-imaged, exclusions removed.  rl2 is formed as
 * the reference forms it, (0.5f*(cutoff+skin))^2 * 4.0f (neighbor_list.cpp:847,
 * 1005).  Writes row offsets (n+1) and the j's of every row sorted ascending;
 * returns the number of pairs, or -(needed) if cap is too small. */
SNBO_API int64_t snbo_nl_pairs(int n, const float* crd, const float* cell,
                               const float* rcell, float cutoff, float skin,
                               const int* excl_start, const int* excl_numbers,
                               const int* excl_list, int64_t* row_start,
                               int* cols, int64_t cap)
{
    float grid_length = 0.5f * (cutoff + skin);
    float rl2 = grid_length * grid_length * 4.0f;
    jlist* rows = (jlist*)calloc((size_t)n, sizeof(jlist));
    int orth = cell[1] == 0.0f && cell[3] == 0.0f && cell[4] == 0.0f;
    float rl = sqrtf(rl2);
    int nc[3] = {0, 0, 0};
    if (orth)
    {
        nc[0] = (int)floor(cell[0] / (rl * 1.0001f));
        nc[1] = (int)floor(cell[2] / (rl * 1.0001f));
        nc[2] = (int)floor(cell[5] / (rl * 1.0001f));
    }
    if (orth && nc[0] >= 3 && nc[1] >= 3 && nc[2] >= 3)
    {
        int ncell = nc[0] * nc[1] * nc[2];
        int* head = (int*)malloc(sizeof(int) * (size_t)ncell);
        int* next = (int*)malloc(sizeof(int) * (size_t)n);
        int* cid = (int*)malloc(sizeof(int) * (size_t)n);
        for (int c = 0; c < ncell; ++c) head[c] = -1;
        double L[3] = {cell[0], cell[2], cell[5]};
        for (int i = n - 1; i >= 0; --i)
        {
            int c3[3];
            for (int d = 0; d < 3; ++d)
            {
                double x = crd[3 * i + d];
                x -= floor(x / L[d]) * L[d];
                int k = (int)(x / L[d] * nc[d]);
                if (k < 0) k = 0;
                if (k >= nc[d]) k = nc[d] - 1;
                c3[d] = k;
            }
            int c = (c3[0] * nc[1] + c3[1]) * nc[2] + c3[2];
            cid[i] = c;
            next[i] = head[c];
            head[c] = i;
        }
#pragma omp parallel for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i)
        {
            int c = cid[i];
            int cx = c / (nc[1] * nc[2]), cy = (c / nc[2]) % nc[1],
                cz = c % nc[2];
            for (int ox = -1; ox <= 1; ++ox)
                for (int oy = -1; oy <= 1; ++oy)
                    for (int oz = -1; oz <= 1; ++oz)
                    {
                        int x = (cx + ox + nc[0]) % nc[0];
                        int y = (cy + oy + nc[1]) % nc[1];
                        int z = (cz + oz + nc[2]) % nc[2];
                        for (int j = head[(x * nc[1] + y) * nc[2] + z]; j >= 0;
                             j = next[j])
                        {
                            if (j <= i) continue;
                            float dr[3];
                            min_image_f32(crd + 3 * i, crd + 3 * j, cell, rcell,
                                          dr);
                            float d2 = dr[0] * dr[0];
                            d2 = d2 + dr[1] * dr[1];
                            d2 = d2 + dr[2] * dr[2];
                            if (d2 < rl2 &&
                                !is_excluded(i, j, excl_start, excl_numbers,
                                             excl_list))
                                jl_push(&rows[i], j);
                        }
                    }
        }
        free(head);
        free(next);
        free(cid);
    }
    else
    {
#pragma omp parallel for schedule(dynamic, 16)
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j)
            {
                float dr[3];
                min_image_f32(crd + 3 * i, crd + 3 * j, cell, rcell, dr);
                float d2 = dr[0] * dr[0];
                d2 = d2 + dr[1] * dr[1];
                d2 = d2 + dr[2] * dr[2];
                if (d2 < rl2 &&
                    !is_excluded(i, j, excl_start, excl_numbers, excl_list))
                    jl_push(&rows[i], j);
            }
    }
    int64_t total = 0;
    for (int i = 0; i < n; ++i) total += rows[i].n;
    if (total > cap || !row_start || !cols)
    {
        for (int i = 0; i < n; ++i) free(rows[i].j);
        free(rows);
        return total > cap ? -total : total;
    }
    int64_t off = 0;
    for (int i = 0; i < n; ++i)
    {
        row_start[i] = off;
        if (rows[i].n) qsort(rows[i].j, (size_t)rows[i].n, sizeof(int), cmp_int);
        memcpy(cols + off, rows[i].j, sizeof(int) * (size_t)rows[i].n);
        off += rows[i].n;
        free(rows[i].j);
    }
    row_start[n] = off;
    free(rows);
    return total;
}

/* ------------------------------------------------------------------ */
/* Direct-space LJ + erfc-Coulomb over a half list, FP64 run of
 * Lennard_Jones_And_Direct_Coulomb_Device (Lennard_Jones_force.cpp:45-137):
 * for pair (i, j) of row i, dr = crd[j] - crd[i] (min image), r < cutoff:
 *   F/r  = (B' - A' r^-6) r^-8 - q_i q_j r^-3 (2 beta r/sqrt(pi) e^{-b^2r^2}
 *          + erfc(beta r))
 *   f_i += (F/r) dr, f_j -= (F/r) dr, virial_i -= (F/r) dr (x) dr,
 *   E_LJ,i += (A'/12 r^-6 - B'/6) r^-6,  E_C,i += q_i q_j erfc(beta r)/r.
 * Outputs are accumulated (+=) like the reference. */
SNBO_API void snbo_direct_f64(int n, const float* crd, const float* charge,
                              const int* lj_type, const float* lj_A,
                              const float* lj_B, const float* cell,
                              const float* rcell, float cutoff, float beta,
                              const int64_t* row_start, const int* cols,
                              double* frc, double* atom_energy,
                              double* lj_energy, double* coul_energy,
                              double* virial)
{
    const double two_over_sqrt_pi = 1.1283791670955126;
    double* fj = (double*)calloc((size_t)3 * n, sizeof(double));
    double b = beta;
#pragma omp parallel
    {
        double* fj_local = (double*)calloc((size_t)3 * n, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i)
        {
            double fi[3] = {0, 0, 0}, vir[6] = {0, 0, 0, 0, 0, 0};
            double elj = 0, ec = 0;
            int ti = lj_type[i];
            double qi = charge[i];
            for (int64_t k = row_start[i]; k < row_start[i + 1]; ++k)
            {
                int j = cols[k];
                double dr[3];
                min_image_f64(crd + 3 * j, crd + 3 * i, cell, rcell, dr);
                double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
                double r = sqrt(r2);
                if (!(r < cutoff)) continue;
                int tj = lj_type[j];
                int hi = ti > tj ? ti : tj, lo = ti > tj ? tj : ti;
                int pidx = hi * (hi + 1) / 2 + lo;
                double A = lj_A[pidx], B = lj_B[pidx];
                double ir2 = 1.0 / r2, ir6 = ir2 * ir2 * ir2;
                double flj = (B - A * ir6) * ir6 * ir2;
                double qq = qi * (double)charge[j];
                double br = b * r;
                double fc = qq / (r2 * r) *
                            (br * two_over_sqrt_pi * exp(-br * br) + erfc(br));
                double fabs_ = flj - fc;
                double fl[3] = {fabs_ * dr[0], fabs_ * dr[1], fabs_ * dr[2]};
                fi[0] += fl[0];
                fi[1] += fl[1];
                fi[2] += fl[2];
                fj_local[3 * j + 0] -= fl[0];
                fj_local[3 * j + 1] -= fl[1];
                fj_local[3 * j + 2] -= fl[2];
                virial_add(vir, fl, dr, -1.0);
                elj += (A / 12.0 * ir6 - B / 6.0) * ir6;
                ec += qq * erfc(br) / r;
            }
            frc[3 * i + 0] += fi[0];
            frc[3 * i + 1] += fi[1];
            frc[3 * i + 2] += fi[2];
            if (atom_energy) atom_energy[i] += elj + ec;
            if (lj_energy) lj_energy[i] += elj;
            if (coul_energy) coul_energy[i] += ec;
            if (virial)
                for (int c = 0; c < 6; ++c) virial[6 * i + c] += vir[c];
        }
#pragma omp critical
        for (int k = 0; k < 3 * n; ++k) fj[k] += fj_local[k];
        free(fj_local);
    }
    for (int k = 0; k < 3 * n; ++k) frc[k] += fj[k];
    free(fj);
}

/* ------------------------------------------------------------------ */
/* Soft-core LJ + direct Coulomb, FP64 run of
 * Lennard_Jones_And_Direct_Coulomb_Soft_Core_CUDA (LJ_soft_core.cpp:196-461)
 * with the pair forms of VECTOR_LJ_SOFT_TYPE (LJ_soft_core.h:33-149), single
 * process (ij_factor 1).  Pairs come from the half-list rows (i, j > i);
 * energies, the inter/intra split by mask and the virial go to i.  dudl[0]
 * and dudl[1] receive the LJ and direct-Coulomb dU/dlambda sums. */
static double sc_lj_e(double A, double B, double r)
{
    double r6 = pow(r, -6.0);
    return (A / 12.0 * r6 - B / 6.0) * r6;
}
static double sc_lj_f(double A, double B, double r)
{
    return (B - A * pow(r, -6.0)) * pow(r, -8.0);
}
static double sc_coul_e(double qq, double beta, double r)
{
    return qq * erfc(beta * r) / r;
}
static double sc_coul_f(double qq, double beta, double r)
{
    double br = beta * r;
    return qq * pow(r, -3.0) *
           (br * 1.1283791670955126 * exp(-br * br) + erfc(br));
}
static double sc_sigma6(double A, double B, double s6, double s6min)
{
    return (A == 0 || B == 0) ? s6 : fmax(0.5 * A / B, s6min);
}
static double sc_dudl(double F, double sigma6, double rs, double alpha,
                      double p, double lambda)
{
    const double flt_min = 1.17549435082228751e-38;
    return p * alpha * (1 - lambda) * pow(lambda + flt_min, p - 1.0) * F *
           pow(rs, -4.0) * sigma6 / 6.0;
}

SNBO_API void snbo_soft_f64(int n, const float* crd, const float* charge,
                            const float* charge_ba, const int* tA, const int* tB,
                            const int* mask, int nA, int nB, const float* AA_t,
                            const float* AB_t, const float* BA_t,
                            const float* BB_t, const float* cell,
                            const float* rcell, float cutoff, float beta,
                            float lambda_f, float alpha_f, float p_f,
                            float sigma6_f, float sigma6_min_f,
                            const int64_t* row_start, const int* cols,
                            double* frc, double* atom_energy, double* lj_energy,
                            double* inter, double* intra, double* coul_energy,
                            double* virial, double* dudl)
{
    const double lam = lambda_f, lam_ = 1.0 - lam, alpha = alpha_f, p = p_f;
    const double b = beta, s6 = sigma6_f, s6min = sigma6_min_f;
    const double alp_A = alpha * pow(lam, p), alp_B = alpha * pow(lam_, p);
    double* fj = (double*)calloc((size_t)3 * n, sizeof(double));
    double du_lj = 0, du_c = 0;
    (void)nA;
    (void)nB;
#pragma omp parallel reduction(+ : du_lj, du_c)
    {
        double* fj_local = (double*)calloc((size_t)3 * n, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int i = 0; i < n; ++i)
        {
            double fi[3] = {0, 0, 0}, vir[6] = {0, 0, 0, 0, 0, 0};
            double elj = 0, ec = 0, e_in = 0, e_out = 0;
            const double qi = charge[i], dqi = charge_ba ? charge_ba[i] : 0.0;
            for (int64_t k = row_start[i]; k < row_start[i + 1]; ++k)
            {
                int j = cols[k];
                double dr[3];
                min_image_f64(crd + 3 * j, crd + 3 * i, cell, rcell, dr);
                double r = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
                if (!(r < cutoff)) continue;
                int a1 = tA[i], a2 = tA[j], b1 = tB[i], b2 = tB[j];
                int pa = (a1 > a2 ? a1 * (a1 + 1) / 2 + a2 : a2 * (a2 + 1) / 2 + a1);
                int pb = (b1 > b2 ? b1 * (b1 + 1) / 2 + b2 : b2 * (b2 + 1) / 2 + b1);
                double AA = AA_t[pa], AB = AB_t[pa], BA = BA_t[pb], BB = BB_t[pb];
                double qq = qi * (double)charge[j];
                double dqj = charge_ba ? charge_ba[j] : 0.0;
                double qd = dqj * qi + (double)charge[j] * dqi;
                double fs, e_lj_pair, e_c_pair;
                if (BA * AA != 0 || BA + AA == 0)
                {
                    fs = lam_ * sc_lj_f(AA, AB, r) + lam * sc_lj_f(BA, BB, r) -
                         sc_coul_f(qq, b, r);
                    e_c_pair = sc_coul_e(qq, b, r);
                    e_lj_pair = lam_ * sc_lj_e(AA, AB, r) + lam * sc_lj_e(BA, BB, r);
                    du_lj += sc_lj_e(BA, BB, r) - sc_lj_e(AA, AB, r);
                    du_c += erfc(b * r) * qd / r;
                }
                else
                {
                    double sA = sc_sigma6(AA, AB, s6, s6min);
                    double sB = sc_sigma6(BA, BB, s6, s6min);
                    double r6 = pow(r, 6.0);
                    double rA = pow(r6 + alp_A * sA, 1.0 / 6.0);
                    double rB = pow(r6 + alp_B * sB, 1.0 / 6.0);
                    double r4 = pow(r, 4.0);
                    double flA = r4 * (AB - AA * pow(rA, -6.0)) * pow(rA, -12.0);
                    double flB = r4 * (BB - BA * pow(rB, -6.0)) * pow(rB, -12.0);
                    double bA = b * rA, bB = b * rB;
                    double fcA = qq * r4 *
                                 (exp(-bA * bA) * 1.1283791670955126 * b +
                                  erfc(bA) / rA) * pow(rA, -6.0);
                    double fcB = qq * r4 *
                                 (exp(-bB * bB) * 1.1283791670955126 * b +
                                  erfc(bB) / rB) * pow(rB, -6.0);
                    fs = lam_ * flA + lam * flB - (lam_ * fcA + lam * fcB);
                    e_c_pair = lam_ * sc_coul_e(qq, b, rA) + lam * sc_coul_e(qq, b, rB);
                    e_lj_pair = lam_ * sc_lj_e(AA, AB, rA) + lam * sc_lj_e(BA, BB, rB);
                    du_lj += sc_lj_e(BA, BB, rB) - sc_lj_e(AA, AB, rA);
                    du_lj += sc_dudl(sc_lj_f(AA, AB, rA), sA, rA, alpha, p, lam) -
                             sc_dudl(sc_lj_f(BA, BB, rB), sB, rB, alpha, p, lam_);
                    du_c += sc_coul_e(qq, b, rB) - sc_coul_e(qq, b, rA);
                    du_c += sc_dudl(sc_coul_f(qq, b, rB), sB, rB, alpha, p, lam_) -
                            sc_dudl(sc_coul_f(qq, b, rA), sA, rA, alpha, p, lam);
                    du_c += lam * erfc(b * rB) * qd / rB + lam_ * erfc(b * rA) * qd / rA;
                }
                double fl[3] = {fs * dr[0], fs * dr[1], fs * dr[2]};
                for (int c = 0; c < 3; ++c)
                {
                    fi[c] += fl[c];
                    fj_local[3 * j + c] -= fl[c];
                }
                virial_add(vir, fl, dr, -1.0);
                elj += e_lj_pair;
                ec += e_c_pair;
                if (mask[i] == mask[j])
                    e_in += e_lj_pair;
                else
                    e_out += e_lj_pair;
            }
            for (int c = 0; c < 3; ++c) frc[3 * i + c] += fi[c];
            if (atom_energy) atom_energy[i] += elj + ec;
            if (lj_energy) lj_energy[i] += elj;
            if (coul_energy) coul_energy[i] += ec;
            if (intra) intra[i] += e_in;
            if (inter) inter[i] += e_out;
            if (virial)
                for (int c = 0; c < 6; ++c) virial[6 * i + c] += vir[c];
        }
#pragma omp critical
        for (int k = 0; k < 3 * n; ++k) fj[k] += fj_local[k];
        free(fj_local);
    }
    for (int k = 0; k < 3 * n; ++k) frc[k] += fj[k];
    free(fj);
    if (dudl)
    {
        dudl[0] = du_lj;
        dudl[1] = du_c;
    }
}

/* Tail factors of LJ_SOFT_CORE::Initial (LJ_soft_core.cpp:640-672): the
 * lambda-mixed sum over all atom pairs of B' (Total_C6_Get) and the state
 * difference (Total_C6_B_A_Get), each times -2/3 pi / rc^3 / 6. */
SNBO_API void snbo_soft_lrc(int n, const int* tA, const int* tB, const float* AB,
                            const float* BB, float lambda, float cutoff,
                            double* factor, double* factor_ti)
{
    double s = 0, sti = 0;
    const double lam = lambda, lam_ = 1.0 - lam;
#pragma omp parallel for reduction(+ : s, sti)
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            int a1 = tA[i], a2 = tA[j], b1 = tB[i], b2 = tB[j];
            int pa = (a1 > a2 ? a1 * (a1 + 1) / 2 + a2 : a2 * (a2 + 1) / 2 + a1);
            int pb = (b1 > b2 ? b1 * (b1 + 1) / 2 + b2 : b2 * (b2 + 1) / 2 + b1);
            s += lam_ * AB[pa] + lam * BB[pb];
            sti += (double)BB[pb] - AB[pa];
        }
    const double k = -2.0 / 3.0 * 3.14159265358979323846 / cutoff / cutoff / cutoff / 6.0;
    *factor = s * k;
    *factor_ti = sti * k;
}

/* ------------------------------------------------------------------ */
/* Excluded-pair correction, FP64 run of
 * MPI_PME_Excluded_Force_With_Atom_Energy_Correction (PM_force.cpp:1745-1817)
 * with factor 1 (single process). */
SNBO_API void snbo_excluded_f64(int n, const float* crd, const float* charge,
                                const float* cell, const float* rcell,
                                float beta, const int* excl_start,
                                const int* excl_numbers, const int* excl_list,
                                double* frc, double* atom_energy,
                                double* virial)
{
    const double two_over_sqrt_pi = 1.1283791670955126;
    for (int i = 0; i < n; ++i)
    {
        int cnt = excl_numbers[i];
        if (cnt <= 0) continue;
        double qi = charge[i];
        double fi[3] = {0, 0, 0}, vir[6] = {0, 0, 0, 0, 0, 0}, e = 0;
        for (int k = excl_start[i]; k < excl_start[i] + cnt; ++k)
        {
            int j = excl_list[k];
            double dr[3];
            min_image_f64(crd + 3 * j, crd + 3 * i, cell, rcell, dr);
            double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
            double r = sqrt(r2);
            double br = (double)beta * r;
            double f = br * two_over_sqrt_pi * exp(-br * br) + erfc(br);
            f = (f - 1.0) / r2 / r;
            f = -qi * (double)charge[j] * f;
            double fl[3] = {f * dr[0], f * dr[1], f * dr[2]};
            frc[3 * j + 0] -= fl[0];
            frc[3 * j + 1] -= fl[1];
            frc[3 * j + 2] -= fl[2];
            fi[0] += fl[0];
            fi[1] += fl[1];
            fi[2] += fl[2];
            e -= qi * (double)charge[j] * erf(br) / r;
            virial_add(vir, fl, dr, -1.0);
        }
        frc[3 * i + 0] += fi[0];
        frc[3 * i + 1] += fi[1];
        frc[3 * i + 2] += fi[2];
        if (atom_energy) atom_energy[i] += e;
        if (virial)
            for (int c = 0; c < 6; ++c) virial[6 * i + c] += vir[c];
    }
}

/* ------------------------------------------------------------------ */
/* 1-4 terms, FP64 run of
 * Dihedral_14_LJ_CF_Force_With_Atom_Energy_And_Virial_Device
 * (nb14/nb14.cpp:8-103): for pair t, dr = r_b - r_a (minimum image),
 * F/r = -A r^-14 + B r^-8 - c q_a q_b r^-3 applied +F to a and -F to b;
 * energy (A/12 r^-12 - B/6 r^-6 + c q_a q_b / r, with the reference's
 * constants 0.08333333 and 0.1666666) and virial -(F (x) dr) to atom a;
 * a charge below 1e-10 in magnitude is taken as 1e-10 (nb14.cpp:4,55-58).
 * sums[0] = LJ, sums[1] = Coulomb (Step_Print, nb14.cpp:307-324). */
SNBO_API void snbo_nb14_f64(int m, const int* ia, const int* ib, const float* A,
                            const float* B, const float* cf, const float* crd,
                            const float* charge, const float* cell,
                            const float* rcell, double* frc, double* atom_energy,
                            double* virial, double* sums)
{
    for (int t = 0; t < m; ++t)
    {
        int a = ia[t], b = ib[t];
        double dr[3];
        min_image_f64(crd + 3 * b, crd + 3 * a, cell, rcell, dr);
        double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        double r = sqrt(r2);
        double ir2 = 1.0 / r2, ir = 1.0 / r;
        double ir4 = ir2 * ir2, ir8 = ir4 * ir4, ir14 = ir8 * ir4 * ir2;
        double qa = charge[a], qb = charge[b];
        if (fabs(qa) < 1e-10) qa = (double)1e-10f;
        if (fabs(qb) < 1e-10) qb = (double)1e-10f;
        double f = -(double)A[t] * ir14 + (double)B[t] * ir8 -
                   (double)cf[t] * ir2 * ir * qa * qb;
        double g[3] = {f * dr[0], f * dr[1], f * dr[2]};
        for (int c = 0; c < 3; ++c)
        {
            frc[3 * a + c] += g[c];
            frc[3 * b + c] -= g[c];
        }
        double ec = (double)cf[t] * ir * qa * qb;
        double el = (double)0.08333333f * A[t] * ir4 * ir8 -
                    (double)0.1666666f * B[t] * ir4 * ir2;
        if (atom_energy) atom_energy[a] += ec + el;
        if (sums)
        {
            sums[0] += el;
            sums[1] += ec;
        }
        if (virial) virial_add(virial + 6 * a, g, dr, -1.0);
    }
}

/* ------------------------------------------------------------------ */
/* Harmonic bonds (BOND, bond/bond.cpp:15-60) and angles (ANGLE,
 * angle/angle.cpp:6-80) in FP64.
 * Bond t of atoms (i, j): dr = r_i - r_j (minimum image), r = |dr|,
 *   E = k (r - r0)^2, f_i = -2 k (r - r0) / r dr, f_j = -f_i;
 *   energy and virial f_i (x) dr (off-diagonal pairs summed) on atom i.
 * Angle t of atoms (i, j, k), j the vertex: a = r_i - r_j, b = r_k - r_j,
 *   cos = a.b / (|a| |b|) clamped to [-0.999999, 0.999999], theta = acos,
 *   E = K (theta - theta0)^2, c = -2 K (theta - theta0) / sin(theta),
 *   f_i = c (cos a / |a|^2 - b / (|a||b|)), f_k = c (cos b / |b|^2 - a /
 *   (|a||b|)), f_j = -f_i - f_k; energy and virial f_i (x) a + f_k (x) b
 *   on atom i.
 * Each family's forces, per-atom energies and virials [n*6] are added to
 * its own arrays; sums[0..1] += the bond and the angle energy. */
SNBO_API void snbo_bonded_f64(int nb, const int* ba, const int* bb, const float* bk,
                              const float* br0, int na, const int* aa,
                              const int* ab, const int* ac, const float* ak,
                              const float* at0, const float* crd,
                              const float* cell, const float* rcell,
                              double* bond_frc, double* bond_energy,
                              double* bond_virial, double* angle_frc,
                              double* angle_energy, double* angle_virial,
                              double* sums)
{
    for (int t = 0; t < nb; ++t)
    {
        int i = ba[t], j = bb[t];
        double dr[3];
        min_image_f64(crd + 3 * i, crd + 3 * j, cell, rcell, dr);
        double r = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        double dev = r - (double)br0[t];
        double s = -2.0 * (double)bk[t] * dev / r;
        double f[3] = {s * dr[0], s * dr[1], s * dr[2]};
        for (int c = 0; c < 3; ++c)
        {
            bond_frc[3 * i + c] += f[c];
            bond_frc[3 * j + c] -= f[c];
        }
        double e = (double)bk[t] * dev * dev;
        bond_energy[i] += e;
        sums[0] += e;
        virial_add(bond_virial + 6 * i, f, dr, 1.0);
    }
    for (int t = 0; t < na; ++t)
    {
        int i = aa[t], j = ab[t], k = ac[t];
        double a[3], b[3];
        min_image_f64(crd + 3 * i, crd + 3 * j, cell, rcell, a);
        min_image_f64(crd + 3 * k, crd + 3 * j, cell, rcell, b);
        double ia2 = 1.0 / (a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        double ib2 = 1.0 / (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        double iab = sqrt(ia2 * ib2);
        double cs = (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) * iab;
        if (cs > 0.999999) cs = 0.999999;
        if (cs < -0.999999) cs = -0.999999;
        double th = acos(cs);
        double dth = th - (double)at0[t];
        double c = -2.0 * (double)ak[t] * dth / sin(th);
        double fi[3], fk[3];
        for (int d = 0; d < 3; ++d)
        {
            fi[d] = c * cs * ia2 * a[d] - c * iab * b[d];
            fk[d] = c * cs * ib2 * b[d] - c * iab * a[d];
            angle_frc[3 * i + d] += fi[d];
            angle_frc[3 * k + d] += fk[d];
            angle_frc[3 * j + d] -= fi[d] + fk[d];
        }
        double e = (double)ak[t] * dth * dth;
        angle_energy[i] += e;
        sums[1] += e;
        virial_add(angle_virial + 6 * i, fi, a, 1.0);
        virial_add(angle_virial + 6 * i, fk, b, 1.0);
    }
}

/* ------------------------------------------------------------------ */
/* Virtual atoms of types 0-3 in FP64 (virtual_atoms/virtual_atom_math.h,
 * virtual_atoms.h:8-105), record by record: positions in the given order,
 * then each virtual atom's force moved onto its sources in reverse order
 * and zeroed.  r_ij is the minimum-image r_i - r_j.
 *   0: x_v = x_1, y_v = y_1, z_v = 2h - z_1;   F_1 += (Fx, Fy, -Fz).
 *   1: r_v = r_1 + a r_21;                     F_1 += (1-a) F, F_2 += a F.
 *   2: r_v = r_1 + a r_21 + b r_31;            F_1 += (1-a-b) F, F_2 += a F,
 *                                              F_3 += b F.
 *   3: q = r_21 + k r_32, u = q/|q|, r_v = r_1 + d u; g = d/|q| (F - (F.u) u),
 *      F_1 += F - g, F_2 += (1-k) g, F_3 += k g; |d| <= 1e-6 puts the site
 *      on atom 1 with all its force; |q|^2 <= 1e-12 is an invalid geometry
 *      (site on atom 1, no force, and 1 + the record is returned).
 * crd [n*3] and frc [n*3] in double, updated in place. */
static void min_image_d(const double* a, const double* b, const float* cell,
                        const float* rcell, double* out);

SNBO_API int snbo_vatom_f64(int m, const int* type, const int* virt, const int* from,
                            const float* param, const float* cell,
                            const float* rcell, double* crd, double* frc)
{
    int bad = 0;
    for (int t = 0; t < m; ++t)
    {
        const int v = virt[t], a = from[3 * t], b = from[3 * t + 1], c = from[3 * t + 2];
        const double p = param[2 * t], q = param[2 * t + 1];
        double* xv = crd + 3 * v;
        const double* x1 = crd + 3 * a;
        if (type[t] == 0)
        {
            xv[0] = x1[0];
            xv[1] = x1[1];
            xv[2] = 2.0 * p - x1[2];
        }
        else if (type[t] == 1 || type[t] == 2)
        {
            double r21[3], r31[3] = {0.0, 0.0, 0.0};
            min_image_d(crd + 3 * b, x1, cell, rcell, r21);
            if (type[t] == 2) min_image_d(crd + 3 * c, x1, cell, rcell, r31);
            double o[3];
            for (int d = 0; d < 3; ++d) o[d] = x1[d] + p * r21[d] + q * r31[d];
            for (int d = 0; d < 3; ++d) xv[d] = o[d];
        }
        else
        {
            double r21[3], r32[3], w[3];
            min_image_d(crd + 3 * b, x1, cell, rcell, r21);
            min_image_d(crd + 3 * c, crd + 3 * b, cell, rcell, r32);
            for (int d = 0; d < 3; ++d) w[d] = r21[d] + q * r32[d];
            const double n2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
            double o[3] = {x1[0], x1[1], x1[2]};
            if (fabs(p) > 1e-6)
            {
                if (n2 <= 1e-12)
                {
                    if (!bad) bad = 1 + t;
                }
                else
                {
                    const double s = p / sqrt(n2);
                    for (int d = 0; d < 3; ++d) o[d] += s * w[d];
                }
            }
            for (int d = 0; d < 3; ++d) xv[d] = o[d];
        }
    }
    for (int t = m - 1; t >= 0; --t)
    {
        const int v = virt[t], a = from[3 * t], b = from[3 * t + 1], c = from[3 * t + 2];
        const double p = param[2 * t], q = param[2 * t + 1];
        double F[3] = {frc[3 * v], frc[3 * v + 1], frc[3 * v + 2]};
        if (type[t] == 0)
        {
            frc[3 * a] += F[0];
            frc[3 * a + 1] += F[1];
            frc[3 * a + 2] -= F[2];
        }
        else if (type[t] == 1 || type[t] == 2)
        {
            const double q2 = type[t] == 2 ? q : 0.0;
            for (int d = 0; d < 3; ++d)
            {
                frc[3 * a + d] += (1.0 - p - q2) * F[d];
                frc[3 * b + d] += p * F[d];
                if (type[t] == 2) frc[3 * c + d] += q2 * F[d];
            }
        }
        else if (fabs(p) <= 1e-6)
        {
            for (int d = 0; d < 3; ++d) frc[3 * a + d] += F[d];
        }
        else
        {
            double r21[3], r32[3], w[3];
            min_image_d(crd + 3 * b, crd + 3 * a, cell, rcell, r21);
            min_image_d(crd + 3 * c, crd + 3 * b, cell, rcell, r32);
            for (int d = 0; d < 3; ++d) w[d] = r21[d] + q * r32[d];
            const double n2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
            if (n2 <= 1e-12)
            {
                if (!bad) bad = 1 + t;
            }
            else
            {
                const double in = 1.0 / sqrt(n2);
                const double u[3] = {w[0] * in, w[1] * in, w[2] * in};
                const double fu = F[0] * u[0] + F[1] * u[1] + F[2] * u[2];
                for (int d = 0; d < 3; ++d)
                {
                    const double g = p * in * (F[d] - fu * u[d]);
                    frc[3 * a + d] += F[d] - g;
                    frc[3 * b + d] += (1.0 - q) * g;
                    frc[3 * c + d] += q * g;
                }
            }
        }
        frc[3 * v] = frc[3 * v + 1] = frc[3 * v + 2] = 0.0;
    }
    return bad;
}

/* ------------------------------------------------------------------ */
/* Rigid-geometry constraints in FP64 by iterated SHAKE (Ryckaert,
 * Ciccotti and Berendsen, J. Comput. Phys. 23, 327 (1977)): every listed
 * constraint (ai, aj, r0) moves its atoms along the bond vector at the
 * start of the step (from crd_old) until each length is r0 to `tol`
 * relative.  SETTLE (constrain/settle.cpp) solves the same equations
 * analytically, so for its rigid triangles and pairs the two agree.
 * crd / vel are updated in place: vel += v_factor / (dt x_factor) times
 * the position change.  virial[6] (LTMatrix3 order, off-diagonal pairs
 * summed) = sum over constraints of F (x) s_old with F = the total
 * multiplier times s_old / (dt^2 x_factor).  Returns the sweeps used, or
 * -1 without convergence in 10000 sweeps. */
static void min_image_d(const double* a, const double* b, const float* cell,
                        const float* rcell, double* out)
{
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    double sx = dx * rcell[0] + dy * rcell[1] + dz * rcell[3];
    double sy = dy * rcell[2] + dz * rcell[4];
    double sz = dz * rcell[5];
    double fx = floor(sx + 0.5), fy = floor(sy + 0.5), fz = floor(sz + 0.5);
    out[0] = dx - (fx * cell[0] + fy * cell[1] + fz * cell[3]);
    out[1] = dy - (fy * cell[2] + fz * cell[4]);
    out[2] = dz - fz * cell[5];
}

SNBO_API int snbo_shake_f64(int n, int m, const int* ai, const int* aj,
                            const double* r0, const double* mass,
                            const float* cell, const float* rcell,
                            const double* crd_old, double* crd, double* vel,
                            double dt, double v_factor, double x_factor,
                            double tol, double* virial)
{
    double* s = (double*)malloc(sizeof(double) * 3 * (m > 0 ? m : 1));
    double* g = (double*)calloc(m > 0 ? m : 1, sizeof(double));
    double* x0 = (double*)malloc(sizeof(double) * 3 * (n > 0 ? n : 1));
    memcpy(x0, crd, sizeof(double) * 3 * n);
    for (int k = 0; k < m; ++k)
        min_image_d(crd_old + 3 * aj[k], crd_old + 3 * ai[k], cell, rcell, s + 3 * k);
    int sweep = 0, done = 0;
    for (; sweep < 10000 && !done; ++sweep)
    {
        done = 1;
        for (int k = 0; k < m; ++k)
        {
            int i = ai[k], j = aj[k];
            double d[3];
            min_image_d(crd + 3 * j, crd + 3 * i, cell, rcell, d);
            double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            double t2 = r0[k] * r0[k];
            if (fabs(d2 - t2) > tol * t2) done = 0;
            double ds = d[0] * s[3 * k] + d[1] * s[3 * k + 1] + d[2] * s[3 * k + 2];
            double wi = 1.0 / mass[i], wj = 1.0 / mass[j];
            double gk = (t2 - d2) / (2.0 * ds * (wi + wj));
            for (int c = 0; c < 3; ++c)
            {
                crd[3 * i + c] -= gk * wi * s[3 * k + c];
                crd[3 * j + c] += gk * wj * s[3 * k + c];
            }
            g[k] += gk;
        }
    }
    for (int i = 0; i < 3 * n; ++i)
        vel[i] += v_factor / (dt * x_factor) * (crd[i] - x0[i]);
    for (int c = 0; c < 6; ++c) virial[c] = 0.0;
    for (int k = 0; k < m; ++k)
    {
        double f[3], c = g[k] / (dt * dt * x_factor);
        for (int q = 0; q < 3; ++q) f[q] = c * s[3 * k + q];
        virial_add(virial, f, s + 3 * k, 1.0);
    }
    free(s);
    free(g);
    free(x0);
    return done ? sweep : -1;
}

/* ------------------------------------------------------------------ */
/* PME reciprocal part in FP64 (PM_force.cpp:541-612 tables, 699-893 spread and
 * gather, 896-919 + 1142-1166 energies, 1024-1068 virial). */

/* |b(k)|^2 for order-4 B-splines: 1 / |sum_{j=0}^{2} M4(j+1) e^{2 pi i k j/K}|^2
 * (getb, PM_force.cpp:40-64). */
static double bspline_mod2(int k, int K)
{
    const double two_pi = 6.283185307179586476925286766559;
    const double m4[3] = {1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0};
    double re = 0, im = 0;
    for (int j = 0; j < 3; ++j)
    {
        double a = two_pi * k * j / K;
        re += m4[j] * cos(a);
        im += m4[j] * sin(a);
    }
    return 1.0 / (re * re + im * im);
}

/* order-4 cardinal B-spline weights of the four points u, u-1, u-2, u-3 and
 * their derivatives (power form of PME_Ma..PME_dMc, PM_force.cpp:20-26) */
static void bspline4(double x, double* w, double* dw)
{
    double x2 = x * x, x3 = x2 * x;
    w[0] = x3 / 6.0;
    w[1] = -0.5 * x3 + 0.5 * x2 + 0.5 * x + 1.0 / 6.0;
    w[2] = 0.5 * x3 - x2 + 4.0 / 6.0;
    w[3] = -x3 / 6.0 + 0.5 * x2 - 0.5 * x + 1.0 / 6.0;
    dw[0] = 0.5 * x2;
    dw[1] = -1.5 * x2 + x + 0.5;
    dw[2] = 1.5 * x2 - 2.0 * x;
    dw[3] = -0.5 * x2 + x - 0.5;
}

/* Fractional coordinate handling of PME_Atom_Near (PM_force.cpp:707-733):
 * frac = crd*rcell - floor(.), scaled by K, base u = (int) clamped, fraction. */
static void pme_base(const float* r, const float* rcell, const int* K,
                     int* u, double* fr)
{
    double f[3];
    f[0] = (double)r[0] * rcell[0] + (double)r[1] * rcell[1] +
           (double)r[2] * rcell[3];
    f[1] = (double)r[1] * rcell[2] + (double)r[2] * rcell[4];
    f[2] = (double)r[2] * rcell[5];
    for (int d = 0; d < 3; ++d)
    {
        f[d] -= floor(f[d]);
        if (!isfinite(f[d])) f[d] = 0.0;
        f[d] *= K[d];
        int t = (int)f[d];
        t = t < 0 ? 0 : (t < K[d] ? t : K[d] - 1);
        u[d] = t;
        double x = f[d] - t;
        fr[d] = x - floor(x);
    }
}

/* Outputs: frc += reciprocal force (times update_interval = 1), *e_recip,
 * *e_self (self + neutralising), virial6 (reference sign convention),
 * optional phi (the convolved grid, Nall doubles). */
SNBO_API void snbo_pme_f64(int n, const float* crd, const float* charge,
                           const float* cell, const float* rcell, int K0,
                           int K1, int K2, float beta, double* frc,
                           double* e_recip, double* e_self, double* virial6,
                           double* phi_out)
{
    const double pi = 3.141592653589793238462643383;
    int K[3] = {K0, K1, K2};
    size_t nall = (size_t)K0 * K1 * K2;
    int nc = K2 / 2 + 1;
    size_t nfft = (size_t)K0 * K1 * nc;
    double* Q = (double*)calloc(nall, sizeof(double));
    int* U = (int*)malloc(sizeof(int) * 3 * (size_t)n);
    double* FR = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    for (int a = 0; a < n; ++a)
    {
        pme_base(crd + 3 * a, rcell, K, U + 3 * a, FR + 3 * a);
        double wx[4], wy[4], wz[4], d[4];
        bspline4(FR[3 * a + 0], wx, d);
        bspline4(FR[3 * a + 1], wy, d);
        bspline4(FR[3 * a + 2], wz, d);
        double q = charge[a];
        for (int ix = 0; ix < 4; ++ix)
        {
            int gx = (U[3 * a] - ix + K0) % K0;
            for (int iy = 0; iy < 4; ++iy)
            {
                int gy = (U[3 * a + 1] - iy + K1) % K1;
                for (int iz = 0; iz < 4; ++iz)
                {
                    int gz = (U[3 * a + 2] - iz + K2) % K2;
                    Q[((size_t)gx * K1 + gy) * K2 + gz] +=
                        q * wx[ix] * wy[iy] * wz[iz];
                }
            }
        }
    }
    fftm_cplx* FQ = (fftm_cplx*)malloc(sizeof(fftm_cplx) * nfft);
    fftm_r2c_3d(Q, FQ, K0, K1, K2);
    /* tables and virial over the half spectrum */
    double vol = (double)cell[0] * cell[2] * cell[5];
    double b = beta;
    double mpre = pi * pi / (b * b);
    double vir[6] = {0, 0, 0, 0, 0, 0};
    double* B0 = (double*)malloc(sizeof(double) * K0);
    double* B1 = (double*)malloc(sizeof(double) * K1);
    double* B2 = (double*)malloc(sizeof(double) * K2);
    for (int k = 0; k < K0; ++k) B0[k] = bspline_mod2(k, K0);
    for (int k = 0; k < K1; ++k) B1[k] = bspline_mod2(k, K1);
    for (int k = 0; k < K2; ++k) B2[k] = bspline_mod2(k, K2);
    for (int kx = 0; kx < K0; ++kx)
    {
        double kxr = kx > K0 / 2 ? kx - K0 : kx;
        for (int ky = 0; ky < K1; ++ky)
        {
            double kyr = ky > K1 / 2 ? ky - K1 : ky;
            for (int kz = 0; kz < nc; ++kz)
            {
                double kzr = kz;
                /* m = MultiplyTranspose(k, rcell) (vector.hpp:286-291) */
                double m[3] = {kxr * rcell[0], kxr * rcell[1] + kyr * rcell[2],
                               kxr * rcell[3] + kyr * rcell[4] +
                                   kzr * rcell[5]};
                double msq = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
                size_t idx = ((size_t)kx * K1 + ky) * nc + kz;
                double bc = 0.0, vb[6] = {0, 0, 0, 0, 0, 0};
                if (kx + ky + kz != 0)
                {
                    bc = 1.0 / pi / msq * exp(-mpre * msq) / vol;
                    double c = 2.0 / msq * (1.0 + mpre * msq);
                    vb[0] = 1.0 - c * m[0] * m[0];
                    vb[1] = 0.0 - c * m[1] * m[0];
                    vb[2] = 1.0 - c * m[1] * m[1];
                    vb[3] = 0.0 - c * m[2] * m[0];
                    vb[4] = 0.0 - c * m[2] * m[1];
                    vb[5] = 1.0 - c * m[2] * m[2];
                }
                bc *= B0[kx] * B1[ky] * B2[kz];
                double f2 = FQ[idx].re * FQ[idx].re + FQ[idx].im * FQ[idx].im;
                double factor = (kz == 0 || kz == nc - 1) ? 0.5 : 1.0;
                for (int c = 0; c < 6; ++c)
                    vir[c] -= factor * f2 * (0.5 * bc * vb[c]);
                FQ[idx].re *= bc;
                FQ[idx].im *= bc;
            }
        }
    }
    double* phi = (double*)malloc(sizeof(double) * nall);
    fftm_c2r_3d(FQ, phi, K0, K1, K2);
    double er = 0.0;
    for (size_t g = 0; g < nall; ++g) er += Q[g] * phi[g];
    *e_recip = 0.5 * er;
    double q2 = 0, qs = 0;
    for (int a = 0; a < n; ++a)
    {
        q2 += (double)charge[a] * charge[a];
        qs += charge[a];
    }
    *e_self = -b / sqrt(pi) * q2 - 0.5 * pi / (b * b * vol) * qs * qs;
    for (int c = 0; c < 6; ++c) virial6[c] += vir[c];
    /* gather (PME_Final, PM_force.cpp:829-893) */
#pragma omp parallel for
    for (int a = 0; a < n; ++a)
    {
        double wx[4], wy[4], wz[4], dx[4], dy[4], dz[4];
        bspline4(FR[3 * a + 0], wx, dx);
        bspline4(FR[3 * a + 1], wy, dy);
        bspline4(FR[3 * a + 2], wz, dz);
        double q = charge[a];
        double acc[3] = {0, 0, 0};
        for (int ix = 0; ix < 4; ++ix)
        {
            int gx = (U[3 * a] - ix + K0) % K0;
            for (int iy = 0; iy < 4; ++iy)
            {
                int gy = (U[3 * a + 1] - iy + K1) % K1;
                for (int iz = 0; iz < 4; ++iz)
                {
                    int gz = (U[3 * a + 2] - iz + K2) % K2;
                    double p = -phi[((size_t)gx * K1 + gy) * K2 + gz] * q;
                    double g0 = dx[ix] * wy[iy] * wz[iz] * K0;
                    double g1 = dy[iy] * wx[ix] * wz[iz] * K1;
                    double g2 = dz[iz] * wx[ix] * wy[iy] * K2;
                    acc[0] += p * (g0 * rcell[0]);
                    acc[1] += p * (g0 * rcell[1] + g1 * rcell[2]);
                    acc[2] += p * (g0 * rcell[3] + g1 * rcell[4] + g2 * rcell[5]);
                }
            }
        }
        frc[3 * a + 0] += acc[0];
        frc[3 * a + 1] += acc[1];
        frc[3 * a + 2] += acc[2];
    }
    if (phi_out) memcpy(phi_out, phi, sizeof(double) * nall);
    free(Q);
    free(U);
    free(FR);
    free(FQ);
    free(phi);
    free(B0);
    free(B1);
    free(B2);
}

/* Plain Ewald reciprocal sum (no mesh) in FP64 for small systems: the exact
 * quantity PME approximates, used to check the oracle's own PME. */
SNBO_API double snbo_ewald_recip_f64(int n, const float* crd,
                                     const float* charge, float box, float beta,
                                     int kmax, double* frc)
{
    const double pi = 3.141592653589793238462643383;
    double L = box, vol = L * L * L, e = 0.0;
    for (int kx = -kmax; kx <= kmax; ++kx)
        for (int ky = -kmax; ky <= kmax; ++ky)
            for (int kz = -kmax; kz <= kmax; ++kz)
            {
                if (!kx && !ky && !kz) continue;
                double m[3] = {kx / L, ky / L, kz / L};
                double m2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
                double pre = exp(-pi * pi * m2 / ((double)beta * beta)) / m2;
                double sr = 0, si = 0;
                for (int a = 0; a < n; ++a)
                {
                    double ph = 2 * pi *
                                (m[0] * crd[3 * a] + m[1] * crd[3 * a + 1] +
                                 m[2] * crd[3 * a + 2]);
                    sr += charge[a] * cos(ph);
                    si += charge[a] * sin(ph);
                }
                e += pre * (sr * sr + si * si);
                if (frc)
                    for (int a = 0; a < n; ++a)
                    {
                        double ph = 2 * pi *
                                    (m[0] * crd[3 * a] + m[1] * crd[3 * a + 1] +
                                     m[2] * crd[3 * a + 2]);
                        double s = sin(ph) * sr - cos(ph) * si;
                        double f = 2.0 / vol * pre * charge[a] * s;
                        frc[3 * a + 0] += f * m[0];
                        frc[3 * a + 1] += f * m[1];
                        frc[3 * a + 2] += f * m[2];
                    }
            }
    return e / (2 * pi * vol);
}

/* ------------------------------------------------------------------ */
/* Long-range LJ correction factor as the reference forms it
 * (Lennard_Jones_force.cpp:212-235): type histogram, double C6 sum, then
 * float scaling by -2/3 pi / rc^3 / 6.  E_lrc = factor/V, W_lrc = 2 factor/V
 * on the diagonal (:279-306). */
SNBO_API float snbo_lrc_factor(int n, const int* lj_type, int n_types,
                               const float* lj_B, float cutoff)
{
    int64_t* cnt = (int64_t*)calloc((size_t)n_types, sizeof(int64_t));
    for (int i = 0; i < n; ++i) cnt[lj_type[i]] += 1;
    double c6 = 0.0;
    for (int a = 0; a < n_types; ++a)
    {
        if (!cnt[a]) continue;
        double inner = 0.0;
        for (int b = 0; b < n_types; ++b)
        {
            if (!cnt[b]) continue;
            int hi = a > b ? a : b, lo = a > b ? b : a;
            inner += (double)cnt[b] * (double)lj_B[hi * (hi + 1) / 2 + lo];
        }
        c6 += (double)cnt[a] * inner;
    }
    free(cnt);
    float f = (float)c6;
    f *= -2.0f / 3.0f * 3.1415926535897932f / cutoff / cutoff / cutoff / 6.0f;
    return f;
}
