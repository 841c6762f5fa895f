/* TEST INFRASTRUCTURE ONLY.  Part of the oracle: never linked into the product.
 *
 * Double-precision mixed-radix complex FFT (recursive Cooley-Tukey over the
 * smallest prime factor, O(n * sum of factors)), used by the FP64 oracle for
 * the PME convolution and by the FFTW-compatible shim that lets the reference's
 * own PM_force.cpp run on CPU (FFTW itself is not installed here).
 * Sign convention: forward = exp(-2*pi*i*k*n/N), inverse unnormalised, the
 * same as FFTW and cuFFT.
 */
#ifndef SNB_ORACLE_FFT_MIXED_H
#define SNB_ORACLE_FFT_MIXED_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } fftm_cplx;

/* In-place 3-D complex transform of a row-major [n0][n1][n2] array.
 * sign = -1 forward, +1 inverse (unnormalised). */
void fftm_3d(fftm_cplx* data, int n0, int n1, int n2, int sign);

/* Real -> half spectrum [n0][n1][n2/2+1], and back (unnormalised). */
void fftm_r2c_3d(const double* in, fftm_cplx* out, int n0, int n1, int n2);
void fftm_c2r_3d(const fftm_cplx* in, double* out, int n0, int n1, int n2);

#ifdef __cplusplus
}
#endif
#endif
