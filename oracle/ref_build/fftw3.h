/* TEST INFRASTRUCTURE ONLY.  FFTW3 (single precision) API shim for compiling
 * the reference's own CPU sources without FFTW, which is not installed here.
 * Only the entry points SPONGE/utils/fft.hpp uses are provided; they are
 * backed by the oracle's double-precision mixed-radix FFT (fft_mixed.c).
 * FFTW itself is an un-vendored third-party dependency of the reference. */
#ifndef SNB_FFTW3_SHIM_H
#define SNB_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct snb_fftwf_plan_s* fftwf_plan;

#define FFTW_ESTIMATE (1U << 6)

void* fftwf_malloc(size_t n);
void fftwf_free(void* p);
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                   float* in, const int* inembed, int istride,
                                   int idist, fftwf_complex* out,
                                   const int* onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                   fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out,
                                   const int* onembed, int ostride, int odist,
                                   unsigned flags);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
#endif
