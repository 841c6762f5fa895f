/* TEST INFRASTRUCTURE ONLY.  FFTW3 single-precision entry points used by the
 * reference's utils/fft.hpp, implemented over the oracle's double-precision
 * mixed-radix FFT.  Supports what PM_force.cpp plans: contiguous rank-3
 * real<->half-complex transforms, any batch count (`howmany`) with the
 * default dense distances. */
#include <stdlib.h>
#include <string.h>

#include "../fft_mixed.h"
#include "fftw3.h"

struct snb_fftwf_plan_s
{
    int rank, n[3], howmany, r2c;
};

void* fftwf_malloc(size_t n) { return malloc(n ? n : 1); }
void fftwf_free(void* p) { free(p); }

static fftwf_plan make(int rank, const int* n, int howmany, int r2c)
{
    if (rank < 1 || rank > 3) return NULL;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->rank = 3;
    p->n[0] = p->n[1] = p->n[2] = 1;
    for (int i = 0; i < rank; ++i) p->n[3 - rank + i] = n[i];
    p->howmany = howmany;
    p->r2c = r2c;
    return p;
}

fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany,
                                   float* in, const int* inembed, int istride,
                                   int idist, fftwf_complex* out,
                                   const int* onembed, int ostride, int odist,
                                   unsigned flags)
{
    (void)in; (void)inembed; (void)istride; (void)idist; (void)out;
    (void)onembed; (void)ostride; (void)odist; (void)flags;
    return make(rank, n, howmany, 1);
}

fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                   fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out,
                                   const int* onembed, int ostride, int odist,
                                   unsigned flags)
{
    (void)in; (void)inembed; (void)istride; (void)idist; (void)out;
    (void)onembed; (void)ostride; (void)odist; (void)flags;
    return make(rank, n, howmany, 0);
}

void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out)
{
    size_t nall = (size_t)p->n[0] * p->n[1] * p->n[2];
    size_t nc = (size_t)p->n[0] * p->n[1] * (p->n[2] / 2 + 1);
    double* r = (double*)malloc(sizeof(double) * nall);
    fftm_cplx* c = (fftm_cplx*)malloc(sizeof(fftm_cplx) * nc);
    for (int b = 0; b < p->howmany; ++b)
    {
        for (size_t i = 0; i < nall; ++i) r[i] = in[b * nall + i];
        fftm_r2c_3d(r, c, p->n[0], p->n[1], p->n[2]);
        for (size_t i = 0; i < nc; ++i)
        {
            out[b * nc + i][0] = (float)c[i].re;
            out[b * nc + i][1] = (float)c[i].im;
        }
    }
    free(r);
    free(c);
}

void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out)
{
    size_t nall = (size_t)p->n[0] * p->n[1] * p->n[2];
    size_t nc = (size_t)p->n[0] * p->n[1] * (p->n[2] / 2 + 1);
    double* r = (double*)malloc(sizeof(double) * nall);
    fftm_cplx* c = (fftm_cplx*)malloc(sizeof(fftm_cplx) * nc);
    for (int b = 0; b < p->howmany; ++b)
    {
        for (size_t i = 0; i < nc; ++i)
        {
            c[i].re = in[b * nc + i][0];
            c[i].im = in[b * nc + i][1];
        }
        fftm_c2r_3d(c, r, p->n[0], p->n[1], p->n[2]);
        for (size_t i = 0; i < nall; ++i) out[b * nall + i] = (float)r[i];
    }
    free(r);
    free(c);
}

void fftwf_destroy_plan(fftwf_plan p) { free(p); }
