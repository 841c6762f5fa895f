/* TEST INFRASTRUCTURE ONLY.  Part of the oracle: never linked into the product.
 * Mixed-radix complex FFT in double precision; see fft_mixed.h. */
#include "fft_mixed.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static int smallest_factor(int n)
{
    for (int p = 2; p * p <= n; ++p)
        if (n % p == 0) return p;
    return n;
}

/* out[k] = sum_j in[j*stride] * w^(j*k), w = exp(sign*2*pi*i/n).
 * tw holds exp(sign*2*pi*i*t/n_top) for t in [0, n_top); n divides n_top. */
static void fft_rec(int n, const fftm_cplx* in, int stride, fftm_cplx* out,
                    const fftm_cplx* tw, int n_top, fftm_cplx* scratch)
{
    if (n == 1)
    {
        out[0] = in[0];
        return;
    }
    int p = smallest_factor(n);
    int m = n / p;
    for (int r = 0; r < p; ++r)
        fft_rec(m, in + (size_t)r * stride, stride * p, out + (size_t)r * m, tw,
                n_top, scratch + n);
    int step = n_top / n; /* tw index scale so that tw[t*step] = w_n^t */
    for (int k = 0; k < m; ++k)
    {
        for (int q = 0; q < p; ++q)
        {
            int kk = k + q * m;
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; ++r)
            {
                int t = (int)(((long long)r * kk) % n);
                fftm_cplx w = tw[(size_t)t * step];
                fftm_cplx x = out[(size_t)r * m + k];
                sr += x.re * w.re - x.im * w.im;
                si += x.re * w.im + x.im * w.re;
            }
            scratch[kk].re = sr;
            scratch[kk].im = si;
        }
    }
    memcpy(out, scratch, sizeof(fftm_cplx) * (size_t)n);
}

static fftm_cplx* make_twiddles(int n, int sign)
{
    fftm_cplx* tw = (fftm_cplx*)malloc(sizeof(fftm_cplx) * (size_t)n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int t = 0; t < n; ++t)
    {
        double a = sign * two_pi * (double)t / (double)n;
        tw[t].re = cos(a);
        tw[t].im = sin(a);
    }
    return tw;
}

/* Transform every line of length n (elements `stride` apart), lines starting
 * at base + l*line_step for l in [0, nlines). */
static void fft_lines(fftm_cplx* data, int n, size_t stride, size_t nlines,
                      size_t (*line_base)(size_t, const int*), const int* dims,
                      int sign)
{
    fftm_cplx* tw = make_twiddles(n, sign);
#pragma omp parallel
    {
        fftm_cplx* line = (fftm_cplx*)malloc(sizeof(fftm_cplx) * (size_t)n);
        fftm_cplx* res = (fftm_cplx*)malloc(sizeof(fftm_cplx) * (size_t)n);
        fftm_cplx* scr = (fftm_cplx*)malloc(sizeof(fftm_cplx) * (size_t)n * 4);
#pragma omp for schedule(static)
        for (long long l = 0; l < (long long)nlines; ++l)
        {
            size_t b = line_base((size_t)l, dims);
            for (int i = 0; i < n; ++i) line[i] = data[b + (size_t)i * stride];
            fft_rec(n, line, 1, res, tw, n, scr);
            for (int i = 0; i < n; ++i) data[b + (size_t)i * stride] = res[i];
        }
        free(line);
        free(res);
        free(scr);
    }
    free(tw);
}

/* line bases for the three axes of an [n0][n1][n2] array */
static size_t base_axis2(size_t l, const int* d) { return l * (size_t)d[2]; }
static size_t base_axis1(size_t l, const int* d)
{
    size_t i0 = l / (size_t)d[2], i2 = l % (size_t)d[2];
    return i0 * (size_t)d[1] * d[2] + i2;
}
static size_t base_axis0(size_t l, const int* d) { return l; }

void fftm_3d(fftm_cplx* data, int n0, int n1, int n2, int sign)
{
    int dims[3] = {n0, n1, n2};
    fft_lines(data, n2, 1, (size_t)n0 * n1, base_axis2, dims, sign);
    fft_lines(data, n1, (size_t)n2, (size_t)n0 * n2, base_axis1, dims, sign);
    fft_lines(data, n0, (size_t)n1 * n2, (size_t)n1 * n2, base_axis0, dims, sign);
}

void fftm_r2c_3d(const double* in, fftm_cplx* out, int n0, int n1, int n2)
{
    size_t nall = (size_t)n0 * n1 * n2;
    fftm_cplx* full = (fftm_cplx*)malloc(sizeof(fftm_cplx) * nall);
    for (size_t i = 0; i < nall; ++i)
    {
        full[i].re = in[i];
        full[i].im = 0.0;
    }
    fftm_3d(full, n0, n1, n2, -1);
    int nc = n2 / 2 + 1;
    for (int a = 0; a < n0; ++a)
        for (int b = 0; b < n1; ++b)
            for (int c = 0; c < nc; ++c)
                out[((size_t)a * n1 + b) * nc + c] =
                    full[((size_t)a * n1 + b) * n2 + c];
    free(full);
}

void fftm_c2r_3d(const fftm_cplx* in, double* out, int n0, int n1, int n2)
{
    size_t nall = (size_t)n0 * n1 * n2;
    int nc = n2 / 2 + 1;
    fftm_cplx* full = (fftm_cplx*)malloc(sizeof(fftm_cplx) * nall);
    for (int a = 0; a < n0; ++a)
        for (int b = 0; b < n1; ++b)
            for (int c = 0; c < n2; ++c)
            {
                fftm_cplx v;
                if (c < nc)
                    v = in[((size_t)a * n1 + b) * nc + c];
                else
                {
                    /* Hermitian partner of (-a, -b, -c) */
                    int ma = (n0 - a) % n0, mb = (n1 - b) % n1, mc = n2 - c;
                    v = in[((size_t)ma * n1 + mb) * nc + mc];
                    v.im = -v.im;
                }
                full[((size_t)a * n1 + b) * n2 + c] = v;
            }
    fftm_3d(full, n0, n1, n2, +1);
    for (size_t i = 0; i < nall; ++i) out[i] = full[i].re;
    free(full);
}
