/*
 * FP64 2-D complex DFT behind the FFTW3 calls PCMBIR_3D makes (test
 * infrastructure only; see fftw3.h). Each dimension is transformed with an
 * iterative radix-2 Cooley-Tukey FFT when its length is a power of two and
 * with a direct O(n^2) DFT otherwise. Twiddles are computed with cos/sin of
 * 2 pi k / n in double. Validated against numpy.fft by tests/test_oracle_pc.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

struct oracle_fftw_plan_s {
    int n0, n1, sign;
    fftw_complex *in, *out;
};

static void dft1(double *re, double *im, int n, int stride, int sign, double *tr, double *ti)
{
    int k, j;
    if ((n & (n - 1)) == 0) {
        /* bit-reverse permutation, then butterflies */
        int i, bits = 0, len;
        while ((1 << bits) < n) bits++;
        for (i = 0; i < n; i++) {
            int r = 0, b;
            for (b = 0; b < bits; b++) if (i & (1 << b)) r |= 1 << (bits - 1 - b);
            tr[r] = re[(size_t)i * stride];
            ti[r] = im[(size_t)i * stride];
        }
        for (len = 2; len <= n; len <<= 1) {
            int half = len / 2;
            for (i = 0; i < n; i += len)
                for (k = 0; k < half; k++) {
                    double ang = sign * 2.0 * M_PI * k / len;
                    double wr = cos(ang), wi = sin(ang);
                    double ar = tr[i + k], ai = ti[i + k];
                    double br = tr[i + k + half], bi = ti[i + k + half];
                    double xr = br * wr - bi * wi, xi = br * wi + bi * wr;
                    tr[i + k] = ar + xr;
                    ti[i + k] = ai + xi;
                    tr[i + k + half] = ar - xr;
                    ti[i + k + half] = ai - xi;
                }
        }
    } else {
        for (k = 0; k < n; k++) {
            double sr = 0, si = 0;
            for (j = 0; j < n; j++) {
                double ang = sign * 2.0 * M_PI * (double)((long long)j * k % n) / n;
                double wr = cos(ang), wi = sin(ang);
                double xr = re[(size_t)j * stride], xi = im[(size_t)j * stride];
                sr += xr * wr - xi * wi;
                si += xr * wi + xi * wr;
            }
            tr[k] = sr;
            ti[k] = si;
        }
    }
    for (k = 0; k < n; k++) {
        re[(size_t)k * stride] = tr[k];
        im[(size_t)k * stride] = ti[k];
    }
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags)
{
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    (void)flags;
    p->n0 = n0;
    p->n1 = n1;
    p->sign = sign;
    p->in = in;
    p->out = out;
    return p;
}

void fftw_execute(const fftw_plan p)
{
    int n0 = p->n0, n1 = p->n1, i, nmax = n0 > n1 ? n0 : n1;
    size_t n = (size_t)n0 * n1;
    double *re = (double *)malloc(sizeof(double) * n), *im = (double *)malloc(sizeof(double) * n);
    double *tr = (double *)malloc(sizeof(double) * nmax), *ti = (double *)malloc(sizeof(double) * nmax);
    size_t q;
    for (q = 0; q < n; q++) {
        re[q] = p->in[q][0];
        im[q] = p->in[q][1];
    }
    for (i = 0; i < n0; i++) dft1(re + (size_t)i * n1, im + (size_t)i * n1, n1, 1, p->sign, tr, ti);
    for (i = 0; i < n1; i++) dft1(re + i, im + i, n0, n1, p->sign, tr, ti);
    for (q = 0; q < n; q++) {
        p->out[q][0] = re[q];
        p->out[q][1] = im[q];
    }
    free(re);
    free(im);
    free(tr);
    free(ti);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
