/*
 * FP64 2-D complex DFT behind the FFTW3 calls PCMBIR_3D makes (test
 * infrastructure only; see fftw3.h). Each dimension is transformed with an
 * iterative radix-2 Cooley-Tukey FFT when its length is a power of two and
 * with a direct O(n^2) DFT otherwise. Twiddles are cos/sin of 2 pi k / len in
 * double for every butterfly stage len, tabulated once per plan (the same
 * expression per stage, so the values do not depend on the tabulation).
 * Validated against numpy.fft by tests/test_oracle_pc.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

/* Butterfly twiddles of one power-of-two length n: for stage len = 2, 4, ...,
 * n the half = len / 2 values cos/sin(sign 2 pi k / len), k < half, stored
 * one stage after another (n - 1 values), plus the bit-reversal permutation. */
typedef struct {
    int n;
    double *wr, *wi;
    int *rev;
} twiddles;

struct oracle_fftw_plan_s {
    int n0, n1, sign;
    fftw_complex *in, *out;
    twiddles t0, t1;
};

static void twiddles_init(twiddles *t, int n, int sign)
{
    int len, k, i, bits = 0, off = 0;
    memset(t, 0, sizeof(*t));
    t->n = n;
    if (n < 2 || (n & (n - 1)) != 0) return;
    t->wr = (double *)malloc(sizeof(double) * (size_t)n);
    t->wi = (double *)malloc(sizeof(double) * (size_t)n);
    t->rev = (int *)malloc(sizeof(int) * (size_t)n);
    for (len = 2; len <= n; len <<= 1) {
        int half = len / 2;
        for (k = 0; k < half; k++) {
            double ang = sign * 2.0 * M_PI * k / len;
            t->wr[off + k] = cos(ang);
            t->wi[off + k] = sin(ang);
        }
        off += half;
    }
    while ((1 << bits) < n) bits++;
    for (i = 0; i < n; i++) {
        int r = 0, b;
        for (b = 0; b < bits; b++) if (i & (1 << b)) r |= 1 << (bits - 1 - b);
        t->rev[i] = r;
    }
}

static void twiddles_free(twiddles *t)
{
    free(t->wr);
    free(t->wi);
    free(t->rev);
}

static void dft1(double *re, double *im, int n, int stride, int sign, const twiddles *tw, double *tr, double *ti)
{
    int k, j;
    if ((n & (n - 1)) == 0) {
        /* bit-reverse permutation, then butterflies */
        int i, len, off = 0;
        if (n < 2) return;
        for (i = 0; i < n; i++) {
            const int r = tw->rev[i];
            tr[r] = re[(size_t)i * stride];
            ti[r] = im[(size_t)i * stride];
        }
        for (len = 2; len <= n; len <<= 1) {
            int half = len / 2;
            const double *wrs = tw->wr + off, *wis = tw->wi + off;
            for (i = 0; i < n; i += len)
                for (k = 0; k < half; k++) {
                    double wr = wrs[k], wi = wis[k];
                    double ar = tr[i + k], ai = ti[i + k];
                    double br = tr[i + k + half], bi = ti[i + k + half];
                    double xr = br * wr - bi * wi, xi = br * wi + bi * wr;
                    tr[i + k] = ar + xr;
                    ti[i + k] = ai + xi;
                    tr[i + k + half] = ar - xr;
                    ti[i + k + half] = ai - xi;
                }
            off += half;
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
    twiddles_init(&p->t0, n0, sign);
    twiddles_init(&p->t1, n1, sign);
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
    for (i = 0; i < n0; i++) dft1(re + (size_t)i * n1, im + (size_t)i * n1, n1, 1, p->sign, &p->t1, tr, ti);
    for (i = 0; i < n1; i++) dft1(re + i, im + i, n0, n1, p->sign, &p->t0, tr, ti);
    for (q = 0; q < n; q++) {
        p->out[q][0] = re[q];
        p->out[q][1] = im[q];
    }
    free(re);
    free(im);
    free(tr);
    free(ti);
}

void fftw_destroy_plan(fftw_plan p)
{
    if (!p) return;
    twiddles_free(&p->t0);
    twiddles_free(&p->t1);
    free(p);
}
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
