/*
 * FP64 stand-in for the part of the FFTW3 API that PCMBIR_3D calls
 * (TEST INFRASTRUCTURE ONLY). FFTW is not installed in this image; the
 * reference's phase-contrast code (PCMBIR_3D/XT_FresnelTran.c:23,68,94,126,
 * XT_Paganin.c:93,116, plans XT_Init.c:345-351) needs only in-place complex
 * 2-D transforms. Sign convention as FFTW: FFTW_FORWARD = exp(-2 pi i jk/n),
 * FFTW_BACKWARD = exp(+2 pi i jk/n), both unnormalised.
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
#include <stddef.h>

typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#endif
