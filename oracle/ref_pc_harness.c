/*
 * Harness around the reference PCMBIR_3D C sources (phase-contrast path),
 * built from source by oracle/Makefile (target `ref_pc`) into
 * oracle/_ref/libref_pcmbir.so with the FP64 FFTW-API shim of
 * oracle/fftw_shim/. TEST INFRASTRUCTURE ONLY: it pins the numpy
 * restatement in oracle/pcmbir_oracle.py. The entry points below call the
 * reference's own functions on caller-supplied per-view state; the structures
 * they need (ScannedObject, TomoInputs of PCMBIR_3D/XT_Structures.h) are filled
 * the way initStructures fills them (PCMBIR_3D/XT_Init.c:251-549).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdint.h>
#include <stdbool.h>
#include <unistd.h>
#include <fcntl.h>
#include "XT_Structures.h"
#include "XT_FresnelTran.h"
#include "XT_PhaseRet.h"
#include "XT_Search.h"
#include "XT_CmplxProjEst.h"
#include "XT_Paganin.h"
#include "allocate.h"

double oracle_ref_pc_mrf_p = 1.2;
/* phantom sizes of the data simulator (PHANTOM_XY_SIZE / PHANTOM_Z_SIZE) */
int oracle_ref_phantom_xy = 512;
int oracle_ref_phantom_z = 128;
int oracle_ref_pret_max_iter = 100; /* PRet_MaxIter of XT_Init.c:516 */

void initFilter(ScannedObject *ScannedObjectPtr, TomoInputs *TomoInputsPtr);
void create_FresnelTranWindow(Real_arr_t **Freq_Window, int32_t rows, int32_t cols, Real_t delta_rows, Real_t delta_cols, Real_t sigma);
void compute_DecorrObjTransform(Real_t DecorrTran[2][2], Real_t delta_over_beta, uint8_t recon_type);

typedef struct {
    int32_t rows, cols;
    double delta_rows, delta_cols, wavelength, distance, window_sigma;
    double mag_sig_s, mag_c_s, phase_sig_s, phase_c_s, delta_over_beta, mrf_p;
} PcParams;

static int quiet_begin(void)
{
    int saved;
    fflush(stdout);
    saved = dup(1);
    int nul = open("/dev/null", O_WRONLY);
    dup2(nul, 1);
    close(nul);
    return saved;
}

static void quiet_end(int saved)
{
    fflush(stdout);
    dup2(saved, 1);
    close(saved);
}

static Real_arr_t **window(const PcParams *p)
{
    Real_arr_t **w = (Real_arr_t **)multialloc(sizeof(Real_arr_t), 2, p->rows, p->cols);
    create_FresnelTranWindow(w, p->rows, p->cols, p->delta_rows, p->delta_cols, p->window_sigma);
    return w;
}

static Real_arr_t **as2d(double *data, int32_t rows, int32_t cols)
{
    Real_arr_t **a = (Real_arr_t **)malloc(sizeof(Real_arr_t *) * rows);
    int32_t i;
    for (i = 0; i < rows; i++) a[i] = data + (size_t)i * cols;
    return a;
}

static void setup_prior(const PcParams *p, ScannedObject *O, TomoInputs *T)
{
    memset(O, 0, sizeof(*O));
    memset(T, 0, sizeof(*T));
    oracle_ref_pc_mrf_p = p->mrf_p;
    O->mult_xy = 1;
    O->Mag_Sigma_S = p->mag_sig_s;
    O->Mag_C_S = p->mag_c_s;
    O->Phase_Sigma_S = p->phase_sig_s;
    O->Phase_C_S = p->phase_c_s;
    T->Mag_Sigma_S_Q = pow((O->Mag_Sigma_S * O->mult_xy), MRF_Q);
    T->Mag_Sigma_S_Q_P = pow(O->Mag_Sigma_S * O->mult_xy, MRF_Q - MRF_P);
    T->Phase_Sigma_S_Q = pow((O->Phase_Sigma_S * O->mult_xy), MRF_Q);
    T->Phase_Sigma_S_Q_P = pow(O->Phase_Sigma_S * O->mult_xy, MRF_Q - MRF_P);
    T->debug_file_ptr = stderr;
    initFilter(O, T);
    compute_DecorrObjTransform(O->DecorrTran, p->delta_over_beta, 2);
}

/* y = H x (herm = 0, compute_FresnelTran) or the reference's Hermitian
 * transform (herm = 1, compute_HermFresnelTran); x, y interleaved complex. */
void ref_pc_fresnel(const PcParams *p, const double *in, double *out, int herm)
{
    int32_t n = p->rows * p->cols, i;
    fftw_complex *a = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex *b = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_plan pf = fftw_plan_dft_2d(p->rows, p->cols, a, a, FFTW_FORWARD, FFTW_ESTIMATE);
    fftw_plan pb = fftw_plan_dft_2d(p->rows, p->cols, b, b, FFTW_BACKWARD, FFTW_ESTIMATE);
    Real_arr_t **w = window(p);
    for (i = 0; i < n; i++) { a[i][0] = in[2 * i]; a[i][1] = in[2 * i + 1]; }
    if (herm) compute_HermFresnelTran(p->rows, p->cols, p->delta_rows, p->delta_cols, a, &pf, b, &pb, p->wavelength, p->distance, w);
    else compute_FresnelTran(p->rows, p->cols, p->delta_rows, p->delta_cols, a, &pf, b, &pb, p->wavelength, p->distance, w);
    for (i = 0; i < n; i++) { out[2 * i] = b[i][0]; out[2 * i + 1] = b[i][1]; }
    multifree(w, 2);
    fftw_destroy_plan(pf);
    fftw_destroy_plan(pb);
    fftw_free(a);
    fftw_free(b);
}

/* One steepest-descent step (steepest_descent_iter, XT_PhaseRet.c:205-270) on
 * planar arrays; updates w and Omega in place and returns the step's
 * threshold statistic. */
double ref_pc_sd_iter(const PcParams *p, double *y_re, double *y_im, double *om_re, double *om_im, double *D_re,
                      double *D_im, double *w_re, double *w_im, double *lam, double *v_re, double *v_im, double nu)
{
    int32_t n = p->rows * p->cols, R = p->rows, C = p->cols;
    fftw_complex *a = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex *b = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_plan pf = fftw_plan_dft_2d(R, C, a, a, FFTW_FORWARD, FFTW_ESTIMATE);
    fftw_plan pb = fftw_plan_dft_2d(R, C, b, b, FFTW_BACKWARD, FFTW_ESTIMATE);
    Real_arr_t **win = window(p);
    Real_arr_t **Yr = as2d(y_re, R, C), **Yi = as2d(y_im, R, C), **Or = as2d(om_re, R, C), **Oi = as2d(om_im, R, C);
    Real_arr_t **Dr = as2d(D_re, R, C), **Di = as2d(D_im, R, C), **Wr = as2d(w_re, R, C), **Wi = as2d(w_im, R, C);
    Real_arr_t **L = as2d(lam, R, C), **Vr = as2d(v_re, R, C), **Vi = as2d(v_im, R, C);
    double t = steepest_descent_iter(Yr, Yi, Or, Oi, Dr, Di, Wr, Wi, L, Vr, Vi, nu, R, C, p->delta_rows, p->delta_cols,
                                     a, &pf, b, &pb, p->wavelength, p->distance, win);
    free(Yr); free(Yi); free(Or); free(Oi); free(Dr); free(Di); free(Wr); free(Wi); free(L); free(Vr); free(Vi);
    multifree(win, 2);
    fftw_destroy_plan(pf);
    fftw_destroy_plan(pb);
    fftw_free(a);
    fftw_free(b);
    return t;
}

/* Omega = phase of y / H(D w) (compute_phase_projection, XT_PhaseRet.c:10-33). */
void ref_pc_phase_projection(const PcParams *p, double *y_re, double *y_im, double *D_re, double *D_im, double *w_re,
                             double *w_im, double *om_re, double *om_im)
{
    int32_t n = p->rows * p->cols, R = p->rows, C = p->cols;
    fftw_complex *a = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex *b = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_plan pf = fftw_plan_dft_2d(R, C, a, a, FFTW_FORWARD, FFTW_ESTIMATE);
    fftw_plan pb = fftw_plan_dft_2d(R, C, b, b, FFTW_BACKWARD, FFTW_ESTIMATE);
    Real_arr_t **win = window(p);
    Real_arr_t **Yr = as2d(y_re, R, C), **Yi = as2d(y_im, R, C), **Or = as2d(om_re, R, C), **Oi = as2d(om_im, R, C);
    Real_arr_t **Dr = as2d(D_re, R, C), **Di = as2d(D_im, R, C), **Wr = as2d(w_re, R, C), **Wi = as2d(w_im, R, C);
    compute_phase_projection(Yr, Yi, Or, Oi, Dr, Di, Wr, Wi, R, C, p->delta_rows, p->delta_cols, a, &pf, b, &pb,
                             p->wavelength, p->distance, win);
    free(Yr); free(Yi); free(Or); free(Oi); free(Dr); free(Di); free(Wr); free(Wi);
    multifree(win, 2);
    fftw_destroy_plan(pf);
    fftw_destroy_plan(pb);
    fftw_free(a);
    fftw_free(b);
}

/* Nelder-Mead proximal search for n independent pixels
 * (Nelder_Mead_Simplex_2DSearch, XT_Search.c:112-215). z[4*i+1] is the
 * starting / returned point; nbr_r/nbr_i/flag hold each pixel's 3x3
 * neighbourhood; iters receives the iteration counts. */
void ref_pc_nms(const PcParams *p, int32_t n, double *zr, double *zi, const double *br, const double *bi,
                const double *nbr_r, const double *nbr_i, const uint8_t *flag, double nu, int32_t max_iter,
                double thresh, int32_t *iters)
{
    ScannedObject O;
    TomoInputs T;
    int32_t i, a, b;
    setup_prior(p, &O, &T);
    for (i = 0; i < n; i++) {
        Real_t nr[3][3], ni[3][3];
        bool f[3][3];
        for (a = 0; a < 3; a++)
            for (b = 0; b < 3; b++) {
                nr[a][b] = nbr_r[i * 9 + a * 3 + b];
                ni[a][b] = nbr_i[i * 9 + a * 3 + b];
                f[a][b] = flag[i * 9 + a * 3 + b] != 0;
            }
        iters[i] = Nelder_Mead_Simplex_2DSearch(zr + 4 * i, zi + 4 * i, 0, 0, br[i], bi[i], 1, 2, 0.5, 0.5, thresh,
                                                max_iter, 0.5, nu, stderr, nr, ni, f, &O, &T);
    }
}

/* The per-view phase-retrieval ADMM (estimate_complex_projection,
 * XT_CmplxProjEst.c:91-229) on one view; z_r/z_i are [rows*cols][4] simplex
 * arrays, everything else planar rows*cols. Writes its residual/cost files
 * into the working directory, as the reference does. */
void ref_pc_estimate(const PcParams *p, double *y_re, double *y_im, double *om_re, double *om_im, double *D_re,
                     double *D_im, double *z_r, double *z_i, double *lam, double *a_re, double *a_im, double *w_re,
                     double *w_im, double *v_re, double *v_im, int32_t nms_iters, int32_t sd_iters, int32_t pret_iters,
                     double mu, double nu)
{
    int32_t n = p->rows * p->cols, R = p->rows, C = p->cols, i, j;
    ScannedObject O;
    TomoInputs T;
    fftw_complex *a = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex *b = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_plan pf = fftw_plan_dft_2d(R, C, a, a, FFTW_FORWARD, FFTW_ESTIMATE);
    fftw_plan pb = fftw_plan_dft_2d(R, C, b, b, FFTW_BACKWARD, FFTW_ESTIMATE);
    Real_arr_t **win = window(p);
    Real_arr_t **Yr = as2d(y_re, R, C), **Yi = as2d(y_im, R, C), **Or = as2d(om_re, R, C), **Oi = as2d(om_im, R, C);
    Real_arr_t **Dr = as2d(D_re, R, C), **Di = as2d(D_im, R, C), **Wr = as2d(w_re, R, C), **Wi = as2d(w_im, R, C);
    Real_arr_t **L = as2d(lam, R, C), **Vr = as2d(v_re, R, C), **Vi = as2d(v_im, R, C);
    Real_arr_t **Ar = as2d(a_re, R, C), **Ai = as2d(a_im, R, C);
    Real_arr_t ***Zr = (Real_arr_t ***)malloc(sizeof(Real_arr_t **) * R), ***Zi = (Real_arr_t ***)malloc(sizeof(Real_arr_t **) * R);
    int saved;
    setup_prior(p, &O, &T);
    for (i = 0; i < R; i++) {
        Zr[i] = (Real_arr_t **)malloc(sizeof(Real_arr_t *) * C);
        Zi[i] = (Real_arr_t **)malloc(sizeof(Real_arr_t *) * C);
        for (j = 0; j < C; j++) {
            Zr[i][j] = z_r + ((size_t)i * C + j) * 4;
            Zi[i][j] = z_i + ((size_t)i * C + j) * 4;
        }
    }
    saved = quiet_begin();
    estimate_complex_projection(Yr, Yi, Or, Oi, Dr, Di, Zr, Zi, L, Ar, Ai, Wr, Wi, Vr, Vi, R, C, p->delta_rows,
                                p->delta_cols, 1, 2, 0.5, 0.5, 0.005, nms_iters, 0.0005, sd_iters, 0.0000001, pret_iters,
                                mu, nu, a, &pf, b, &pb, p->wavelength, p->distance, win, 0, &O, &T);
    quiet_end(saved);
    for (i = 0; i < R; i++) { free(Zr[i]); free(Zi[i]); }
    free(Zr); free(Zi);
    free(Yr); free(Yi); free(Or); free(Oi); free(Dr); free(Di); free(Wr); free(Wi); free(L); free(Vr); free(Vi);
    free(Ar); free(Ai);
    multifree(win, 2);
    fftw_destroy_plan(pf);
    fftw_destroy_plan(pb);
    fftw_free(a);
    fftw_free(b);
}

/* Single-material Paganin retrieval (paganins_1mat_phase_retrieval,
 * XT_Paganin.c:77-134). */
void ref_pc_paganin(const PcParams *p, double *meas, double *D_re, double *D_im, double wavenumber, double *z_r,
                    double *z_i)
{
    int32_t n = p->rows * p->cols, R = p->rows, C = p->cols;
    fftw_complex *a = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_complex *b = (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n);
    fftw_plan pf = fftw_plan_dft_2d(R, C, a, a, FFTW_FORWARD, FFTW_ESTIMATE);
    fftw_plan pb = fftw_plan_dft_2d(R, C, b, b, FFTW_BACKWARD, FFTW_ESTIMATE);
    Real_arr_t **M = as2d(meas, R, C), **Dr = as2d(D_re, R, C), **Di = as2d(D_im, R, C);
    Real_arr_t **Zr = as2d(z_r, R, C), **Zi = as2d(z_i, R, C);
    paganins_1mat_phase_retrieval(M, Dr, Di, Zr, Zi, R, C, p->delta_rows, p->delta_cols, a, &pf, b, &pb, wavenumber,
                                  p->wavelength, p->distance, p->delta_over_beta);
    free(M); free(Dr); free(Di); free(Zr); free(Zi);
    fftw_destroy_plan(pf);
    fftw_destroy_plan(pb);
    fftw_free(a);
    fftw_free(b);
}

void ref_pc_filter(const PcParams *p, double *filt27, double *decorr4)
{
    ScannedObject O;
    TomoInputs T;
    int32_t i;
    setup_prior(p, &O, &T);
    for (i = 0; i < 27; i++) filt27[i] = (&T.Spatial_Filter[0][0][0])[i];
    for (i = 0; i < 4; i++) decorr4[i] = (&O.DecorrTran[0][0])[i];
}
