/*
 * Harness around the reference MBIR_4D C sources, built from source by
 * oracle/Makefile into oracle/_ref/libref_mbir4d.so.
 *
 * TEST INFRASTRUCTURE ONLY: it exists to pin the C restatement in
 * oracle/mbir_oracle.c and to time the reference CPU path. Nothing in the
 * product links it.
 *
 * The Makefile compiles a scratch copy of Source_Code/MBIR_4D in which four
 * compile-time constants of XT_Constants.h / XT_Engine.c became globals that
 * this file owns (MRF_P, MAX_NUM_ITERATIONS, the multi-resolution stage count
 * clamp of XT_Engine.c:114-115, TIFF writes off) and a voxel-update counter was
 * added beside the call at XT_VoxUpdate.c:264. Everything else is the
 * reference's own code, reached through its own structures (XT_Structures.h).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdint.h>
#include <stdbool.h>
#include <omp.h>
#include "XT_Structures.h"
#include "XT_Init.h"
#include "XT_Profile.h"
#include "XT_AMatrix.h"
#include "XT_ICD_update.h"
#include "allocate.h"
#include "randlib.h"
#include "XT_NHICD.h"

/* Globals read by the patched reference (see the sed recipe in the Makefile). */
double oracle_ref_mrf_p = 1.2;
int oracle_ref_max_iter = 1000;
int oracle_ref_num_stages = 0; /* 0 keeps the reference's own stage plan */
long long oracle_ref_vox_updates = 0;

void oracle_ref_vox_updates_inc(void) { __atomic_fetch_add(&oracle_ref_vox_updates, 1, __ATOMIC_RELAXED); }

/* Reference functions that have no header prototype. */
Real_t computeCost(Sinogram *SinogramPtr, ScannedObject *ScannedObjectPtr, TomoInputs *TomoInputsPtr, Real_arr_t ***ErrorSino);
int32_t initErrorSinogam(Sinogram *SinogramPtr, ScannedObject *ScannedObjectPtr, TomoInputs *TomoInputsPtr, Real_arr_t **DetectorResponse, Real_arr_t ***ErrorSino);
int reconstruct(float **object, float *projections, float *weights, float *proj_angles, float *proj_times, float *recon_times, int32_t proj_rows, int32_t proj_cols, int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center, float sig_s, float sig_t, float c_s, float c_t, float convg_thresh, int32_t remove_rings, int32_t quad_convex, float huber_delta, float huber_T, uint8_t restart, FILE *debug_msg_ptr);

void ref_set_options(double mrf_p, int max_iter, int num_stages)
{
    oracle_ref_mrf_p = mrf_p;
    oracle_ref_max_iter = max_iter;
    oracle_ref_num_stages = num_stages;
}

long long ref_vox_updates(void) { return oracle_ref_vox_updates; }
void ref_reset_vox_updates(void) { oracle_ref_vox_updates = 0; }

/* One problem description shared by the entry points below. */
typedef struct {
    float *projections, *weights, *proj_angles, *proj_times, *recon_times;
    int32_t proj_rows, proj_cols, proj_num, recon_num;
    float vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh;
    int32_t quad_convex;
    float huber_delta, huber_T;
    int32_t mult_xy, mult_z;
} RefProblem;

typedef struct {
    Sinogram S;
    ScannedObject O;
    TomoInputs T;
    Real_arr_t **H_r;
    Real_arr_t *H_t;
} RefState;

static FILE *ref_log(void)
{
    static FILE *f = NULL;
    if (!f) f = fopen("/dev/null", "w");
    return f;
}

static int ref_init_rings(RefState *st, const RefProblem *pb, int32_t remove_rings)
{
    int32_t mxy[1], mz[1];
    memset(st, 0, sizeof(*st));
    mxy[0] = pb->mult_xy;
    mz[0] = pb->mult_z;
    st->T.debug_file_ptr = ref_log();
    if (initStructures(&st->S, &st->O, &st->T, 0, mxy, mz, pb->projections, pb->weights, pb->proj_angles,
                       pb->proj_times, pb->recon_times, pb->proj_rows, pb->proj_cols, pb->proj_num, pb->recon_num,
                       pb->vox_wid, pb->rot_center, pb->sig_s, pb->sig_t, pb->c_s, pb->c_t, pb->convg_thresh,
                       remove_rings, pb->quad_convex, pb->huber_delta, pb->huber_T))
        return -1;
    st->H_r = (Real_arr_t **)multialloc(sizeof(Real_arr_t), 2, st->S.N_p, DETECTOR_RESPONSE_BINS + 1);
    st->H_t = (Real_arr_t *)get_spc(DETECTOR_RESPONSE_BINS + 1, sizeof(Real_arr_t));
    DetectorResponseProfile(st->H_r, st->H_t, &st->S, &st->O, &st->T);
    return 0;
}

static int ref_init(RefState *st, const RefProblem *pb) { return ref_init_rings(st, pb, 0); }

static void ref_fini(RefState *st, int projection_freed)
{
    if (!projection_freed && st->S.Projection) multifree(st->S.Projection, 3);
    multifree(st->H_r, 2);
    free(st->H_t);
    free(Arr4DToArr1D(st->O.Object));
    freeMemory(&st->S, &st->O, &st->T);
}

/*
 * Geometry and prior constants after XT_Init.c:211-432 and the detector
 * response of XT_Profile.c:129-218.
 *   scal[0..15] = delta_r, delta_t, R0, RMax, T0, TMax, x0, y0, z0, delta_xy,
 *                 delta_z, OffsetR, OffsetT, delta_recon, radius_obj, z_overlap_num
 *   scal[16..22]= Sigma_S_Q, Sigma_S_Q_P, Sigma_T_Q, Sigma_T_Q_P, Time_Filter[0], N_z, num_z_blocks
 *   filt[27]    = Spatial_Filter[3][3][3]
 *   H_r[N_p*65], H_t[65]; proj_idx[N_p] (views per frame, frame-major), proj_cnt[N_time]
 */
int ref_geometry(const RefProblem *pb, double *scal, double *filt, float *H_r, float *H_t, int32_t *proj_idx, int32_t *proj_cnt)
{
    RefState st;
    int32_t i, j, k, n;
    if (ref_init(&st, pb)) return -1;
    scal[0] = st.S.delta_r; scal[1] = st.S.delta_t; scal[2] = st.S.R0; scal[3] = st.S.RMax;
    scal[4] = st.S.T0; scal[5] = st.S.TMax; scal[6] = st.O.x0; scal[7] = st.O.y0; scal[8] = st.O.z0;
    scal[9] = st.O.delta_xy; scal[10] = st.O.delta_z; scal[11] = st.S.OffsetR; scal[12] = st.S.OffsetT;
    scal[13] = st.O.delta_recon; scal[14] = st.T.radius_obj; scal[15] = st.S.z_overlap_num;
    scal[16] = st.T.Sigma_S_Q; scal[17] = st.T.Sigma_S_Q_P; scal[18] = st.T.Sigma_T_Q; scal[19] = st.T.Sigma_T_Q_P;
    scal[20] = st.T.Time_Filter[0]; scal[21] = st.O.N_z; scal[22] = st.T.num_z_blocks;
    for (i = 0; i < 3; i++) for (j = 0; j < 3; j++) for (k = 0; k < 3; k++)
        filt[(i * 3 + j) * 3 + k] = st.T.Spatial_Filter[i][j][k];
    for (i = 0; i < st.S.N_p; i++)
        for (j = 0; j <= DETECTOR_RESPONSE_BINS; j++) H_r[i * (DETECTOR_RESPONSE_BINS + 1) + j] = st.H_r[i][j];
    for (j = 0; j <= DETECTOR_RESPONSE_BINS; j++) H_t[j] = st.H_t[j];
    n = 0;
    for (i = 0; i < st.O.N_time; i++) {
        proj_cnt[i] = st.O.ProjNum[i];
        for (j = 0; j < st.O.ProjNum[i]; j++) proj_idx[n++] = st.O.ProjIdxPtr[i][j];
    }
    ref_fini(&st, 0);
    return 0;
}

/*
 * All A-matrix columns of XT_AMatrix.c:50-110 for every view and voxel
 * column: count[N_p][N_y][N_x], index/value[N_p][N_y][N_x][kmax].
 */
int ref_amatrix(const RefProblem *pb, int32_t kmax, uint8_t *count, int32_t *index, double *value)
{
    RefState st;
    AMatrixCol col;
    int32_t p, j, k, q;
    size_t base;
    if (ref_init(&st, pb)) return -1;
    col.values = (Real_t *)get_spc(64, sizeof(Real_t));
    col.index = (int32_t *)get_spc(64, sizeof(int32_t));
    for (p = 0; p < st.S.N_p; p++)
        for (j = 0; j < st.O.N_y; j++)
            for (k = 0; k < st.O.N_x; k++) {
                calcAMatrixColumnforAngle(&st.S, &st.O, st.H_r, &col, j, k, p);
                base = ((size_t)p * st.O.N_y + j) * st.O.N_x + k;
                count[base] = col.count;
                for (q = 0; q < col.count && q < kmax; q++) {
                    index[base * kmax + q] = col.index[q];
                    value[base * kmax + q] = col.values[q];
                }
            }
    free(col.values);
    free(col.index);
    ref_fini(&st, 0);
    return 0;
}

/*
 * Error sinogram e = y - Ax - d of XT_ICD_update.c:651-712 for an object
 * given without halo as [N_time][N_z][N_y][N_x]; e is returned in the
 * reference's internal layout [N_p][N_r][N_t] with the ProjSelect mask, and
 * the MAP cost of XT_ICD_update.c:185-318 for that state.
 */
int ref_error_sino_and_cost(const RefProblem *pb, const float *object, float *err, uint8_t *proj_select, double *cost)
{
    RefState st;
    Real_arr_t ***E;
    int32_t i, z, j, k, n;
    if (ref_init(&st, pb)) return -1;
    n = 0;
    for (i = 0; i < st.O.N_time; i++)
        for (z = 0; z < st.O.N_z; z++)
            for (j = 0; j < st.O.N_y; j++)
                for (k = 0; k < st.O.N_x; k++) st.O.Object[i][z + 1][j][k] = object[n++];
    E = (Real_arr_t ***)multialloc(sizeof(Real_arr_t), 3, st.S.N_p, st.S.N_r, st.S.N_t);
    if (initErrorSinogam(&st.S, &st.O, &st.T, st.H_r, E)) return -1;
    memcpy(err, &E[0][0][0], sizeof(float) * (size_t)st.S.N_p * st.S.N_r * st.S.N_t);
    for (i = 0; i < st.S.N_p * st.S.N_r * st.S.N_t; i++) proj_select[i] = (&st.S.ProjSelect[0][0][0])[i] ? 1 : 0;
    *cost = computeCost(&st.S, &st.O, &st.T, E);
    multifree(E, 3);
    ref_fini(&st, 1);
    return 0;
}

/*
 * The voxel surrogate solve CE_FunctionalSubstitution (XT_ICD_update.c:133-182)
 * on one neighbourhood, with the prior constants taken from a problem set up
 * by initStructures. nhood[27] is [z][y][x] around the voxel; flags likewise.
 */
int ref_functional_substitution(const RefProblem *pb, int32_t n, const double *V, const double *theta1,
                                const double *theta2, const double *nhood, const uint8_t *nflag,
                                const double *tnhood, const uint8_t *tflag, double *out)
{
    RefState st;
    Real_t sn[3][3][3], tn[2];
    bool sf[3][3][3], tf[2];
    int32_t m, a;
    if (ref_init(&st, pb)) return -1;
    for (m = 0; m < n; m++) {
        for (a = 0; a < 27; a++) {
            (&sn[0][0][0])[a] = nhood[m * 27 + a];
            (&sf[0][0][0])[a] = nflag[m * 27 + a] != 0;
        }
        for (a = 0; a < 2; a++) { tn[a] = tnhood[m * 2 + a]; tf[a] = tflag[m * 2 + a] != 0; }
        out[m] = CE_FunctionalSubstitution(V[m], theta1[m], theta2[m], &st.O, &st.T, sn, tn, sf, tf);
    }
    ref_fini(&st, 0);
    return 0;
}

/*
 * The reference's NH-ICD voxel-line selection (VSC_based_Voxel_Line_Select,
 * XT_NHICD.c:164-216) for one frame and one z block: mag is the update-
 * magnitude map [ny][nx], n_lines the number of voxel lines of the block
 * (UpdateSelectNum). sel[ny][nx] receives 1 for every selected line; the
 * return value is the number selected. RandomizedSelect draws from random2,
 * seeded here so the call is repeatable (its result does not depend on it).
 */
int32_t ref_vsc_select(int32_t ny, int32_t nx, const float *mag, int32_t n_lines, uint8_t *sel)
{
    ScannedObject O;
    TomoInputs T;
    int32_t i, n;
    memset(&O, 0, sizeof(O));
    memset(&T, 0, sizeof(T));
    O.N_time = 1;
    O.N_y = ny;
    O.N_x = nx;
    O.NHICD_Iterations = 10; /* XT_Init.c:406 */
    T.num_z_blocks = 1;
    T.UpdateSelectNum = (int32_t **)multialloc(sizeof(int32_t), 2, 1, 1);
    T.NHICDSelectNum = (int32_t **)multialloc(sizeof(int32_t), 2, 1, 1);
    T.x_NHICD_select = (int32_t ***)multialloc(sizeof(int32_t), 3, 1, 1, ny * nx);
    T.y_NHICD_select = (int32_t ***)multialloc(sizeof(int32_t), 3, 1, 1, ny * nx);
    Real_arr_t ****map = (Real_arr_t ****)multialloc(sizeof(Real_arr_t), 4, 1, 1, ny, nx);
    for (i = 0; i < ny * nx; i++) (&map[0][0][0][0])[i] = mag[i];
    T.UpdateSelectNum[0][0] = n_lines;
    srandom2(761521);
    VSC_based_Voxel_Line_Select(&O, &T, map);
    n = T.NHICDSelectNum[0][0];
    memset(sel, 0, (size_t)ny * nx);
    for (i = 0; i < n; i++) sel[T.y_NHICD_select[0][0][i] * nx + T.x_NHICD_select[0][0][i]] = 1;
    multifree(map, 4);
    multifree(T.x_NHICD_select, 3);
    multifree(T.y_NHICD_select, 3);
    multifree(T.UpdateSelectNum, 2);
    multifree(T.NHICDSelectNum, 2);
    return n;
}

/* The reference's Park-Miller generator (randlib.c:119-172). */
void ref_random2_sequence(uint32_t seed, int32_t n, double *out)
{
    int32_t i;
    srandom2(seed);
    for (i = 0; i < n; i++) out[i] = random2();
}

/*
 * The reference's top-level entry point (XT_Engine.c:81), run in the caller's
 * working directory (it writes cost.bin, object_time_*.bin, status.bin ...).
 * The returned buffer is the reference's own allocation and must be passed to
 * ref_free.
 */
int ref_reconstruct(const RefProblem *pb, int32_t threads, int32_t remove_rings, float **object)
{
    int rc;
    if (threads > 0) omp_set_num_threads(threads);
    *object = NULL;
    rc = reconstruct(object, pb->projections, pb->weights, pb->proj_angles, pb->proj_times, pb->recon_times,
                     pb->proj_rows, pb->proj_cols, pb->proj_num, pb->recon_num, pb->vox_wid, pb->rot_center,
                     pb->sig_s, pb->sig_t, pb->c_s, pb->c_t, pb->convg_thresh, remove_rings, pb->quad_convex,
                     pb->huber_delta, pb->huber_T, 0, ref_log());
    return rc;
}

void ref_free(void *p) { free(p); }

/*
 * One ring-correction update, update_Sinogram_Offset (XT_ICD_update.c:916-923),
 * of a problem set up by initStructures with remove_rings = mode: err
 * [N_p][N_r][N_t] (the error sinogram y - Ax - d) and d [N_r][N_t] (the
 * offset) are updated in place. ProjSelect is set from err first, as the
 * reference keeps it (|e sqrt(w)| < ErrorSinoThresh).
 */
void update_Sinogram_Offset(Sinogram *SinogramPtr, TomoInputs *TomoInputsPtr, Real_arr_t ***ErrorSino);

int ref_offset_update(const RefProblem *pb, int32_t mode, float *err, float *d)
{
    RefState st;
    Real_arr_t ***E;
    size_t i, n, nrt;
    if (ref_init_rings(&st, pb, mode)) return -1;
    n = (size_t)st.S.N_p * st.S.N_r * st.S.N_t;
    nrt = (size_t)st.S.N_r * st.S.N_t;
    E = (Real_arr_t ***)multialloc(sizeof(Real_arr_t), 3, st.S.N_p, st.S.N_r, st.S.N_t);
    memcpy(&E[0][0][0], err, n * sizeof(float));
    memcpy(&st.S.ProjOffset[0][0], d, nrt * sizeof(float));
    for (i = 0; i < n; i++)
        (&st.S.ProjSelect[0][0][0])[i] =
            fabs((&E[0][0][0])[i] * sqrt((&st.T.Weight[0][0][0])[i])) < st.T.ErrorSinoThresh;
    update_Sinogram_Offset(&st.S, &st.T, E);
    memcpy(err, &E[0][0][0], n * sizeof(float));
    memcpy(d, &st.S.ProjOffset[0][0], nrt * sizeof(float));
    multifree(E, 3);
    ref_fini(&st, 0);
    return 0;
}

/*
 * One noise-variance re-estimation, update_variance_parameter
 * (XT_ICD_update.c:716-747), of a problem set up by initStructures: err
 * [N_p][N_r][N_t], w [N_p][N_r][N_t] (the current weights, updated in place)
 * and *var_est (updated). ProjSelect is set from err and w first.
 */
void update_variance_parameter(Sinogram *SinogramPtr, TomoInputs *TomoInputsPtr, Real_arr_t ***ErrorSino);

int ref_variance_update(const RefProblem *pb, const float *err, float *w, double *var_est)
{
    RefState st;
    Real_arr_t ***E;
    size_t i, n;
    if (ref_init(&st, pb)) return -1;
    n = (size_t)st.S.N_p * st.S.N_r * st.S.N_t;
    E = (Real_arr_t ***)multialloc(sizeof(Real_arr_t), 3, st.S.N_p, st.S.N_r, st.S.N_t);
    memcpy(&E[0][0][0], err, n * sizeof(float));
    memcpy(&st.T.Weight[0][0][0], w, n * sizeof(float));
    st.T.var_est = *var_est;
    for (i = 0; i < n; i++)
        (&st.S.ProjSelect[0][0][0])[i] =
            fabs((&E[0][0][0])[i] * sqrt((&st.T.Weight[0][0][0])[i])) < st.T.ErrorSinoThresh;
    update_variance_parameter(&st.S, &st.T, E);
    memcpy(w, &st.T.Weight[0][0][0], n * sizeof(float));
    *var_est = st.T.var_est;
    multifree(E, 3);
    ref_fini(&st, 0);
    return 0;
}
