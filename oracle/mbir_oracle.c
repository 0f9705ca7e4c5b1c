/*
 * CPU restatement of the phasecon MBIR_4D hot path (TEST INFRASTRUCTURE ONLY).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, as the checker or the timed CPU baseline. The product path
 * never calls it. Arithmetic follows the reference operation by operation
 * (double precision where the reference uses Real_t = double, float where it
 * stores Real_arr_t = float, MBIR_4D/XT_Constants.h:42-43) and the library is
 * built with -ffp-contract=off so that no multiply-add is fused, which keeps
 * the geometry, detector response and A-matrix values bit-identical to the
 * reference built from source.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "mbir_oracle.h"

#define PROFILE_RES 1536 /* PROFILE_RESOLUTION, MBIR_4D/XT_Constants.h:77 */
#define BEAM_RES 512     /* BEAM_RESOLUTION, XT_Constants.h:78 */
#define HALF_PI 1.57079632679489661923132169163975144
#define QUARTER_PI 0.785398163397448309615660845819875721

/* Distance to a neighbour in the 4-D (t,z,y,x) prior grid, XT_Init.c:138-141. */
static double nb_distance(int i, int j, int k, int l)
{
    return sqrt(pow((double)i - 1.0, 2.0) + pow((double)j - 1.0, 2.0) + pow((double)k - 1.0, 2.0) +
                pow((double)l - 1.0, 2.0));
}

/*
 * Geometry, view-to-frame map and prior constants of initStructures
 * (MBIR_4D/XT_Init.c:211-432) for a single stage with voxel scale mult_xy,
 * mult_z on one rank; view map per initSparseAnglesOfObject (XT_Init.c:69-96),
 * filters per initFilter (XT_Init.c:144-190), z-block count XT_Init.c:379-384.
 * proj_idx receives the views of every frame back to back (frame-major).
 */
int orc_init_geometry(OrcGeom *g, int32_t proj_rows, int32_t proj_cols, int32_t proj_num, int32_t recon_num,
                      double vox_wid, double rot_center, double sig_s, double sig_t, double c_s, double c_t,
                      int32_t mult_xy, int32_t mult_z, double mrf_p, int32_t quad_convex, double huber_delta,
                      double huber_T, int32_t num_threads, const float *proj_times, const float *recon_times,
                      int32_t *proj_idx, int32_t *proj_cnt)
{
    double length_R, length_T, sum, prior_const, tf, total;
    int32_t i, j, k, start, n, nb;
    memset(g, 0, sizeof(*g));
    g->mult_xy = mult_xy;
    g->mult_z = mult_z;
    g->p = mrf_p;
    g->q = 2.0;     /* MRF_Q, XT_Constants.h:63 */
    g->alpha = 1.5; /* OVER_RELAXATION_FACTOR, XT_Constants.h:87 */
    g->c_s = c_s;
    g->c_t = c_t;
    length_R = vox_wid * proj_cols;
    length_T = vox_wid * proj_rows;
    g->N_time = recon_num;
    g->N_p = proj_num;
    g->N_r = proj_cols;
    g->N_t = proj_rows;
    g->radius_obj = vox_wid * proj_cols / 2;
    g->delta_r = length_R / g->N_r;
    g->delta_t = length_T / g->N_t;
    g->R0 = -rot_center * g->delta_r;
    g->RMax = (g->N_r - rot_center) * g->delta_r;
    g->T0 = -length_T / 2.0;
    g->TMax = length_T / 2.0;
    g->N_x = (int32_t)(g->N_r / (double)mult_xy);
    g->N_y = g->N_x;
    g->N_z = (int32_t)(g->N_t / (double)mult_z);
    g->delta_xy = mult_xy * g->delta_r;
    g->delta_z = mult_z * g->delta_t;
    g->z_overlap = mult_z;
    g->x0 = g->R0;
    g->z0 = g->T0;
    g->y0 = -length_R / 2.0;
    g->OffsetR = (g->delta_xy / sqrt(2.0) + g->delta_r / 2.0) / ORC_RESP_BINS;
    g->OffsetT = ((g->delta_z / 2) + g->delta_t / 2) / ORC_RESP_BINS;
    if (quad_convex) {
        g->huber_T = 100000; /* ZINGER_DISABLE_PARAM_T, XT_Constants.h:97 */
        g->huber_delta = 1;  /* ZINGER_DISABLE_PARAM_DELTA, XT_Constants.h:98 */
    } else {
        g->huber_T = huber_T;
        g->huber_delta = huber_delta;
    }
    nb = num_threads / recon_num;
    if (nb < 2) nb = 2;
    else if (nb > g->N_z) nb = g->N_z;
    g->num_z_blocks = (nb / 2) * 2;

    for (i = 0; i + 1 < proj_num; i++)
        if (proj_times[i + 1] < proj_times[i]) return -1; /* XT_Init.c:109-110 */
    for (i = 0; i < recon_num; i++)
        if (recon_times[i + 1] < recon_times[i]) return -1; /* XT_Init.c:112-113 */
    start = 0;
    n = 0;
    total = 0;
    for (i = 0; i < recon_num; i++) {
        proj_cnt[i] = 0;
        for (j = start; j < proj_num; j++) {
            double t = proj_times[j];
            if (t >= recon_times[i] && t < recon_times[i + 1]) {
                proj_idx[n++] = j;
                proj_cnt[i]++;
            }
            if (t >= recon_times[i + 1]) {
                start = j;
                break;
            }
        }
        total += proj_cnt[i];
    }
    g->delta_recon = total / g->N_time;
    g->sigma_s_q = pow(sig_s * mult_xy, g->q);
    g->sigma_s_q_p = pow(sig_s * mult_xy, g->q - g->p);
    g->sigma_t_q = pow(sig_t * g->delta_recon, g->q);
    g->sigma_t_q_p = pow(sig_t * g->delta_recon, g->q - g->p);

    prior_const = (double)mult_xy * (double)mult_xy * (double)mult_xy * g->delta_recon;
    tf = 1.0 / nb_distance(0, 1, 1, 1);
    sum = 2.0 * tf;
    for (i = 0; i < 3; i++)
        for (j = 0; j < 3; j++)
            for (k = 0; k < 3; k++) {
                double v = 0;
                if (i != 1 || j != 1 || k != 1) {
                    v = 1.0 / nb_distance(1, i, j, k);
                    sum = sum + v;
                }
                g->spatial_filter[(i * 3 + j) * 3 + k] = v;
            }
    for (i = 0; i < 27; i++) g->spatial_filter[i] = prior_const * g->spatial_filter[i] / sum;
    g->time_filter = prior_const * tf / sum;
    return 0;
}

/*
 * Per-view detector response H_r[view][0..64] of DetectorResponseProfile
 * (XT_Profile.c:129-218): the voxel's trapezoidal line-integral profile
 * (calculateVoxelProfile, XT_Profile.c:47-104, stored as float) convolved with
 * a normalised Hamming beam (initializeBeamProfile, XT_Profile.c:108-124),
 * sampled every OffsetR; entry 64 is zero.
 */
void orc_detector_response(const OrcGeom *g, const float *angles, float *H_r)
{
    double beam[BEAM_RES], bsum = 0;
    float *prof = (float *)malloc(sizeof(float) * PROFILE_RES);
    double r0 = -(g->delta_r) / 2, step = (g->delta_r) / BEAM_RES;
    double scale = (PROFILE_RES) / (2 * g->delta_xy);
    int32_t v, i, j, p;
    for (i = 0; i < BEAM_RES; i++) {
        beam[i] = 0.54 - 0.46 * cos((2 * 3.14159265358979323846 / BEAM_RES) * i);
        bsum = bsum + beam[i];
    }
    for (i = 0; i < BEAM_RES; i++) beam[i] /= bsum;

    for (v = 0; v < g->N_p; v++) {
        double angle = angles[v], peak, c45, d1, d2, lc, ln, rn, rc;
        while (angle > HALF_PI) angle -= HALF_PI;
        while (angle < 0) angle += HALF_PI;
        if (angle <= QUARTER_PI) peak = g->delta_xy / cos(angle);
        else peak = g->delta_xy / cos(HALF_PI - angle);
        c45 = cos(QUARTER_PI);
        d1 = c45 * cos((QUARTER_PI - angle));
        d2 = c45 * fabs((cos((QUARTER_PI + angle))));
        lc = 1 - d1;
        ln = 1 - d2;
        rn = 1 + d2;
        rc = 1 + d1;
        for (j = 0; j < PROFILE_RES; j++) {
            double t = 2.0 * j / PROFILE_RES;
            if (t <= lc || t >= rc) prof[j] = 0;
            else if (t > rn) prof[j] = (float)(peak * (rc - t) / (rc - rn));
            else if (t >= ln) prof[j] = (float)peak;
            else prof[j] = (float)(peak * (t - lc) / (ln - lc));
        }
        for (i = 0; i < ORC_RESP_BINS; i++) {
            double center = i * g->OffsetR, rmin = center - g->delta_xy, s = 0;
            for (p = 0; p < BEAM_RES; p++) {
                double r = r0 + p * step;
                int32_t idx = (int32_t)floor((r - rmin) * scale);
                if (idx >= 0 && idx <= PROFILE_RES - 1) s += (prof[idx] * beam[p]);
            }
            H_r[v * (ORC_RESP_BINS + 1) + i] = (float)s;
        }
        H_r[v * (ORC_RESP_BINS + 1) + ORC_RESP_BINS] = 0.0f;
    }
    free(prof);
}

/*
 * One column of the sparse system matrix: the detector channels a voxel
 * column (row, col) projects onto at one view, with their weights, per
 * calcAMatrixColumnforAngle (XT_AMatrix.c:50-110). Returns the count.
 */
int32_t orc_amatrix_column(const OrcGeom *g, const float *H_r, double cosv, double sinv, int32_t view, int32_t row,
                           int32_t col, int32_t *index, double *value)
{
    const float *h = H_r + (size_t)view * (ORC_RESP_BINS + 1);
    double x = g->x0 + ((double)col + 0.5) * g->delta_xy;
    double y = g->y0 + ((double)row + 0.5) * g->delta_xy;
    double r = x * cosv - y * sinv;
    double rmin = r - g->delta_xy, rmax = r + g->delta_xy;
    int32_t imin, imax, j, count = 0;
    if (rmax < g->R0 || rmin > g->RMax) return 0;
    imin = (int32_t)(floor(((rmin - g->R0) / g->delta_r)));
    imax = (int32_t)(floor((rmax - g->R0) / g->delta_r));
    if (imax >= g->N_r) imax = g->N_r - 1;
    if (imin < 0) imin = 0;
    for (j = imin; j <= imax; j++) {
        double center = (g->R0 + (((double)j) + 0.5) * (g->delta_r));
        double d = fabs(r - center);
        int32_t bin = (int32_t)(floor((d / g->OffsetR)));
        if (bin >= 0 && bin < ORC_RESP_BINS) {
            double w1 = d - bin * g->OffsetR;
            double w2 = g->OffsetR - w1;
            double f1 = (w2 * h[bin] + w1 * h[bin + 1]) / g->OffsetR;
            if (f1 > 0) {
                value[count] = f1;
                index[count] = j;
                count++;
            }
        }
    }
    return count;
}

/*
 * Forward projection A x in double precision, as scattered by
 * initErrorSinogam / forward_project_voxel_AMat1D (XT_ICD_update.c:651-682,
 * XT_ForwardProject.c:44-61): each voxel slice covers z_overlap detector rows
 * with its A value unscaled. object is [N_time][N_z][N_y][N_x] without halo;
 * Ax is [N_p][N_r][N_t]. The error sinogram is y - Ax - d.
 */
void orc_forward_project(const OrcGeom *g, const float *H_r, const float *angles, const int32_t *proj_idx,
                         const int32_t *proj_cnt, const float *object, double *Ax)
{
    int32_t i, j, k, p, s, m, n, base = 0;
    int32_t idx[64];
    double val[64];
    memset(Ax, 0, sizeof(double) * (size_t)g->N_p * g->N_r * g->N_t);
    for (i = 0; i < g->N_time; i++) {
        for (p = 0; p < proj_cnt[i]; p++) {
            int32_t v = proj_idx[base + p];
            double cv = cos(angles[v]), sv = sin(angles[v]);
            double *row = Ax + (size_t)v * g->N_r * g->N_t;
            for (j = 0; j < g->N_y; j++)
                for (k = 0; k < g->N_x; k++) {
                    int32_t cnt = orc_amatrix_column(g, H_r, cv, sv, v, j, k, idx, val);
                    for (s = 0; s < g->N_z; s++) {
                        double px = object[(((size_t)i * g->N_z + s) * g->N_y + j) * g->N_x + k];
                        for (m = 0; m < cnt; m++)
                            for (n = 0; n < g->z_overlap; n++)
                                row[(size_t)idx[m] * g->N_t + s * g->z_overlap + n] += px * val[m];
                    }
                }
        }
        base += proj_cnt[i];
    }
}

/* qGGMRF potential and its derivative, XT_ICD_update.c:82-118. */
static double qg_value(const OrcGeom *g, double d, double sq, double sqp, double c)
{
    return ((pow(fabs(d), g->q) / sq) / (c + pow(fabs(d), g->q - g->p) / sqp));
}

static double qg_deriv(const OrcGeom *g, double d, double sq, double sqp, double c)
{
    double t1 = pow(fabs(d), g->q - g->p) / (sqp);
    double t2 = pow(fabs(d), g->q - 1);
    double t3 = c + t1;
    if (d < 0) return ((-1 * t2 / (t3 * sq)) * (g->q - ((g->q - g->p) * t1) / (t3)));
    return ((t2 / (t3 * sq)) * (g->q - ((g->q - g->p) * t1) / (t3)));
}

/*
 * MAP cost of computeCost (XT_ICD_update.c:185-318): half the weighted
 * squared error (generalised-Huber branch where |e sqrt(w)| >= T) plus the
 * causal-half-neighbourhood qGGMRF prior (13 spatial pairs and 1 temporal
 * pair per voxel); the log-variance term is zero for var_est = 1.
 * parts[0] = data term, parts[1] = prior term.
 */
double orc_cost(const OrcGeom *g, const float *err, const float *weight, const float *object, double *parts)
{
    size_t n, total = (size_t)g->N_p * g->N_r * g->N_t;
    double data = 0, prior = 0;
    int32_t i, z, j, k;
    const int32_t NX = g->N_x, NY = g->N_y, NZ = g->N_z, NT = g->N_time;
#define OBJ(ii, zz, jj, kk) (object[(((size_t)(ii) * NZ + (zz)) * NY + (jj)) * NX + (kk)])
#define SF(a, b, c) (g->spatial_filter[((a) * 3 + (b)) * 3 + (c)])
#define SV(d) qg_value(g, (double)(float)(d), g->sigma_s_q, g->sigma_s_q_p, g->c_s)
    for (n = 0; n < total; n++) {
        double t = err[n] * sqrt(weight[n]);
        if (fabs(t) < g->huber_T) t = t * t;
        else t = 2.0 * g->huber_delta * g->huber_T * fabs(t) + g->huber_T * g->huber_T * (1.0 - 2.0 * g->huber_delta);
        data += t;
    }
    data /= 2.0;
    for (i = 0; i < NT; i++)
        for (z = 0; z < NZ; z++)
            for (j = 0; j < NY; j++)
                for (k = 0; k < NX; k++) {
                    /* neighbour differences are taken in float, as the reference's
                       float - float (XT_ICD_update.c:226) */
                    float c = OBJ(i, z, j, k);
                    int jm = j - 1 >= 0, km = k - 1 >= 0, zp = z + 1 < NZ, ip = i + 1 < NT;
                    int jp = j + 1 < NY, kp = k + 1 < NX;
                    if (kp) prior += SF(1, 1, 2) * SV(c - OBJ(i, z, j, k + 1));
                    if (jp) {
                        if (km) prior += SF(1, 2, 0) * SV(c - OBJ(i, z, j + 1, k - 1));
                        prior += SF(1, 2, 1) * SV(c - OBJ(i, z, j + 1, k));
                        if (kp) prior += SF(1, 2, 2) * SV(c - OBJ(i, z, j + 1, k + 1));
                    }
                    if (zp) {
                        if (jm) prior += SF(2, 0, 1) * SV(c - OBJ(i, z + 1, j - 1, k));
                        prior += SF(2, 1, 1) * SV(c - OBJ(i, z + 1, j, k));
                        if (jp) prior += SF(2, 2, 1) * SV(c - OBJ(i, z + 1, j + 1, k));
                        if (jm) {
                            if (km) prior += SF(2, 0, 0) * SV(c - OBJ(i, z + 1, j - 1, k - 1));
                            if (kp) prior += SF(2, 0, 2) * SV(c - OBJ(i, z + 1, j - 1, k + 1));
                        }
                        if (km) prior += SF(2, 1, 0) * SV(c - OBJ(i, z + 1, j, k - 1));
                        if (jp) {
                            if (km) prior += SF(2, 2, 0) * SV(c - OBJ(i, z + 1, j + 1, k - 1));
                            if (kp) prior += SF(2, 2, 2) * SV(c - OBJ(i, z + 1, j + 1, k + 1));
                        }
                        if (kp) prior += SF(2, 1, 2) * SV(c - OBJ(i, z + 1, j, k + 1));
                    }
                    if (ip)
                        prior += g->time_filter * qg_value(g, (double)(float)(c - OBJ(i + 1, z, j, k)), g->sigma_t_q, g->sigma_t_q_p, g->c_t);
                }
#undef OBJ
#undef SF
#undef SV
    if (parts) {
        parts[0] = data;
        parts[1] = prior;
    }
    return data + prior;
}

/*
 * One-voxel surrogate solve of CE_FunctionalSubstitution
 * (XT_ICD_update.c:133-182): qGGMRF surrogate weights b = w rho'(d)/d (or
 * q/(sigma^q c) at d = 0, :119-128), minimiser u of the quadratic, then
 * over-relaxation x = V + alpha (u - V). nhood is [z][y][x] around the voxel
 * (its centre ignored), tnhood = {previous frame, next frame}.
 */
double orc_functional_substitution(const OrcGeom *g, double V, double theta1, double theta2, const double *nhood,
                                   const uint8_t *nflag, const double *tnhood, const uint8_t *tflag)
{
    double num = 0, den = 0, u;
    int32_t a;
    for (a = 0; a < 27; a++) {
        if (nflag[a] && a != 13) {
            double d = V - nhood[a], b, c;
            if (d != 0) b = qg_deriv(g, d, g->sigma_s_q, g->sigma_s_q_p, g->c_s) / d;
            else b = g->q / (g->sigma_s_q * g->c_s);
            c = g->spatial_filter[a] * b;
            num += c * nhood[a];
            den += c;
        }
    }
    for (a = 0; a < 2; a++) {
        if (tflag[a]) {
            double d = V - tnhood[a], b, c;
            if (d != 0) b = qg_deriv(g, d, g->sigma_t_q, g->sigma_t_q_p, g->c_t) / d;
            else b = g->q / (g->sigma_t_q * g->c_t);
            c = g->time_filter * b;
            num += c * tnhood[a];
            den += c;
        }
    }
    u = (num + (theta2 * V) - theta1) / (den + theta2);
    return V + g->alpha * (u - V);
}

/* Park-Miller minimal-standard generator of randlib.c:119-172, in 64-bit form. */
void orc_random2_sequence(uint32_t seed, int32_t n, double *out)
{
    uint64_t s = seed;
    int32_t i;
    for (i = 0; i < n; i++) {
        s = (s * 16807u) % 2147483647u;
        out[i] = (double)s / 2147483647.0;
    }
}

/*
 * Sequential ICD over a list of voxel columns (flat (frame*N_y + row)*N_x + col
 * indices), every slice of a column in ascending z, restating
 * updateVoxels_Atten (XT_VoxUpdate.c:119-283: neighbourhood with boundary
 * flags :168-236, zero skipping :238-261) and compute_voxel_update_Atten
 * (XT_VoxUpdate.c:45-117: theta1/theta2 over the column's A entries scaled by
 * delta_t, Huber weights where |e sqrt(w)| >= T, error-sinogram update).
 * object is [N_time][N_z][N_y][N_x]; err and weight are [N_p][N_r][N_t].
 * Returns the number of voxel updates performed (zero-skipped ones excluded).
 */
int64_t orc_icd_pass(const OrcGeom *g, const float *H_r, const float *angles, const int32_t *proj_idx,
                     const int32_t *proj_cnt, const uint8_t *mask, const int32_t *order, int32_t n_order,
                     int32_t iter, float *object, float *err, const float *weight)
{
    const int32_t NX = g->N_x, NY = g->N_y, NZ = g->N_z, NT = g->N_time, ZO = g->z_overlap;
    int32_t *first = (int32_t *)malloc(sizeof(int32_t) * (NT + 1));
    int32_t maxv = 0, t, o;
    int64_t updates = 0;
    int32_t *cnt, *idx;
    double *val;
    first[0] = 0;
    for (t = 0; t < NT; t++) {
        first[t + 1] = first[t] + proj_cnt[t];
        if (proj_cnt[t] > maxv) maxv = proj_cnt[t];
    }
    cnt = (int32_t *)malloc(sizeof(int32_t) * (maxv + 1));
    idx = (int32_t *)malloc(sizeof(int32_t) * (maxv + 1) * 64);
    val = (double *)malloc(sizeof(double) * (maxv + 1) * 64);
#define OBJ(ii, zz, jj, kk) object[(((size_t)(ii) * NZ + (zz)) * NY + (jj)) * NX + (kk)]
    for (o = 0; o < n_order; o++) {
        int32_t flat = order[o], i = flat / (NX * NY), j = (flat / NX) % NY, k = flat % NX, p, s;
        if (!mask[(size_t)j * NX + k]) continue;
        for (p = 0; p < proj_cnt[i]; p++) {
            int32_t v = proj_idx[first[i] + p];
            cnt[p] = orc_amatrix_column(g, H_r, cos(angles[v]), sin(angles[v]), v, j, k, idx + p * 64, val + p * 64);
        }
        for (s = 0; s < NZ; s++) {
            double nh[27], tn[2], V, th1 = 0, th2 = 0, xn;
            uint8_t nf[27], tf[2];
            int32_t dz, dy, dx, zs = 1;
            tf[0] = i - 1 >= 0;
            tn[0] = tf[0] ? OBJ(i - 1, s, j, k) : 0.0;
            tf[1] = i + 1 < NT;
            tn[1] = tf[1] ? OBJ(i + 1, s, j, k) : 0.0;
            for (dz = 0; dz < 3; dz++)
                for (dy = 0; dy < 3; dy++)
                    for (dx = 0; dx < 3; dx++) {
                        int32_t zz = s + dz - 1, yy = j + dy - 1, xx = k + dx - 1, a = (dz * 3 + dy) * 3 + dx;
                        int ok = zz >= 0 && zz < NZ && yy >= 0 && yy < NY && xx >= 0 && xx < NX;
                        nf[a] = (uint8_t)ok;
                        nh[a] = ok ? OBJ(i, zz, yy, xx) : 0.0;
                    }
            nh[13] = 0.0;
            V = OBJ(i, s, j, k);
            if (V == 0.0 && iter > 1) {
                int32_t a;
                if (tn[0] > 0.0 || tn[1] > 0.0) zs = 0;
                for (a = 0; a < 27; a++)
                    if (nh[a] > 0.0) zs = 0;
            } else {
                zs = 0;
            }
            if (zs) continue;
            for (p = 0; p < proj_cnt[i]; p++) {
                int32_t v = proj_idx[first[i] + p], q, r;
                for (q = 0; q < cnt[p]; q++) {
                    double a = val[p * 64 + q] * g->delta_t;
                    for (r = 0; r < ZO; r++) {
                        size_t e = ((size_t)v * g->N_r + idx[p * 64 + q]) * g->N_t + s * ZO + r;
                        if (fabs(err[e] * sqrt(weight[e])) < g->huber_T) {
                            th2 += (a * a * weight[e]);
                            th1 += -(err[e] * a * weight[e]);
                        } else {
                            double hw = g->huber_T * g->huber_delta * sqrt(weight[e]) / fabs(err[e]);
                            th2 += (a * a * hw);
                            th1 += -(err[e] * a * hw);
                        }
                    }
                }
            }
            xn = orc_functional_substitution(g, V, th1, th2, nh, nf, tn, tf);
            OBJ(i, s, j, k) = (float)xn;
            for (p = 0; p < proj_cnt[i]; p++) {
                int32_t v = proj_idx[first[i] + p], q, r;
                for (q = 0; q < cnt[p]; q++) {
                    double a = val[p * 64 + q] * g->delta_t;
                    for (r = 0; r < ZO; r++) {
                        size_t e = ((size_t)v * g->N_r + idx[p * 64 + q]) * g->N_t + s * ZO + r;
                        err[e] -= (a * (OBJ(i, s, j, k) - V));
                    }
                }
            }
            updates++;
        }
    }
#undef OBJ
    free(first);
    free(cnt);
    free(idx);
    free(val);
    return updates;
}
