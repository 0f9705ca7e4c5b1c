/*
 * CPU restatement of the phasecon MBIR_4D hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This is the oracle the CUDA path is checked against. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only
 * as the checker or the timed CPU baseline; the product never calls it.
 * Each function cites the reference file:line it restates (paths relative to
 * the phasecon project root). The restatement is pinned against the reference
 * C built from source (oracle/Makefile, target `ref`) by tests/test_oracle.py.
 */
#ifndef MBIR_ORACLE_H
#define MBIR_ORACLE_H
#include <stdint.h>

#define ORC_RESP_BINS 64 /* DETECTOR_RESPONSE_BINS, MBIR_4D/XT_Constants.h:79 */

typedef struct {
    /* detector / sinogram (Sinogram, MBIR_4D/XT_Structures.h:61-89) */
    int32_t N_r, N_t, N_p, z_overlap;
    double delta_r, delta_t, R0, RMax, T0, TMax, OffsetR, OffsetT;
    /* object (ScannedObject, XT_Structures.h:91-125) */
    int32_t N_time, N_x, N_y, N_z, mult_xy, mult_z;
    double x0, y0, z0, delta_xy, delta_z, delta_recon, radius_obj;
    /* prior and solver (TomoInputs, XT_Structures.h:135-190) */
    double p, q, alpha, c_s, c_t;
    double sigma_s_q, sigma_s_q_p, sigma_t_q, sigma_t_q_p;
    double spatial_filter[27]; /* [z][y][x] offsets -1..1 */
    double time_filter;
    double huber_T, huber_delta;
    int32_t num_z_blocks;
} OrcGeom;

int orc_init_geometry(OrcGeom *g, int32_t proj_rows, int32_t proj_cols, int32_t proj_num, int32_t recon_num,
                      double vox_wid, double rot_center, double sig_s, double sig_t, double c_s, double c_t,
                      int32_t mult_xy, int32_t mult_z, double mrf_p, int32_t quad_convex, double huber_delta,
                      double huber_T, int32_t num_threads, const float *proj_times, const float *recon_times,
                      int32_t *proj_idx, int32_t *proj_cnt);

void orc_detector_response(const OrcGeom *g, const float *angles, float *H_r);

int32_t orc_amatrix_column(const OrcGeom *g, const float *H_r, double cosv, double sinv, int32_t view, int32_t row,
                           int32_t col, int32_t *index, double *value);

void orc_forward_project(const OrcGeom *g, const float *H_r, const float *angles, const int32_t *proj_idx,
                         const int32_t *proj_cnt, const float *object, double *Ax);

double orc_cost(const OrcGeom *g, const float *err, const float *weight, const float *object, double *parts);

double orc_functional_substitution(const OrcGeom *g, double V, double theta1, double theta2, const double *nhood,
                                   const uint8_t *nflag, const double *tnhood, const uint8_t *tflag);

void orc_random2_sequence(uint32_t seed, int32_t n, double *out);

int64_t orc_icd_pass(const OrcGeom *g, const float *H_r, const float *angles, const int32_t *proj_idx,
                     const int32_t *proj_cnt, const uint8_t *mask, const int32_t *order, int32_t n_order,
                     int32_t iter, float *object, float *err, const float *weight);

#endif
