/*
 * mbirgpu -- B200 (sm_100a) implementation of phasecon's MBIR hot path.
 *
 * C ABI of libmbirgpu.so (phasecon_b200/libmbirgpu.so). Plain pointers and
 * sizes only. Every function returns 0 on success and -1 on failure, like the
 * reference's check_error/goto error convention (MBIR_4D/XT_Debug.h:22); the
 * message of the last failure on the calling thread is mbirgpu_last_error().
 * All pointers are HOST pointers unless the parameter name starts with d_.
 *
 * Paths cited below are relative to the phasecon project root.
 */
#ifndef MBIRGPU_H
#define MBIRGPU_H

#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* --------------------------------------------------------------------------
 * Drop-in entry point.
 *
 * Replaces reconstruct() of MBIR_4D/XT_Engine.c:81 (declared void in
 * include/mbir4d.h:35; defined int, returns 0 / -1). Same arguments, same
 * meaning, same output: *object receives a malloc'ed buffer the caller
 * free()s, laid out [recon_num][proj_rows+2][proj_cols][proj_cols] -- the
 * reference returns its backing array with one halo slice above and below
 * each frame's volume (MBIR_4D/XT_IOMisc.c:331-336, XT_Init.c:362-363); the
 * halo slices are zero. Writes the reference's side-effect files in the
 * working directory (object_time_<i>.bin, cost.bin, status.bin,
 * variance_estimate.bin, mag_update.bin, proj_offset.bin) unless disabled by
 * mbirgpu_set_options. remove_rings 1-3 estimates the per-detector-pixel
 * offset as the reference does (none in the coarsest stage, from zero in the
 * second, carried over after that; see mbirgpu_session_set_ring_correction).
 * restart = 1 resumes from status.bin like XT_Engine.c:143-150.
 * No MPI is required.
 * ------------------------------------------------------------------------ */
int reconstruct(float **object, float *projections, float *weights, float *proj_angles, float *proj_times,
                float *recon_times, int32_t proj_rows, int32_t proj_cols, int32_t proj_num, int32_t recon_num,
                float vox_wid, float rot_center, float sig_s, float sig_t, float c_s, float c_t,
                float convg_thresh, int32_t remove_rings, int32_t quad_convex, float huber_delta, float huber_T,
                uint8_t restart, FILE *debug_msg_ptr);

/* --------------------------------------------------------------------------
 * Former compile-time constants of MBIR_4D/XT_Constants.h, now runtime.
 * ------------------------------------------------------------------------ */
typedef struct {
    double mrf_p;            /* MRF_P (XT_Constants.h:62), default 1.2 */
    double mrf_q;            /* MRF_Q (XT_Constants.h:63), default 2.0 */
    double alpha;            /* OVER_RELAXATION_FACTOR (XT_Constants.h:87), default 1.5 */
    int32_t max_iterations;  /* MAX_NUM_ITERATIONS (XT_Constants.h:86), default 1000 */
    int32_t num_stages;      /* multi-resolution stages: 0 = reference plan (XT_Engine.c:111-141),
                                n > 0 = the n finest stages of that plan */
    double cost_rel_tol;     /* also stop a stage when |cost_k - cost_{k-1}| / |cost_k| < tol; 0 = off */
    int32_t zero_skipping;   /* ZERO_SKIPPING (XT_Constants.h:47), default 1 */
    int32_t write_files;     /* reference side-effect files, default 1 */
    int32_t compute_cost;    /* FP64 MAP cost every iteration (cost.bin), default 1 */
    int32_t refresh_every;   /* FP64 recomputation of e = y - Ax every n iterations, default 8 */
    int32_t sv_size;         /* super-voxel edge in voxel columns; 0 = by rule or autotuned */
    int32_t cta_warps;       /* warps cooperating on one voxel column; 0 = by rule or autotuned */
    int32_t icd_unroll;      /* views whose A records and sinogram entries one lane keeps in flight
                                (1, 2 or 4); 0 = autotuned */
    uint64_t seed;           /* voxel-order seed */
    int32_t nhicd_passes;    /* non-homogeneous ICD (XT_ICD_update.c:1007-1047, XT_NHICD.c:164-216):
                                from iteration 2, after the full sweep, n passes each re-update the
                                voxel columns with the largest 5x5-Hamming-filtered update magnitude
                                (1/NHICD_Iterations of the masked columns per frame, as the
                                reference); 0 = off, up to 16. Default 10 (the reference's
                                NHICD_Iterations, XT_Init.c:406; NO_NHICD is 0) */
    int32_t sv_colors;       /* super-voxel colouring: K x K colour classes, K = 2 (4 phases per
                                sweep) or 4 (16 phases: same-colour super-voxels twice as far
                                apart); 0 = by rule or autotuned */
    int32_t stage_records;   /* 1 (default): the ICD sweep copies each next voxel column's A
                                records into shared memory while it updates the current one;
                                0: records are read from global memory where they are used */
    int32_t nh_sv_size;      /* super-voxel edge of the non-homogeneous passes; 0 = autotuned */
    int32_t nh_sv_colors;    /* K of their K x K colouring (2 or 4); 0 = autotuned */
    int32_t nh_cta_warps;    /* warps cooperating on one voxel column in those passes; 0 = autotuned */
    int32_t nh_work_lists;   /* 1 (default): those passes visit only super-voxels holding selected
                                columns, the ones with the most first; 0: every super-voxel */
    int32_t autotune;        /* 0 (default): the schedule fields left at 0 follow a fixed rule of
                                the problem's shape (super-voxels 4 x 4, K = 2, 4 warps per column
                                when a frame has >= 64 views, else 2), so the same inputs give the
                                same schedule and the same image on every run; 1: a single
                                session measures the candidate schedules on its own problem and
                                keeps the fastest (timing-dependent); batches always measure */
    int32_t graph_iterations;/* 1 (default): a session on a stream of its own (not the legacy
                                default stream) replays each ICD iteration -- colour phases,
                                non-homogeneous passes, FP64 refresh -- from a CUDA graph captured
                                on first use (one graph per kind of iteration; the kernels read the
                                iteration number from device memory); iterations with ring
                                correction or variance re-estimation, and the legacy default
                                stream, launch directly. 0: always launch directly */
} mbirgpu_options;

/* Defaults as listed above. */
void mbirgpu_default_options(mbirgpu_options *opt);
int mbirgpu_set_options(const mbirgpu_options *opt);
int mbirgpu_get_options(mbirgpu_options *opt);
const char *mbirgpu_last_error(void);

/* --------------------------------------------------------------------------
 * Session API: one problem resident in GPU memory at one voxel scale.
 *
 * The problem fields carry the same meaning as reconstruct()'s arguments
 * (MBIR_4D/XT_Engine.c:50-80). A session is one stage of the reference's
 * multi-resolution loop: initStructures (MBIR_4D/XT_Init.c:211-432) plus the
 * state ICD_BackProject keeps (XT_ICD_update.c:1095-1230).
 * Device layouts: sinograms [N_p][N_r][N_t] (t fastest, as the reference's
 * internal arrays, XT_Init.c:292-301); the object [N_time][N_y][N_x][N_z]
 * (z fastest). Host object buffers exchanged through this API use the
 * reference's volume order [N_time][N_z][N_y][N_x] without halo.
 * ------------------------------------------------------------------------ */
typedef struct mbirgpu_session mbirgpu_session;

typedef struct {
    const float *projections; /* [proj_num][proj_rows][proj_cols] */
    const float *weights;     /* [proj_num][proj_rows][proj_cols] */
    const float *proj_angles; /* [proj_num], radians */
    const float *proj_times;  /* [proj_num], nondecreasing */
    const float *recon_times; /* [recon_num + 1] frame edges */
    int32_t proj_rows, proj_cols, proj_num, recon_num;
    float vox_wid, rot_center, sig_s, sig_t, c_s, c_t, convg_thresh;
    int32_t quad_convex;
    float huber_delta, huber_T;
} mbirgpu_problem;

typedef struct {
    int32_t N_r, N_t, N_p, N_time, N_x, N_y, N_z, mult_xy, mult_z;
    int32_t max_views;       /* most views in one frame */
    int32_t kmax;            /* most detector channels one voxel column hits per view */
    int32_t sv_size, cta_warps;
    int64_t masked_columns;  /* voxel columns inside the reconstruction circle, all frames */
    int64_t nnz;             /* A-matrix nonzeros (view, channel) of the columns inside the circle,
                                summed over frames; one voxel slice reads nnz*z_overlap entries */
    double delta_t;
    size_t device_bytes;     /* device memory the session holds */
    int32_t sv_colors;       /* K of the K x K super-voxel colouring in use */
} mbirgpu_session_info;

typedef struct {
    int64_t voxel_updates;   /* updates that ran (zero-skipped ones excluded) */
    int64_t zero_skipped;
    double sum_abs_update;   /* sum |x_new - x_old| */
    double sum_abs_value;    /* sum |x_new| over updated voxels */
    double kernel_ms;        /* device time of the ICD sweep kernels (when timing is on) */
    int32_t kernel_launches;
} mbirgpu_iter_stats;

/* Replaces initStructures + DetectorResponseProfile (MBIR_4D/XT_Init.c:211,
 * XT_Profile.c:129) for one stage with voxel scale (mult_xy, mult_z), and
 * builds the compressed A-matrix table on the device. stream may be NULL
 * (the default stream) or a cudaStream_t every launch of the session uses. */
int mbirgpu_session_create(mbirgpu_session **out, const mbirgpu_problem *pb, const mbirgpu_options *opt,
                           int32_t mult_xy, int32_t mult_z, void *stream);
int mbirgpu_session_destroy(mbirgpu_session *s);
int mbirgpu_session_info_get(const mbirgpu_session *s, mbirgpu_session_info *info);
int mbirgpu_session_set_stream(mbirgpu_session *s, void *stream);
int mbirgpu_session_set_timing(mbirgpu_session *s, int32_t enable);

/* Object upload / download, [N_time][N_z][N_y][N_x] without halo. */
int mbirgpu_session_set_object(mbirgpu_session *s, const float *object);
int mbirgpu_session_get_object(mbirgpu_session *s, float *object);
/* Device pointer to the resident object ([N_time][N_y][N_x][N_z]). */
int mbirgpu_session_object_device(mbirgpu_session *s, float **d_object);

/* Replaces initErrorSinogam (MBIR_4D/XT_ICD_update.c:651-712): e = y - A x
 * with the projection accumulated in FP64; also the periodic refresh. */
int mbirgpu_session_refresh_error(mbirgpu_session *s);
int mbirgpu_session_get_error(mbirgpu_session *s, float *err); /* [N_p][N_r][N_t] */

/* Replaces computeCost (MBIR_4D/XT_ICD_update.c:185-318); FP64. */
int mbirgpu_session_cost(mbirgpu_session *s, double *total, double *data_term, double *prior_term);

/* One ICD iteration: every voxel column inside the reconstruction circle of
 * every frame updated once, super-voxel parallel. Replaces
 * updateVoxelsTimeSlices (MBIR_4D/XT_ICD_update.c:932-1092) with
 * updateVoxels_Atten / compute_voxel_update_Atten (XT_VoxUpdate.c:45-283). */
int mbirgpu_session_icd_iteration(mbirgpu_session *s, int32_t iter, mbirgpu_iter_stats *stats);

/* Forward projection A x of a host object (no error, no weights) and the
 * adjoint A^T s of a host sinogram, both FP64-accumulated; replaces
 * forward_project_voxel_AMat1D (MBIR_4D/XT_ForwardProject.c:44-61) and the
 * back-projection implicit in theta1 (XT_VoxUpdate.c:56-85). */
int mbirgpu_session_forward_project(mbirgpu_session *s, const float *object, float *sino);
int mbirgpu_session_back_project(mbirgpu_session *s, const float *sino, float *object);

/* Filtered back-projection of the measurements (Ram-Lak ramp filter, then
 * the adjoint of the A matrix per frame, scaled by pi / views of the frame):
 * the classical initial image. _fbp returns it ([N_time][N_z][N_y][N_x]);
 * _set_object_fbp makes it the current object, zero outside the
 * reconstruction circle like every object ICD works on (and recomputes e).
 * The reference starts from zero or a restart file (initObject,
 * MBIR_4D/XT_ICD_update.c:540-647); FBP has no counterpart there. */
int mbirgpu_session_fbp(mbirgpu_session *s, float *object);
int mbirgpu_session_set_object_fbp(mbirgpu_session *s);
/* The current object becomes zero on the device (the reference's zero
 * initialisation, XT_ICD_update.c:540-647 with no previous stage), then
 * e = y - A x - d; no host buffer is involved. */
int mbirgpu_session_set_object_zero(mbirgpu_session *s);

/* Ring correction (remove_rings of reconstruct, MBIR_4D/XT_Engine.c:73):
 * the session estimates one offset d per detector pixel, shared by all views,
 * so that e = y - Ax - d (update_Sinogram_Offset, XT_ICD_update.c:749-923);
 * mode 1 leaves d free, 2 constrains its mean to zero, 3 is the reference's
 * rectangular-window mode, whose windows its reconstruct never builds
 * (gen_offset_constraint_windows runs only in the simulator's set-up), so d
 * becomes the weighted mean of e + d over the views; 0 turns it off. d is
 * re-estimated after every full-sweep colour phase and every NH pass.
 * offset: the starting d, [proj_cols][proj_rows] (the reference's
 * ProjOffset[N_r][N_t]), or NULL for zero. The error sinogram is recomputed. */
int mbirgpu_session_set_ring_correction(mbirgpu_session *s, int32_t remove_rings, const float *offset);
/* Noise-variance re-estimation of the generalised-Huber data term
 * (update_variance_parameter, MBIR_4D/XT_ICD_update.c:716-747), which
 * reconstruct runs after its first multires stage when quad_convex = 0: with
 * on != 0 the variance (starting at 1) is re-estimated at the end of every
 * ICD iteration and the weights are rescaled by it; the cost then includes
 * N log(var) / 2 (XT_ICD_update.c:307). update_variance runs one
 * re-estimation now; get_variance returns the current value. */
int mbirgpu_session_set_variance_estimation(mbirgpu_session *s, int32_t on);
int mbirgpu_session_update_variance(mbirgpu_session *s);
int mbirgpu_session_get_variance(mbirgpu_session *s, double *var_est);
/* One offset update with the object fixed (the step the ICD iteration runs
 * after each phase): d and e change together. */
int mbirgpu_session_update_offset(mbirgpu_session *s);
/* The current offset d, [proj_cols][proj_rows] (zero without ring correction). */
int mbirgpu_session_get_offset(mbirgpu_session *s, float *offset);
/* The NH-ICD voxel-line selection for a given update-magnitude map (for
 * inspection): mag [N_time][N_y][N_x] (sum over z of |update| of each voxel
 * column's latest visit, MagUpdateMap), sel [N_time][N_y][N_x] receives 1
 * for the columns an NH pass would visit -- the masked columns among the
 * masked/NHICD_Iterations largest 5x5-Hamming-filtered values of the frame
 * (VSC_based_Voxel_Line_Select, MBIR_4D/XT_NHICD.c:164-216). */
int mbirgpu_session_nh_select(mbirgpu_session *s, const float *mag, uint8_t *sel);

/* No counterpart in the reference. The forward projection of
 * mbirgpu_session_forward_project for callers that may not allocate device
 * memory (a framework allocator or a fixed budget owns it; cudaMalloc would
 * synchronise a latency-critical loop): object_dev [N_time][N_z][N_y][N_x]
 * and sino_dev [N_p][N_r][N_t] are device pointers, and the FP64 scratch is
 * a fixed 16 MiB array in the library (N_p * N_r * N_t <= 2,097,152, larger
 * sessions are rejected). Enqueued on the session's stream, not waited for.
 * Runs on the session's device whichever device is current (the caller's
 * current device is restored). Make the first call on each device before any
 * stream capture (it looks the scratch up; later calls outside capture look
 * it up again). The call clears the scratch it uses itself. The scratch is
 * shared by every call on a device: calls in flight at the same time on one
 * device race, so order them. */
int mbirgpu_session_forward_project_noalloc(mbirgpu_session *s, const float *object_dev, float *sino_dev);

/* The device A-matrix table, for inspection: per (frame view, voxel column)
 * the first detector channel, the count and kmax FP32 values.
 * first/count: [N_p][N_y][N_x]; values: [N_p][N_y][N_x][kmax]. */
int mbirgpu_session_get_amatrix(mbirgpu_session *s, int32_t *first, int32_t *count, float *values);

/* H_r detector response [N_p][65] as built on the host (XT_Profile.c:129-218). */
int mbirgpu_session_get_detector_response(mbirgpu_session *s, float *H_r);

/* Run ICD iterations until the reference's convergence test
 * (100 sum|dx| / sum|x| < convg_thresh after iteration 1, XT_ICD_update.c:1083-1090),
 * the cost test of opt->cost_rel_tol, or max_iter. costs (may be NULL) gets
 * the FP64 cost before iteration 1 and after each iteration; returns the
 * iteration count in *iters. */
int mbirgpu_session_run(mbirgpu_session *s, int32_t max_iter, double *costs, int32_t *iters,
                        mbirgpu_iter_stats *total);

/* --------------------------------------------------------------------------
 * Batched reconstruction of many independent problems (no counterpart in the
 * reference, which solves one problem per process).
 *
 * All problems stay resident; one ICD iteration of all of them is one
 * persistent launch per colour phase (and per detector-row class) whose CTAs
 * drain a queue over every problem's super-voxels, captured once as a CUDA
 * graph. Each problem is a single stage at voxel scale 1 (mult_xy = mult_z =
 * 1, the finest stage of reconstruct()), starts from zero and stops on its own
 * convergence test (100 sum|dx| / sum|x| < convg_thresh after the first
 * iteration, MBIR_4D/XT_ICD_update.c:1083-1090). The super-voxel size and
 * CTA width are autotuned for the whole batch unless fixed in the options.
 * ------------------------------------------------------------------------ */
typedef struct mbirgpu_batch mbirgpu_batch;

typedef struct {
    int64_t voxel_updates;     /* updates that ran in all problems since creation */
    double device_ms;          /* device time of this run (CUDA events) */
    int32_t graph_launches;    /* CUDA graph launches of this run (one per iteration) */
    int32_t kernel_launches_per_iteration;
    int32_t problems_converged;
    int32_t sv_size, cta_warps, sv_colors;
} mbirgpu_batch_stats;

int mbirgpu_batch_create(mbirgpu_batch **out, const mbirgpu_problem *problems, int32_t n,
                         const mbirgpu_options *opt, void *stream);
int mbirgpu_batch_destroy(mbirgpu_batch *b);
/* Run `iterations` more iterations of every problem that has not converged. */
int mbirgpu_batch_run(mbirgpu_batch *b, int32_t iterations, mbirgpu_batch_stats *stats);
int mbirgpu_batch_problem_info(mbirgpu_batch *b, int32_t i, mbirgpu_session_info *info, int32_t *iterations,
                               int32_t *converged);
/* Object of problem i, [N_time][N_z][N_y][N_x] without halo. */
int mbirgpu_batch_get_object(mbirgpu_batch *b, int32_t i, float *object);
/* FP64 MAP cost of problem i (MBIR_4D/XT_ICD_update.c:185-318). */
int mbirgpu_batch_cost(mbirgpu_batch *b, int32_t i, double *total);
/* Drop-in style: reconstruct n problems together with the current options,
 * up to `iterations` iterations each; objects[i] receives a malloc'ed buffer in
 * reconstruct()'s layout [recon_num][proj_rows+2][proj_cols][proj_cols]. */
int mbirgpu_reconstruct_batch(float **objects, const mbirgpu_problem *problems, int32_t n, int32_t iterations);

/* --------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference, which starts from zero
 * or a restart file). A 3-D U-Net -- four levels of c, 2c, 4c, 8c channels,
 * 3x3x3 convolutions with ReLU, 2x2x2 max-pooling, nearest upsampling with
 * skip concatenation, a 1x1x1 head added to the input -- trained and run by
 * the library's own BF16 tensor-core kernels (FP32 accumulation, FP32 master
 * weights, Adam). It maps a filtered back-projection frame to a converged
 * MBIR frame; ICD then runs to its usual convergence test from that image,
 * so the network changes the starting point only, never the solution.
 * Volumes are FP32 device arrays [D][H][W] with D, H, W multiples of 8.
 * ------------------------------------------------------------------------ */
typedef struct mbirgpu_unet mbirgpu_unet;

int mbirgpu_unet_create(mbirgpu_unet **out, int32_t base_channels, uint64_t seed, void *stream);
int mbirgpu_unet_destroy(mbirgpu_unet *u);
int64_t mbirgpu_unet_num_params(const mbirgpu_unet *u);
/* The network sees scale x input (values of order one) and returns
 * input + correction / scale; default 1. */
int mbirgpu_unet_set_input_scale(mbirgpu_unet *u, float scale);
float mbirgpu_unet_get_input_scale(const mbirgpu_unet *u);
/* Parameters (FP32 master copy), in layer order: per convolution the weights
 * [27][C_in][C_out] then the biases [C_out]; the head's weights [c] and bias. */
int mbirgpu_unet_get_params(mbirgpu_unet *u, float *params);
int mbirgpu_unet_set_params(mbirgpu_unet *u, const float *params);
int mbirgpu_unet_forward(mbirgpu_unet *u, const float *d_input, float *d_output, int32_t D, int32_t H, int32_t W);
/* Loss mean((net(input) - target)^2) and its gradient w.r.t. every parameter
 * (host, layer order as above; may be NULL). */
int mbirgpu_unet_gradients(mbirgpu_unet *u, const float *d_input, const float *d_target, int32_t D, int32_t H,
                           int32_t W, double *loss, float *grads);
/* One Adam step (beta 0.9 / 0.999) on one (input, target) pair. */
int mbirgpu_unet_train_step(mbirgpu_unet *u, const float *d_input, const float *d_target, int32_t D, int32_t H,
                            int32_t W, float lr, double *loss);
/* Which tensor-core kernels run the 3x3x3 convolutions: 1 (default) the
 * tcgen05 kernels (TMEM accumulators, TMA-staged operands) wherever input and
 * output channel counts are multiples of 16, 0 the mma.sync kernels
 * everywhere. No counterpart in the reference (the network has none). */
int mbirgpu_unet_set_tensor_path(mbirgpu_unet *u, int32_t path);
int32_t mbirgpu_unet_get_tensor_path(const mbirgpu_unet *u);
/* The session's object becomes the network applied to each frame of the
 * filtered back-projection, zero outside the reconstruction circle; e = y - A x
 * is recomputed. */
int mbirgpu_session_set_object_unet(mbirgpu_session *s, mbirgpu_unet *u);

/* --------------------------------------------------------------------------
 * Phase-contrast tomography (PCMBIR_3D): per-view phase retrieval.
 *
 * Drop-in for phcontomo_reconstruct of PCMBIR_3D/XT_Engine.c:82-197
 * (include/pcmbir4d.h:35). recon_type 1 runs single-material Paganin
 * retrieval on every view and writes pag_mag_ret.bin / pag_phase_ret.bin
 * (FP64, [proj_num][proj_cols][proj_rows] as the reference); recon_type 2
 * reads them and runs the per-view phase-retrieval ADMM of
 * estimate_complex_projection (PCMBIR_3D/XT_CmplxProjEst.c:91-229), writing
 * mag_tomo_aux / phase_tomo_aux (the estimated complex projections),
 * mag_pret_aux / phase_pret_aux, mag_pret_dual / phase_pret_dual,
 * omega_real / omega_imag and the per-view pret_cost / pret_primal /
 * pret_dual histories. Like the reference (XT_Engine.c:177-178) it returns
 * *magobject = *phaseobject = NULL; results go to files. The tomographic
 * ICD inside the ADMM is compiled out in the reference (ENABLE_TOMO_RECONS is
 * never defined) and is not part of this entry point either.
 * ------------------------------------------------------------------------ */
int phcontomo_reconstruct(float **magobject, float **phaseobject, float *measurements, float *brights,
                          float *proj_angles, float *proj_times, float *recon_times, int32_t proj_rows,
                          int32_t proj_cols, int32_t proj_num, int32_t recon_num, float vox_wid, float rot_center,
                          float mag_sig_s, float mag_sig_t, float mag_c_s, float mag_c_t, float phase_sig_s,
                          float phase_sig_t, float phase_c_s, float phase_c_t, float convg_thresh,
                          float obj2det_dist, float light_energy, float pag_regparam, uint8_t restart,
                          uint8_t recon_type, FILE *debug_msg_ptr);

typedef struct mbirgpu_pc_session mbirgpu_pc_session;

typedef struct {
    const float *measurements; /* [proj_num][proj_rows][proj_cols] intensities */
    const float *brights;      /* [proj_rows][proj_cols] bright field */
    int32_t proj_rows, proj_cols, proj_num;
    float vox_wid;             /* detector pitch; delta_r = delta_t = vox_wid (XT_Init.c:278-279, 391-392) */
    float mag_sig_s, mag_c_s, phase_sig_s, phase_c_s;
    float obj2det_dist;        /* propagation distance, same unit as vox_wid (um) */
    float light_energy;        /* keV; wavelength = hc / E (XT_Init.c:258) */
    float pag_regparam;        /* delta / beta */
} mbirgpu_pc_problem;

typedef struct {
    int32_t pret_max_iter;     /* PRet_MaxIter, XT_Init.c:517: 100 */
    int32_t sd_max_iter;       /* SteepDes_MaxIter, :518: 100 */
    int32_t nms_max_iter;      /* NMS_MaxIter, :515: 50 */
    double pret_threshold;     /* PRet_threshold, :522: 1e-7 */
    double sd_threshold;       /* SteepDes_threshold, :523: 5e-4 */
    double nms_threshold;      /* NMS_threshold, :520: 5e-3 */
    double mu, nu;             /* ADMM_mu, ADMM_nu for recon_type 2, :496-497: 0.5 */
    double mrf_p, mrf_q;       /* MRF_P, MRF_Q of PCMBIR_3D/XT_Constants.h:146-147 */
    int32_t nms_order;         /* proximal sweep order: 0 = the reference's raster order,
                                  kept exactly by anti-diagonal wavefronts (default);
                                  1 = four colour classes (more parallel, other order) */
    int32_t fft_radix;         /* largest radix of the FFT stages: 2, 4, 8 or 16; 0 = the
                                  library's choice. Every stage keeps its points in registers
                                  between two passes through shared memory */
    int32_t nms_lanes;         /* lanes that share one pixel's Nelder-Mead search: 1, 2, 4
                                  or 8; 0 = the library's choice */
    int32_t nms_ctas_per_view; /* raster order: CTAs (one thread-block cluster) per view,
                                  1, 2 or 4; 0 = the library's choice */
} mbirgpu_pc_options;

typedef struct {
    int64_t sd_steps;          /* steepest-descent steps run, summed over views */
    int64_t fresnel_transforms;/* Fresnel transforms run, summed over views */
    double kernel_ms;          /* device time of the run (CUDA events) */
    int64_t kernel_launches;   /* kernels the run launched */
} mbirgpu_pc_stats;

void mbirgpu_pc_default_options(mbirgpu_pc_options *opt);

/* Replaces the phase-contrast part of initStructures (PCMBIR_3D/XT_Init.c:
 * 251-549): measurements -> sqrt(I) / sqrt(mean bright), D = sqrt(bright) /
 * sqrt(mean bright), transfer tables of the Fresnel and Hermitian transforms.
 * Host images exchanged with a session are [proj_num][proj_cols][proj_rows]
 * (the reference's [N_p][N_r][N_t]); complex images are interleaved
 * (re, im) floats. */
int mbirgpu_pc_session_create(mbirgpu_pc_session **out, const mbirgpu_pc_problem *pb,
                              const mbirgpu_pc_options *opt, void *stream);
int mbirgpu_pc_session_destroy(mbirgpu_pc_session *s);
/* Batched Fresnel transform of every view (herm = 0: compute_FresnelTran,
 * herm = 1: compute_HermFresnelTran). */
int mbirgpu_pc_fresnel(mbirgpu_pc_session *s, const float *in, float *out, int32_t herm);
/* No counterpart in the reference (a measurement aid). n Fresnel-type
 * transforms (herm: the Hermitian one) of every view of the session, on its
 * resident buffers (whatever they hold), enqueued back to back on the
 * session's stream; *ms receives their device time (CUDA events). */
int mbirgpu_pc_time_fresnel(mbirgpu_pc_session *s, int32_t n, int32_t herm, double *ms);
/* Paganin retrieval of every view into the session's z (and, if not NULL, zr/zi). */
int mbirgpu_pc_paganin(mbirgpu_pc_session *s, float *zr, float *zi);
int mbirgpu_pc_set_z(mbirgpu_pc_session *s, const float *zr, const float *zi);
/* ADMM start of initErrorSinogam (PCMBIR_3D/XT_ICD_update.c:680-799):
 * w = e^{-z}, v = 0, Omega = phase of y / H(D w). */
int mbirgpu_pc_init_admm(mbirgpu_pc_session *s);
int mbirgpu_pc_set_state(mbirgpu_pc_session *s, const float *w, const float *v, const float *omega);
int mbirgpu_pc_get_state(mbirgpu_pc_session *s, float *zr, float *zi, float *w, float *v, float *omega);
/* One steepest-descent step of every view towards buf (steepest_descent_iter,
 * PCMBIR_3D/XT_PhaseRet.c:205-270); thresh[proj_num] receives each view's statistic. */
int mbirgpu_pc_sd_step(mbirgpu_pc_session *s, const float *buf, float *thresh);
/* One Nelder-Mead proximal sweep over every pixel of every view with b = w - v. */
int mbirgpu_pc_nms_sweep(mbirgpu_pc_session *s);
/* The per-view ADMM: costs [proj_num][pret_max_iter + 1] (may be NULL, FP64
 * phase-retrieval cost before and after each iteration, NaN after a view
 * stops), iters [proj_num] (may be NULL). */
int mbirgpu_pc_run(mbirgpu_pc_session *s, double *costs, int32_t *iters, mbirgpu_pc_stats *stats);

/* --------------------------------------------------------------------------
 * Phase-contrast data simulator.
 *
 * Drop-in for phcontomo_forward_project of PCMBIR_3D/XT_Engine.c:199-253
 * (include/pcmbir4d.h:36), which runs ForwardProject
 * (PCMBIR_3D/XT_genSinogram.c:59-343) on the geometry of
 * initPhantomStructures (PCMBIR_3D/XT_Init.c:611-684): the absorption and
 * refractive-index-decrement phantoms [phantom_z][phantom_xy][phantom_xy]
 * (float32 files) are projected with the A matrix times the wavenumber, the
 * exit field sqrt(expected_count) e^{-P_mag} e^{-i P_phase} is propagated by
 * the windowed Fresnel transform, |.|^2 is averaged over the
 * (phantom_z / proj_rows) x (phantom_xy / proj_cols) phantom pixels of each
 * detector pixel, and noise |m + sqrt|m| n| is added with n the reference's
 * randlib normal() sequence after srandom2(761521). *measurements
 * ([proj_num][proj_rows][proj_cols]) and *brights ([proj_rows][proj_cols],
 * = expected_count) are caller-allocated, as in the reference driver
 * (reconstruct/phase_data/XT_Main.c:130-134). With write_files the
 * reference's SimMagProjs.bin / SimPhaseProjs.bin (FP64
 * [proj_num][phantom_z][phantom_xy]) and mag_phantom.bin / phase_phantom.bin
 * (FP64 phantoms) are written to the working directory. Returns 0 or -1.
 * ------------------------------------------------------------------------ */
int phcontomo_forward_project(float **measurements, float **brights, float *proj_angles, int32_t proj_rows,
                              int32_t proj_cols, int32_t proj_num, float vox_wid, float rot_center,
                              float obj2det_dist, float light_energy, float pag_regparam, FILE *debug_msg_ptr);

/* The simulator's compile-time constants of PCMBIR_3D/XT_Constants.h as
 * run-time settings; defaults are the reference's values. */
typedef struct {
    char mag_phantom_path[1024];   /* MAG_PHANTOM_FILEPATH (:91) */
    char phase_phantom_path[1024]; /* PHASE_PHANTOM_FILEPATH (:92) */
    int32_t phantom_xy;            /* PHANTOM_XY_SIZE (:203): 512 */
    int32_t phantom_z;             /* PHANTOM_Z_SIZE (:204): 128 */
    float expected_count;          /* EXPECTED_COUNT_MEASUREMENT (:89): 2500 */
    int32_t write_files;           /* the reference's output files (default 1) */
} mbirgpu_pc_sim_options;

void mbirgpu_pc_sim_default_options(mbirgpu_pc_sim_options *opt);
int mbirgpu_pc_sim_set_options(const mbirgpu_pc_sim_options *opt);
int mbirgpu_pc_sim_get_options(mbirgpu_pc_sim_options *opt);

/* The simulator on phantoms in host memory (no files are read; files are
 * written only if opt->write_files). sim_mag_projs / sim_phase_projs
 * ([proj_num][phantom_z][phantom_xy] FP64, the reference's projs_real /
 * projs_imag) and measurement_avg may be NULL. opt NULL = the current
 * settings. No counterpart in the reference, which reads the phantoms from
 * fixed paths. */
int mbirgpu_pc_simulate(const float *mag_phantom, const float *phase_phantom, const mbirgpu_pc_sim_options *opt,
                        float *measurements, float *brights, const float *proj_angles, int32_t proj_rows,
                        int32_t proj_cols, int32_t proj_num, float vox_wid, float rot_center, float obj2det_dist,
                        float light_energy, double *sim_mag_projs, double *sim_phase_projs,
                        double *measurement_avg);

#ifdef __cplusplus
}
#endif
#endif
