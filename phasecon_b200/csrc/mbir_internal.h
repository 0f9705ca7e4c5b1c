// Internal declarations shared by the host code and the CUDA kernels of
// libmbirgpu. Not part of the public ABI (include/mbirgpu.h is).
#pragma once
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <cuda_runtime.h>

namespace mbirgpu {

constexpr int kRespBins = 64;  // DETECTOR_RESPONSE_BINS, MBIR_4D/XT_Constants.h:79
constexpr int kMaxKmax = 9;    // channels per (column, view) at voxel scale 4: 2*4+1
constexpr int kMaxNt = 32;     // detector rows handled by the lane-per-row kernels

// One stage's geometry and prior constants, passed by value to kernels.
// Field meanings follow Sinogram / ScannedObject / TomoInputs of
// MBIR_4D/XT_Structures.h:61-190.
struct Geom {
    int N_r, N_t, N_p, z_overlap;
    int N_time, N_x, N_y, N_z, mult_xy, mult_z;
    double delta_r, delta_t, R0, RMax, T0, TMax, OffsetR, OffsetT;
    double x0, y0, z0, delta_xy, delta_z, delta_recon, radius_obj;
    double p, q, alpha, c_s, c_t;
    double sigma_s_q, sigma_s_q_p, sigma_t_q, sigma_t_q_p;
    double spatial_filter[27];  // [dz][dy][dx], offsets -1..1
    double time_filter;
    double huber_T, huber_delta;
    int huber;       // generalised-Huber data term active (quad_convex == 0)
    int kmax;        // slots per A record: 2*mult_xy + 1
    int rec_words;   // 32-bit words per A record (header + kmax values, padded to 4)
    int max_views;   // most views in a frame
};

// Host-side setup of a stage (restates MBIR_4D/XT_Init.c:211-432).
struct HostSetup {
    Geom g{};
    std::vector<int32_t> view_first;  // [N_time + 1] offsets into views
    std::vector<int32_t> views;       // frame-major view indices
    std::vector<float> H_r;           // [N_p][65]
    std::vector<double> cosv, sinv;   // [N_p]
    std::vector<uint8_t> mask;        // [N_y][N_x]
};

struct ProblemDesc {
    int proj_rows, proj_cols, proj_num, recon_num;
    float vox_wid, rot_center, sig_s, sig_t, c_s, c_t;
    int quad_convex;
    float huber_delta, huber_T;
    double mrf_p, mrf_q, alpha;
};

// Returns "" on success, else the failure message.
std::string build_setup(HostSetup &hs, const ProblemDesc &pd, const float *angles, const float *proj_times,
                        const float *recon_times, int mult_xy, int mult_z);

// ---- kernel launchers (kernels_*.cu); all asynchronous on `st` -------------
void launch_transpose_sino(const float *h_layout_dev, float *d_out, int N_p, int N_t, int N_r, cudaStream_t st);
void launch_untranspose_sino(const float *d_in, float *d_out, int N_p, int N_r, int N_t, cudaStream_t st);
void launch_vol_to_zfast(const float *d_in, float *d_out, int N_time, int N_z, int N_y, int N_x, cudaStream_t st);
void launch_zfast_to_vol(const float *d_in, float *d_out, int N_time, int N_z, int N_y, int N_x, cudaStream_t st);

// d_view_first: [N_time+1] offsets into d_views; d_view_frame: [N_p] frame of d_views[i].
void launch_build_amatrix(const Geom &g, const float *d_Hr, const double *d_cos, const double *d_sin,
                          const int32_t *d_views, const int32_t *d_view_first, const int32_t *d_view_frame,
                          uint32_t *d_table, int *d_err, cudaStream_t st);

void launch_count_masked_nnz(const Geom &g, int n_assigned, const int32_t *d_view_first, const int32_t *d_view_frame,
                             const uint8_t *d_mask, const uint32_t *d_table, unsigned long long *d_out,
                             cudaStream_t st);

// e = y - A x (FP64 accumulation in d_acc, N_p*N_r*N_t doubles); when d_y is
// null the result is A x itself. Rows of views outside every frame get y (or 0).
void launch_forward_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                            const float *d_x, const float *d_y, double *d_acc, float *d_out, cudaStream_t st);
void launch_back_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                         const int32_t *d_views, const float *d_sino, float *d_x, cudaStream_t st);

// FP64 MAP cost: out[0] = data term, out[1] = prior term (device doubles).
void launch_cost(const Geom &g, const float *d_err, const float *d_w, const float *d_x, double *d_partials,
                 int n_partials, double *d_out, cudaStream_t st);
int cost_partials_needed(const Geom &g);

// ICD sweep over one colour phase.
struct IcdLaunch {
    int sv;               // super-voxel edge (columns)
    int n_sv_x, n_sv_y;   // super-voxels per row / column of the image
    int warps;            // warps per CTA (cooperating on one column)
    int phase;            // 0..3
    int iter;             // 1-based iteration (zero-skipping starts at 2)
    int zero_skipping;
    int unroll;           // views in flight per lane (1, 2, 4); the launcher caps it by record width
    uint64_t seed;
};
struct IcdStats {  // device accumulators
    unsigned long long updates, skipped;
    double sum_abs_dx, sum_abs_x;
};
// d_queue: one zeroed counter per launch (the persistent CTAs' work queue).
void launch_icd_phase(const Geom &g, const IcdLaunch &L, const uint32_t *d_table, const int32_t *d_view_first,
                      const uint8_t *d_mask, float *d_x, float *d_err, const float *d_w, float *d_mag,
                      IcdStats *d_stats, unsigned int *d_queue, cudaStream_t st);

}  // namespace mbirgpu
