// Internal declarations shared by the host code and the CUDA kernels of
// libmbirgpu. Not part of the public ABI (include/mbirgpu.h is).
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>
#include <cuda_runtime.h>

namespace mbirgpu {

constexpr int kRespBins = 64;  // DETECTOR_RESPONSE_BINS, MBIR_4D/XT_Constants.h:79
constexpr int kMaxKmax = 9;    // channels per (column, view) at voxel scale 4: 2*4+1
constexpr int kRowChunk = 32;  // detector rows one warp covers (lane = row); taller columns are chunked

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

// Detector response H_r [N_p][bins + 1] of the views' angles for g's geometry
// (XT_Profile.c:129-218): MBIR_4D's (float, 64 bins, a 512-sample beam) and
// PCMBIR_3D's (double; 256 bins and a 256-sample beam, PCMBIR_3D/XT_Constants.h:162-163).
void detector_response(const Geom &g, const float *angles, float *H_r);
void detector_response_f64(const Geom &g, const float *angles, double *H_r, int bins, int beam_res);

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

// e = y - A x - d (FP64 accumulation in d_acc, N_p*N_r*N_t doubles; d the
// per-detector-pixel offset [N_r][N_t], may be null); when d_y is null the
// result is A x itself. Rows of views outside every frame get y - d (or 0).
void launch_forward_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                            const float *d_x, const float *d_y, double *d_acc, float *d_out, cudaStream_t st,
                            const float *d_off = nullptr);

// Ring correction (kernels_offset.cu): one update of the per-detector-pixel
// offset d (mode 1 unconstrained, 2 zero mean, 3 the reference's window mode,
// which in its reconstruct has no windows) with e changed by the offset's
// change in every view. Scratch: d_num, d_lam ([N_r][N_t] doubles), d_gamma
// (1 double), d_x ([N_r][N_t] floats). Returns 0 or -1.
int offset_update(const Geom &g, int mode, int N_p, float *d_err, const float *d_w, float *d_off, double *d_num,
                  double *d_lam, double *d_gamma, float *d_x, cudaStream_t st);
// Noise variance re-estimation of the generalised-Huber data term: scales the
// weights in place (W <- W v_old / v_new) and updates *var_est (host);
// d_scratch holds variance_scratch_doubles() doubles.
size_t variance_scratch_doubles();
int variance_update(const Geom &g, int N_p, const float *d_err, float *d_w, double *var_est, double *d_scratch,
                    cudaStream_t st);
void launch_back_project(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first,
                         const int32_t *d_views, const float *d_sino, float *d_x, cudaStream_t st);

// Filtered back-projection of d_y into d_x ([N_time][N_y][N_x][N_z]); d_q is a
// sinogram-sized scratch for the ramp-filtered data. The ramp filter keeps one
// view ([N_r][N_t] floats) in shared memory.
void launch_fbp(const Geom &g, const uint32_t *d_table, const int32_t *d_view_first, const int32_t *d_views,
                const float *d_y, float *d_q, float *d_x, cudaStream_t st);
// Zero the voxel columns of d_x ([N_time][N_y][N_x][N_z]) outside the
// reconstruction circle: ICD never updates them, and the reference keeps them 0.
void launch_mask_object(const Geom &g, const uint8_t *d_mask, float *d_x, cudaStream_t st);
inline bool fbp_supported(const Geom &g) { return ((size_t)g.N_r * g.N_t + 2 * (size_t)g.N_r) * 4 <= 200 * 1024; }

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
    const uint8_t *sel;   // [N_time][N_y][N_x] columns this sweep may visit (with the mask); null = all
    int perm;             // queue order inside a frame: SV slot = (queue index * perm) mod slots
    int colors_k;         // K x K colour classes; phase p updates colour (p + frame) mod K^2
    long long max_ctas;   // cap on the persistent grid (sv_max_concurrent); 0 = none
    int stage_records;    // prefetch each next column's A records into shared memory (cp.async)
    const int *iter_dev;  // if set, the iteration number is read here (graph-captured iterations)
    // optional explicit work list of the phase (non-homogeneous passes): items[i]
    // = frame << 22 | sv_y << 11 | sv_x, *n_items of them (device memory);
    // null = every SV slot of the phase's colour in every frame
    const uint32_t *items;
    const int *n_items;
};

// SV slots of one colour per frame and the items (all frames) of one phase.
inline int sv_slots(int N_x, int N_y, int sv, int K)
{
    const int nx = (N_x + sv - 1) / sv, ny = (N_y + sv - 1) / sv;
    return ((nx + K - 1) / K) * ((ny + K - 1) / K);
}

// Multiplier of the SV queue order: coprime with n and near n / golden ratio,
// so consecutive queue positions -- the SVs CTAs work on at the same time --
// land far apart in the image instead of in one band of SV rows.
inline int spread_multiplier(int n)
{
    if (n <= 2) return 1;
    auto gcd = [](long long a, long long b) {
        while (b) {
            const long long t = a % b;
            a = b;
            b = t;
        }
        return a;
    };
    long long p = (long long)(0.6180339887498949 * n);
    if (p < 1) p = 1;
    while (gcd(p, n) != 1) p++;
    return (int)p;
}
struct IcdStats {  // device accumulators
    unsigned long long updates, skipped;
    double sum_abs_dx, sum_abs_x;
    unsigned int stage_timeouts, pad;  // staged record copies that did not land within the wait limit
};
// Per-problem constants of the voxel update, in FP32.
struct IcdConst {
    float sf[27];
    float tf;
    float q, qmp, ssq, ssqp, stq, stqp, cs, ct, bs0, bt0, alpha, dt;
    float issq, issqp, istq, istqp;  // reciprocals of ssq, ssqp, stq, stqp
    float huber_T, huber_delta;
    int huber;
};
IcdConst make_icd_const(const Geom &g);

// d_queue: one zeroed counter per launch (the persistent CTAs' work queue).
void launch_icd_phase(const Geom &g, const IcdLaunch &L, const uint32_t *d_table, const int32_t *d_view_first,
                      const uint8_t *d_mask, float *d_x, float *d_err, const float *d_w, float *d_mag,
                      IcdStats *d_stats, unsigned int *d_queue, cudaStream_t st);

// One problem of a batched launch (device-resident descriptor).
constexpr int kMaxBatch = 256;
struct __align__(16) BatchDesc {
    Geom g;
    IcdLaunch L;
    IcdConst K;
    const uint32_t *table;
    const int32_t *view_first;
    const uint8_t *mask;
    float *x, *err;
    const float *w;
    float *mag;
    IcdStats *stats;
    unsigned long long total_updates;  // voxel updates of all iterations run
    double last_pct;                   // last convergence statistic 100 sum|dx| / sum|x|
    float convg_thresh;                // the problem's convg_thresh (percent)
    int active;                        // 0 once converged: its items are skipped
    int iters_done;
};
int batch_grid(int vec, int warps);
void launch_icd_batch(int vec, int warps, int grid, const BatchDesc *d_descs, const int2 *d_item_map, int total,
                      int phase, unsigned int *d_queue, cudaStream_t st);
// persistent grid of the one-problem sweep kernel at `warps` warps per CTA
int icd_grid(int warps);
// Stability of concurrent super-voxel updates: CTAs update different columns
// at the same time, and columns of one frame on a common ray couple like a
// Jacobi step, more strongly the closer they are. Same-colour SVs are K sv
// columns apart; with C columns of a frame in flight, spread over the image
// (spread_multiplier), the over-relaxed updates stay convergent for
// 32 C <= N_y (K sv / 2)^2. Measured on 256 x 256 single-frame problems
// (90-360 views, no temporal prior): sv 4 with K = 2 converges at C <= 256
// and diverges at C = 512 (one problem already at 256); sv 8 with K = 2
// converges at C = 256, all its SVs of a colour. Launches cap their
// persistent grid at this many CTAs (frames are interleaved in the queue,
// so each frame gets its share).
inline long long sv_max_concurrent(int N_x, int N_y, int frames, int sv, int K)
{
    const long long spacing = (long long)K * sv / 2;
    (void)N_x;
    return std::max(1LL, (long long)std::max(1, frames) * ((long long)N_y * spacing * spacing / 32));
}

// Relative iterations to convergence by same-colour spacing K sv / 2
// (4: 1, 8: 51/56, 16: 38/56, measured on the 4-D workload with K = 2).
inline double sv_convergence_factor(int sv, int K)
{
    const int spacing = K * sv / 2;
    return spacing >= 16 ? 38.0 / 56.0 : spacing >= 8 ? 51.0 / 56.0 : 1.0;
}
void launch_batch_begin(BatchDesc *d_descs, int n, cudaStream_t st);
void launch_batch_end(BatchDesc *d_descs, int n, cudaStream_t st);

// Non-homogeneous ICD selection (VSC_based_Voxel_Line_Select, XT_NHICD.c:164-216):
// per frame, the 5x5 Hamming-filtered update-magnitude map (ComputeVSC,
// :128-161) and sel = mask && filtered > the (N - k)-th smallest filtered
// value, N = N_x N_y (RandomizedSelect's threshold), i.e. the k largest.
constexpr int kMaxNhPasses = 16;
constexpr int kNhicdIterations = 10;  // NHICD_Iterations, XT_Init.c:406
// d_sel_scratch: nh_select_scratch_bytes(n_frames) bytes of device memory
// (the radix select's per-frame state and digit histograms).
void launch_nh_select(int n_frames, int N_y, int N_x, const float *d_mag, const uint8_t *d_mask, int k,
                      float *d_filt, uint8_t *d_sel, cudaStream_t st, void *d_sel_scratch);
size_t nh_select_scratch_bytes(int n_frames);
// Work lists of the non-homogeneous passes: for each of the K x K phases of
// the (sv, K) tiling (phase p of frame f updates colour (p + f) mod K^2), the
// super-voxels holding selected columns, ordered by their number of selected
// columns, most first (the longest chains of sequential column updates start
// first), and in the phases' spread queue order within equal counts. Buffers:
// items [K^2][items_per_phase], n_items [K^2], scratch of nh_items_scratch_ints().
int nh_items_per_phase(int n_frames, int N_y, int N_x, int sv, int K);
size_t nh_items_scratch_ints(int n_frames, int N_y, int N_x, int sv, int K);
bool nh_items_supported(int n_frames, int N_y, int N_x, int sv);
void launch_nh_items(int n_frames, int N_y, int N_x, int sv, int K, const uint8_t *d_sel, uint32_t *d_items,
                     int *d_n_items, int *d_scratch, cudaStream_t st);

}  // namespace mbirgpu
