// Session object behind the opaque mbirgpu_session handle.
#pragma once
#include <utility>
#include <vector>
#include "../../include/mbirgpu.h"
#include "mbir_internal.h"

namespace mbirgpu {

int fail(const char *fmt, ...);
mbirgpu_options current_options();
struct UNet;

struct Session {
    HostSetup hs;
    mbirgpu_options opt{};
    cudaStream_t st = nullptr;
    int device = 0;  // the CUDA device that was current when the session was created
    float convg_thresh = 0;
    size_t n_sino = 0, n_vox = 0, device_bytes = 0;
    int n_assigned = 0;  // views that belong to some frame
    int64_t masked_columns = 0;
    int64_t masked_nnz = 0;  // A nonzeros over masked columns, all frames, per voxel slice
    int sv = 8, warps = 4, colors = 2;
    int nh_sv = 8, nh_colors = 2, nh_warps = 4;  // schedule of the non-homogeneous passes
    bool timing = false;

    float *d_y = nullptr, *d_w = nullptr, *d_err = nullptr, *d_x = nullptr, *d_tmp = nullptr;
    uint32_t *d_table = nullptr;
    float *d_Hr = nullptr;
    double *d_cos = nullptr, *d_sin = nullptr;
    int32_t *d_views = nullptr, *d_view_first = nullptr, *d_view_frame = nullptr;
    uint8_t *d_mask = nullptr;
    float *d_mag = nullptr;
    IcdStats *d_stats = nullptr;
    double *d_cost_partials = nullptr, *d_cost_out = nullptr;
    int *d_flag = nullptr;
    double *d_acc = nullptr;  // FP64 sinogram accumulator of the forward projector
    unsigned int *d_queue = nullptr;  // super-voxel work-queue counters, one per ICD launch of an iteration
    static constexpr int kMaxPhases = 16;  // K x K colours, K <= 4
    static constexpr int kQueueCounters = kMaxPhases * (1 + kMaxNhPasses);
    float *d_filt = nullptr;          // NH-ICD filtered update magnitudes [N_time][N_y][N_x]
    uint8_t *d_sel = nullptr;         // NH-ICD selected columns [N_time][N_y][N_x]
    uint32_t *d_nh_items = nullptr;   // NH-ICD work lists (launch_nh_items), per phase
    int *d_nh_n = nullptr;            // their lengths [kMaxPhases]
    int *d_nh_scratch = nullptr;
    uint64_t *d_nh_selstate = nullptr;  // radix-select state (nh_select_scratch_bytes)
    size_t nh_items_cap = 0, nh_scratch_cap = 0;  // ints allocated
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pairs;
    // CUDA graphs of one ICD iteration, by [non-homogeneous passes][FP64
    // refresh]; the iteration number the kernels read lives in d_iter
    cudaGraphExec_t graphs[2][2] = {};
    bool graphs_timed = false;  // the captured graphs record the timing events
    bool tuning = false;        // schedule candidates are being measured: no graphs
    int *d_iter = nullptr;
    int h_iter = 0;
    int graph_launches_[2][2] = {};  // kernel launches inside each graph
    int graph_seen[2][2] = {};       // direct runs of each kind of iteration so far
    // ring correction: offset d [N_r][N_t] of e = y - Ax - d, updated after
    // every full-sweep phase and every NH pass while rings != 0
    int rings = 0;
    float *d_off = nullptr, *d_offx = nullptr;
    double *d_onum = nullptr, *d_olam = nullptr, *d_ogamma = nullptr;
    // noise variance of the generalised-Huber data term, re-estimated at the
    // end of every iteration while update_var (weights scaled in place)
    int update_var = 0;
    double var_est = 1.0;
    double *d_var = nullptr;

    ~Session();
    int init(const mbirgpu_problem *pb, const mbirgpu_options *o, int mult_xy, int mult_z, void *stream);
    void choose_schedule();
    int autotune();
    void sync_nh_schedule();
    struct TuneEntry {
        int sv, warps;
        double ms;
    };
    std::vector<TuneEntry> tune_log;
    int refresh_error();
    int set_object(const float *obj);
    int get_object(float *obj);
    int cost(double *total, double *data, double *prior);
    int icd_iteration(int iter, mbirgpu_iter_stats *out);
    int enqueue_iteration(int iter, bool graph_mode, int *launches);  // every launch of one iteration
    bool graph_ok() const;
    void drop_graphs();
    int run(int max_iter, double *costs, int *iters, mbirgpu_iter_stats *total);
    int amatrix(int32_t *first, int32_t *count, float *values);
    int forward_project(const float *obj, float *sino);
    int back_project(const float *sino, float *obj);
    int fbp(float *obj);              // host [N_time][N_z][N_y][N_x]
    int set_object_fbp();             // x = FBP, then e = y - A x
    int set_object_unet(UNet *u);     // x = U-Net(FBP) per frame, then e = y - A x
    int set_ring_correction(int mode, const float *offset);  // mode 0..3, offset host [N_r][N_t] or null
    int update_offset();
    int set_variance_estimation(int on);
};

}  // namespace mbirgpu
